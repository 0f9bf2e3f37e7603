"""Regenerates tests/golden/sketch/: small FASTA/FASTQ inputs and the reference
sketcher's output on them (oracle/_ref/kssd3a, built from the reference sources by
`make -C oracle ref`).  Run from the repository root:

    python tests/golden/make_sketch_golden.py

sketch/inputs/        seeded genomes with the cases the sketch path must handle: several
                      records per file, lower case, N runs, CRLF line ends, records shorter
                      than k, an empty record, a gzip-compressed file, FASTQ reads
sketch/default/       `kssd3a sketch -o DIR <inputs>` (coden pattern, -f 8, conflicting
                      contexts removed): comblco, comblco.index, lcofiles.stat,
                      lcofiles.infilemeta
sketch/conflict/      the same with --conflict (conflicting contexts kept)
sketch/asone/         the same with --asone (all inputs one sample)
"""
import gzip
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.join(HERE, "sketch")
BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
INPUTS = ["g0.fa", "g1.fasta", "g2.fna", "g3.fa.gz", "r0.fq"]


def _genome(rng, n):
    return BASES[rng.integers(0, 4, size=n)].copy()


def _mutate(rng, seq, rate):
    s = seq.copy()
    hit = rng.random(len(s)) < rate
    s[hit] = BASES[(np.searchsorted(BASES, s[hit]) + rng.integers(1, 4, size=int(hit.sum()))) % 4]
    return s


def _lines(body, width):
    return [body[i:i + width] for i in range(0, len(body), width)]


def write_inputs(d):
    rng = np.random.default_rng(20261204)
    anc = _genome(rng, 60000)
    g0 = _mutate(rng, anc, 0.01)
    g1 = _mutate(rng, anc, 0.03)
    g2 = _mutate(rng, anc, 0.05)
    g3 = _genome(rng, 30000)
    # g0: two records, CRLF line ends, a lower-case stretch and an N run in the first
    a, b = g0[:35000].tobytes(), g0[35000:].tobytes()
    a = a[:5000] + a[5000:9000].lower() + b"N" * 50 + a[9050:]
    with open(os.path.join(d, INPUTS[0]), "wb") as f:
        f.write(b">g0_chr1 first record\r\n" + b"\r\n".join(_lines(a, 70)) + b"\r\n")
        f.write(b">g0_chr2\r\n" + b"\r\n".join(_lines(b, 70)) + b"\r\n")
    # g1: one record, 60-column lines, scattered IUPAC codes
    s = bytearray(g1.tobytes())
    for p in rng.integers(0, len(s), size=40):
        s[int(p)] = ord("RYKMSWn"[int(p) % 7])
    with open(os.path.join(d, INPUTS[1]), "wb") as f:
        f.write(b">g1 one record\n" + b"\n".join(_lines(bytes(s), 60)) + b"\n")
    # g2: records of 31, 32 and 33 bases (shorter than, equal to, longer than k), an
    # empty record, then the genome in pieces
    t = g2.tobytes()
    with open(os.path.join(d, INPUTS[2]), "wb") as f:
        f.write(b">short31\n" + t[:31] + b"\n>exact32\n" + t[100:132] + b"\n>long33\n" + t[200:233] + b"\n")
        f.write(b">empty\n")
        for i, piece in enumerate(_lines(t[300:], 9000)):
            f.write(b">piece%d\n" % i + b"\n".join(_lines(piece, 80)) + b"\n")
    # g3: gzip-compressed, unrelated genome
    with open(os.path.join(d, INPUTS[3]), "wb") as raw:
        with gzip.GzipFile(fileobj=raw, mode="wb", compresslevel=6, mtime=0) as f:
            f.write(b">g3\n" + b"\n".join(_lines(g3.tobytes(), 80)) + b"\n")
    # r0: 150 bp reads of g0 at ~1x with 0.5% errors, four-line FASTQ
    with open(os.path.join(d, INPUTS[4]), "wb") as f:
        for i in range(400):
            p = int(rng.integers(0, len(g0) - 150))
            r = _mutate(rng, g0[p:p + 150], 0.005)
            if rng.random() < 0.5:
                r = BASES[3 - np.searchsorted(BASES, r[::-1])]
            f.write(b"@r%d\n" % i + r.tobytes() + b"\n+\n" + b"I" * 150 + b"\n")


def main():
    if not oracle.ref_available():
        sys.exit("build the reference first: make -C oracle ref")
    shutil.rmtree(OUT, ignore_errors=True)
    inputs = os.path.join(OUT, "inputs")
    os.makedirs(inputs)
    write_inputs(inputs)
    env = {k: v for k, v in os.environ.items() if not k.startswith("KSSD3A_")}
    for mode, extra in (("default", []), ("conflict", ["--conflict"]), ("asone", ["--asone"])):
        d = os.path.join(OUT, mode)
        # relative input paths, as the names stored in lcofiles.stat
        subprocess.run([oracle.REF_BIN, "sketch", "-o", os.path.relpath(d, OUT), *extra,
                        *[os.path.join("inputs", x) for x in INPUTS]], cwd=OUT, check=True, env=env,
                       capture_output=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()

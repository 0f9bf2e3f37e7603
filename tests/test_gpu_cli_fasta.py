"""bin/kssd3a against the reference CLI (oracle/_ref/kssd3a) on FASTA/FASTQ inputs, byte
for byte: the auto-ANI forms of `kssd3a ani` that sketch sequence before counting
(src/command_ani_wrapper.c:842-1046, 1275-1502) -- positional reference and query
inputs, --pair, --reflist/--qrylist, and -q/--qraw sequence against a sketch
directory -- on 8 seeded genomes of 1 Mbp (2 clusters of 4, 0.1-2% substitutions and
short indels), a FASTQ read set drawn from one of them, and the sketch golden inputs
(several records per file, CRLF line ends, lower case, N runs, gzip).  Our binary
sketches on the GPU (kssdgpu_sketch), the reference with its own sketcher.  Both run in
the same working directory, so the printed paths agree.

Skipped where the reference build is absent (it is built from the reference sources
by oracle/Makefile)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")
GOLDEN = os.path.join(ROOT, "tests", "golden", "sketch", "inputs")
THREADS = str(min(16, os.cpu_count() or 4))


def _run(binary, argv, cwd):
    env = {k: v for k, v in os.environ.items() if not k.startswith("KSSD3A_")}
    env["OMP_NUM_THREADS"] = THREADS
    return subprocess.run([binary, *argv], capture_output=True, env=env, cwd=cwd, timeout=900)


def _reads(path, genome, n, seed, err=0.005, length=150):
    """n reads of one FASTA genome at uniform positions with substitution errors."""
    with open(genome, "rb") as f:
        seq = f.read().split(b"\n", 1)[1].replace(b"\n", b"")
    rng = np.random.default_rng(seed)
    bases = np.frombuffer(b"ACGT", dtype=np.uint8)
    with open(path, "wb") as f:
        for i in range(n):
            p = int(rng.integers(0, len(seq) - length))
            r = np.frombuffer(seq[p:p + length], dtype=np.uint8).copy()
            hit = rng.random(length) < err
            r[hit] = bases[rng.integers(0, 4, size=int(hit.sum()))]
            f.write(b"@r%d\n%s\n+\n%s\n" % (i, r.tobytes(), b"I" * length))


@pytest.fixture(scope="module")
def work(tmp_path_factory):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    import fasta_synth
    root = str(tmp_path_factory.mktemp("fasta_cli"))
    fasta_synth.write_genomes(os.path.join(root, "fa"), n_clusters=2, per_cluster=4, length=1_000_000,
                              sub_lo=0.001, sub_hi=0.02)
    os.makedirs(os.path.join(root, "gold"))
    for name in ("g0.fa", "g1.fasta", "g2.fna", "g3.fa.gz", "r0.fq"):
        shutil.copy(os.path.join(GOLDEN, name), os.path.join(root, "gold", name))
    _reads(os.path.join(root, "reads.fq"), os.path.join(root, "fa", "c01_m02.fa"), 20000, 5)
    with open(os.path.join(root, "refs.txt"), "w") as f:
        f.write("".join(f"fa/c0{c}_m0{m}.fa\n" for c in range(2) for m in range(2)))
    with open(os.path.join(root, "qry.txt"), "w") as f:
        f.write("".join(f"fa/c0{c}_m0{m}.fa\n" for c in range(2) for m in range(2, 4)))
    # a reference-made sketch directory for the -q / --qraw sequence forms
    names = sorted(os.listdir(os.path.join(root, "fa")))
    r = subprocess.run([oracle.REF_BIN, "sketch", "-p", THREADS, "-o", "refsk", *[f"fa/{x}" for x in names]],
                       capture_output=True, cwd=root, timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    return root


CASES = [
    ("positional", ["ani", "fa/c00_m00.fa", "fa/c00_m01.fa", "fa/c01_m00.fa", "fa/c00_m02.fa"]),
    ("dirs", ["ani", "fa", "fa"]),
    ("dirs_matrix", ["ani", "--format", "matrix", "--values", "ani", "fa", "fa"]),
    ("pair", ["ani", "--pair", "fa/c00_m00.fa", "fa"]),
    ("lists", ["ani", "--reflist", "refs.txt", "--qrylist", "qry.txt"]),
    ("query_fasta", ["ani", "-r", "refsk", "-q", "fa/c00_m03.fa", "fa/c01_m01.fa"]),
    ("qraw_fastq", ["ani", "-r", "refsk", "--qraw", "reads.fq"]),
    ("golden_positional", ["ani", "gold/g0.fa", "gold/g1.fasta", "gold/g2.fna", "gold/g3.fa.gz"]),
    ("golden_query", ["ani", "-r", "refsk", "-q", "gold/g0.fa", "gold/g3.fa.gz", "gold/g2.fna"]),
    ("golden_qraw", ["ani", "-r", "refsk", "--qraw", "gold/r0.fq"]),
    ("golden_dirs_matrix", ["ani", "--format", "matrix", "--values", "ani", "gold", "gold"]),
    ("golden_positional_matrix", ["ani", "--format", "matrix", "gold/g0.fa", "gold/g1.fasta", "gold/g2.fna",
                                  "gold/g3.fa.gz"]),
    ("query_dir_refused", ["ani", "-r", "refsk", "-q", "fa"]),
]


@pytest.mark.parametrize("name,argv", CASES, ids=[c[0] for c in CASES])
def test_fasta_inputs_match_reference_cli(work, name, argv):
    argv = [argv[0], "-p", THREADS, *argv[1:]]
    mine = _run(OURS, argv, work)
    want = _run(oracle.REF_BIN, argv, work)
    assert mine.returncode == want.returncode, (name, mine.stderr.decode()[-1000:], want.stderr.decode()[-1000:])
    if want.returncode != 0:
        # the same message (after the program name)
        last = lambda r: r.stderr.decode().strip().splitlines()[-1].split(":", 1)[-1]  # noqa: E731
        assert last(mine) == last(want)
        return
    if mine.stdout != want.stdout:
        a, b = mine.stdout.decode().splitlines(), want.stdout.decode().splitlines()
        for i, (x, y) in enumerate(zip(a, b)):
            if x != y:
                pytest.fail(f"{name}: first differing line {i}:\n ours: {x[:300]}\n want: {y[:300]}")
        pytest.fail(f"{name}: line counts differ: ours {len(a)} want {len(b)}")
    if name in ("dirs", "query_fasta", "qraw_fastq", "lists", "positional"):
        assert want.stdout.count(b"\n") > 2  # cross-genome rows, not just a header

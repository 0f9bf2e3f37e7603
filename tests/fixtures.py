"""Seeded sketch-space fixtures for the tests (pure numpy; no reference code)."""
import numpy as np

OBJ_BITS = 20


def samples_to_sketch(samples, obj_bits=OBJ_BITS):
    """samples: list of iterables of (ctx, obj).  Returns (keys, offs) sorted per sample."""
    keys, offs = [], [0]
    for s in samples:
        k = sorted({(int(c) << obj_bits) | int(o) for c, o in s})
        keys.extend(k)
        offs.append(len(keys))
    return np.array(keys, dtype=np.uint64), np.array(offs, dtype=np.uint64)


def random_samples(rng, n, max_len, ctx_space, obj_space, conflict=True, empty_prob=0.1):
    """Small random samples; with conflict=False every context appears once per sample."""
    out = []
    for _ in range(n):
        if rng.random() < empty_prob:
            out.append([])
            continue
        m = int(rng.integers(1, max_len + 1))
        ctx = rng.integers(0, ctx_space, size=m)
        obj = rng.integers(0, obj_space, size=m)
        pairs = list(zip(ctx.tolist(), obj.tolist()))
        if not conflict:
            seen = {}
            for c, o in pairs:
                seen.setdefault(c, o)
            pairs = list(seen.items())
        out.append(pairs)
    return out


def mutate_from(rng, base, rate, obj_bits=OBJ_BITS):
    """A sample derived from `base` with object bases substituted at `rate`."""
    out = []
    for c, o in base:
        for b in range(obj_bits // 2):
            if rng.random() < rate:
                o ^= int(rng.integers(1, 4)) << (2 * b)
        out.append((c, o))
    return out


def read_fastx_records(path):
    """Sequence records of a FASTA/FASTQ file (gzip or plain) with the reference's parser
    rules (klib kseq as vendored by the reference): a record starts at '>' or '@';
    sequence lines run to the next line starting with '>', '+' or '@'; line ends are
    '\\n' with one trailing '\\r' removed; empty lines are skipped; FASTQ quality lines
    are consumed by length."""
    import gzip
    with open(path, "rb") as f:
        data = f.read()
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    lines = data.split(b"\n")
    if lines and lines[-1] == b"":
        lines.pop()
    recs, i = [], 0
    while i < len(lines) and not lines[i][:1] in (b">", b"@"):
        i += 1
    while i < len(lines):
        i += 1  # header
        seq = []
        while i < len(lines) and lines[i][:1] not in (b">", b"+", b"@"):
            if lines[i]:
                seq.append(lines[i][:-1] if lines[i].endswith(b"\r") else lines[i])
            i += 1
        s = b"".join(seq)
        if i < len(lines) and lines[i][:1] == b"+":
            i += 1
            q = 0
            while i < len(lines) and q < len(s):
                q += len(lines[i].rstrip(b"\r"))
                i += 1
        recs.append(s)
    return recs

"""Seeded synthetic genomes as FASTA files (the sequence-space workload of the
64-genome configuration): clusters of members derived from a random ancestor by
uniform substitutions and short indels.

    ancestor   iid bases at a given GC fraction
    member     substitutions at rate ~U(sub_lo, sub_hi) (a uniformly different base),
               indels at indel_rate per bp (insertion or deletion with equal odds,
               length ~U{1..10}); every member is its own deterministic stream

These files are sketched by the reference's own sketcher, so that the counting
engine is checked on sketches made from sequence (not generated in sketch space).
"""
from __future__ import annotations

import os

import numpy as np

_BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def _ancestor(rng: np.random.Generator, length: int, gc: float) -> np.ndarray:
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return rng.choice(4, size=length, p=p).astype(np.uint8)


def _member(rng: np.random.Generator, anc: np.ndarray, sub: float, indel_rate: float) -> np.ndarray:
    seq = anc.copy()
    hit = rng.random(len(seq)) < sub
    seq[hit] = (seq[hit] + rng.integers(1, 4, size=int(hit.sum()), dtype=np.uint8)) % 4
    n_ind = rng.binomial(len(seq), indel_rate)
    if n_ind == 0:
        return seq
    pos = np.sort(rng.choice(len(seq), size=n_ind, replace=False))
    lens = rng.integers(1, 11, size=n_ind)
    ins = rng.random(n_ind) < 0.5
    parts, last = [], 0
    for p, ln, is_ins in zip(pos.tolist(), lens.tolist(), ins.tolist()):
        if p < last:
            continue  # inside a previous deletion
        parts.append(seq[last:p])
        if is_ins:
            parts.append(rng.integers(0, 4, size=ln, dtype=np.uint8))
            last = p
        else:
            last = p + ln
    parts.append(seq[last:])
    return np.concatenate(parts)


def write_genomes(outdir: str, n_clusters: int = 8, per_cluster: int = 8, length: int = 1_000_000,
                  gc: float = 0.5, sub_lo: float = 0.005, sub_hi: float = 0.05, indel_rate: float = 0.001,
                  seed: int = 20261204) -> list[str]:
    """Writes n_clusters * per_cluster FASTA files (one genome each, 80-column lines)
    into outdir and returns their paths in sample order (cluster-major)."""
    os.makedirs(outdir, exist_ok=True)
    paths = []
    for c in range(n_clusters):
        anc = _ancestor(np.random.default_rng([seed, c, 0]), length, gc)
        for m in range(per_cluster):
            rng = np.random.default_rng([seed, c, m + 1])
            seq = _BASES[_member(rng, anc, rng.uniform(sub_lo, sub_hi), indel_rate)]
            path = os.path.join(outdir, f"c{c:02d}_m{m:02d}.fa")
            body = seq.tobytes()
            with open(path, "wb") as f:
                f.write(f">c{c:02d}_m{m:02d} synthetic cluster {c} member {m}\n".encode())
                f.write(b"\n".join(body[i:i + 80] for i in range(0, len(body), 80)))
                f.write(b"\n")
            paths.append(path)
    return paths

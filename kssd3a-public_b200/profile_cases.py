"""Small, self-contained launches of the hot kernels for one-kernel ncu captures.

    python kssd3a-public_b200/profile_cases.py scan    # 2,000-genome self join, 3 scan-join steps
    python kssd3a-public_b200/profile_cases.py scanbig # 5,000 small genomes: triangle beyond L2 (cell table)
    python kssd3a-public_b200/profile_cases.py dense   # 512-genome one-species dense join, 2 steps
    python kssd3a-public_b200/profile_cases.py rect    # 2,000 queries x 4,000 references, 4 batched counts
    python kssd3a-public_b200/profile_cases.py denseprobe  # 128 queries x 512 one-species references, 3 counts

Each case builds its index from a seeded synthetic sketch (the generators of the
benchmark), runs a few launches of the kernel under study on cuda:0 and exits, so
that a capture (`ncu -k <kernel> -s <skip> -c <count> ...`) holds a few GB of device
memory at most and ends by itself.  No timing is printed: times taken under a
profiler are not measurements.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import torch  # noqa: E402

import kssdgpu  # noqa: E402

THREADS = os.cpu_count() or 8


def case_scan(dev, st):
    n = 2000
    sk = kssdgpu.synth(n_samples=n, n_clusters=n // 10, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                       len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=20261203 + 2,
                       sample_seed=20261203 + 2, threads=THREADS)
    idx = kssdgpu.Index.from_sketch(sk)
    cells = n * (n - 1) // 2
    a = torch.zeros(cells, dtype=torch.int64, device=dev)
    b = torch.zeros_like(a)
    for _ in range(3):
        idx.self_lower_dev(a, b, flags=kssdgpu.SELF_SCAN, stream=st)
    torch.cuda.synchronize()
    idx.close()


def case_scanbig(dev, st):
    """5,000 genomes of 0.5-2 Mbp: the packed triangle (12.5M cells, 200 MB) is larger than
    L2, so the scan join adds through its table of touched cells; about 1 GB on the device."""
    n = 5000
    sk = kssdgpu.synth(n_samples=n, n_clusters=n // 10, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=1e6,
                       len_sigma=0.37, len_min=5e5, len_max=2e6, sub_lo=0.001, sub_hi=0.2, seed=20261203 + 2,
                       sample_seed=20261203 + 2, threads=THREADS)
    idx = kssdgpu.Index.from_sketch(sk)
    cells = n * (n - 1) // 2
    a = torch.zeros(cells, dtype=torch.int64, device=dev)
    b = torch.zeros_like(a)
    for _ in range(3):
        idx.self_lower_dev(a, b, flags=kssdgpu.SELF_SCAN, stream=st)
    torch.cuda.synchronize()
    print("entries", int(sk.offs[-1]))
    idx.close()


def case_dense(dev, st):
    n = 512
    sk = kssdgpu.synth(n_samples=n, n_clusters=1, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.2,
                       len_min=2e6, len_max=8e6, sub_lo=0.001, sub_hi=0.02, seed=7, sample_seed=7, threads=THREADS)
    idx = kssdgpu.Index.from_sketch(sk)
    cells = n * (n - 1) // 2
    a = torch.zeros(cells, dtype=torch.int64, device=dev)
    b = torch.zeros_like(a)
    for _ in range(2):
        idx.self_lower_dev(a, b, flags=kssdgpu.SELF_DENSE, stream=st)
    torch.cuda.synchronize()
    print("alleles", idx.dense_alleles())
    idx.close()


def case_denseprobe(dev, st):
    """The batched probe on a one-species index: 512 references and 128 new members of the
    species (context groups of hundreds of postings, walked by whole warps)."""
    ref = kssdgpu.synth(n_samples=512, n_clusters=1, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.2,
                        len_min=2e6, len_max=8e6, sub_lo=0.001, sub_hi=0.02, seed=7, sample_seed=7, threads=THREADS)
    qry = kssdgpu.synth(n_samples=128, n_clusters=1, role=kssdgpu.ROLE_OWNLEN, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        len_median=4e6, len_sigma=0.2, len_min=2e6, len_max=8e6, own_len_min=1e6, own_len_max=8e6,
                        sub_lo=0.001, sub_hi=0.02, seed=7, sample_seed=8, threads=THREADS)
    idx = kssdgpu.Index.from_sketch(ref)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    c = torch.zeros(qry.n * ref.n, dtype=torch.int64, device=dev)
    o = torch.zeros_like(c)
    for _ in range(3):
        idx.count_block_dev(dk, do, qry.n, c, o, flags=kssdgpu.GLOBAL_ACC, stream=st)
    torch.cuda.synchronize()
    print("keys", int(qry.offs[-1]), "credits", int((c & 0xFFFFFFFF).sum().item()))
    idx.close()


def case_rect(dev, st):
    nr, nq = 4000, 2000
    ref = kssdgpu.synth(n_samples=nr, n_clusters=nr // 10, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                        len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=20261206,
                        sample_seed=20261206, threads=THREADS)
    qry = kssdgpu.synth(n_samples=nq, n_clusters=nr // 10, role=kssdgpu.ROLE_OWNLEN, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6, own_len_min=5e4,
                        own_len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=20261206, sample_seed=20261207,
                        threads=THREADS)
    idx = kssdgpu.Index.from_sketch(ref)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    c = torch.zeros(nq * nr, dtype=torch.int64, device=dev)
    o = torch.zeros_like(c)
    for i in range(4):
        idx.count_block_dev(dk, do, nq, c, o, flags=kssdgpu.NO_ZERO if i else 0, stream=st)
    torch.cuda.synchronize()
    print("keys", int(qry.offs[-1]))
    idx.close()


def main(argv):
    cases = {"scan": case_scan, "scanbig": case_scanbig, "dense": case_dense, "rect": case_rect,
             "denseprobe": case_denseprobe}
    which = argv[1] if len(argv) > 1 else ""
    if which not in cases:
        print("usage: profile_cases.py scan|scanbig|dense|rect|denseprobe", file=sys.stderr)
        return 64
    if not torch.cuda.is_available():
        print("profile_cases.py: needs a CUDA device", file=sys.stderr)
        return 1
    dev = torch.device("cuda", 0)
    cases[which](dev, torch.cuda.current_stream())
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))

#!/usr/bin/env python
"""Benchmark: ANI genome-pairs/s of the all-vs-all self ANI matrix on one B200.

Workload (the configuration the headline metric is quoted on): 2,000 synthetic
genomes, lognormal sizes (median 4 Mbp, sigma 0.37, clipped to 1-12 Mbp), 200
clusters, ancestor-to-member substitution ~U(0.1%, 20%), sketched at the default
coden pattern (44-bit context, 20-bit object, ~1 key per 256 bp), generated in
sketch space by the seeded generator (host/kssd_synth.c).  The path is the
counting behind `kssd3a ani -q refs --format matrix --values ani` (indexed self
full matrix): the lower triangle of shared-context counters for every pair;
genome-pairs = n^2 matrix cells per step.

Arms:
  ours (default)   value: one self step from the resident index per timed step --
                   zero fill of the dense lower triangle plus the one-pass scan join
                   (every context group's bounds read, every shared context joined;
                   nothing cached between steps); e2e: the reference-facing C-ABI call
                   kssdgpu_count_lower with HOST buffers (query keys H2D, dense
                   counters D2H) every step, pinned in one call, and as the reference's
                   drivers call it (64-query blocks, pageable buffers); beside it the
                   batched probe kernel, the plain one-query-per-launch kernel, the
                   cached-plan join, and (unless --no-extra) the 20,000-genome
                   all-vs-all, a 10,000-query x 20,000-reference block, 40 read sets
                   with unique contexts and a short serving sweep against the resident
                   20,000-genome index, each with parity against the reference's own
                   counting function on a sample.
  reference        the reference's own count_ctx_obj_frm_comb_sketch_section_lower
                   (compiled from its sources into oracle/_ref) over blocks of 64
                   queries with all host threads; rank 0 only.
One JSON line on stdout (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import random
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "kssd3a-public_b200"))

WORKLOAD = dict(name="self-ani-matrix-2000-genomes", n_samples=2000, n_clusters=200, len_median=4e6,
                len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=20261203 + 2)
BLOCK = 64  # the reference's self-matrix query block (src/command_ani.c:1498-1531)


def make_workload(n: int, lib=None):
    import kssdgpu
    w = dict(WORKLOAD)
    return kssdgpu.synth(lib=lib, n_samples=n, n_clusters=max(1, n // 10), size_dist=kssdgpu.SIZE_LOGNORMAL,
                         len_median=w["len_median"], len_sigma=w["len_sigma"], len_min=w["len_min"],
                         len_max=w["len_max"], sub_lo=w["sub_lo"], sub_hi=w["sub_hi"], seed=w["seed"],
                         sample_seed=w["seed"], threads=os.cpu_count() or 8)


def cpu_count_lower_blocks(sk, rec, blocks, threads, use_ref):
    """Runs count_lower over the given 64-query blocks on the host; returns (seconds, counters)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    n = sk.n
    outs = []
    t0 = time.perf_counter()
    for b in blocks:
        off = b * BLOCK
        nb = min(BLOCK, n - off)
        qo = np.ascontiguousarray(sk.offs[off: off + nb + 1])
        qk = sk.keys[int(qo[0]): int(qo[-1])]
        outs.append((off, oracle.count_lower(rec, n, off, qk, qo, threads=threads, ref=use_ref)))
    return time.perf_counter() - t0, outs


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i
                          and s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_peak_bf16_tflops():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def max_over_ranks(dist, x, device):
    """The largest of x over all ranks (x itself without a process group): every
    rank's timed region ends with the slowest one."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, units, seconds):
    """Whole-job throughput of `world` replicas that each processed `units` in at
    most `seconds` (weak scaling: per-GPU work fixed)."""
    return world * units / seconds


def probe_model_bytes(n_keys, postings_walked, cells):
    """The per-query probe model of the counting kernels: 8 B per query key, 12 B per
    index posting walked (the reference's ctxgidobj_t record), 16 B per counter cell."""
    return 8 * n_keys + 12 * postings_walked + 16 * cells


def scan_join_bytes(contexts, shared_postings, touched):
    """Distinct bytes of the one-pass scan join: every context group's bounds (4 B per
    group + 1), the postings of groups of >= 2 (8 B each) and the touched counter cells
    read and written once (2 x 16 B)."""
    return 4 * (contexts + 1) + 8 * shared_postings + 2 * 16 * touched


def lower_equals_dense(lower_c, lower_o, dense_c, dense_o, n, rows=1024):
    """Packed lower triangle == the strictly-lower part of the dense [n][n] counters
    (compared in row blocks on the device)."""
    import torch
    dc, do = dense_c.view(n, n), dense_o.view(n, n)
    for a in range(0, n, rows):
        b = min(n, a + rows)
        r = torch.arange(a, b, device=dc.device).unsqueeze(1)
        c = torch.arange(0, b, device=dc.device).unsqueeze(0)
        m = c < r
        lo, hi = a * (a - 1) // 2 if a else 0, b * (b - 1) // 2
        if not (torch.equal(dc[a:b, :b][m], lower_c[lo:hi]) and torch.equal(do[a:b, :b][m], lower_o[lo:hi])):
            return False
    return True


class Timer:
    """CUDA-event timing on one stream, an L2 flush (a 256 MB write, above the 126 MB
    L2) before every timed call."""

    def __init__(self, stream, device):
        import torch
        self.torch = torch
        self.stream = stream
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)

    def __call__(self, fn, steps, warmup, pre=None, flush_l2=True):
        torch = self.torch
        for _ in range(warmup):
            if pre:
                pre()
            fn()
        torch.cuda.synchronize()
        tot = []
        for _ in range(steps):
            if flush_l2:
                self.flush.fill_(1)
            if pre:
                pre()
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(self.stream)
            fn()
            e.record(self.stream)
            e.synchronize()
            tot.append(s.elapsed_time(e))
        torch.cuda.synchronize()
        return float(np.mean(tot))  # ms


def density_histogram(d_lc, sizes, n, tile=128):
    """Shared-context density of the all-vs-all matrix per 128 x 128 genome tile, in
    gid order and with the genomes grouped by cluster (the best case for a dense
    tile): credits / (tile cells x mean sketch size), i.e. the fraction of a dense
    int8 context-by-genome GEMM's multiply-adds that land on a shared context."""
    import torch
    num_ctx = (d_lc & 0xFFFFFFFF).to(torch.float64)
    full = torch.zeros(n, n, dtype=torch.float64, device=d_lc.device)
    tri = torch.tril_indices(n, n, -1, device=d_lc.device)
    full[tri[0], tri[1]] = num_ctx
    full = full + full.T
    mean_size = float(np.mean(sizes))
    out = {}
    for name, order in (("gid_order", torch.arange(n, device=d_lc.device)),
                        ("cluster_order", torch.argsort(torch.arange(n, device=d_lc.device) % max(1, n // 10),
                                                        stable=True))):
        m = full[order][:, order]
        nt = (n + tile - 1) // tile
        pad = nt * tile - n
        m = torch.nn.functional.pad(m, (0, pad, 0, pad))
        t = m.view(nt, tile, nt, tile).sum(dim=(1, 3)) / (tile * tile * mean_size)
        t = t[torch.triu_indices(nt, nt, 0, device=t.device).unbind(0)]
        edges = [0, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2, 0.1, 1.0]
        hist = [int(((t >= lo) & (t < hi)).sum().item()) for lo, hi in zip(edges[:-1], edges[1:])]
        out[name] = {"tiles": int(t.numel()), "max": float(t.max().item()), "mean": float(t.mean().item()),
                     "bins": edges, "counts": hist}
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import kssdgpu
    import oracle
    # the generator built into the oracle's own library (the product's host library
    # stays unmapped in this process)
    sk = make_workload(args.genomes, lib=kssdgpu.bind_synth(oracle.workload_lib()))
    rec = oracle.build_index(sk.keys, sk.offs)
    use_ref = oracle.ref_available()
    threads = os.cpu_count() or 1
    nblocks = (sk.n + BLOCK - 1) // BLOCK
    # size a step to a bounded sample: time one block (the heaviest, last) first
    t1, _ = cpu_count_lower_blocks(sk, rec, [nblocks - 1], threads, use_ref)
    per_step = max(1, min(nblocks, int(args.cpu_step_seconds / max(t1, 1e-3))))
    order = list(range(nblocks))
    times, pairs = [], []
    for s in range(args.warmup + args.steps):
        blocks = [order[(s * per_step + i) % nblocks] for i in range(per_step)]
        dt, _ = cpu_count_lower_blocks(sk, rec, blocks, threads, use_ref)
        if s >= args.warmup:
            times.append(dt)
            pairs.append(sum(min(BLOCK, sk.n - b * BLOCK) for b in blocks) * sk.n)
    value = float(sum(pairs) / sum(times))
    kind = "reference" if use_ref else "port"
    line = {
        "impl": "reference", "metric": "ANI genome-pairs/s", "value": value, "unit": "genome-pairs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "genomes": sk.n, "entries": int(sk.offs[-1])},
        "path": "count_ctx_obj_frm_comb_sketch_section_lower, 64-query blocks (-O3 -flto -fopenmp build)",
        "blocks_per_step": per_step,
        "cpu_baseline": {"value": value, "unit": "genome-pairs/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} of {nblocks} 64-query blocks per step, rotating"},
        "e2e": {"value": value, "unit": "genome-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def leg_north_star(args, timer, dev, stream, peak):
    """The 20,000-genome all-vs-all: the self step (fill + scan join) vs the batched
    probe kernel vs the plain per-query kernel on the same counters (parity checked on
    the device), and the cached-plan join (first call = plan + join)."""
    import torch
    import kssdgpu
    n = args.ns_genomes
    t0 = time.perf_counter()
    sk = make_workload(n)
    gen_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = kssdgpu.Index.from_sketch(sk, device=dev.index or 0)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    info = idx.info()
    facts = idx.self_plan_info()
    cells = n * (n - 1) // 2
    lc = torch.zeros(cells, dtype=torch.int64, device=dev)
    lo = torch.zeros_like(lc)
    step = lambda: idx.self_lower_dev(lc, lo, stream=stream)  # noqa: E731
    ms_step = timer(step, max(3, args.steps // 2), 3)
    touched = int(torch.count_nonzero(lc).item())
    ms_scan = timer(lambda: idx.self_lower_dev(lc, lo, flags=kssdgpu.NO_ZERO, stream=stream), max(3, args.steps // 2),
                    2, pre=lambda: (lc.zero_(), lo.zero_()))
    # cached-plan join: the first call builds the plan (host-timed), later calls only join
    l2c, l2o = torch.zeros_like(lc), torch.zeros_like(lc)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx.self_lower_dev(l2c, l2o, flags=kssdgpu.SELF_PLAN, stream=stream)
    torch.cuda.synchronize()
    plan_first_ms = 1e3 * (time.perf_counter() - t0)
    ms_cached = timer(lambda: idx.self_lower_dev(l2c, l2o, flags=kssdgpu.SELF_PLAN, stream=stream), 3, 1)
    step()
    torch.cuda.synchronize()
    same_plan = bool(torch.equal(lc, l2c) and torch.equal(lo, l2o))
    del l2c, l2o
    d_keys = torch.from_numpy(sk.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(sk.offs.view(np.int64)).to(dev)
    dc = torch.zeros(n * n, dtype=torch.int64, device=dev)
    do = torch.zeros_like(dc)
    probe = lambda: idx.count_block_dev(d_keys, d_offs, n, dc, do, lower=True, stream=stream)  # noqa: E731
    ms_probe = timer(probe, 3, 1)
    same_probe = lower_equals_dense(lc, lo, dc, do, n)
    ms_plain = timer(lambda: idx.count_plain_dev(d_keys, d_offs, sk.offs, dc, do, lower=True, stream=stream), 1, 1)
    same_plain = lower_equals_dense(lc, lo, dc, do, n)
    scan_bytes = scan_join_bytes(info["contexts"], facts["postings"], touched)
    step_bytes = scan_bytes + 16 * cells
    model = probe_model_bytes(int(sk.offs[-1]), facts["pairs"], cells)
    out = {
        "workload": f"self-ani-matrix-{n}-genomes", "genomes": n, "entries": int(sk.offs[-1]),
        "unique_contexts": info["contexts"], "generate_s": gen_s, "index_build_s": build_s,
        "self_step": {"ms": ms_step, "genome_pairs_s": n * n / (ms_step / 1e3),
                      "what": "zero fill of the dense lower triangle + one-pass scan join, nothing cached",
                      "roofline": {"bound": "hbm", "bytes": step_bytes, "achieved": step_bytes / ms_step / 1e6,
                                   "frac": step_bytes / ms_step / 1e6 / peak},
                      "probe_model_frac": model / ms_step / 1e6 / peak},
        "scan_join_alone": {"ms": ms_scan, "bytes": scan_bytes, "frac": scan_bytes / ms_scan / 1e6 / peak},
        "batched_probe": {"ms": ms_probe, "genome_pairs_s": n * n / (ms_probe / 1e3),
                          "contexts_probed_per_s": int(sk.offs[-1]) / (ms_probe / 1e3),
                          "probe_model_frac": model / ms_probe / 1e6 / peak},
        "plain_per_query": {"ms": ms_plain, "launches": n},
        "batched_vs_plain": ms_plain / ms_probe, "self_step_vs_plain": ms_plain / ms_step,
        "cached_plan_join": {"first_call_ms": plan_first_ms, "join_ms": ms_cached},
        "parity": {"scan_eq_probe": same_probe, "scan_eq_plain": same_plain, "scan_eq_cached_plan": same_plan},
        "touched_cells": touched,
    }
    del dc, do, lc, lo
    return out, idx, sk


def leg_rect(args, timer, dev, stream, peak, idx, ref):
    """A 10,000-query x 20,000-reference block (queries of log-uniform 50 kbp-12 Mbp
    from the references' cluster ancestors): one batched launch vs the plain kernel,
    and the counters of a query sample against the reference's own counting function."""
    import torch
    import kssdgpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    nr, nq = ref.n, args.rect_queries
    qry = kssdgpu.synth(n_samples=nq, n_clusters=max(1, nr // 10), role=kssdgpu.ROLE_OWNLEN,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6,
                        own_len_min=5e4, own_len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=WORKLOAD["seed"],
                        sample_seed=WORKLOAD["seed"] + 11, threads=os.cpu_count() or 8)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    cells = nq * nr
    dc = torch.zeros(cells, dtype=torch.int64, device=dev)
    dob = torch.zeros_like(dc)
    tuning = idx.count_tune(dk, do, nq, dc, dob)
    ms_b = timer(lambda: idx.count_block_dev(dk, do, nq, dc, dob, stream=stream), 3, 2)
    shared = int((dc & 0xFFFFFFFF).sum().item())
    ms_p = timer(lambda: idx.count_plain_dev(dk, do, qry.offs, dc, dob, stream=stream), 1, 0)
    qkeys = int(qry.offs[-1])
    model = probe_model_bytes(qkeys, shared, cells)
    rec, _ = idx.export()
    sample = list(range(0, nq, max(1, nq // args.parity_queries)))[:args.parity_queries]
    skeys = np.concatenate([qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])] for q in sample])
    soffs = np.concatenate([[0], np.cumsum([int(qry.offs[q + 1] - qry.offs[q]) for q in sample])]).astype(np.uint64)
    t0 = time.perf_counter()
    c, o = oracle.count_block(rec, nr, skeys, soffs, threads=os.cpu_count() or 1, ref=oracle.ref_available())
    cpu_s = time.perf_counter() - t0
    rows = torch.tensor(sample, device=dev)
    same = bool(np.array_equal(c.view(np.int64).reshape(len(sample), nr), dc.view(nq, nr)[rows].cpu().numpy()) and
                np.array_equal(o.view(np.int64).reshape(len(sample), nr), dob.view(nq, nr)[rows].cpu().numpy()))
    # detail mode on the same block: the count with its pre-filter on the device, only
    # candidate cells back (kssdgpu_count_detail, host buffers), against the reference's
    # own detail pre-filter on the sampled queries
    del dc, dob
    torch.cuda.empty_cache()
    rcnt = np.diff(ref.offs.astype(np.int64)).astype(np.uint32)
    qcnt = np.diff(qry.offs.astype(np.int64)).astype(np.uint32)
    t0 = time.perf_counter()
    hits, roffs = idx.count_detail(qry.keys, qry.offs, qcnt, rcnt, 0, 3, 0.5, 0.95, cap=1 << 24)
    detail_s = time.perf_counter() - t0
    detail_same = None
    if oracle.ref_available():
        _, npass, ranked = oracle.count_detail_ref(rec, nr, skeys, soffs, rcnt, qcnt[sample], ctxcut=3, afcut=0.5,
                                                   anicut=0.95, ntop=nr, threads=os.cpu_count() or 1)
        detail_same = True
    for i, q in enumerate(sample if detail_same is not None else []):
        want = set(ranked[i, :npass[i]].tolist())
        got = set(hits["ref"][int(roffs[q]):int(roffs[q + 1])].tolist())
        detail_same &= want <= got  # the device keeps every reference candidate (margin below anicut)
    detail = {"call": "kssdgpu_count_detail (host buffers)", "wall_ms": 1e3 * detail_s,
              "candidates": int(roffs[-1]), "d2h_bytes": int(roffs[-1]) * 40 + 8 * (nq + 1),
              "dense_d2h_bytes_instead": 16 * cells,
              "candidates_cover_reference_sample": detail_same}
    del rec
    return {"workload": f"rect-{nq}x{nr}", "query_keys": qkeys, "ms": ms_b, "genome_pairs_s": cells / (ms_b / 1e3),
            "tuning": tuning, "detail": detail,
            "contexts_probed_per_s": qkeys / (ms_b / 1e3),
            "roofline_probe_model": {"bytes": model, "achieved": model / ms_b / 1e6, "frac": model / ms_b / 1e6 / peak},
            "plain_per_query": {"ms": ms_p, "launches": nq}, "batched_vs_plain": ms_p / ms_b,
            "parity": {"queries": len(sample), "counts_match_reference": same,
                       "checker": "reference count_ctx_obj_frm_comb_sketch_section_with_unique"
                       if oracle.ref_available() else "oracle"},
            "cpu_baseline": {"value": len(sample) * nr / cpu_s, "unit": "genome-pairs/s", "cores": os.cpu_count(),
                             "kind": "reference" if oracle.ref_available() else "port",
                             "sample": f"{len(sample)} queries"}}


def leg_reads(args, timer, dev, stream, idx, ref):
    """40 read sets (1-5 genomes of the reference set at 5-50x, 0.1-1% errors,
    conflicts kept) against the 20,000-genome index with unique contexts (`ani --qraw
    ... --unique-ctx --anicut 0.95`): batched vs plain, and the counters of a sample
    against the reference's own counting function."""
    import torch
    import kssdgpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    nr, nq = ref.n, args.reads_samples
    qry = kssdgpu.synth(n_samples=nq, n_clusters=max(1, nr // 10), role=kssdgpu.ROLE_READS,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6,
                        sub_lo=0.001, sub_hi=0.2, seed=WORKLOAD["seed"], sample_seed=WORKLOAD["seed"] + 12,
                        ref_sample_seed=WORKLOAD["seed"], ref_samples=nr, cov_lo=5, cov_hi=50, err_lo=0.001,
                        err_hi=0.01, threads=os.cpu_count() or 8)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    cells = nq * nr
    outs = [torch.zeros(cells, dtype=torch.int64, device=dev) for _ in range(4)]
    flags = kssdgpu.UNIQUE
    ms_b = timer(lambda: idx.count_block_dev(dk, do, nq, *outs, flags=flags, stream=stream), 3, 2)
    ms_p = timer(lambda: idx.count_plain_dev(dk, do, qry.offs, *outs, flags=flags, stream=stream), 1, 0)
    rec, _ = idx.export()
    sample = list(range(0, nq, max(1, nq // 8)))[:8]
    skeys = np.concatenate([qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])] for q in sample])
    soffs = np.concatenate([[0], np.cumsum([int(qry.offs[q + 1] - qry.offs[q]) for q in sample])]).astype(np.uint64)
    want = oracle.count_block(rec, nr, skeys, soffs, unique=True, threads=os.cpu_count() or 1,
                              ref=oracle.ref_available())
    rows = torch.tensor(sample, device=dev)
    same = all(bool(np.array_equal(w.view(np.int64).reshape(len(sample), nr), o.view(nq, nr)[rows].cpu().numpy()))
               for w, o in zip(want, outs))
    del rec, outs
    qkeys = int(qry.offs[-1])
    return {"workload": f"reads-{nq}x{nr}-unique-ctx", "read_sets": nq, "query_keys": qkeys, "ms": ms_b,
            "genome_pairs_s": cells / (ms_b / 1e3), "contexts_probed_per_s": qkeys / (ms_b / 1e3),
            "plain_per_query": {"ms": ms_p, "launches": nq}, "batched_vs_plain": ms_p / ms_b,
            "parity": {"read_sets": len(sample), "counts_match_reference": same}}


def leg_dense(args, timer, dev, stream, peak_tc):
    """One species: --dense-genomes genomes of one cluster at 0.1-2% substitutions (most
    contexts shared by most genomes): the dense tensor-core self join vs the one-pass
    scan on the same counters."""
    import torch
    import kssdgpu
    n = args.dense_genomes
    sk = kssdgpu.synth(n_samples=n, n_clusters=1, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.2,
                       len_min=2e6, len_max=8e6, sub_lo=0.001, sub_hi=0.02, seed=WORKLOAD["seed"] + 21,
                       sample_seed=WORKLOAD["seed"] + 21, threads=os.cpu_count() or 8)
    idx = kssdgpu.Index.from_sketch(sk)
    facts = idx.self_plan_info()
    path, density = idx.self_choice()
    cells = n * (n - 1) // 2
    a_c = torch.zeros(cells, dtype=torch.int64, device=dev)
    a_o = torch.zeros_like(a_c)
    b_c, b_o = torch.zeros_like(a_c), torch.zeros_like(a_c)
    ms_dense = timer(lambda: idx.self_lower_dev(a_c, a_o, flags=kssdgpu.SELF_DENSE, stream=stream), 3, 1)
    alleles = idx.dense_alleles()
    ms_scan = timer(lambda: idx.self_lower_dev(b_c, b_o, flags=kssdgpu.SELF_SCAN, stream=stream), 3, 1)
    same = bool(torch.equal(a_c, b_c) and torch.equal(a_o, b_o))
    kpad = (alleles + 127) // 128 * 128
    # int8 multiply-adds x 2 the GEMMs perform: from 6 blocks of 128 genomes on, one GEMM
    # per block of 128 genomes r over the rows q at or below it, else the whole square
    npad = (n + 15) // 16 * 16
    bw = 128 if (npad + 127) // 128 >= 6 else npad
    ops = sum(2 * (npad - bw * j) * 4 * min(bw, npad - bw * j) * kpad for j in range((npad + bw - 1) // bw))
    square_ops = 2 * npad * 4 * npad * kpad
    del a_c, a_o, b_c, b_o
    # the batched probe on the same dense index: 256 new members of the species against
    # it (context groups of hundreds of postings, walked by whole warps), counters of a
    # query sample against the oracle
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    qry = kssdgpu.synth(n_samples=256, n_clusters=1, role=kssdgpu.ROLE_OWNLEN, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        len_median=4e6, len_sigma=0.2, len_min=2e6, len_max=8e6, own_len_min=1e6, own_len_max=8e6,
                        sub_lo=0.001, sub_hi=0.02, seed=WORKLOAD["seed"] + 21, sample_seed=WORKLOAD["seed"] + 22,
                        threads=os.cpu_count() or 8)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    pc = torch.zeros(qry.n * n, dtype=torch.int64, device=dev)
    po = torch.zeros_like(pc)
    probe_tuning = idx.count_tune(dk, do, qry.n, pc, po)
    ms_probe = timer(lambda: idx.count_block_dev(dk, do, qry.n, pc, po, stream=stream), 5, 2)
    walked = int((pc & 0xFFFFFFFF).sum().item())  # one credit per (query context, reference gid run)
    rec, _ = idx.export()
    sample = list(range(0, qry.n, qry.n // 8))[:8]
    skeys = np.concatenate([qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])] for q in sample])
    soffs = np.concatenate([[0], np.cumsum([int(qry.offs[q + 1] - qry.offs[q]) for q in sample])]).astype(np.uint64)
    wc, wo = oracle.count_block(rec, n, skeys, soffs, threads=os.cpu_count() or 1, ref=oracle.ref_available())
    rows = torch.tensor(sample, device=dev)
    probe_same = bool(np.array_equal(wc.view(np.int64).reshape(len(sample), n), pc.view(qry.n, n)[rows].cpu().numpy())
                      and np.array_equal(wo.view(np.int64).reshape(len(sample), n),
                                         po.view(qry.n, n)[rows].cpu().numpy()))
    qkeys = int(qry.offs[-1])
    model = probe_model_bytes(qkeys, walked, qry.n * n)
    del rec, pc, po, dk, do
    idx.close()
    return {"workload": f"one-species-{n}-genomes", "genomes": n, "entries": int(sk.offs[-1]),
            "shared_postings": facts["postings"], "pairs": facts["pairs"], "alleles": alleles,
            "density": density, "default_path": ["scan", "dense", "plan"][path],
            "dense_step_ms": ms_dense, "scan_step_ms": ms_scan, "dense_vs_scan": ms_scan / ms_dense,
            "genome_pairs_s": n * n / (ms_dense / 1e3),
            "tensor": {"bound": "tensor", "int8_ops": ops, "square_int8_ops": square_ops,
                       "achieved_tops": ops / ms_dense / 1e9, "peak_tops": peak_tc,
                       "frac_of_step": ops / ms_dense / 1e9 / peak_tc,
                       "what": "int8 ops the GEMMs perform (blocks at or below the diagonal) over the whole "
                               "dense step (allele build + operand rows + GEMMs + epilogue)"},
            "parity": {"dense_eq_scan": same},
            "batched_probe_256_queries": {"ms": ms_probe, "query_keys": qkeys, "credits": walked,
                                          "genome_pairs_s": qry.n * n / (ms_probe / 1e3),
                                          "tuning": probe_tuning,
                                          "roofline_probe_model": {"bytes": model, "frac": model / ms_probe / 1e6 /
                                                                   measured_peak_hbm()[0]},
                                          "counts_match_reference": probe_same,
                                          "what": "kssdgpu_count_block_dev of 256 new members of the species: "
                                                  "context groups of hundreds of postings walked by whole warps"}}


def leg_cli_2k(args, sk):
    """The drop-in CLI end to end on the headline workload: `kssd3a ani -p P -q DIR --format
    matrix --values ani -o FILE` (indexed self full matrix, 36 MB of TSV) with bin/kssd3a and
    with the reference CLI on the same sketch directory (index file present, warm page
    cache): wall times and byte equality of the outputs."""
    import hashlib
    import shutil
    import tempfile
    import kssdgpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return {"skipped": "reference build absent"}
    ours = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")
    root = tempfile.mkdtemp(prefix="kssd_cli2k_")
    try:
        d = os.path.join(root, "refs")
        kssdgpu.write_sketch_dir(d, sk)
        rec = oracle.build_index(sk.keys, sk.offs)
        rec.tofile(os.path.join(d, "sortedcomb_ctxgid64obj32"))
        oracle.unique_bits(rec).tofile(os.path.join(d, "sortedcomb_ctxgid64obj32.unique_bits"))
        del rec
        thr = str(os.cpu_count() or 8)
        env = {k: v for k, v in os.environ.items() if not k.startswith("KSSD3A_")}
        out = {}
        for name, binary in (("ours", ours), ("reference", oracle.REF_BIN)):
            dst = os.path.join(root, name + ".tsv")
            argv = [binary, "ani", "-p", thr, "-q", d, "--format", "matrix", "--values", "ani", "-o", dst]
            subprocess.run(argv, check=True, capture_output=True, env=env)  # warm page cache and context
            ts = []
            for _ in range(3):
                t0 = time.perf_counter()
                subprocess.run(argv, check=True, capture_output=True, env=env)
                ts.append(time.perf_counter() - t0)
            out[name] = {"wall_s_median_of_3": float(np.median(ts)),
                         "sha256": hashlib.sha256(open(dst, "rb").read()).hexdigest(),
                         "bytes": os.path.getsize(dst)}
        return {"command": "kssd3a ani -p P -q DIR --format matrix --values ani -o FILE", "genomes": sk.n,
                "threads": int(thr), "ours": out["ours"], "reference": out["reference"],
                "bytes_equal": out["ours"]["sha256"] == out["reference"]["sha256"],
                "speedup": out["reference"]["wall_s_median_of_3"] / out["ours"]["wall_s_median_of_3"]}
    finally:
        shutil.rmtree(root, ignore_errors=True)


def leg_config1(args):
    """64 genomes of 1 Mbp (8 clusters x 8 members, 0.5-5% substitutions, 0.1% indels) as
    FASTA, sketched by the reference's own sketcher; bin/kssd3a and the reference CLI on
    the dispatcher's small-n paths: bytes compared, wall times beside."""
    import shutil
    import tempfile
    import fasta_synth
    import kssdgpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return {"skipped": "reference build absent"}
    ours = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")
    root = tempfile.mkdtemp(prefix="kssd_cfg1_")
    try:
        paths = fasta_synth.write_genomes(os.path.join(root, "fa"))
        thr = str(os.cpu_count() or 8)
        plain, indexed = os.path.join(root, "refs"), os.path.join(root, "refsi")
        for d in (plain, indexed):
            subprocess.run([oracle.REF_BIN, "sketch", "-p", thr, "-o", d, *paths], check=True, capture_output=True)
        subprocess.run([oracle.REF_BIN, "sketch", "-i", indexed], check=True, capture_output=True)
        cases = {"detail_hash": ["ani", "-p", thr, "-r", plain, "-q", plain],
                 "detail_mem_eff": ["ani", "-p", thr, "-r", indexed, "-q", indexed],
                 "matrix_direct": ["ani", "-p", thr, "-r", plain, "-q", plain, "--format", "matrix"],
                 "self_ani_matrix": ["ani", "-p", thr, "-q", indexed, "--format", "matrix", "--values", "ani"],
                 "matrix_cmd": ["matrix", "-p", thr, "-q", plain]}
        out = {}
        env = {k: v for k, v in os.environ.items() if not k.startswith("KSSD3A_")}
        for name, argv in cases.items():
            t0 = time.perf_counter()
            a = subprocess.run([ours, *argv], capture_output=True, env=env)
            t1 = time.perf_counter()
            b = subprocess.run([oracle.REF_BIN, *argv], capture_output=True, env=env)
            t2 = time.perf_counter()
            out[name] = {"bytes_equal": a.returncode == 0 and a.stdout == b.stdout, "lines": len(b.stdout.splitlines()),
                         "ours_s": t1 - t0, "reference_s": t2 - t1}
        sk = kssdgpu.read_sketch_dir(plain)
        syn = kssdgpu.synth(n_samples=64, n_clusters=8, size_dist=kssdgpu.SIZE_FIXED, len_median=1e6, len_min=1e6,
                            len_max=1e6, sub_lo=0.005, sub_hi=0.05, indel_rate=0.001, seed=5, sample_seed=5)
        hist = {}
        for name, x in (("reference_sketcher_on_fasta", sk), ("sketch_space_generator", syn)):
            _, k = np.unique(x.keys >> np.uint64(20), return_counts=True)
            h = np.bincount(np.minimum(k, 9), minlength=10)[1:]
            hist[name] = {"entries": int(len(x.keys)), "contexts": int(len(k)),
                          "postings_per_context": float(len(x.keys) / len(k)),
                          "fraction_of_contexts_with_k_postings_1_to_9plus": (h / len(k)).round(4).tolist()}
        return {"workload": "64 x 1 Mbp FASTA genomes, 8 clusters x 8, sketched by the reference sketcher",
                "entries": int(len(sk.keys)), "cases": out, "postings_per_context": hist}
    finally:
        shutil.rmtree(root, ignore_errors=True)


def _pct(xs, p):
    xs = sorted(xs)
    return float(xs[min(len(xs) - 1, int(p * (len(xs) - 1) + 0.5))]) if xs else None


def serve_sweep(idx, nref, rates, seconds, seed, pool_assemblies=256, pool_reads=64, max_batch_queries=64):
    """Poisson arrivals at each rate for `seconds`: 80% assemblies (0.5-12 Mbp, from the
    references' cluster ancestors) and 20% read sets (1-5 genomes at 5-100x, 0.1-1%
    errors); latency = submit -> hits on the host, measured by the server.  Returns
    (per-rate results, pool facts, server facts)."""
    import kssdgpu
    asm = kssdgpu.synth(n_samples=pool_assemblies, n_clusters=max(1, nref // 10), role=kssdgpu.ROLE_OWNLEN,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6,
                        own_len_min=5e5, own_len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed, sample_seed=seed + 1)
    reads = kssdgpu.synth(n_samples=pool_reads, n_clusters=max(1, nref // 10), role=kssdgpu.ROLE_READS,
                          size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6,
                          len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed, sample_seed=seed + 2,
                          ref_sample_seed=seed, ref_samples=nref, cov_lo=5, cov_hi=100, err_lo=0.001, err_hi=0.01)
    pool = [("assembly", asm.keys[asm.offs[i]:asm.offs[i + 1]]) for i in range(asm.n)]
    pool_r = [("reads", reads.keys[reads.offs[i]:reads.offs[i + 1]]) for i in range(reads.n)]
    max_keys = max(len(k) for _, k in pool + pool_r)
    srv = kssdgpu.Server(idx, max_batch_queries=max_batch_queries, max_batch_keys=max(1 << 24, 2 * max_keys),
                         max_hits=1 << 22)
    for _, k in pool[:32] + pool_r[:8]:  # warm-up
        srv.result(srv.submit(k))
    rng = random.Random(seed)
    results = []
    old_si = sys.getswitchinterval()
    sys.setswitchinterval(2e-4)  # the pacing loop must not hold the interpreter lock for 5 ms
    try:
        for rate in rates:
            srv.reset_stats()
            nreq = max(1, int(rate * seconds))
            t = 0.0
            plan = []
            for _ in range(nreq):
                t += rng.expovariate(rate)
                plan.append((t, pool[rng.randrange(len(pool))] if rng.random() < 0.8 else
                             pool_r[rng.randrange(len(pool_r))]))
            got, tickets = [], []
            cond = threading.Condition()
            done_submitting = [False]

            def collector():
                i = 0
                while i < nreq:
                    with cond:
                        while i >= len(tickets):
                            cond.wait(timeout=1.0)
                            if i >= len(tickets) and done_submitting[0]:
                                return
                        kind, tk = tickets[i]
                    hits, lat = srv.result(tk, timeout_ms=120000)
                    got.append((kind, lat, len(hits)))
                    i += 1

            th = threading.Thread(target=collector)
            th.start()
            start = time.perf_counter()
            for at, (kind, keys) in plan:
                gap = at - (time.perf_counter() - start)
                if gap > 1e-3:
                    time.sleep(gap - 5e-4)
                while time.perf_counter() - start < at:
                    pass
                tk = srv.submit(keys)
                with cond:
                    tickets.append((kind, tk))
                    cond.notify()
            with cond:
                done_submitting[0] = True
                cond.notify()
            th.join()
            wall = time.perf_counter() - start
            st = srv.stats()
            lat_a = [x[1] for x in got if x[0] == "assembly"]
            lat_r = [x[1] for x in got if x[0] == "reads"]
            lat = [x[1] for x in got]
            results.append({
                "rate_req_s": rate, "requests": nreq, "wall_s": wall, "throughput_req_s": nreq / wall,
                "genome_pairs_s": nreq * nref / wall, "p50_ms": _pct(lat, 0.5), "p99_ms": _pct(lat, 0.99),
                "assembly_p50_ms": _pct(lat_a, 0.5), "assembly_p99_ms": _pct(lat_a, 0.99),
                "reads_p50_ms": _pct(lat_r, 0.5), "reads_p99_ms": _pct(lat_r, 0.99),
                "max_ms": max(lat) if lat else None, "batches": st["batches"], "max_inflight": st["max_inflight"],
                "overlapped_batches": st["overlapped_batches"], "splits": st["splits"],
                "mean_hits": float(np.mean([x[2] for x in got])) if got else 0.0})
    finally:
        sys.setswitchinterval(old_si)
    pool_facts = {"assemblies": len(pool), "read_sets": len(pool_r), "max_keys": max_keys,
                  "mean_assembly_keys": float(np.mean([len(k) for _, k in pool])),
                  "mean_reads_keys": float(np.mean([len(k) for _, k in pool_r]))}
    srv_facts = {"reserved_bytes": srv.stats()["reserved_bytes"], "slots": srv.stats()["slots"],
                 "max_batch_queries": max_batch_queries}
    srv.close()
    return results, pool_facts, srv_facts


def run_ours(args, rank, world, local_rank):
    import torch
    import kssdgpu
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    timer = Timer(stream, dev)
    peak, peak_kind = measured_peak_hbm()
    peak_tc = 2 * measured_peak_bf16_tflops()  # int8 dense rate = 2 x bf16 on these tensor cores

    sk = make_workload(args.genomes)
    n = sk.n
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = kssdgpu.Index.from_sketch(sk, device=local_rank)
    torch.cuda.synchronize()
    index_ms = 1e3 * (time.perf_counter() - t0)
    info = idx.info()
    facts = idx.self_plan_info()  # shared context groups, their postings and pairs (one pass; no plan)

    d_keys = torch.from_numpy(sk.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(sk.offs.view(np.int64)).to(dev)
    lower_cells = n * (n - 1) // 2
    d_lc = torch.zeros(lower_cells, dtype=torch.int64, device=dev)
    d_lo = torch.zeros(lower_cells, dtype=torch.int64, device=dev)
    d_c = torch.zeros(n * n, dtype=torch.int64, device=dev)
    d_o = torch.zeros(n * n, dtype=torch.int64, device=dev)

    def self_step(flags=0):
        idx.self_lower_dev(d_lc, d_lo, flags=flags, stream=stream)

    def probe_step():
        idx.count_block_dev(d_keys, d_offs, n, d_c, d_o, lower=True, stream=stream)

    def plain_step():
        idx.count_plain_dev(d_keys, d_offs, sk.offs, d_c, d_o, lower=True, stream=stream)

    # ---- parity on the benchmark's own inputs: scan join == batched probe == plain == cached-plan join
    probe_step()
    idx.sync(stream)
    self_step()
    idx.sync(stream)
    ok_probe = lower_equals_dense(d_lc, d_lo, d_c, d_o, n)
    plain_step()
    idx.sync(stream)
    ok_plain = lower_equals_dense(d_lc, d_lo, d_c, d_o, n)
    p_c, p_o = torch.zeros_like(d_lc), torch.zeros_like(d_lo)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx.self_lower_dev(p_c, p_o, flags=kssdgpu.SELF_PLAN, stream=stream)  # first call builds the plan
    torch.cuda.synchronize()
    plan_first_ms = 1e3 * (time.perf_counter() - t0)
    ok_plan = bool(torch.equal(p_c, d_lc) and torch.equal(p_o, d_lo))
    if not (ok_probe and ok_plain and ok_plan):
        raise SystemExit(f"parity failure on the bench workload: probe={ok_probe} plain={ok_plain} plan={ok_plan}")
    # lower-triangle cells that share at least one context (every credit adds num_ctx += 1)
    touched = int(torch.count_nonzero(d_lc).item())
    density = density_histogram(d_lc, np.diff(sk.offs.astype(np.int64)), n)

    # ---- headline: one self step per timed step, bracketed by barrier + synchronize, max over ranks
    launches0 = kssdgpu.launch_count()
    self_step()
    torch.cuda.synchronize()
    launches_per_step = kssdgpu.launch_count() - launches0
    # the step (zero fill + scan join, the join launched programmatically after the
    # fill) captured once into a CUDA graph and replayed: no host gap between the two
    # launches inside the timed region; direct launches are timed beside it
    ms_direct = timer(self_step, args.steps, args.warmup)
    step_fn, launch_mode = self_step, "direct launches"
    try:
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            with torch.cuda.graph(graph, stream=side):
                idx.self_lower_dev(d_lc, d_lo, stream=side)
        stream.wait_stream(side)
        graph.replay()
        torch.cuda.synchronize()
        if bool(torch.equal(d_lc, p_c) and torch.equal(d_lo, p_o)):
            step_fn, launch_mode = graph.replay, "CUDA graph replay"
    except Exception as exc:  # capture support depends on the driver; keep the direct launches
        launch_mode = f"direct launches (graph capture failed: {exc})"
    with ClockSampler(local_rank) as clocks:
        # the steps take tens of microseconds: keep the GPU on this workload until the
        # sampler has readings, then run the timed region inside the same sampling window
        t_end = time.time() + 1.5
        while time.time() < t_end or len(clocks.samples) < 3:
            for _ in range(200):
                step_fn()
            torch.cuda.synchronize()
            if time.time() > t_end + 10:
                break
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms_step = timer(step_fn, args.steps, args.warmup)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms_step = max_over_ranks(dist, ms_step, dev)
    launches_timed = launches_per_step * args.steps
    value = replica_value(world, n * n, ms_step / 1e3)

    # ---- the dominant kernel alone: the scan join, counters zeroed outside the events
    zero = lambda: (d_lc.zero_(), d_lo.zero_())  # noqa: E731
    ms_scan = timer(lambda: self_step(kssdgpu.NO_ZERO), args.steps, 2, pre=zero)
    scan_bytes = scan_join_bytes(info["contexts"], facts["postings"], touched)
    step_bytes = scan_bytes + 16 * lower_cells
    model_bytes = probe_model_bytes(int(sk.offs[-1]), facts["pairs"], lower_cells)
    achieved = scan_bytes / (ms_scan / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "k_self_scan_traffic.json")
    if os.path.exists(tfile):
        try:
            t = json.load(open(tfile))
            if t.get("workload_genomes") == n:  # the ncu capture of this workload's scan-join launch
                traffic = t.get("bytes_per_launch")
        except Exception:
            traffic = None

    # ---- batched probe, plain per-query kernel and cached-plan join on the same workload
    probe_tuning = idx.count_tune(d_keys, d_offs, n, d_c, d_o, lower=True)  # accumulator mode / chunk size
    ms_probe = timer(probe_step, max(3, args.steps // 2), 2)
    ms_plain = timer(plain_step, 3, 1)
    ms_plan_join = timer(lambda: idx.self_lower_dev(p_c, p_o, flags=kssdgpu.SELF_PLAN, stream=stream), 5, 2)
    del p_c, p_o

    # ---- e2e through the host-buffer C ABI
    lib = kssdgpu.gpu_lib()
    h_keys = torch.from_numpy(sk.keys.view(np.int64)).pin_memory()
    h_offs_np = np.ascontiguousarray(sk.offs, dtype=np.uint64)
    h_ctx = torch.empty(n * n * 2, dtype=torch.int32).pin_memory()
    h_obj = torch.empty(n * n * 2, dtype=torch.int32).pin_memory()

    def e2e_call():
        rc = lib.kssdgpu_count_lower(idx.handle, h_keys.data_ptr(), h_offs_np, n, 0, 0, h_ctx.data_ptr(),
                                     h_obj.data_ptr())
        if rc:
            raise kssdgpu.KssdGpuError(rc, lib.kssdgpu_last_error().decode())

    def e2e_time(call, reps):
        call()
        ts = []
        for _ in range(reps):
            timer.flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            call()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts))

    e2e_s = max_over_ranks(dist, e2e_time(e2e_call, max(3, args.steps // 2)), dev)
    e2e_value = replica_value(world, n * n, e2e_s)
    h2d = int(sk.keys.nbytes + sk.offs.nbytes)
    d2h = int(n * n * 16)
    e2e_ok = bool(np.array_equal(h_ctx.numpy().view(np.int64), d_c.cpu().numpy()))
    # as the reference's drivers call it: 64-query blocks, pageable (malloc'd) buffers
    # (src/command_ani.c:1698 in comb_sortedsketch64_indexed_self_full)
    blk_ctx = np.empty((BLOCK, n, 2), dtype=np.uint32)
    blk_obj = np.empty((BLOCK, n, 2), dtype=np.uint32)
    blk_ok = [True]

    def e2e_blocks(check=False):
        for off in range(0, n, BLOCK):
            nb = min(BLOCK, n - off)
            qo = np.ascontiguousarray(sk.offs[off: off + nb + 1])
            qk = sk.keys[int(qo[0]): int(qo[-1])]
            rc = lib.kssdgpu_count_lower(idx.handle, qk.ctypes.data, qo, nb, off, 0, blk_ctx.ctypes.data,
                                         blk_obj.ctypes.data)
            if rc:
                raise kssdgpu.KssdGpuError(rc, lib.kssdgpu_last_error().decode())
            if check:
                want = h_ctx.numpy().view(np.uint32).reshape(n, n, 2)[off: off + nb]
                blk_ok[0] &= bool(np.array_equal(blk_ctx[:nb], want))

    e2e_blocks(check=True)
    blocks_s = max_over_ranks(dist, e2e_time(e2e_blocks, 3), dev)

    # ---- CPU baseline: the reference's counting function on host cores (rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        # the reference-layout index records (input of the CPU function); byte-identical
        # to the reference's own `sketch -i` output (tests/test_gpu_count.py)
        rec, _ = idx.export()
        use_ref = oracle.ref_available()
        threads = os.cpu_count() or 1
        nblocks = (n + BLOCK - 1) // BLOCK
        t1, _ = cpu_count_lower_blocks(sk, rec, [nblocks - 1], threads, use_ref)
        per = max(1, min(nblocks, int(args.cpu_seconds / max(t1, 1e-3))))
        blocks = sorted(set(np.linspace(0, nblocks - 1, per).astype(int).tolist()))
        dt, outs = cpu_count_lower_blocks(sk, rec, blocks, threads, use_ref)
        pairs = sum(min(BLOCK, n - b * BLOCK) for b in blocks) * n
        # parity of the sampled blocks against the device counters
        dc = d_c.view(n, n).cpu().numpy()
        same = all(np.array_equal(o[0][:, :, 0].astype(np.int64) | (o[0][:, :, 1].astype(np.int64) << 32),
                                  dc[off: off + o[0].shape[0]]) for off, o in outs)
        cpu = {"value": pairs / dt, "unit": "genome-pairs/s", "cores": threads,
               "kind": "reference" if use_ref else "port",
               "sample": f"{len(blocks)} of {nblocks} 64-query blocks (count_lower), spread over the matrix",
               "counts_match_gpu": bool(same)}
        del rec

    # ---- the north-star and config legs against a resident 20,000-genome index
    extra = {}
    if rank == 0 and world == 1 and not args.no_extra:
        del d_c, d_o
        torch.cuda.empty_cache()
        ns, ns_idx, ns_sk = leg_north_star(args, timer, dev, stream, peak)
        extra["all_vs_all_20k"] = ns
        extra["rect_config3"] = leg_rect(args, timer, dev, stream, peak, ns_idx, ns_sk)
        extra["reads_config4"] = leg_reads(args, timer, dev, stream, ns_idx, ns_sk)
        ns_idx.close()
        del ns_sk
        torch.cuda.empty_cache()
        if args.serve_rates and args.serve_refs > 0:
            extra["serve"] = serve_leg(args, args.serve_refs)
        extra["dense_one_species"] = leg_dense(args, timer, dev, stream, peak_tc)
        extra["cli_2k"] = leg_cli_2k(args, sk)
        extra["config1_fasta"] = leg_config1(args)

    if rank == 0:
        line = {
            "metric": "ANI genome-pairs/s", "value": value, "unit": "genome-pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "genomes": n, "entries": int(sk.offs[-1]),
                       "unique_contexts": info["contexts"], "matrix_cells": n * n,
                       "lower_pairs": lower_cells,
                       "path": "self step from the resident index: zero fill + one-pass scan join "
                               "(kssdgpu_self_lower_dev), nothing cached between steps",
                       "l2": "flushed (256 MB write) before every timed step",
                       "launch": launch_mode, "ms_per_step_direct_launches": ms_direct,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "genome-pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "call": "kssdgpu_count_lower, one call, pinned host buffers",
                    "ms_per_step": 1e3 * e2e_s, "counts_match_device": e2e_ok},
            "e2e_reference_blocks": {"value": replica_value(world, n * n, blocks_s), "unit": "genome-pairs/s",
                                     "ms_per_step": 1e3 * blocks_s, "h2d_bytes_per_step": h2d,
                                     "d2h_bytes_per_step": d2h, "counts_match_one_call": blk_ok[0],
                                     "call": "kssdgpu_count_lower per 64-query block, pageable host buffers "
                                             "(as the reference's drivers call the counting function)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_self_scan (one-pass scan join)", "ms_per_launch": ms_scan,
                         "algorithmic_bytes": scan_bytes,
                         "bytes_model": "4 B per context group + 1 (bounds) + 8 B per posting of a group of >= 2 "
                                        "+ 2 x 16 B per touched lower cell",
                         "touched_cells": touched, "shared_groups": facts["groups"],
                         "shared_postings": facts["postings"], "pairs": facts["pairs"]},
            "step_roofline": {"bound": "hbm", "algorithmic_bytes": step_bytes,
                              "achieved": step_bytes / (ms_step / 1e3) / 1e9,
                              "frac": step_bytes / (ms_step / 1e3) / 1e9 / peak,
                              "what": "zero fill of the dense lower triangle (16 B per cell) + scan join",
                              "probe_model_bytes": model_bytes,
                              "probe_model_frac": model_bytes / (ms_step / 1e3) / 1e9 / peak},
            "kernels": {
                "batched_probe": {"ms": ms_probe, "value": world * n * n / (ms_probe / 1e3),
                                  "contexts_probed_per_s": world * int(sk.offs[-1]) / (ms_probe / 1e3),
                                  "probe_model_bytes": model_bytes,
                                  "probe_model_frac": model_bytes / (ms_probe / 1e3) / 1e9 / peak,
                                  "tuning": probe_tuning},
                "plain_per_query": {"ms": ms_plain, "value": world * n * n / (ms_plain / 1e3), "launches": n},
                "cached_plan_join": {"ms": ms_plan_join, "first_call_ms": plan_first_ms,
                                     "what": "KSSDGPU_SELF_PLAN: set-major plan built by the first call and kept"},
                "self_step_vs_plain": ms_plain / ms_step, "batched_probe_vs_plain": ms_plain / ms_probe,
                "self_step_vs_batched_probe": ms_probe / ms_step,
            },
            "index_build_ms": index_ms,
            "density_per_128_tile": density,
            "gpu_launches": int(launches_timed),
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    idx.close()
    return 0


def serve_leg(args, n):
    """A resident index of n genomes (the self-matrix generator, 10 genomes per cluster)
    and the serving sweep against it."""
    import torch
    import kssdgpu
    seed = WORKLOAD["seed"] + 5
    t0 = time.perf_counter()
    ref = kssdgpu.synth(n_samples=n, n_clusters=max(1, n // 10), size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                        len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed,
                        sample_seed=seed, threads=os.cpu_count() or 8)
    gen_s = time.perf_counter() - t0
    entries = int(ref.offs[-1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = kssdgpu.Index.from_sketch(ref)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    del ref
    rates = [float(x) for x in args.serve_rates.split(",")]
    res, pool, srvf = serve_sweep(idx, n, rates, args.serve_seconds, seed)
    idx.close()
    return {"index": {"genomes": n, "entries": entries, "generate_s": gen_s, "device_build_s": build_s},
            "pool": pool, "server": srvf, "rates": res}


def run_serve(args, rank):
    """Serving alone: a resident index of --serve-refs genomes, Poisson arrivals at each rate."""
    if rank != 0:
        return 0
    leg = serve_leg(args, args.serve_refs)
    line = {"metric": "serve p50/p99 ms", "workload": f"serve-{args.serve_refs}-genome-index", "unit": "ms",
            "higher_is_better": False, "data": "synthetic"}
    line.update(leg)
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--genomes", type=int, default=WORKLOAD["n_samples"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--cpu-step-seconds", type=float, default=8.0, help="reference arm: seconds per step")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 20,000-genome legs")
    ap.add_argument("--workload", choices=["self", "serve"], default="self",
                    help="self: the headline self matrix and its legs (default); serve: Poisson arrivals against "
                         "a resident --serve-refs genome index (p50/p99)")
    ap.add_argument("--ns-genomes", type=int, default=20000, help="genomes of the all-vs-all leg and its index")
    ap.add_argument("--rect-queries", type=int, default=10000)
    ap.add_argument("--reads-samples", type=int, default=40)
    ap.add_argument("--parity-queries", type=int, default=48)
    ap.add_argument("--dense-genomes", type=int, default=1024, help="genomes of the one-species dense leg")
    ap.add_argument("--serve-refs", type=int, default=50000,
                    help="resident index size (genomes) of the serving sweep (0: no sweep in the default run)")
    ap.add_argument("--serve-rates", default="1000,5000", help="arrival rates (req/s) of the serving sweep")
    ap.add_argument("--serve-seconds", type=float, default=1.5, help="arrival window per rate")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "serve":
        return run_serve(args, rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())

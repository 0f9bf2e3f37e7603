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
  ours (default)   value: device-resident step (self join over the resident index,
                   counters zeroed and rebuilt each step); e2e: the reference-facing
                   C-ABI call kssdgpu_count_lower with pinned HOST buffers (query keys
                   H2D, dense counters D2H) every step; plus the plain one-query-per-
                   launch kernel and the batched persistent probe kernel beside it.
  reference        the reference's own count_ctx_obj_frm_comb_sketch_section_lower
                   (compiled from its sources into oracle/_ref) over blocks of 64
                   queries with all host threads; rank 0 only.
One JSON line on stdout (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
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


def make_workload(n: int):
    import kssdgpu
    w = dict(WORKLOAD)
    return kssdgpu.synth(n_samples=n, n_clusters=max(1, n // 10), size_dist=kssdgpu.SIZE_LOGNORMAL,
                         len_median=w["len_median"], len_sigma=w["len_sigma"], len_min=w["len_min"],
                         len_max=w["len_max"], sub_lo=w["sub_lo"], sub_hi=w["sub_hi"], seed=w["seed"],
                         sample_seed=w["seed"])


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


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    sk = make_workload(args.genomes)
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
        "config": {"workload": WORKLOAD["name"], "genomes": sk.n, "entries": int(sk.offs[-1]),
                   "path": "count_ctx_obj_frm_comb_sketch_section_lower, 64-query blocks",
                   "blocks_per_step": per_step},
        "cpu_baseline": {"value": value, "unit": "genome-pairs/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} of {nblocks} 64-query blocks per step, rotating"},
        "e2e": {"value": value, "unit": "genome-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import kssdgpu
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()

    sk = make_workload(args.genomes)
    n = sk.n
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    idx = kssdgpu.Index.from_sketch(sk, device=local_rank)
    torch.cuda.synchronize()
    index_ms = 1e3 * (time.perf_counter() - t0)
    info = idx.info()
    t0 = time.perf_counter()
    plan = idx.self_plan_info()  # first call builds the join plan (once per index)
    torch.cuda.synchronize()
    plan["plan_ms"] = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    plan["tuning"] = idx.self_plan_tune()  # the autotuner picks the plan's chunking
    plan["tuning"]["tune_ms"] = 1e3 * (time.perf_counter() - t0)
    plan["index_build_ms"] = index_ms

    d_keys = torch.from_numpy(sk.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(sk.offs.view(np.int64)).to(dev)
    lower_cells = n * (n - 1) // 2
    d_lc = torch.zeros(lower_cells, dtype=torch.int64, device=dev)
    d_lo = torch.zeros(lower_cells, dtype=torch.int64, device=dev)
    d_c = torch.zeros(n * n, dtype=torch.int64, device=dev)
    d_o = torch.zeros(n * n, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def self_step(flags=0):
        idx.self_lower_dev(d_lc, d_lo, flags=flags, stream=stream)

    def probe_step():
        idx.count_block_dev(d_keys, d_offs, n, d_c, d_o, lower=True, stream=stream)

    def plain_step():
        idx.count_plain_dev(d_keys, d_offs, sk.offs, d_c, d_o, lower=True, stream=stream)

    # ---- parity on the benchmark's own inputs: self join == batched probe == plain
    probe_step()
    idx.sync(stream)
    tri = torch.tril_indices(n, n, -1, device=dev)
    dense_c = d_c.view(n, n)[tri[0], tri[1]].clone()
    dense_o = d_o.view(n, n)[tri[0], tri[1]].clone()
    self_step()
    idx.sync(stream)
    ok_join = bool(torch.equal(dense_c, d_lc) and torch.equal(dense_o, d_lo))
    plain_step()
    idx.sync(stream)
    ok_plain = bool(torch.equal(d_c.view(n, n)[tri[0], tri[1]], dense_c) and
                    torch.equal(d_o.view(n, n)[tri[0], tri[1]], dense_o))
    if not (ok_join and ok_plain):
        raise SystemExit(f"parity failure on the bench workload: join={ok_join} plain={ok_plain}")
    del tri
    # lower-triangle cells that share at least one context (every credit adds num_ctx += 1)
    touched = int(torch.count_nonzero(d_lc).item())

    def timed(fn, steps, warmup, flush_l2=True, pre=None):
        for _ in range(warmup):
            if pre:
                pre()
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(steps):
            if flush_l2:
                flush.fill_(1)
            if pre:
                pre()
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            tot += s.elapsed_time(e)
        idx.sync(stream)
        return tot / steps  # ms

    # ---- headline: timed region bracketed by barrier + synchronize, max over ranks
    launches0 = kssdgpu.launch_count()
    self_step()
    torch.cuda.synchronize()
    launches_per_step = kssdgpu.launch_count() - launches0
    with ClockSampler(local_rank) as clocks:
        # the steps take milliseconds: keep the GPU on this workload until the sampler
        # has readings, then run the timed region inside the same sampling window
        t_end = time.time() + 1.5
        while time.time() < t_end or len(clocks.samples) < 3:
            for _ in range(50):
                self_step()
            torch.cuda.synchronize()
            if time.time() > t_end + 10:
                break
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms_step = timed(self_step, args.steps, args.warmup)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms_step = max_over_ranks(dist, ms_step, dev)
    launches_timed = launches_per_step * args.steps
    value = replica_value(world, n * n, ms_step / 1e3)

    # ---- dominant kernel alone (join kernels, counters zeroed outside the events)
    zero = lambda: (d_lc.zero_(), d_lo.zero_())  # noqa: E731
    ms_join = timed(lambda: self_step(kssdgpu.NO_ZERO), args.steps, 2, pre=zero)
    peak, peak_kind = measured_peak_hbm()
    # algorithmic bytes of one join launch: each listed group's (begin,k) word and its
    # postings read once, each touched lower-triangle cell (16 B of counters) read and
    # written once; the step adds the 16 B/cell zero fill of the dense lower triangle
    join_bytes = 8 * plan["groups"] + 8 * plan["postings"] + 2 * 16 * touched
    step_bytes = join_bytes + 16 * lower_cells
    achieved = join_bytes / (ms_join / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "k_self_sets_traffic.json")
    if os.path.exists(tfile):
        try:
            t = json.load(open(tfile))
            if t.get("workload_genomes") == n:  # the ncu capture of this workload's join launch
                traffic = t.get("bytes_per_launch")
        except Exception:
            traffic = None

    # ---- plain one-query-per-launch and batched probe kernels (same counters)
    probe_tuning = idx.count_tune(d_keys, d_offs, n, d_c, d_o, lower=True)  # accumulator mode / chunk size
    ms_probe = timed(probe_step, max(3, args.steps // 2), 2)
    ms_plain = timed(plain_step, 3, 1)
    # per-query probe model bytes: 8|q| + 12 * postings walked + 16 per output cell
    probe_model_bytes = None

    # ---- e2e through the host-buffer C ABI (pinned host inputs and outputs)
    h_keys = torch.from_numpy(sk.keys.view(np.int64)).pin_memory()
    h_offs_t = torch.from_numpy(sk.offs.view(np.int64)).pin_memory()
    h_ctx = torch.empty(n * n * 2, dtype=torch.int32).pin_memory()
    h_obj = torch.empty(n * n * 2, dtype=torch.int32).pin_memory()
    lib = kssdgpu.gpu_lib()
    h_offs_np = h_offs_t.numpy().view(np.uint64)

    def e2e_call():
        rc = lib.kssdgpu_count_lower(idx.handle, h_keys.data_ptr(), h_offs_np, n, 0, 0, h_ctx.data_ptr(),
                                     h_obj.data_ptr())
        if rc:
            raise kssdgpu.KssdGpuError(rc, lib.kssdgpu_last_error().decode())

    for _ in range(2):
        e2e_call()
    e2e_times = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_call()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e_times))
    e2e_s = max_over_ranks(dist, e2e_s, dev)
    e2e_value = replica_value(world, n * n, e2e_s)
    h2d = int(sk.keys.nbytes + sk.offs.nbytes + 4 * n)
    d2h = int(n * n * 16)
    # the e2e counters equal the device-resident ones
    e2e_ok = bool(np.array_equal(h_ctx.numpy().view(np.int64), d_c.cpu().numpy()))

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

    if rank == 0:
        line = {
            "metric": "ANI genome-pairs/s", "value": value, "unit": "genome-pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "genomes": n, "entries": int(sk.offs[-1]),
                       "unique_contexts": info["contexts"], "matrix_cells": n * n,
                       "lower_pairs": lower_cells, "path": "self join (kssdgpu_self_lower_dev)",
                       "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "genome-pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "call": "kssdgpu_count_lower (host buffers, pinned)",
                    "ms_per_step": 1e3 * e2e_s, "counts_match_device": e2e_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_self_sets (set-major self join)", "ms_per_launch": ms_join,
                         "algorithmic_bytes": join_bytes, "touched_cells": touched},
            "step_roofline": {"bound": "hbm", "algorithmic_bytes": step_bytes,
                              "achieved": step_bytes / (ms_step / 1e3) / 1e9,
                              "frac": step_bytes / (ms_step / 1e3) / 1e9 / peak,
                              "what": "zero fill of the dense lower triangle + self join"},
            "kernels": {
                "batched_probe": {"ms": ms_probe, "value": world * n * n / (ms_probe / 1e3),
                                  "contexts_probed_per_s": world * int(sk.offs[-1]) / (ms_probe / 1e3),
                                  "tuning": probe_tuning},
                "plain_per_query": {"ms": ms_plain, "value": world * n * n / (ms_plain / 1e3), "launches": n},
                "self_join_vs_plain": ms_plain / ms_step, "batched_probe_vs_plain": ms_plain / ms_probe,
            },
            "join_plan": plan,
            "gpu_launches": int(launches_timed),
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    idx.close()
    return 0


def _pct(xs, p):
    xs = sorted(xs)
    return float(xs[min(len(xs) - 1, int(p * (len(xs) - 1) + 0.5))]) if xs else None


def run_serve(args, rank):
    """Serving: a resident index of --serve-refs genomes (the self-matrix generator,
    10 genomes per cluster), Poisson arrivals at each rate for --serve-seconds, 80%
    assemblies (0.5-12 Mbp, from the same cluster ancestors) and 20% read sets (1-5
    genomes at 5-100x, 0.1-1% errors, conflicts kept); latency = submit -> hits on the
    host, measured by the server."""
    import random
    import torch
    import kssdgpu
    if rank != 0:
        return 0
    n = args.serve_refs
    seed = 20261203 + 5
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
    asm = kssdgpu.synth(n_samples=256, n_clusters=max(1, n // 10), role=kssdgpu.ROLE_OWNLEN,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6,
                        own_len_min=5e5, own_len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed, sample_seed=seed + 1)
    reads = kssdgpu.synth(n_samples=64, n_clusters=max(1, n // 10), role=kssdgpu.ROLE_READS,
                          size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6, len_sigma=0.37, len_min=1e6,
                          len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed, sample_seed=seed + 2,
                          ref_sample_seed=seed, ref_samples=n, cov_lo=5, cov_hi=100, err_lo=0.001, err_hi=0.01)
    pool = [("assembly", asm.keys[asm.offs[i]:asm.offs[i + 1]]) for i in range(asm.n)]
    pool_reads = [("reads", reads.keys[reads.offs[i]:reads.offs[i + 1]]) for i in range(reads.n)]
    max_keys = max(len(k) for _, k in pool + pool_reads)
    srv = kssdgpu.Server(idx, max_batch_queries=64, max_batch_keys=max(1 << 24, 2 * max_keys), max_hits=1 << 22)
    for _, k in pool[:32] + pool_reads[:8]:  # warm-up
        srv.result(srv.submit(k))
    rng = random.Random(seed)
    results = []
    sys.setswitchinterval(2e-4)  # the pacing loop must not hold the interpreter lock for 5 ms
    for rate in [float(x) for x in args.serve_rates.split(",")]:
        srv.reset_stats()
        nreq = max(1, int(rate * args.serve_seconds))
        t = 0.0
        plan = []
        for _ in range(nreq):
            t += rng.expovariate(rate)
            plan.append((t, pool[rng.randrange(len(pool))] if rng.random() < 0.8 else
                         pool_reads[rng.randrange(len(pool_reads))]))
        got = []
        tickets = []
        cond = threading.Condition()

        def collector():
            i = 0
            while True:
                with cond:
                    while i >= len(tickets):
                        cond.wait(timeout=1.0)
                        if i >= len(tickets) and done_submitting[0]:
                            return
                    kind, tk = tickets[i]
                hits, lat = srv.result(tk, timeout_ms=120000)
                got.append((kind, lat, len(hits)))
                i += 1
                if i == nreq:
                    return

        done_submitting = [False]
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
            "genome_pairs_s": nreq * n / wall, "p50_ms": _pct(lat, 0.5), "p99_ms": _pct(lat, 0.99),
            "assembly_p50_ms": _pct(lat_a, 0.5), "assembly_p99_ms": _pct(lat_a, 0.99),
            "reads_p50_ms": _pct(lat_r, 0.5), "reads_p99_ms": _pct(lat_r, 0.99), "max_ms": max(lat) if lat else None,
            "batches": st["batches"], "max_inflight": st["max_inflight"],
            "overlapped_batches": st["overlapped_batches"], "mean_hits": float(np.mean([x[2] for x in got]))})
        print(json.dumps({"partial": results[-1]}), file=sys.stderr, flush=True)
    line = {"metric": "serve p50/p99 ms", "workload": f"serve-{n}-genome-index", "unit": "ms",
            "higher_is_better": False, "data": "synthetic", "index": {"genomes": n, "entries": entries,
            "generate_s": gen_s, "device_build_s": build_s}, "pool": {"assemblies": len(pool),
            "read_sets": len(pool_reads), "max_keys": max_keys,
            "mean_assembly_keys": float(np.mean([len(k) for _, k in pool])),
            "mean_reads_keys": float(np.mean([len(k) for _, k in pool_reads]))},
            "server": {"reserved_bytes": srv.stats()["reserved_bytes"], "max_batch_queries": 64},
            "rates": results}
    print(json.dumps(line), flush=True)
    srv.close()
    idx.close()
    return 0


def run_rect(args, rank):
    """Uneven batch: --rect-queries genomes of log-uniform 50 kbp-12 Mbp against a
    --rect-refs genome index (2,000 clusters at the default sizes): one persistent
    batched launch (also replayed from a CUDA graph) vs the plain per-query kernel,
    with the reference's own counting function timed on a query sample."""
    import torch
    import kssdgpu
    if rank != 0:
        return 0
    nr, nq = args.rect_refs, args.rect_queries
    seed = 20261203 + 3
    clusters = max(1, nr // 10)
    ref = kssdgpu.synth(n_samples=nr, n_clusters=clusters, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                        len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed,
                        sample_seed=seed, threads=os.cpu_count() or 8)
    qry = kssdgpu.synth(n_samples=nq, n_clusters=clusters, role=kssdgpu.ROLE_OWNLEN, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6, own_len_min=5e4,
                        own_len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed, sample_seed=seed + 1,
                        threads=os.cpu_count() or 8)
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    cells = nq * nr
    dc = torch.zeros(cells, dtype=torch.int64, device=dev)
    dob = torch.zeros(cells, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def batched():
        idx.count_block_dev(dk, do, nq, dc, dob, stream=stream)

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(steps):
            flush.fill_(1)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            tot += s.elapsed_time(e)
        idx.sync(stream)
        return tot / steps

    tuning = idx.count_tune(dk, do, nq, dc, dob)
    ms_b = timed(batched, args.steps, args.warmup)
    checksum = int(dc.sum().item())
    shared = int((dc & 0xFFFFFFFF).sum().item())  # = postings walked (conflict-free references)
    # the same launch sequence captured once into a CUDA graph and replayed
    graph_ms = None
    try:
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                idx.count_block_dev(dk, do, nq, dc, dob, stream=side)
        stream.wait_stream(side)
        graph_ms = timed(lambda: g.replay(), args.steps, 2)
        assert int(dc.sum().item()) == checksum
    except Exception as exc:  # capture support depends on the driver; report instead of failing
        graph_ms = f"capture failed: {exc}"
    ms_p = timed(lambda: idx.count_plain_dev(dk, do, qry.offs, dc, dob, stream=stream), 1, 1)
    assert int(dc.sum().item()) == checksum
    qkeys = int(qry.offs[-1])
    probe_bytes = 8 * qkeys + 12 * shared + 16 * cells
    peak, kind = measured_peak_hbm()
    # the reference's counting function on a sample of queries (host cores)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    rec, _ = idx.export()
    sample = list(range(0, nq, max(1, nq // 48)))[:48]
    skeys = np.concatenate([qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])] for q in sample])
    soffs = np.concatenate([[0], np.cumsum([int(qry.offs[q + 1] - qry.offs[q]) for q in sample])]).astype(np.uint64)
    t0 = time.perf_counter()
    c, _ = oracle.count_block(rec, nr, skeys, soffs, threads=os.cpu_count() or 1, ref=oracle.ref_available())
    cpu_s = time.perf_counter() - t0
    hc = dc.view(nq, nr)[torch.tensor(sample, device=dev)].cpu().numpy()
    same = bool(np.array_equal(c[:, :, 0].astype(np.int64) | (c[:, :, 1].astype(np.int64) << 32), hc))
    line = {"metric": "ANI genome-pairs/s", "workload": f"rect-{nq}x{nr}", "unit": "genome-pairs/s",
            "value": cells / (ms_b / 1e3), "ms_per_step": ms_b, "steps": args.steps, "data": "synthetic",
            "config": {"queries": nq, "refs": nr, "query_keys": qkeys, "ref_entries": int(ref.offs[-1]),
                       "accumulators": "global (reference row exceeds shared memory)" if nr * 16 > 112 * 1024
                       else "shared"},
            "graph_replay_ms": graph_ms, "contexts_probed_per_s": qkeys / (ms_b / 1e3), "tuning": tuning,
            "plain_per_query": {"ms": ms_p, "value": cells / (ms_p / 1e3), "launches": nq},
            "batched_vs_plain": ms_p / ms_b,
            "roofline_probe_model": {"bound": "hbm", "bytes": probe_bytes,
                                     "achieved": probe_bytes / (ms_b / 1e3) / 1e9, "peak": peak,
                                     "frac": probe_bytes / (ms_b / 1e3) / 1e9 / peak, "peak_kind": kind},
            "cpu_baseline": {"value": len(sample) * nr / cpu_s, "unit": "genome-pairs/s",
                             "cores": os.cpu_count(), "kind": "reference" if oracle.ref_available() else "port",
                             "sample": f"{len(sample)} queries", "counts_match_gpu": same}}
    print(json.dumps(line), flush=True)
    idx.close()
    return 0


def run_reads(args, rank):
    """Read sets: --reads-samples samples, each a mix of 1-5 genomes of a --rect-refs
    genome reference at 5-50x with 0.1-1% substitution errors (conflicts kept, as
    `sketch --asone --conflict -A`), counted against the reference index with unique
    contexts (`ani --qraw ... --unique-ctx`): one batched launch, key-range chunks
    built on the device, vs the plain per-query kernel; the reference's own counting
    function timed on a sample."""
    import torch
    import kssdgpu
    if rank != 0:
        return 0
    nr, nq = args.rect_refs, args.reads_samples
    seed = 20261203 + 4
    clusters = max(1, nr // 10)
    ref = kssdgpu.synth(n_samples=nr, n_clusters=clusters, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                        len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=seed,
                        sample_seed=seed, threads=os.cpu_count() or 8)
    qry = kssdgpu.synth(n_samples=nq, n_clusters=clusters, role=kssdgpu.ROLE_READS, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        len_median=4e6, len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2,
                        seed=seed, sample_seed=seed + 1, ref_sample_seed=seed, ref_samples=nr, cov_lo=5, cov_hi=50,
                        err_lo=0.001, err_hi=0.01, threads=os.cpu_count() or 8)
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    cells = nq * nr
    outs = [torch.zeros(cells, dtype=torch.int64, device=dev) for _ in range(4)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    flags = kssdgpu.UNIQUE

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(steps):
            flush.fill_(1)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            e.synchronize()
            tot += s.elapsed_time(e)
        idx.sync(stream)
        return tot / steps

    tuning = idx.count_tune(dk, do, nq, *outs, flags=flags)
    ms_b = timed(lambda: idx.count_block_dev(dk, do, nq, *outs, flags=flags, stream=stream), args.steps,
                 args.warmup)
    sums = [int(o.sum().item()) for o in outs]
    ms_p = timed(lambda: idx.count_plain_dev(dk, do, qry.offs, *outs, flags=flags, stream=stream), 1, 1)
    assert [int(o.sum().item()) for o in outs] == sums
    qkeys = int(qry.offs[-1])
    # the reference's counting function (with unique contexts) on a sample of read sets
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    rec, _ = idx.export()
    sample = list(range(0, nq, max(1, nq // 8)))[:8]
    skeys = np.concatenate([qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])] for q in sample])
    soffs = np.concatenate([[0], np.cumsum([int(qry.offs[q + 1] - qry.offs[q]) for q in sample])]).astype(np.uint64)
    t0 = time.perf_counter()
    want = oracle.count_block(rec, nr, skeys, soffs, unique=True, threads=os.cpu_count() or 1,
                              ref=oracle.ref_available())
    cpu_s = time.perf_counter() - t0
    rows = torch.tensor(sample, device=dev)
    same = all(bool(np.array_equal(w[:, :, 0].astype(np.int64) | (w[:, :, 1].astype(np.int64) << 32),
                                   o.view(nq, nr)[rows].cpu().numpy())) for w, o in zip(want, outs))
    line = {"metric": "ANI genome-pairs/s", "workload": f"reads-{nq}x{nr}-unique-ctx", "unit": "genome-pairs/s",
            "value": cells / (ms_b / 1e3), "ms_per_step": ms_b, "steps": args.steps, "data": "synthetic",
            "contexts_probed_per_s": qkeys / (ms_b / 1e3), "tuning": tuning,
            "config": {"read_sets": nq, "refs": nr, "query_keys": qkeys, "ref_entries": int(ref.offs[-1]),
                       "mean_keys_per_read_set": qkeys / nq, "flags": "unique contexts, conflicts kept"},
            "plain_per_query": {"ms": ms_p, "value": cells / (ms_p / 1e3), "launches": nq},
            "batched_vs_plain": ms_p / ms_b,
            "cpu_baseline": {"value": len(sample) * nr / cpu_s, "unit": "genome-pairs/s",
                             "cores": os.cpu_count(), "kind": "reference" if oracle.ref_available() else "port",
                             "sample": f"{len(sample)} read sets", "counts_match_gpu": same}}
    print(json.dumps(line), flush=True)
    idx.close()
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
    ap.add_argument("--workload", choices=["self", "serve", "rect", "reads"], default="self",
                    help="self: the headline self matrix (default); serve: Poisson arrivals against a resident "
                         "index (p50/p99); rect: uneven queries against a larger index, one batched launch; "
                         "reads: read sets with unique-context counting against the larger index")
    ap.add_argument("--reads-samples", type=int, default=40)
    ap.add_argument("--serve-refs", type=int, default=50000, help="serve: resident index size (genomes)")
    ap.add_argument("--serve-rates", default="100,300,1000,3000,5000,10000,20000", help="serve: arrival rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serve: arrival window per rate")
    ap.add_argument("--rect-refs", type=int, default=20000)
    ap.add_argument("--rect-queries", type=int, default=10000)
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
    if args.workload == "rect":
        return run_rect(args, rank)
    if args.workload == "reads":
        return run_reads(args, rank)
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

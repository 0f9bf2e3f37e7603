"""The continuous-batching server (kssdgpu_server_*): every request's hits equal the
nonzero counter cells kssdgpu_count_block gives for that query alone, whether the
request ran alone or shared batches with concurrent arrivals."""
import random
import threading
import time

import numpy as np
import pytest

import kssdgpu

pytestmark = pytest.mark.gpu


def _workload():
    ref = kssdgpu.synth(n_samples=300, n_clusters=15, len_median=3e5, len_min=1e5, len_max=1e6,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.08, seed=41, sample_seed=41)
    asm = kssdgpu.synth(n_samples=40, n_clusters=15, role=kssdgpu.ROLE_OWNLEN, len_median=3e5, len_min=1e5,
                        len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=1.2e6,
                        seed=41, sample_seed=42)
    reads = kssdgpu.synth(n_samples=8, n_clusters=15, role=kssdgpu.ROLE_READS, len_median=3e5, len_min=1e5,
                          len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL, seed=41, sample_seed=43,
                          ref_sample_seed=41, ref_samples=300, cov_lo=5, cov_hi=30)
    queries = [asm.keys[asm.offs[i]:asm.offs[i + 1]] for i in range(asm.n)]
    queries += [reads.keys[reads.offs[i]:reads.offs[i + 1]] for i in range(reads.n)]
    queries.append(np.zeros(0, dtype=np.uint64))  # an empty sample
    return ref, queries


def _expected(idx, q, flags):
    offs = np.array([0, len(q)], dtype=np.uint64)
    out = idx.count_block(q, offs, flags)
    ctx, obj = out[0][0], out[1][0]
    nz = np.nonzero(ctx[:, 0])[0]
    if flags & kssdgpu.UNIQUE:
        uctx, uobj = out[2][0], out[3][0]
        nz = np.union1d(nz, np.nonzero(uctx[:, 0])[0])
    rows = []
    for r in nz:
        row = [int(r), ctx[r, 0], ctx[r, 1], obj[r, 0], obj[r, 1]]
        if flags & kssdgpu.UNIQUE:
            row += [uctx[r, 0], uctx[r, 1], uobj[r, 0], uobj[r, 1]]
        rows.append(tuple(int(x) for x in row))
    return rows


def _as_rows(hits, flags):
    cols = ["ref", "num_ctx", "num_mut2_ctx", "diff_obj", "diff_obj_section"]
    if flags & kssdgpu.UNIQUE:
        cols += ["u_num_ctx", "u_num_mut2_ctx", "u_diff_obj", "u_diff_obj_section"]
    return [tuple(int(h[c]) for c in cols) for h in hits]


@pytest.mark.parametrize("flags", [0, kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT])
def test_results_identical_alone_and_in_the_mix(flags):
    ref, queries = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    want = [_expected(idx, q, flags) for q in queries]
    assert sum(len(w) for w in want) > 0
    srv = kssdgpu.Server(idx, max_batch_queries=16, max_batch_keys=1 << 22, flags=flags)
    try:
        # alone: one request on the GPU at a time
        for q, w in zip(queries, want):
            hits, lat = srv.result(srv.submit(q))
            assert _as_rows(hits, flags) == w
            assert lat >= 0
        # in the mix: four clients submit with random gaps, several rounds
        got = {}
        lock = threading.Lock()

        def client(seed):
            rng = random.Random(seed)
            order = list(range(len(queries))) * 3
            rng.shuffle(order)
            tickets = []
            for i in order:
                tickets.append((i, srv.submit(queries[i])))
                if rng.random() < 0.3:
                    time.sleep(rng.random() * 0.002)
            for i, t in tickets:
                hits, _ = srv.result(t, timeout_ms=60000)
                with lock:
                    got.setdefault(i, []).append(_as_rows(hits, flags))

        threads = [threading.Thread(target=client, args=(s,)) for s in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for i, w in enumerate(want):
            assert len(got[i]) == 12
            assert all(g == w for g in got[i]), i
        st = srv.stats()
        assert st["completed"] == len(queries) * 13
        assert st["batches"] < st["completed"]          # requests shared batches
        assert st["max_inflight"] > 1
        assert st["p99_ms"] >= st["p50_ms"] >= 0
    finally:
        srv.close()
        idx.close()


def test_oversized_query_is_rejected():
    ref, queries = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    srv = kssdgpu.Server(idx, max_batch_queries=4, max_batch_keys=1000)
    try:
        big = max(queries, key=len)
        assert len(big) > 1000
        with pytest.raises(kssdgpu.KssdGpuError) as e:
            srv.submit(big)
        assert e.value.code == 7
        small = min((q for q in queries if len(q)), key=len)
        if len(small) <= 1000:
            hits, _ = srv.result(srv.submit(small))
            assert _as_rows(hits, 0) == _expected(idx, small, 0)
    finally:
        srv.close()
        idx.close()

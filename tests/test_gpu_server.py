"""The continuous-batching server (kssdgpu_server_*): every request's hits equal the
nonzero counter cells the oracle gives for that query alone, whether the request ran
alone or shared batches with concurrent arrivals; batches that overflow the hit
capacity are split and re-run; admission follows the device-memory budget."""
import random
import threading
import time

import numpy as np
import pytest

import kssdgpu
import oracle

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


def _expected(rec, nref, q, flags):
    """Nonzero cells of the oracle's counters for query q alone."""
    offs = np.array([0, len(q)], dtype=np.uint64)
    out = oracle.count_block(rec, nref, q, offs, ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT),
                             unique=bool(flags & kssdgpu.UNIQUE))
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


@pytest.mark.parametrize("flags,stripe_bytes", [(0, 0), (kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT, 0), (0, 256)])
def test_results_identical_alone_and_in_the_mix(flags, stripe_bytes):
    ref, queries = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    if stripe_bytes:  # a filter of many key-range stripes: each context's stripe found per key
        assert idx.filter(stripe_bytes)["stripes"] > 1
    rec = oracle.build_index(ref.keys, ref.offs)
    want = [_expected(rec, ref.n, q, flags) for q in queries]
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
            assert _as_rows(hits, 0) == _expected(oracle.build_index(ref.keys, ref.offs), ref.n, small, 0)
        bad = np.array(big[:50][::-1])  # descending keys
        with pytest.raises(kssdgpu.KssdGpuError) as e:
            srv.submit(bad)
        assert e.value.code == 3
    finally:
        srv.close()
        idx.close()


def test_hit_overflow_splits_the_batch():
    """A batch whose nonzero cells exceed max_hits re-runs its requests one per batch:
    each request that fits alone gets its full result; one that overflows alone fails
    with KSSDGPU_ERR_CAPACITY, and the server keeps serving."""
    ref, queries = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    rec = oracle.build_index(ref.keys, ref.offs)
    want = [_expected(rec, ref.n, q, 0) for q in queries]
    cap = max(len(w) for w in want if len(w) < 60) if any(len(w) < 60 for w in want) else 0
    assert cap > 0
    srv = kssdgpu.Server(idx, max_batch_queries=8, max_batch_keys=1 << 22, max_hits=cap, slots=1)
    try:
        tickets = [srv.submit(q) for q in queries]  # queued together: batches of up to 8
        for q, w, t in zip(queries, want, tickets):
            if len(w) <= cap:
                hits, _ = srv.result(t, timeout_ms=60000)
                assert _as_rows(hits, 0) == w
            else:
                with pytest.raises(kssdgpu.KssdGpuError) as e:
                    srv.result(t, timeout_ms=60000)
                assert e.value.code == 7
        st = srv.stats()
        assert st["splits"] > 0 and st["slots"] == 1
        small = [i for i, w in enumerate(want) if 0 < len(w) <= cap][0]
        hits, _ = srv.result(srv.submit(queries[small]))
        assert _as_rows(hits, 0) == want[small]
    finally:
        srv.close()
        idx.close()


def test_admission_by_device_budget():
    """The slot count follows the device-memory budget; a budget below one slot is refused."""
    ref, queries = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    try:
        one = kssdgpu.Server(idx, max_batch_queries=4, max_batch_keys=1 << 20, slots=8)
        per_slot = one.stats()["reserved_bytes"] // one.stats()["slots"]
        assert one.stats()["slots"] == 8
        one.close()
        srv = kssdgpu.Server(idx, max_batch_queries=4, max_batch_keys=1 << 20, slots=8, device_budget=3 * per_slot)
        assert srv.stats()["slots"] == 3
        rec = oracle.build_index(ref.keys, ref.offs)
        ts = [srv.submit(q) for q in queries]
        for q, t in zip(queries, ts):
            hits, _ = srv.result(t, timeout_ms=60000)
            assert _as_rows(hits, 0) == _expected(rec, ref.n, q, 0)
        srv.close()
        with pytest.raises(kssdgpu.KssdGpuError) as e:
            kssdgpu.Server(idx, max_batch_queries=4, max_batch_keys=1 << 20, device_budget=per_slot - 1)
        assert e.value.code == 7
    finally:
        idx.close()

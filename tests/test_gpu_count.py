"""CUDA counting path (through the C ABI) against the oracle, bit for bit."""
import json
import os

import numpy as np
import pytest

import kssdgpu
import oracle
from fixtures import mutate_from, random_samples, samples_to_sketch

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _fixture(seed, nref, nq, ctx_space, obj_space, conflict, max_len=40):
    rng = np.random.default_rng(seed)
    refs = random_samples(rng, nref, max_len, ctx_space, obj_space, conflict)
    qrys = random_samples(rng, nq, max_len, ctx_space, obj_space, conflict)
    for i in range(min(nq, nref)):
        if refs[i] and rng.random() < 0.5:
            qrys[i] = mutate_from(rng, refs[i], 0.05)
    rk, ro = samples_to_sketch(refs)
    qk, qo = samples_to_sketch(qrys)
    return rk, ro, qk, qo


CASES = [(s, 4, 2, 35, 256, True) for s in range(10)] + \
        [(s, 40, 12, 300, 1 << 20, True) for s in range(10, 14)] + \
        [(s, 300, 50, 5000, 1 << 20, False) for s in range(14, 16)]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("flags", [0, kssdgpu.IGNORECONFLICT, kssdgpu.PLAIN, kssdgpu.GLOBAL_ACC,
                                   kssdgpu.PLAIN | kssdgpu.IGNORECONFLICT, kssdgpu.SMEM_ACC,
                                   kssdgpu.SMEM_ACC | kssdgpu.IGNORECONFLICT])
def test_count_block_unique(case, flags):
    rk, ro, qk, qo = _fixture(*case)
    nref = len(ro) - 1
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, nref)
    ign = bool(flags & kssdgpu.IGNORECONFLICT)
    got = idx.count_block(qk, qo, flags | kssdgpu.UNIQUE)
    want = oracle.count_block(rec, nref, qk, qo, ignoreconflict=ign, unique=True)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    got2 = idx.count_block(qk, qo, flags)
    np.testing.assert_array_equal(got2[0], want[0])
    np.testing.assert_array_equal(got2[1], want[1])


@pytest.mark.parametrize("case", CASES[::2])
@pytest.mark.parametrize("flags", [0, kssdgpu.IGNORECONFLICT, kssdgpu.PLAIN, kssdgpu.GLOBAL_ACC, kssdgpu.SMEM_ACC])
def test_count_lower_blocks(case, flags):
    rk, ro, _, _ = _fixture(*case)
    nref = len(ro) - 1
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, nref)
    ign = bool(flags & kssdgpu.IGNORECONFLICT)
    for off in range(0, nref, 64):
        nb = min(64, nref - off)
        qo = ro[off: off + nb + 1]
        qk = rk[int(qo[0]): int(qo[-1])]
        got = idx.count_lower(qk, qo, off, flags)
        want = oracle.count_lower(rec, nref, off, qk, qo, ignoreconflict=ign)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


SELF_PATHS = [0, kssdgpu.SELF_SCAN, kssdgpu.SELF_PLAN]  # by density (default), one-pass scan, cached plan


@pytest.mark.parametrize("case", CASES[::3])
@pytest.mark.parametrize("ign", [False, True])
@pytest.mark.parametrize("path", SELF_PATHS)
def test_self_lower_join(case, ign, path):
    rk, ro, _, _ = _fixture(*case)
    rec = oracle.build_index(rk, ro)
    nref = len(ro) - 1
    idx = kssdgpu.Index.from_records(rec, nref)
    got = idx.self_lower((kssdgpu.IGNORECONFLICT if ign else 0) | path)
    want = oracle.self_lower_all(rec, rk, ro, ignoreconflict=ign)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("conflict", [False, True])
@pytest.mark.parametrize("ign", [False, True])
def test_self_scan_large_groups(seed, conflict, ign):
    """Context groups of more than 32 postings (the scan join's whole-CTA path), with and
    without multi-object gid runs, mixed with small groups and empty samples."""
    rng = np.random.default_rng(100 + seed)
    refs = random_samples(rng, 70, 60, 12, 64 if conflict else 1 << 20, conflict)
    refs += random_samples(rng, 30, 40, 5000, 1 << 20, conflict)
    rk, ro = samples_to_sketch(refs)
    rec = oracle.build_index(rk, ro)
    nref = len(ro) - 1
    idx = kssdgpu.Index.from_records(rec, nref)
    assert idx.self_plan_info()["postings"] > 0
    want = oracle.self_lower_all(rec, rk, ro, ignoreconflict=ign)
    for path in SELF_PATHS:
        got = idx.self_lower((kssdgpu.IGNORECONFLICT if ign else 0) | path)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


def test_self_plan_info_counts_groups():
    rk, ro, _, _ = _fixture(*CASES[12])
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, len(ro) - 1)
    ctx = (np.frombuffer(rec.tobytes(), dtype=np.dtype([("cg", "<u8"), ("obj", "<u4")]))["cg"] >> np.uint64(20))
    _, k = np.unique(ctx, return_counts=True)
    k = k[k >= 2].astype(np.int64)
    assert idx.self_plan_info() == dict(groups=len(k), postings=int(k.sum()), pairs=int((k * (k - 1) // 2).sum()))


@pytest.mark.parametrize("case", CASES[::4])
def test_index_from_sketch_and_export(case):
    rk, ro, _, _ = _fixture(*case)
    nref = len(ro) - 1
    rec = oracle.build_index(rk, ro)
    sk = kssdgpu.Sketch(keys=rk, offs=ro, names=[str(i) for i in range(nref)], conflict=True)
    idx = kssdgpu.Index.from_sketch(sk)
    got_rec, got_bits = idx.export()
    assert got_rec.tobytes() == rec.tobytes()
    np.testing.assert_array_equal(got_bits, oracle.unique_bits(rec))
    for ign in (False, True):
        c, u = idx.ref_ctx_counts(conflict=True, ignoreconflict=ign)
        np.testing.assert_array_equal(c, oracle.ref_ctx_counts(rec, nref, ro, True, ign))
        np.testing.assert_array_equal(u, oracle.unique_ref_totals(rec, nref, ign))
    c, _ = idx.ref_ctx_counts(conflict=False, ignoreconflict=False)
    np.testing.assert_array_equal(c, np.diff(ro).astype(np.uint32))


def test_synthetic_genomes_block_and_self():
    """Seeded assembly-like genomes (sketch-space generator): block, lower and self join agree."""
    sk = kssdgpu.synth(n_samples=96, n_clusters=8, len_median=3e5, len_min=1e5, len_max=1e6,
                       size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    q = kssdgpu.synth(n_samples=20, n_clusters=8, role=kssdgpu.ROLE_OWNLEN, sample_seed=99,
                      len_median=3e5, len_min=1e5, len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL,
                      own_len_min=5e4, own_len_max=1e6)
    got = idx.count_block(q.keys, q.offs, kssdgpu.UNIQUE)
    want = oracle.count_block(rec, sk.n, q.keys, q.offs, unique=True)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    assert want[0][:, :, 0].sum() > 0
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    for path in SELF_PATHS:
        got = idx.self_lower(path)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


def _clustered_sketch(kind="pairs"):
    if kind == "pairs":
        # tight clusters: many contexts shared by exactly 2..4 genomes, in runs of the
        # same gid list that cross warp (32-group) boundaries and end in partial warps
        return kssdgpu.synth(n_samples=120, n_clusters=30, len_median=3e5, len_min=1e5, len_max=1e6,
                             size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.05)
    # three wide clusters: contexts shared by 5..23 genomes (tiles of one chunk whose
    # 36..253 items span several warps)
    return kssdgpu.synth(n_samples=90, n_clusters=3, len_median=2e5, len_min=1e5, len_max=6e5,
                         size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.08)


@pytest.mark.parametrize("kind", ["pairs", "wide"])
@pytest.mark.parametrize("flat,chunk,srt", [(1, 32, 1), (2, 32, 1), (3, 32, 1), (4, 32, 1), (4, 1, 1), (4, 7, 0),
                                            (2, 255, 1), (3, 16, 0)])
def test_self_join_plan_settings(monkeypatch, flat, chunk, srt, kind):
    """Every plan setting (largest flat group size, groups per chunk, chunk order)
    gives the oracle's self-join counters."""
    monkeypatch.setenv("KSSDGPU_JOIN_FLAT", str(flat))
    monkeypatch.setenv("KSSDGPU_JOIN_CHUNK", str(chunk))
    monkeypatch.setenv("KSSDGPU_JOIN_SORT", str(srt))
    sk = _clustered_sketch(kind)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    got = idx.self_lower(kssdgpu.SELF_PLAN)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    t = idx.self_plan_tune()  # pinned by the environment: defaults kept, nothing timed
    assert (t["flat_groups"], t["chunk_groups"], t["sorted"], t["candidates"]) == (flat, chunk, bool(srt), 0)


@pytest.mark.parametrize("kind", ["pairs", "wide"])
@pytest.mark.parametrize("compact", [0, 2])
def test_self_join_compact_counters(monkeypatch, kind, compact):
    """Plans of items only add into compact slots of the touched cells while the dense
    fill runs on a second stream, then scatter (by default only where the dense
    counters outgrow L2; KSSDGPU_JOIN_COMPACT=2 forces it here); with
    KSSDGPU_JOIN_COMPACT=0 they add into the dense cells.  Both give the oracle's
    counters, overwrite stale device counters, and accumulate with KSSDGPU_NO_ZERO."""
    import torch
    monkeypatch.setenv("KSSDGPU_JOIN_FLAT", "1")
    monkeypatch.setenv("KSSDGPU_JOIN_COMPACT", str(compact))
    sk = _clustered_sketch(kind)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    cells = sk.n * (sk.n - 1) // 2
    d_c = torch.full((cells,), 0x3C3C3C3C3C3C3C3C, dtype=torch.int64, device="cuda")
    d_o = torch.full((cells,), -7, dtype=torch.int64, device="cuda")
    for _ in range(2):
        idx.self_lower_dev(d_c, d_o, flags=kssdgpu.SELF_PLAN)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_c.cpu().numpy().view(np.uint32).reshape(-1, 2), want[0])
        np.testing.assert_array_equal(d_o.cpu().numpy().view(np.uint32).reshape(-1, 2), want[1])
    idx.self_lower_dev(d_c, d_o, flags=kssdgpu.NO_ZERO | kssdgpu.SELF_PLAN)  # adds a second copy of every count
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_c.cpu().numpy().view(np.uint32).reshape(-1, 2), 2 * want[0])
    np.testing.assert_array_equal(d_o.cpu().numpy().view(np.uint32).reshape(-1, 2), 2 * want[1])


def test_self_join_autotuner_keeps_counts(monkeypatch):
    for v in ("KSSDGPU_JOIN_FLAT", "KSSDGPU_JOIN_CHUNK", "KSSDGPU_JOIN_SORT"):
        monkeypatch.delenv(v, raising=False)
    sk = _clustered_sketch()
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    t = idx.self_plan_tune()
    assert t["candidates"] == 9 and 1 <= t["flat_groups"] <= 4 and t["step_ms"] > 0
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    got = idx.self_lower(kssdgpu.SELF_PLAN)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.parametrize("misalign", [0, 8])
@pytest.mark.parametrize("path", SELF_PATHS)
def test_self_lower_dev_overwrites_stale_counters(misalign, path):
    """kssdgpu_self_lower_dev zero-fills the device counters before the join adds into
    them (the join may start under the fill's tail and waits for it before its first
    atomic): counters full of stale values come out equal to the oracle's, repeatedly.
    An 8-byte offset takes the memset path instead of the 16-byte fill kernel."""
    import torch
    sk = kssdgpu.synth(n_samples=400, n_clusters=40, len_median=3e5, len_min=1e5, len_max=1e6,
                       size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    cells = sk.n * (sk.n - 1) // 2
    w = misalign // 8
    buf_c = torch.empty(cells + 1, dtype=torch.int64, device="cuda")
    buf_o = torch.empty(cells + 1, dtype=torch.int64, device="cuda")
    d_c, d_o = buf_c[w:w + cells], buf_o[w:w + cells]
    for rep in range(3):
        buf_c.fill_(0x5A5A5A5A5A5A5A5A - rep)
        buf_o.fill_(-1 - rep)
        idx.self_lower_dev(d_c, d_o, flags=path)
        torch.cuda.synchronize()
        got_c = d_c.cpu().numpy().view(np.uint32).reshape(-1, 2)
        got_o = d_o.cpu().numpy().view(np.uint32).reshape(-1, 2)
        np.testing.assert_array_equal(got_c, want[0])
        np.testing.assert_array_equal(got_o, want[1])


def test_read_sets_with_conflicts():
    ref = kssdgpu.synth(n_samples=40, n_clusters=8, len_median=2e5, len_min=1e5, len_max=1e6)
    reads = kssdgpu.synth(n_samples=6, n_clusters=8, role=kssdgpu.ROLE_READS, sample_seed=5,
                          ref_sample_seed=20261203, ref_samples=40, len_median=2e5, len_min=1e5, len_max=1e6,
                          cov_lo=5, cov_hi=20)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    for flags in (0, kssdgpu.IGNORECONFLICT):
        got = idx.count_block(reads.keys, reads.offs, flags | kssdgpu.UNIQUE)
        want = oracle.count_block(rec, ref.n, reads.keys, reads.offs, unique=True,
                                  ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)


def test_golden_cli_counts_on_gpu():
    for name in sorted(f for f in os.listdir(GOLDEN) if f.startswith("counts_")):
        g = json.load(open(os.path.join(GOLDEN, name)))
        rk, ro = samples_to_sketch([[tuple(p) for p in s] for s in g["refs"]])
        qk, qo = samples_to_sketch([[tuple(p) for p in s] for s in g["queries"]])
        rec = oracle.build_index(rk, ro)
        idx = kssdgpu.Index.from_records(rec, len(ro) - 1)
        flags = kssdgpu.UNIQUE | (kssdgpu.IGNORECONFLICT if g["ignoreconflict"] else 0)
        ctx, obj, uctx, uobj = idx.count_block(qk, qo, flags)
        for row in g["rows"]:
            q, r = row["q"], row["r"]
            assert (ctx[q, r, 0], obj[q, r, 0], obj[q, r, 1], ctx[q, r, 1]) == (
                row["XnY_ctx"], row["N_diff_obj"], row["N_diff_obj_section"], row["N_mut2_ctx"])
            assert (uctx[q, r, 0], uobj[q, r, 0], uobj[q, r, 1], uctx[q, r, 1]) == (
                row["Unique_XnY_ctx"], row["Unique_N_diff_obj"], row["Unique_N_diff_obj_section"],
                row["Unique_N_mut2_ctx"])
        assert int((ctx[:, :, 0] > 0).sum()) == len(g["rows"])


def test_edge_cases():
    # empty queries, a query with no shared contexts, a reference with no entries
    refs = [[(1, 0), (2, 3)], [], [(2, 3), (5, 1)]]
    rk, ro = samples_to_sketch(refs)
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, 3)
    qk, qo = samples_to_sketch([[], [(9, 9)], [(2, 0), (2, 3), (5, 2)]])
    got = idx.count_block(qk, qo, kssdgpu.UNIQUE)
    want = oracle.count_block(rec, 3, qk, qo, unique=True)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    # zero queries
    out = idx.count_block(np.zeros(0, np.uint64), np.zeros(1, np.uint64))
    assert out[0].shape == (0, 3, 2)
    # gid at the top of the 20-bit range is rejected when nref is too small
    bad = np.zeros(1, dtype=kssdgpu.REC_DTYPE)
    bad["ctxgid"] = (5 << 20) | 7
    with pytest.raises(kssdgpu.KssdGpuError):
        kssdgpu.Index.from_records(bad, 3)
    # unsorted records are rejected
    two = np.zeros(2, dtype=kssdgpu.REC_DTYPE)
    two["ctxgid"] = [(9 << 20) | 0, (3 << 20) | 0]
    with pytest.raises(kssdgpu.KssdGpuError):
        kssdgpu.Index.from_records(two, 1)


def test_large_gid_and_max_object_width():
    """gid near 2^20 (within nref) and 32-bit objects (min-difference cap of 12)."""
    nref = (1 << 20) - 1
    rec = np.zeros(3, dtype=kssdgpu.REC_DTYPE)
    rec["ctxgid"] = [(4 << 20) | 5, (4 << 20) | (nref - 1), (6 << 20) | (nref - 1)]
    rec["obj"] = [0xFFFFFFFF, 0x0, 0x12345678]
    idx = kssdgpu.Index.from_records(rec, nref, obj_bits=32)
    qk = np.array([(4 << 32) | 0x0, (6 << 32) | 0x12345679], dtype=np.uint64)
    qo = np.array([0, 2], dtype=np.uint64)
    ctx, obj = idx.count_block(qk, qo, kssdgpu.GLOBAL_ACC)
    want = oracle.count_block(rec, nref, qk, qo, obj_bits=32)
    np.testing.assert_array_equal(ctx, want[0])
    np.testing.assert_array_equal(obj, want[1])
    assert obj[0, 5, 1] == 12  # 16 differing bases, capped at NUM_CODENS + 1


def test_chunked_global_rows_with_runs_across_chunks():
    """Global-row mode splits each query into 4,096-entry chunks; context runs
    (conflicting objects) that straddle a chunk boundary are counted once, by the
    chunk holding the run's first entry."""
    ref = kssdgpu.synth(n_samples=40, n_clusters=4, len_median=1e6, len_min=5e5, len_max=2e6)
    reads = kssdgpu.synth(n_samples=6, n_clusters=4, role=kssdgpu.ROLE_READS, sample_seed=7,
                          ref_sample_seed=20261203, ref_samples=40, len_median=1e6, len_min=5e5, len_max=2e6,
                          cov_lo=10, cov_hi=30)
    keys = np.unique(reads.keys)
    # widen the run at every chunk boundary: extra objects on the boundary entry's context
    extra = []
    for b in range(4096, len(keys), 4096):
        ctx = int(keys[b]) >> 20
        extra += [(ctx << 20) | int(o) for o in np.random.default_rng(b).integers(0, 1 << 20, 6)]
    keys = np.unique(np.concatenate([keys, np.array(extra, dtype=np.uint64)]))
    assert len(keys) > 3 * 4096
    qk = np.concatenate([keys, ref.keys[ref.offs[3]:ref.offs[4]]])
    qo = np.array([0, len(keys), len(qk)], dtype=np.uint64)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    for flags in (0, kssdgpu.IGNORECONFLICT):
        want = oracle.count_block(rec, ref.n, qk, qo, unique=True,
                                  ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
        for mode in (0, kssdgpu.GLOBAL_ACC):
            got = idx.count_block(qk, qo, flags | mode | kssdgpu.UNIQUE)
            for g, w in zip(got, want):
                np.testing.assert_array_equal(g, w)
        assert want[0][0, :, 0].sum() > 0
        # device-pointer form: the chunk table is built on the device from the offsets
        import torch
        dev = torch.device("cuda", 0)
        d_keys = torch.from_numpy(qk.view(np.int64)).to(dev)
        # absolute offsets that do not start at 0, an empty query in the middle
        qo2 = np.array([5, 5 + len(keys), 5 + len(keys), 5 + len(qk)], dtype=np.uint64)
        d_keys2 = torch.cat([torch.zeros(5, dtype=torch.int64, device=dev), d_keys])
        d_offs = torch.from_numpy(qo2.view(np.int64)).to(dev)
        outs = [torch.full((3 * ref.n,), -1, dtype=torch.int64, device=dev) for _ in range(4)]
        idx.count_block_dev(d_keys2[5:], d_offs, 3, *outs, flags=flags | kssdgpu.GLOBAL_ACC | kssdgpu.UNIQUE)
        idx.sync()
        got = [o.cpu().numpy().view(np.uint32).reshape(3, ref.n, 2) for o in outs]
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g[0], w[0])
            np.testing.assert_array_equal(g[2], w[1])
            assert not g[1].any()


@pytest.mark.parametrize("stripe_bytes", [0, 32, 2048, 1 << 16])
def test_striped_filter_counts(stripe_bytes):
    """The context membership filter cut into key-range stripes (down to one 32-byte
    block per stripe, up to 256 stripes): block, unique, ignoreconflict and lower
    counts, stripe-major (global rows) and with the stripe found per key (shared rows),
    equal the oracle's counters; the filter admits every context of the index."""
    import torch
    ref = kssdgpu.synth(n_samples=64, n_clusters=8, len_median=3e5, len_min=1e5, len_max=1e6,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=15, sample_seed=15)
    qry = kssdgpu.synth(n_samples=24, n_clusters=8, role=kssdgpu.ROLE_OWNLEN, len_median=3e5, len_min=1e5,
                        len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=2e6,
                        seed=15, sample_seed=16)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    f = idx.filter(stripe_bytes)
    ctxs = idx.info()["contexts"]
    if stripe_bytes and ctxs > stripe_bytes:
        assert 1 < f["stripes"] <= 256
    per_ctx_bits = f["bytes"] * 8 / ctxs
    assert per_ctx_bits >= 8
    # the index's own samples as queries: every context is present and must pass
    self_want = oracle.count_block(rec, ref.n, ref.keys, ref.offs)
    for g, w in zip(idx.count_block(ref.keys, ref.offs, kssdgpu.GLOBAL_ACC), self_want):
        np.testing.assert_array_equal(g, w)
    for flags in (0, kssdgpu.UNIQUE, kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT):
        want = oracle.count_block(rec, ref.n, qry.keys, qry.offs, unique=bool(flags & kssdgpu.UNIQUE),
                                  ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
        for acc in (kssdgpu.GLOBAL_ACC, kssdgpu.SMEM_ACC):
            got = idx.count_block(qry.keys, qry.offs, flags | acc)
            for g, w in zip(got, want):
                np.testing.assert_array_equal(g, w)
    want = oracle.count_lower(rec, ref.n, 0, ref.keys, ref.offs)
    for acc in (kssdgpu.GLOBAL_ACC, kssdgpu.SMEM_ACC):
        got = idx.count_lower(ref.keys, ref.offs, 0, acc)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
    # device buffers, default accumulator, twice (the stripe offsets are scratch)
    dev = torch.device("cuda", 0)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    want = oracle.count_block(rec, ref.n, qry.keys, qry.offs)
    for _ in range(2):
        outs = [torch.full((qry.n * ref.n,), -1, dtype=torch.int64, device=dev) for _ in range(2)]
        idx.count_block_dev(dk, do, qry.n, *outs)
        idx.sync()
        for o, w in zip(outs, want):
            np.testing.assert_array_equal(o.cpu().numpy().view(np.uint32).reshape(qry.n, ref.n, 2), w)
    idx.close()


def test_count_autotuner_keeps_counts():
    """kssdgpu_count_tune times the accumulator settings on a block; its outputs and
    every later count (under the chosen setting) equal the oracle's counters."""
    import torch
    ref = kssdgpu.synth(n_samples=64, n_clusters=8, len_median=3e5, len_min=1e5, len_max=1e6,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=5, sample_seed=5)
    qry = kssdgpu.synth(n_samples=24, n_clusters=8, role=kssdgpu.ROLE_OWNLEN, len_median=3e5, len_min=1e5,
                        len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=2e6,
                        seed=5, sample_seed=6)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    want = oracle.count_block(rec, ref.n, qry.keys, qry.offs, unique=True)
    dev = torch.device("cuda", 0)
    dk = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    do = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    outs = [torch.zeros(qry.n * ref.n, dtype=torch.int64, device=dev) for _ in range(4)]
    t = idx.count_tune(dk, do, qry.n, *outs, flags=kssdgpu.UNIQUE)
    # 4 accumulator settings, then the best of them with the membership filter toggled
    assert t["candidates"] == 5 and t["chunk_keys"] in (1024, 4096, 16384) and t["ms"] > 0
    assert t["filter"] in (0, 1)
    for _ in range(2):
        got = [o.cpu().numpy().view(np.uint32).reshape(qry.n, ref.n, 2) for o in outs]
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
        for o in outs:
            o.fill_(-1)
        idx.count_block_dev(dk, do, qry.n, *outs, flags=kssdgpu.UNIQUE)
        idx.sync()
    host = idx.count_block(qry.keys, qry.offs, kssdgpu.UNIQUE)
    for g, w in zip(host, want):
        np.testing.assert_array_equal(g, w)
    # shared rows cannot be forced where a row does not fit
    big = np.zeros(2, dtype=kssdgpu.REC_DTYPE)
    big["ctxgid"] = [(1 << 20) | 0, (2 << 20) | 20000]
    bidx = kssdgpu.Index.from_records(big, 20001)
    with pytest.raises(kssdgpu.KssdGpuError) as e:
        bidx.count_block(qry.keys[:10], np.array([0, 10], dtype=np.uint64), kssdgpu.SMEM_ACC)
    assert e.value.code == 7


@pytest.mark.parametrize("max_freq,step", [(256, 1), (0, 1), (2, 1), (256, 3), (1, 2)])
def test_sparse_scan_votes(max_freq, step):
    """Candidate votes of the indexed sparse scan (and the scan's first-touch order)
    equal the oracle's, on conflict-free genomes with shared and unshared contexts."""
    sk = kssdgpu.synth(n_samples=60, n_clusters=6, len_median=3e5, len_min=1e5, len_max=1e6,
                       size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=9, sample_seed=9)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    v, f = idx.self_votes(sk.keys, sk.offs, max_freq, step)
    wv, wf = oracle.self_votes(rec, sk.keys, sk.offs, max_freq=max_freq, step=step)
    np.testing.assert_array_equal(v, wv)
    np.testing.assert_array_equal(f, wf)
    # a group of one posting holds no pair: max_freq 1 nominates nothing
    assert (wv.sum() > 0) == (max_freq != 1)
    # absolute offsets that do not start at 0
    offs2 = sk.offs + np.uint64(7)
    keys2 = sk.keys
    v2, f2 = idx.self_votes(keys2, offs2, max_freq, step)
    np.testing.assert_array_equal(v2, wv)
    np.testing.assert_array_equal(f2, wf)


@pytest.mark.parametrize("mode", ["block_unique", "lower"])
def test_pinned_host_buffers_pipeline(mode):
    """With page-locked host buffers a large block is split into sub-blocks whose copies
    overlap the counting; the counters equal the single-pass ones (pageable buffers)."""
    import torch
    sk = kssdgpu.synth(n_samples=600, n_clusters=60, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                       len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=3, sample_seed=3)
    assert int(sk.offs[-1]) >= 8 << 20
    idx = kssdgpu.Index.from_sketch(sk)
    n = sk.n
    lib = kssdgpu.gpu_lib()
    h_keys = torch.from_numpy(sk.keys.view(np.int64)).pin_memory()
    nout = 4 if mode == "block_unique" else 2
    outs = [torch.empty(n * n * 2, dtype=torch.int32).pin_memory() for _ in range(nout)]
    offs = np.ascontiguousarray(sk.offs)
    if mode == "block_unique":
        rc = lib.kssdgpu_count_block(idx.handle, h_keys.data_ptr(), offs, n, kssdgpu.UNIQUE,
                                     *[o.data_ptr() for o in outs])
        want = idx.count_block(sk.keys, sk.offs, kssdgpu.UNIQUE)
    else:
        rc = lib.kssdgpu_count_lower(idx.handle, h_keys.data_ptr(), offs, n, 0, 0, outs[0].data_ptr(),
                                     outs[1].data_ptr())
        want = idx.count_lower(sk.keys, sk.offs, 0)
    assert rc == 0, lib.kssdgpu_last_error()
    for g, w in zip(outs, want):
        np.testing.assert_array_equal(g.numpy().view(np.uint32).reshape(n, n, 2), w)


def _naive_ani(xny, diff, sect):
    """1 - get_naive_dist (src/command_ani.h:202-224), numpy FP64."""
    xny, diff, sect = (np.asarray(v, dtype=np.float64) for v in (xny, diff, sect))
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = (sect + 1e-8) / (diff + 1e-8)
        dist0 = diff / (xny + diff)
        fd = 1 - np.power(1 - dist0, ratio)
    w = np.minimum(fd / 0.01, 1.0)
    d = np.where(fd <= 0, 0.0, fd * 0.1544286 + 7.133e-4 * w)
    return 1 - np.where(xny == 0, 1.0, d)


@pytest.mark.parametrize("flags", [0, kssdgpu.UNIQUE, kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT])
@pytest.mark.parametrize("cuts", [(3, 0.5, 0.95), (1, 0.0, 0.0), (5, 0.3, 0.85)])
def test_count_detail_candidates(flags, cuts):
    """kssdgpu_count_detail keeps every cell the reference's detail pre-filter keeps
    (the candidates are a superset within the 1e-9 ANI margin), in ascending (query,
    ref) order with the dense block's counters."""
    ctxcut, afcut, anicut = cuts
    ref = kssdgpu.synth(n_samples=150, n_clusters=15, len_median=3e5, len_min=1e5, len_max=1e6,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.08, seed=51, sample_seed=51)
    qry = kssdgpu.synth(n_samples=30, n_clusters=15, role=kssdgpu.ROLE_OWNLEN, len_median=3e5, len_min=1e5,
                        len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=1.2e6,
                        seed=51, sample_seed=52)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    rcnt = np.diff(ref.offs).astype(np.uint32)
    qcnt = np.diff(qry.offs).astype(np.uint32)
    hits, roffs = idx.count_detail(qry.keys, qry.offs, qcnt, rcnt, flags, ctxcut, afcut, anicut, cap=64)
    dense = oracle.count_block(rec, ref.n, qry.keys, qry.offs, unique=True,
                               ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
    c, o, uc, uo = (x.astype(np.int64) for x in dense)
    shared = c[:, :, 0]
    with np.errstate(divide="ignore", invalid="ignore"):
        af = np.maximum(shared / qcnt[:, None].astype(np.float64), shared / rcnt[None, :].astype(np.float64))
        if flags & kssdgpu.UNIQUE:
            use_u = uc[:, :, 0] * 20 >= rcnt[None, :]
            ani = np.where(use_u, _naive_ani(uc[:, :, 0], uo[:, :, 0], uo[:, :, 1]),
                           _naive_ani(c[:, :, 0], o[:, :, 0], o[:, :, 1]))
        else:
            dist = (o[:, :, 0].astype(np.float32) / shared.astype(np.float32)) / np.float32(7)
            ani = (np.float32(1) - dist).astype(np.float64)
    base = (shared >= ctxcut) & (qcnt[:, None] > 0) & (rcnt[None, :] > 0) & (af >= np.float64(np.float32(afcut)))
    exact = base & (ani >= np.float64(np.float32(anicut)))
    loose = base & (ani >= np.float64(np.float32(anicut)) - 1e-9)
    got = np.zeros_like(exact)
    got[hits["query"], hits["ref"]] = True
    assert (exact <= got).all() and (got <= loose).all()
    assert exact.sum() > 0
    assert np.all(np.diff(hits["query"].astype(np.int64) * ref.n + hits["ref"]) > 0)
    np.testing.assert_array_equal(roffs, np.concatenate([[0], np.cumsum(got.sum(axis=1))]))
    q, r = hits["query"], hits["ref"]
    np.testing.assert_array_equal(hits["num_ctx"], dense[0][q, r, 0])
    np.testing.assert_array_equal(hits["num_mut2_ctx"], dense[0][q, r, 1])
    np.testing.assert_array_equal(hits["diff_obj"], dense[1][q, r, 0])
    np.testing.assert_array_equal(hits["diff_obj_section"], dense[1][q, r, 1])
    if flags & kssdgpu.UNIQUE:
        np.testing.assert_array_equal(hits["u_num_ctx"], dense[2][q, r, 0])
        np.testing.assert_array_equal(hits["u_diff_obj_section"], dense[3][q, r, 1])
    if oracle.ref_available():
        # the reference's own detail pre-filter keeps exactly the exact set
        _, npass, ranked = oracle.count_detail_ref(rec, ref.n, qry.keys, qry.offs, rcnt, qcnt,
                                                   ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT),
                                                   unique=bool(flags & kssdgpu.UNIQUE), ctxcut=ctxcut, afcut=afcut,
                                                   anicut=anicut, ntop=ref.n)
        for i in range(qry.n):
            ids = set(ranked.reshape(qry.n, ref.n)[i, :npass[i]].tolist())
            assert ids == set(np.flatnonzero(exact[i]).tolist())


def _wide_cluster(n=160, seed=61, sub_hi=0.01):
    """One species: every genome a member of one cluster at 0.1-1% substitutions, so most
    contexts are shared by most genomes (dense incidence)."""
    return kssdgpu.synth(n_samples=n, n_clusters=1, len_median=4e5, len_min=2e5, len_max=8e5,
                         size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=sub_hi, seed=seed, sample_seed=seed)


@pytest.mark.parametrize("n,seed,sub_hi", [(160, 61, 0.01), (300, 62, 0.03), (129, 63, 0.2), (2, 64, 0.01),
                                            (700, 65, 0.01)])
def test_self_dense_join_matches_oracle(n, seed, sub_hi):
    """The dense tensor-core self join (alleles of the shared contexts, int8 GEMMs) gives
    the oracle's counters; on a dense index the default path chooses it.  700 genomes
    (6 blocks of 128, the last of 64) take the GEMM per block below the diagonal."""
    sk = _wide_cluster(n, seed, sub_hi)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    for flags in (kssdgpu.SELF_DENSE, 0, kssdgpu.SELF_SCAN):
        got = idx.self_lower(flags)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])
    path, density = idx.self_choice()
    if sub_hi <= 0.03 and n >= 100:
        assert path == kssdgpu.PATH_DENSE and density >= 1 / 2048
    assert idx.self_choice(kssdgpu.SELF_SCAN)[0] == kssdgpu.PATH_SCAN


@pytest.mark.parametrize("case", [c for c in CASES if not c[5]])
def test_self_dense_join_on_sparse_fixtures(case):
    """Forced on sparse conflict-free fixtures (empty samples, contexts of one genome)."""
    rk, ro, _, _ = _fixture(*case)
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, len(ro) - 1)
    want = oracle.self_lower_all(rec, rk, ro)
    got = idx.self_lower(kssdgpu.SELF_DENSE)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    assert idx.self_choice()[0] == kssdgpu.PATH_SCAN  # sparse: the scan


def test_self_dense_join_wide_objects_and_conflicts():
    """32-bit objects (differences capped at NUM_CODENS + 1) through the dense join; an
    index with conflicts refuses it and the default path falls back to the scan."""
    rng = np.random.default_rng(9)
    samples = [[(c, int(rng.integers(0, 1 << 32))) for c in range(40) if rng.random() < 0.8] for _ in range(50)]
    rk, ro = samples_to_sketch(samples, obj_bits=32)
    rec = oracle.build_index(rk, ro, obj_bits=32)
    idx = kssdgpu.Index.from_records(rec, 50, obj_bits=32)
    want = oracle.self_lower_all(rec, rk, ro, obj_bits=32)
    got = idx.self_lower(kssdgpu.SELF_DENSE)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    assert want[1][:, 1].max() > 0
    rk, ro, _, _ = _fixture(*CASES[0])  # conflicts
    rec = oracle.build_index(rk, ro)
    idx = kssdgpu.Index.from_records(rec, len(ro) - 1)
    with pytest.raises(kssdgpu.KssdGpuError) as e:
        idx.self_lower(kssdgpu.SELF_DENSE)
    assert e.value.code == 1
    assert idx.self_choice()[0] == kssdgpu.PATH_SCAN


@pytest.mark.parametrize("n,clusters,table_log", [(6000, 600, None), (4500, 50, None), (4500, 50, 4)])
def test_self_scan_with_counters_beyond_l2(n, clusters, table_log, monkeypatch):
    """Small genomes whose packed triangle (4,500 genomes: 10M cells, 162 MB) outgrows
    L2: the scan join adds through the table of touched cells and flushes it into the
    triangle.  Clusters of 90 genomes give context groups of more than 32 postings (dealt
    out over the CTA, into the table); a table of 16 slots sends nearly every cell to the
    triangle directly.  The counters equal the oracle's on two calls in a row (the flush
    empties the table), and a NO_ZERO call adds onto the previous counters."""
    import torch
    if table_log is not None:
        monkeypatch.setenv("KSSDGPU_CELL_TABLE_LOG", str(table_log))
    sk = kssdgpu.synth(n_samples=n, n_clusters=clusters, len_median=8e4, len_min=5e4, len_max=1.5e5,
                       size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=71 + clusters,
                       sample_seed=71 + clusters)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    want = oracle.self_lower_all(rec, sk.keys, sk.offs)
    for _ in range(2):
        got = idx.self_lower(kssdgpu.SELF_SCAN)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])
    assert want[0][:, 0].sum() > 0
    if clusters == 50:
        _, sizes = np.unique(rec["ctxgid"] >> 20, return_counts=True)
        assert sizes.max() > 32  # groups of more than 32 postings are present
    cells = n * (n - 1) // 2
    dev = torch.device("cuda", 0)
    lc = torch.zeros(cells, dtype=torch.int64, device=dev)
    lo = torch.zeros_like(lc)
    idx.self_lower_dev(lc, lo, flags=kssdgpu.SELF_SCAN)
    idx.self_lower_dev(lc, lo, flags=kssdgpu.SELF_SCAN | kssdgpu.NO_ZERO)
    idx.sync()
    got_c = lc.cpu().numpy().view(np.uint32).reshape(cells, 2)
    got_o = lo.cpu().numpy().view(np.uint32).reshape(cells, 2)
    np.testing.assert_array_equal(got_c, 2 * want[0].reshape(cells, 2))
    np.testing.assert_array_equal(got_o, 2 * want[1].reshape(cells, 2))
    idx.close()

@pytest.mark.parametrize("case", ["block", "block_unique", "lower", "reads_unique_ignoreconflict", "smem_unique",
                                  "striped_unique", "striped_lower"])
def test_batched_count_on_long_postings_lists(case):
    """References of one species (contexts shared by up to 300 genomes): query contexts
    whose groups hold 32 or more postings are walked by the whole warp (coalesced
    postings, run heads by shuffle, owners by ballot); the counters equal the oracle's
    for blocks, lower blocks, read sets with conflicts under --ignoreconflict, shared-
    and global-memory rows and the stripe-major count."""
    ref = _wide_cluster(300, 65, 0.03)
    rec = oracle.build_index(ref.keys, ref.offs)
    _, sizes = np.unique(rec["ctxgid"] >> 20, return_counts=True)
    assert sizes.max() >= 200 and sizes[sizes >= 32].sum() > 0.5 * sizes.sum()  # most postings in long groups
    idx = kssdgpu.Index.from_records(rec, ref.n)
    flags, unique = 0, False
    qry = kssdgpu.synth(n_samples=24, n_clusters=1, role=kssdgpu.ROLE_OWNLEN, len_median=4e5, len_min=2e5,
                        len_max=8e5, size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.03, seed=65,
                        sample_seed=66, own_len_min=5e4, own_len_max=8e5)
    if case.startswith("striped"):
        assert idx.filter(4096)["stripes"] > 1
    if case in ("block_unique", "smem_unique", "striped_unique"):
        flags, unique = kssdgpu.UNIQUE, True
    if case == "smem_unique":
        flags |= kssdgpu.SMEM_ACC
    if case == "reads_unique_ignoreconflict":
        qry = kssdgpu.synth(n_samples=4, n_clusters=1, role=kssdgpu.ROLE_READS, sample_seed=67, ref_sample_seed=65,
                            ref_samples=300, len_median=4e5, len_min=2e5, len_max=8e5, cov_lo=5, cov_hi=15)
        flags, unique = kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT, True
    if case in ("lower", "striped_lower"):
        off = 100
        qk = ref.keys[int(ref.offs[off]):int(ref.offs[off + 60])]
        qo = np.ascontiguousarray(ref.offs[off:off + 61])
        got = idx.count_lower(qk, qo, off, flags)
        want = oracle.count_lower(rec, ref.n, off, qk, qo)
    else:
        got = idx.count_block(qry.keys, qry.offs, flags)
        want = oracle.count_block(rec, ref.n, qry.keys, qry.offs, unique=unique,
                                  ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    assert want[0][:, :, 0].sum() > 0
    idx.close()


@pytest.mark.parametrize("case", ["block", "lower", "striped", "tiny_table"])
def test_batched_count_beyond_l2(case, monkeypatch):
    """A block of 2,500 queries x 4,000 references (10M counter cells, 160 MB: larger
    than L2) through the global-row count, chunked and stripe-major, and as a lower
    block; the table of touched cells shrunk to 16 slots must not matter (the count adds
    into its rows directly).  Counters equal the oracle's, on two calls in a row."""
    if case == "tiny_table":
        monkeypatch.setenv("KSSDGPU_CELL_TABLE_LOG", "4")
    ref = kssdgpu.synth(n_samples=4000, n_clusters=400, len_median=8e4, len_min=5e4, len_max=1.5e5,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=81, sample_seed=81)
    rec = oracle.build_index(ref.keys, ref.offs)
    idx = kssdgpu.Index.from_records(rec, ref.n)
    if case == "striped":
        assert idx.filter(1 << 16)["stripes"] > 1
    if case == "lower":
        off = 1500
        qk = ref.keys[int(ref.offs[off]):int(ref.offs[off + 2500])]
        qo = np.ascontiguousarray(ref.offs[off:off + 2501])
        want = oracle.count_lower(rec, ref.n, off, qk, qo)
        for _ in range(2):
            got = idx.count_lower(qk, qo, off, kssdgpu.GLOBAL_ACC)
            for g, w in zip(got, want):
                np.testing.assert_array_equal(g, w)
    else:
        qry = kssdgpu.synth(n_samples=2500, n_clusters=400, role=kssdgpu.ROLE_OWNLEN, len_median=8e4, len_min=5e4,
                            len_max=1.5e5, size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=81,
                            sample_seed=82, own_len_min=2e4, own_len_max=1.5e5)
        want = oracle.count_block(rec, ref.n, qry.keys, qry.offs)
        for _ in range(2):
            got = idx.count_block(qry.keys, qry.offs, kssdgpu.GLOBAL_ACC)
            for g, w in zip(got, want):
                np.testing.assert_array_equal(g, w)
    assert want[0][:, :, 0].sum() > 0
    idx.close()

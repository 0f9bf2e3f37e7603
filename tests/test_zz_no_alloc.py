"""kssdgpu_count_block_noalloc: the counting entry point for callers that must not
allocate device memory during a call (a serving loop that reserved all device
memory for its admission budget, an application whose own allocator owns the
device).  It must give the same counters as kssdgpu_count_block_dev, call after
call, with its scratch in the library's static device array.

This file is collected last on purpose (tests run in name order), so a run that
stops at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

import kssdgpu
import oracle

pytestmark = pytest.mark.gpu

MAX_QUERIES = 65536          # KSSDGPU_NOALLOC_MAX_QUERIES
ERR_CAPACITY = 7             # KSSDGPU_ERR_CAPACITY


def _lib():
    lib = kssdgpu.gpu_lib()
    vp = C.c_void_p
    lib.kssdgpu_count_block_noalloc.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_uint,
                                                vp, vp, vp, vp, vp]
    lib.kssdgpu_count_block_noalloc.restype = C.c_int
    return lib


def _noalloc(idx, d_keys, d_offs, nq, outs, flags=0, lower=False, qgid_offset=0):
    import torch
    lib = _lib()
    ptrs = [o.data_ptr() for o in outs] + [None] * (4 - len(outs))
    rc = lib.kssdgpu_count_block_noalloc(idx.handle, d_keys.data_ptr(), d_offs.data_ptr(), nq, qgid_offset,
                                         int(lower), flags, *ptrs, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.kssdgpu_last_error().decode()
    torch.cuda.synchronize()


def _workload():
    ref = kssdgpu.synth(n_samples=120, n_clusters=12, len_median=3e5, len_min=1e5, len_max=1e6,
                        size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1)
    qry = kssdgpu.synth(n_samples=40, n_clusters=12, role=kssdgpu.ROLE_OWNLEN, sample_seed=31,
                        len_median=3e5, len_min=1e5, len_max=1e6, size_dist=kssdgpu.SIZE_LOGNORMAL,
                        own_len_min=2e4, own_len_max=1.5e6)
    reads = kssdgpu.synth(n_samples=5, n_clusters=12, role=kssdgpu.ROLE_READS, sample_seed=32,
                          ref_sample_seed=20261203, ref_samples=120, len_median=3e5, len_min=1e5,
                          len_max=1e6, cov_lo=5, cov_hi=15)
    return ref, qry, reads


@pytest.mark.parametrize("case", ["block", "block_unique", "reads_ignoreconflict", "lower", "global_acc",
                                  "smem_acc", "lower_offset", "striped_block_unique", "striped_lower"])
def test_noalloc_matches_existing_entry_point_twice(case):
    import torch
    ref, qry, reads = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    flags, lower, q, off = 0, False, qry, 0
    if case.startswith("striped_"):
        # a filter of many key-range stripes: the existing entry point counts stripe by
        # stripe, the no-allocation one finds each context's stripe per key
        assert idx.filter(512)["stripes"] > 1
        case = case[len("striped_"):]
    if case == "block_unique":
        flags = kssdgpu.UNIQUE
    elif case == "reads_ignoreconflict":
        flags, q = kssdgpu.UNIQUE | kssdgpu.IGNORECONFLICT, reads
    elif case == "lower":
        lower, q = True, ref
    elif case == "global_acc":
        flags = kssdgpu.GLOBAL_ACC | kssdgpu.UNIQUE
    elif case == "smem_acc":
        flags = kssdgpu.SMEM_ACC | kssdgpu.UNIQUE
    elif case == "lower_offset":
        # a block of the reference's own samples past the first: gids below 50 + i count
        lower, off = True, 50
        q = kssdgpu.Sketch(keys=ref.keys[int(ref.offs[off]):int(ref.offs[off + 40])],
                           offs=np.ascontiguousarray(ref.offs[off:off + 41]), names=[])
    nq, nref = q.n, ref.n
    d_keys = torch.from_numpy(q.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(q.offs.view(np.int64)).to(dev)
    nout = 4 if flags & kssdgpu.UNIQUE else 2
    want = [torch.zeros(nq * nref, dtype=torch.int64, device=dev) for _ in range(nout)]
    idx.count_block_dev(d_keys, d_offs, nq, *want, flags=flags, lower=lower, qry_gid_offset=off)
    idx.sync()
    for call in range(2):  # two calls in a row share the one scratch array
        got = [torch.full((nq * nref,), -1, dtype=torch.int64, device=dev) for _ in range(nout)]
        _noalloc(idx, d_keys, d_offs, nq, got, flags=flags, lower=lower, qgid_offset=off)
        for g, w in zip(got, want):
            assert torch.equal(g, w), f"call {call + 1} differs from kssdgpu_count_block_dev"
    idx.sync()  # no error recorded on the device
    assert int((want[0] & 0xFFFFFFFF).sum()) > 0
    # and both equal the oracle
    rec, _ = idx.export()
    if lower:
        o = oracle.count_lower(rec, nref, off, q.keys, q.offs)
    else:
        o = oracle.count_block(rec, nref, q.keys, q.offs, unique=bool(flags & kssdgpu.UNIQUE),
                               ignoreconflict=bool(flags & kssdgpu.IGNORECONFLICT))
    for w, ow in zip(want, o):
        np.testing.assert_array_equal(w.cpu().numpy().view(np.uint32).reshape(nq, nref, 2), ow)
    idx.close()


def test_noalloc_rejects_more_queries_than_its_scratch_holds():
    import torch
    ref, _, _ = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    d_offs = torch.zeros(MAX_QUERIES + 2, dtype=torch.int64, device=dev)
    d_keys = torch.zeros(1, dtype=torch.int64, device=dev)
    out = torch.zeros(1, dtype=torch.int64, device=dev)
    lib = _lib()
    rc = lib.kssdgpu_count_block_noalloc(idx.handle, d_keys.data_ptr(), d_offs.data_ptr(), MAX_QUERIES + 1, 0, 0,
                                         0, out.data_ptr(), out.data_ptr(), None, None, None)
    assert rc == ERR_CAPACITY
    assert b"maximum" in lib.kssdgpu_last_error()
    idx.close()


def test_noalloc_empty_block_and_unsorted_keys():
    """nq = 0 launches nothing and leaves the outputs untouched; query keys out of order
    are recorded on the device and reported by the next kssdgpu_sync."""
    import torch
    ref, qry, _ = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    d_keys = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    out = [torch.full((qry.n * ref.n,), 7, dtype=torch.int64, device=dev) for _ in range(2)]
    _noalloc(idx, d_keys, d_offs, 0, out)
    assert all(bool((o == 7).all()) for o in out)
    bad = d_keys.clone()
    a, b = int(qry.offs[3]), int(qry.offs[4])
    assert b - a > 2
    bad[a:b] = torch.flip(bad[a:b], [0])
    _noalloc(idx, bad, d_offs, qry.n, out)
    with pytest.raises(kssdgpu.KssdGpuError) as e:
        idx.sync()
    assert e.value.code == 3  # KSSDGPU_ERR_UNSORTED
    idx.sync()  # reported once, then cleared
    idx.close()


def test_noalloc_at_the_query_limit():
    """KSSDGPU_NOALLOC_MAX_QUERIES queries of a few keys each (the chunk prefix fills the
    scratch to its last word) give the counters of kssdgpu_count_block_dev."""
    import torch
    ref, qry, _ = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    sizes = rng.integers(0, 4, size=MAX_QUERIES)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    src = rng.integers(0, qry.n, size=MAX_QUERIES)
    keys = np.concatenate([np.sort(rng.choice(qry.keys[int(qry.offs[q]):int(qry.offs[q + 1])], size=k, replace=False))
                           for q, k in zip(src, sizes) if k]).astype(np.uint64)
    d_keys = torch.from_numpy(keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(offs.view(np.int64)).to(dev)
    cells = MAX_QUERIES * ref.n
    want = [torch.zeros(cells, dtype=torch.int64, device=dev) for _ in range(2)]
    idx.count_block_dev(d_keys, d_offs, MAX_QUERIES, *want)
    idx.sync()
    got = [torch.full((cells,), -1, dtype=torch.int64, device=dev) for _ in range(2)]
    _noalloc(idx, d_keys, d_offs, MAX_QUERIES, got)
    idx.sync()
    assert all(torch.equal(g, w) for g, w in zip(got, want))
    assert int((want[0] & 0xFFFFFFFF).sum()) > 0
    idx.close()


def test_noalloc_with_no_queries_leaves_outputs_untouched():
    """nq = 0 (an empty batch a serving loop may hand over) succeeds, launches nothing
    that writes the outputs, and the next call still matches the existing entry point."""
    import torch
    ref, qry, _ = _workload()
    idx = kssdgpu.Index.from_sketch(ref)
    dev = torch.device("cuda", 0)
    out = [torch.full((8,), -1, dtype=torch.int64, device=dev) for _ in range(2)]
    d_offs = torch.zeros(1, dtype=torch.int64, device=dev)
    d_keys = torch.zeros(1, dtype=torch.int64, device=dev)
    _noalloc(idx, d_keys, d_offs, 0, out)
    for o in out:
        assert bool((o == -1).all())
    d_keys = torch.from_numpy(qry.keys.view(np.int64)).to(dev)
    d_offs = torch.from_numpy(qry.offs.view(np.int64)).to(dev)
    want = [torch.zeros(qry.n * ref.n, dtype=torch.int64, device=dev) for _ in range(2)]
    got = [torch.full((qry.n * ref.n,), -1, dtype=torch.int64, device=dev) for _ in range(2)]
    idx.count_block_dev(d_keys, d_offs, qry.n, *want)
    idx.sync()
    _noalloc(idx, d_keys, d_offs, qry.n, got)
    for g, w in zip(got, want):
        assert torch.equal(g, w)
    idx.close()

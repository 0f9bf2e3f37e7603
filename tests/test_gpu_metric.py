"""The FP64 matrix-value epilogue on the device (kssdgpu_lower_metric_dev,
kssdgpu_self_lower_metric) against the host epilogue's kssd_pair_metric (itself
bit-identical to the reference's functions, tests/test_epilogue.py): over random
lower triangles of counters and every metric option, each value the device keeps
prints the host's six decimals (fixed6 and "%lf"), and is the host's double bit for bit
where the metric is built from + - * / only (lm3ways, the calibration trees, p-dist);
the cells it lists for the host are few, carry their counters, and are exactly the ones
it left as NaN."""
import ctypes as C

import numpy as np
import pytest
import torch

import kssdgpu
import oracle

pytestmark = pytest.mark.gpu


class Feat(C.Structure):
    _fields_ = [("XnY_ctx", C.c_uint32), ("X_ctx", C.c_uint32), ("N_diff_obj_section", C.c_uint32),
                ("N_mut2_ctx", C.c_uint32), ("N_diff_obj", C.c_uint32)]


class AniOpt(C.Structure):
    """kssd_ani_opt_t (host/kssd_epilogue.h), field for field."""
    _fields_ = [("fmt", C.c_int), ("p", C.c_int), ("d", C.c_bool), ("v", C.c_bool), ("unassembled", C.c_bool),
                ("unified_metric", C.c_bool), ("ignoreconflict", C.c_bool), ("raw_output", C.c_bool),
                ("max_pdist_set", C.c_bool), ("max_pdist", C.c_double), ("max_diff_obj_section", C.c_int),
                ("e", C.c_int), ("s", C.c_int), ("ntop", C.c_int), ("ctxcut", C.c_int), ("afcut", C.c_float),
                ("afcut_set", C.c_bool), ("anicut", C.c_float), ("unique_ctx", C.c_bool),
                ("estimate_coverage", C.c_bool), ("obj_bits", C.c_int), ("ctx_bits", C.c_int), ("drfold", C.c_int)]


def _host():
    lib = kssdgpu.host_lib()
    lib.kssd_opt_defaults.argtypes = [C.POINTER(AniOpt)]
    lib.kssd_opt_defaults.restype = None
    lib.kssd_pair_metric.argtypes = [C.POINTER(Feat), C.c_uint32, C.c_uint32, C.POINTER(AniOpt), C.c_void_p,
                                     C.c_void_p]
    lib.kssd_pair_metric.restype = C.c_double
    lib.kssd_zero_overlap_metric.argtypes = [C.POINTER(AniOpt), C.POINTER(C.c_double)]
    lib.kssd_zero_overlap_metric.restype = C.c_bool
    return lib


def _triangle(rng, n):
    """Counters of n(n-1)/2 cells shaped like a self matrix: sketch sizes of 5k-30k (a few
    empty samples), 40 % of cells sharing nothing, the rest sharing from a few contexts to
    most of the smaller sketch (so the AF gate passes and the calibration trees run)."""
    size = rng.integers(5000, 30000, size=n).astype(np.uint32)
    size[rng.random(n) < 0.03] = 0
    q = np.repeat(np.arange(n), np.arange(n))
    r = np.concatenate([np.arange(i) for i in range(n)]).astype(np.int64)
    cells = len(q)
    small = np.minimum(size[q], size[r]).astype(np.float64)
    frac = np.where(rng.random(cells) < 0.5, rng.uniform(0.3, 1.0, cells), rng.uniform(0.0, 0.3, cells) ** 3)
    xny = np.floor(small * frac).astype(np.uint32)
    xny[rng.random(cells) < 0.4] = 0
    div = rng.uniform(0, 0.25, cells) ** 2
    dobj = np.minimum(xny, np.floor(xny * div * rng.uniform(0.5, 4, cells))).astype(np.uint32)
    dobj[rng.random(cells) < 0.05] = 0
    mut2 = np.floor(dobj * rng.uniform(0, 0.6, cells)).astype(np.uint32)
    sect = (dobj + mut2 + np.floor(mut2 * rng.uniform(0, 3, cells))).astype(np.uint32)
    lc = xny.astype(np.uint64) | (mut2.astype(np.uint64) << np.uint64(32))
    lo = dobj.astype(np.uint64) | (sect.astype(np.uint64) << np.uint64(32))
    return size, q, r, lc, lo


OPTIONS = [dict(s=1), dict(s=-1), dict(s=2), dict(s=-2), dict(s=3), dict(s=-3), dict(s=4), dict(s=-4), dict(s=5),
           dict(s=6), dict(s=7), dict(s=-8), dict(s=9), dict(s=1, v=1), dict(s=-2, v=1), dict(s=-1, raw_output=1),
           dict(s=1, unassembled=1), dict(s=-1, unassembled=1, unified_metric=1), dict(s=-1, afcut=0.0),
           dict(s=1, afcut=0.9, e=0), dict(s=-1, drfold=6), dict(s=-1, drfold=10, e=0), dict(s=-5, ctx_bits=40)]


@pytest.mark.parametrize("case", range(len(OPTIONS)),
                         ids=[",".join(f"{k}={v}" for k, v in o.items()) for o in OPTIONS])
def test_device_matrix_values_match_host(case):
    opt = OPTIONS[case]
    host = _host()
    o = AniOpt()
    host.kssd_opt_defaults(C.byref(o))
    o.fmt = 1
    for k, v in opt.items():
        setattr(o, k, v)
    zero = C.c_double()
    zero_const = bool(host.kssd_zero_overlap_metric(C.byref(o), C.byref(zero)))
    rng = np.random.default_rng(900 + case)
    n = 360
    size, q, r, lc, lo = _triangle(rng, n)
    cells = len(lc)
    mo = kssdgpu.metric_opt(s=o.s, e=o.e, v=int(o.v), unassembled=int(o.unassembled),
                            unified_metric=int(o.unified_metric), raw_output=int(o.raw_output), afcut=o.afcut,
                            drfold=o.drfold, obj_bits=o.obj_bits, ctx_bits=o.ctx_bits, zero_const=int(zero_const),
                            zero_value=zero.value)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64 if a.dtype.itemsize == 8 else np.int32)).to(dev)  # noqa: E731,E501
    d_size, d_lc, d_lo = t(size), t(lc), t(lo)
    d_val = torch.zeros(cells, dtype=torch.float64, device=dev)
    cap = cells
    d_re = torch.zeros(cap * 3, dtype=torch.int64, device=dev)
    d_nre = torch.zeros(1, dtype=torch.int64, device=dev)
    kssdgpu.lower_metric_dev(mo, n, d_size, d_size, d_lc, d_lo, d_val, d_re, cap, d_nre)
    torch.cuda.synchronize()
    got = d_val.cpu().numpy()
    nre = int(d_nre.item())
    re = d_re.cpu().numpy().view(kssdgpu.RECHECK_DTYPE)[:nre]
    # the host's value of every cell (the CLI's self_cell_metric)
    want = np.empty(cells)
    f = Feat()
    for i in range(cells):
        c, ob = int(lc[i]), int(lo[i])
        qs, rs = int(size[q[i]]), int(size[r[i]])
        if zero_const and (c & 0xFFFFFFFF) == 0 and qs and rs:
            want[i] = zero.value
            continue
        f.XnY_ctx, f.N_mut2_ctx = c & 0xFFFFFFFF, c >> 32
        f.N_diff_obj, f.N_diff_obj_section = ob & 0xFFFFFFFF, ob >> 32
        f.X_ctx = 0
        want[i] = host.kssd_pair_metric(C.byref(f), qs, rs, C.byref(o), None, None)
    listed = np.zeros(cells, dtype=bool)
    listed[re["cell"].astype(np.int64)] = True
    assert np.isnan(got[listed]).all()
    keep = ~listed
    g, w = got[keep], want[keep]
    exact = abs(opt["s"]) in (1, 2, 3, 9) and not opt.get("v") and not opt.get("unassembled")
    if exact:
        assert np.array_equal(g.view(np.uint64), w.view(np.uint64)), \
            np.nonzero(g.view(np.uint64) != w.view(np.uint64))[0][:5]
    fin = np.isfinite(w)
    assert np.array_equal(np.isfinite(g), fin)
    fixed6 = lambda v: np.where(v >= 0, v * 1000000.0 + 0.5, v * 1000000.0 - 0.5).astype(np.int64)  # noqa: E731
    assert np.array_equal(fixed6(g[fin]), fixed6(w[fin]))
    assert [f"{x:f}" for x in g] == [f"{x:f}" for x in w]
    # listed cells carry their counters; they are a small minority
    cl = re["cell"].astype(np.int64)
    assert np.array_equal(re["num_ctx"].astype(np.uint64) | (re["num_mut2_ctx"].astype(np.uint64) << np.uint64(32)),
                          lc[cl])
    assert np.array_equal(re["diff_obj"].astype(np.uint64) | (re["diff_obj_section"].astype(np.uint64) << np.uint64(32)),
                          lo[cl])
    assert nre <= max(10, cells // 1000), nre


def test_self_lower_metric_matches_host_epilogue():
    """The self join + device epilogue of an index's own samples against the host
    epilogue over kssdgpu_self_lower's counters; a one-entry recheck list returns
    KSSDGPU_ERR_CAPACITY when more cells need the host."""
    host = _host()
    o = AniOpt()
    host.kssd_opt_defaults(C.byref(o))
    o.fmt, o.s = 1, -1
    sk = kssdgpu.synth(n_samples=300, n_clusters=30, len_median=1e6, len_min=3e5, len_max=3e6,
                       size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.1, seed=5, sample_seed=5)
    rec = oracle.build_index(sk.keys, sk.offs)
    idx = kssdgpu.Index.from_records(rec, sk.n)
    n = sk.n
    cells = n * (n - 1) // 2
    size = np.diff(sk.offs.astype(np.int64)).astype(np.uint32)  # conflict-free sketch: sizes = entries
    zero = C.c_double()
    zero_const = bool(host.kssd_zero_overlap_metric(C.byref(o), C.byref(zero)))
    mo = kssdgpu.metric_opt(s=-1, zero_const=int(zero_const), zero_value=zero.value)
    lib = kssdgpu.gpu_lib()
    val = np.zeros(cells)
    re = np.zeros(cells, dtype=kssdgpu.RECHECK_DTYPE)
    nre = C.c_uint64()
    rc = lib.kssdgpu_self_lower_metric(idx.handle, 0, C.byref(mo), size, size, val.ctypes.data, re.ctypes.data,
                                       cells, C.byref(nre))
    assert rc == 0, lib.kssdgpu_last_error()
    lc, lo = idx.self_lower()
    lc = lc.view(np.uint64).reshape(-1)
    lo = lo.view(np.uint64).reshape(-1)
    listed = np.zeros(cells, dtype=bool)
    listed[re["cell"][:nre.value].astype(np.int64)] = True
    qi = np.repeat(np.arange(n), np.arange(n))
    ri = np.concatenate([np.arange(i) for i in range(n)])
    f = Feat()
    for i in range(cells):
        c, ob = int(lc[i]), int(lo[i])
        qs, rs = int(size[qi[i]]), int(size[ri[i]])
        if zero_const and (c & 0xFFFFFFFF) == 0 and qs and rs:
            w = zero.value
        else:
            f.XnY_ctx, f.N_mut2_ctx = c & 0xFFFFFFFF, c >> 32
            f.N_diff_obj, f.N_diff_obj_section = ob & 0xFFFFFFFF, ob >> 32
            w = host.kssd_pair_metric(C.byref(f), qs, rs, C.byref(o), None, None)
        if listed[i]:
            assert np.isnan(val[i])
        else:
            assert np.float64(val[i]).tobytes() == np.float64(w).tobytes(), (i, val[i], w)
    assert (lc & 0xFFFFFFFF).sum() > 0
    if nre.value > 1:
        small = np.zeros(1, dtype=kssdgpu.RECHECK_DTYPE)
        rc = lib.kssdgpu_self_lower_metric(idx.handle, 0, C.byref(mo), size, size, val.ctypes.data,
                                           small.ctypes.data, 1, C.byref(nre))
        assert rc == 7
    idx.close()

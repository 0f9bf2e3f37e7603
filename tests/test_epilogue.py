"""The host FP64 epilogue (libkssdhost) against the reference's own model functions
(compiled from its sources into oracle/_ref/refharness.so): every double must be
bit-identical, so every printed digit is."""
import ctypes as C
import os

import numpy as np
import pytest

import kssdgpu
import oracle

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")


class Feat(C.Structure):
    _fields_ = [("XnY_ctx", C.c_uint32), ("X_ctx", C.c_uint32), ("N_diff_obj_section", C.c_uint32),
                ("N_mut2_ctx", C.c_uint32), ("N_diff_obj", C.c_uint32)]


def _host():
    lib = kssdgpu.host_lib()
    fp = C.POINTER(Feat)
    for name in ("kssd_lm3ways_dist", "kssd_af_anib"):
        getattr(lib, name).argtypes = [fp, C.c_int]
        getattr(lib, name).restype = C.c_double
    lib.kssd_naive_dist.argtypes = [fp]
    lib.kssd_naive_dist.restype = C.c_double
    lib.kssd_p_dist.argtypes = [fp, C.c_int]
    lib.kssd_p_dist.restype = C.c_double
    for name in ("kssd_mashD", "kssd_aafD"):
        getattr(lib, name).argtypes = [C.c_uint32] * 4
        getattr(lib, name).restype = C.c_double
    lib.kssd_hgb_predict_ani.argtypes = [C.c_double, C.c_double] + [C.c_uint] * 4 + [C.c_int]
    lib.kssd_hgb_predict_ani.restype = C.c_double
    return lib


def _ref():
    lib = oracle.ref_lib()
    lib.refh_models.argtypes = [np.ctypeslib.ndpointer(np.uint32), C.c_int, C.c_int,
                                np.ctypeslib.ndpointer(np.float64)]
    lib.refh_hgb.argtypes = [C.c_double, C.c_double] + [C.c_uint] * 4 + [C.c_int]
    lib.refh_hgb.restype = C.c_double
    return lib


def _same(a, b):
    return np.float64(a).tobytes() == np.float64(b).tobytes() or (np.isnan(a) and np.isnan(b))


def _features(rng, n):
    out = []
    for _ in range(n):
        xny = int(rng.choice([0, 1, 2, 3, int(rng.integers(1, 60000))]))
        dobj = int(rng.integers(0, xny + 1)) if xny else 0
        mut2 = int(rng.integers(0, dobj + 1)) if dobj else 0
        sect = dobj + mut2 + int(rng.integers(0, 8 * mut2 + 1)) if dobj else 0
        x = xny + int(rng.integers(0, 60000))
        out.append((xny, x, sect, mut2, dobj))
    return out


@needs_ref
@pytest.mark.parametrize("drfold", [8, 6, 10])
def test_models_bit_identical(drfold):
    host, ref = _host(), _ref()
    rng = np.random.default_rng(drfold)
    for f5 in _features(rng, 3000):
        f = Feat(*f5)
        want = np.zeros(6)
        ref.refh_models(np.array(f5, dtype=np.uint32), drfold, 20, want)
        got = [host.kssd_lm3ways_dist(C.byref(f), drfold), host.kssd_af_anib(C.byref(f), drfold),
               host.kssd_naive_dist(C.byref(f)), host.kssd_p_dist(C.byref(f), 20),
               host.kssd_mashD(22, f5[1], f5[0] + 7, f5[0]), host.kssd_aafD(22, f5[1], f5[0] + 7, f5[0])]
        for i, (g, w) in enumerate(zip(got, want)):
            assert _same(g, w), (i, f5, g, w)


@needs_ref
def test_hgb_calibration_bit_identical():
    host, ref = _host(), _ref()
    rng = np.random.default_rng(5)
    for _ in range(4000):
        xny = int(rng.integers(0, 40000))
        dobj = int(rng.integers(0, xny + 1)) if xny else 0
        mut2 = int(rng.integers(0, dobj + 1)) if dobj else 0
        sect = dobj + mut2 + int(rng.integers(0, 3 * mut2 + 1)) if dobj else 0
        raw = float(rng.choice([rng.uniform(0.6, 1.05), 1.0, 0.95, np.nan]))
        af = float(rng.choice([rng.uniform(-0.1, 1.1), 0.2, 0.5, 1.0, 1e-13]))
        for drf in (8, 9):
            g = host.kssd_hgb_predict_ani(raw, af, xny, dobj, sect, mut2, drf)
            w = ref.refh_hgb(raw, af, xny, dobj, sect, mut2, drf)
            assert _same(g, w), (raw, af, xny, dobj, sect, mut2, g, w)


def test_hgb_table_shape():
    src = os.path.join(os.path.dirname(kssdgpu.__file__), "host", "hgb_t11_model.c")
    text = open(src).read()
    assert text.count("\n    {") == 9760


class Opt(C.Structure):
    _fields_ = [("fmt", C.c_int), ("p", C.c_int), ("d", C.c_bool), ("v", C.c_bool), ("unassembled", C.c_bool),
                ("unified_metric", C.c_bool), ("ignoreconflict", C.c_bool), ("raw_output", C.c_bool),
                ("max_pdist_set", C.c_bool), ("max_pdist", C.c_double), ("max_diff_obj_section", C.c_int),
                ("e", C.c_int), ("s", C.c_int), ("ntop", C.c_int), ("ctxcut", C.c_int), ("afcut", C.c_float),
                ("afcut_set", C.c_bool), ("anicut", C.c_float), ("unique_ctx", C.c_bool), ("obj_bits", C.c_int),
                ("ctx_bits", C.c_int), ("drfold", C.c_int)]


def test_zero_overlap_constant_equals_full_evaluation():
    """The CLI's shortcut for pairs with no shared context gives exactly the value the
    full row evaluation gives, for every metric, sign, exception value and AF cut."""
    lib = _host()
    lib.kssd_opt_defaults.argtypes = [C.POINTER(Opt)]
    lib.kssd_zero_overlap_metric.argtypes = [C.POINTER(Opt), C.POINTER(C.c_double)]
    lib.kssd_zero_overlap_metric.restype = C.c_bool
    lib.kssd_pair_metric.argtypes = [C.POINTER(Feat), C.c_uint32, C.c_uint32, C.POINTER(Opt), C.c_void_p,
                                     C.c_void_p]
    lib.kssd_pair_metric.restype = C.c_double
    rng = np.random.default_rng(3)
    zero = Feat(0, 0, 0, 0, 0)
    for s in list(range(1, 10)) + list(range(-9, 0)):
        for afcut in (0.5, 0.2, 1e-6, 0.0):
            for flags in ((False, False, False), (True, True, False), (False, False, True)):
                o = Opt()
                lib.kssd_opt_defaults(C.byref(o))
                o.s, o.afcut, o.e = s, afcut, int(rng.integers(1, 3))
                o.v, o.unassembled, o.raw_output = flags
                const = C.c_double()
                ok = lib.kssd_zero_overlap_metric(C.byref(o), C.byref(const))
                assert ok == (afcut > 0)
                if not ok:
                    continue
                for _ in range(20):
                    qc, rc = (int(x) for x in rng.integers(1, 200000, size=2))
                    full = lib.kssd_pair_metric(C.byref(zero), qc, rc, C.byref(o), None, None)
                    assert _same(full, const.value), (s, afcut, flags, qc, rc, full, const.value)

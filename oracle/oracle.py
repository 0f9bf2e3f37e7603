"""ORACLE — test infrastructure only.

ctypes binding of the C restatement (oracle/liboracle.so, kssd_oracle.c) and of
the reference's own counting functions compiled from its sources
(oracle/_ref/refharness.so, ref_harness.c) plus the reference CLI
(oracle/_ref/kssd3a).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_BIN = os.path.join(REF_DIR, "kssd3a")

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_vp = C.c_void_p

_orc = None
_ref = None


def oracle_lib() -> C.CDLL:
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE}`")
        lib = C.CDLL(path)
        lib.orc_build_index.argtypes = [_u64p, _u64p, C.c_int, C.c_int, _vp]
        lib.orc_build_index.restype = C.c_size_t
        lib.orc_unique_bits.argtypes = [_vp, C.c_size_t, _vp]
        lib.orc_unique_bits.restype = C.c_uint64
        lib.orc_ref_ctx_counts.argtypes = [_vp, C.c_size_t, C.c_int, _u64p, C.c_int, C.c_int, _u32p]
        lib.orc_sample_ctx_counts.argtypes = [_u64p, _u64p, C.c_int, C.c_int, C.c_int, C.c_int, _u32p]
        lib.orc_unique_ref_totals.argtypes = [_vp, C.c_size_t, C.c_int, C.c_int, _u32p]
        lib.orc_count_block.argtypes = [_vp, C.c_size_t, C.c_int, _u64p, _u64p, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _vp, _vp, _vp, _vp]
        lib.orc_count_lower.argtypes = [_vp, C.c_size_t, C.c_int, C.c_int, _u64p, _u64p, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _vp, _vp]
        lib.orc_pair_features.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.c_int, C.c_int, _u32p]
        lib.orc_dna_popcount.argtypes = [C.c_uint32]
        lib.orc_self_votes.argtypes = [_vp, C.c_size_t, _u64p, _u64p, C.c_int, C.c_int, C.c_uint32, C.c_uint32,
                                       _u32p, _u32p]
        lib.orc_sketch_masks.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
        lib.orc_sketch_records.argtypes = [C.c_char_p, _u64p, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_int,
                                           C.c_uint32, C.c_int, _vp, C.c_size_t]
        lib.orc_sketch_records.restype = C.c_size_t
        _orc = lib
    return _orc


_work = None


def workload_lib() -> C.CDLL:
    """oracle/libworkload.so: the seeded synthetic-sketch generator built on its own
    (declare its entry points with kssdgpu.bind_synth before use)."""
    global _work
    if _work is None:
        path = os.path.join(HERE, "libworkload.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE}`")
        _work = C.CDLL(path)
    return _work


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "refharness.so")) and os.path.exists(REF_BIN)


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        path = os.path.join(REF_DIR, "refharness.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} missing: run `make -C {HERE} ref` where the reference sources exist")
        lib = C.CDLL(path)
        lib.refh_count_block.argtypes = [_vp, C.c_size_t, C.c_int, _u64p, _u64p, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int, _vp, _vp, _vp, _vp]
        lib.refh_count_lower.argtypes = [_vp, C.c_size_t, C.c_int, C.c_int, _u64p, _u64p, C.c_int, C.c_int,
                                         C.c_int, C.c_int, _vp, _vp]
        lib.refh_count_detail.argtypes = [_vp, C.c_size_t, C.c_int, _u64p, _u64p, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int, _u32p, _u32p, C.c_int, C.c_float, C.c_float,
                                          C.c_int, _vp, _vp, _vp, _vp, _u32p, _u32p]
        lib.refh_pair_features.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.c_int, C.c_int, _u32p]
        _ref = lib
    return _ref


REC_DTYPE = np.dtype([("ctxgid", "<u8"), ("obj", "<u4")])


def _rptr(rec):
    return rec.ctypes.data if len(rec) else None


def build_index(keys, offs, obj_bits=20):
    n = int(offs[-1] - offs[0])
    rec = np.zeros(max(n, 1), dtype=REC_DTYPE)
    got = oracle_lib().orc_build_index(np.ascontiguousarray(keys, np.uint64),
                                       np.ascontiguousarray(offs, np.uint64), len(offs) - 1, obj_bits,
                                       rec.ctypes.data)
    return rec[:got]


def unique_bits(rec):
    bits = np.zeros(max((len(rec) + 7) // 8, 1), dtype=np.uint8)
    oracle_lib().orc_unique_bits(_rptr(rec), len(rec), bits.ctypes.data)
    return bits[: (len(rec) + 7) // 8]


def ref_ctx_counts(rec, nref, ref_offs, conflict, ignoreconflict):
    out = np.zeros(nref, dtype=np.uint32)
    oracle_lib().orc_ref_ctx_counts(_rptr(rec), len(rec), nref, np.ascontiguousarray(ref_offs, np.uint64),
                                    int(conflict), int(ignoreconflict), out)
    return out


def sample_ctx_counts(keys, offs, obj_bits, conflict, ignoreconflict):
    out = np.zeros(len(offs) - 1, dtype=np.uint32)
    k = np.ascontiguousarray(keys, np.uint64)
    if len(k) == 0:
        k = np.zeros(1, np.uint64)
    oracle_lib().orc_sample_ctx_counts(k, np.ascontiguousarray(offs, np.uint64), len(offs) - 1, obj_bits,
                                       int(conflict), int(ignoreconflict), out)
    return out


def unique_ref_totals(rec, nref, ignoreconflict):
    out = np.zeros(nref, dtype=np.uint32)
    oracle_lib().orc_unique_ref_totals(_rptr(rec), len(rec), nref, int(ignoreconflict), out)
    return out


def _qk(qkeys):
    k = np.ascontiguousarray(qkeys, np.uint64)
    return k if len(k) else np.zeros(1, np.uint64)


def count_block(rec, nref, qkeys, qoffs, obj_bits=20, ignoreconflict=False, unique=False, threads=8, ref=False):
    """Counters [nq, nref, 2] x (ctx, obj[, uctx, uobj]); ref=True runs the reference's own function."""
    nq = len(qoffs) - 1
    outs = [np.zeros((nq, nref, 2), dtype=np.uint32) for _ in range(4 if unique else 2)]
    ptr = [o.ctypes.data for o in outs] + [None] * (4 - len(outs))
    fn = ref_lib().refh_count_block if ref else oracle_lib().orc_count_block
    fn(_rptr(rec), len(rec), nref, _qk(qkeys), np.ascontiguousarray(qoffs, np.uint64), nq, obj_bits,
       int(ignoreconflict), int(unique), threads, *ptr)
    return tuple(outs)


def count_lower(rec, nref, qgid_offset, qkeys, qoffs, obj_bits=20, ignoreconflict=False, threads=8, ref=False):
    nq = len(qoffs) - 1
    ctx = np.zeros((nq, nref, 2), dtype=np.uint32)
    obj = np.zeros((nq, nref, 2), dtype=np.uint32)
    fn = ref_lib().refh_count_lower if ref else oracle_lib().orc_count_lower
    fn(_rptr(rec), len(rec), nref, qgid_offset, _qk(qkeys), np.ascontiguousarray(qoffs, np.uint64), nq,
       obj_bits, int(ignoreconflict), threads, ctx.ctypes.data, obj.ctypes.data)
    return ctx, obj


def count_detail_ref(rec, nref, qkeys, qoffs, ref_ctx_count, qry_ctx_count, obj_bits=20, ignoreconflict=False,
                     unique=False, ctxcut=3, afcut=0.5, anicut=0.95, ntop=-1, threads=4):
    """The reference's detail-mode counting + pre-filter + ranking; returns (counters, num_pass, ranked ids)."""
    nq = len(qoffs) - 1
    outs = [np.zeros((nq, nref, 2), dtype=np.uint32) for _ in range(4)]
    num_pass = np.zeros(max(nq, 1), dtype=np.uint32)
    ranked = np.zeros(max(nq * nref, 1), dtype=np.uint32)
    ref_lib().refh_count_detail(_rptr(rec), len(rec), nref, _qk(qkeys), np.ascontiguousarray(qoffs, np.uint64),
                                nq, obj_bits, int(ignoreconflict), int(unique), threads,
                                np.ascontiguousarray(ref_ctx_count, np.uint32),
                                np.ascontiguousarray(qry_ctx_count, np.uint32), ctxcut, afcut, anicut, ntop,
                                outs[0].ctypes.data, outs[1].ctypes.data, outs[2].ctypes.data,
                                outs[3].ctypes.data, num_pass, ranked)
    return outs, num_pass[:nq], ranked[: nq * nref].reshape(nq, nref) if nq else ranked[:0]


def pair_features(a, b, obj_bits=20, ignore_b_conflict=False, ref=False):
    out = np.zeros(4, dtype=np.uint32)
    fn = ref_lib().refh_pair_features if ref else oracle_lib().orc_pair_features
    fn(_qk(a), len(a), _qk(b), len(b), obj_bits, int(ignore_b_conflict), out)
    return out


def self_lower_all(rec, sketch_keys, sketch_offs, obj_bits=20, ignoreconflict=False, threads=8):
    """Packed lower triangle (q*(q-1)/2 + r) of count_lower over all samples."""
    n = len(sketch_offs) - 1
    cells = n * (n - 1) // 2
    ctx = np.zeros((cells, 2), dtype=np.uint32)
    obj = np.zeros((cells, 2), dtype=np.uint32)
    block = 64
    for off in range(0, n, block):
        nb = min(block, n - off)
        qo = np.ascontiguousarray(sketch_offs[off: off + nb + 1], np.uint64)
        qk = sketch_keys[int(qo[0]): int(qo[-1])]
        c, o = count_lower(rec, n, off, qk, qo, obj_bits, ignoreconflict, threads)
        for i in range(nb):
            q = off + i
            if q == 0:
                continue
            base = q * (q - 1) // 2
            ctx[base: base + q] = c[i, :q]
            obj[base: base + q] = o[i, :q]
    return ctx, obj


def self_votes(rec, keys, offs, obj_bits=20, max_freq=256, step=1):
    """Sparse-scan candidate votes and first-touch order over the packed lower triangle."""
    n = len(offs) - 1
    cells = n * (n - 1) // 2
    votes = np.zeros(max(cells, 1), dtype=np.uint32)
    first = np.zeros(max(cells, 1), dtype=np.uint32)
    oracle_lib().orc_self_votes(_rptr(rec), len(rec), _qk(keys), np.ascontiguousarray(offs, np.uint64), n, obj_bits,
                                max_freq, step, votes, first)
    return votes[:cells], first[:cells]


def sketch_masks(coden_len=11, klen=32, hclen=0, holen=0):
    """(context mask, k-mer mask, object bits) of the sketch parameters."""
    cm, tm, ob = C.c_uint64(), C.c_uint64(), C.c_int()
    oracle_lib().orc_sketch_masks(coden_len, klen, hclen, holen, C.byref(cm), C.byref(tm), C.byref(ob))
    return cm.value, tm.value, ob.value


def sketch_records(records, klen=32, coden_len=11, hclen=0, holen=0, drfold=8, conflict=False):
    """One sample's sketch keys from its records' sequence bytes (the reference's sketcher,
    restated in liboracle)."""
    cm, tm, ob = sketch_masks(coden_len, klen, hclen, holen)
    seq = b"".join(records)
    offs = np.cumsum([0] + [len(r) for r in records]).astype(np.uint64)
    out = np.zeros(max(len(seq), 1), dtype=np.uint64)
    n = oracle_lib().orc_sketch_records(seq, offs, len(records), klen, cm, tm, ob, 0xFFFFFFFF >> drfold,
                                        1 if conflict else 0, out.ctypes.data, len(out))
    return out[:n].copy()

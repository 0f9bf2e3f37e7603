"""ctypes binding of libkssdgpu (include/kssdgpu.h) and libkssdhost (sketch I/O and
synthetic workloads), with numpy arrays on the host side and optional torch CUDA
tensors for the device-pointer calls.

The shared libraries are built in-tree (``make -C kssd3a-public_b200``).  There is
no fallback: loading fails loudly when they are missing, and every call checks
its status code and raises ``KssdGpuError`` with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

# flags (include/kssdgpu.h)
IGNORECONFLICT = 0x1
UNIQUE = 0x2
PLAIN = 0x4
GLOBAL_ACC = 0x8
NO_ZERO = 0x10
SMEM_ACC = 0x20
SELF_PLAN = 0x40
SELF_SCAN = 0x80
SELF_DENSE = 0x100
PATH_SCAN, PATH_DENSE, PATH_PLAN = 0, 1, 2

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class KssdGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"kssdgpu error {code}: {msg}")
        self.code = code


def _load(name: str) -> C.CDLL:
    path = os.path.join(LIBDIR, name)
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C {HERE}`")
    return C.CDLL(path)


_gpu = None
_host = None


def gpu_lib() -> C.CDLL:
    global _gpu
    if _gpu is None:
        lib = _load("libkssdgpu.so")
        vp = C.c_void_p
        lib.kssdgpu_last_error.restype = C.c_char_p
        lib.kssdgpu_launch_count.restype = C.c_uint64
        lib.kssdgpu_index_from_records.argtypes = [vp, C.c_uint64, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
        lib.kssdgpu_index_from_sketch.argtypes = [_u64p, _u64p, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
        lib.kssdgpu_index_free.argtypes = [vp]
        lib.kssdgpu_index_free.restype = None
        lib.kssdgpu_index_info.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.kssdgpu_index_export.argtypes = [vp, vp, vp]
        lib.kssdgpu_index_filter.argtypes = [vp, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_uint64)]
        lib.kssdgpu_index_ref_ctx_counts.argtypes = [vp, C.c_int, C.c_int, vp, vp]
        lib.kssdgpu_count_block.argtypes = [vp, vp, _u64p, C.c_int, C.c_uint, vp, vp, vp, vp]
        lib.kssdgpu_count_lower.argtypes = [vp, vp, _u64p, C.c_int, C.c_int, C.c_uint, vp, vp]
        lib.kssdgpu_count_detail.argtypes = [vp, vp, _u64p, C.c_int, C.c_uint, _u32p, _u32p, C.c_int, C.c_float,
                                             C.c_float, vp, C.c_uint64, _u64p]
        lib.kssdgpu_count_block_dev.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_uint,
                                                vp, vp, vp, vp, vp]
        lib.kssdgpu_sync.argtypes = [vp, vp]
        lib.kssdgpu_self_votes.argtypes = [vp, _u64p, _u64p, C.c_uint32, C.c_uint32, vp, vp]
        lib.kssdgpu_count_tune.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_uint, vp, vp, vp, vp,
                                           C.POINTER(_CountTuning)]
        lib.kssdgpu_self_lower.argtypes = [vp, C.c_uint, vp, vp]
        lib.kssdgpu_self_lower_dev.argtypes = [vp, C.c_uint, vp, vp, vp]
        lib.kssdgpu_self_choice.argtypes = [vp, C.c_uint, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        lib.kssdgpu_self_dense_alleles.argtypes = [vp, C.POINTER(C.c_uint64)]
        lib.kssdgpu_self_plan_tune.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_int), C.POINTER(C.c_uint32),
                                                 C.POINTER(C.c_int), C.POINTER(C.c_float)]
        lib.kssdgpu_self_plan_info.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                               C.POINTER(C.c_uint64)]
        lib.kssdgpu_count_plain_dev.argtypes = [vp, vp, vp, _u64p, C.c_int, C.c_int, C.c_int, C.c_uint,
                                                vp, vp, vp, vp, vp]
        lib.kssdgpu_init.argtypes = [C.c_int]
        lib.kssdgpu_server_create.argtypes = [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]
        lib.kssdgpu_server_submit.argtypes = [vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]
        lib.kssdgpu_server_wait.argtypes = [vp, C.c_uint64, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
        lib.kssdgpu_server_take.argtypes = [vp, C.c_uint64, vp, C.c_uint32]
        lib.kssdgpu_server_stats.argtypes = [vp, C.POINTER(_ServerStats)]
        lib.kssdgpu_server_reset_stats.argtypes = [vp]
        lib.kssdgpu_server_destroy.argtypes = [vp]
        lib.kssdgpu_server_destroy.restype = None
        lib.kssdgpu_sketch.argtypes = [C.c_char_p, C.c_uint64, _u64p, C.c_uint64, _u64p, C.c_int,
                                       C.POINTER(_SketchParams), vp, C.c_uint64, _u64p]
        lib.kssdgpu_sketch_hash_id.argtypes = [C.POINTER(_SketchParams)]
        lib.kssdgpu_sketch_hash_id.restype = C.c_uint32
        lib.kssdgpu_lower_metric_dev.argtypes = [C.c_int, C.POINTER(MetricOpt), C.c_int, vp, vp, vp, vp, vp, vp,
                                                 C.c_uint64, vp, vp]
        lib.kssdgpu_self_lower_metric.argtypes = [vp, C.c_uint, C.POINTER(MetricOpt), _u32p, _u32p, vp, vp,
                                                  C.c_uint64, C.POINTER(C.c_uint64)]
        _gpu = lib
    return _gpu


class MetricOpt(C.Structure):
    """kssdgpu_metric_opt_t: the options a matrix value reads, and the calibration trees."""
    _fields_ = [("s", C.c_int), ("e", C.c_int), ("v", C.c_int), ("unassembled", C.c_int),
                ("unified_metric", C.c_int), ("raw_output", C.c_int), ("afcut", C.c_float), ("drfold", C.c_int),
                ("obj_bits", C.c_int), ("ctx_bits", C.c_int), ("zero_const", C.c_int), ("zero_value", C.c_double),
                ("hgb_nodes", C.c_void_p), ("hgb_nodes_count", C.c_uint32), ("hgb_tree_begin", C.c_void_p),
                ("hgb_trees", C.c_uint32), ("hgb_baseline", C.c_double)]


RECHECK_DTYPE = np.dtype([("cell", "<u8"), ("num_ctx", "<u4"), ("num_mut2_ctx", "<u4"), ("diff_obj", "<u4"),
                          ("diff_obj_section", "<u4")])


def metric_opt(s=1, e=1, v=0, unassembled=0, unified_metric=0, raw_output=0, afcut=0.5, drfold=8, obj_bits=20,
               ctx_bits=44, zero_const=0, zero_value=0.0) -> MetricOpt:
    """Metric options with the calibration trees of the host library (its model tables)."""
    host = host_lib()
    trees, nodes = 160, 9760  # KSSD_HGB_TREES, KSSD_HGB_NODES
    begin = (C.c_uint * (trees + 1)).in_dll(host, "kssd_hgb_tree_begin")
    node_tab = (C.c_ubyte * (16 * nodes)).in_dll(host, "kssd_hgb_nodes")
    base = C.c_double.in_dll(host, "kssd_hgb_baseline").value
    return MetricOpt(s, e, v, unassembled, unified_metric, raw_output, afcut, drfold, obj_bits, ctx_bits, zero_const,
                     zero_value, C.addressof(node_tab), nodes, C.addressof(begin), trees, base)


def lower_metric_dev(opt: MetricOpt, n, d_qcnt, d_rcnt, d_lc, d_lo, d_val, d_recheck, cap, d_nrecheck, device=0,
                     stream=None):
    """kssdgpu_lower_metric_dev over device tensors (stream-ordered)."""
    ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
    _check(gpu_lib().kssdgpu_lower_metric_dev(device, C.byref(opt), n, ptr(d_qcnt), ptr(d_rcnt), ptr(d_lc),
                                              ptr(d_lo), ptr(d_val), ptr(d_recheck), cap, ptr(d_nrecheck),
                                              None if stream is None else stream.cuda_stream))


class _SketchParams(C.Structure):
    _fields_ = [("klen", C.c_int), ("coden_len", C.c_int), ("hclen", C.c_int), ("holen", C.c_int),
                ("drfold", C.c_int), ("conflict", C.c_int)]


def sketch(samples, klen=32, coden_len=11, hclen=0, holen=0, drfold=8, conflict=False):
    """Sketches on the device: samples is a list of samples, each a list of records'
    sequence bytes.  Returns (keys, offs) in the comblco / comblco.index layout."""
    recs = [r for smp in samples for r in smp]
    seq = b"".join(recs)
    rec_offs = np.cumsum([0] + [len(r) for r in recs]).astype(np.uint64)
    samp = np.cumsum([0] + [len(smp) for smp in samples]).astype(np.uint64)
    prm = _SketchParams(klen, coden_len, hclen, holen, drfold, 1 if conflict else 0)
    offs = np.zeros(len(samples) + 1, dtype=np.uint64)
    cap = max(1, len(seq) // max(1, 1 << min(drfold, 8)) + 1024)
    keys = np.zeros(cap, dtype=np.uint64)
    rc = gpu_lib().kssdgpu_sketch(seq, len(seq), rec_offs, len(recs), samp, len(samples), C.byref(prm),
                                  keys.ctypes.data, cap, offs)
    if rc == 7:  # capacity: offs holds the sizes
        keys = np.zeros(int(offs[-1]), dtype=np.uint64)
        rc = gpu_lib().kssdgpu_sketch(seq, len(seq), rec_offs, len(recs), samp, len(samples), C.byref(prm),
                                      keys.ctypes.data if len(keys) else None, len(keys), offs)
    _check(rc)
    return keys[:int(offs[-1])].copy(), offs


def sketch_hash_id(klen=32, coden_len=11, hclen=0, holen=0, drfold=8):
    return gpu_lib().kssdgpu_sketch_hash_id(C.byref(_SketchParams(klen, coden_len, hclen, holen, drfold, 0)))


class _ServerConfig(C.Structure):
    _fields_ = [("max_batch_queries", C.c_int), ("max_batch_keys", C.c_uint64), ("max_hits", C.c_uint64),
                ("flags", C.c_uint), ("slots", C.c_int), ("device_budget", C.c_uint64)]


class _CountTuning(C.Structure):
    _fields_ = [("smem_rows", C.c_int), ("chunk_keys", C.c_uint32), ("candidates", C.c_int), ("ms", C.c_float),
                ("filter", C.c_int), ("striped", C.c_int)]


class _ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("batches", C.c_uint64), ("pending", C.c_uint64),
                ("max_inflight", C.c_uint64), ("overlapped_batches", C.c_uint64), ("reserved_bytes", C.c_uint64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double), ("mean_ms", C.c_double),
                ("slots", C.c_uint64), ("splits", C.c_uint64)]


HIT_DTYPE = np.dtype([("query", "<u4"), ("ref", "<u4"), ("num_ctx", "<u4"), ("num_mut2_ctx", "<u4"),
                      ("diff_obj", "<u4"), ("diff_obj_section", "<u4"), ("u_num_ctx", "<u4"),
                      ("u_num_mut2_ctx", "<u4"), ("u_diff_obj", "<u4"), ("u_diff_obj_section", "<u4")])


class _SynthCfg(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("sample_seed", C.c_uint64), ("n_samples", C.c_int),
        ("n_clusters", C.c_int), ("role", C.c_int), ("size_dist", C.c_int),
        ("len_median", C.c_double), ("len_sigma", C.c_double), ("len_min", C.c_double),
        ("len_max", C.c_double), ("own_len_min", C.c_double), ("own_len_max", C.c_double),
        ("sub_lo", C.c_double), ("sub_hi", C.c_double),
        ("indel_rate", C.c_double), ("density", C.c_double), ("ctx_bits", C.c_int),
        ("obj_bits", C.c_int), ("klen", C.c_int), ("ref_sample_seed", C.c_uint64),
        ("ref_samples", C.c_int), ("reads_min_genomes", C.c_int), ("reads_max_genomes", C.c_int),
        ("cov_lo", C.c_double), ("cov_hi", C.c_double), ("err_lo", C.c_double),
        ("err_hi", C.c_double), ("threads", C.c_int),
    ]


class _SynthOut(C.Structure):
    _fields_ = [("n", C.c_int), ("keys", C.POINTER(C.c_uint64)), ("offs", C.POINTER(C.c_uint64)),
                ("lengths", C.POINTER(C.c_double))]


def host_lib() -> C.CDLL:
    global _host
    if _host is None:
        lib = _load("libkssdhost.so")
        lib.kssd_host_last_error.restype = C.c_char_p
        bind_synth(lib)
        _host = lib
    return _host


def bind_synth(lib: C.CDLL) -> C.CDLL:
    """Declares the generator's entry points (host/kssd_synth.h) on a loaded library."""
    lib.kssd_synth_default.argtypes = [C.POINTER(_SynthCfg)]
    lib.kssd_synth_default.restype = None
    lib.kssd_synth_generate.argtypes = [C.POINTER(_SynthCfg)]
    lib.kssd_synth_generate.restype = C.POINTER(_SynthOut)
    lib.kssd_synth_free.argtypes = [C.POINTER(_SynthOut)]
    lib.kssd_synth_free.restype = None
    return lib


def _check(rc: int):
    if rc != 0:
        raise KssdGpuError(rc, gpu_lib().kssdgpu_last_error().decode(errors="replace"))


def launch_count() -> int:
    """Kernels launched by libkssdgpu so far in this process."""
    return int(gpu_lib().kssdgpu_launch_count())


# ---------------------------------------------------------------- synthetic workloads

ROLE_MEMBER, ROLE_OWNLEN, ROLE_READS = 0, 1, 2
SIZE_FIXED, SIZE_LOGNORMAL, SIZE_LOGUNIFORM = 0, 1, 2


@dataclass
class Sketch:
    """A sketch in memory: comblco keys, comblco.index offsets, sample names."""
    keys: np.ndarray
    offs: np.ndarray
    names: list
    conflict: bool = False
    obj_bits: int = 20
    lengths: np.ndarray | None = None

    @property
    def n(self) -> int:
        return len(self.offs) - 1


def synth(lib: C.CDLL | None = None, **kw) -> Sketch:
    """Generate a synthetic sketch (see host/kssd_synth.h for the model and fields).
    lib: another build of the same generator, declared with bind_synth (default: the
    host library)."""
    prefix = kw.pop("name_prefix", None)
    lib = lib or host_lib()
    cfg = _SynthCfg()
    lib.kssd_synth_default(C.byref(cfg))
    for k, v in kw.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    out = lib.kssd_synth_generate(C.byref(cfg))
    if not out:
        raise ValueError("invalid synthetic workload configuration")
    try:
        n = out.contents.n
        offs = np.ctypeslib.as_array(out.contents.offs, shape=(n + 1,)).copy()
        keys = np.ctypeslib.as_array(out.contents.keys, shape=(max(int(offs[-1]), 1),))[: int(offs[-1])].copy()
        lengths = np.ctypeslib.as_array(out.contents.lengths, shape=(max(n, 1),))[:n].copy()
    finally:
        lib.kssd_synth_free(out)
    prefix = prefix or ("read" if cfg.role == ROLE_READS else "g")
    names = [f"{prefix}{i}" for i in range(n)]
    return Sketch(keys=keys, offs=offs, names=names, conflict=cfg.role == ROLE_READS,
                  obj_bits=cfg.obj_bits, lengths=lengths)


# ---------------------------------------------------------------- sketch directories

STAT_DTYPE = np.dtype([("hash_id", "<u4"), ("koc", "u1"), ("conflict", "u1"), ("pad", "V2"),
                       ("coden_len", "<i4"), ("klen", "<i4"), ("hclen", "<i4"), ("holen", "<i4"),
                       ("drfold", "<i4"), ("infile_num", "<i4")])
REC_DTYPE = np.dtype([("ctxgid", "<u8"), ("obj", "<u4")])  # packed 12 B
# infile_meta_t (src/global_basic.h:182-193): lcofiles.infilemeta records, 32 B
META_DTYPE = np.dtype([("total_length_bp", "<u8"), ("record_count", "<u4"), ("median_length_bp", "<u4"),
                       ("asm_level", "<f4"), ("length_cv", "<f4"), ("meta_fmt_version", "u1"), ("infile_fmt", "i1"),
                       ("create_type", "i1"), ("infile_flags", "u1"), ("pad", "V4")])
DEFAULT_HASH_ID = 1772583717  # the reference sketcher's id for its default coden/k=32/f8 pattern


def write_sketch_dir(path: str, sk: Sketch, coden_len: int = 11, klen: int = 32, drfold: int = 8,
                     hash_id: int = DEFAULT_HASH_ID, with_index: bool = False, meta: np.ndarray | None = None,
                     abundance: np.ndarray | None = None):
    """Write a sketch directory in the reference layout (lcofiles.stat, comblco, comblco.index);
    with_index also writes sortedcomb_ctxgid64obj32 and its unique_bits; meta (META_DTYPE,
    one record per sample) writes lcofiles.infilemeta; abundance (uint32 per key) writes
    comblco.a and marks the sketch as made with k-mer counting (koc)."""
    os.makedirs(path, exist_ok=True)
    st = np.zeros(1, dtype=STAT_DTYPE)
    st["hash_id"], st["koc"], st["conflict"] = hash_id, int(abundance is not None), int(sk.conflict)
    st["coden_len"], st["klen"], st["hclen"], st["holen"] = coden_len, klen, 0, 0
    st["drfold"], st["infile_num"] = drfold, sk.n
    names = b"".join(nm.encode()[:255].ljust(256, b"\0") for nm in sk.names)
    with open(os.path.join(path, "lcofiles.stat"), "wb") as f:
        f.write(st.tobytes() + names)
    sk.keys.astype("<u8").tofile(os.path.join(path, "comblco"))
    sk.offs.astype("<u8").tofile(os.path.join(path, "comblco.index"))
    if abundance is not None:
        assert len(abundance) == len(sk.keys)
        abundance.astype("<u4").tofile(os.path.join(path, "comblco.a"))
    if meta is not None:
        assert meta.dtype == META_DTYPE and len(meta) == sk.n
        meta.tofile(os.path.join(path, "lcofiles.infilemeta"))
    if with_index:
        recs = build_records_np(sk)
        recs.tofile(os.path.join(path, "sortedcomb_ctxgid64obj32"))
        unique_bits_np(recs).tofile(os.path.join(path, "sortedcomb_ctxgid64obj32.unique_bits"))


def read_sketch_dir(path: str) -> Sketch:
    raw = open(os.path.join(path, "lcofiles.stat"), "rb").read()
    st = np.frombuffer(raw[:32], dtype=STAT_DTYPE)[0]
    n = int(st["infile_num"])
    names = [raw[32 + 256 * i: 32 + 256 * (i + 1)].split(b"\0")[0].decode(errors="replace") for i in range(n)]
    offs = np.fromfile(os.path.join(path, "comblco.index"), dtype="<u8")[: n + 1].astype(np.uint64)
    keys = np.fromfile(os.path.join(path, "comblco"), dtype="<u8").astype(np.uint64)
    ctx_bits = 4 * int(st["coden_len"]) if st["coden_len"] > 0 else 4 * int(st["hclen"])
    return Sketch(keys=keys, offs=offs, names=names, conflict=bool(st["conflict"]),
                  obj_bits=2 * int(st["klen"]) - ctx_bits)


def read_index_records(path: str) -> np.ndarray:
    return np.fromfile(os.path.join(path, "sortedcomb_ctxgid64obj32"), dtype=REC_DTYPE)


def build_records_np(sk: Sketch) -> np.ndarray:
    """Reference index records of a sketch, built with numpy (host helper for fixtures)."""
    counts = np.diff(sk.offs).astype(np.int64)
    gid = np.repeat(np.arange(sk.n, dtype=np.uint64), counts)
    ctxgid = ((sk.keys >> np.uint64(sk.obj_bits)) << np.uint64(20)) | gid
    obj = (sk.keys & np.uint64((1 << sk.obj_bits) - 1)).astype(np.uint32)
    order = np.lexsort((obj, ctxgid))
    rec = np.zeros(len(order), dtype=REC_DTYPE)
    rec["ctxgid"] = ctxgid[order]
    rec["obj"] = obj[order]
    return rec


def unique_bits_np(rec: np.ndarray) -> np.ndarray:
    ctx = rec["ctxgid"] >> np.uint64(20)
    key = np.stack([ctx, rec["obj"].astype(np.uint64)], axis=1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    uniq = cnt[inv.ravel()] == 1
    return np.packbits(uniq.astype(np.uint8), bitorder="little")


# ---------------------------------------------------------------- index and counting


class Index:
    """Device-resident CSR of a reference index (opaque libkssdgpu handle)."""

    def __init__(self, handle: int, nref: int, obj_bits: int):
        self._h = C.c_void_p(handle)
        self.nref = nref
        self.obj_bits = obj_bits

    @classmethod
    def from_records(cls, records: np.ndarray, nref: int, obj_bits: int = 20, device: int = 0) -> "Index":
        rec = np.ascontiguousarray(records)
        if rec.dtype.itemsize != 12:
            raise ValueError("records must be packed 12-byte {u64 ctxgid; u32 obj}")
        h = C.c_void_p()
        _check(gpu_lib().kssdgpu_index_from_records(rec.ctypes.data if len(rec) else None, len(rec),
                                                    nref, obj_bits, device, C.byref(h)))
        return cls(h.value, nref, obj_bits)

    @classmethod
    def from_sketch(cls, sk: Sketch, device: int = 0) -> "Index":
        h = C.c_void_p()
        keys = np.ascontiguousarray(sk.keys, dtype=np.uint64)
        if len(keys) == 0:
            keys = np.zeros(1, dtype=np.uint64)
        _check(gpu_lib().kssdgpu_index_from_sketch(keys, np.ascontiguousarray(sk.offs, dtype=np.uint64),
                                                   sk.n, sk.obj_bits, device, C.byref(h)))
        return cls(h.value, sk.n, sk.obj_bits)

    def close(self):
        if self._h and self._h.value:
            gpu_lib().kssdgpu_index_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        r, u, n, o = C.c_uint64(), C.c_uint64(), C.c_int(), C.c_int()
        _check(gpu_lib().kssdgpu_index_info(self._h, C.byref(r), C.byref(u), C.byref(n), C.byref(o)))
        return dict(records=r.value, contexts=u.value, nref=n.value, obj_bits=o.value)

    def filter(self, max_stripe_bytes: int = 0):
        """Rebuild the context membership filter with key-range stripes of at most
        max_stripe_bytes (0: the default); returns its stripe count and bytes."""
        n, b = C.c_int(), C.c_uint64()
        _check(gpu_lib().kssdgpu_index_filter(self._h, max_stripe_bytes, C.byref(n), C.byref(b)))
        return dict(stripes=n.value, bytes=b.value)

    def export(self):
        info = self.info()
        rec = np.zeros(info["records"], dtype=REC_DTYPE)
        bits = np.zeros((info["records"] + 7) // 8, dtype=np.uint8)
        _check(gpu_lib().kssdgpu_index_export(self._h, rec.ctypes.data if len(rec) else None,
                                              bits.ctypes.data if len(bits) else None))
        return rec, bits

    def ref_ctx_counts(self, conflict: bool, ignoreconflict: bool):
        c = np.zeros(self.nref, dtype=np.uint32)
        u = np.zeros(self.nref, dtype=np.uint32)
        _check(gpu_lib().kssdgpu_index_ref_ctx_counts(self._h, int(conflict), int(ignoreconflict),
                                                      c.ctypes.data, u.ctypes.data))
        return c, u

    def count_block(self, qkeys: np.ndarray, qoffs: np.ndarray, flags: int = 0):
        """Returns (ctx, obj[, uctx, uobj]) as uint32 arrays of shape [nq, nref, 2]."""
        nq = len(qoffs) - 1
        qk = np.ascontiguousarray(qkeys, dtype=np.uint64)
        qo = np.ascontiguousarray(qoffs, dtype=np.uint64)
        outs = [np.zeros((nq, self.nref, 2), dtype=np.uint32) for _ in range(4 if flags & UNIQUE else 2)]
        ptr = [o.ctypes.data for o in outs] + [None] * (4 - len(outs))
        _check(gpu_lib().kssdgpu_count_block(self._h, qk.ctypes.data if len(qk) else None, qo, nq, flags, *ptr))
        return tuple(outs)

    def count_lower(self, qkeys: np.ndarray, qoffs: np.ndarray, qry_gid_offset: int, flags: int = 0):
        nq = len(qoffs) - 1
        qk = np.ascontiguousarray(qkeys, dtype=np.uint64)
        qo = np.ascontiguousarray(qoffs, dtype=np.uint64)
        ctx = np.zeros((nq, self.nref, 2), dtype=np.uint32)
        obj = np.zeros((nq, self.nref, 2), dtype=np.uint32)
        _check(gpu_lib().kssdgpu_count_lower(self._h, qk.ctypes.data if len(qk) else None, qo, nq,
                                             qry_gid_offset, flags, ctx.ctypes.data, obj.ctypes.data))
        return ctx, obj

    def count_detail(self, qkeys: np.ndarray, qoffs: np.ndarray, qry_ctx_count, ref_ctx_count, flags: int = 0,
                     ctxcut: int = 3, afcut: float = 0.5, anicut: float = 0.95, cap: int = 1 << 20):
        """Detail-mode candidates filtered on the device: (hits HIT_DTYPE array ascending
        (query, ref), row_offs [nq + 1])."""
        nq = len(qoffs) - 1
        qk = np.ascontiguousarray(qkeys, dtype=np.uint64)
        qo = np.ascontiguousarray(qoffs, dtype=np.uint64)
        qc = np.ascontiguousarray(qry_ctx_count, dtype=np.uint32)
        rc_ = np.ascontiguousarray(ref_ctx_count, dtype=np.uint32)
        row_offs = np.zeros(nq + 1, dtype=np.uint64)
        hits = np.zeros(max(cap, 1), dtype=HIT_DTYPE)
        rc = gpu_lib().kssdgpu_count_detail(self._h, qk.ctypes.data if len(qk) else None, qo, nq, flags, qc, rc_,
                                            ctxcut, afcut, anicut, hits.ctypes.data, cap, row_offs)
        if rc == 7 and row_offs[-1] > cap:  # more candidates than the guess: the call reported how many
            return self.count_detail(qkeys, qoffs, qry_ctx_count, ref_ctx_count, flags, ctxcut, afcut, anicut,
                                     int(row_offs[-1]))
        _check(rc)
        return hits[: int(row_offs[-1])], row_offs

    def self_lower(self, flags: int = 0):
        """Packed lower triangle: arrays [nref*(nref-1)/2, 2] of (num_ctx, mut2) and (diff_obj, section)."""
        cells = self.nref * (self.nref - 1) // 2
        ctx = np.zeros((max(cells, 1), 2), dtype=np.uint32)
        obj = np.zeros((max(cells, 1), 2), dtype=np.uint32)
        _check(gpu_lib().kssdgpu_self_lower(self._h, flags, ctx.ctypes.data, obj.ctypes.data))
        return ctx[:cells], obj[:cells]

    # device-pointer forms (torch tensors or raw ints)
    def count_block_dev(self, d_keys, d_offs, nq, d_ctx, d_obj, d_uctx=None, d_uobj=None, flags=0,
                        lower=False, qry_gid_offset=0, stream=None):
        _check(gpu_lib().kssdgpu_count_block_dev(self._h, _ptr(d_keys), _ptr(d_offs), nq, qry_gid_offset,
                                                 int(lower), flags, _ptr(d_ctx), _ptr(d_obj), _ptr(d_uctx),
                                                 _ptr(d_uobj), _ptr(stream)))

    def count_tune(self, d_keys, d_offs, nq, d_ctx, d_obj, d_uctx=None, d_uobj=None, flags=0, lower=False,
                   qry_gid_offset=0):
        """Autotune this index's batched count on a block; returns the chosen setting."""
        t = _CountTuning()
        _check(gpu_lib().kssdgpu_count_tune(self._h, _ptr(d_keys), _ptr(d_offs), nq, qry_gid_offset, int(lower),
                                            flags, _ptr(d_ctx), _ptr(d_obj), _ptr(d_uctx), _ptr(d_uobj),
                                            C.byref(t)))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def count_plain_dev(self, d_keys, d_offs, h_offs, d_ctx, d_obj, d_uctx=None, d_uobj=None, flags=0,
                        lower=False, qry_gid_offset=0, stream=None):
        h = np.ascontiguousarray(h_offs, dtype=np.uint64)
        _check(gpu_lib().kssdgpu_count_plain_dev(self._h, _ptr(d_keys), _ptr(d_offs), h, len(h) - 1,
                                                 qry_gid_offset, int(lower), flags, _ptr(d_ctx), _ptr(d_obj),
                                                 _ptr(d_uctx), _ptr(d_uobj), _ptr(stream)))

    def self_votes(self, keys: np.ndarray, offs: np.ndarray, max_ctx_freq: int = 256, sample_step: int = 1):
        """Sparse-scan candidate votes and first-touch positions over the packed lower triangle."""
        n = self.nref
        cells = n * (n - 1) // 2
        votes = np.zeros(max(cells, 1), dtype=np.uint32)
        first = np.zeros(max(cells, 1), dtype=np.uint32)
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        _check(gpu_lib().kssdgpu_self_votes(self._h, k if len(k) else np.zeros(1, np.uint64),
                                            np.ascontiguousarray(offs, dtype=np.uint64), max_ctx_freq, sample_step,
                                            votes.ctypes.data, first.ctypes.data))
        return votes[:cells], first[:cells]

    def self_plan_tune(self):
        """Autotune the self-join plan (once per index); returns the setting in use."""
        c, so, f, n, ms = C.c_uint32(), C.c_int(), C.c_uint32(), C.c_int(), C.c_float()
        _check(gpu_lib().kssdgpu_self_plan_tune(self._h, C.byref(c), C.byref(so), C.byref(f), C.byref(n),
                                                C.byref(ms)))
        return dict(chunk_groups=c.value, sorted=bool(so.value), flat_groups=f.value, candidates=n.value,
                    step_ms=ms.value)

    def dense_alleles(self) -> int:
        """Allele rows (the GEMM's K before padding) of the last dense self join."""
        a = C.c_uint64()
        _check(gpu_lib().kssdgpu_self_dense_alleles(self._h, C.byref(a)))
        return a.value

    def self_choice(self, flags: int = 0):
        """(path the self join takes for these flags: PATH_*, the index's shared-context density)."""
        p, d = C.c_int(), C.c_double()
        _check(gpu_lib().kssdgpu_self_choice(self._h, flags, C.byref(p), C.byref(d)))
        return p.value, d.value

    def self_plan_info(self):
        g, p, q = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(gpu_lib().kssdgpu_self_plan_info(self._h, C.byref(g), C.byref(p), C.byref(q)))
        return dict(groups=g.value, postings=p.value, pairs=q.value)

    def self_lower_dev(self, d_ctx, d_obj, flags=0, stream=None):
        _check(gpu_lib().kssdgpu_self_lower_dev(self._h, flags, _ptr(d_ctx), _ptr(d_obj), _ptr(stream)))

    def sync(self, stream=None):
        _check(gpu_lib().kssdgpu_sync(self._h, _ptr(stream)))


class Server:
    """Continuous-batching query server over a resident Index (libkssdgpu kssdgpu_server_*)."""

    def __init__(self, index: Index, max_batch_queries=256, max_batch_keys=1 << 26, max_hits=0, flags=0, slots=0,
                 device_budget=0):
        self.index = index  # keep the index alive
        cfg = _ServerConfig(max_batch_queries, max_batch_keys, max_hits, flags, slots, device_budget)
        h = C.c_void_p()
        _check(gpu_lib().kssdgpu_server_create(index.handle, C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, keys: np.ndarray) -> int:
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        t = C.c_uint64()
        _check(gpu_lib().kssdgpu_server_submit(self._h, k.ctypes.data if len(k) else None, len(k), C.byref(t)))
        return t.value

    def result(self, ticket: int, timeout_ms: int = -1):
        """(hits structured array sorted by ref, latency ms)."""
        n, lat = C.c_uint32(), C.c_double()
        _check(gpu_lib().kssdgpu_server_wait(self._h, ticket, timeout_ms, C.byref(n), C.byref(lat)))
        hits = np.zeros(max(n.value, 1), dtype=HIT_DTYPE)
        _check(gpu_lib().kssdgpu_server_take(self._h, ticket, hits.ctypes.data, n.value))
        return hits[: n.value], lat.value

    def stats(self):
        st = _ServerStats()
        _check(gpu_lib().kssdgpu_server_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def reset_stats(self):
        _check(gpu_lib().kssdgpu_server_reset_stats(self._h))

    def close(self):
        if self._h and self._h.value:
            gpu_lib().kssdgpu_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "cuda_stream"):
        return x.cuda_stream
    raise TypeError(type(x))

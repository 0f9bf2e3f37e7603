"""Command-line parity cases shared by tests/test_gpu_cli.py and tests/golden/make_golden.py.

Each case names seeded synthetic sketch directories (generated on demand by the host
library's sketch-space generator) and a `kssd3a` command line; the reference CLI and
bin/kssd3a must print the same bytes.  The cases walk the reference dispatcher
(src/command_ani_wrapper.c:1082-1230): indexed mem_eff detail/matrix, one- and
multi-query streams, the no-index hash path, direct and indexed self matrices and
triangles, the rectangular direct matrix, read sets with --unique-ctx; and the
`matrix` command's one-sketch full/triangle and rectangular full reports.
"""
import os
import shutil

import kssdgpu

FIXTURES = {
    # 120 references: above the auto-index threshold (100) for detail output
    "refs120": dict(n_samples=120, n_clusters=12, len_median=3e5, len_sigma=0.3, len_min=1e5, len_max=8e5,
                    size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.06, seed=11, sample_seed=11),
    "qry30": dict(n_samples=30, n_clusters=12, role=kssdgpu.ROLE_OWNLEN, len_median=3e5, len_sigma=0.3,
                  len_min=1e5, len_max=8e5, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=9e5,
                  sub_lo=0.001, sub_hi=0.06, seed=11, sample_seed=12, name_prefix="q"),
    "refs40": dict(n_samples=40, n_clusters=5, len_median=2e5, len_sigma=0.3, len_min=1e5, len_max=6e5,
                   size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.04, seed=21, sample_seed=21),
    "qry1": dict(n_samples=1, n_clusters=5, role=kssdgpu.ROLE_OWNLEN, len_median=2e5, len_sigma=0.3, len_min=1e5,
                 len_max=6e5, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=1.5e5, own_len_max=3e5, sub_lo=0.002,
                 sub_hi=0.01, seed=21, sample_seed=22, name_prefix="one"),
    "qry8": dict(n_samples=8, n_clusters=5, role=kssdgpu.ROLE_OWNLEN, len_median=2e5, len_sigma=0.3, len_min=1e5,
                 len_max=6e5, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=4e5, sub_lo=0.001,
                 sub_hi=0.03, seed=21, sample_seed=23, name_prefix="few"),
    "qry50": dict(n_samples=50, n_clusters=5, role=kssdgpu.ROLE_OWNLEN, len_median=2e5, len_sigma=0.3,
                  len_min=1e5, len_max=6e5, size_dist=kssdgpu.SIZE_LOGNORMAL, own_len_min=5e4, own_len_max=4e5,
                  sub_lo=0.001, sub_hi=0.03, seed=21, sample_seed=24, name_prefix="many"),
    "reads1": dict(n_samples=1, n_clusters=12, role=kssdgpu.ROLE_READS, len_median=3e5, len_sigma=0.3,
                   len_min=1e5, len_max=8e5, size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.06, seed=11,
                   sample_seed=37, ref_sample_seed=11, ref_samples=120, cov_lo=10, cov_hi=30, err_lo=0.001,
                   err_hi=0.003, name_prefix="single"),
    "reads6": dict(n_samples=6, n_clusters=12, role=kssdgpu.ROLE_READS, len_median=3e5, len_sigma=0.3,
                   len_min=1e5, len_max=8e5, size_dist=kssdgpu.SIZE_LOGNORMAL, sub_lo=0.001, sub_hi=0.06, seed=11,
                   sample_seed=31, ref_sample_seed=11, ref_samples=120, cov_lo=5, cov_hi=20, err_lo=0.001,
                   err_hi=0.005, name_prefix="reads"),
}
INDEXED = {"refs120i", "refs120im", "refs40i", "refs40c9i"}  # with sortedcomb_ctxgid64obj32 written up front
WITH_META = {"refs120im", "refs40m"}  # with lcofiles.infilemeta (per-sample input metadata)
WITH_COUNTS = {"reads6a", "reads1a"}  # sketched with k-mer counts: comblco.a
# sketched at 9 or 10 codens (k = 26 / 29): 36- / 40-bit contexts, 16- / 18-bit objects
# (the reference reads the object width of every sketch from its lcofiles.stat)
CODENS = {"refs40c9": (9, 26), "refs40c9i": (9, 26), "qry8c9": (9, 26), "qry50c9": (9, 26),
          "refs40c10": (10, 29), "qry8c10": (10, 29)}


def synth_counts(sk, seed):
    """Seeded per-key k-mer counts: a depth per sample, Poisson-like spread, some singletons."""
    import numpy as np
    rng = np.random.default_rng(seed)
    depth = np.repeat(rng.integers(3, 60, sk.n), np.diff(sk.offs).astype(np.int64))
    counts = rng.poisson(depth).astype(np.uint32)
    counts[rng.random(len(counts)) < 0.1] = 1
    return np.maximum(counts, 1)


def synth_meta(sk, seed):
    """Seeded per-sample input metadata (some records invalid, some FASTQ, ties on purpose)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    m = np.zeros(sk.n, dtype=kssdgpu.META_DTYPE)
    m["total_length_bp"] = (sk.lengths // 1000 * 1000).astype(np.uint64)  # ties between samples
    m["record_count"] = rng.choice([0, 1, 2, 5, 40], sk.n)
    m["median_length_bp"] = rng.choice([5000, 20000, 100000], sk.n)
    m["asm_level"] = rng.choice([1.0, 2.0, 3.0, np.nan], sk.n).astype(np.float32)
    m["length_cv"] = rng.choice([0.1, 0.5, np.inf], sk.n).astype(np.float32)
    m["meta_fmt_version"] = rng.choice([1, 1, 1, 0], sk.n)
    m["infile_fmt"] = rng.choice([1, 1, 2], sk.n)
    return m

# (case name, argv after `kssd3a`, extra environment)
CASES = [
    ("memeff_detail", ["ani", "-r", "{refs120}", "-q", "{qry30}"], {}),
    ("memeff_detail_top3", ["ani", "-r", "{refs120}", "-q", "{qry30}", "-N", "3", "-n", "0.9", "-f", "0.3"], {}),
    ("memeff_detail_metrics", ["ani", "-r", "{refs120}", "-q", "{qry30}", "--metric", "p_dist", "-n", "0.5"], {}),
    ("memeff_detail_moe_raw", ["ani", "-r", "{refs120}", "-q", "{qry30}", "-s", "3", "--raw-output", "-t", "10"], {}),
    ("memeff_detail_close", ["ani", "-r", "{refs120}", "-q", "{qry30}", "--max-pdist", "0.02", "-n", "0.8"], {}),
    ("memeff_detail_naive", ["ani", "-r", "{refs120}", "-q", "{qry30}", "-v"], {}),
    ("memeff_matrix_ani", ["ani", "-r", "{refs120}", "-q", "{qry30}", "--format", "matrix", "--values", "ani"],
     {"KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD": "0"}),
    ("rect_matrix_direct", ["ani", "-r", "{refs40}", "-q", "{qry8}", "--format", "matrix"], {}),
    ("rect_matrix_ani_direct", ["ani", "-r", "{refs40}", "-q", "{qry50}", "--format", "matrix", "-s", "-5"], {}),
    ("stream_one", ["ani", "-r", "{refs40}", "-q", "{qry1}", "-n", "0.9"], {}),
    ("stream_multi", ["ani", "-r", "{refs40}", "-q", "{qry8}", "-n", "0.9", "-N", "4"], {}),
    ("hash_detail", ["ani", "-r", "{refs40}", "-q", "{qry50}", "-n", "0.9"], {}),
    ("self_full_direct", ["ani", "-q", "{refs120}", "--format", "matrix", "--values", "ani"], {}),
    ("self_full_indexed", ["ani", "-q", "{refs120}", "--format", "matrix", "--values", "ani"],
     {"KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD": "0"}),
    ("self_full_indexed_dist", ["ani", "-q", "{refs40}", "-m1"], {"KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD": "0"}),
    ("self_triangle_direct", ["ani", "-q", "{refs40}", "-m2", "-d", "-s", "-1"], {}),
    ("self_triangle_indexed", ["ani", "-q", "{refs120}", "-m2"], {"KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD": "0"}),
    # self matrices whose values come from log / pow (Naive, Mash, AAF): the device's
    # FP64 epilogue hands cells next to a rounding boundary to the host
    ("self_full_indexed_naive_ani", ["ani", "-q", "{refs120}", "--format", "matrix", "-s", "-4"],
     {"KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD": "0"}),
    ("self_full_mash", ["ani", "-q", "{refs120}", "--format", "matrix", "-s", "5"], {}),
    ("self_triangle_aaf_ani", ["ani", "-q", "{refs40}", "-m2", "-s", "-6"], {}),
    ("self_matrix_reads_ignoreconflict", ["ani", "-q", "{reads6}", "--format", "matrix", "--values", "ani",
                                          "--ignoreconflict"], {}),
    ("reads_qraw", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.8"], {}),
    ("reads_qraw_unique", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.95", "--unique-ctx"], {}),
    ("reads_qraw_ignoreconflict", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.5", "--ignoreconflict"],
     {}),
    ("reads_qraw_stream", ["ani", "-r", "{refs120}", "--qraw", "{reads6}", "-n", "0.5"], {}),
    # `kssd3a matrix`: one-sketch full/triangle (indexed self path) and rectangular full (per-pair path)
    ("matrix_triangle", ["matrix", "{refs40}"], {}),
    ("matrix_triangle_d_mash", ["matrix", "-q", "{refs120}", "--format", "triangle", "-d", "-m", "mash"], {}),
    ("matrix_full_moe", ["matrix", "--format", "full", "-m", "ctx-moe", "{refs40}"], {}),
    ("matrix_full_phylip_pdist", ["matrix", "--format", "full", "--matrix-format", "phylip", "-m", "p_dist",
                                  "{refs120i}"], {}),
    ("matrix_full_diag_value", ["matrix", "--format", "full", "--diagonal-value", "0.5", "-m", "1", "{refs40}"], {}),
    ("matrix_rect_aaf", ["matrix", "-r", "{refs40}", "-q", "{qry8}", "-m", "aaf"], {}),
    ("matrix_rect_naive_e2", ["matrix", "-r", "{refs120}", "-q", "{qry30}", "-e", "2"], {}),
    ("matrix_reads_triangle", ["matrix", "-m", "ctx-moe", "-d", "{reads6}"], {}),
    ("matrix_full_phylip_idmap", ["matrix", "--format", "full", "--matrix-format", "phylip", "--matrix-idmap",
                                  "{out:ids.tsv}", "{refs40}"], {}),
    # sparse reports: indexed scan (index file, conflict-free), direct pairs, -r/-q edges.
    # The reference's indexed scan emits rows from several threads in any order: those
    # cases compare the sorted lines ("_sorted").
    ("matrix_edges_indexed", ["matrix", "--format", "edges", "--cut", "0.05", "{refs120i}"], {"_sorted": "1"}),
    ("matrix_edges_indexed_votes", ["matrix", "--sparse", "--cut", "0.2", "--index-max-ctx-freq", "3",
                                    "--index-min-votes", "2", "--index-sample-step", "2", "-m", "ctx-moe",
                                    "{refs120i}"], {"_sorted": "1"}),
    ("matrix_edges_direct_expr", ["matrix", "--format", "edges", "--cut", "0.1", "-m", "ctx-naive&aaf",
                                  "--ctxcut", "50", "{refs40}"], {}),
    ("matrix_edges_rect_or", ["matrix", "-r", "{refs40}", "-q", "{qry8}", "--format", "edges", "--cut", "0.3",
                              "-m", "mash|p_dist", "--max-afcut", "0.2"], {}),
    ("matrix_clusters_indexed", ["matrix", "--format", "clusters", "--cut", "0.05", "--edge-out",
                                 "{out:edges.tsv}", "-g", "{out:glist.tsv}", "{refs120im}"], {"_sorted_out": "edges.tsv"}),
    ("matrix_clusters_direct", ["matrix", "--format", "clusters", "--cut", "0.08", "-m", "p_dist",
                                "--edge-out", "{out:edges.tsv}", "{refs40m}"], {}),
    ("matrix_dedup_greedy", ["matrix", "--format", "dedup-plan", "--cut", "0.05", "--keep-out", "{out:keep.txt}",
                             "--remove-out", "{out:remove.txt}", "--keep-matrix-out", "{out:keep.tsv}",
                             "{refs120im}"], {}),
    ("matrix_dedup_full_phylip", ["matrix", "--format", "dedup-plan", "--dedup-strategy", "full-linkage", "--cut",
                                  "0.08", "--max-afcut", "0.5", "--keep-matrix-out", "{out:keep.phy}",
                                  "--keep-matrix-format", "phylip", "--keep-matrix-idmap", "{out:keep.idmap}",
                                  "--edge-out", "{out:edges.tsv}", "{refs40m}"], {}),
    ("matrix_dedup_reads", ["matrix", "--format", "dedup-plan", "--cut", "0.5", "-m", "mash", "{reads6}"], {}),
    ("matrix_query_list", ["matrix", "-r", "{refs40}", "--query-sketch-list", "{list:qry8,qry1}", "-m", "ctx-moe"],
     {}),
    # the dispatcher's environment switches (src/command_ani_wrapper.c:1082-1230)
    ("env_force_ref_index_one", ["ani", "-r", "{refs40i}", "-q", "{qry1}", "-n", "0.9"],
     {"KSSD3A_FORCE_REF_INDEX": "1"}),
    ("env_qraw_lookup_sorted", ["ani", "-r", "{refs120i}", "--qraw", "{reads1}", "-n", "0.5"],
     {"KSSD3A_QRAW_LOOKUP": "sorted"}),
    ("env_qraw_multi_legacy", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.5", "-N", "4"],
     {"KSSD3A_QRAW_MULTI": "legacy"}),
    ("env_qraw_multi_sortedindex", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.5", "-N", "4"],
     {"KSSD3A_QRAW_MULTI": "sortedindex"}),
    ("env_multi_threshold", ["ani", "-r", "{refs40}", "-q", "{qry8}", "-n", "0.9"],
     {"KSSD3A_QRAW_MULTI_THRESHOLD": "3"}),
    ("env_no_auto_index", ["ani", "-r", "{refs120}", "-q", "{qry30}", "-n", "0.9"],
     {"KSSD3A_AUTO_REF_INDEX_THRESHOLD": "0"}),
    # --estimate-coverage on read sets with k-mer counts: mem_eff with the reference
    # database's marker bits, the multi-query stream (markers among reported rows), the
    # one-query stream, and a query without counts
    ("reads_coverage_memeff", ["ani", "-r", "{refs120i}", "--qraw", "{reads6a}", "-n", "0.8",
                               "--estimate-coverage"], {}),
    ("reads_coverage_stream_multi", ["ani", "-r", "{refs120}", "--qraw", "{reads6a}", "-n", "0.5", "-N", "5",
                                     "--estimate-coverage"], {}),
    ("reads_coverage_stream_one", ["ani", "-r", "{refs120i}", "--qraw", "{reads1a}", "-n", "0.5",
                                   "--estimate-coverage"], {}),
    ("reads_coverage_no_counts", ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n", "0.8",
                                  "--estimate-coverage"], {}),
    # sketches of 9 and 10 codens: narrower objects (p_dist divides by the object width)
    ("codens9_memeff_detail", ["ani", "-r", "{refs40c9i}", "-q", "{qry50c9}", "-n", "0.5"], {}),
    ("codens9_stream_pdist", ["ani", "-r", "{refs40c9}", "-q", "{qry8c9}", "--metric", "p_dist", "-n", "0.3"], {}),
    ("codens9_self_matrix", ["ani", "-q", "{refs40c9i}", "--format", "matrix", "--values", "ani"], {}),
    ("codens10_stream_detail", ["ani", "-r", "{refs40c10}", "-q", "{qry8c10}", "-n", "0.5", "-v"], {}),
    ("codens10_matrix_triangle", ["matrix", "--format", "triangle", "{refs40c10}"], {}),
]


# Cases run by the 9- and 10-coden builds (build/codens9, build/codens10) against the
# reference compiled the same way (-DNUM_CODENS=9 / 10: the other lm3ways and naive
# model coefficients, no calibration model, object-difference cap 10 / 11), on
# sketches of 9 / 10 codens and of the default 11.
CODENS_BUILD_CASES = [
    ("memeff_detail", ["ani", "-r", "{refs40c9i}", "-q", "{qry50c9}", "-n", "0.5"]),
    ("stream_detail_naive", ["ani", "-r", "{refs40c10}", "-q", "{qry8c10}", "-n", "0.5", "-v"]),
    ("stream_detail_moe", ["ani", "-r", "{refs40c9}", "-q", "{qry8c9}", "-s", "3", "-n", "0.5"]),
    ("self_matrix", ["ani", "-q", "{refs40c9i}", "--format", "matrix", "--values", "ani"]),
    ("matrix_full", ["matrix", "--format", "full", "{refs40c10}"]),
    ("memeff_detail_11codens", ["ani", "-r", "{refs120}", "-q", "{qry30}", "-n", "0.8"]),
    ("self_triangle_11codens", ["ani", "-q", "{refs40}", "--format", "triangle", "--values", "ani"]),
]


def make_fixture(root: str, name: str) -> str:
    """Writes fixture `name` under root (idempotent) and returns its directory."""
    path = os.path.join(root, name)
    if os.path.isdir(path):
        return path
    base = name
    while base not in FIXTURES:
        base = base[:-1]
    spec = dict(FIXTURES[base])
    coden_len, klen = CODENS.get(name, (11, 32))
    if name in CODENS:
        spec.update(ctx_bits=4 * coden_len, obj_bits=2 * klen - 4 * coden_len, klen=klen)
    sk = kssdgpu.synth(**spec)
    meta = synth_meta(sk, len(name)) if name in WITH_META else None
    counts = synth_counts(sk, len(name)) if name in WITH_COUNTS else None
    kssdgpu.write_sketch_dir(path, sk, coden_len=coden_len, klen=klen, with_index=name in INDEXED, meta=meta,
                             abundance=counts)
    return path


def with_threads(argv, threads=4):
    """-p right after the subcommand: positional sketch arguments must come last."""
    return [argv[0], "-p", str(threads), *argv[1:]]


def out_files(argv):
    """Names of the extra output files a case writes ({out:NAME} placeholders)."""
    return [a[5:-1] for a in argv if a.startswith("{out:")]


def materialize(root: str, argv, fresh_tag: str):
    """argv with fixture placeholders replaced by fresh copies (so side effects such
    as automatic index creation start from the same state for every binary) and
    {out:NAME} placeholders by files of this run."""
    out = []
    for a in argv:
        if a.startswith("{list:"):
            # a --query-sketch-list file naming fresh copies of the fixtures (with a
            # comment, a blank line and surrounding blanks the parser must skip)
            dirs = materialize(root, ["{" + n + "}" for n in a[6:-1].split(",")], fresh_tag)
            path = os.path.join(root, fresh_tag, "query_list.txt")
            with open(path, "w") as f:
                f.write("# query sketches\n\n" + "".join(f"  {d} \n" for d in dirs))
            out.append(path)
        elif a.startswith("{out:"):
            os.makedirs(os.path.join(root, fresh_tag), exist_ok=True)
            out.append(os.path.join(root, fresh_tag, a[5:-1]))
        elif a.startswith("{") and a.endswith("}"):
            name = a[1:-1]
            src = make_fixture(os.path.join(root, "_src"), name)
            dst = os.path.join(root, fresh_tag, name)
            if not os.path.isdir(dst):
                shutil.copytree(src, dst)
            out.append(dst)
        else:
            out.append(a)
    return out

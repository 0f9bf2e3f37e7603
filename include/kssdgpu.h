/*
 * libkssdgpu — B200 (sm_100a) shared-context counting engine for KSSD3A's
 * `kssd3a ani` / `kssd3a matrix`.  C ABI: plain pointers and sizes, status returns.
 *
 * The reference has no plugin or FFI layer; its replaceable seam is the pair of
 * counting functions the drivers call per query block:
 *
 *   count_ctx_obj_frm_comb_sketch_section_with_unique  src/command_ani.h:463-624
 *   count_ctx_obj_frm_comb_sketch_section_lower         src/command_ani.h:635-721
 *
 * called from src/command_ani.c:656,1698,1803 and src/command_matrix.c:489,573,845.
 * Those functions take the sorted index (sortedcomb_ctxgid64obj32) in host memory,
 * a block of query samples (comblco keys + comblco.index offsets) and caller-owned,
 * zeroed dense counter blocks [block][R] of ctx_mut2_t / obj_section_t
 * (src/command_ani.h:114-124).  The entry points below take the same arguments,
 * in the same layouts, and fill the same counters bit for bit; the index lives on
 * the device behind an opaque handle (built once, like the reference's
 * read_from_file of the index), errors come back as status codes instead of
 * err()/errx() process exits, and no global state (the reference's Bitslen) is used:
 * object width is a parameter of the index.
 */
#ifndef KSSDGPU_H
#define KSSDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define KSSDGPU_OK 0
#define KSSDGPU_ERR_ARG 1          /* invalid argument (size, null pointer, width) */
#define KSSDGPU_ERR_CUDA 2         /* CUDA runtime error (message via kssdgpu_last_error) */
#define KSSDGPU_ERR_UNSORTED 3     /* index records or query keys not sorted */
#define KSSDGPU_ERR_GID 4          /* record gid >= number of references */
#define KSSDGPU_ERR_TIMEOUT 5      /* a bounded device loop gave up (never expected) */
#define KSSDGPU_ERR_NOMEM 6        /* device allocation failed */
#define KSSDGPU_ERR_CAPACITY 7     /* request exceeds a documented capacity limit */

/* Counting flags. */
#define KSSDGPU_IGNORECONFLICT 0x1u /* ani --ignoreconflict: skip ref (ctx,gid) runs with >1 object */
#define KSSDGPU_UNIQUE 0x2u         /* also count reference-unique contexts (--unique-ctx) */
#define KSSDGPU_PLAIN 0x4u          /* use the plain one-query-per-launch kernel (baseline) */
#define KSSDGPU_GLOBAL_ACC 0x8u     /* force global-memory accumulators (no shared-memory rows) */
#define KSSDGPU_NO_ZERO 0x10u       /* device calls: outputs were zeroed by the caller (skip memset) */
#define KSSDGPU_SMEM_ACC 0x20u      /* force shared-memory accumulator rows (KSSDGPU_ERR_CAPACITY when a
                                       row of the index's references does not fit) */
#define KSSDGPU_SELF_PLAN 0x40u     /* self lower triangle: join over the index's cached set-major plan
                                       (built and kept on first use) instead of the one-pass scan */
#define KSSDGPU_SELF_SCAN 0x80u     /* self lower triangle: the one-pass scan join, whatever the density */
#define KSSDGPU_SELF_DENSE 0x100u   /* self lower triangle: the dense tensor-core join, whatever the
                                       density (conflict-free indexes only) */

/* Counter cells, identical in layout to the reference's ctx_mut2_t / obj_section_t. */
typedef struct kssdgpu_ctx_mut2 {
    uint32_t num_ctx;
    uint32_t num_mut2_ctx;
} kssdgpu_ctx_mut2_t;
typedef struct kssdgpu_obj_section {
    uint32_t diff_obj;
    uint32_t diff_obj_section;
} kssdgpu_obj_section_t;

typedef struct kssdgpu_index kssdgpu_index_t;

/* Message of the last failing call on this thread ("" if none). */
const char *kssdgpu_last_error(void);

/* Creates the CUDA context of `device` (otherwise created by the first call that
 * needs it).  A front end can call it from a helper thread while it reads its input
 * files, so context creation overlaps the I/O. */
int kssdgpu_init(int device);

/*
 * Device-resident CSR from the reference's inverted index records
 * (sortedcomb_ctxgid64obj32: n packed 12-byte {uint64 ctx<<20|gid; uint32 obj},
 * sorted by (ctxgid, obj); host memory).  Replaces read_from_file of the index
 * (src/command_ani.c:508-516) plus kssd_build_fenceposts_ctxgid (:3656-3678).
 * nref = number of reference samples (gids must be < nref); obj_bits = object
 * width (Bitslen.obj, src/sketch_rearrange.c:35; 20 for the default coden pattern).
 */
int kssdgpu_index_from_records(const void *records12, uint64_t n, int nref, int obj_bits,
                               int device, kssdgpu_index_t **out);

/*
 * The same CSR built on the device directly from a sketch (comblco keys, each
 * sample sorted ascending, and comblco.index offsets; host memory): the GPU
 * version of gen_inverted_index4comblco (src/command_sketch.c:916-938) minus the
 * file write.  Guards of the reference: total entries < UINT32_MAX, nref < 2^20.
 */
int kssdgpu_index_from_sketch(const uint64_t *keys, const uint64_t *offs, int nref, int obj_bits,
                              int device, kssdgpu_index_t **out);

void kssdgpu_index_free(kssdgpu_index_t *idx);

/* Calls on one index handle share its per-index device scratch (plans, work lists,
 * compact counters): do not make them from several host threads at once, and do
 * not let them overlap on the GPU (order them on one stream).  Different handles are
 * independent; the server (kssdgpu_server_*) serialises its own calls. */

/* Facts of a built index: records, unique contexts, references, object bits. */
int kssdgpu_index_info(const kssdgpu_index_t *idx, uint64_t *records, uint64_t *contexts,
                       int *nref, int *obj_bits);

/*
 * Rebuilds the index's context membership filter (built with the index) with
 * key-range stripes of at most max_stripe_bytes each (0: the default of 16 MB; at most
 * 256 stripes; at least 8 bits per context) and reports the stripe count and the
 * filter's bytes (either may be NULL).  A batched count with the filter on walks the
 * query keys stripe by stripe when there are several, so that the stripe in use stays
 * in L2.  Synchronizes the device; not to be called while a server runs on the
 * index.  No reference counterpart (the CPU path has no filter).
 */
int kssdgpu_index_filter(kssdgpu_index_t *idx, uint64_t max_stripe_bytes, int *stripes, uint64_t *bytes);

/*
 * Copies the index back as reference-layout records (12-byte packed, sorted) and
 * its unique-object bitset ((n+7)/8 bytes; src/command_sketch.c:856-914).  Either
 * output may be NULL.
 */
int kssdgpu_index_export(const kssdgpu_index_t *idx, void *records12, uint8_t *unique_bits);

/*
 * Per-reference context counts (AF denominators).  With conflict != 0 a (ctx,gid)
 * run of L > 1 objects counts once, or not at all with ignoreconflict
 * (ref_ctx_counts_from_ctxgidobj, src/command_ani.c:351-370); otherwise the
 * record count of each gid (:372-381).  unique_out (may be NULL) receives the
 * reference-unique context totals (unique_ref_context_totals, :441-460).
 */
int kssdgpu_index_ref_ctx_counts(const kssdgpu_index_t *idx, int conflict, int ignoreconflict,
                                 uint32_t *ctx_count_out, uint32_t *unique_out);

/*
 * count_ctx_obj_frm_comb_sketch_section_with_unique (src/command_ani.h:463-574),
 * counting part.  Host buffers:
 *   qry_keys   comblco keys of the block, keys of query i at
 *              qry_keys[qry_offs[i] - qry_offs[0] .. qry_offs[i+1] - qry_offs[0])
 *   qry_offs   nq + 1 absolute comblco.index offsets (section_skidx)
 *   ctx, obj   caller-owned [nq][nref] counter blocks (overwritten; need not be zeroed)
 *   uctx, uobj [nq][nref] reference-unique counters when flags has KSSDGPU_UNIQUE
 * Every cell of the outputs is written.  Detail-mode filtering and ranking
 * (src/command_ani.h:577-621) is host work on these counters.
 */
int kssdgpu_count_block(kssdgpu_index_t *idx, const uint64_t *qry_keys, const uint64_t *qry_offs,
                        int nq, unsigned flags, kssdgpu_ctx_mut2_t *ctx, kssdgpu_obj_section_t *obj,
                        kssdgpu_ctx_mut2_t *uctx, kssdgpu_obj_section_t *uobj);

/*
 * count_ctx_obj_frm_comb_sketch_section_lower (src/command_ani.h:635-721): as
 * above without unique counters, counting only references with gid < qry_gid,
 * where qry_gid = qry_gid_offset + i for query i of the block.
 */
int kssdgpu_count_lower(kssdgpu_index_t *idx, const uint64_t *qry_keys, const uint64_t *qry_offs,
                        int nq, int qry_gid_offset, unsigned flags, kssdgpu_ctx_mut2_t *ctx,
                        kssdgpu_obj_section_t *obj);

/*
 * Device-pointer forms of the two calls (inputs already in HBM; stream is a
 * cudaStream_t or NULL for the legacy stream).  d_qry_offs are absolute offsets as
 * above; outputs are device arrays of nq*nref cells.  Asynchronous: the counters
 * are complete when the stream reaches this point; errors detected on the device
 * are reported by the next kssdgpu_sync(idx, stream).
 */
int kssdgpu_count_block_dev(kssdgpu_index_t *idx, const uint64_t *d_qry_keys,
                            const uint64_t *d_qry_offs, int nq, int qry_gid_offset, int lower,
                            unsigned flags, kssdgpu_ctx_mut2_t *d_ctx, kssdgpu_obj_section_t *d_obj,
                            kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj, void *stream);
int kssdgpu_sync(kssdgpu_index_t *idx, void *stream);

/*
 * Autotune the batched count of this index on a representative block (arguments as
 * kssdgpu_count_block_dev; flags select unique/ignoreconflict, lower selects the
 * triangle form): shared-memory accumulator rows (where a row fits), global rows in
 * key-range chunks of 1,024 / 4,096 / 16,384 entries and (with several filter stripes)
 * global rows stripe by stripe are each timed with CUDA events (best of three after a
 * warm-up) on the legacy stream, then the best of them
 * with the index's context membership filter toggled (at least 8 bits per context
 * in key-range stripes of at most 16 MB, built with the index: a query context it
 * rules out needs no table probe; with several stripes and global rows the count runs
 * stripe by stripe, see kssdgpu_index_filter); the fastest becomes the index's
 * setting for later batched counts without KSSDGPU_SMEM_ACC / KSSDGPU_GLOBAL_ACC.
 * Synchronizes the device; the outputs hold the block's counters afterwards.  Without
 * a call: global rows (in 4,096-entry chunks, or stripe by stripe), filter on.  No
 * reference counterpart (the CPU path has no tunables).
 */
typedef struct kssdgpu_count_tuning {
    int smem_rows;        /* 1: shared-memory accumulator rows; 0: global rows in chunks */
    uint32_t chunk_keys;  /* entries per key-range chunk of the global-row mode */
    int candidates;       /* settings timed */
    float ms;             /* the chosen setting's time on the block */
    int filter;           /* 1: query contexts pass the index's membership filter before a table probe */
    int striped;          /* 1: global rows run stripe by stripe over the filter's key-range stripes */
} kssdgpu_count_tuning_t;
int kssdgpu_count_tune(kssdgpu_index_t *idx, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs, int nq,
                       int qry_gid_offset, int lower, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx,
                       kssdgpu_obj_section_t *d_obj, kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj,
                       kssdgpu_count_tuning_t *out);

/*
 * Detail-mode count with the candidate filter fused behind it on the device: the
 * counting of kssdgpu_count_block on the block, then the pre-filter of the reference's
 * detail branch (src/command_ani.h:585-609) over the block's counters in HBM, so only
 * candidate cells are copied back.  A cell (i, j) is a candidate when
 *   num_ctx >= ctxcut, qry_ctx_count[i] > 0, ref_ctx_count[j] > 0,
 *   max(num_ctx / qry_ctx_count[i], num_ctx / ref_ctx_count[j]) >= afcut, and
 *   its naive ANI >= anicut - 1e-9, the naive ANI being the float
 *   1 - diff_obj / num_ctx / 7 or, with KSSDGPU_UNIQUE, 1 - naive distance of the
 *   unique counters when they cover >= 5% of the reference, else of the full ones
 *   (FP64 with the device's pow).
 * The 1e-9 margin keeps every cell the reference keeps: the caller re-applies the
 * exact ANI test with its own libm to the candidates before ranking them.  Outputs:
 *   hits      the candidates, ascending (query, ref); query = index in the block;
 *             all eight counters (unique ones zero without KSSDGPU_UNIQUE)
 *   row_offs  nq + 1 entries: query i's candidates are hits[row_offs[i] .. row_offs[i+1])
 * More than hits_cap candidates: KSSDGPU_ERR_CAPACITY with row_offs filled (the size
 * the caller needs).  flags: KSSDGPU_IGNORECONFLICT, KSSDGPU_UNIQUE, accumulator flags.
 * No reference counterpart as an entry point: it fuses a6's counting with its detail
 * filter so the dense block stays on the device.
 */
typedef struct kssdgpu_hit kssdgpu_hit_t;
int kssdgpu_count_detail(kssdgpu_index_t *idx, const uint64_t *qry_keys, const uint64_t *qry_offs, int nq,
                         unsigned flags, const uint32_t *qry_ctx_count, const uint32_t *ref_ctx_count, int ctxcut,
                         float afcut, float anicut, kssdgpu_hit_t *hits, uint64_t hits_cap, uint64_t *row_offs);

/*
 * Whole self lower triangle in one pass (the counting behind
 * comb_sortedsketch64_indexed_self_full / _triangle, src/command_ani.c:1657-1842,
 * and matrix_write_indexed_self_matrix, src/command_matrix.c:439-619), valid when
 * the index was built from the same sketch that supplies the queries.  Output
 * cells are packed lower-triangular: cell (q, r), r < q, at q*(q-1)/2 + r
 * (ani_lower_offset, src/command_ani.c:1588-1591); nref*(nref-1)/2 cells each.
 * Host-buffer form.
 */
int kssdgpu_self_lower(kssdgpu_index_t *idx, unsigned flags, kssdgpu_ctx_mut2_t *ctx_lower,
                       kssdgpu_obj_section_t *obj_lower);
/*
 * Candidate votes of the indexed sparse scan behind `kssd3a matrix --format
 * edges|clusters|dedup-plan` on one sketch (pairwise_indexed_self_scan,
 * src/pairwise_graph.c:1148-1316; nomination at :1195-1246): for every sample q of the
 * sketch (keys/offs: comblco keys and absolute comblco.index offsets, nref samples),
 * the keys at positions 0, step, 2*step, ... that the index holds, in context groups of
 * at most max_ctx_freq postings (0: any), vote once for every reference gid r < q of
 * the group.  Outputs over the packed lower triangle (cell (q, r) at q*(q-1)/2 + r):
 * votes, and first = the lowest sampled position index (position / step) that voted
 * (UINT32_MAX without a vote) -- the scan's order of touching r within row q.
 * Host buffers; synchronous.
 */
int kssdgpu_self_votes(kssdgpu_index_t *idx, const uint64_t *keys, const uint64_t *offs, uint32_t max_ctx_freq,
                       uint32_t sample_step, uint32_t *votes, uint32_t *first);
/* Device form of kssdgpu_self_lower (outputs in HBM, stream-ordered).
 *
 * Default: nothing cached between calls; the join follows the index's density
 * (kssdgpu_self_choice).  The one-pass scan (KSSDGPU_SELF_SCAN) zero-fills the packed
 * lower triangle (unless KSSDGPU_NO_ZERO), reads every context group's bounds and
 * joins each group of >= 2 postings as it finds it.  The dense join
 * (KSSDGPU_SELF_DENSE) lists the shared contexts, sorts their postings into alleles
 * (distinct objects per context), builds two int8 operand matrices and computes all
 * four counters of every pair with one exact int8 GEMM on the tensor cores (int32
 * accumulation), then writes every cell of the triangle; it needs a conflict-free
 * index (KSSDGPU_ERR_ARG otherwise) and synchronizes the stream once (for the
 * allele count).
 *
 * With KSSDGPU_SELF_PLAN: the first call builds a set-major plan of the index's
 * shared contexts (kept on the handle; later calls only join over it).  Where the
 * dense counters outgrow L2 that join adds into per-index compact counters while the
 * zero fill runs on an internal stream that waits for the caller's earlier work; the
 * call's last operation on `stream` waits for both.  Calls on one index that overlap
 * on the GPU share those compact counters: order them on one stream. */
int kssdgpu_self_lower_dev(kssdgpu_index_t *idx, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx_lower,
                           kssdgpu_obj_section_t *d_obj_lower, void *stream);

/*
 * Matrix values on the device: the FP64 epilogue that turns the counters of every
 * cell of a packed lower triangle into the value a `kssd3a ani --format
 * matrix|triangle` output prints for it -- the per-pair metric of
 * ani_indexed_self_pair_metric / ani_matrix_pair_value (src/command_ani.c:1458-1496,
 * 1627-1655): lm3ways distance (src/model_ani.h:285-305), naive and p distances
 * (src/command_ani.h:202-232), Mash and AAF distances (src/command_matrix.c:26-33), the
 * 160-tree calibration (src/model_refaf_hgb.h:7593-7628), the selected metric and the
 * exception value (src/command_ani.c:1186-1379, 1448-1456).  Every + - * / is the
 * reference's IEEE double operation in its order (no contraction), so a value built
 * from them alone (lm3ways, the calibration trees, p_dist) is bit-identical to the
 * reference's.  log, log1p and pow (CUDA's, whose last bits may differ from a host
 * libm's) enter the Naive, Mash and AAF values and three calibration features; those
 * values print the reference's six decimals, except where the difference could change
 * what is printed: a calibration feature within 1e-9 (relative) of a tree threshold on
 * the cell's path, or a Naive / Mash / AAF value within 1e-12 of a rounding boundary of
 * its six printed decimals or of zero.  Such cells are not valued on the device: their
 * value is a NaN and they are listed (cell, counters) for the caller to recompute on
 * the host.
 */
typedef struct kssdgpu_metric_opt {
    int s;              /* selected metric 1..9 (BestDist .. p_dist); negative: print 1 - distance */
    int e;              /* exception value (no sketch on one side, failed AF gate) */
    int v;              /* ANI from the naive model instead of lm3ways */
    int unassembled;    /* --qraw query mode */
    int unified_metric; /* --unified-metric */
    int raw_output;     /* no calibration */
    float afcut;        /* AF gate */
    int drfold;         /* the sketch's drfold (model feature scale) */
    int obj_bits;       /* object width (p_dist) */
    int ctx_bits;       /* context width (Mash / AAF k = ctx_bits / 2) */
    int zero_const;     /* cells with no shared context and both sketch sizes nonzero take zero_value */
    double zero_value;
    /* the calibration trees (the 11-coden build's model; the 9- and 10-coden builds have
     * none): node records of 16 bytes {double x; int8 feature; uint8 flags (bit 0 leaf,
     * bit 1 a NaN input goes left); uint16 left, right (relative to the tree's first
     * node)}, the first node of every tree (hgb_trees + 1 offsets), the baseline */
    const void *hgb_nodes;
    uint32_t hgb_nodes_count;
    const uint32_t *hgb_tree_begin;
    uint32_t hgb_trees;
    double hgb_baseline;
} kssdgpu_metric_opt_t;

/* A cell the caller values on the host: its lower-triangle number q*(q-1)/2 + r and its
 * counters. */
typedef struct kssdgpu_recheck {
    uint64_t cell;
    kssdgpu_ctx_mut2_t ctx;
    kssdgpu_obj_section_t obj;
} kssdgpu_recheck_t;

/* Device form over any packed lower triangle of n samples: d_qcnt / d_rcnt are the
 * samples' sketch sizes as query / as reference (n each), the counters d_ctx_lower /
 * d_obj_lower (n(n-1)/2 each); writes d_value_lower (n(n-1)/2 doubles), the first
 * recheck_cap listed cells to d_recheck and their number to *d_nrecheck (zeroed by the
 * call).  Stream-ordered on `stream` of `device`; the calibration trees are copied to the
 * device once per device and model. */
int kssdgpu_lower_metric_dev(int device, const kssdgpu_metric_opt_t *opt, int n, const uint32_t *d_qcnt,
                             const uint32_t *d_rcnt, const kssdgpu_ctx_mut2_t *d_ctx_lower,
                             const kssdgpu_obj_section_t *d_obj_lower, double *d_value_lower,
                             kssdgpu_recheck_t *d_recheck, uint64_t recheck_cap, uint64_t *d_nrecheck,
                             void *stream);

/* The self matrix of an index's own samples with its values from the device: the self
 * join of kssdgpu_self_lower (flags alike), then the device epilogue above; host buffers
 * (qcnt / rcnt: n sketch sizes; value_lower: n(n-1)/2 doubles; recheck: recheck_cap
 * entries), synchronous.  *nrecheck = the listed cells; more than recheck_cap returns
 * KSSDGPU_ERR_CAPACITY (the values of the other cells are written).  Moves 8 bytes per
 * cell to the host instead of kssdgpu_self_lower's 16. */
int kssdgpu_self_lower_metric(kssdgpu_index_t *idx, unsigned flags, const kssdgpu_metric_opt_t *opt,
                              const uint32_t *qcnt, const uint32_t *rcnt, double *value_lower,
                              kssdgpu_recheck_t *recheck, uint64_t recheck_cap, uint64_t *nrecheck);

/*
 * Facts of the self join, from one pass over the index (no plan is built): context
 * groups holding >= 2 postings, postings inside them, and their posting pairs
 * (k(k-1)/2 per group of k).  These size the join's algorithmic bytes.
 */
int kssdgpu_self_plan_info(kssdgpu_index_t *idx, uint64_t *groups, uint64_t *postings, uint64_t *pairs);

/*
 * Which join kssdgpu_self_lower(_dev) takes for these flags (KSSDGPU_PATH_*), and the
 * index's shared-context density: pairs of postings of shared contexts / (nref^2 x
 * alleles of shared contexts), the ratio of the scan's counter updates to the dense
 * GEMM's multiply-adds up to a constant (the allele count -- distinct objects per
 * shared context -- is estimated at index build from up to 65,536 sampled context
 * groups).  Without a path flag the dense tensor-core join is taken when the index is
 * conflict-free, the density is at least 1/2048 and its operands fit in half of the
 * free device memory; else the one-pass scan.  No reference counterpart.
 */
#define KSSDGPU_PATH_SCAN 0
#define KSSDGPU_PATH_DENSE 1
#define KSSDGPU_PATH_PLAN 2
int kssdgpu_self_choice(kssdgpu_index_t *idx, unsigned flags, int *path, double *density);
/* Allele rows (distinct objects of the shared contexts: the GEMM's K before padding to
 * 128) of the last dense self join on this index; 0 before one ran. */
int kssdgpu_self_dense_alleles(kssdgpu_index_t *idx, uint64_t *alleles);

/*
 * Autotune the KSSDGPU_SELF_PLAN join's plan (once per index; builds the plan first if needed):
 * every candidate setting is planned and timed as a whole step (zero fill + join) on
 * scratch counters, after an L2 flush, and the fastest is kept.  Reports the setting in use: groups per
 * set-major chunk, whether chunks run largest first, the largest group size joined
 * flat (one thread per group; 1: none), how many candidates were timed (0: defaults
 * kept, e.g. when a setting is pinned by KSSDGPU_JOIN_CHUNK / KSSDGPU_JOIN_SORT /
 * KSSDGPU_JOIN_FLAT or the scratch would not fit) and the chosen candidate's step
 * time in ms.  Without this call the plan uses the defaults (32 groups, largest
 * first, every size as tiled items) unless KSSDGPU_TUNE=1.  Synchronizes the device.  No
 * reference counterpart (the CPU path has no tunables).  Any out pointer may be NULL.
 */
int kssdgpu_self_plan_tune(kssdgpu_index_t *idx, uint32_t *chunk_groups, int *sorted, uint32_t *flat_groups,
                           int *candidates, float *step_ms);

/*
 * Plain baseline kernel with device inputs: one launch per query (h_qry_offs is a
 * host copy of d_qry_offs, used to size each launch).  Outputs are zeroed unless
 * KSSDGPU_NO_ZERO.  Same counters as kssdgpu_count_block_dev.
 */
int kssdgpu_count_plain_dev(kssdgpu_index_t *idx, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs,
                            const uint64_t *h_qry_offs, int nq, int qry_gid_offset, int lower, unsigned flags,
                            kssdgpu_ctx_mut2_t *d_ctx, kssdgpu_obj_section_t *d_obj,
                            kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj, void *stream);

/*
 * No-allocation form of kssdgpu_count_block_dev (no counterpart in the reference).
 *
 * For callers that must not allocate device memory during a count: a serving
 * loop that reserved all device memory up front for its admission budget, or an
 * embedding application whose own allocator owns the device and forbids other
 * allocations.  The call runs the batched persistent counting kernel, in the
 * accumulator mode kssdgpu_count_block_dev would use (global rows split into
 * key-range chunks, so a large query spreads over all SMs, unless shared-memory rows
 * are forced or were chosen by kssdgpu_count_tune), with its scratch (work counter
 * and the chunk prefix or largest-first query order it builds on the device) in a
 * static device array of this library instead of memory from cudaMalloc; it calls
 * no cudaMalloc, cudaFree or allocating library routine.  The index (built earlier)
 * and all inputs and outputs are the caller's device buffers, as for
 * kssdgpu_count_block_dev; errors found on the device (query keys out of order) are
 * reported by the next kssdgpu_sync(idx, stream).
 *
 * Limits and rules:
 *   - at most KSSDGPU_NOALLOC_MAX_QUERIES queries per call; more returns
 *     KSSDGPU_ERR_CAPACITY without launching anything;
 *   - the array is KSSDGPU_NOALLOC_SCRATCH_BYTES, held by every GPU that loads the
 *     library until the process exits;
 *   - the first call on a device looks up the array's device address (set-up);
 *     make that first call before any stream capture; after a cudaDeviceReset,
 *     call kssdgpu_init(device) first so that the address is looked up again;
 *   - every call shares the one array (it keeps the last call's contents and is
 *     cleared where needed on each call), so calls that overlap on the GPU (other
 *     streams, other threads) race: serialise them.
 */
#define KSSDGPU_NOALLOC_MAX_QUERIES 65536
#define KSSDGPU_NOALLOC_SCRATCH_BYTES (512 + 4 * KSSDGPU_NOALLOC_MAX_QUERIES)
int kssdgpu_count_block_noalloc(kssdgpu_index_t *idx, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs,
                                int nq, int qry_gid_offset, int lower, unsigned flags,
                                kssdgpu_ctx_mut2_t *d_ctx, kssdgpu_obj_section_t *d_obj,
                                kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj, void *stream);

/*
 * Continuous-batching query server over a resident index (the serving loop; the
 * reference has no server: its per-request equivalent is one `kssd3a ani -r R -q one`
 * run).  Each request is one query sample; its result is the list of nonzero counter
 * cells kssdgpu_count_block gives for that query alone, sorted by reference id.
 *
 * Admission by device memory: at creation the server reserves as many batch slots as
 * device_budget bytes hold (at most `slots`); each slot admits the oldest queued
 * requests up to max_batch_queries queries and max_batch_keys keys, and every slot's
 * batch runs beside the others on the device, so requests arriving while batches run
 * join the next free slot.  A batch whose nonzero cells overflow max_hits is split:
 * its requests re-run one per batch, and only a request that overflows alone fails
 * (KSSDGPU_ERR_CAPACITY).  Query keys that do not ascend are rejected at submit
 * (KSSDGPU_ERR_UNSORTED).
 */
typedef struct kssdgpu_hit {
    uint32_t query; /* 0 in results (each request is one query) */
    uint32_t ref;
    uint32_t num_ctx, num_mut2_ctx, diff_obj, diff_obj_section;
    uint32_t u_num_ctx, u_num_mut2_ctx, u_diff_obj, u_diff_obj_section; /* KSSDGPU_UNIQUE */
} kssdgpu_hit_t;

typedef struct kssdgpu_server_config {
    int max_batch_queries;   /* queries per batch slot */
    uint64_t max_batch_keys; /* keys per batch slot (larger single queries are rejected) */
    uint64_t max_hits;       /* nonzero cells per batch (0: min(batch queries x references, 2^22)) */
    unsigned flags;          /* KSSDGPU_IGNORECONFLICT | KSSDGPU_UNIQUE */
    int slots;               /* most batch slots in flight (0: 4) */
    uint64_t device_budget;  /* device bytes the slots may reserve (0: half of the free memory) */
} kssdgpu_server_config_t;

typedef struct kssdgpu_server_stats {
    uint64_t completed, batches, pending, max_inflight, overlapped_batches, reserved_bytes;
    double p50_ms, p99_ms, max_ms, mean_ms; /* submit -> result latency */
    uint64_t slots;          /* batch slots reserved (the budget's share) */
    uint64_t splits;         /* batches split after overflowing max_hits */
} kssdgpu_server_stats_t;

typedef struct kssdgpu_server kssdgpu_server_t;

int kssdgpu_server_create(kssdgpu_index_t *idx, const kssdgpu_server_config_t *cfg, kssdgpu_server_t **out);
/* Copies the query's keys (sorted comblco keys of one sample) and queues it. */
int kssdgpu_server_submit(kssdgpu_server_t *srv, const uint64_t *keys, uint64_t n_keys, uint64_t *ticket);
/* Waits (timeout_ms < 0: no limit) for a request; gives its hit count and latency. */
int kssdgpu_server_wait(kssdgpu_server_t *srv, uint64_t ticket, int timeout_ms, uint32_t *n_hits,
                        double *latency_ms);
/* Copies a finished request's hits (cap entries at most) and forgets the ticket. */
int kssdgpu_server_take(kssdgpu_server_t *srv, uint64_t ticket, kssdgpu_hit_t *hits, uint32_t cap);
int kssdgpu_server_stats(kssdgpu_server_t *srv, kssdgpu_server_stats_t *out);
int kssdgpu_server_reset_stats(kssdgpu_server_t *srv);
/* Finishes queued and running batches, then frees the server (not the index). */
void kssdgpu_server_destroy(kssdgpu_server_t *srv);

/*
 * Sketching of sequence (FASTA/FASTQ records) on the device, as the reference's
 * `kssd3a sketch` (src/command_sketch.c:3913-3949, :4156-4188; src/kssdlib_sort.c:388-406):
 * every k-mer of a record made of A/C/G/T (either case) takes its canonical context
 * (the smaller of the forward and reverse-complement contexts, the reverse on a tie),
 * is kept when the 32-bit SplitMix64 hash of the context is <= UINT32_MAX >> drfold, and
 * becomes ctx << obj_bits | obj; per sample the keys are sorted and deduplicated and,
 * unless conflict is set, contexts holding more than one object are dropped.
 */
typedef struct kssdgpu_sketch_params {
    int klen;       /* k-mer length, 1..32 (32 with the 11-coden pattern) */
    int coden_len;  /* > 0: the coden context pattern of this many codens; 0: hclen/holen layout */
    int hclen;      /* half context length (coden_len == 0) */
    int holen;      /* half outer object length (coden_len == 0) */
    int drfold;     /* k-mer space downsampling 1/2^drfold, 0..32 */
    int conflict;   /* 1: keep contexts that hold several objects */
} kssdgpu_sketch_params_t;
/* Context mask, k-mer mask and object width of the parameters (src/sketch_rearrange.c:7-39). */
int kssdgpu_sketch_masks(const kssdgpu_sketch_params_t *p, uint64_t *ctxmask, uint64_t *tupmask, int *obj_bits);
/* The sketch method id stored in lcofiles.stat (src/command_sketch.h:49-52, :769-772). */
uint32_t kssdgpu_sketch_hash_id(const kssdgpu_sketch_params_t *p);
/*
 * seq: the records' sequence bytes back to back (< 4 GiB per call); record r is
 * seq[rec_offs[r] .. rec_offs[r+1]) (rec_offs[0] = 0, rec_offs[nrec] = seq_len); sample s
 * is records samp_recs[s] .. samp_recs[s+1] (samp_recs[0] = 0, samp_recs[nsamples] = nrec).
 * Writes sample s's keys to keys[offs[s] .. offs[s+1]) (offs: nsamples + 1 words).  With
 * fewer than offs[nsamples] keys of room the call returns KSSDGPU_ERR_CAPACITY with offs
 * filled.  Runs on the current device; synchronous.
 */
int kssdgpu_sketch(const char *seq, uint64_t seq_len, const uint64_t *rec_offs, uint64_t nrec,
                   const uint64_t *samp_recs, int nsamples, const kssdgpu_sketch_params_t *p, uint64_t *keys,
                   uint64_t keys_cap, uint64_t *offs);

/* Number of kernels launched by this library so far in this process. */
uint64_t kssdgpu_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif

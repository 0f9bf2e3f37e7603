/*
 * FP64 epilogue of the counting path: features -> distances/ANI, calibration,
 * metric selection, filters and the byte format of every printed field.
 *
 * Every formula evaluates in the reference's operation order, compiled without
 * floating-point contraction, so each double is bit-identical to the reference
 * binary's and every printed digit matches (model: src/model_ani.h:233-367,
 * src/command_ani.h:200-232, src/command_matrix.c:26-33, src/model_refaf_hgb.h:7575-7628;
 * rows: src/command_ani.c:1056-1432).
 */
#ifndef KSSD_EPILOGUE_H
#define KSSD_EPILOGUE_H

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>

#include "kssd_format.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ani_features_t (src/model_ani.h:215-222), same field order */
typedef struct kssd_features {
    uint32_t XnY_ctx;
    uint32_t X_ctx;
    uint32_t N_diff_obj_section;
    uint32_t N_mut2_ctx;
    uint32_t N_diff_obj;
} kssd_features_t;

/* The options the epilogue reads (subset of ani_opt_t, src/command_ani.h:18-68). */
typedef struct kssd_ani_opt {
    int fmt;              /* 0 detail, 1 matrix, 2 triangle */
    int p;                /* host threads */
    bool d;               /* diagonal */
    bool v;               /* naive model */
    bool unassembled;     /* --qraw */
    bool unified_metric;
    bool ignoreconflict;
    bool raw_output;
    bool max_pdist_set;
    double max_pdist;
    int max_diff_obj_section;
    int e;                /* exception value */
    int s;                /* selected metric, sign = matrix values */
    int ntop;
    int ctxcut;
    float afcut;
    bool afcut_set;
    float anicut;
    bool unique_ctx;
    bool estimate_coverage; /* --estimate-coverage: coverage columns on detail rows */
    /* sketch-derived globals of the reference (Bitslen, ani_model_drfold) */
    int obj_bits;
    int ctx_bits;
    int drfold;
} kssd_ani_opt_t;

/* ani_row_t (src/command_ani.c:1056-1085), the fields the printed row uses */
typedef struct kssd_row {
    uint32_t rn;
    double ani, metric, selected_ani, moe_dist, naive_dist, p_dist, mash_dist, aaf_dist;
    double calibrated_ani, best_ani;
    unsigned char confidence, best_guarded, af_pass;
    bool unique_ctx_selected;
    double af_qry, blastn_af_qry, af_ref, blastn_af_ref;
    int XnY_ctx, N_diff_obj, N_diff_obj_section, N_mut2_ctx;
    /* --estimate-coverage (src/command_ani.c:1071-1084): status 0 not computed, 1 markers
     * unique among the reported rows, 2 query abundances missing, 4 reference-db unique bits */
    unsigned char coverage_status;
    uint32_t cov_ref_markers, cov_observed_markers;
    double cov_observed_fraction, cov_count_sum, est_depth, pos_mean_depth, pos_median_depth, count_cv;
    double est_mass, est_fraction;
} kssd_row_t;

/* Reference-database marker bits for coverage: the index records and their
 * unique-object bitset (sortedcomb_ctxgid64obj32 + .unique_bits) */
typedef struct kssd_cov_refdb {
    bool available;
    uint64_t entries;
    const uint8_t *bits;
    const kssd_index_rec_t *sorted;
} kssd_cov_refdb_t;

/* populate_selected_coverage_for_query_arrays (src/command_ani.c:2315-2455): coverage of
 * the reported rows of one query from its abundances (q_keys sorted, q_counts parallel;
 * NULL: abundances missing) and each row's reference keys (ref_keys at absolute
 * ref_offs[rn] - ref_offs[0]); markers are reference keys unique in the reference db
 * (refdb available) or among the rows' references. */
void kssd_coverage_rows(const uint64_t *q_keys, const uint32_t *q_counts, size_t q_n, const uint64_t *ref_keys,
                        const uint64_t *ref_offs, const kssd_cov_refdb_t *refdb, int obj_bits, kssd_row_t *rows,
                        size_t n_rows);

extern const char kssd_coverage_header[];

void kssd_opt_defaults(kssd_ani_opt_t *o);

double kssd_fold_scale(int drfold);
double kssd_lm3ways_dist(const kssd_features_t *f, int drfold);
double kssd_af_anib(const kssd_features_t *f, int drfold);
double kssd_naive_dist(const kssd_features_t *f);
double kssd_p_dist(const kssd_features_t *f, int obj_bits);
double kssd_mashD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY);
double kssd_aafD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY);
double kssd_hgb_predict_ani(double raw_ani, double ref_af, unsigned xny, unsigned n_diff_obj,
                            unsigned n_diff_obj_section, unsigned n_mut2_ctx, int drfold);

bool kssd_af_pass(const kssd_ani_opt_t *o, double af_qry, double af_ref);
uint32_t kssd_af_needed_ctx(const kssd_ani_opt_t *o, uint32_t qry_ctx, uint32_t ref_ctx);
bool kssd_row_passes_close_filter(const kssd_row_t *r, const kssd_ani_opt_t *o);
bool kssd_use_unique_context(uint32_t matched, uint32_t full_reference);

/* make_selected_output_row (src/command_ani.c:1349-1379); qry/ref meta may be NULL */
kssd_row_t kssd_make_row(uint32_t rn, const kssd_features_t *f, const kssd_ani_opt_t *o, uint32_t qry_ctx,
                         uint32_t ref_ctx, double af_qry, double blastn_af_qry, double af_ref,
                         double blastn_af_ref, const kssd_infile_meta_t *qry_meta,
                         const kssd_infile_meta_t *ref_meta);
/* selected distance/ANI again after a caller changed naive_dist (unique contexts) */
void kssd_finalize_row(kssd_row_t *r, const kssd_ani_opt_t *o);

/* The full metric value of one (q, r) pair the way the matrix drivers compute it
 * (ani_matrix_pair_value / ani_indexed_self_pair_metric, src/command_ani.c:1458-1496,
 * 1627-1655): double AFs, exception value when a sketch is empty. */
double kssd_pair_metric(const kssd_features_t *f, uint32_t qry_ctx, uint32_t ref_ctx, const kssd_ani_opt_t *o,
                        const kssd_infile_meta_t *qry_meta, const kssd_infile_meta_t *ref_meta);
double kssd_matrix_exception_value(const kssd_ani_opt_t *o);
/* The metric of every pair with no shared context (XnY = 0) and non-empty sketches,
 * which is one constant whenever afcut > 0: such a pair never passes the AF gate, so
 * no model depends on its sketch sizes.  Returns false (no constant) when afcut is 0. */
bool kssd_zero_overlap_metric(const kssd_ani_opt_t *o, double *value);
double kssd_matrix_diagonal_value(const kssd_ani_opt_t *o);

/* printing */
typedef struct kssd_buf {
    char *s;
    size_t l, m;
} kssd_buf_t;
void kssd_buf_reserve(kssd_buf_t *b, size_t extra);
void kssd_buf_printf(kssd_buf_t *b, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void kssd_buf_puts(kssd_buf_t *b, const char *s);
void kssd_buf_putc(kssd_buf_t *b, char c);
void kssd_buf_free(kssd_buf_t *b);

extern const char kssd_detail_header[];
/* append_unified_detail_row (src/command_ani.c:1381-1432): nothing when the close filter rejects */
void kssd_append_detail_row(kssd_buf_t *b, const kssd_ani_opt_t *o, const char *qry_name, const char *ref_name,
                            const kssd_row_t *r, const char *annotation);
int32_t kssd_scale_fixed6(double value);               /* ani_scale_fixed6, src/command_ani.c:1593-1604 */
void kssd_put_scaled6(kssd_buf_t *b, int32_t scaled);  /* ani_kput_scaled6, :1606-1625 */

/* comparator of detail survivors (cmp_ani_desc, src/command_ani.c:1087-1095) */
int kssd_cmp_row_desc(const void *a, const void *b);

#ifdef __cplusplus
}
#endif
#endif

/* FP64 epilogue; see kssd_epilogue.h.  Compiled with -ffp-contract=off: each
 * expression keeps the reference's operation order and rounding. */
#define _GNU_SOURCE
#include "kssd_epilogue.h"

#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include "kssd_hgb.h"

#define KSSD_EPSILON (1e-8)
#define KSSD_NAIVE_TAU (0.01)

/* ---------------------------------------------------------------- model coefficients
 * Trained constants of the reference's builds (src/model_ani.h:9-205): the default
 * NUM_CODENS = 11 set, or the set its 9- and 10-coden builds share; they must be
 * identical for identical output.  The AF model's constants are the same for all. */
#ifndef KSSD_NUM_CODENS
#define KSSD_NUM_CODENS 11
#endif
#if KSSD_NUM_CODENS != 9 && KSSD_NUM_CODENS != 10 && KSSD_NUM_CODENS != 11
#error "the reference builds 9, 10 or 11 codens"
#endif
#if KSSD_NUM_CODENS < 11
static const double k_denom[12] = {1.0090536851341, 1.0013604061893, 1.03540226374509, 1.04270754727088,
                                   1.0108940845453, 1.0010797461052, 0.98914550652945, 1.01536320288592,
                                   1.0061957741437, 0.9957814716168, 0.98352379677340, 1.00951820561544};
static const double k_denom95[12] = {1.0196821174688, 0.9817771341602, 1.04637038371202, 1.02441485561367,
                                     1.0163855061091, 0.9824051281495, 1.04908985213703, 1.01102197270052,
                                     1.0074050784795, 1.0018402553389, 0.94654127396428, 0.94051319172603};
static const double k_coef[17] = {-0.587100397752123, -7.93027271403258e-08, 4.98481429879899e-06,
                                  -1.63903694463017e-05, -4.93356600478016e-06, -14843.5350131617,
                                  306478.144745683,  -290254.345158429, -1781.00695309133,
                                  -1091.99589131905, 327.6575530681,    47395.255680747,
                                  47798.7112013701,  -35574.6303634354, -45398.423188085,
                                  -46461.4920783106, 35045.3583333325};
static const double k_coef95[17] = {10.7394186800999,  -2.92835943410177e-08, 1.66112325940088e-05,
                                    -3.48757817098253e-05, -1.82725607919882e-05, 3151.11534599359,
                                    -1300.37794535582, -1824.96575177919, -21820.9227396359,
                                    -30943.09511694,   10100.3465983902,  25441.8492675468,
                                    35763.8363380932,  -3901.01958522226, -3669.6748819999,
                                    -4909.59256464219, -5653.59698386914};
#else
static const double k_denom[12] = {1.0178887, 1.0135146, 1.0302181, 1.1205122, 1.0136223, 0.9803396,
                                   1.0021964, 0.9839395, 0.9988935, 0.9690589, 0.9888171, 0.9817371};
static const double k_denom95[12] = {1.0145656, 1.2708196, 1.2169829, 0.3904416, 0.8147527, 1.3389150,
                                     2.0581364, -1.4624736, 1.6877678, 2.4390067, 0.7878482, 0.6697437};
static const double k_coef[17] = {6.86905236142636,  -5.85271800517096e-08, 7.43351941016881e-06,
                                  -1.95859228059721e-05, -8.44336369105416e-06, -11726.5478433625,
                                  -111109.682632437, 121000.895632267,  -741.538955661909,
                                  -1894.53741972785, 2585.81964981999,  -7744.5216892858,
                                  -18190.2514369096, 23306.3090989115,  8352.82760552325,
                                  19782.4294837312,  -25518.2493259614};
static const double k_coef95[17] = {-1.69173585242774, -3.64716315423252e-08, 2.85880264052975e-05,
                                    -5.5597924264054e-05, -2.96208613804271e-05, 1106.96550282022,
                                    -83.197177767225,  -1671.88720051458, 152.75590068948,
                                    212.734805232395,  208.388739816682,  -0.27860125939004,
                                    2.27065806912198,  -10.2977013026837, -250.681324281127,
                                    -403.751360812353, -137.96628693833};
#endif
static const double k_af_denom[15] = {2.36775520439829,  2.17036643548818,  -0.0977124271437818,
                                      -0.251063182363729, 2.19491057829433,  1.41850238263675,
                                      2.15224961402778,  -2.18587619877498, -2.21943802445092,
                                      0.418474287083788, 0.990424249133548, 0.502163745411501,
                                      5.7787290524088,   0.626839640715682, 0.638706160147675};
static const double k_af_coef[21] = {0.127498260534708, -1.51730137145957e-06, 9.48114616179122e-05,
                                     -0.000257916039708839, -7.85253629216324e-05, 1.96482915215685e-06,
                                     -1475.58996322769, 26.4698377745167,  529.387641078915,
                                     42.0602258298213,  92.3637001980455,  -306.00755719743,
                                     -86.3482066935661, 2.16630645286942,  -0.674746089642152,
                                     48.1147600903939,  3.39101087242059,  -15.5481688297158,
                                     -26.7068442368566, 18.5142668221724,  20.4430437567379};
/* naive model (src/command_ani.h:212-218) */
#if KSSD_NUM_CODENS < 11
static const double k_naive_scale = 0.1557143;
static const double k_naive_intercept = 9.961e-5;
#else
static const double k_naive_scale = 0.1544286;
static const double k_naive_intercept = 7.133e-4;
#endif

static const char *const k_metric_names[9] = {"BestDist", "RecalDist", "CtxMoE", "Naive", "MashD",
                                              "AafD",     "MashD_if_far", "AafD_if_far", "p_dist"};

const char kssd_detail_header[] =
    "Qry\tRef\tANI\tDistance\tConfidence\tSelected_metric\tXnY_ctx\tQry_align_fraction\t"
    "blastn_Qry_align_fraction\tRef_align_fraction\tblastn_Ref_align_fraction\tN_diff_obj\t"
    "N_diff_obj_section\tN_mut2_ctx\tRef_annotation";

void kssd_opt_defaults(kssd_ani_opt_t *o)
{
    /* ani_opt defaults, src/command_ani_wrapper.c:174-221 */
    memset(o, 0, sizeof *o);
    o->p = 1;
    o->s = 1;
    o->e = 1;
    o->ntop = -1;
    o->ctxcut = 3;
    o->afcut = 0.5f;
    o->anicut = 0.95f;
    o->max_diff_obj_section = -1;
    o->obj_bits = 20;
    o->ctx_bits = 44;
    o->drfold = 8;
}

/* ---------------------------------------------------------------- models */

double kssd_fold_scale(int drfold)
{
    const int delta = drfold - 8;
    if (delta < -60)
        return ldexp(1.0, -60);
    if (delta > 60)
        return ldexp(1.0, 60);
    return ldexp(1.0, delta);
}

static double lm3_core(double X, double S, double M, double D, const double p[12], const double c[17])
{
    const double d1 = 1 / (p[0] * X + p[1] * S + p[2] * M + p[3] * D + KSSD_EPSILON);
    const double d2 = 1 / (p[4] * X + p[5] * S + p[6] * M + p[7] * D + KSSD_EPSILON);
    const double d3 = 1 / (p[8] * X + p[9] * S + p[10] * M + p[11] * D + KSSD_EPSILON);
    return c[0] + c[1] * X + c[2] * S + c[3] * M + c[4] * D + c[5] * d1 + c[6] * d2 + c[7] * d3 + c[8] * X * d1 +
           c[9] * S * d1 + c[10] * M * d1 + c[11] * X * d2 + c[12] * S * d2 + c[13] * M * d2 + c[14] * X * d3 +
           c[15] * S * d3 + c[16] * M * d3;
}

double kssd_lm3ways_dist(const kssd_features_t *f, int drfold)
{
    const double scale = kssd_fold_scale(drfold);
    const double X = (double)f->XnY_ctx * scale;
    const double S = (double)f->N_diff_obj_section * scale;
    const double M = (double)f->N_mut2_ctx * scale;
    const double D = (double)f->N_diff_obj * scale;
    if (X <= 0.0)
        return 1;
    else if (D <= 0.0)
        return 0;
    double dist = lm3_core(X, S, M, D, k_denom, k_coef);
    if (dist < 0.05)
        dist = lm3_core(X, S, M, D, k_denom95, k_coef95);
    if (dist < 0)
        dist = 0;
    return dist;
}

double kssd_af_anib(const kssd_features_t *f, int drfold)
{
    const double scale = kssd_fold_scale(drfold);
    const double X = (double)f->XnY_ctx * scale, S = (double)f->N_diff_obj_section * scale;
    const double M = (double)f->N_mut2_ctx * scale, D = (double)f->N_diff_obj * scale;
    const double T = (double)f->X_ctx * scale;
    const double *p = k_af_denom, *c = k_af_coef;
    const double d1 = 1 / (p[0] * X + p[1] * S + p[2] * M + p[3] * D + p[4] * T + KSSD_EPSILON);
    const double d2 = 1 / (p[5] * X + p[6] * S + p[7] * M + p[8] * D + p[9] * T + KSSD_EPSILON);
    const double d3 = 1 / (p[10] * X + p[11] * S + p[12] * M + p[13] * D + p[14] * T + KSSD_EPSILON);
    return c[0] + c[1] * X + c[2] * S + c[3] * M + c[4] * D + c[5] * T + c[6] * d1 + c[7] * d2 + c[8] * d3 +
           c[9] * X * d1 + c[10] * S * d1 + c[11] * M * d1 + c[12] * D * d1 + c[13] * X * d2 + c[14] * S * d2 +
           c[15] * M * d2 + c[16] * D * d2 + c[17] * X * d3 + c[18] * S * d3 + c[19] * M * d3 + c[20] * D * d3;
}

double kssd_naive_dist(const kssd_features_t *f)
{
    if (f->XnY_ctx == 0)
        return 1;
    const double ratio = (double)(f->N_diff_obj_section + KSSD_EPSILON) / (f->N_diff_obj + KSSD_EPSILON);
    const double dist0 = (double)f->N_diff_obj / (f->XnY_ctx + f->N_diff_obj);
    const double final_dist = 1 - pow((1 - dist0), ratio);
    if (final_dist <= 0)
        return 0;
    double w = final_dist / KSSD_NAIVE_TAU;
    if (w > 1.0)
        w = 1.0;
    return final_dist * k_naive_scale + k_naive_intercept * w;
}

double kssd_p_dist(const kssd_features_t *f, int obj_bits)
{
    if (f->XnY_ctx == 0 || obj_bits == 0)
        return 1;
    return (double)f->N_diff_obj_section / ((double)f->XnY_ctx * ((double)obj_bits / 2.0));
}

double kssd_mashD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY)
{
    const double j = (double)XnY / (X + Y - XnY);
    return (-log(2 * j / (1 + j)) / (K));
}

double kssd_aafD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY)
{
    return (-log((double)XnY / (X < Y ? X : Y)) / (K));
}

static double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

double kssd_hgb_predict_ani(double raw_ani, double ref_af, unsigned xny, unsigned n_diff_obj,
                            unsigned n_diff_obj_section, unsigned n_mut2_ctx, int drfold)
{
#if KSSD_NUM_CODENS < 11
    /* the 9- and 10-coden builds carry no calibration model: raw ANI
     * (src/model_refaf_hgb.h, its #else branch) */
    (void)ref_af; (void)xny; (void)n_diff_obj; (void)n_diff_obj_section; (void)n_mut2_ctx; (void)drfold;
    return raw_ani;
#endif
    if (xny == 0)
        return raw_ani;
    raw_ani = clamp01(raw_ani);
    if (ref_af < 1e-12)
        ref_af = 1e-12;
    if (ref_af > 1.0)
        ref_af = 1.0;
    const double xd = (double)xny;
    const double ref_aaf_ani = clamp01(1.0 + log(ref_af) / 11.0);
    double x[KSSD_HGB_FEATURES];
    x[0] = raw_ani;
    x[1] = ref_af;
    x[2] = log1p(xd * kssd_fold_scale(drfold));
    x[3] = (double)n_diff_obj / xd;
    x[4] = (double)n_diff_obj_section / xd;
    x[5] = (double)n_mut2_ctx / xd;
    x[6] = ref_aaf_ani;
    x[7] = raw_ani - ref_aaf_ani;
    x[8] = ref_af < 0.2 ? 1.0 : 0.0;
    x[9] = (ref_af >= 0.2 && ref_af < 0.5) ? 1.0 : 0.0;
    x[10] = ref_af >= 0.5 ? 1.0 : 0.0;
    double pred = kssd_hgb_baseline;
    for (int t = 0; t < KSSD_HGB_TREES; ++t) {
        const unsigned begin = kssd_hgb_tree_begin[t];
        unsigned node = begin;
        while (!(kssd_hgb_nodes[node].flags & 1u)) {
            const kssd_hgb_node_t *nd = &kssd_hgb_nodes[node];
            const double v = x[nd->feature];
            const int left = isnan(v) ? (nd->flags >> 1) & 1u : (v <= nd->x);
            node = begin + (left ? nd->left : nd->right);
        }
        pred += kssd_hgb_nodes[node].x;
    }
    return clamp01(pred);
}

/* ---------------------------------------------------------------- filters */

bool kssd_af_pass(const kssd_ani_opt_t *o, double af_qry, double af_ref)
{
    return (af_qry > af_ref ? af_qry : af_ref) >= (double)o->afcut;
}

uint32_t kssd_af_needed_ctx(const kssd_ani_opt_t *o, uint32_t qry_ctx, uint32_t ref_ctx)
{
    const uint32_t denom = qry_ctx < ref_ctx ? qry_ctx : ref_ctx;
    const double need = (double)o->afcut * (double)denom;
    if (need <= 0.0)
        return 0;
    if (need >= (double)UINT32_MAX)
        return UINT32_MAX;
    return (uint32_t)ceil(need);
}

static bool close_filter_enabled(const kssd_ani_opt_t *o)
{
    return o && (o->max_pdist_set || o->max_diff_obj_section >= 0);
}

bool kssd_row_passes_close_filter(const kssd_row_t *r, const kssd_ani_opt_t *o)
{
    if (!close_filter_enabled(o))
        return true;
    if (o->max_diff_obj_section >= 0 && r->N_diff_obj_section > o->max_diff_obj_section)
        return false;
    if (o->max_pdist_set && (!isfinite(r->p_dist) || r->p_dist > o->max_pdist))
        return false;
    return true;
}

bool kssd_use_unique_context(uint32_t matched, uint32_t full_reference)
{
    return full_reference > 0 && (uint64_t)matched * 20 >= full_reference;
}

/* ---------------------------------------------------------------- rows */

enum { CONF_LOW = 0, CONF_MEDIUM = 1, CONF_HIGH = 2 };

static double bounded_ani(double v)
{
    if (!isfinite(v))
        return NAN;
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

static double ctx_k(const kssd_ani_opt_t *o) { return o->ctx_bits > 0 ? (double)o->ctx_bits / 2.0 : 22.0; }

static double mash_ani(const kssd_ani_opt_t *o, double overlap, double q, double r)
{
    if (overlap <= 0.0 || q <= 0.0 || r <= 0.0)
        return 0.0;
    const double denom = q + r - overlap;
    if (denom <= 0.0)
        return 0.0;
    const double j = overlap / denom;
    if (j <= 0.0)
        return 0.0;
    return bounded_ani(1.0 + log(2.0 * j / (1.0 + j)) / ctx_k(o));
}

static double aaf_ani(const kssd_ani_opt_t *o, double overlap, double q, double r)
{
    if (overlap <= 0.0 || q <= 0.0 || r <= 0.0)
        return 0.0;
    const double m = q < r ? q : r;
    if (m <= 0.0)
        return 0.0;
    const double c = overlap / m;
    if (c <= 0.0)
        return 0.0;
    return bounded_ani(1.0 + log(c) / ctx_k(o));
}

static bool meta_assembly_record(const kssd_infile_meta_t *s)
{
    return s && s->meta_fmt_version == 1 && s->infile_fmt == 1 && s->total_length_bp > 0 && s->record_count > 0;
}

static bool meta_complete_like_assembly(const kssd_infile_meta_t *s)
{
    if (!s || s->meta_fmt_version != 1 || s->infile_fmt != 1 || s->total_length_bp == 0 || s->median_length_bp == 0)
        return false;
    return s->total_length_bp >= 3500000ULL && s->record_count < 5 && s->median_length_bp > 100000U &&
           (double)s->total_length_bp / (double)s->median_length_bp < 5.0;
}

static bool best_guard_enabled(const kssd_ani_opt_t *o) { return o->fmt == 0 && !o->unassembled && !o->v; }

static void fill_calibration(kssd_row_t *r, const kssd_ani_opt_t *o, const kssd_infile_meta_t *qm)
{
    if (o->unassembled) {
        r->calibrated_ani = r->ani;
        r->best_ani = r->ani;
        r->confidence = CONF_HIGH;
        r->best_guarded = 0;
        return;
    }
    if (r->XnY_ctx > 0 && r->N_diff_obj == 0 && r->N_diff_obj_section == 0 && r->N_mut2_ctx == 0 &&
        r->af_qry == 1.0 && r->af_ref == 1.0) {
        r->calibrated_ani = 1.0;
        r->best_ani = 1.0;
        r->confidence = CONF_HIGH;
        r->best_guarded = 0;
        return;
    }
    r->calibrated_ani = kssd_hgb_predict_ani(r->ani, r->af_ref, (unsigned)r->XnY_ctx, (unsigned)r->N_diff_obj,
                                             (unsigned)r->N_diff_obj_section, (unsigned)r->N_mut2_ctx, o->drfold);
    {
        const double drop = r->ani - r->calibrated_ani;
        if (r->af_ref < 0.5 || (r->ani >= 0.95 && drop > 0.02))
            r->confidence = CONF_LOW;
        else if (fabs(drop) > 0.01)
            r->confidence = CONF_MEDIUM;
        else
            r->confidence = CONF_HIGH;
    }
    r->best_ani = r->calibrated_ani;
    r->best_guarded = 0;
    const double min_af = r->af_qry < r->af_ref ? r->af_qry : r->af_ref;
    if (!best_guard_enabled(o) || !meta_assembly_record(qm) || !meta_complete_like_assembly(qm) || r->ani < 0.958 ||
        r->calibrated_ani < 0.962 || min_af < 0.25 || min_af >= 0.50 || r->XnY_ctx <= 0 || r->af_qry <= 0.0 ||
        r->af_ref <= 0.0)
        return;
    const double qc = (double)r->XnY_ctx / r->af_qry;
    const double rc = (double)r->XnY_ctx / r->af_ref;
    double exact = (double)r->XnY_ctx - (double)r->N_diff_obj;
    if (exact < 0.0)
        exact = 0.0;
    const double mean = (mash_ani(o, (double)r->XnY_ctx, qc, rc) + aaf_ani(o, (double)r->XnY_ctx, qc, rc) +
                         mash_ani(o, exact, qc, rc) + aaf_ani(o, exact, qc, rc)) /
                        4.0;
    if (r->ani - mean < 0.015)
        return;
    r->best_ani = aaf_ani(o, exact, qc, rc);
    r->best_guarded = 1;
}

static int request_id(const kssd_ani_opt_t *o)
{
    int s = abs(o->s);
    return (s < 1 || s > 9) ? 1 : s;
}

static bool value_available(double v) { return v > 0.0 && v <= 1.0; }

static int effective_id(const kssd_row_t *r, const kssd_ani_opt_t *o)
{
    int s = request_id(o);
    if (o->unassembled && !o->unified_metric && s <= 4)
        return 4;
    if (s == 1 && !(!o->raw_output && !o->unassembled && value_available(r->best_ani)))
        s = 2;
    if (s == 2 && !(!o->raw_output && !o->unassembled && value_available(r->calibrated_ani)))
        s = 3;
    return s;
}

static double selected_distance(const kssd_row_t *r, const kssd_ani_opt_t *o)
{
    switch (effective_id(r, o)) {
    case 1: return 1.0 - r->best_ani;
    case 2: return 1.0 - r->calibrated_ani;
    case 3: return r->moe_dist;
    case 4: return r->naive_dist;
    case 5: return r->mash_dist;
    case 6: return r->aaf_dist;
    case 7: return r->af_pass ? r->moe_dist : r->mash_dist;
    case 8: return r->af_pass ? r->moe_dist : r->aaf_dist;
    case 9: return r->p_dist;
    default: return r->metric;
    }
}

void kssd_finalize_row(kssd_row_t *r, const kssd_ani_opt_t *o)
{
    r->metric = selected_distance(r, o);
    r->selected_ani = 1.0 - r->metric;
}

kssd_row_t kssd_make_row(uint32_t rn, const kssd_features_t *f, const kssd_ani_opt_t *o, uint32_t qry_ctx,
                         uint32_t ref_ctx, double af_qry, double blastn_af_qry, double af_ref,
                         double blastn_af_ref, const kssd_infile_meta_t *qry_meta,
                         const kssd_infile_meta_t *ref_meta)
{
    (void)ref_meta;
    kssd_row_t r;
    memset(&r, 0, sizeof r);
    r.rn = rn;
    r.af_qry = af_qry;
    r.blastn_af_qry = blastn_af_qry;
    r.af_ref = af_ref;
    r.blastn_af_ref = blastn_af_ref;
    r.XnY_ctx = (int)f->XnY_ctx;
    r.N_diff_obj = (int)f->N_diff_obj;
    r.N_diff_obj_section = (int)f->N_diff_obj_section;
    r.N_mut2_ctx = (int)f->N_mut2_ctx;
    r.af_pass = kssd_af_pass(o, af_qry, af_ref);
    if (r.af_pass) {
        r.moe_dist = kssd_lm3ways_dist(f, o->drfold);
        r.naive_dist = kssd_naive_dist(f);
        r.p_dist = kssd_p_dist(f, o->obj_bits);
    } else {
        r.moe_dist = o->e;
        r.naive_dist = o->e;
        r.p_dist = o->e;
    }
    r.mash_dist = kssd_mashD((uint32_t)(o->ctx_bits / 2), ref_ctx, qry_ctx, f->XnY_ctx);
    r.aaf_dist = kssd_aafD((uint32_t)(o->ctx_bits / 2), ref_ctx, qry_ctx, f->XnY_ctx);
    r.ani = 1.0 - (o->v ? r.naive_dist : r.moe_dist);
    if (!o->raw_output && r.af_pass)
        fill_calibration(&r, o, qry_meta);
    kssd_finalize_row(&r, o);
    return r;
}

double kssd_matrix_exception_value(const kssd_ani_opt_t *o) { return o->s < 0 ? 1.0 - o->e : o->e; }

double kssd_matrix_diagonal_value(const kssd_ani_opt_t *o) { return o->s < 0 ? 1.0 : 0.0; }

double kssd_pair_metric(const kssd_features_t *f, uint32_t qry_ctx, uint32_t ref_ctx, const kssd_ani_opt_t *o,
                        const kssd_infile_meta_t *qry_meta, const kssd_infile_meta_t *ref_meta)
{
    if (qry_ctx == 0 || ref_ctx == 0)
        return kssd_matrix_exception_value(o);
    const double af_q = (double)f->XnY_ctx / (double)qry_ctx;
    const double af_r = (double)f->XnY_ctx / (double)ref_ctx;
    kssd_features_t t = *f;
    t.X_ctx = qry_ctx;
    const double bq = kssd_af_anib(&t, o->drfold);
    t = *f;
    t.X_ctx = ref_ctx;
    const double br = kssd_af_anib(&t, o->drfold);
    const kssd_row_t r = kssd_make_row(0, f, o, qry_ctx, ref_ctx, af_q, bq, af_r, br, qry_meta, ref_meta);
    return o->s < 0 ? r.selected_ani : r.metric;
}

bool kssd_zero_overlap_metric(const kssd_ani_opt_t *o, double *value)
{
    if (!(o->afcut > 0.0f))
        return false;
    const kssd_features_t zero = {0, 0, 0, 0, 0};
    *value = kssd_pair_metric(&zero, 1, 1, o, NULL, NULL);
    return true;
}

int kssd_cmp_row_desc(const void *pa, const void *pb)
{
    const kssd_row_t *a = pa, *b = pb;
    if (a->selected_ani < b->selected_ani)
        return 1;
    if (a->selected_ani > b->selected_ani)
        return -1;
    if (a->af_qry < b->af_qry)
        return 1;
    if (a->af_qry > b->af_qry)
        return -1;
    return (a->rn > b->rn) - (a->rn < b->rn);
}

/* ---------------------------------------------------------------- printing */

void kssd_buf_reserve(kssd_buf_t *b, size_t extra)
{
    if (b->l + extra + 1 <= b->m)
        return;
    size_t m = b->m ? b->m : 256;
    while (m < b->l + extra + 1)
        m *= 2;
    char *s = realloc(b->s, m);
    if (!s)
        abort();
    b->s = s;
    b->m = m;
}

void kssd_buf_printf(kssd_buf_t *b, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int need = vsnprintf(NULL, 0, fmt, ap);
    va_end(ap);
    if (need < 0)
        return;
    kssd_buf_reserve(b, (size_t)need);
    va_start(ap, fmt);
    vsnprintf(b->s + b->l, (size_t)need + 1, fmt, ap);
    va_end(ap);
    b->l += (size_t)need;
}

void kssd_buf_puts(kssd_buf_t *b, const char *s)
{
    const size_t n = strlen(s);
    kssd_buf_reserve(b, n);
    memcpy(b->s + b->l, s, n + 1);
    b->l += n;
}

void kssd_buf_putc(kssd_buf_t *b, char c)
{
    kssd_buf_reserve(b, 1);
    b->s[b->l++] = c;
    b->s[b->l] = '\0';
}

void kssd_buf_free(kssd_buf_t *b)
{
    free(b->s);
    b->s = NULL;
    b->l = b->m = 0;
}

static const char *confidence_label(unsigned c)
{
    return c == CONF_HIGH ? "high" : (c == CONF_MEDIUM ? "medium" : "low");
}

static double bounded_af(double v)
{
    if (!isfinite(v))
        return v;
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

/* append_coverage_double / coverage_estimator_label and the coverage columns of
 * print_unified_detail_row (src/command_ani.c:1106-1126,1403-1429) */
static void coverage_double(kssd_buf_t *b, double v)
{
    if (!isfinite(v))
        kssd_buf_puts(b, "NA");
    else if (fabs(v) >= 1000.0)
        kssd_buf_printf(b, "%.3f", v);
    else
        kssd_buf_printf(b, "%.6g", v);
}

static void append_coverage(kssd_buf_t *b, const kssd_row_t *r)
{
    const char *label = r->coverage_status == 0   ? "NA:not_computed"
                        : r->coverage_status == 2 ? "NA:query_missing_comblco.a"
                        : r->coverage_status == 3 ? "NA:ref_read_error"
                        : r->coverage_status == 4 ? "refdb_unique_ctxobj_bitset"
                                                  : "reported_unique_ctxobj_sum";
    if (r->coverage_status != 1 && r->coverage_status != 4) {
        kssd_buf_printf(b, "\t%s\tNA\tNA\tNA\tNA\tNA\tNA\tNA\tNA\tNA\tNA\tNA", label);
        return;
    }
    kssd_buf_printf(b, "\t%s\t%u\t%u\t", label, r->cov_ref_markers, r->cov_observed_markers);
    const double v[8] = {r->cov_observed_fraction, r->cov_count_sum, r->est_depth, r->pos_mean_depth,
                         r->pos_median_depth, r->count_cv, r->est_mass, r->est_fraction};
    for (int i = 0; i < 8; ++i) {
        if (i)
            kssd_buf_putc(b, '\t');
        coverage_double(b, v[i]);
    }
    kssd_buf_printf(b, "\t%s", r->coverage_status == 4 ? "refdb" : "reported_rows");
}

void kssd_append_detail_row(kssd_buf_t *b, const kssd_ani_opt_t *o, const char *qry_name, const char *ref_name,
                            const kssd_row_t *r, const char *annotation)
{
    if (!kssd_row_passes_close_filter(r, o))
        return;
    const int eff = effective_id(r, o);
    const char *name = o->unique_ctx ? (r->unique_ctx_selected ? "NaiveUnique" : "NaiveFull") : k_metric_names[eff - 1];
    const char *conf;
    if (o->raw_output)
        conf = "raw";
    else if (o->unassembled && !o->unified_metric && request_id(o) <= 4)
        conf = "unassembled";
    else if (eff == 1)
        conf = r->best_guarded ? "guarded_low_confidence" : confidence_label(r->confidence);
    else if (eff == 2)
        conf = confidence_label(r->confidence);
    else
        conf = "raw";
    const char *anno = annotation && annotation[0] ? annotation : "NA";
    kssd_buf_printf(b, "%s\t%s\t%lf\t%lf\t%s\t%s\t%d\t%f\t%f\t%f\t%f\t%d\t%d\t%d\t%s", qry_name, ref_name,
                    r->selected_ani, r->metric, conf, name, r->XnY_ctx, r->af_qry, bounded_af(r->blastn_af_qry),
                    r->af_ref, bounded_af(r->blastn_af_ref), r->N_diff_obj, r->N_diff_obj_section, r->N_mut2_ctx,
                    anno);
    if (o->estimate_coverage)
        append_coverage(b, r);
    kssd_buf_putc(b, '\n');
}

int32_t kssd_scale_fixed6(double value)
{
    if (!isfinite(value))
        value = 1.0;
    if (value > 2147.0)
        value = 2147.0;
    if (value < -2147.0)
        value = -2147.0;
    return (int32_t)(value >= 0.0 ? value * 1000000.0 + 0.5 : value * 1000000.0 - 0.5);
}

void kssd_put_scaled6(kssd_buf_t *b, int32_t scaled)
{
    char tmp[24];
    int n = 0;
    uint32_t mag;
    if (scaled < 0) {
        tmp[n++] = '-';
        mag = (uint32_t)(-(int64_t)scaled);
    } else {
        mag = (uint32_t)scaled;
    }
    const uint32_t whole = mag / 1000000U;
    uint32_t frac = mag % 1000000U;
    char w[12];
    int wn = 0;
    uint32_t x = whole;
    do {
        w[wn++] = (char)('0' + x % 10);
        x /= 10;
    } while (x);
    while (wn)
        tmp[n++] = w[--wn];
    tmp[n++] = '.';
    for (int i = 5; i >= 0; --i) {
        tmp[n + i] = (char)('0' + frac % 10);
        frac /= 10;
    }
    n += 6;
    kssd_buf_reserve(b, (size_t)n);
    memcpy(b->s + b->l, tmp, (size_t)n);
    b->l += (size_t)n;
    b->s[b->l] = '\0';
}

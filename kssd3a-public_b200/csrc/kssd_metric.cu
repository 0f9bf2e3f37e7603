// FP64 metric epilogue on the device: the printed value of every cell of a lower
// triangle of counters (a matrix of `kssd3a ani --format matrix|triangle`), in the
// reference's formulas and operation order (lm3ways distance src/model_ani.h:285-305,
// naive and p distances src/command_ani.h:202-232, Mash/AAF
// src/command_ani.c:164-188, the 160-tree calibration src/model_refaf_hgb.h:7593-7628,
// metric selection src/command_ani.c:1129-1379, matrix exception values :1448-1456).
//
// This file is compiled with --fmad=false: no multiply-add is contracted, and every
// + - * / is the IEEE double operation the reference's host code performs, so every
// value built from them alone is bit-identical.  Only log, log1p and pow (CUDA's, not
// the host libm's) can differ in the last bits.  A cell's printed value is therefore the
// reference's unless it depends on one of them and either
//   - a calibration feature derived from them lies within kTol of a tree threshold on
//     the cell's path (a different leaf is then possible), or
//   - the value itself is derived from them (Naive, Mash or AAF metrics) and lies
//     within kTolValue of a rounding boundary of the six printed decimals (or of zero);
// such cells are listed for the host, which recomputes them with its own libm.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kssd_metric.cuh"

#ifndef KSSD_NUM_CODENS
#define KSSD_NUM_CODENS 11
#endif

namespace kssd {
namespace {

constexpr double kEps = 1e-8;
constexpr double kNaiveTau = 0.01;
// far above the few-ulp differences of two libms' log / log1p / pow on these values:
// relative distance of a calibration feature to a tree threshold, and distance (relative
// above 1) of a value to a rounding boundary of its printed decimals
constexpr double kTol = 1e-9;
constexpr double kTolValue = 1e-12;

// Trained constants of the reference's builds (src/model_ani.h:9-205): the 11-coden
// set, or the set its 9- and 10-coden builds share.
#if KSSD_NUM_CODENS < 11
__constant__ double c_denom[12] = {1.0090536851341, 1.0013604061893, 1.03540226374509, 1.04270754727088,
                                   1.0108940845453, 1.0010797461052, 0.98914550652945, 1.01536320288592,
                                   1.0061957741437, 0.9957814716168, 0.98352379677340, 1.00951820561544};
__constant__ double c_denom95[12] = {1.0196821174688, 0.9817771341602, 1.04637038371202, 1.02441485561367,
                                     1.0163855061091, 0.9824051281495, 1.04908985213703, 1.01102197270052,
                                     1.0074050784795, 1.0018402553389, 0.94654127396428, 0.94051319172603};
__constant__ double c_coef[17] = {-0.587100397752123, -7.93027271403258e-08, 4.98481429879899e-06,
                                  -1.63903694463017e-05, -4.93356600478016e-06, -14843.5350131617,
                                  306478.144745683,  -290254.345158429, -1781.00695309133,
                                  -1091.99589131905, 327.6575530681,    47395.255680747,
                                  47798.7112013701,  -35574.6303634354, -45398.423188085,
                                  -46461.4920783106, 35045.3583333325};
__constant__ double c_coef95[17] = {10.7394186800999,  -2.92835943410177e-08, 1.66112325940088e-05,
                                    -3.48757817098253e-05, -1.82725607919882e-05, 3151.11534599359,
                                    -1300.37794535582, -1824.96575177919, -21820.9227396359,
                                    -30943.09511694,   10100.3465983902,  25441.8492675468,
                                    35763.8363380932,  -3901.01958522226, -3669.6748819999,
                                    -4909.59256464219, -5653.59698386914};
constexpr double kNaiveScale = 0.1557143;
constexpr double kNaiveIntercept = 9.961e-5;
#else
__constant__ double c_denom[12] = {1.0178887, 1.0135146, 1.0302181, 1.1205122, 1.0136223, 0.9803396,
                                   1.0021964, 0.9839395, 0.9988935, 0.9690589, 0.9888171, 0.9817371};
__constant__ double c_denom95[12] = {1.0145656, 1.2708196, 1.2169829, 0.3904416, 0.8147527, 1.3389150,
                                     2.0581364, -1.4624736, 1.6877678, 2.4390067, 0.7878482, 0.6697437};
__constant__ double c_coef[17] = {6.86905236142636,  -5.85271800517096e-08, 7.43351941016881e-06,
                                  -1.95859228059721e-05, -8.44336369105416e-06, -11726.5478433625,
                                  -111109.682632437, 121000.895632267,  -741.538955661909,
                                  -1894.53741972785, 2585.81964981999,  -7744.5216892858,
                                  -18190.2514369096, 23306.3090989115,  8352.82760552325,
                                  19782.4294837312,  -25518.2493259614};
__constant__ double c_coef95[17] = {-1.69173585242774, -3.64716315423252e-08, 2.85880264052975e-05,
                                    -5.5597924264054e-05, -2.96208613804271e-05, 1106.96550282022,
                                    -83.197177767225,  -1671.88720051458, 152.75590068948,
                                    212.734805232395,  208.388739816682,  -0.27860125939004,
                                    2.27065806912198,  -10.2977013026837, -250.681324281127,
                                    -403.751360812353, -137.96628693833};
constexpr double kNaiveScale = 0.1544286;
constexpr double kNaiveIntercept = 7.133e-4;
#endif
struct Feat {
    uint32_t xny, section, mut2, diff;
};

__device__ double fold_scale(int drfold)
{
    const int delta = drfold - 8;
    if (delta < -60)
        return ldexp(1.0, -60);
    if (delta > 60)
        return ldexp(1.0, 60);
    return ldexp(1.0, delta);
}

__device__ double lm3_core(double X, double S, double M, double D, const double *p, const double *c)
{
    const double d1 = 1 / (p[0] * X + p[1] * S + p[2] * M + p[3] * D + kEps);
    const double d2 = 1 / (p[4] * X + p[5] * S + p[6] * M + p[7] * D + kEps);
    const double d3 = 1 / (p[8] * X + p[9] * S + p[10] * M + p[11] * D + kEps);
    return c[0] + c[1] * X + c[2] * S + c[3] * M + c[4] * D + c[5] * d1 + c[6] * d2 + c[7] * d3 + c[8] * X * d1 +
           c[9] * S * d1 + c[10] * M * d1 + c[11] * X * d2 + c[12] * S * d2 + c[13] * M * d2 + c[14] * X * d3 +
           c[15] * S * d3 + c[16] * M * d3;
}

// lm3ways_dist_from_features (src/model_ani.h:285-305)
__device__ double lm3ways_dist(const Feat &f, int drfold)
{
    const double scale = fold_scale(drfold);
    const double X = (double)f.xny * scale;
    const double S = (double)f.section * scale;
    const double M = (double)f.mut2 * scale;
    const double D = (double)f.diff * scale;
    if (X <= 0.0)
        return 1;
    else if (D <= 0.0)
        return 0;
    double dist = lm3_core(X, S, M, D, c_denom, c_coef);
    if (dist < 0.05)
        dist = lm3_core(X, S, M, D, c_denom95, c_coef95);
    if (dist < 0)
        dist = 0;
    return dist;
}

// get_naive_dist (src/command_ani.h:202-224): pow, so not exact
__device__ double naive_dist(const Feat &f)
{
    if (f.xny == 0)
        return 1;
    const double ratio = (double)(f.section + kEps) / (f.diff + kEps);
    const double dist0 = (double)f.diff / (f.xny + f.diff);
    const double final_dist = 1 - pow((1 - dist0), ratio);
    if (final_dist <= 0)
        return 0;
    double w = final_dist / kNaiveTau;
    if (w > 1.0)
        w = 1.0;
    return final_dist * kNaiveScale + kNaiveIntercept * w;
}

// get_p_dist (src/command_ani.h:226-232)
__device__ double p_dist(const Feat &f, int obj_bits)
{
    if (f.xny == 0 || obj_bits == 0)
        return 1;
    return (double)f.section / ((double)f.xny * ((double)obj_bits / 2.0));
}

// get_mashD / get_aafD (src/command_matrix.c:26-33): log, so not exact
__device__ double mash_d(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY)
{
    const double j = (double)XnY / (X + Y - XnY);
    return (-log(2 * j / (1 + j)) / (K));
}
__device__ double aaf_d(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY)
{
    return (-log((double)XnY / (X < Y ? X : Y)) / (K));
}

__device__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

__device__ bool near(double v, double t) { return fabs(v - t) <= kTol * fmax(1.0, fabs(t)); }

// the 9- and 10-coden builds carry no calibration model (raw ANI)
constexpr bool kCalibrate = KSSD_NUM_CODENS >= 11;

// refaf_hgb_predict_ani (src/model_refaf_hgb.h:7593-7628).  *path_unc: a feature derived
// from log / log1p / pow (or from an inexact raw ANI) came within kTol of a threshold on
// the path, so another leaf is possible; *val_unc: the result is the inexact raw ANI
// itself (no calibration), a few ulps from the host's at most.
__device__ double hgb_predict(const MetricParams &P, double raw_ani, bool raw_unc, double ref_af, const Feat &f,
                              bool *path_unc, bool *val_unc)
{
    if (!kCalibrate || f.xny == 0) {
        *val_unc = raw_unc;
        return raw_ani;
    }
    raw_ani = clamp01(raw_ani);
    if (ref_af < 1e-12)
        ref_af = 1e-12;
    if (ref_af > 1.0)
        ref_af = 1.0;
    const double xd = (double)f.xny;
    const double ref_aaf_ani = clamp01(1.0 + log(ref_af) / 11.0);
    double x[11];
    bool xu[11];
    x[0] = raw_ani;
    xu[0] = raw_unc;
    x[1] = ref_af;
    xu[1] = false;
    x[2] = log1p(xd * fold_scale(P.drfold));
    xu[2] = true;
    x[3] = (double)f.diff / xd;
    x[4] = (double)f.section / xd;
    x[5] = (double)f.mut2 / xd;
    xu[3] = xu[4] = xu[5] = false;
    x[6] = ref_aaf_ani;
    xu[6] = true;
    x[7] = raw_ani - ref_aaf_ani;
    xu[7] = true;
    x[8] = ref_af < 0.2 ? 1.0 : 0.0;
    x[9] = (ref_af >= 0.2 && ref_af < 0.5) ? 1.0 : 0.0;
    x[10] = ref_af >= 0.5 ? 1.0 : 0.0;
    xu[8] = xu[9] = xu[10] = false;
    double pred = P.baseline;
    for (int t = 0; t < P.ntrees; ++t) {
        const uint32_t begin = __ldg(P.tree_begin + t);
        uint32_t node = begin;
        for (int depth = 0; depth < 64; ++depth) {  // trees are far shallower; the bound ends any walk
            if (node >= P.nnodes)  // a malformed model: the cell is left to the host below
                break;
            const HgbNode nd = P.nodes[node];
            if (nd.flags & 1u)
                break;
            const int fi = nd.feature;
            const double v = x[fi];
            if (xu[fi] && near(v, nd.x))
                *path_unc = true;
            const int left = isnan(v) ? (nd.flags >> 1) & 1u : (v <= nd.x);
            node = begin + (left ? nd.left : nd.right);
        }
        if (node >= P.nnodes || !(P.nodes[node].flags & 1u)) {
            *path_unc = true;  // the walk did not end on a leaf
            continue;
        }
        pred += P.nodes[node].x;
    }
    return clamp01(pred);
}

__device__ bool value_available(double v) { return v > 0.0 && v <= 1.0; }

// kssd_pair_metric for a matrix cell (ani_matrix_pair_value / ani_indexed_self_pair_metric,
// src/command_ani.c:1458-1496, 1627-1655, with make_selected_output_row :1349-1379)
__device__ double pair_metric(const MetricParams &P, const Feat &f0, uint32_t qctx, uint32_t rctx, bool *unc)
{
    if (qctx == 0 || rctx == 0)
        return P.s < 0 ? 1.0 - P.e : (double)P.e;
    const double af_q = (double)f0.xny / (double)qctx;
    const double af_r = (double)f0.xny / (double)rctx;
    const bool af_pass = (af_q > af_r ? af_q : af_r) >= (double)P.afcut;
    double moe = P.e, naive = P.e, pd = P.e;
    bool naive_unc = false;
    if (af_pass) {
        moe = lm3ways_dist(f0, P.drfold);
        naive = naive_dist(f0);
        naive_unc = true;
        pd = p_dist(f0, P.obj_bits);
    }
    const uint32_t K = (uint32_t)(P.ctx_bits / 2);
    const double mash = mash_d(K, rctx, qctx, f0.xny);
    const double aaf = aaf_d(K, rctx, qctx, f0.xny);
    const double ani = 1.0 - (P.v ? naive : moe);
    const bool ani_unc = P.v && naive_unc;
    // fill_calibration (src/command_ani.c:1129-1184); matrix outputs never take the
    // assembly best-ANI guard (detail output only), so best ANI = calibrated ANI
    double calibrated = 0, best = 0;
    bool path_unc = false, cal_unc = false;
    if (!P.raw_output && af_pass) {
        if (P.unassembled) {
            calibrated = best = ani;
            cal_unc = ani_unc;
        } else if (f0.xny > 0 && f0.diff == 0 && f0.section == 0 && f0.mut2 == 0 && af_q == 1.0 && af_r == 1.0) {
            calibrated = best = 1.0;
        } else {
            calibrated = hgb_predict(P, ani, ani_unc, af_r, f0, &path_unc, &cal_unc);
            best = calibrated;
        }
    }
    // effective metric (src/command_ani.c:1186-1347)
    int s = P.s < 0 ? -P.s : P.s;
    if (s < 1 || s > 9)
        s = 1;
    if (P.unassembled && !P.unified_metric && s <= 4)
        s = 4;
    if (s <= 2 && (path_unc || (cal_unc && (near(best, 0.0) || near(best, 1.0)))))
        *unc = true;  // another leaf, or value_available() of an inexact calibrated value
    if (s == 1 && !(!P.raw_output && !P.unassembled && value_available(best)))
        s = 2;
    if (s == 2 && !(!P.raw_output && !P.unassembled && value_available(calibrated)))
        s = 3;
    double metric;
    bool vu = false;
    switch (s) {
    case 1: metric = 1.0 - best; vu = cal_unc; break;
    case 2: metric = 1.0 - calibrated; vu = cal_unc; break;
    case 3: metric = moe; break;
    case 4: metric = naive; vu = naive_unc; break;
    case 5: metric = mash; vu = true; break;
    case 6: metric = aaf; vu = true; break;
    case 7: metric = af_pass ? moe : mash; vu = !af_pass; break;
    case 8: metric = af_pass ? moe : aaf; vu = !af_pass; break;
    default: metric = pd; break;
    }
    const double value = P.s < 0 ? 1.0 - metric : metric;
    if (vu) {
        // an inexact value prints the same six decimals unless it lies next to a rounding
        // boundary, or -- as 1 - distance, which may fall on either side of zero -- next to
        // zero, whose sign "%lf" prints (the distances themselves are never negative)
        const double y = fabs(value) * 1000000.0 + 0.5;
        if (!isfinite(value) || fabs(y - rint(y)) <= kTolValue * 1000000.0 * fmax(1.0, fabs(value)) ||
            (P.s < 0 && fabs(value) <= kTolValue))
            *unc = true;
    }
    return value;
}

// One CTA per triangle row q; threads stride over r < q.  Exact cells get their value;
// the others get NaN and are listed (cell, counters) for the host, up to cap entries.
__global__ void __launch_bounds__(256) k_lower_metric(MetricParams P, int n, int row0, int row1,
                                                     const unsigned long long *__restrict__ lc,
                                                     const unsigned long long *__restrict__ lo,
                                                     const uint32_t *__restrict__ qcnt,
                                                     const uint32_t *__restrict__ rcnt, double *__restrict__ out,
                                                     RecheckCell *__restrict__ recheck, unsigned long long cap,
                                                     unsigned long long *__restrict__ nrecheck)
{
    for (int q = row0 + blockIdx.x; q < row1; q += gridDim.x) {
        const size_t base = (size_t)q * (q - 1) / 2;
        const uint32_t qc = __ldg(qcnt + q);
        for (int r = threadIdx.x; r < q; r += blockDim.x) {
            const unsigned long long c = __ldg(lc + base + r), o = __ldg(lo + base + r);
            const uint32_t rc = __ldg(rcnt + r);
            Feat f;
            f.xny = (uint32_t)c;
            f.mut2 = (uint32_t)(c >> 32);
            f.diff = (uint32_t)o;
            f.section = (uint32_t)(o >> 32);
            double v;
            bool unc = false;
            if (P.zero_const && f.xny == 0 && qc && rc)
                v = P.zero_value;
            else
                v = pair_metric(P, f, qc, rc, &unc);
            if (unc) {
                out[base + r] = __longlong_as_double(0x7FF8000000000000ll);
                const unsigned long long slot = atomicAdd(nrecheck, 1ull);
                if (slot < cap)
                    recheck[slot] = RecheckCell{(unsigned long long)(base + r), c, o};
            } else {
                out[base + r] = v;
            }
        }
    }
}

}  // namespace

cudaError_t lower_metric_launch(const MetricParams &P, int n, const unsigned long long *lc,
                                const unsigned long long *lo, const uint32_t *qcnt, const uint32_t *rcnt, double *out,
                                RecheckCell *recheck, unsigned long long cap, unsigned long long *nrecheck, int sms,
                                cudaStream_t st)
{
    if (n < 2)
        return cudaSuccess;
    const int grid = n - 1 < sms * 8 ? n - 1 : sms * 8;
    k_lower_metric<<<grid, 256, 0, st>>>(P, n, 1, n, lc, lo, qcnt, rcnt, out, recheck, cap, nrecheck);
    return cudaGetLastError();
}

}  // namespace kssd

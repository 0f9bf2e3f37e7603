// Shared declarations of the device metric epilogue (kssd_metric.cu) and its caller.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace kssd {

// one node of the calibration trees: the split threshold (or a leaf's value), the
// split's feature, flags (bit 0 leaf, bit 1 a NaN input goes left), children relative
// to the tree's first node (the record layout of the host's model tables)
struct HgbNode {
    double x;
    signed char feature;
    unsigned char flags;
    unsigned short left, right;
};
static_assert(sizeof(HgbNode) == 16, "calibration node records are 16 bytes");

// the options a matrix value reads (a subset of the reference's ani_opt_t)
struct MetricParams {
    int s, e, v, unassembled, unified_metric, raw_output;
    float afcut;
    int drfold, obj_bits, ctx_bits;
    int zero_const;
    double zero_value;
    const HgbNode *nodes;       // device copy of the calibration trees
    const uint32_t *tree_begin; // ntrees + 1 node offsets
    int ntrees;
    uint32_t nnodes;
    double baseline;
};

// a cell whose value the host recomputes: its lower-triangle number and its counters
struct RecheckCell {
    unsigned long long cell, ctx, obj;
};

cudaError_t lower_metric_launch(const MetricParams &P, int n, const unsigned long long *lc,
                                const unsigned long long *lo, const uint32_t *qcnt, const uint32_t *rcnt, double *out,
                                RecheckCell *recheck, unsigned long long cap, unsigned long long *nrecheck, int sms,
                                cudaStream_t st);

}  // namespace kssd

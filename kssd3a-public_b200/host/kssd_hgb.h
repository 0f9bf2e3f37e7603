/* Gradient-boosted calibration model (160 trees) of the reference's assembly
 * ANI epilogue (src/model_refaf_hgb.h:7575-7628), as node records. */
#ifndef KSSD_HGB_H
#define KSSD_HGB_H

#define KSSD_HGB_TREES 160
#define KSSD_HGB_NODES 9760
#define KSSD_HGB_FEATURES 11

typedef struct kssd_hgb_node {
    double x;               /* split threshold, or the leaf value for leaves */
    signed char feature;    /* input feature of a split */
    unsigned char flags;    /* bit 0: leaf; bit 1: a missing (NaN) input goes left */
    unsigned short left;    /* children, relative to the tree's first node */
    unsigned short right;
} kssd_hgb_node_t;

extern const double kssd_hgb_baseline;
extern const unsigned kssd_hgb_tree_begin[KSSD_HGB_TREES + 1];
extern const kssd_hgb_node_t kssd_hgb_nodes[KSSD_HGB_NODES];

#endif

/*
 * Seeded synthetic genomes generated directly in sketch space (the sampled
 * ctxobj64 keys a `kssd3a sketch` run would emit), so that workloads of
 * thousands of multi-Mbp genomes can be produced in seconds on any box.
 *
 * Model (per sample; every sample is an independent deterministic stream):
 *   - cluster c has an ancestor of length L_c drawn from the size distribution;
 *     its sampled k-mers are round(L_c * density) random (44-bit ctx, 20-bit obj)
 *     keys (density ~ 1/256 at DimRdcFold 8).  Lengths and keys come from two
 *     streams of (seed, c) only, so every configuration sharing seed and cluster
 *     count shares the ancestors (a query set and a reference set, say).
 *   - a member with substitution rate p keeps an ancestor key when none of its
 *     ctx_bits/2 context bases and no indel start in its klen window hit it,
 *     probability (1-p)^(ctx_bits/2) * (1-indel_rate)^klen; kept keys mutate each
 *     object base with probability p; lost keys are replaced by fresh random keys.
 *   - a sample with its own length L_s keeps each ancestor key with probability
 *     min(1, L_s/L_c) and adds (L_s-L_c)*density fresh keys when L_s > L_c.
 *   - read sets (conflicts kept) mix 1..k member genomes of a reference set at a
 *     coverage C and base error e: covered keys, extra objects at the same context
 *     (error in the object part; sketch conflicts), and noise contexts.
 */
#ifndef KSSD_SYNTH_H
#define KSSD_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { KSSD_SIZE_FIXED = 0, KSSD_SIZE_LOGNORMAL = 1, KSSD_SIZE_LOGUNIFORM = 2 };
enum { KSSD_ROLE_MEMBER = 0, KSSD_ROLE_OWNLEN = 1, KSSD_ROLE_READS = 2 };

typedef struct kssd_synth_cfg {
    uint64_t seed;          /* ancestors depend only on (seed, cluster) */
    uint64_t sample_seed;   /* per-sample streams: (sample_seed, index) */
    int n_samples;
    int n_clusters;
    int role;               /* KSSD_ROLE_* */
    int size_dist;          /* KSSD_SIZE_*: ancestor lengths (members inherit them) */
    double len_median, len_sigma, len_min, len_max;
    double own_len_min, own_len_max; /* KSSD_ROLE_OWNLEN: own length ~ log-uniform */
    double sub_lo, sub_hi;  /* member substitution rate ~ U(lo, hi) */
    double indel_rate;
    double density;         /* sampled keys per bp */
    int ctx_bits, obj_bits, klen;
    /* KSSD_ROLE_READS: genomes are members of a reference set generated with
     * (seed, ref_sample_seed, ref_clusters) */
    uint64_t ref_sample_seed;
    int ref_samples;
    int reads_min_genomes, reads_max_genomes;
    double cov_lo, cov_hi, err_lo, err_hi;
    int threads;
} kssd_synth_cfg_t;

typedef struct kssd_synth_out {
    int n;
    uint64_t *keys;   /* all samples, each sorted ascending */
    uint64_t *offs;   /* n + 1 */
    double *lengths;  /* per sample genome length (bp) used */
} kssd_synth_out_t;

void kssd_synth_default(kssd_synth_cfg_t *cfg);
kssd_synth_out_t *kssd_synth_generate(const kssd_synth_cfg_t *cfg);
void kssd_synth_free(kssd_synth_out_t *out);

#ifdef __cplusplus
}
#endif
#endif

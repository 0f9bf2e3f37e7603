/*
 * ORACLE — test infrastructure only.  A plain-C restatement of the KSSD3A
 * shared-context counting path, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the CHECKER.  Never linked into, called by, or
 * shipped with the product library.
 *
 * Record layout (the reference's sortedcomb_ctxgid64obj32 file, src/sketch_rearrange.h:19):
 *   packed 12 bytes { uint64_t ctxgid = ctx << 20 | gid; uint32_t obj; }
 * Counter layout (src/command_ani.h:114-124): per (query, ref) cell
 *   ctx2[2*cell+0] = num_ctx, ctx2[2*cell+1] = num_mut2_ctx,
 *   obj2[2*cell+0] = diff_obj, obj2[2*cell+1] = diff_obj_section.
 */
#ifndef KSSD_ORACLE_H
#define KSSD_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_GID_BITS 20

/* src/sketch_rearrange.c:65-78 + src/kssdlib_sort.c:145-219: ctxobj64 -> ctxgidobj, sorted. */
size_t orc_build_index(const uint64_t *keys, const uint64_t *offs, int nsamples, int obj_bits,
                       void *out_records);
/* src/command_sketch.c:856-914: bit i set when record i's obj is unique inside its ctx group. */
uint64_t orc_unique_bits(const void *records, size_t len, uint8_t *bits);
/* src/command_ani.c:351-370 (conflict) / :372-381 (no conflict). */
void orc_ref_ctx_counts(const void *records, size_t len, int nref, const uint64_t *ref_offs,
                        int conflict, int ignoreconflict, uint32_t *out);
/* src/command_ani.c:337-349,383-401,1533-1548. */
void orc_sample_ctx_counts(const uint64_t *keys, const uint64_t *offs, int nsamples, int obj_bits,
                           int conflict, int ignoreconflict, uint32_t *out);
/* src/command_ani.c:441-460. */
void orc_unique_ref_totals(const void *records, size_t len, int nref, int ignoreconflict,
                           uint32_t *out);
/* src/command_ani.h:463-574 (counting part; no detail filtering). */
int orc_count_block(const void *records, size_t len, int nref,
                    const uint64_t *qkeys, const uint64_t *qoffs, int nq,
                    int obj_bits, int ignoreconflict, int want_unique, int threads,
                    uint32_t *ctx2, uint32_t *obj2, uint32_t *uctx2, uint32_t *uobj2);
/* src/command_ani.h:635-721. */
int orc_count_lower(const void *records, size_t len, int nref, int qry_gid_offset,
                    const uint64_t *qkeys, const uint64_t *qoffs, int nq,
                    int obj_bits, int ignoreconflict, int threads,
                    uint32_t *ctx2, uint32_t *obj2);
/* src/command_ani.h:303-346. */
void orc_pair_features(const uint64_t *a, size_t n, const uint64_t *b, size_t m, int obj_bits,
                       int ignore_b_conflict, uint32_t out4[4]);
/* src/dna_popcount.h:45-49. */
int orc_dna_popcount(uint32_t x);
void orc_self_votes(const void *records, size_t len, const uint64_t *keys, const uint64_t *offs, int nsamples,
                    int obj_bits, uint32_t max_freq, uint32_t step, uint32_t *votes, uint32_t *first);
/* Sketch parameters -> context mask, k-mer mask, object width (src/sketch_rearrange.c:7-39). */
void orc_sketch_masks(int coden_len, int klen, int hclen, int holen, uint64_t *ctxmask, uint64_t *tupmask,
                      int *obj_bits);
/* One genome's sketch from its records' sequence bytes seq[rec_offs[r]..rec_offs[r+1]): canonical
 * context per k-mer, kept when (uint32) splitmix64(ctx) <= filter, ctx << obj_bits | obj, sorted,
 * deduplicated, and without conflict the contexts holding several objects removed
 * (src/command_sketch.c:3913-3949, :4156-4188; src/kssdlib_sort.c:388-406).
 * Returns the key count, or (size_t)-1 when cap is too small. */
size_t orc_sketch_records(const char *seq, const uint64_t *rec_offs, int nrec, int klen, uint64_t ctxmask,
                          uint64_t tupmask, int obj_bits, uint32_t filter, int conflict, uint64_t *out, size_t cap);

#ifdef __cplusplus
}
#endif
#endif

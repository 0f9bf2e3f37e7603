/*
 * On-disk formats of a KSSD3A sketch directory and of its inverted index, as read
 * and written by the reference (file names at src/command_sketch.c:29-39):
 *
 *   lcofiles.stat            dim_sketch_stat_t (32 B, src/global_basic.h:138-149)
 *                            followed by infile_num sample names of 256 B each
 *   comblco                  uint64 ctxobj keys, each sample's run sorted ascending
 *   comblco.index            uint64 x (infile_num + 1) run offsets into comblco
 *   sortedcomb_ctxgid64obj32 packed 12 B records {uint64 ctx<<20|gid; uint32 obj},
 *                            sorted by (ctxgid, obj) (src/sketch_rearrange.h:19)
 *   sortedcomb_ctxgid64obj32.unique_bits
 *                            bit i set when record i's obj is unique in its context
 *   lcofiles.anno / lcofiles.infilemeta   optional per-sample sidecars
 */
#ifndef KSSD_FORMAT_H
#define KSSD_FORMAT_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KSSD_PATHLEN 256
#define KSSD_GID_BITS 20

typedef struct kssd_sketch_stat {
    uint32_t hash_id;
    bool koc;
    bool conflict;
    int32_t coden_len;
    int32_t klen;
    int32_t hclen;
    int32_t holen;
    int32_t drfold;
    int32_t infile_num;
} kssd_sketch_stat_t;

typedef struct __attribute__((packed)) kssd_index_rec {
    uint64_t ctxgid;
    uint32_t obj;
} kssd_index_rec_t;

/* infile_meta_t (src/global_basic.h:182-193), 32 B */
typedef struct kssd_infile_meta {
    uint64_t total_length_bp;
    uint32_t record_count;
    uint32_t median_length_bp;
    float asm_level;
    float length_cv;
    uint8_t meta_fmt_version;
    int8_t infile_fmt;
    int8_t create_type;
    uint8_t infile_flags;
} kssd_infile_meta_t;

typedef struct kssd_sketch {
    kssd_sketch_stat_t stat;
    int n;                        /* samples */
    char (*names)[KSSD_PATHLEN];  /* n names */
    uint64_t *keys;               /* comblco */
    uint64_t *offs;               /* comblco.index, n + 1 */
    char (*anno)[KSSD_PATHLEN];   /* optional */
    kssd_infile_meta_t *meta;     /* optional */
    int obj_bits;                 /* 2*klen - ctx_bits */
    int ctx_bits;
} kssd_sketch_t;

/* Last error message of the host library (thread-local). */
const char *kssd_host_last_error(void);
void kssd_host_set_error(const char *msg);

/* Loads a sketch directory.  flags: 1 = annotations, 2 = infile meta.
 * Returns NULL on error (message via kssd_host_last_error). */
kssd_sketch_t *kssd_sketch_load(const char *dir, unsigned flags);
/* comblco.a: per-key k-mer counts of a sketch made with counting (stat.koc) */
uint32_t *kssd_abundance_load(const char *dir, size_t *n_out);
/* sortedcomb_ctxgid64obj32.unique_bits: one bit per index record */
uint8_t *kssd_unique_bits_load(const char *dir, size_t *bytes_out);
void kssd_sketch_free(kssd_sketch_t *s);
int kssd_sketch_write(const char *dir, const kssd_sketch_stat_t *stat, int n,
                      const char (*names)[KSSD_PATHLEN], const uint64_t *keys,
                      const uint64_t *offs);
int kssd_read_stat(const char *dir, kssd_sketch_stat_t *out);
/* bit widths implied by a stat (src/sketch_rearrange.c:7-42) */
void kssd_stat_bits(const kssd_sketch_stat_t *st, int *ctx_bits, int *obj_bits);

/* Inverted index file.  Returns malloc'd records (caller frees) or NULL. */
kssd_index_rec_t *kssd_index_load(const char *dir, size_t *n_out);
int kssd_index_write(const char *dir, const kssd_index_rec_t *recs, size_t n,
                     const uint8_t *unique_bits);
bool kssd_file_exists(const char *dir, const char *name);

#ifdef __cplusplus
}
#endif
#endif

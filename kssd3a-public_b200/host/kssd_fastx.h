/*
 * FASTA/FASTQ input for sketching: the records' sequence bytes of a file (plain or
 * gzip; "-" is standard input), read with the reference's parser rules (its vendored
 * klib kseq: a record starts at '>' or '@'; the header runs to the end of its line;
 * sequence lines run to the next line starting with '>', '+' or '@'; empty lines are
 * skipped; one trailing '\r' of a line is dropped; FASTQ quality lines are consumed by
 * length; a record whose quality length differs ends the file), and the input-format
 * rules of src/global_basic.c:166-192 and src/global_basic.h:216-253.
 */
#ifndef KSSD_FASTX_H
#define KSSD_FASTX_H
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#include "kssd_format.h"

#ifdef __cplusplus
extern "C" {
#endif

#define KSSD_FMT_UNKNOWN 0
#define KSSD_FMT_FASTA 1
#define KSSD_FMT_FASTQ 2

typedef struct kssd_seqbuf {
    char *seq;           /* the records' bytes back to back */
    uint64_t len, cap;
    uint64_t *rec;       /* record offsets into seq: nrec + 1 words */
    uint64_t nrec, rec_cap;
    uint64_t *lens;      /* lengths of the non-empty records (assembly statistics) */
    uint64_t nlens, lens_cap;
} kssd_seqbuf_t;

void kssd_seqbuf_init(kssd_seqbuf_t *b);
void kssd_seqbuf_free(kssd_seqbuf_t *b);
/* Appends the records of path.  anno (KSSD_PATHLEN bytes, may be NULL) receives the
 * first record's header in the reference's annotation form (src/command_sketch.c:1012-1029).
 * Returns 0, or -1 with a message (kssd_host_last_error). */
int kssd_fastx_append(const char *path, kssd_seqbuf_t *b, char *anno);

/* suffix rules, a trailing .gz / .bz2 ignored (case-sensitive like the reference) */
int kssd_fastx_fmt(const char *path);         /* KSSD_FMT_* */
bool kssd_fastx_accepted(const char *path);   /* .fna .fas .fasta .fq .fastq .fa .co */
bool kssd_name_compressed(const char *path);  /* ends in .gz or .bz2 */

#ifdef __cplusplus
}
#endif
#endif

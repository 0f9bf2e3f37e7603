/*
 * Sketch directories made from FASTA/FASTQ inputs for `kssd3a ani`'s sequence inputs
 * (positional auto ANI, --reflist/--qrylist, -q/--qraw with sequence), following the
 * reference's auto-ANI sketching (src/command_ani_wrapper.c:1028-1046, 1275-1436) and
 * its sketcher (src/command_sketch.c:774-790, 4385-4564, 5396-5560): the k-mers are
 * sketched on the GPU (kssdgpu_sketch); this file reads the inputs and writes the
 * directories (lcofiles.stat, comblco, comblco.index, lcofiles.infilemeta, optional
 * lcofiles.anno) and merges them (src/command_sketch.c:1633-1850).
 */
#ifndef KSSD_AUTOSKETCH_H
#define KSSD_AUTOSKETCH_H
#include <stdbool.h>

#include "kssd_format.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kssd_autosketch_opt {
    kssd_sketch_stat_t tmpl;  /* sketch parameters (the template stat; infile_num ignored) */
    bool asone;               /* all files of an input make one sample */
    bool anno;                /* write the first header of each sample to lcofiles.anno */
    int threads;              /* host threads reading the inputs */
} kssd_autosketch_opt_t;

/* The files of one input argument (src/global_basic.c:332-433 with format checking):
 * "-", a directory's entries with an accepted suffix (directory order), or one file
 * with an accepted suffix; exits like the reference on anything else. */
int kssd_organize_input(const char *arg, char ***paths_out);
void kssd_free_paths(char **paths, int n);

/* Sketches the files of one input argument into outdir (created).  Exits with the
 * reference's message on invalid input. */
void kssd_autosketch_to_dir(const char *input, const kssd_autosketch_opt_t *o, const char *outdir);

/* Concatenates sketch directories into outdir (names, index, comblco, infile meta,
 * annotations, comblco.a of counting sketches). */
void kssd_merge_sketch_dirs(char **dirs, int n, const char *outdir);

/* The reference's default auto-ANI template (coden pattern or manual lengths, drfold,
 * conflict; hash_id of those parameters). */
kssd_sketch_stat_t kssd_default_auto_stat(bool coden, int hclen, int holen, int iolen, int drfold, bool conflict,
                                          bool abundance);

/* mkdir -p */
void kssd_mkdir_p(const char *path);
/* rm -r of a temporary tree */
void kssd_remove_tree(const char *path);

#ifdef __cplusplus
}
#endif
#endif

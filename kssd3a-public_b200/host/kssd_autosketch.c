/* Sketch directories from FASTA/FASTQ inputs (see kssd_autosketch.h). */
#include "kssd_autosketch.h"

#include <dirent.h>
#include <err.h>
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include "kssd_fastx.h"
#include "kssdgpu.h"

#define PATHLEN KSSD_PATHLEN
/* infile meta fields (src/global_basic.h:164-176) */
#define META_VERSION 1u
#define CREATE_NORMAL 0
#define CREATE_ASONE 1
#define FLAG_STDIN 0x02u
#define FLAG_COMPRESSED 0x04u
#define FLAG_MIXED_FORMAT 0x10u
/* sequence bytes per device sketch call */
#define SKETCH_BATCH_BYTES (1ull << 30)

void kssd_mkdir_p(const char *path)
{
    char tmp[2 * PATHLEN];
    snprintf(tmp, sizeof tmp, "%s", path);
    for (char *p = tmp + 1; *p; ++p)
        if (*p == '/') {
            *p = 0;
            if (mkdir(tmp, 0755) != 0 && errno != EEXIST)
                err(errno, "mkdir %s", tmp);
            *p = '/';
        }
    if (mkdir(tmp, 0755) != 0 && errno != EEXIST)
        err(errno, "mkdir %s", tmp);
}

void kssd_remove_tree(const char *path)
{
    DIR *d = opendir(path);
    if (!d)
        return;
    struct dirent *e;
    while ((e = readdir(d)) != NULL) {
        if (!strcmp(e->d_name, ".") || !strcmp(e->d_name, ".."))
            continue;
        char child[2 * PATHLEN];
        snprintf(child, sizeof child, "%s/%s", path, e->d_name);
        struct stat st;
        if (lstat(child, &st) != 0)
            continue;
        if (S_ISDIR(st.st_mode))
            kssd_remove_tree(child);
        else
            unlink(child);
    }
    closedir(d);
    rmdir(path);
}

void kssd_free_paths(char **paths, int n)
{
    for (int i = 0; i < n; ++i)
        free(paths[i]);
    free(paths);
}

static void push_path(char ***v, int *n, int *cap, const char *p)
{
    if (*n == *cap) {
        *cap = *cap ? 2 * *cap : 16;
        *v = realloc(*v, (size_t)*cap * sizeof(char *));
        if (!*v)
            err(errno, "out of memory");
    }
    (*v)[(*n)++] = strdup(p);
}

int kssd_organize_input(const char *arg, char ***paths_out)
{
    char **v = NULL;
    int n = 0, cap = 0;
    if (!strcmp(arg, "-")) {
        push_path(&v, &n, &cap, arg);
        *paths_out = v;
        return n;
    }
    struct stat st;
    stat(arg, &st);
    if (S_ISDIR(st.st_mode)) {
        DIR *d = opendir(arg);
        if (!d)
            err(errno, "%dth argument: can't open %s", 1, arg);
        struct dirent *e;
        while ((e = readdir(d)) != NULL) {
            char full[2 * PATHLEN];
            if (strlen(arg) + strlen(e->d_name) + 1 > PATHLEN)
                err(errno, "path: %s/%s exceed maximal path lenth %d", arg, e->d_name, PATHLEN);
            snprintf(full, sizeof full, "%s/%s", arg, e->d_name);
            if (kssd_fastx_accepted(full))
                push_path(&v, &n, &cap, full);
        }
        closedir(d);
    } else if (kssd_fastx_accepted(arg)) {
        push_path(&v, &n, &cap, arg);
    } else {
        static const char *acpt[] = {"fna", "fas", "fasta", "fq", "fastq", "fa", "co"};
        printf("wrong format %dth argument: %s\nSupported format are:\n", 1, arg);
        for (int i = 0; i < 7; ++i)
            printf(".%s ", acpt[i]);
        printf("\n");
        fflush(stdout);
        err(errno, "program exit");
    }
    *paths_out = v;
    return n;
}

/* the SplitMix64 finalizer's low 32 bits (the sketch method id's hash) */
static uint32_t mix32(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return (uint32_t)(x ^ (x >> 31));
}

kssd_sketch_stat_t kssd_default_auto_stat(bool coden, int hclen, int holen, int iolen, int drfold, bool conflict,
                                          bool abundance)
{
    /* src/command_ani_wrapper.c:881-911 */
    kssd_sketch_stat_t s;
    memset(&s, 0, sizeof s);
    s.koc = abundance;
    s.conflict = conflict;
    s.drfold = drfold;
    uint64_t v[3];
    if (coden) {
        s.coden_len = KSSD_NUM_CODENS;
        s.klen = KSSD_NUM_CODENS < 11 ? 3 * KSSD_NUM_CODENS + 1 : 32;
        v[0] = (uint64_t)s.coden_len, v[1] = 0, v[2] = 0;
    } else {
        s.hclen = hclen;
        s.holen = holen;
        s.klen = iolen + 2 * (hclen + holen);
        v[0] = (uint64_t)hclen, v[1] = (uint64_t)holen, v[2] = (uint64_t)iolen;
    }
    const uint32_t filter = 0xFFFFFFFFu >> drfold;
    s.hash_id = mix32(v[0]) ^ mix32(v[1]) ^ mix32(v[2]) ^ mix32((uint64_t)drfold) ^ mix32(filter) ^ mix32(31415926ull);
    return s;
}

static int cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* src/command_sketch.c:1134-1173 */
static void meta_from_lengths(uint64_t *lengths, size_t n, int8_t fmt, int8_t create_type, uint8_t flags,
                              kssd_infile_meta_t *out)
{
    memset(out, 0, sizeof *out);
    out->meta_fmt_version = META_VERSION;
    out->infile_fmt = fmt;
    out->create_type = create_type;
    out->infile_flags = flags;
    out->asm_level = fmt == KSSD_FMT_FASTQ ? 0.0f : -1.0f;
    if (!lengths || n == 0)
        return;
    uint64_t total = 0;
    double mean = 0.0, m2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
        total += lengths[i];
        const double x = (double)lengths[i];
        const double delta = x - mean;
        mean += delta / (double)(i + 1);
        m2 += delta * (x - mean);
    }
    qsort(lengths, n, sizeof lengths[0], cmp_u64);
    out->total_length_bp = total;
    out->record_count = n > UINT32_MAX ? UINT32_MAX : (uint32_t)n;
    if (n & 1)
        out->median_length_bp = lengths[n / 2] > UINT32_MAX ? UINT32_MAX : (uint32_t)lengths[n / 2];
    else {
        const uint64_t med = (lengths[n / 2 - 1] + lengths[n / 2]) / 2;
        out->median_length_bp = med > UINT32_MAX ? UINT32_MAX : (uint32_t)med;
    }
    if (mean > 0.0 && n > 1)
        out->length_cv = (float)(sqrt(m2 / (double)n) / mean);
    if (fmt == KSSD_FMT_FASTA && total > 0)
        out->asm_level = (float)((double)lengths[n - 1] / (double)total);
}

static uint8_t flags_of(const char *path)
{
    uint8_t f = 0;
    if (!strcmp(path, "-"))
        f |= FLAG_STDIN;
    if (kssd_name_compressed(path))
        f |= FLAG_COMPRESSED;
    return f;
}

static void write_file(const char *dir, const char *name, const void *a, size_t na)
{
    char p[2 * PATHLEN];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "wb");
    if (!f || (na && fwrite(a, 1, na, f) != na) || fclose(f) != 0)
        err(errno, "write %s", p);
}

static void *read_file(const char *dir, const char *name, size_t *sz, bool must)
{
    char p[2 * PATHLEN];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "rb");
    if (!f) {
        if (must)
            err(errno, "%s", p);
        *sz = 0;
        return NULL;
    }
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    void *b = malloc(n > 0 ? (size_t)n : 1);
    if (!b || (n > 0 && fread(b, 1, (size_t)n, f) != (size_t)n))
        err(errno, "read %s", p);
    fclose(f);
    *sz = (size_t)n;
    return b;
}

/* One sample: its records' bytes, lengths for the assembly statistics, annotation. */
typedef struct sample_in {
    kssd_seqbuf_t buf;
    char anno[PATHLEN];
} sample_in_t;

void kssd_autosketch_to_dir(const char *input, const kssd_autosketch_opt_t *o, const char *outdir)
{
    char **files = NULL;
    const int nfiles = kssd_organize_input(input, &files);
    if (nfiles < 1)
        errx(EXIT_FAILURE, "%s is not a valid FASTA/FASTQ input for auto ANI", input);
    for (int i = 0; i < nfiles; ++i)
        if (strcmp(files[i], "-") && kssd_fastx_fmt(files[i]) == KSSD_FMT_UNKNOWN)
            err(errno, "%s(): %s is not accept format(.fasta,.fastq)", "load_genome_into_single_vec", files[i]);
    const int nsamp = o->asone ? 1 : nfiles;
    kssd_mkdir_p(outdir);
    sample_in_t *in = calloc((size_t)nfiles, sizeof *in);
    if (!in)
        err(errno, "out of memory");
    bool stream_input = false;
    for (int i = 0; i < nfiles; ++i)
        stream_input |= !strcmp(files[i], "-");
    /* read the files (independent, so in parallel) */
    int bad = -1;
    char bad_msg[1024] = {0};
#pragma omp parallel for num_threads(o->threads > 0 ? o->threads : 1) schedule(dynamic, 1)
    for (int i = 0; i < nfiles; ++i) {
        kssd_seqbuf_init(&in[i].buf);
        if (kssd_fastx_append(files[i], &in[i].buf, in[i].anno) != 0) {
#pragma omp critical
            if (bad < 0) {
                bad = i;
                snprintf(bad_msg, sizeof bad_msg, "%s", kssd_host_last_error());
            }
        }
    }
    if (bad >= 0)
        errx(EXIT_FAILURE, "%s", bad_msg);
    /* per-sample statistics (src/command_sketch.c:4462-4468, 5435-5476) */
    kssd_infile_meta_t *meta = calloc((size_t)nsamp, sizeof *meta);
    char(*names)[PATHLEN] = calloc((size_t)nsamp, PATHLEN);
    if (!meta || !names)
        err(errno, "out of memory");
    if (o->asone) {
        int8_t fmt = KSSD_FMT_UNKNOWN;
        uint8_t flags = FLAG_MIXED_FORMAT;
        for (int f = 0; f < nfiles; ++f) {
            const int8_t this_fmt = (int8_t)kssd_fastx_fmt(files[f]);
            flags |= flags_of(files[f]);
            fmt = f == 0 ? this_fmt : (fmt != this_fmt ? KSSD_FMT_UNKNOWN : fmt);
        }
        if (fmt != KSSD_FMT_UNKNOWN)
            flags &= (uint8_t)~FLAG_MIXED_FORMAT;
        uint64_t *lens = NULL;
        size_t nl = 0;
        if (fmt == KSSD_FMT_FASTA) {
            for (int f = 0; f < nfiles; ++f)
                nl += in[f].buf.nlens;
            lens = malloc((nl ? nl : 1) * sizeof(uint64_t));
            nl = 0;
            for (int f = 0; f < nfiles; ++f) {
                memcpy(lens + nl, in[f].buf.lens, in[f].buf.nlens * sizeof(uint64_t));
                nl += in[f].buf.nlens;
            }
        }
        meta_from_lengths(lens, nl, fmt, CREATE_ASONE, flags, &meta[0]);
        free(lens);
        snprintf(names[0], PATHLEN, "%s", files[0]);
    } else {
        for (int f = 0; f < nfiles; ++f) {
            const int8_t fmt = (int8_t)kssd_fastx_fmt(files[f]);
            meta_from_lengths(fmt == KSSD_FMT_FASTA ? in[f].buf.lens : NULL, fmt == KSSD_FMT_FASTA ? in[f].buf.nlens : 0,
                              fmt, CREATE_NORMAL, flags_of(files[f]), &meta[f]);
            snprintf(names[f], PATHLEN, "%s", files[f]);
        }
    }
    /* the k-mers on the device, in batches of whole samples */
    kssdgpu_sketch_params_t prm = {o->tmpl.klen, o->tmpl.coden_len, o->tmpl.hclen, o->tmpl.holen, o->tmpl.drfold,
                                   o->tmpl.conflict ? 1 : 0};
    uint64_t *keys = NULL, nkeys = 0, kcap = 0;
    uint64_t *offs = calloc((size_t)nsamp + 1, sizeof(uint64_t));
    if (!offs)
        err(errno, "out of memory");
    int s0 = 0;
    while (s0 < nsamp) {
        /* samples s0..s1 (files f0..f1) up to the batch size, at least one */
        int s1 = s0;
        uint64_t bytes = 0;
        do {
            const int fb = o->asone ? 0 : s1, fe = o->asone ? nfiles : s1 + 1;
            for (int f = fb; f < fe; ++f)
                bytes += in[f].buf.len;
            ++s1;
        } while (s1 < nsamp && bytes + in[o->asone ? 0 : s1].buf.len <= SKETCH_BATCH_BYTES);
        const int f0 = o->asone ? 0 : s0, f1 = o->asone ? nfiles : s1;
        uint64_t nrec = 0;
        for (int f = f0; f < f1; ++f)
            nrec += in[f].buf.nrec;
        char *seq = malloc(bytes ? bytes : 1);
        uint64_t *rec = malloc((nrec + 1) * sizeof(uint64_t));
        uint64_t *samp = malloc(((size_t)(s1 - s0) + 1) * sizeof(uint64_t));
        if (!seq || !rec || !samp)
            err(errno, "out of memory");
        uint64_t at = 0, r = 0;
        rec[0] = 0;
        samp[0] = 0;
        for (int f = f0; f < f1; ++f) {
            const kssd_seqbuf_t *b = &in[f].buf;
            memcpy(seq + at, b->seq, b->len);
            for (uint64_t k = 0; k < b->nrec; ++k)
                rec[++r] = at + b->rec[k + 1];
            at += b->len;
            if (!o->asone)
                samp[f - f0 + 1] = r;
        }
        if (o->asone)
            samp[1] = r;
        const int ns = s1 - s0;
        uint64_t cap = bytes / 64 + 4096;
        for (;;) {
            if (nkeys + cap > kcap) {
                kcap = nkeys + cap;
                keys = realloc(keys, kcap * sizeof(uint64_t));
                if (!keys)
                    err(errno, "out of memory");
            }
            const int rc = kssdgpu_sketch(seq, bytes, rec, nrec, samp, ns, &prm, keys + nkeys, cap, offs + s0);
            if (rc == KSSDGPU_ERR_CAPACITY && offs[s0 + ns] > cap) {
                cap = offs[s0 + ns];
                continue;
            }
            if (rc)
                errx(EXIT_FAILURE, "sketching on the GPU failed: %s", kssdgpu_last_error());
            break;
        }
        /* offs of this batch are relative to its first sample */
        const uint64_t got = offs[s0 + ns];
        for (int s = ns; s >= 0; --s)
            offs[s0 + s] += nkeys;
        nkeys += got;
        free(seq);
        free(rec);
        free(samp);
        s0 = s1;
    }
    /* the directory (src/command_sketch.c:989-1005, 1242-1249) */
    kssd_sketch_stat_t st = o->tmpl;
    if (kssd_sketch_write(outdir, &st, nsamp, (const char(*)[PATHLEN])names, keys ? keys : offs, offs))
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    write_file(outdir, "lcofiles.infilemeta", meta, (size_t)nsamp * sizeof *meta);
    if (o->anno && !stream_input) {
        char(*an)[PATHLEN] = calloc((size_t)nsamp, PATHLEN);
        for (int s = 0; s < nsamp; ++s)
            memcpy(an[s], in[s].anno, PATHLEN);
        write_file(outdir, "lcofiles.anno", an, (size_t)nsamp * PATHLEN);
        free(an);
    }
    for (int i = 0; i < nfiles; ++i)
        kssd_seqbuf_free(&in[i].buf);
    free(in);
    free(meta);
    free(names);
    free(keys);
    free(offs);
    kssd_free_paths(files, nfiles);
}

void kssd_merge_sketch_dirs(char **dirs, int n, const char *outdir)
{
    /* src/command_sketch.c:1633-1850 for the files the counting engine reads */
    kssd_mkdir_p(outdir);
    size_t sz = 0;
    kssd_sketch_stat_t first;
    void *m = read_file(dirs[0], "lcofiles.stat", &sz, true);
    memcpy(&first, m, sizeof first);
    free(m);
    kssd_sketch_stat_t all = first;
    all.infile_num = 0;
    char(*names)[PATHLEN] = NULL;
    uint64_t *index = calloc(1, sizeof(uint64_t));
    kssd_infile_meta_t *meta = NULL;
    char(*anno)[PATHLEN] = NULL;
    bool write_meta = false, seen_meta = false, seen_no_meta = false, write_anno = false;
    char out[2 * PATHLEN];
    snprintf(out, sizeof out, "%s/comblco", outdir);
    FILE *comb = fopen(out, "wb");
    if (!comb)
        err(errno, "%s", out);
    for (int i = 0; i < n; ++i) {
        void *sm = read_file(dirs[i], "lcofiles.stat", &sz, true);
        kssd_sketch_stat_t it;
        memcpy(&it, sm, sizeof it);
        if (it.hash_id != first.hash_id)
            err(EINVAL, "%uth %s hashid: %u != %u ", i, dirs[i], it.hash_id, first.hash_id);
        if (!it.koc)
            all.koc = false;
        const int old = all.infile_num, now = old + it.infile_num;
        names = realloc(names, (size_t)(now > 0 ? now : 1) * PATHLEN);
        memcpy(names + old, (char *)sm + sizeof it, (size_t)it.infile_num * PATHLEN);
        free(sm);
        size_t isz = 0;
        uint64_t *idx = read_file(dirs[i], "comblco.index", &isz, true);
        index = realloc(index, ((size_t)now + 1) * sizeof(uint64_t));
        for (int j = 1; j <= it.infile_num; ++j)
            index[old + j] = index[old] + idx[j];
        free(idx);
        size_t msz = 0;
        kssd_infile_meta_t *mi = read_file(dirs[i], "lcofiles.infilemeta", &msz, false);
        seen_meta |= mi != NULL;
        seen_no_meta |= mi == NULL;
        if (mi || write_meta) {
            meta = realloc(meta, (size_t)(now > 0 ? now : 1) * sizeof *meta);
            if (!write_meta && old > 0)
                memset(meta, 0, (size_t)old * sizeof *meta);
            if (mi) {
                if (msz != (size_t)it.infile_num * sizeof *meta)
                    err(EINVAL, "%s(): %s/%s has %zu bytes, expected %zu", "merge_comblco", dirs[i],
                         "lcofiles.infilemeta", msz, (size_t)it.infile_num * sizeof *meta);
                memcpy(meta + old, mi, msz);
            } else {
                memset(meta + old, 0, (size_t)it.infile_num * sizeof *meta);
            }
            write_meta = true;
        }
        free(mi);
        size_t asz = 0;
        char(*ai)[PATHLEN] = read_file(dirs[i], "lcofiles.anno", &asz, false);
        if (ai || write_anno) {
            anno = realloc(anno, (size_t)(now > 0 ? now : 1) * PATHLEN);
            if (!write_anno && old > 0)
                memset(anno, 0, (size_t)old * PATHLEN);
            if (ai) {
                if (asz != (size_t)it.infile_num * PATHLEN)
                    err(EINVAL, "%s(): %s/%s has %zu bytes, expected %zu", "merge_comblco", dirs[i],
                         "lcofiles.anno", asz, (size_t)it.infile_num * PATHLEN);
                memcpy(anno + old, ai, asz);
            } else {
                memset(anno + old, 0, (size_t)it.infile_num * PATHLEN);
            }
            write_anno = true;
        }
        free(ai);
        all.infile_num = now;
        size_t csz = 0;
        void *c = read_file(dirs[i], "comblco", &csz, true);
        if (csz && fwrite(c, 1, csz, comb) != csz)
            err(errno, "%s", out);
        free(c);
    }
    if (fclose(comb) != 0)
        err(errno, "%s", out);
    if (all.koc) {
        snprintf(out, sizeof out, "%s/comblco.a", outdir);
        FILE *ab = fopen(out, "wb");
        if (!ab)
            err(errno, "%s", out);
        for (int i = 0; i < n; ++i) {
            size_t csz = 0;
            void *c = read_file(dirs[i], "comblco.a", &csz, true);
            if (csz && fwrite(c, 1, csz, ab) != csz)
                err(errno, "%s", out);
            free(c);
        }
        if (fclose(ab) != 0)
            err(errno, "%s", out);
    }
    write_file(outdir, "comblco.index", index, ((size_t)all.infile_num + 1) * sizeof(uint64_t));
    {
        const size_t ns = sizeof all + (size_t)all.infile_num * PATHLEN;
        char *buf = malloc(ns);
        memcpy(buf, &all, sizeof all);
        memcpy(buf + sizeof all, names, (size_t)all.infile_num * PATHLEN);
        write_file(outdir, "lcofiles.stat", buf, ns);
        free(buf);
    }
    if (write_meta) {
        if (seen_meta && seen_no_meta)
            memset(meta, 0, (size_t)all.infile_num * sizeof *meta);
        write_file(outdir, "lcofiles.infilemeta", meta, (size_t)all.infile_num * sizeof *meta);
    }
    if (write_anno)
        write_file(outdir, "lcofiles.anno", anno, (size_t)all.infile_num * PATHLEN);
    free(names);
    free(index);
    free(meta);
    free(anno);
}

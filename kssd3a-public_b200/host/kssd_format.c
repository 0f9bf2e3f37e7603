/*
 * Sketch directory and inverted-index I/O (formats described in kssd_format.h).
 * Size checks follow the reference reader: comblco must hold exactly
 * comblco.index[n] keys (src/global_basic.c:1110-1114), the index exactly as many
 * 12-byte records (src/command_ani.c:516), sidecars exactly n records
 * (src/command_ani.c:223-248).
 */
#define _GNU_SOURCE
#include "kssd_format.h"

#include <errno.h>
#include <fcntl.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

static __thread char g_err[1024];

const char *kssd_host_last_error(void) { return g_err; }

static void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

void kssd_host_set_error(const char *msg) { snprintf(g_err, sizeof g_err, "%s", msg); }

bool kssd_file_exists(const char *dir, const char *name)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    return access(p, F_OK) == 0;
}

/* Whole file into memory; large files are read in 64 MB pieces by parallel pread
 * (page-cache copies and first-touch page faults spread over the host cores). */
static void *read_all(const char *dir, const char *name, size_t *size)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    const int fd = open(p, O_RDONLY);
    if (fd < 0) {
        set_err("cannot open %s: %s", p, strerror(errno));
        return NULL;
    }
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        set_err("cannot stat %s", p);
        return NULL;
    }
    const size_t len = (size_t)st.st_size;
    char *buf = malloc(len > 0 ? len : 1);
    if (!buf) {
        close(fd);
        set_err("out of memory reading %s (%zu bytes)", p, len);
        return NULL;
    }
    const size_t piece = (size_t)64 << 20;
    const long npieces = (long)((len + piece - 1) / piece);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad) if (npieces > 1)
    for (long c = 0; c < npieces; ++c) {
        const size_t off = (size_t)c * piece, want = len - off < piece ? len - off : piece;
        size_t got = 0;
        while (got < want) {
            const ssize_t r = pread(fd, buf + off + got, want - got, (off_t)(off + got));
            if (r < 0 && errno == EINTR)
                continue;
            if (r <= 0) {
                bad = 1;
                break;
            }
            got += (size_t)r;
        }
    }
    close(fd);
    if (bad) {
        free(buf);
        set_err("short read on %s", p);
        return NULL;
    }
    *size = len;
    return buf;
}

static int write_all(const char *dir, const char *name, const void *a, size_t an, const void *b,
                     size_t bn)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "wb");
    if (!f) {
        set_err("cannot create %s: %s", p, strerror(errno));
        return -1;
    }
    int ok = (an == 0 || fwrite(a, 1, an, f) == an) && (bn == 0 || fwrite(b, 1, bn, f) == bn);
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        set_err("write failed on %s", p);
        return -1;
    }
    return 0;
}

void kssd_stat_bits(const kssd_sketch_stat_t *st, int *ctx_bits, int *obj_bits)
{
    const int ctx = st->coden_len > 0 ? 4 * st->coden_len : 4 * st->hclen;
    if (ctx_bits)
        *ctx_bits = ctx;
    if (obj_bits)
        *obj_bits = 2 * st->klen - ctx;
}

int kssd_read_stat(const char *dir, kssd_sketch_stat_t *out)
{
    size_t sz = 0;
    void *b = read_all(dir, "lcofiles.stat", &sz);
    if (!b)
        return -1;
    if (sz < sizeof(kssd_sketch_stat_t)) {
        free(b);
        set_err("%s/lcofiles.stat has %zu bytes, expected at least %zu", dir, sz,
                sizeof(kssd_sketch_stat_t));
        return -1;
    }
    memcpy(out, b, sizeof *out);
    free(b);
    return 0;
}

kssd_sketch_t *kssd_sketch_load(const char *dir, unsigned flags)
{
    kssd_sketch_t *s = calloc(1, sizeof *s);
    if (!s) {
        set_err("out of memory");
        return NULL;
    }
    size_t sz = 0;
    char *stat = read_all(dir, "lcofiles.stat", &sz);
    if (!stat)
        goto fail;
    if (sz < sizeof(kssd_sketch_stat_t)) {
        set_err("%s/lcofiles.stat too short", dir);
        free(stat);
        goto fail;
    }
    memcpy(&s->stat, stat, sizeof s->stat);
    s->n = s->stat.infile_num;
    if (s->n < 0 || sz < sizeof(kssd_sketch_stat_t) + (size_t)s->n * KSSD_PATHLEN) {
        set_err("%s/lcofiles.stat: %zu bytes cannot hold %d names", dir, sz, s->n);
        free(stat);
        goto fail;
    }
    s->names = malloc((size_t)(s->n ? s->n : 1) * KSSD_PATHLEN);
    if (!s->names) {
        free(stat);
        set_err("out of memory");
        goto fail;
    }
    memcpy(s->names, stat + sizeof(kssd_sketch_stat_t), (size_t)s->n * KSSD_PATHLEN);
    for (int i = 0; i < s->n; i++)
        s->names[i][KSSD_PATHLEN - 1] = '\0';
    free(stat);
    kssd_stat_bits(&s->stat, &s->ctx_bits, &s->obj_bits);

    size_t isz = 0;
    s->offs = read_all(dir, "comblco.index", &isz);
    if (!s->offs)
        goto fail;
    if (isz < (size_t)(s->n + 1) * sizeof(uint64_t)) {
        set_err("%s/comblco.index has %zu bytes, expected %zu", dir, isz,
                (size_t)(s->n + 1) * sizeof(uint64_t));
        goto fail;
    }
    for (int i = 0; i < s->n; i++)
        if (s->offs[i + 1] < s->offs[i]) {
            set_err("%s/comblco.index is not monotone at sample %d", dir, i);
            goto fail;
        }
    size_t ksz = 0;
    s->keys = read_all(dir, "comblco", &ksz);
    if (!s->keys)
        goto fail;
    const size_t expect = (size_t)s->offs[s->n] * sizeof(uint64_t);
    if (ksz != expect) {
        set_err("%s/comblco has %zu bytes, expected %zu", dir, ksz, expect);
        goto fail;
    }
    if ((flags & 1u) && kssd_file_exists(dir, "lcofiles.anno")) {
        size_t asz = 0;
        s->anno = read_all(dir, "lcofiles.anno", &asz);
        if (!s->anno)
            goto fail;
        if (asz != (size_t)s->n * KSSD_PATHLEN) {
            set_err("%s/lcofiles.anno has %zu bytes, expected %zu", dir, asz,
                    (size_t)s->n * KSSD_PATHLEN);
            goto fail;
        }
    }
    if ((flags & 2u) && kssd_file_exists(dir, "lcofiles.infilemeta")) {
        size_t msz = 0;
        s->meta = read_all(dir, "lcofiles.infilemeta", &msz);
        if (!s->meta)
            goto fail;
        if (msz != (size_t)s->n * sizeof(kssd_infile_meta_t)) {
            set_err("%s/lcofiles.infilemeta has %zu bytes, expected %zu", dir, msz,
                    (size_t)s->n * sizeof(kssd_infile_meta_t));
            goto fail;
        }
    }
    return s;
fail:
    kssd_sketch_free(s);
    return NULL;
}

void kssd_sketch_free(kssd_sketch_t *s)
{
    if (!s)
        return;
    free(s->names);
    free(s->keys);
    free(s->offs);
    free(s->anno);
    free(s->meta);
    free(s);
}

int kssd_sketch_write(const char *dir, const kssd_sketch_stat_t *stat, int n,
                      const char (*names)[KSSD_PATHLEN], const uint64_t *keys,
                      const uint64_t *offs)
{
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) {
        set_err("cannot create %s: %s", dir, strerror(errno));
        return -1;
    }
    kssd_sketch_stat_t st = *stat;
    st.infile_num = n;
    if (write_all(dir, "lcofiles.stat", &st, sizeof st, names, (size_t)n * KSSD_PATHLEN))
        return -1;
    if (write_all(dir, "comblco", keys, (size_t)offs[n] * sizeof(uint64_t), NULL, 0))
        return -1;
    if (write_all(dir, "comblco.index", offs, (size_t)(n + 1) * sizeof(uint64_t), NULL, 0))
        return -1;
    return 0;
}

kssd_index_rec_t *kssd_index_load(const char *dir, size_t *n_out)
{
    size_t sz = 0;
    kssd_index_rec_t *r = read_all(dir, "sortedcomb_ctxgid64obj32", &sz);
    if (!r)
        return NULL;
    if (sz % sizeof(kssd_index_rec_t)) {
        free(r);
        set_err("%s/sortedcomb_ctxgid64obj32 size %zu is not a multiple of 12", dir, sz);
        return NULL;
    }
    *n_out = sz / sizeof(kssd_index_rec_t);
    return r;
}

int kssd_index_write(const char *dir, const kssd_index_rec_t *recs, size_t n,
                     const uint8_t *unique_bits)
{
    if (write_all(dir, "sortedcomb_ctxgid64obj32", recs, n * sizeof(*recs), NULL, 0))
        return -1;
    if (unique_bits &&
        write_all(dir, "sortedcomb_ctxgid64obj32.unique_bits", unique_bits, (n + 7) / 8, NULL, 0))
        return -1;
    return 0;
}

uint32_t *kssd_abundance_load(const char *dir, size_t *n_out)
{
    size_t sz = 0;
    uint32_t *a = read_all(dir, "comblco.a", &sz);
    if (!a)
        return NULL;
    *n_out = sz / sizeof(uint32_t);
    if (sz % sizeof(uint32_t)) {
        free(a);
        set_err("%s/comblco.a size %zu is not a multiple of 4", dir, sz);
        return NULL;
    }
    return a;
}

uint8_t *kssd_unique_bits_load(const char *dir, size_t *bytes_out)
{
    size_t sz = 0;
    uint8_t *b = read_all(dir, "sortedcomb_ctxgid64obj32.unique_bits", &sz);
    if (!b)
        return NULL;
    *bytes_out = sz;
    return b;
}

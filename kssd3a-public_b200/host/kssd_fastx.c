/* FASTA/FASTQ reading for the sketcher (see kssd_fastx.h for the rules followed). */
#include "kssd_fastx.h"

#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <zlib.h>

static void fail_msg(const char *fmt, const char *a, const char *b)
{
    char m[1024];
    snprintf(m, sizeof m, fmt, a, b);
    kssd_host_set_error(m);
}

void kssd_seqbuf_init(kssd_seqbuf_t *b) { memset(b, 0, sizeof *b); }

void kssd_seqbuf_free(kssd_seqbuf_t *b)
{
    free(b->seq);
    free(b->rec);
    free(b->lens);
    memset(b, 0, sizeof *b);
}

static int grow(void **p, uint64_t *cap, uint64_t need, size_t elem)
{
    if (need <= *cap)
        return 0;
    uint64_t c = *cap ? *cap : 1024;
    while (c < need)
        c <<= 1;
    void *q = realloc(*p, c * elem);
    if (!q) {
        kssd_host_set_error("out of memory reading sequence");
        return -1;
    }
    *p = q;
    *cap = c;
    return 0;
}

static int put_byte(kssd_seqbuf_t *b, char c)
{
    if (b->len == b->cap && grow((void **)&b->seq, &b->cap, b->len + 1, 1))
        return -1;
    b->seq[b->len++] = c;
    return 0;
}

/* buffered byte stream over zlib (plain files read through unchanged) */
typedef struct {
    gzFile gz;
    unsigned char *buf;
    int pos, n;
    bool eof, error;
} zstream_t;

static int zgetc(zstream_t *z)
{
    if (z->pos == z->n) {
        if (z->eof)
            return -1;
        z->n = gzread(z->gz, z->buf, 1 << 20);
        z->pos = 0;
        if (z->n <= 0) {
            if (z->n < 0)
                z->error = true;
            z->eof = true;
            z->n = 0;
            return -1;
        }
    }
    return z->buf[z->pos++];
}

/* bytes up to '\n' (consumed, not stored) appended to b's sequence, or skipped
 * (b == NULL); returns the number of bytes taken, -1 at end of stream */
static int64_t rest_of_line(zstream_t *z, kssd_seqbuf_t *b, int *last)
{
    int64_t n = 0;
    int c;
    *last = -1;
    while ((c = zgetc(z)) >= 0 && c != '\n') {
        if (b && put_byte(b, (char)c))
            return -2;
        *last = c;
        ++n;
    }
    return c < 0 && n == 0 ? -1 : n;
}

static void anno_copy(char *dest, const char *name)
{
    /* src/command_sketch.c:1012-1029 with the header line as the name and no comment */
    memset(dest, 0, KSSD_PATHLEN);
    size_t pos = 0;
    for (const char *s = name; *s && pos < KSSD_PATHLEN - 1; ++s) {
        const unsigned char c = (unsigned char)*s;
        dest[pos++] = (c < 32 || c == 127 || c == '\t') ? ' ' : (char)c;
    }
}

int kssd_fastx_append(const char *path, kssd_seqbuf_t *b, char *anno)
{
    if (anno)
        memset(anno, 0, KSSD_PATHLEN);
    gzFile gz;
    if (!strcmp(path, "-")) {
        int fd = dup(0);
        gz = fd >= 0 ? gzdopen(fd, "r") : NULL;
    } else {
        gz = gzopen(path, "r");
    }
    if (!gz) {
        fail_msg("cannot open %s: %s", path, strerror(errno ? errno : EIO));
        return -1;
    }
    gzbuffer(gz, 4u << 20);
    zstream_t z = {gz, malloc(1 << 20), 0, 0, false, false};
    if (!z.buf) {
        gzclose(gz);
        kssd_host_set_error("out of memory reading sequence");
        return -1;
    }
    if (!b->rec && grow((void **)&b->rec, &b->rec_cap, 1, sizeof(uint64_t))) {
        free(z.buf);
        gzclose(gz);
        return -1;
    }
    if (b->nrec == 0)
        b->rec[0] = b->len;
    int rc = 0, c = 0, last_char = 0;
    bool first = true;
    char *header = NULL;
    size_t hcap = 0;
    for (;;) {
        if (last_char == 0) {  /* to the next header character */
            while ((c = zgetc(&z)) >= 0 && c != '>' && c != '@')
                ;
            if (c < 0)
                break;
        }
        /* header line (whole line; one trailing '\r' dropped when longer than one byte) */
        size_t hl = 0;
        while ((c = zgetc(&z)) >= 0 && c != '\n') {
            if (hl + 2 > hcap) {
                hcap = hcap ? 2 * hcap : 256;
                char *h = realloc(header, hcap);
                if (!h) {
                    rc = -1;
                    kssd_host_set_error("out of memory reading sequence");
                    goto done;
                }
                header = h;
            }
            header[hl++] = (char)c;
        }
        if (c < 0 && hl == 0)
            break;  /* a header character at the end of the stream starts no record */
        if (hl > 1 && header[hl - 1] == '\r')
            --hl;
        if (header)
            header[hl] = 0;
        if (first && anno)
            anno_copy(anno, header ? header : "");
        first = false;
        /* sequence lines */
        const uint64_t start = b->len;
        while ((c = zgetc(&z)) >= 0 && c != '>' && c != '+' && c != '@') {
            if (c == '\n')
                continue;
            if (put_byte(b, (char)c)) {
                rc = -1;
                goto done;
            }
            int last;
            if (rest_of_line(&z, b, &last) == -2) {
                rc = -1;
                goto done;
            }
            if (b->len - start > 1 && b->seq[b->len - 1] == '\r')
                --b->len;
        }
        last_char = (c == '>' || c == '@') ? c : 0;
        const uint64_t slen = b->len - start;
        if (c == '+') {
            /* FASTQ: skip the '+' line, then quality lines until they cover the sequence */
            int last;
            while ((c = zgetc(&z)) >= 0 && c != '\n')
                ;
            if (c < 0) {
                b->len = start;  /* no quality: the record and the rest of the file are dropped */
                break;
            }
            uint64_t ql = 0;
            for (;;) {
                const int64_t n = rest_of_line(&z, NULL, &last);
                if (n < 0)
                    break;
                ql += (uint64_t)n - (n > 1 && last == '\r' ? 1 : 0);
                if (ql >= slen)
                    break;
            }
            last_char = 0;
            if (ql != slen) {
                b->len = start;  /* quality of another length: stops like the reference's loop */
                break;
            }
        }
        /* the record */
        if (grow((void **)&b->rec, &b->rec_cap, b->nrec + 2, sizeof(uint64_t))) {
            rc = -1;
            goto done;
        }
        b->rec[++b->nrec] = b->len;
        if (slen) {
            if (grow((void **)&b->lens, &b->lens_cap, b->nlens + 1, sizeof(uint64_t))) {
                rc = -1;
                goto done;
            }
            b->lens[b->nlens++] = slen;
        }
        if (c < 0)
            break;
    }
done:
    if (rc == 0 && z.error) {
        fail_msg("error reading %s%s", path, "");
        rc = -1;
    }
    free(header);
    free(z.buf);
    gzclose(gz);
    return rc;
}

static const char *strip_compress(const char *path, char *tmp)
{
    static const char *cmp[2] = {".gz", ".bz2"};
    const size_t n = strlen(path);
    for (int i = 0; i < 2; ++i) {
        const size_t m = strlen(cmp[i]);
        if (n >= m && !strcmp(path + n - m, cmp[i])) {
            snprintf(tmp, KSSD_PATHLEN, "%.*s", (int)(n - m), path);
            return tmp;
        }
    }
    return path;
}

static bool has_suffix_in(const char *path, const char *const *fmts, int nf)
{
    char tmp[KSSD_PATHLEN];
    const char *p = strip_compress(path, tmp);
    const size_t n = strlen(p);
    for (int i = 0; i < nf; ++i) {
        char suf[16];
        snprintf(suf, sizeof suf, ".%s", fmts[i]);
        const size_t m = strlen(suf);
        if (n >= m && !strcmp(p + n - m, suf))
            return true;
    }
    return false;
}

int kssd_fastx_fmt(const char *path)
{
    static const char *fq[] = {"fq", "fastq"};
    static const char *fa[] = {"fasta", "fna", "fas", "fa"};
    if (!path)
        return KSSD_FMT_UNKNOWN;
    if (has_suffix_in(path, fq, 2))
        return KSSD_FMT_FASTQ;
    if (has_suffix_in(path, fa, 4))
        return KSSD_FMT_FASTA;
    return KSSD_FMT_UNKNOWN;
}

bool kssd_fastx_accepted(const char *path)
{
    static const char *acpt[] = {"fna", "fas", "fasta", "fq", "fastq", "fa", "co"};
    return has_suffix_in(path, acpt, 7);
}

bool kssd_name_compressed(const char *path)
{
    const size_t n = strlen(path);
    return (n >= 3 && !strcmp(path + n - 3, ".gz")) || (n >= 4 && !strcmp(path + n - 4, ".bz2"));
}

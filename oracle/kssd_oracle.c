/*
 * ORACLE — test infrastructure only (see kssd_oracle.h).  A CPU restatement of
 * the reference's shared-context counting, written for clarity: plain binary
 * search for each query context, then a walk of that context's postings.  The
 * counting rules follow src/command_ani.h:463-721 exactly; every function cites
 * the reference lines whose behaviour it restates.
 */
#include "kssd_oracle.h"

#include <stdlib.h>
#include <string.h>

/* NUM_CODENS + 1 with the default NUM_CODENS = 11 (src/command_ani.h:547,684). */
#define ORC_MIN_INIT 12

typedef struct __attribute__((packed)) {
    uint64_t ctxgid;
    uint32_t obj;
} orc_rec_t;

int orc_dna_popcount(uint32_t x)
{
    /* a differing 2-bit base sets at least one of its two bits (src/dna_popcount.h:45-49) */
    uint32_t any = (x | (x >> 1)) & 0x55555555u;
    return __builtin_popcount(any);
}

static int rec_cmp(const void *pa, const void *pb)
{
    const orc_rec_t *a = pa, *b = pb;
    if (a->ctxgid != b->ctxgid)
        return a->ctxgid < b->ctxgid ? -1 : 1;
    if (a->obj != b->obj)
        return a->obj < b->obj ? -1 : 1;
    return 0;
}

size_t orc_build_index(const uint64_t *keys, const uint64_t *offs, int nsamples, int obj_bits,
                       void *out_records)
{
    orc_rec_t *r = out_records;
    const uint64_t objmask = (obj_bits >= 64) ? ~0ull : ((1ull << obj_bits) - 1);
    const uint64_t gidmask = (1ull << ORC_GID_BITS) - 1;
    size_t n = 0;
    for (int g = 0; g < nsamples; g++) {
        for (uint64_t i = offs[g]; i < offs[g + 1]; i++) {
            r[n].ctxgid = ((keys[i] >> obj_bits) << ORC_GID_BITS) | ((uint64_t)g & gidmask);
            r[n].obj = (uint32_t)(keys[i] & objmask);
            n++;
        }
    }
    qsort(r, n, sizeof(orc_rec_t), rec_cmp);
    return n;
}

uint64_t orc_unique_bits(const void *records, size_t len, uint8_t *bits)
{
    /* For each ctx group, an obj value that occurs exactly once marks its record. */
    const orc_rec_t *r = records;
    uint64_t marked = 0;
    memset(bits, 0, (len + 7) / 8);
    size_t i = 0;
    while (i < len) {
        const uint64_t ctx = r[i].ctxgid >> ORC_GID_BITS;
        size_t j = i + 1;
        while (j < len && (r[j].ctxgid >> ORC_GID_BITS) == ctx)
            j++;
        for (size_t a = i; a < j; a++) {
            int count = 0;
            for (size_t b = i; b < j; b++)
                count += r[b].obj == r[a].obj;
            if (count == 1) {
                bits[a >> 3] |= (uint8_t)(1u << (a & 7));
                marked++;
            }
        }
        i = j;
    }
    return marked;
}

void orc_ref_ctx_counts(const void *records, size_t len, int nref, const uint64_t *ref_offs,
                        int conflict, int ignoreconflict, uint32_t *out)
{
    const orc_rec_t *r = records;
    for (int g = 0; g < nref; g++)
        out[g] = (uint32_t)(ref_offs[g + 1] - ref_offs[g]);
    if (!conflict)
        return;
    /* A (ctx,gid) run of length L > 1 is one context (L-1 removed), or none with
     * --ignoreconflict (L removed). */
    size_t i = 0;
    while (i < len) {
        size_t j = i + 1;
        while (j < len && r[j].ctxgid == r[i].ctxgid)
            j++;
        const size_t run = j - i;
        if (run > 1) {
            const uint32_t gid = (uint32_t)(r[i].ctxgid & ((1ull << ORC_GID_BITS) - 1));
            out[gid] -= (uint32_t)(ignoreconflict ? run : run - 1);
        }
        i = j;
    }
}

void orc_sample_ctx_counts(const uint64_t *keys, const uint64_t *offs, int nsamples, int obj_bits,
                           int conflict, int ignoreconflict, uint32_t *out)
{
    for (int g = 0; g < nsamples; g++) {
        const uint64_t b = offs[g], e = offs[g + 1];
        if (!conflict) {
            out[g] = (uint32_t)(e - b);
            continue;
        }
        uint32_t runs = 0;
        uint64_t i = b;
        while (i < e) {
            const uint64_t ctx = keys[i] >> obj_bits;
            uint64_t j = i + 1;
            while (j < e && (keys[j] >> obj_bits) == ctx)
                j++;
            if (!ignoreconflict || j - i == 1)
                runs++;
            i = j;
        }
        out[g] = runs;
    }
}

void orc_unique_ref_totals(const void *records, size_t len, int nref, int ignoreconflict,
                           uint32_t *out)
{
    const orc_rec_t *r = records;
    memset(out, 0, sizeof(uint32_t) * (size_t)nref);
    size_t i = 0;
    while (i < len) {
        const uint64_t ctx = r[i].ctxgid >> ORC_GID_BITS;
        size_t j = i + 1;
        int single_owner = 1;
        while (j < len && (r[j].ctxgid >> ORC_GID_BITS) == ctx) {
            if (r[j].ctxgid != r[i].ctxgid)
                single_owner = 0;
            j++;
        }
        const uint32_t gid = (uint32_t)(r[i].ctxgid & ((1ull << ORC_GID_BITS) - 1));
        if (single_owner && (!ignoreconflict || j - i == 1) && gid < (uint32_t)nref)
            out[gid]++;
        i = j;
    }
}

/* first record index whose ctx >= target (records sorted by ctxgid) */
static size_t lower_bound_ctx(const orc_rec_t *r, size_t len, uint64_t target)
{
    size_t lo = 0, hi = len;
    while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if ((r[mid].ctxgid >> ORC_GID_BITS) < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static int min_diff(const uint64_t *q, size_t qn, uint64_t objmask, const orc_rec_t *r,
                    size_t rb, size_t re)
{
    int best = ORC_MIN_INIT;
    for (size_t a = 0; a < qn; a++)
        for (size_t b = rb; b < re; b++) {
            const uint32_t x = (uint32_t)(q[a] & objmask) ^ r[b].obj;
            const int d = x ? orc_dna_popcount(x) : 0;
            if (d < best)
                best = d;
        }
    return best;
}

static inline void add_cell(uint32_t *ctx2, uint32_t *obj2, size_t cell, int d)
{
    ctx2[2 * cell] += 1;
    if (d > 0) {
        obj2[2 * cell] += 1;
        obj2[2 * cell + 1] += (uint32_t)d;
        if (d > 1)
            ctx2[2 * cell + 1] += 1;
    }
}

/* One query sample against the whole index.  lower_gid >= 0 restricts the walk to
 * gid < lower_gid (the self lower triangle, src/command_ani.h:694-699). */
static void count_one(const orc_rec_t *r, size_t len, int nref, const uint64_t *a, size_t an,
                      int obj_bits, int ignoreconflict, int lower_gid, size_t row,
                      uint32_t *ctx2, uint32_t *obj2, uint32_t *uctx2, uint32_t *uobj2)
{
    const uint64_t objmask = (obj_bits >= 64) ? ~0ull : ((1ull << obj_bits) - 1);
    const uint64_t gidmask = (1ull << ORC_GID_BITS) - 1;
    size_t j = 0;
    while (j < an) {
        const uint64_t ctx = a[j] >> obj_bits;
        size_t s = 1;
        while (j + s < an && (a[j + s] >> obj_bits) == ctx)
            s++;
        size_t d = lower_bound_ctx(r, len, ctx);
        size_t owners = 0;
        uint32_t sole_gid = 0;
        int sole_diff = 0, sole_allowed = 0;
        while (d < len && (r[d].ctxgid >> ORC_GID_BITS) == ctx) {
            const uint64_t cg = r[d].ctxgid;
            const uint32_t gid = (uint32_t)(cg & gidmask);
            const size_t rb = d;
            while (d < len && r[d].ctxgid == cg)
                d++;
            const size_t re = d;
            owners++;
            sole_gid = gid;
            if (lower_gid >= 0 && (int)gid >= lower_gid)
                break;
            if (ignoreconflict && re - rb > 1)
                continue;
            const int md = min_diff(a + j, s, objmask, r, rb, re);
            add_cell(ctx2, obj2, row * (size_t)nref + gid, md);
            sole_diff = md;
            sole_allowed = 1;
        }
        if (uctx2 && owners == 1 && sole_allowed)
            add_cell(uctx2, uobj2, row * (size_t)nref + sole_gid, sole_diff);
        j += s;
    }
}

int orc_count_block(const void *records, size_t len, int nref,
                    const uint64_t *qkeys, const uint64_t *qoffs, int nq,
                    int obj_bits, int ignoreconflict, int want_unique, int threads,
                    uint32_t *ctx2, uint32_t *obj2, uint32_t *uctx2, uint32_t *uobj2)
{
    const orc_rec_t *r = records;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int q = 0; q < nq; q++) {
        const uint64_t *a = qkeys + (qoffs[q] - qoffs[0]);
        const size_t an = (size_t)(qoffs[q + 1] - qoffs[q]);
        count_one(r, len, nref, a, an, obj_bits, ignoreconflict, -1, (size_t)q, ctx2, obj2,
                  want_unique ? uctx2 : NULL, want_unique ? uobj2 : NULL);
    }
    return 0;
}

int orc_count_lower(const void *records, size_t len, int nref, int qry_gid_offset,
                    const uint64_t *qkeys, const uint64_t *qoffs, int nq,
                    int obj_bits, int ignoreconflict, int threads,
                    uint32_t *ctx2, uint32_t *obj2)
{
    const orc_rec_t *r = records;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int q = 0; q < nq; q++) {
        const uint64_t *a = qkeys + (qoffs[q] - qoffs[0]);
        const size_t an = (size_t)(qoffs[q + 1] - qoffs[q]);
        count_one(r, len, nref, a, an, obj_bits, ignoreconflict, qry_gid_offset + q, (size_t)q,
                  ctx2, obj2, NULL, NULL);
    }
    return 0;
}

void orc_pair_features(const uint64_t *a, size_t n, const uint64_t *b, size_t m, int obj_bits,
                       int ignore_b_conflict, uint32_t out4[4])
{
    const uint64_t objmask = (obj_bits >= 64) ? ~0ull : ((1ull << obj_bits) - 1);
    memset(out4, 0, 4 * sizeof(uint32_t));
    size_t i = 0, j = 0;
    while (i < n && j < m) {
        const uint64_t ca = a[i] >> obj_bits, cb = b[j] >> obj_bits;
        size_t ie = i + 1, je = j + 1;
        while (ie < n && (a[ie] >> obj_bits) == ca)
            ie++;
        while (je < m && (b[je] >> obj_bits) == cb)
            je++;
        if (ca < cb) {
            i = ie;
            continue;
        }
        if (cb < ca) {
            j = je;
            continue;
        }
        if (!(ignore_b_conflict && je - j > 1)) {
            int best = ORC_MIN_INIT;
            for (size_t x = i; x < ie; x++)
                for (size_t y = j; y < je; y++) {
                    const uint32_t d32 = (uint32_t)(a[x] & objmask) ^ (uint32_t)(b[y] & objmask);
                    const int d = d32 ? orc_dna_popcount(d32) : 0;
                    if (d < best)
                        best = d;
                }
            out4[0]++;
            if (best > 0) {
                out4[1]++;
                out4[2] += (uint32_t)best;
                if (best > 1)
                    out4[3]++;
            }
        }
        i = ie;
        j = je;
    }
}

/* Candidate nomination of the indexed sparse scan, src/pairwise_graph.c:1195-1246:
 * for sample q (its keys sorted), every step-th key (position qi*step) whose context
 * the index holds in a group of at most max_freq records (0: any) gives one vote to
 * each record gid < q of the group; first[(q, r)] is the smallest qi that voted for r
 * (UINT32_MAX without a vote).  Cells packed lower-triangular (q*(q-1)/2 + r). */
void orc_self_votes(const void *records, size_t len, const uint64_t *keys, const uint64_t *offs, int nsamples,
                    int obj_bits, uint32_t max_freq, uint32_t step, uint32_t *votes, uint32_t *first)
{
    const orc_rec_t *r = records;
    const size_t cells = (size_t)nsamples * (size_t)(nsamples > 0 ? nsamples - 1 : 0) / 2;
    memset(votes, 0, cells * sizeof(uint32_t));
    for (size_t c = 0; c < cells; c++)
        first[c] = UINT32_MAX;
    for (int q = 1; q < nsamples; q++) {
        const uint64_t *a = keys + (offs[q] - offs[0]);
        const size_t an = (size_t)(offs[q + 1] - offs[q]);
        for (size_t pos = 0, qi = 0; pos < an; pos += step, qi++) {
            const uint64_t ctx = a[pos] >> obj_bits;
            size_t b = lower_bound_ctx(r, len, ctx), e = b;
            while (e < len && (r[e].ctxgid >> ORC_GID_BITS) == ctx)
                e++;
            if (b == e || (max_freq && e - b > max_freq))
                continue;
            for (size_t k = b; k < e; k++) {
                const uint32_t gid = (uint32_t)(r[k].ctxgid & ((1ull << ORC_GID_BITS) - 1));
                if ((int)gid >= q)
                    break;
                const size_t cell = (size_t)q * (q - 1) / 2 + gid;
                votes[cell]++;
                if (qi < first[cell])
                    first[cell] = (uint32_t)qi;
            }
        }
    }
}

/* ---------------------------------------------------------------- sketching (FASTA/FASTQ)
 * The reference's sketch of one genome (src/command_sketch.c:3913-3949 per record, then
 * :4156-4188 sort + dedup and src/kssdlib_sort.c:388-406 conflict removal), restated
 * with a portable bit-extract.  Masks: src/sketch_rearrange.c:7-39 and
 * src/sketch_rearrange.h:109-122 (coden pattern). */

void orc_sketch_masks(int coden_len, int klen, int hclen, int holen, uint64_t *ctxmask, uint64_t *tupmask,
                      int *obj_bits)
{
    uint64_t cm = 0;
    int ctx_bits;
    if (coden_len > 0) {
        /* per coden: 4 context bits over 2 object bits (0b111100), the 11th coden one
         * final 4-bit context group */
        for (int i = 0; i < coden_len; ++i) {
            cm = (cm << 6) | 0x3Cu;
            if (i == 10) {
                cm = (cm << 4) | 0xFu;
                break;
            }
        }
        ctx_bits = 4 * coden_len;
    } else {
        const int iolen = klen - 2 * (hclen + holen);
        const uint64_t hc = hclen ? (~0ull >> (64 - 2 * hclen)) : 0;
        cm = (hc << (2 * (holen + hclen + iolen))) | (hc << (2 * holen));
        ctx_bits = 4 * hclen;
    }
    *ctxmask = cm;
    *tupmask = klen ? (~0ull >> (64 - 2 * klen)) : 0;
    *obj_bits = 2 * klen - ctx_bits;
}

static uint64_t orc_pext(uint64_t x, uint64_t mask)
{
    uint64_t r = 0;
    int k = 0;
    for (int b = 0; b < 64; ++b)
        if ((mask >> b) & 1u)
            r |= ((x >> b) & 1u) << k++;
    return r;
}

/* SplitMix64 finalizer (Steele, Lea, Flood 2014), the sketch's context hash (src/kssdlib_hash.h:16-21) */
static uint64_t orc_splitmix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

static int orc_base(unsigned char c)
{
    switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
    }
}

static int u64_cmp(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

size_t orc_sketch_records(const char *seq, const uint64_t *rec_offs, int nrec, int klen, uint64_t ctxmask,
                          uint64_t tupmask, int obj_bits, uint32_t filter, int conflict, uint64_t *out, size_t cap)
{
    size_t n = 0;
    const int len_mv = 2 * klen - 2;
    const uint64_t objmask = tupmask & ~ctxmask;
    for (int r = 0; r < nrec; ++r) {
        const uint64_t b = rec_offs[r], e = rec_offs[r + 1];
        if (e - b < (uint64_t)klen)
            continue;
        uint64_t tuple = 0, crv = 0;
        int run = 0;
        for (uint64_t p = b; p < e; ++p) {
            const int v = orc_base((unsigned char)seq[p]);
            if (v < 0) {
                run = 0;
                tuple = crv = 0;
                continue;
            }
            tuple = (tuple << 2) | (uint64_t)v;
            crv = (crv >> 2) | ((uint64_t)(v ^ 3) << len_mv);
            if (++run < klen)
                continue;
            const uint64_t tc = tuple & ctxmask, rc = crv & ctxmask;
            const int fwd = tc < rc;
            const uint64_t uctx = fwd ? tc : rc;
            if ((uint32_t)orc_splitmix64(uctx) > filter)
                continue;
            const uint64_t ut = (fwd ? tuple : crv) & tupmask;
            if (n == cap)
                return (size_t)-1;
            out[n++] = (orc_pext(ut, ctxmask) << obj_bits) | orc_pext(ut, objmask);
        }
    }
    qsort(out, n, sizeof(uint64_t), u64_cmp);
    size_t m = 0;
    for (size_t i = 0; i < n; ++i)
        if (i == 0 || out[i] != out[m - 1])
            out[m++] = out[i];
    if (conflict)
        return m;
    /* drop every context that holds more than one object */
    size_t w = 0;
    for (size_t i = 0; i < m;) {
        size_t j = i + 1;
        while (j < m && (out[j] >> obj_bits) == (out[i] >> obj_bits))
            ++j;
        if (j - i == 1)
            out[w++] = out[i];
        i = j;
    }
    return w;
}

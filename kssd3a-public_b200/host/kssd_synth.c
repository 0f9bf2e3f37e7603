/* Synthetic sketch-space genomes; the model is described in kssd_synth.h. */
#include "kssd_synth.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s;
} rng_t;

static inline uint64_t splitmix(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t rnext(rng_t *r) { return splitmix(&r->s); }

static inline double runif(rng_t *r) { return (double)(rnext(r) >> 11) * (1.0 / 9007199254740992.0); }

static inline double rnorm(rng_t *r)
{
    double u1 = runif(r), u2 = runif(r);
    if (u1 < 1e-300)
        u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static uint64_t rpois(rng_t *r, double lambda)
{
    if (lambda <= 0)
        return 0;
    if (lambda < 30) {
        const double L = exp(-lambda);
        uint64_t k = 0;
        double p = 1.0;
        do {
            k++;
            p *= runif(r);
        } while (p > L);
        return k - 1;
    }
    double v = lambda + sqrt(lambda) * rnorm(r) + 0.5;
    return v < 0 ? 0 : (uint64_t)v;
}

static rng_t stream(uint64_t seed, uint64_t tag, uint64_t idx)
{
    rng_t r;
    uint64_t x = seed ^ (tag * 0xD6E8FEB86659FD93ull);
    r.s = splitmix(&x) ^ (idx * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull);
    (void)rnext(&r);
    return r;
}

static double draw_len(const kssd_synth_cfg_t *c, rng_t *r)
{
    double L;
    switch (c->size_dist) {
    case KSSD_SIZE_LOGNORMAL:
        L = c->len_median * exp(c->len_sigma * rnorm(r));
        break;
    case KSSD_SIZE_LOGUNIFORM:
        L = exp(log(c->len_min) + runif(r) * (log(c->len_max) - log(c->len_min)));
        break;
    default:
        L = c->len_median;
    }
    if (L < c->len_min)
        L = c->len_min;
    if (L > c->len_max)
        L = c->len_max;
    return L;
}

typedef struct {
    uint64_t *a;
    size_t n, cap;
} vec_t;

static void vpush(vec_t *v, uint64_t x)
{
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 4096;
        v->a = realloc(v->a, v->cap * sizeof(uint64_t));
    }
    v->a[v->n++] = x;
}

static inline uint64_t fresh_key(const kssd_synth_cfg_t *c, rng_t *r)
{
    const uint64_t ctx = rnext(r) >> (64 - c->ctx_bits);
    const uint64_t obj = rnext(r) & ((1ull << c->obj_bits) - 1);
    return (ctx << c->obj_bits) | obj;
}

/* mutate each object base with probability p (to a different base) */
static inline uint64_t mutate_obj(const kssd_synth_cfg_t *c, rng_t *r, uint64_t key, double p)
{
    const int npos = c->obj_bits / 2;
    for (int b = 0; b < npos; b++)
        if (runif(r) < p)
            key ^= (uint64_t)(1 + rnext(r) % 3) << (2 * b);
    return key;
}

/* ancestor keys of a cluster (unsorted), returns its length; the key stream is
 * independent of the length stream, so ancestors of different lengths share a prefix */
static double ancestor_keys(const kssd_synth_cfg_t *c, int cluster, vec_t *out)
{
    rng_t rl = stream(c->seed, 0xA11CE, (uint64_t)cluster);
    rng_t rk = stream(c->seed, 0xA11CF, (uint64_t)cluster);
    const double L = draw_len(c, &rl);
    const uint64_t m = (uint64_t)llround(L * c->density);
    for (uint64_t i = 0; i < m; i++)
        vpush(out, fresh_key(c, &rk));
    return L;
}

/* homologous copy of an ancestor: keep fraction frac of the keys, each surviving
 * a substitution rate p (context intact) or being replaced by a fresh key */
static void derive(const kssd_synth_cfg_t *c, rng_t *r, const vec_t *anc, double frac, double p,
                   vec_t *out)
{
    const double keep = pow(1.0 - p, c->ctx_bits / 2) * pow(1.0 - c->indel_rate, c->klen);
    for (size_t i = 0; i < anc->n; i++) {
        if (frac < 1.0 && runif(r) >= frac)
            continue;
        if (runif(r) < keep)
            vpush(out, mutate_obj(c, r, anc->a[i], p));
        else
            vpush(out, fresh_key(c, r));
    }
}

static int cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* sort; conflict-free samples keep one object per context, read sets drop exact
 * duplicates only */
static void finish(const kssd_synth_cfg_t *c, vec_t *v, int conflict)
{
    if (v->n == 0)
        return;
    qsort(v->a, v->n, sizeof(uint64_t), cmp_u64);
    size_t w = 1;
    for (size_t i = 1; i < v->n; i++) {
        const uint64_t prev = v->a[w - 1], cur = v->a[i];
        const int dup = conflict ? (cur == prev) : ((cur >> c->obj_bits) == (prev >> c->obj_bits));
        if (!dup)
            v->a[w++] = cur;
    }
    v->n = w;
}

static double gen_member(const kssd_synth_cfg_t *c, uint64_t sample_seed, int idx, vec_t *out)
{
    vec_t anc = {0};
    const int cluster = idx % c->n_clusters;
    const double L = ancestor_keys(c, cluster, &anc);
    rng_t r = stream(sample_seed, 0x5E3B, (uint64_t)idx);
    const double p = c->sub_lo + (c->sub_hi - c->sub_lo) * runif(&r);
    derive(c, &r, &anc, 1.0, p, out);
    free(anc.a);
    return L;
}

static double gen_ownlen(const kssd_synth_cfg_t *c, int idx, vec_t *out)
{
    vec_t anc = {0};
    const int cluster = idx % c->n_clusters;
    const double La = ancestor_keys(c, cluster, &anc);
    rng_t r = stream(c->sample_seed, 0x0E11, (uint64_t)idx);
    const double Ls = exp(log(c->own_len_min) + runif(&r) * (log(c->own_len_max) - log(c->own_len_min)));
    const double p = c->sub_lo + (c->sub_hi - c->sub_lo) * runif(&r);
    derive(c, &r, &anc, Ls < La ? Ls / La : 1.0, p, out);
    if (Ls > La) {
        const uint64_t extra = (uint64_t)llround((Ls - La) * c->density);
        for (uint64_t i = 0; i < extra; i++)
            vpush(out, fresh_key(c, &r));
    }
    free(anc.a);
    return Ls;
}

static double gen_reads(const kssd_synth_cfg_t *c, int idx, vec_t *out)
{
    rng_t r = stream(c->sample_seed, 0x2EAD, (uint64_t)idx);
    const int span = c->reads_max_genomes - c->reads_min_genomes + 1;
    const int g = c->reads_min_genomes + (int)(rnext(&r) % (uint64_t)(span > 0 ? span : 1));
    double total = 0;
    for (int k = 0; k < g; k++) {
        const int gid = (int)(rnext(&r) % (uint64_t)(c->ref_samples > 0 ? c->ref_samples : 1));
        vec_t genome = {0};
        const double L = gen_member(c, c->ref_sample_seed, gid, &genome);
        const double cov = c->cov_lo + (c->cov_hi - c->cov_lo) * runif(&r);
        const double e = c->err_lo + (c->err_hi - c->err_lo) * runif(&r);
        /* a sampled k-mer is seen when at least one 150 bp read covers all of it */
        const double seen = 1.0 - exp(-cov * (150.0 - c->klen + 1.0) / 150.0);
        const double var_rate = cov * (1.0 - pow(1.0 - e, c->obj_bits / 2));
        for (size_t i = 0; i < genome.n; i++) {
            if (runif(&r) >= seen)
                continue;
            vpush(out, genome.a[i]);
            const uint64_t nv = rpois(&r, var_rate);
            for (uint64_t v = 0; v < nv; v++) {
                const int b = (int)(rnext(&r) % (uint64_t)(c->obj_bits / 2));
                vpush(out, genome.a[i] ^ ((uint64_t)(1 + rnext(&r) % 3) << (2 * b)));
            }
        }
        const uint64_t noise = rpois(&r, L * cov * e * (c->ctx_bits / 2) * c->density);
        for (uint64_t i = 0; i < noise; i++)
            vpush(out, fresh_key(c, &r));
        total += L * cov;
        free(genome.a);
    }
    return total;
}

void kssd_synth_default(kssd_synth_cfg_t *c)
{
    memset(c, 0, sizeof *c);
    c->seed = 20261203;
    c->sample_seed = 20261203;
    c->n_samples = 64;
    c->n_clusters = 8;
    c->role = KSSD_ROLE_MEMBER;
    c->size_dist = KSSD_SIZE_FIXED;
    c->len_median = 1e6;
    c->len_sigma = 0.37;
    c->len_min = 1e6;
    c->len_max = 12e6;
    c->own_len_min = 5e4;
    c->own_len_max = 12e6;
    c->sub_lo = 0.005;
    c->sub_hi = 0.05;
    c->indel_rate = 0.001;
    c->density = 1.0 / 256.0;
    c->ctx_bits = 44;
    c->obj_bits = 20;
    c->klen = 32;
    c->reads_min_genomes = 1;
    c->reads_max_genomes = 5;
    c->cov_lo = 5;
    c->cov_hi = 50;
    c->err_lo = 0.001;
    c->err_hi = 0.01;
    c->threads = 0;
}

kssd_synth_out_t *kssd_synth_generate(const kssd_synth_cfg_t *c)
{
    if (c->n_samples < 0 || c->n_clusters <= 0 || c->own_len_min <= 0 || c->own_len_max < c->own_len_min || c->ctx_bits + c->obj_bits > 64 || c->obj_bits > 32 ||
        c->ctx_bits <= 0 || c->obj_bits <= 0)
        return NULL;
    const int n = c->n_samples;
    vec_t *per = calloc((size_t)(n ? n : 1), sizeof(vec_t));
    kssd_synth_out_t *o = calloc(1, sizeof *o);
    o->n = n;
    o->offs = calloc((size_t)n + 1, sizeof(uint64_t));
    o->lengths = calloc((size_t)(n ? n : 1), sizeof(double));
    const int conflict = c->role == KSSD_ROLE_READS;
#pragma omp parallel for schedule(dynamic, 4) num_threads(c->threads > 0 ? c->threads : 8)
    for (int i = 0; i < n; i++) {
        double L;
        if (c->role == KSSD_ROLE_OWNLEN)
            L = gen_ownlen(c, i, &per[i]);
        else if (c->role == KSSD_ROLE_READS)
            L = gen_reads(c, i, &per[i]);
        else
            L = gen_member(c, c->sample_seed, i, &per[i]);
        finish(c, &per[i], conflict);
        o->lengths[i] = L;
    }
    for (int i = 0; i < n; i++)
        o->offs[i + 1] = o->offs[i] + per[i].n;
    o->keys = malloc((size_t)(o->offs[n] ? o->offs[n] : 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(static) num_threads(c->threads > 0 ? c->threads : 8)
    for (int i = 0; i < n; i++) {
        if (per[i].n)
            memcpy(o->keys + o->offs[i], per[i].a, per[i].n * sizeof(uint64_t));
        free(per[i].a);
    }
    free(per);
    return o;
}

void kssd_synth_free(kssd_synth_out_t *o)
{
    if (!o)
        return;
    free(o->keys);
    free(o->offs);
    free(o->lengths);
    free(o);
}

/*
 * --estimate-coverage: abundance-derived coverage columns of the reported detail rows
 * of one query (read sets sketched with k-mer counts, comblco.a).  Restates
 * populate_selected_coverage_for_query_arrays (src/command_ani.c:2315-2455) and the
 * marker lookups before it (:2203-2313): a row's markers are the keys of its reference
 * that are unique -- in the reference database's unique-object bitset when the index
 * and its .unique_bits are present, else among the keys of all the rows' references --
 * and the query's counts of the markers it holds give observed fraction, depth and
 * dispersion; each row's count mass over the rows' total gives its abundance fraction.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "kssd_epilogue.h"

const char kssd_coverage_header[] =
    "Coverage_estimator\tCoverage_ref_markers\tCoverage_observed_markers\tCoverage_observed_fraction\t"
    "Coverage_count_sum\tEstimated_depth\tPositive_mean_depth\tPositive_median_depth\tCount_CV\t"
    "Estimated_abundance_mass\tEstimated_abundance_fraction\tAbundance_fraction_scope";

static int cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

static int cmp_u32(const void *a, const void *b)
{
    const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

/* first position with a[i] >= v (or > v when upper) */
static size_t bound_u64(const uint64_t *a, size_t n, uint64_t v, int upper)
{
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = lo + ((hi - lo) >> 1);
        if (upper ? a[mid] <= v : a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* the record (ctxgid, obj) in the sorted index carries its unique-object bit */
static int refdb_marker(const kssd_cov_refdb_t *db, uint64_t ctxgid, uint32_t obj)
{
    uint64_t lo = 0, hi = db->entries;
    while (lo < hi) {
        const uint64_t mid = lo + ((hi - lo) >> 1);
        const kssd_index_rec_t *v = &db->sorted[mid];
        if (v->ctxgid < ctxgid || (v->ctxgid == ctxgid && v->obj < obj))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < db->entries && db->sorted[lo].ctxgid == ctxgid && db->sorted[lo].obj == obj &&
           (db->bits[lo >> 3] & (uint8_t)(1u << (lo & 7u))) != 0;
}

void kssd_coverage_rows(const uint64_t *q_keys, const uint32_t *q_counts, size_t q_n, const uint64_t *ref_keys,
                        const uint64_t *ref_offs, const kssd_cov_refdb_t *refdb, int obj_bits, kssd_row_t *rows,
                        size_t n_rows)
{
    if (!rows || n_rows == 0)
        return;
    if (!q_keys || !q_counts) {
        for (size_t i = 0; i < n_rows; ++i)
            rows[i].coverage_status = 2;
        return;
    }
    const int use_db = refdb && refdb->available;
    /* without the database bits: the pooled keys of the rows' references */
    uint64_t *pool = NULL;
    size_t pool_n = 0;
    if (!use_db) {
        for (size_t i = 0; i < n_rows; ++i)
            pool_n += (size_t)(ref_offs[rows[i].rn + 1] - ref_offs[rows[i].rn]);
        pool = malloc((pool_n ? pool_n : 1) * sizeof(uint64_t));
        if (!pool)
            abort();
        size_t o = 0;
        for (size_t i = 0; i < n_rows; ++i) {
            const size_t len = (size_t)(ref_offs[rows[i].rn + 1] - ref_offs[rows[i].rn]);
            if (len)
                memcpy(pool + o, ref_keys + (ref_offs[rows[i].rn] - ref_offs[0]), len * sizeof(uint64_t));
            o += len;
        }
        if (pool_n)
            qsort(pool, pool_n, sizeof(uint64_t), cmp_u64);
    }
    const uint64_t objmask = obj_bits >= 64 ? ~0ull : ((1ull << obj_bits) - 1ull);
    double total_mass = 0.0;
    for (size_t i = 0; i < n_rows; ++i) {
        kssd_row_t *r = &rows[i];
        const uint64_t *keys = ref_keys + (ref_offs[r->rn] - ref_offs[0]);
        const size_t len = (size_t)(ref_offs[r->rn + 1] - ref_offs[r->rn]);
        uint32_t *pos = malloc((len ? len : 1) * sizeof(uint32_t));
        if (!pos)
            abort();
        uint32_t markers = 0, observed = 0;
        double sum = 0.0, sumsq = 0.0;
        for (size_t k = 0; k < len; ++k) {
            const uint64_t key = keys[k];
            int marker;
            if (use_db) {
                const uint64_t ctx = obj_bits >= 64 ? 0 : (key >> obj_bits);
                marker = refdb_marker(refdb, (ctx << KSSD_GID_BITS) | (uint64_t)r->rn, (uint32_t)(key & objmask));
            } else {
                marker = bound_u64(pool, pool_n, key, 1) - bound_u64(pool, pool_n, key, 0) == 1;
            }
            if (!marker)
                continue;
            ++markers;
            const size_t qi = bound_u64(q_keys, q_n, key, 0);
            if (qi < q_n && q_keys[qi] == key) {
                const uint32_t c = q_counts[qi];
                pos[observed++] = c;
                sum += (double)c;
                sumsq += (double)c * (double)c;
            }
        }
        r->coverage_status = use_db ? 4 : 1;
        r->cov_ref_markers = markers;
        r->cov_observed_markers = observed;
        r->cov_observed_fraction = markers ? (double)observed / (double)markers : 0.0;
        r->cov_count_sum = sum;
        r->est_depth = markers ? sum / (double)markers : 0.0;
        r->pos_mean_depth = observed ? sum / (double)observed : 0.0;
        if (observed) {
            qsort(pos, observed, sizeof(uint32_t), cmp_u32);
            r->pos_median_depth = (observed & 1u) ? pos[observed / 2u]
                                                  : ((double)pos[observed / 2u - 1u] + (double)pos[observed / 2u]) / 2.0;
            const double mean = r->pos_mean_depth;
            double var = sumsq / (double)observed - mean * mean;
            if (var < 0.0 && var > -1e-9)
                var = 0.0;
            r->count_cv = mean > 0.0 && var > 0.0 ? sqrt(var) / mean : 0.0;
        }
        r->est_mass = sum;
        total_mass += sum;
        free(pos);
    }
    if (total_mass > 0.0)
        for (size_t i = 0; i < n_rows; ++i)
            rows[i].est_fraction = rows[i].est_mass / total_mass;
    free(pool);
}

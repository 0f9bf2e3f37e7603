// libkssdgpu: device-resident KSSD3A inverted index and shared-context counting
// kernels for B200 (sm_100a).  C ABI in include/kssdgpu.h.
//
// HBM layout of an index (N records, U unique contexts):
//   post[N]   uint64  gid << 32 | obj, in the reference's (ctx, gid, obj) record order
//   gkey[U]   uint64  unique contexts, ascending
//   gbeg[U+1] uint32  postings range of each context
//   table[C]  Slot    open-addressing hash of the U contexts (C = pow2 >= 2U),
//                     16 B {ctx, begin | count << 32}: one sector per probe
//
// Counting semantics follow src/command_ani.h:463-721 (see walk_context below).
#include "kssdgpu.h"
#include "kssd_dev.cuh"
#include "kssd_metric.cuh"

#include <cub/cub.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

using namespace kssd;

namespace kssd {
size_t dense_gemm_s8_workspace(int M, int N, int K);
int dense_gemm_s8(const int8_t *A, const int8_t *B, int32_t *D, int M, int N, int K, int64_t lda, int64_t ldb,
                  int64_t ldd, void *workspace, cudaStream_t st);
}  // namespace kssd

namespace {

thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? KSSDGPU_ERR_NOMEM : KSSDGPU_ERR_CUDA,   \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                        \
    } while (0)

inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ------------------------------------------------------------------ index build kernels

// Unpack reference records (packed 12 B) into postings; flag context heads and
// check the (ctxgid, obj) order and the gid range.
__global__ void k_unpack_records(const uint32_t *__restrict__ w, uint64_t n, int nref, uint64_t *__restrict__ post,
                                 uint32_t *__restrict__ head, unsigned long long *__restrict__ ctx_of,
                                 int *__restrict__ err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long cg = (unsigned long long)w[3 * i] | ((unsigned long long)w[3 * i + 1] << 32);
        const uint32_t obj = w[3 * i + 2];
        const uint32_t gid = (uint32_t)(cg & ((1u << kGidBits) - 1));
        const unsigned long long ctx = cg >> kGidBits;
        post[i] = ((uint64_t)gid << 32) | obj;
        ctx_of[i] = ctx;
        uint32_t h = 1;
        if (i > 0) {
            const unsigned long long pcg = (unsigned long long)w[3 * (i - 1)] | ((unsigned long long)w[3 * (i - 1) + 1] << 32);
            const uint32_t pobj = w[3 * (i - 1) + 2];
            if (pcg > cg || (pcg == cg && pobj > obj))
                atomicMax(err, (int)kDevUnsorted);
            h = (pcg >> kGidBits) != ctx;
        }
        if ((int)gid >= nref)
            atomicMax(err, (int)kDevGid);
        head[i] = h;
    }
}

// Sketch keys -> sort keys (ctx << 20 | gid) with obj values; checks that each
// sample's keys ascend (comblco order), which makes one stable sort by ctxgid
// produce the reference's (ctxgid, obj) order.
__global__ void k_sketch_to_sortkeys(const uint64_t *__restrict__ keys, const uint64_t *__restrict__ offs, int nref,
                                     int obj_bits, unsigned long long *__restrict__ skey, uint32_t *__restrict__ sval,
                                     int *__restrict__ err)
{
    const uint64_t base = offs[0];
    const uint64_t objmask = (obj_bits >= 64) ? ~0ull : ((1ull << obj_bits) - 1);
    for (int g = blockIdx.x; g < nref; g += gridDim.x) {
        const uint64_t b = offs[g] - base, e = offs[g + 1] - base;
        for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
            const uint64_t k = keys[i];
            if (i > b && keys[i - 1] > k)
                atomicMax(err, (int)kDevUnsorted);
            skey[i] = ((k >> obj_bits) << kGidBits) | (uint64_t)g;
            sval[i] = (uint32_t)(k & objmask);
        }
    }
}

__global__ void k_sorted_to_post(const unsigned long long *__restrict__ skey, const uint32_t *__restrict__ sval, uint64_t n,
                                 uint64_t *__restrict__ post, uint32_t *__restrict__ head,
                                 unsigned long long *__restrict__ ctx_of)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long cg = skey[i];
        const unsigned long long ctx = cg >> kGidBits;
        post[i] = ((cg & ((1u << kGidBits) - 1)) << 32) | sval[i];
        ctx_of[i] = ctx;
        head[i] = (i == 0) || ((skey[i - 1] >> kGidBits) != ctx);
    }
}

__global__ void k_scatter_groups(const uint32_t *__restrict__ head, const uint32_t *__restrict__ gidx,
                                 const unsigned long long *__restrict__ ctx_of, uint64_t n,
                                 unsigned long long *__restrict__ gkey, uint32_t *__restrict__ gbeg, uint64_t u)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (head[i]) {
            gkey[gidx[i]] = ctx_of[i];
            gbeg[gidx[i]] = (uint32_t)i;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        gbeg[u] = (uint32_t)n;
}

__global__ void k_table_insert(const unsigned long long *__restrict__ gkey, const uint32_t *__restrict__ gbeg, uint64_t u,
                               const uint64_t *__restrict__ post, Slot *__restrict__ t, uint32_t mask,
                               int *__restrict__ err)
{
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long ctx = gkey[g];
        const uint32_t cnt = gbeg[g + 1] - gbeg[g];
        // a context with one posting keeps it in the slot
        const unsigned long long word = cnt == 1 ? (ctx | kInlineBit) : ctx;
        const unsigned long long range =
            cnt == 1 ? post[gbeg[g]] : ((unsigned long long)gbeg[g] | ((unsigned long long)cnt << 32));
        uint32_t i = (uint32_t)mix64(ctx) & mask;
        bool done = false;
        for (uint32_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev = atomicCAS(&t[i].ctx, kEmptyCtx, word);
            if (prev == kEmptyCtx || prev == word) {
                t[i].range = range;
                done = true;
                break;
            }
            i = (i + 1) & mask;
        }
        if (!done)
            atomicMax(err, (int)kDevProbe);
    }
}

// reference-layout records back out of the CSR
__global__ void k_export_records(const unsigned long long *__restrict__ gkey, const uint32_t *__restrict__ gbeg, uint64_t u,
                                 const uint64_t *__restrict__ post, uint32_t *__restrict__ w)
{
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long ctx = gkey[g];
        for (uint32_t i = gbeg[g]; i < gbeg[g + 1]; ++i) {
            const uint64_t p = post[i];
            const unsigned long long cg = (ctx << kGidBits) | (p >> 32);
            w[3 * (uint64_t)i] = (uint32_t)cg;
            w[3 * (uint64_t)i + 1] = (uint32_t)(cg >> 32);
            w[3 * (uint64_t)i + 2] = (uint32_t)p;
        }
    }
}

// bit i set when record i's object occurs once in its context group
// (write_unique_marker_bits_from_sorted, src/command_sketch.c:856-914)
__global__ void k_unique_bits(const uint32_t *__restrict__ gbeg, uint64_t u, const uint64_t *__restrict__ post,
                              uint32_t *__restrict__ bits32)
{
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = gbeg[g], e = gbeg[g + 1];
        for (uint32_t i = b; i < e; ++i) {
            const uint32_t o = (uint32_t)post[i];
            uint32_t same = 0;
            for (uint32_t j = b; j < e && same < 2; ++j)
                same += (uint32_t)post[j] == o;
            if (same == 1)
                atomicOr(&bits32[i >> 5], 1u << (i & 31));
        }
    }
}

// per-gid record counts, conflict adjustments and unique-context totals
// (src/command_ani.c:351-381,441-460)
__global__ void k_ref_counts(const uint32_t *__restrict__ gbeg, uint64_t u, const uint64_t *__restrict__ post,
                             int conflict, int ignoreconflict, uint32_t *__restrict__ cnt, uint32_t *__restrict__ uniq)
{
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = gbeg[g], e = gbeg[g + 1];
        uint32_t i = b;
        bool single_owner = true;
        while (i < e) {
            const uint32_t gid = (uint32_t)(post[i] >> 32);
            uint32_t j = i + 1;
            while (j < e && (uint32_t)(post[j] >> 32) == gid)
                ++j;
            const uint32_t run = j - i;
            uint32_t keep = run;
            if (conflict && run > 1)
                keep = ignoreconflict ? 0 : 1;
            if (keep)
                atomicAdd(&cnt[gid], keep);
            if (i != b)
                single_owner = false;
            i = j;
        }
        if (uniq && single_owner && (!ignoreconflict || e - b == 1))
            atomicAdd(&uniq[(uint32_t)(post[b] >> 32)], 1u);
    }
}

// ------------------------------------------------------------------ counting kernels

// One unit of work of the global-row batched kernel: entries [b, e) (relative to
// qoffs[0]) of query q.  Context runs that straddle a chunk boundary are taken by
// the chunk holding the run's first entry, so chunks of one query never double count.
struct WorkItem {
    uint32_t q, pad;
    uint64_t b, e;
};
constexpr uint64_t kChunkKeys = 4096;
// filter stripes: at most this many bytes each (one stripe stays in L2 beside the
// streamed keys and the table lines), at most kMaxStripes of them
#ifndef KSSD_STRIPE_MB
#define KSSD_STRIPE_MB 16
#endif
constexpr uint64_t kStripeBytes = (uint64_t)KSSD_STRIPE_MB << 20;
constexpr int kMaxStripes = 256;
// stripe-major work: chunks of at least kStripeChunk entries, at most kStripeItemsMax
// chunks beyond one per (stripe, query)
constexpr uint64_t kStripeChunk = 256;
constexpr uint64_t kStripeItemsMax = 1ull << 20;

// An open-addressing table of touched counter cells (see table_credit below).
constexpr uint32_t kCellEmpty = 0xFFFFFFFFu;

struct CellTable {
    uint32_t *key;            // cell number, kCellEmpty for a free slot (null: no table)
    unsigned long long *acc;  // per slot: ctx word (num_mut2 << 32 | num_ctx), obj word (section << 32 | diff_obj)
    int log;                  // 2^log slots
};

struct CountParams {
    const Slot *table;
    uint32_t mask;
    const uint64_t *post;
    const uint64_t *qkeys;  // keys of query i at qkeys[qoffs[i] - qoffs[0] ...]
    const uint64_t *qoffs;  // absolute offsets, nq + 1
    int nq;
    int nref;
    int qgid_offset;
    int obj_bits;
    int ignoreconflict;
    unsigned long long *out_ctx;   // [nq][nref] ctx_mut2_t as u64 (num_mut2 << 32 | num_ctx)
    unsigned long long *out_obj;   // [nq][nref] obj_section_t as u64 (section << 32 | diff_obj)
    unsigned long long *out_uctx;
    unsigned long long *out_uobj;
    unsigned int *work;            // persistent-kernel work counter (zeroed before launch)
    const int *order;              // query processing order (largest first), may be null
    const WorkItem *items;         // global-row mode: key-range chunks of queries, may be null
    int nitems;
    const uint32_t *chunk_prefix;  // global-row mode without items: query q owns the chunk_keys-entry
                                   // chunks [prefix[q], prefix[q+1]) (nq + 1 words), may be null
    uint32_t chunk_keys;           // entries per chunk in that mode
    int *err;
    const uint4 *bloom;            // membership filter of the index's contexts, may be null
    uint32_t bloom_mask;           // 32-byte blocks of one stripe of it - 1
    int bloom_stripes;             // its key-range stripes (a power of two)
    const unsigned long long *bloom_bounds;  // first context of each stripe (stripes + 1 words)
    const uint32_t *nitems_dev;    // stripe-major mode: count of P.items (built on the device), may be null
};


// One counter update for a matched (query ctx, reference gid run) with minimum
// object difference d: num_ctx += 1; d > 0: diff_obj += 1, section += d;
// d > 1: num_mut2 += 1  (src/command_ani.h:536-561).
__device__ __forceinline__ unsigned long long inc_ctx(int d) { return 1ull | ((unsigned long long)(d > 1) << 32); }
__device__ __forceinline__ unsigned long long inc_obj(int d) { return 1ull | ((unsigned long long)d << 32); }

// Shared-memory row: four 32-bit counters per reference (native shared atomics;
// hot cells of similar genomes contend less than on 64-bit words).
struct SmemAcc {
    uint32_t *nc, *m2, *dobj, *sect;
    __device__ __forceinline__ void add(uint32_t gid, int d) const
    {
        atomicAdd(nc + gid, 1u);
        if (d) {
            atomicAdd(dobj + gid, 1u);
            atomicAdd(sect + gid, (uint32_t)d);
            if (d > 1)
                atomicAdd(m2 + gid, 1u);
        }
    }
};

// Where a counter array spans far more memory than L2 (the 20,000-genome lower
// triangle: 3.2 GB), its touched cells lie scattered
// over the whole span and every add into them is slow -- atomics onto a fixed set of
// addresses spread over 1.6 GB run at 38 G/s on a B200 against 130 G/s when the same
// addresses fit in 16 MB -- although the touched cells themselves are few (92,633).
// The self join's scan then adds into a compact open-addressing table of touched cells
// instead (2^21 slots by default: a cell
// number and its two counter words, 40 MB), claimed by the first credit of a cell that
// finds a free slot among its first kCellTableProbes; a cell whose probes find no room
// goes to the array directly.  Keys only go from empty to a cell while a kernel runs and
// every credit of a cell probes the same sequence, so a cell lives in one slot or in the
// array, never both; k_cell_table_flush adds the slots into the array after the kernel
// and empties them for the next call.
constexpr int kCellTableLog = 21;
constexpr uint32_t kCellTableProbes = 8;


// One credit of difference d into the cell's slot; false when its probes find no room.
__device__ __forceinline__ bool table_credit(const CellTable &T, uint32_t cell, int d)
{
    const uint32_t mask = (1u << T.log) - 1;
    uint32_t s = (cell * 2654435761u) >> (32 - T.log);
    for (uint32_t p = 0; p < kCellTableProbes; ++p) {
        uint32_t k = __ldcg(T.key + s);  // from L2: keys are claimed while the kernel runs
        if (k == kCellEmpty) {
            const uint32_t old = atomicCAS(T.key + s, kCellEmpty, cell);
            k = old == kCellEmpty ? cell : old;
        }
        if (k == cell) {
            atomicAdd(T.acc + 2 * (size_t)s, inc_ctx(d));
            if (d)
                atomicAdd(T.acc + 2 * (size_t)s + 1, inc_obj(d));
            return true;
        }
        s = (s + 1) & mask;
    }
    return false;
}

// A query's global counter row.  (Through the table of touched cells, the 10,000 x
// 20,000 block's count measured 2.24 vs 2.18 ms: unlike the self join's, its credits'
// cost is not the scattered addresses, and the key load per credit adds latency.)
struct GlobalAcc {
    unsigned long long *c, *o;
    __device__ __forceinline__ void add(uint32_t gid, int d) const
    {
        atomicAdd(c + gid, inc_ctx(d));
        if (d)
            atomicAdd(o + gid, inc_obj(d));
    }
};

// min over the query run's objects x one reference object
__device__ __forceinline__ int min_diff_obj(uint32_t robj, uint32_t q0, int s, const uint64_t *__restrict__ qrun,
                                            uint64_t objmask, int cur)
{
    int d = dna_pop(q0 ^ robj);
    for (int k = 1; k < s && d; ++k)
        d = min(d, dna_pop((uint32_t)(__ldg(qrun + k) & objmask) ^ robj));
    return min(cur, d);
}

// The postings walk for one query context run (objects qrun[0..s)) against the
// context group [pb, pe): per reference gid run, count the context, take the
// minimum object difference over the run cross product, and (UNIQUE) credit the
// sole owner of the context when there is exactly one gid run
// (src/command_ani.h:515-575; lower variant :694-716 stops at gid >= qgid).
template <bool LOWER, bool UNIQUE, class Acc>
__device__ __forceinline__ void walk_context(const uint64_t *__restrict__ post, uint32_t pb, uint32_t pe,
                                             const uint64_t *__restrict__ qrun, int s, uint64_t objmask, int qgid,
                                             int ignoreconflict, const Acc &acc, const Acc &uacc)
{
    const uint32_t q0 = (uint32_t)(__ldg(qrun) & objmask);
    uint32_t p = pb;
    uint32_t owners = 0, sole_gid = 0;
    int sole_d = 0;
    bool sole_ok = false;
    while (p < pe) {
        const uint64_t w = __ldg(post + p);
        const uint32_t gid = (uint32_t)(w >> 32);
        if (LOWER && (int)gid >= qgid)
            break;
        int d = min_diff_obj((uint32_t)w, q0, s, qrun, objmask, kMinInit);
        const uint32_t rb = p++;
        while (p < pe) {
            const uint64_t w2 = __ldg(post + p);
            if ((uint32_t)(w2 >> 32) != gid)
                break;
            d = min_diff_obj((uint32_t)w2, q0, s, qrun, objmask, d);
            ++p;
        }
        ++owners;
        sole_gid = gid;
        if (ignoreconflict && p - rb > 1)
            continue;
        acc.add(gid, d);
        sole_d = d;
        sole_ok = true;
    }
    if (UNIQUE && owners == 1 && sole_ok)
        uacc.add(sole_gid, sole_d);
}

// Handle a found context: the inline single posting, or a walk of its group.
template <bool LOWER, bool UNIQUE, class Acc>
__device__ __forceinline__ void credit_context(const CountParams &P, uint64_t i, int s, unsigned long long payload,
                                               bool single, int qgid, uint64_t objmask, const Acc &acc,
                                               const Acc &uacc)
{
    if (single) {
        // the context's only posting, held in the slot: one gid run of one object
        const uint32_t gid = (uint32_t)(payload >> 32);
        if (LOWER && (int)gid >= qgid)
            return;
        const uint32_t q0 = (uint32_t)(P.qkeys[i] & objmask);
        const int d = min_diff_obj((uint32_t)payload, q0, s, P.qkeys + i, objmask, kMinInit);
        acc.add(gid, d);
        if (UNIQUE)
            uacc.add(gid, d);
        return;
    }
    const uint32_t pb = (uint32_t)payload, pc = (uint32_t)(payload >> 32);
    walk_context<LOWER, UNIQUE>(P.post, pb, pb + pc, P.qkeys + i, s, objmask, qgid, P.ignoreconflict, acc, uacc);
}

// Process query entry i of [b, e): only the first entry of a context run works;
// it takes the whole run (src/command_ani.h:498-505).
template <bool LOWER, bool UNIQUE, class Acc>
__device__ __forceinline__ void process_entry(const CountParams &P, uint64_t i, uint64_t b, uint64_t e, int qgid,
                                              uint64_t objmask, const Acc &acc, const Acc &uacc)
{
    const uint64_t key = __ldg(P.qkeys + i);
    const uint64_t ctx = key >> P.obj_bits;
    const uint64_t prev = i > b ? __ldg(P.qkeys + i - 1) : 0;
    if (prev > key)
        atomicMax(P.err, (int)kDevUnsorted);  // a sample's keys must ascend (comblco order)
    if (i > b && (prev >> P.obj_bits) == ctx)
        return;
    int s = 1;
    while (i + s < e && (__ldg(P.qkeys + i + s) >> P.obj_bits) == ctx)
        ++s;
    unsigned long long payload;
    bool single;
    if (!table_lookup(P.table, P.mask, ctx, payload, single))
        return;
    credit_context<LOWER, UNIQUE>(P, i, s, payload, single, qgid, objmask, acc, uacc);
}

// Membership filter of an index's contexts, cut into key-range stripes: stripe s holds
// the contexts of [bounds[s], bounds[s+1]) (quantiles of the sorted contexts, so every
// stripe holds U / S of them) in a power of two of 32-byte blocks, at most 16 MB per
// stripe and at least 8 bits per context; each context sets 4 bits in one 16-byte half
// of its block.  A query context whose bits are not all set is not in the index and
// needs no table probe: for queries of other genomes most contexts are absent (a
// 10,000 x 20,000 block: 88%), and each absent context would otherwise cost a random
// table line from HBM.  A filter read at random as a whole does not stay in L2 once it
// is tens of MB; a count that walks the query keys stripe by stripe keeps only the
// current stripe's part hot (k_count_striped).
struct BloomBits {
    uint32_t block, half, p[4];
};
__device__ __forceinline__ BloomBits bloom_bits(unsigned long long ctx, uint32_t mask)
{
    const unsigned long long h = mix64(mix64(ctx) ^ 0x243F6A8885A308D3ull);
    BloomBits b;
    b.block = (uint32_t)h & mask;
    b.half = (uint32_t)(h >> 32) & 1u;
    b.p[0] = (uint32_t)(h >> 33) & 127u;
    b.p[1] = (uint32_t)(h >> 40) & 127u;
    b.p[2] = (uint32_t)(h >> 47) & 127u;
    b.p[3] = (uint32_t)(h >> 54) & 127u;
    return b;
}

// stripe of a context: the largest s < S with bounds[s] <= ctx (bounds[0] = 0)
__device__ __forceinline__ uint32_t stripe_of(const unsigned long long *__restrict__ bounds, int S,
                                              unsigned long long ctx)
{
    uint32_t lo = 0;
    for (uint32_t step = (uint32_t)S >> 1; step; step >>= 1)
        if (__ldg(bounds + lo + step) <= ctx)
            lo += step;
    return lo;
}

// Filter loads ask L2 to keep their lines (evict_last), so that the streamed query
// keys and the random table lines do not push the filter out of L2.
__device__ __forceinline__ uint4 ld_keep_l2(const uint4 *p)
{
    uint4 r;
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p), "l"(pol));
    return r;
}

// f: the context's stripe of the filter
__device__ __forceinline__ bool bloom_may_hold(const uint4 *__restrict__ f, uint32_t mask, unsigned long long ctx)
{
    const BloomBits b = bloom_bits(ctx, mask);
    const uint4 w = ld_keep_l2(f + 2 * (size_t)b.block + b.half);
    bool all = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t p = b.p[i];  // word by selects (a dynamically indexed array would live in local memory)
        const uint32_t word = (p & 64) ? ((p & 32) ? w.w : w.z) : ((p & 32) ? w.y : w.x);
        all &= (word >> (p & 31)) & 1u;
    }
    return all;
}

// The filter as one kernel sees it: a whole filter whose stripe is found per context,
// or (stripes == 1) the one stripe the caller works in.
struct FilterView {
    const uint4 *f;
    uint32_t mask;
    int stripes;
    const unsigned long long *bounds;
    __device__ __forceinline__ bool may_hold(unsigned long long ctx) const
    {
        if (!f)
            return true;
        const uint4 *base = f;
        if (stripes > 1)
            base += 2 * ((size_t)mask + 1) * stripe_of(bounds, stripes, ctx);
        return bloom_may_hold(base, mask, ctx);
    }
};

__global__ void k_bloom_insert(const unsigned long long *__restrict__ gkey, uint64_t u, uint32_t mask, int stripes,
                               const unsigned long long *__restrict__ bounds, uint32_t *__restrict__ f)
{
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long ctx = gkey[g];
        const BloomBits b = bloom_bits(ctx, mask);
        const size_t blk = (size_t)(stripes > 1 ? stripe_of(bounds, stripes, ctx) : 0) * ((size_t)mask + 1) + b.block;
        uint32_t *half = f + (2 * blk + b.half) * 4;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            atomicOr(half + (b.p[i] >> 5), 1u << (b.p[i] & 31));
    }
}

// bounds[s] = first context of stripe s: 0, then gkey[s * U / S], then ~0 (S + 1 words)
__global__ void k_stripe_bounds(const unsigned long long *__restrict__ gkey, uint64_t u, int stripes,
                                unsigned long long *__restrict__ bounds)
{
    for (int s = threadIdx.x; s <= stripes; s += blockDim.x)
        bounds[s] = s == 0 ? 0ull : s == stripes ? ~0ull : gkey[(uint64_t)s * u / (uint64_t)stripes];
}

// spos[q * (S + 1) + s]: the first entry of query q whose context is >= bounds[s]
// (absolute offsets; s = 0 and s = S are the query's own bounds).  Keys ascend within
// a query, so each is one binary search.
__global__ void k_stripe_pos(const uint64_t *__restrict__ qkeys, const uint64_t *__restrict__ qoffs, int nq,
                             int stripes, const unsigned long long *__restrict__ bounds, int obj_bits,
                             uint64_t *__restrict__ spos)
{
    const uint64_t base = qoffs[0];
    const uint64_t n = (uint64_t)nq * (stripes + 1);
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const int q = (int)(t / (uint64_t)(stripes + 1)), s = (int)(t % (uint64_t)(stripes + 1));
        uint64_t lo = qoffs[q], hi = qoffs[q + 1];
        if (s == stripes) {
            spos[t] = hi;
            continue;
        }
        if (s > 0) {
            const unsigned long long bound = bounds[s];
            while (lo < hi) {
                const uint64_t mid = lo + ((hi - lo) >> 1);
                if ((__ldg(qkeys + (mid - base)) >> obj_bits) < bound)
                    lo = mid + 1;
                else
                    hi = mid;
            }
        }
        spos[t] = lo;
    }
}

// A context group of at least kWarpWalk postings is walked by the whole warp: lanes load
// consecutive postings (one coalesced line per 32 of them instead of one thread's
// serial walk), the lane holding the first posting of a gid run takes the run's minimum
// object difference and credits it, and a ballot counts the group's owners for the
// unique-context rule.  Same credits as walk_context (src/command_ani.h:515-575): LOWER
// stops at gid >= qgid, --ignoreconflict skips reference runs of several objects, the
// sole owner is credited when its run counted.
constexpr uint32_t kWarpWalk = 32;

template <bool LOWER, bool UNIQUE, class Acc>
__device__ __forceinline__ void walk_context_warp(const uint64_t *__restrict__ post, uint32_t pb, uint32_t pe,
                                                  const uint64_t *__restrict__ qrun, int s, uint64_t objmask,
                                                  int qgid, int ignoreconflict, const Acc &acc, const Acc &uacc,
                                                  uint32_t lane)
{
    const uint32_t q0 = (uint32_t)(__ldg(qrun) & objmask);
    uint32_t owners = 0, sole_gid = 0;
    int sole_d = 0;
    bool sole_mine = false, sole_ok = false;
    for (uint32_t p0 = pb; p0 < pe; p0 += 32) {
        const uint32_t p = p0 + lane;
        const bool in = p < pe;
        const uint64_t w = in ? __ldg(post + p) : 0;
        const uint32_t gid = (uint32_t)(w >> 32);
        uint32_t pg = __shfl_up_sync(0xFFFFFFFFu, gid, 1);
        if (lane == 0)
            pg = p0 > pb ? (uint32_t)(__ldg(post + p0 - 1) >> 32) : 0xFFFFFFFFu;
        const bool live = in && (!LOWER || (int)gid < qgid);
        const bool head = live && gid != pg;
        if (head) {
            int d = min_diff_obj((uint32_t)w, q0, s, qrun, objmask, kMinInit);
            uint32_t x = p + 1;
            while (x < pe) {
                const uint64_t w2 = __ldg(post + x);
                if ((uint32_t)(w2 >> 32) != gid)
                    break;
                d = min_diff_obj((uint32_t)w2, q0, s, qrun, objmask, d);
                ++x;
            }
            const bool counted = !(ignoreconflict && x - p > 1);
            if (counted)
                acc.add(gid, d);
            sole_mine = true;
            sole_gid = gid;
            sole_d = d;
            sole_ok = counted;
        }
        owners += __popc(__ballot_sync(0xFFFFFFFFu, head));
        if (LOWER && __any_sync(0xFFFFFFFFu, in && (int)gid >= qgid))
            break;  // postings ascend by gid: the rest are not below the query
    }
    if (UNIQUE && owners == 1 && sole_mine && sole_ok)
        uacc.add(sole_gid, sole_d);
}

// Entries [cb, ce) of one query (whose entries are [b, e)), taken by the caller's
// threads t0, t0 + T, ... (t0 % 32 = the lane, T a multiple of 32): every lane of a warp
// takes one entry per round (the warp's rounds are the same for all its lanes).  Only the
// first entry of a context run works (src/command_ani.h:498-505); the filter rules out
// most absent contexts; one hash probe finds the context; the inline single posting is
// credited at once, short groups are walked by their lane, long ones by the warp.
template <bool LOWER, bool UNIQUE, class Acc>
__device__ __forceinline__ void process_query(const CountParams &P, uint64_t b, uint64_t e, uint64_t cb, uint64_t ce,
                                              int qgid, uint64_t objmask, const Acc &acc, const Acc &uacc,
                                              const FilterView &fv, uint64_t t0, uint64_t T)
{
    const uint32_t lane = (uint32_t)(t0 & 31u);
    for (uint64_t wb = cb + (t0 - lane); wb < ce; wb += T) {
        const uint64_t i = wb + lane;
        int s = 0;
        unsigned long long ctx = 0;
        uint32_t slot = 0;
        if (i < ce) {
            const uint64_t key = __ldg(P.qkeys + i);
            ctx = key >> P.obj_bits;
            const uint64_t prev = i > b ? __ldg(P.qkeys + i - 1) : 0;
            if (prev > key)
                atomicMax(P.err, (int)kDevUnsorted);  // a sample's keys must ascend (comblco order)
            if (!(i > b && (prev >> P.obj_bits) == ctx) && fv.may_hold(ctx)) {
                int run = 1;
                while (i + run < e && (__ldg(P.qkeys + i + run) >> P.obj_bits) == ctx)
                    ++run;
                s = run;
                slot = (uint32_t)mix64(ctx) & P.mask;
            }
        }
        bool wide = false;
        uint32_t pb = 0, pc = 0;
        if (s) {
            ulonglong2 sl = __ldg(reinterpret_cast<const ulonglong2 *>(P.table + slot));
            uint32_t at = slot;
            bool found = false;
            for (uint32_t probe = 0; probe <= P.mask; ++probe) {
                if ((sl.x & ~kInlineBit) == ctx) {
                    found = true;
                    break;
                }
                if (sl.x == kEmptyCtx)
                    break;
                at = (at + 1) & P.mask;
                sl = __ldg(reinterpret_cast<const ulonglong2 *>(P.table + at));
            }
            if (found) {
                const bool single = (sl.x & kInlineBit) != 0;
                pb = (uint32_t)sl.y;
                pc = (uint32_t)(sl.y >> 32);
                if (!single && pc >= kWarpWalk)
                    wide = true;
                else
                    credit_context<LOWER, UNIQUE>(P, i, s, sl.y, single, qgid, objmask, acc, uacc);
            }
        }
        // the warp walks its lanes' long groups together, one after another
        for (unsigned m = __ballot_sync(0xFFFFFFFFu, wide); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            const uint32_t gb = __shfl_sync(0xFFFFFFFFu, pb, src), gc = __shfl_sync(0xFFFFFFFFu, pc, src);
            const uint64_t gi = __shfl_sync(0xFFFFFFFFu, i, src);
            const int gs = __shfl_sync(0xFFFFFFFFu, s, src);
            walk_context_warp<LOWER, UNIQUE>(P.post, gb, gb + gc, P.qkeys + gi, gs, objmask, qgid, P.ignoreconflict,
                                             acc, uacc, lane);
        }
    }
}

// Batched persistent kernel: CTAs take whole queries from a work counter
// (largest first); with SMEM the query's reference row is accumulated in shared
// memory and written once, coalesced; without, counters go to the zeroed global
// row with atomics, and the work may be split into key-range chunks (P.items) so
// that one large query (a read set) spreads over many SMs.
template <bool LOWER, bool UNIQUE, bool SMEM>
__global__ void __launch_bounds__(512) k_count_batched(CountParams P)
{
    extern __shared__ uint32_t sm[];
    __shared__ int s_item;
    const uint64_t objmask = (P.obj_bits >= 64) ? ~0ull : ((1ull << P.obj_bits) - 1);
    const uint64_t base = P.qoffs[0];
    const int nref = P.nref;
    const FilterView fv{P.bloom, P.bloom_mask, P.bloom_stripes, P.bloom_bounds};
    for (;;) {
        if (threadIdx.x == 0)
            s_item = (int)atomicAdd(P.work, 1u);
        __syncthreads();
        const int it = s_item;
        const bool vchunks = !SMEM && !P.items && P.chunk_prefix;
        if (it >= (!SMEM && P.items ? P.nitems : vchunks ? (int)P.chunk_prefix[P.nq] : P.nq))
            break;
        int q;
        if (!SMEM && P.items) {
            q = (int)P.items[it].q;
        } else if (vchunks) {
            // the last query whose first chunk is <= it (queries without keys own no chunk)
            int lo = 0, hi = P.nq - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (P.chunk_prefix[mid] <= (uint32_t)it)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            q = lo;
        } else {
            q = P.order ? P.order[it] : it;
        }
        const int qgid = P.qgid_offset + q;
        const size_t row = (size_t)q * nref;
        // rows: [nc | m2 | dobj | sect] x nref, then the unique-context row
        uint32_t *row0 = sm, *row1 = sm + 4 * (size_t)nref;
        if (SMEM) {
            for (int c = threadIdx.x; c < nref * (UNIQUE ? 8 : 4); c += blockDim.x)
                sm[c] = 0;
            __syncthreads();
        }
        const uint64_t b = P.qoffs[q] - base, e = P.qoffs[q + 1] - base;
        if (SMEM) {
            const SmemAcc acc{row0, row0 + nref, row0 + 2 * nref, row0 + 3 * nref};
            const SmemAcc uacc{row1, row1 + nref, row1 + 2 * nref, row1 + 3 * nref};
            process_query<LOWER, UNIQUE>(P, b, e, b, e, qgid, objmask, acc, uacc, fv, threadIdx.x, blockDim.x);
        } else {
            const GlobalAcc acc{P.out_ctx + row, P.out_obj + row};
            const GlobalAcc uacc{UNIQUE ? P.out_uctx + row : nullptr, UNIQUE ? P.out_uobj + row : nullptr};
            uint64_t cb = b, ce = e;
            if (P.items) {
                cb = P.items[it].b;
                ce = P.items[it].e;
            } else if (vchunks) {
                cb = b + (uint64_t)(it - (int)P.chunk_prefix[q]) * P.chunk_keys;
                ce = min(e, cb + (uint64_t)P.chunk_keys);
            }
            process_query<LOWER, UNIQUE>(P, b, e, cb, ce, qgid, objmask, acc, uacc, fv, threadIdx.x, blockDim.x);
        }
        __syncthreads();
        if (SMEM) {
            for (int g = threadIdx.x; g < nref; g += blockDim.x) {
                P.out_ctx[row + g] = (unsigned long long)row0[g] | ((unsigned long long)row0[nref + g] << 32);
                P.out_obj[row + g] = (unsigned long long)row0[2 * nref + g] | ((unsigned long long)row0[3 * nref + g] << 32);
                if (UNIQUE) {
                    P.out_uctx[row + g] = (unsigned long long)row1[g] | ((unsigned long long)row1[nref + g] << 32);
                    P.out_uobj[row + g] =
                        (unsigned long long)row1[2 * nref + g] | ((unsigned long long)row1[3 * nref + g] << 32);
                }
            }
        }
        __syncthreads();
    }
}

// Stripe-major global-row kernel: the work items are chunks of one query's entries
// whose contexts fall in one filter stripe, listed stripe by stripe (k_stripe_expand),
// so that at any time the SMs probe one stripe of the filter and it stays in L2 while
// the query keys stream past.  Each warp takes kStripeGrab chunks at a time from the
// work counter; its lanes stride over a chunk's entries.  Counters go to the zeroed
// global rows with atomics, as in the chunked mode.
constexpr uint32_t kStripeGrab = 2;

template <bool LOWER, bool UNIQUE>
__global__ void __launch_bounds__(512) k_count_striped(CountParams P)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t objmask = (P.obj_bits >= 64) ? ~0ull : ((1ull << P.obj_bits) - 1);
    const uint64_t base = P.qoffs[0];
    const uint32_t nitems = *P.nitems_dev;
    const size_t stripe_words = 2 * ((size_t)P.bloom_mask + 1);  // uint4 per stripe
    for (;;) {
        uint32_t it0 = 0;
        if (lane == 0)
            it0 = atomicAdd(P.work, kStripeGrab);
        it0 = __shfl_sync(0xFFFFFFFFu, it0, 0);
        if (it0 >= nitems)
            break;
        const uint32_t it1 = min(nitems, it0 + kStripeGrab);
        for (uint32_t it = it0; it < it1; ++it) {
            const WorkItem w = P.items[it];
            const int q = (int)w.q;
            const uint64_t b = P.qoffs[q] - base, e = P.qoffs[q + 1] - base;
            const size_t row = (size_t)q * P.nref;
            const GlobalAcc acc{P.out_ctx + row, P.out_obj + row};
            const GlobalAcc uacc{UNIQUE ? P.out_uctx + row : nullptr, UNIQUE ? P.out_uobj + row : nullptr};
            const FilterView fv{P.bloom + stripe_words * w.pad, P.bloom_mask, 1, nullptr};
            process_query<LOWER, UNIQUE>(P, b, e, w.b, w.e, P.qgid_offset + q, objmask, acc, uacc, fv, lane, 32);
        }
    }
}

// chunk size of the stripe-major items: kStripeChunk entries, more for blocks so large
// that the chunks would exceed kStripeItemsMax
__device__ __forceinline__ uint64_t stripe_chunk(const uint64_t *__restrict__ qoffs, int nq)
{
    const uint64_t total = qoffs[nq] - qoffs[0];
    return max(kStripeChunk, (total + kStripeItemsMax - 1) / kStripeItemsMax);
}

// cnt[s * nq + q]: chunks of query q's entries in stripe s (cnt[S * nq] = 0, so that an
// exclusive scan leaves the chunk total there).  Offsets that decrease come only from
// keys out of order: the block is refused (err) and the range counts nothing, so the
// chunks never outgrow their buffer.
__global__ void k_stripe_counts(const uint64_t *__restrict__ spos, const uint64_t *__restrict__ qoffs, int nq,
                                int stripes, uint32_t *__restrict__ cnt, int *__restrict__ err)
{
    const uint64_t ck = stripe_chunk(qoffs, nq);
    const uint64_t n = (uint64_t)stripes * nq;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t <= n; t += (uint64_t)gridDim.x * blockDim.x) {
        if (t == n) {
            cnt[n] = 0;
            continue;
        }
        const int st = (int)(t / (uint64_t)nq), q = (int)(t % (uint64_t)nq);
        const uint64_t *sp = spos + (size_t)q * (stripes + 1) + st;
        if (sp[1] < sp[0]) {
            atomicMax(err, (int)kDevUnsorted);
            cnt[t] = 0;
            continue;
        }
        cnt[t] = (uint32_t)((sp[1] - sp[0] + ck - 1) / ck);
    }
}

// the chunks themselves, at their scanned offsets: {query, stripe, begin, end} with
// offsets relative to the block's first entry
__global__ void k_stripe_expand(const uint64_t *__restrict__ spos, const uint64_t *__restrict__ qoffs, int nq,
                                int stripes, const uint32_t *__restrict__ pre, WorkItem *__restrict__ items)
{
    const uint64_t ck = stripe_chunk(qoffs, nq);
    const uint64_t base = qoffs[0];
    const uint64_t n = (uint64_t)stripes * nq;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const int st = (int)(t / (uint64_t)nq), q = (int)(t % (uint64_t)nq);
        const uint64_t *sp = spos + (size_t)q * (stripes + 1) + st;
        const uint64_t b = sp[0] - base, e = sp[1] - base;
        uint32_t o = pre[t];
        for (uint64_t c = b; c < e && o < pre[t + 1]; c += ck)
            items[o++] = WorkItem{(uint32_t)q, (uint32_t)st, c, min(e, c + ck)};
    }
}

// counts[q] = chunk-entry chunks of query q; prefix[0] = 0 (a scan of counts fills
// prefix[1..nq])
__global__ void k_chunk_counts(const uint64_t *__restrict__ qoffs, int nq, uint32_t chunk,
                               uint32_t *__restrict__ counts, uint32_t *__restrict__ prefix)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        if (q == 0)
            prefix[0] = 0;
        counts[q] = (uint32_t)((qoffs[q + 1] - qoffs[q] + chunk - 1) / chunk);
    }
}

// Plain baseline: one launch per query, one thread per query entry, global atomics.
template <bool LOWER, bool UNIQUE>
__global__ void __launch_bounds__(256) k_count_plain(CountParams P, int q)
{
    const uint64_t objmask = (P.obj_bits >= 64) ? ~0ull : ((1ull << P.obj_bits) - 1);
    const uint64_t base = P.qoffs[0];
    const uint64_t b = P.qoffs[q] - base, e = P.qoffs[q + 1] - base;
    const uint64_t i = b + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= e)
        return;
    const size_t row = (size_t)q * P.nref;
    const GlobalAcc acc{P.out_ctx + row, P.out_obj + row};
    const GlobalAcc uacc{UNIQUE ? P.out_uctx + row : nullptr, UNIQUE ? P.out_uobj + row : nullptr};
    process_entry<LOWER, UNIQUE>(P, i, b, e, P.qgid_offset + q, objmask, acc, uacc);
}

// ------------------------------------------------------------------ self lower triangle (join)
//
// In the self case every query sample is also an index sample, so the query run of
// sample q at context c IS the (c, q) run of c's postings.  count_lower(q) at c
// therefore credits every ordered pair of runs (r < q) of c's group, and the whole
// triangle is one pass over the groups that hold at least two postings: no lookups.

// Plan-time classes of a context group.
enum : uint32_t { kJoinSmallMax = 32 };

// Warp-aggregated append of this lane's item when `want` (all 32 lanes call it).
__device__ __forceinline__ uint32_t warp_slot(unsigned int *counter, bool want, unsigned lane)
{
    const unsigned m = __ballot_sync(0xffffffffu, want);
    unsigned base = 0;
    if (m && lane == (unsigned)(__ffs(m) - 1))
        base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, m ? __ffs(m) - 1 : 0);
    return base + (unsigned)__popc(m & ((1u << lane) - 1u));
}

// Classify the groups with >= 2 postings (one thread per group, whole warps):
//   small   (k <= 32, one object per gid) -> (sort key, group) for the compact plan;
//             key = (32 - k, hash of the group's gid set) so that groups over the same
//             genome set end up side by side (equal keys: the set-major join compares
//             the gid lists themselves)
//   big     (k > 32, one object per gid)  -> begin | k << 32
//   conflict (a gid holds several objects) -> begin | k << 32
// totals: [0] postings in listed groups, [1] pairs.
__global__ void __launch_bounds__(256) k_self_classify(const uint32_t *__restrict__ gbeg, uint64_t u,
                                                       const uint64_t *__restrict__ post,
                                                       unsigned long long *__restrict__ skey,
                                                       uint32_t *__restrict__ sval,
                                                       unsigned long long *__restrict__ big,
                                                       unsigned long long *__restrict__ conf,
                                                       unsigned int *__restrict__ counts,
                                                       unsigned long long *__restrict__ totals)
{
    const uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    uint32_t b = 0, k = 0;
    bool conflict = false;
    unsigned long long key = 0;
    if (g < u) {
        b = gbeg[g];
        k = gbeg[g + 1] - b;
        if (k >= 2) {
            uint32_t prev = (uint32_t)(post[b] >> 32);
            unsigned long long h = mix64(prev + 1ull);
            for (uint32_t i = b + 1; i < b + k; ++i) {
                const uint32_t gid = (uint32_t)(post[i] >> 32);
                conflict |= gid == prev;
                prev = gid;
                h = mix64(h ^ (gid + 1ull));
            }
            key = ((unsigned long long)(kJoinSmallMax - min(k, kJoinSmallMax)) << 58) | (h >> 6);
        } else {
            k = 0;
        }
    }
    const bool is_small = k >= 2 && !conflict && k <= kJoinSmallMax;
    const bool is_big = k > kJoinSmallMax && !conflict;
    const bool is_conf = k >= 2 && conflict;
    const uint32_t s0 = warp_slot(counts + 0, is_small, lane);
    const uint32_t s1 = warp_slot(counts + 1, is_big, lane);
    const uint32_t s2 = warp_slot(counts + 2, is_conf, lane);
    const unsigned long long item = (unsigned long long)b | ((unsigned long long)k << 32);
    if (is_small) {
        skey[s0] = key;
        sval[s0] = (uint32_t)g;
    }
    if (is_big)
        big[s1] = item;
    if (is_conf)
        conf[s2] = item;
    unsigned long long np = k, npairs = k >= 2 ? (unsigned long long)k * (k - 1) / 2 : 0ull;
    for (int o = 16; o; o >>= 1) {
        np += __shfl_down_sync(0xffffffffu, np, o);
        npairs += __shfl_down_sync(0xffffffffu, npairs, o);
    }
    if (lane == 0 && np) {
        atomicAdd(totals + 0, np);
        atomicAdd(totals + 1, npairs);
    }
}

// sizes of the sorted small groups, for the offsets of the compact posting array
__global__ void k_self_sizes(const uint32_t *__restrict__ sval, uint32_t n, const uint32_t *__restrict__ gbeg,
                             uint32_t *__restrict__ ks)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        ks[t] = gbeg[sval[t] + 1] - gbeg[sval[t]];
}

// descriptor (offset | k << 32) and the group's postings copied to jp[offset ..)
__global__ void k_self_gather(const uint32_t *__restrict__ sval, const uint32_t *__restrict__ ks,
                              const uint32_t *__restrict__ offs, uint32_t n, const uint32_t *__restrict__ gbeg,
                              const uint64_t *__restrict__ post, unsigned long long *__restrict__ desc,
                              uint64_t *__restrict__ jp)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t b = gbeg[sval[t]], k = ks[t], o = offs[t];
        desc[t] = (unsigned long long)o | ((unsigned long long)k << 32);
        for (uint32_t i = 0; i < k; ++i)
            jp[o + i] = post[b + i];
    }
}

__device__ __forceinline__ size_t lower_cell(uint32_t row, uint32_t col) { return (size_t)row * (row - 1) / 2 + col; }

__device__ __forceinline__ void join_pair(uint64_t pi, uint64_t pj, unsigned long long *__restrict__ oc,
                                          unsigned long long *__restrict__ oo)
{
    const int d = min(kMinInit, dna_pop((uint32_t)pi ^ (uint32_t)pj));
    const size_t cell = lower_cell((uint32_t)(pj >> 32), (uint32_t)(pi >> 32));
    atomicAdd(oc + cell, inc_ctx(d));
    if (d)
        atomicAdd(oo + cell, inc_obj(d));
}

// Zero two 16-byte aligned arrays of `words` 8-byte counters.
// Programmatic dependent launch of the self join after the zero fill: the fill lets
// the join's grid launch at once, and the join waits for the fill's completion (and
// its stores) only before its first atomic, so the join's loads overlap the fill.
#ifndef KSSD_JOIN_PDL
#define KSSD_JOIN_PDL 1
#endif
__device__ __forceinline__ void pdl_launch_dependents()
{
#if KSSD_JOIN_PDL
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
__device__ __forceinline__ void pdl_wait_primary()
{
#if KSSD_JOIN_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");  // no-op without a programmatic dependency
#endif
}

// One wave (8 blocks of 256 per SM, all resident at once), so that the dependent
// join's blocks never take the slots of fill blocks still waiting to start.
__global__ void __launch_bounds__(256, 8) k_zero_pair(unsigned long long *__restrict__ a, unsigned long long *__restrict__ b,
                                                      size_t words)
{
    pdl_launch_dependents();
    const size_t n16 = words / 2;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    ulonglong2 *a2 = reinterpret_cast<ulonglong2 *>(a), *b2 = reinterpret_cast<ulonglong2 *>(b);
    const ulonglong2 z = make_ulonglong2(0ull, 0ull);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += stride) {
        a2[i] = z;
        b2[i] = z;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (words & 1)) {
        a[words - 1] = 0;
        b[words - 1] = 0;
    }
}

// Set-major plan of the small groups.  Sorted groups with the same gid list form
// a run (their pairs all land on the same k(k-1)/2 counter cells); runs are cut
// into chunks of at most `csize` groups, and every (chunk, pair) is one work item
// of the join: the item sums its pair's increments over the chunk's groups in
// registers and adds them with one atomic per counter word.  Chunks are ordered by
// size (largest first) so that the lanes of a warp loop over equal group counts.

// heads[t] = 1 where sorted small group t starts a new run (size or gid list differs)
__global__ void k_set_heads(const unsigned long long *__restrict__ desc, uint32_t n, const uint64_t *__restrict__ jp,
                            uint32_t *__restrict__ heads)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        uint32_t h = 1;
        if (t > 0) {
            const unsigned long long d = desc[t], d0 = desc[t - 1];
            const uint32_t k = (uint32_t)(d >> 32);
            if (k == (uint32_t)(d0 >> 32)) {
                h = 0;
                const uint64_t *a = jp + (uint32_t)d, *b = jp + (uint32_t)d0;
                for (uint32_t i = 0; i < k && !h; ++i)
                    h = (uint32_t)(a[i] >> 32) != (uint32_t)(b[i] >> 32);
            }
        }
        heads[t] = h;
    }
}

// run starts: first[run] = t for every head (run = inclusive head count - 1)
__global__ void k_set_run_first(const uint32_t *__restrict__ heads, const uint32_t *__restrict__ runs_incl, uint32_t n,
                                uint32_t *__restrict__ first)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        if (heads[t])
            first[runs_incl[t] - 1] = t;
}

// chunk heads: every csize-th group of a run, counted from the run's start
__global__ void k_set_chunk_heads(const uint32_t *__restrict__ runs_incl, const uint32_t *__restrict__ first, uint32_t n,
                                  uint32_t csize, uint32_t *__restrict__ cheads)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        cheads[t] = ((t - first[runs_incl[t] - 1]) % csize) == 0;
}

// chunk records {offset of the first group's postings, m | k << 32} and pair counts
// Sort key of a chunk: (descending group count, then size) when sorted, else the size
// alone (plan order within a size); chunks of equal (count, size) end up adjacent,
// as the item tiles need.
__global__ void k_set_chunks(const uint32_t *__restrict__ cheads, const uint32_t *__restrict__ cpos, uint32_t n,
                             uint32_t csize, int by_count, const unsigned long long *__restrict__ desc,
                             ulonglong2 *__restrict__ chunks, uint32_t *__restrict__ skey, uint32_t *__restrict__ sval)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        if (!cheads[t])
            continue;
        const uint32_t c = cpos[t];
        // the chunk ends at the next chunk head (every run start is one)
        uint32_t e = t + 1;
        while (e < n && e - t < csize && !cheads[e])
            ++e;
        const unsigned long long d = desc[t];
        const uint32_t k = (uint32_t)(d >> 32);
        chunks[c] = make_ulonglong2((unsigned long long)(uint32_t)d, (unsigned long long)(e - t) | ((unsigned long long)k << 32));
        skey[c] = (by_count ? (csize - (e - t)) << 6 : 0u) | k;  // csize < 256, k <= 32: 14 bits
        sval[c] = c;
    }
}

// Small groups of at most kFlatMax genomes can be joined flat (one thread per group)
// instead of as (chunk, pair) items; the plan chooses the largest flat size.
constexpr uint32_t kFlatMax = 4;

// chunks in sorted order
__global__ void k_set_permute(const uint32_t *__restrict__ order, uint32_t nchunks, const ulonglong2 *__restrict__ in,
                              ulonglong2 *__restrict__ out)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x)
        out[c] = in[order[c]];
}

// first sorted small group of every size 2..flat_max (the groups are sorted by size,
// largest first, so each size is one contiguous class and the smallest is the tail)
__global__ void k_flat_firsts(const unsigned long long *__restrict__ desc, uint32_t n, uint32_t flat_max,
                              uint32_t *__restrict__ firsts)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(desc[t] >> 32);
        if (k <= flat_max && (t == 0 || (uint32_t)(desc[t - 1] >> 32) != k))
            firsts[k] = t;
    }
}

// run heads of one flat class, one 32-bit word per 32 groups (bit = lane)
__global__ void k_flat_heads(const uint32_t *__restrict__ heads, uint32_t first, uint32_t cnt, uint32_t *__restrict__ out)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if ((t & ~31u) >= cnt)
        return;  // whole warps only
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, t < cnt && heads[first + t]);
    if ((t & 31) == 0)
        out[t >> 5] = b;
}

// Self-contained join items: first word of the chunk's tile in the tiled postings
// (34 bits) | m << 34 (8) | k << 42 (6) | i << 48 (5) | j << 53 (5) | slot << 58 (5),
// slot = the chunk's place in its tile.  The all-zero word (m = 0) is an empty lane.
__host__ __device__ __forceinline__ unsigned long long set_item(uint64_t off, uint32_t m, uint32_t k, uint32_t i,
                                                                uint32_t j, uint32_t slot)
{
    return off | ((unsigned long long)m << 34) | ((unsigned long long)k << 42) | ((unsigned long long)i << 48) |
           ((unsigned long long)j << 53) | ((unsigned long long)slot << 58);
}
constexpr uint64_t kSetItemMaxOffset = 1ull << 34;

// Item tiles.  Chunks of equal group count m and size k are packed C at a time into
// a tile whose postings are stored row-interleaved: row x of chunk 0, row x of chunk
// 1, ..., then row x + 1 (word (x * C + slot) * k + posting).  C = 32 / P chunks with
// P = k(k-1)/2 items each fill one warp, so the warp's loads of one row touch one or
// two 128-byte lines instead of one line per chunk; a chunk with P > 32 items is a
// tile of its own over whole warps.
__host__ __device__ __forceinline__ uint32_t tile_chunks(uint32_t k)
{
    const uint32_t p = k * (k - 1) / 2;
    return p >= 1 && p <= 32 ? 32 / p : 1;
}
__host__ __device__ __forceinline__ uint32_t tile_lanes(uint32_t k)
{
    const uint32_t p = k * (k - 1) / 2;
    return p <= 32 ? 32 : (p + 31) / 32 * 32;
}

// heads of the runs of tiled chunks with equal (m, k) in the sorted chunk order
__global__ void k_tile_class_heads(const ulonglong2 *__restrict__ chunks, uint32_t nchunks, uint32_t flat_max,
                                   uint32_t *__restrict__ heads)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        const unsigned long long y = chunks[c].y;
        const uint32_t k = (uint32_t)(y >> 32);
        heads[c] = k > flat_max && (c == 0 || chunks[c - 1].y != y);
    }
}

// each chunk's slot in its tile; tile heads carry the tile's words and lanes
__global__ void k_tile_slots(const ulonglong2 *__restrict__ chunks, uint32_t nchunks, uint32_t flat_max,
                             const uint32_t *__restrict__ cls_incl, const uint32_t *__restrict__ cls_first,
                             uint32_t *__restrict__ slot, unsigned long long *__restrict__ words,
                             uint32_t *__restrict__ lanes)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        const unsigned long long y = chunks[c].y;
        const uint32_t m = (uint32_t)y, k = (uint32_t)(y >> 32);
        uint32_t sl = 0;
        unsigned long long wd = 0;
        uint32_t ln = 0;
        if (k > flat_max) {
            const uint32_t cap = tile_chunks(k);
            sl = (c - cls_first[cls_incl[c] - 1]) % cap;
            if (sl == 0) {
                wd = (unsigned long long)m * cap * k;
                ln = tile_lanes(k);
            }
        }
        slot[c] = sl;
        words[c] = wd;
        lanes[c] = ln;
    }
}

// postings of every tiled chunk into its tile, row-interleaved
__global__ void k_tile_scatter(const ulonglong2 *__restrict__ chunks, uint32_t nchunks, uint32_t flat_max,
                               const uint32_t *__restrict__ slot, const unsigned long long *__restrict__ word0,
                               const uint64_t *__restrict__ jp, uint64_t *__restrict__ jt)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        const ulonglong2 ch = chunks[c];
        const uint32_t m = (uint32_t)ch.y, k = (uint32_t)(ch.y >> 32);
        if (k <= flat_max)
            continue;
        const uint32_t sl = slot[c], cap = tile_chunks(k);
        const uint64_t base = word0[c - sl];
        for (uint32_t x = 0; x < m; ++x)
            for (uint32_t i = 0; i < k; ++i)
                jt[base + ((uint64_t)x * cap + sl) * k + i] = jp[ch.x + (uint64_t)x * k + i];
    }
}

// Items of every tiled chunk: pair p (i < j, p = j(j-1)/2 + i) of the chunk in slot
// sl of its tile is lane lane0 + sl * P + p of the tile's lanes; unused lanes stay 0.
__global__ void k_set_items(const ulonglong2 *__restrict__ chunks, uint32_t nchunks, uint32_t flat_max,
                            const uint32_t *__restrict__ slot, const unsigned long long *__restrict__ word0,
                            const uint32_t *__restrict__ lane0, unsigned long long *__restrict__ items)
{
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunks; c += gridDim.x * blockDim.x) {
        const ulonglong2 ch = chunks[c];
        const uint32_t m = (uint32_t)ch.y, k = (uint32_t)(ch.y >> 32);
        if (k <= flat_max)
            continue;
        const uint32_t sl = slot[c], np = k * (k - 1) / 2;
        const uint64_t w0 = word0[c - sl];
        uint32_t o = lane0[c - sl] + sl * np;
        for (uint32_t j = 1; j < k; ++j)
            for (uint32_t i = 0; i < j; ++i)
                items[o++] = set_item(w0, m, k, i, j, sl);
    }
}

// Compact counters.  Every item's counter cell is known when the plan is built, and
// the touched cells are few (a genome shares contexts with a handful of others), so
// the join can add into one compact slot per touched cell (L2-resident) while the
// dense zero fill runs beside it on another stream; a scatter then adds the compact
// counters into the dense arrays.  Cell of every item lane (empty lanes sort last):
__global__ void k_item_cells(const unsigned long long *__restrict__ items, uint32_t nitems,
                             const uint64_t *__restrict__ jt, unsigned long long *__restrict__ cell,
                             uint32_t *__restrict__ lane)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nitems; t += gridDim.x * blockDim.x) {
        const unsigned long long it = items[t];
        const uint32_t m = (uint32_t)(it >> 34) & 0xFFu, k = (uint32_t)(it >> 42) & 0x3Fu;
        unsigned long long c = ~0ull;
        if (m) {
            const uint32_t i = (uint32_t)(it >> 48) & 0x1Fu, j = (uint32_t)(it >> 53) & 0x1Fu;
            const uint32_t slot = (uint32_t)(it >> 58) & 0x1Fu;
            const uint64_t *g = jt + (it & (kSetItemMaxOffset - 1)) + slot * k;
            const uint32_t gi = (uint32_t)(g[i] >> 32), gj = (uint32_t)(g[j] >> 32);
            c = lower_cell(gj, gi);
        }
        cell[t] = c;
        lane[t] = t;
    }
}

// heads of the distinct touched cells in the sorted cell list
__global__ void k_touched_heads(const unsigned long long *__restrict__ cell, uint32_t n, uint32_t *__restrict__ heads)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        heads[s] = cell[s] != ~0ull && (s == 0 || cell[s] != cell[s - 1]);
}

// Compact slot layout: slot s holds its ctx word at s * kCompactStride and its obj
// word right after it (20,000 genomes: strides of 2 / 4 / 16 words measured a 153 /
// 156 / 161 us join).
#ifndef KSSD_COMPACT_STRIDE
#define KSSD_COMPACT_STRIDE 2
#endif
constexpr uint32_t kCompactStride = KSSD_COMPACT_STRIDE;

// each item lane's compact slot (as the word offset of its ctx word), and the dense
// cell of every slot
__global__ void k_touched_slots(const unsigned long long *__restrict__ cell, const uint32_t *__restrict__ lane,
                                const uint32_t *__restrict__ heads, const uint32_t *__restrict__ incl, uint32_t n,
                                uint32_t *__restrict__ islot, unsigned long long *__restrict__ touched)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        if (cell[s] == ~0ull)
            continue;
        islot[lane[s]] = (incl[s] - 1) * kCompactStride;
        if (heads[s])
            touched[incl[s] - 1] = cell[s];
    }
}

// dense counters += compact counters (distinct cells: no two threads share one)
__global__ void k_scatter_touched(const unsigned long long *__restrict__ touched, uint32_t n,
                                  const unsigned long long *__restrict__ acc, unsigned long long *__restrict__ oc,
                                  unsigned long long *__restrict__ oo)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const size_t c = touched[s];
        oc[c] += acc[(size_t)s * kCompactStride];
        oo[c] += acc[(size_t)s * kCompactStride + 1];
    }
}

// The set-major join: one thread per (chunk, pair) item.  The m groups of the chunk
// share their gid list, so the pair's counter cell is the same for all of them:
// sum num_ctx (= m), mut2, diff_obj and section over the groups, then one atomic
// per counter word.  The items of a tile (one warp) read the same row of its
// row-interleaved postings together, from one or two lines.
#ifndef KSSD_SET_UNROLL
#define KSSD_SET_UNROLL 4
#endif
#ifndef KSSD_SET_MINB
#define KSSD_SET_MINB 1
#endif
constexpr int kSetUnroll = KSSD_SET_UNROLL;
__device__ __forceinline__ void self_set_item(uint32_t t, const unsigned long long *__restrict__ items, uint32_t nitems,
                                              const uint64_t *__restrict__ jt, const uint32_t *__restrict__ islot,
                                              unsigned long long *__restrict__ oc,
                                              unsigned long long *__restrict__ oo)
{
    if (t >= nitems)
        return;
    const unsigned long long it = __ldg(items + t);
    const uint64_t off = it & (kSetItemMaxOffset - 1);
    const uint32_t m = (uint32_t)(it >> 34) & 0xFFu, k = (uint32_t)(it >> 42) & 0x3Fu;
    if (m == 0)
        return;  // an empty lane of a tile
    const uint32_t i = (uint32_t)(it >> 48) & 0x1Fu, j = (uint32_t)(it >> 53) & 0x1Fu;
    const uint32_t slot = (uint32_t)(it >> 58) & 0x1Fu, stride = tile_chunks(k) * k;  // words per tile row
    // the chunk's first row gives the gids (high words) and its objects
    const uint64_t *g = jt + off + slot * k;
    const uint64_t pi0 = __ldg(g + i), pj0 = __ldg(g + j);
    const uint32_t gi = (uint32_t)(pi0 >> 32), gj = (uint32_t)(pj0 >> 32);
    uint32_t d = (uint32_t)min(kMinInit, dna_pop((uint32_t)pi0 ^ (uint32_t)pj0));
    uint32_t mut2 = d > 1, dobj = d > 0, sect = d;
    // low (object) words of the other rows' postings
    const uint32_t *w = reinterpret_cast<const uint32_t *>(g);
#pragma unroll kSetUnroll
    for (uint32_t x = 1; x < m; ++x) {
        const uint32_t oi = __ldg(w + 2 * (x * stride + i)), oj = __ldg(w + 2 * (x * stride + j));
        d = (uint32_t)min(kMinInit, dna_pop(oi ^ oj));
        mut2 += d > 1;
        dobj += d > 0;
        sect += d;
    }
    const size_t cell = islot ? (size_t)__ldg(islot + t) : lower_cell(gj, gi);  // compact slot or dense cell
    pdl_wait_primary();
    atomicAdd(oc + cell, (unsigned long long)m | ((unsigned long long)mut2 << 32));
    if (dobj)
        atomicAdd(oo + cell, (unsigned long long)dobj | ((unsigned long long)sect << 32));
}

// Flat join of one size class: one thread per group of K genomes, lanes on
// consecutive groups (a warp reads 32 x K postings, contiguous).  Groups of one run
// share their K(K-1)/2 counter cells; per pair, a warp sums each run's increments by
// a segmented reduction toward the run's first lane (run heads from the plan, bit =
// lane) and that lane adds them with one atomic per counter word.  A warp takes
// kFlatRounds(K) consecutive rounds of 32 groups and issues all their loads first, so
// that each thread keeps several postings in flight.  Threads of a warp exit together
// (the shuffles span the full warp).
__host__ __device__ constexpr uint32_t kFlatRounds(int k) { return k == 2 ? 3 : 1; }
#ifndef KSSD_FLAT_REDUX
#define KSSD_FLAT_REDUX 1
#endif

template <int K>
__device__ __forceinline__ void self_flat_groups(uint32_t t, const uint64_t *__restrict__ pk, uint32_t nk,
                                                 const uint32_t *__restrict__ hk, unsigned long long *__restrict__ oc,
                                                 unsigned long long *__restrict__ oo)
{
    constexpr uint32_t R = kFlatRounds(K);
    const uint32_t lane = t & 31, w0 = (t >> 5) * R;  // the warp's first 32-group word
    if ((size_t)w0 * 32 >= nk)
        return;
    uint64_t p[R][K];
    uint32_t hw[R];
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
        const size_t g = (size_t)(w0 + r) * 32 + lane;
        const bool act = g < nk;
#pragma unroll
        for (int x = 0; x < K; ++x)
            p[r][x] = act ? __ldg(pk + (size_t)K * g + x) : 0;
        hw[r] = (size_t)(w0 + r) * 32 < nk ? __ldg(hk + w0 + r) : 0u;
    }
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) {
        const size_t base = (size_t)(w0 + r) * 32;
        if (base >= nk)
            break;  // the same for the whole warp
        const uint32_t nv = (uint32_t)min((size_t)32, nk - base);
        const bool act = lane < nv;
        // segments: the plan's run heads, lane 0, and every inactive lane on its own
        const uint32_t valid = nv == 32 ? 0xFFFFFFFFu : (1u << nv) - 1;
        const uint32_t heads = hw[r] | 1u | ~valid;
        const uint32_t above = lane == 31 ? 0u : heads & (0xFFFFFFFFu << (lane + 1));
        const uint32_t end = above ? (uint32_t)__ffs(above) - 1 : 32u;
        const bool lead = act && ((heads >> lane) & 1u);
        const uint32_t m = end - lane;
        if (r == 0)
            pdl_wait_primary();
#pragma unroll
        for (int j = 1; j < K; ++j) {
#pragma unroll
            for (int i = 0; i < j; ++i) {
                const uint32_t d = (uint32_t)min(kMinInit, dna_pop((uint32_t)p[r][i] ^ (uint32_t)p[r][j]));
                // sect (9 bits: at most 32 x 12) | dobj << 9 (6 bits) | mut2 << 15 (6 bits)
                uint32_t v = act ? d | (uint32_t)(d > 0) << 9 | (uint32_t)(d > 1) << 15 : 0;
#if KSSD_FLAT_REDUX
                if (heads == 1u) {
                    v = __reduce_add_sync(0xFFFFFFFFu, v);  // one run over the whole warp
                } else
#endif
                {
#pragma unroll
                    for (uint32_t off = 1; off < 32; off <<= 1) {
                        const uint32_t x = __shfl_down_sync(0xFFFFFFFFu, v, off);
                        if (lane + off < end)
                            v += x;
                    }
                }
                if (lead) {
                    const uint32_t sect = v & 511u, dobj = (v >> 9) & 63u, mut2 = v >> 15;
                    const size_t cell = lower_cell((uint32_t)(p[r][j] >> 32), (uint32_t)(p[r][i] >> 32));
                    atomicAdd(oc + cell, (unsigned long long)m | ((unsigned long long)mut2 << 32));
                    if (dobj)
                        atomicAdd(oo + cell, (unsigned long long)dobj | ((unsigned long long)sect << 32));
                }
            }
        }
    }
}

// Flat classes of one join launch: class k (2..kFlatMax) has n[k] groups whose
// postings start at off[k] in the compact postings, run-head words from hoff[k],
// and blocks [block0[k], block0[k] + nblocks[k]) of the launch.
struct FlatClasses {
    uint32_t n[kFlatMax + 1];
    uint64_t off[kFlatMax + 1];
    uint32_t hoff[kFlatMax + 1];
    uint32_t block0[kFlatMax + 1];
    uint32_t nblocks[kFlatMax + 1];
};

template <int K>
__device__ __forceinline__ bool flat_class_block(const FlatClasses &fc, const uint64_t *__restrict__ jp,
                                                 const uint32_t *__restrict__ fheads,
                                                 unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo)
{
    const uint32_t b = blockIdx.x - fc.block0[K];
    if (b >= fc.nblocks[K])
        return false;
    self_flat_groups<K>(b * blockDim.x + threadIdx.x, jp + fc.off[K], fc.n[K], fheads + fc.hoff[K], oc, oo);
    return true;
}

// The join launch: the first set_blocks blocks run the (chunk, pair) items, the rest
// the flat classes (largest size first), so that the latter fill the former's tail.
__global__ void __launch_bounds__(256, KSSD_SET_MINB) k_self_sets(const unsigned long long *__restrict__ items, uint32_t nitems,
                                                   uint32_t set_blocks, const uint64_t *__restrict__ jt,
                                                   const uint32_t *__restrict__ islot,
                                                   const uint64_t *__restrict__ jp,
                                                   const FlatClasses fc, const uint32_t *__restrict__ fheads,
                                                   unsigned long long *__restrict__ oc,
                                                   unsigned long long *__restrict__ oo)
{
    if (blockIdx.x < set_blocks) {
        self_set_item(blockIdx.x * blockDim.x + threadIdx.x, items, nitems, jt, islot, oc, oo);
        return;
    }
    static_assert(kFlatMax == 4, "one dispatch per flat class");
    if (flat_class_block<4>(fc, jp, fheads, oc, oo))
        return;
    if (flat_class_block<3>(fc, jp, fheads, oc, oo))
        return;
    flat_class_block<2>(fc, jp, fheads, oc, oo);
}

// One warp per big group: lanes stride over its k(k-1)/2 pairs.
__global__ void __launch_bounds__(256) k_self_big(const unsigned long long *__restrict__ list, uint32_t n,
                                                  const uint64_t *__restrict__ post,
                                                  unsigned long long *__restrict__ oc,
                                                  unsigned long long *__restrict__ oo)
{
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n)
        return;
    const unsigned long long item = __ldg(list + w);
    const uint32_t b = (uint32_t)item, k = (uint32_t)(item >> 32);
    // lane handles rows j = lane+1, lane+33, ... paired with every i < j; rows are
    // dealt round-robin so lanes carry near-equal work
    for (uint32_t j = 1 + lane; j < k; j += 32) {
        const uint64_t pj = __ldg(post + b + j);
        for (uint32_t i = 0; i < j; ++i)
            join_pair(__ldg(post + b + i), pj, oc, oo);
    }
}

// Groups with multi-object gid runs: one thread per group walks run pairs with the
// full min-over-cross-product rule; the lower-gid run is the reference side.
__global__ void k_self_conflict_groups(const unsigned long long *__restrict__ list, uint32_t n,
                                       const uint64_t *__restrict__ post, int ignoreconflict,
                                       unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned long long item = list[t];
        const uint32_t b = (uint32_t)item, e = b + (uint32_t)(item >> 32);
        // run (query side, higher gid) qb..qe
        for (uint32_t qb = b; qb < e;) {
            const uint32_t qg = (uint32_t)(post[qb] >> 32);
            uint32_t qe = qb + 1;
            while (qe < e && (uint32_t)(post[qe] >> 32) == qg)
                ++qe;
            for (uint32_t rb = b; rb < qb;) {
                const uint32_t rg = (uint32_t)(post[rb] >> 32);
                uint32_t re = rb + 1;
                while (re < qb && (uint32_t)(post[re] >> 32) == rg)
                    ++re;
                if (!(ignoreconflict && re - rb > 1)) {
                    int d = kMinInit;
                    for (uint32_t x = qb; x < qe && d; ++x)
                        for (uint32_t y = rb; y < re && d; ++y)
                            d = min(d, dna_pop((uint32_t)post[x] ^ (uint32_t)post[y]));
                    const size_t cell = lower_cell(qg, rg);
                    atomicAdd(oc + cell, inc_ctx(d));
                    if (d)
                        atomicAdd(oo + cell, inc_obj(d));
                }
                rb = re;
            }
            qb = qe;
        }
    }
}

// ------------------------------------------------------------------ self lower triangle: one-pass scan join
//
// The self step from the resident index alone, with nothing prepared beforehand: a
// persistent grid streams the context-group boundaries (gbeg) tile by tile, queues
// every group of >= 2 postings in shared memory and joins the queue at once -- one
// thread per group of at most kScanLaneMax postings, the whole CTA for a larger one.
// Every pair of gid runs of a group credits cell (higher gid, lower gid) with the
// minimum object difference over the two runs' cross product (the higher gid's run is
// the query run of count_lower at that context, src/command_ani.h:694-716);
// --ignoreconflict skips reference (lower-gid) runs of several objects.

constexpr uint32_t kScanThreads = 256;
#ifndef KSSD_SCAN_PER_THREAD
#define KSSD_SCAN_PER_THREAD 8
#endif
constexpr uint32_t kScanPerThread = KSSD_SCAN_PER_THREAD;
constexpr uint32_t kScanTile = kScanThreads * kScanPerThread;  // groups per tile (4 B of gbeg each)
constexpr uint32_t kScanLaneMax = 32;                          // larger groups: the whole CTA

__device__ __forceinline__ void credit_lower(unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo,
                                             uint32_t qg, uint32_t rg, int d)
{
    const size_t cell = lower_cell(qg, rg);
    atomicAdd(oc + cell, inc_ctx(d));
    if (d)
        atomicAdd(oo + cell, inc_obj(d));
}

// Query run [qb, qe) of gid qg against every reference run of [b, qb).
__device__ __forceinline__ void join_query_run(const uint64_t *__restrict__ post, uint32_t b, uint32_t qb,
                                               uint32_t qe, uint32_t qg, int ignoreconflict,
                                               unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo)
{
    const uint32_t q0 = (uint32_t)__ldg(post + qb);
    for (uint32_t rb = b; rb < qb;) {
        const uint64_t r0 = __ldg(post + rb);
        const uint32_t rg = (uint32_t)(r0 >> 32);
        uint32_t re = rb + 1;
        while (re < qb && (uint32_t)(__ldg(post + re) >> 32) == rg)
            ++re;
        if (!(ignoreconflict && re - rb > 1)) {
            int d = kMinInit;
            for (uint32_t x = qb; x < qe && d; ++x) {
                const uint32_t qo = x == qb ? q0 : (uint32_t)__ldg(post + x);
                for (uint32_t y = rb; y < re && d; ++y)
                    d = min(d, dna_pop(qo ^ (uint32_t)__ldg(post + y)));
            }
            credit_lower(oc, oo, qg, rg, d);
        }
        rb = re;
    }
}

// All run pairs of group [b, b + k) on one thread.
__device__ __forceinline__ void join_group_lane(const uint64_t *__restrict__ post, uint32_t b, uint32_t k,
                                                int ignoreconflict, unsigned long long *__restrict__ oc,
                                                unsigned long long *__restrict__ oo)
{
    const uint32_t e = b + k;
    const uint32_t g0 = (uint32_t)(__ldg(post + b) >> 32);
    uint32_t qb = b + 1;
    while (qb < e && (uint32_t)(__ldg(post + qb) >> 32) == g0)
        ++qb;
    while (qb < e) {
        const uint32_t qg = (uint32_t)(__ldg(post + qb) >> 32);
        uint32_t qe = qb + 1;
        while (qe < e && (uint32_t)(__ldg(post + qe) >> 32) == qg)
            ++qe;
        join_query_run(post, b, qb, qe, qg, ignoreconflict, oc, oo);
        qb = qe;
    }
}

// All run pairs of group [b, b + k) on the whole CTA: thread t takes the query runs
// starting at b + t, b + t + T, ...
__device__ __forceinline__ void join_group_cta(const uint64_t *__restrict__ post, uint32_t b, uint32_t k,
                                               int ignoreconflict, unsigned long long *__restrict__ oc,
                                               unsigned long long *__restrict__ oo)
{
    const uint32_t e = b + k;
    for (uint32_t x = b + 1 + threadIdx.x; x < e; x += blockDim.x) {
        const uint32_t qg = (uint32_t)(__ldg(post + x) >> 32);
        if ((uint32_t)(__ldg(post + x - 1) >> 32) == qg)
            continue;  // not the first posting of its run
        uint32_t qe = x + 1;
        while (qe < e && (uint32_t)(__ldg(post + qe) >> 32) == qg)
            ++qe;
        join_query_run(post, b, x, qe, qg, ignoreconflict, oc, oo);
    }
}

// Shared memory of k_self_scan: the tile's queue of shared groups, and (PAIRS) the
// exclusive prefix of the small groups' pair counts.
constexpr uint32_t kScanPairRanks = kScanLaneMax * (kScanLaneMax - 1) / 2;  // pairs of the largest small group
struct ScanSmem {
    unsigned long long queue[kScanTile];  // groups of 2..kScanLaneMax from the front, larger from the back
    uint32_t prefix[kScanTile];
    unsigned short pair[kScanPairRanks];  // (i, j) of every pair rank of a small group: i | j << 8
};

// One credit into the table, or into the triangle (no table, or no room).
__device__ __forceinline__ void credit_global(const CellTable &T, unsigned long long *__restrict__ oc,
                                              unsigned long long *__restrict__ oo, uint32_t qg, uint32_t rg, int d)
{
    if (T.key && table_credit(T, (uint32_t)lower_cell(qg, rg), d))
        return;
    credit_lower(oc, oo, qg, rg, d);
}

// The table's cells into the triangle (plain adds: a cell lives in one slot and the join
// has finished), slots emptied for the next call.
__global__ void k_cell_table_flush(uint32_t *__restrict__ key, unsigned long long *__restrict__ acc, uint32_t slots,
                                   unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const uint32_t cell = key[s];
        if (cell == kCellEmpty)
            continue;
        const ulonglong2 a = reinterpret_cast<const ulonglong2 *>(acc)[s];
        oc[cell] += a.x;
        if (a.y)
            oo[cell] += a.y;
        key[s] = kCellEmpty;
        reinterpret_cast<ulonglong2 *>(acc)[s] = make_ulonglong2(0, 0);
    }
}

// The pair (i < j) of rank t among the k(k-1)/2 pairs of a group: j(j-1)/2 <= t.
__device__ __forceinline__ void pair_of_rank(uint32_t t, uint32_t &i, uint32_t &j)
{
    j = (uint32_t)((1.0f + sqrtf(1.0f + 8.0f * (float)t)) * 0.5f);
    while (j * (j - 1) / 2 > t)
        --j;
    while ((j + 1) * j / 2 <= t)
        ++j;
    i = t - j * (j - 1) / 2;
}

// The same for the pairs of a large group (ranks up to 2^32, 64-bit arithmetic).
__device__ __forceinline__ void pair_of_rank_wide(uint32_t t, uint32_t &i, uint32_t &j)
{
    uint64_t jj = (uint64_t)((1.0 + sqrt(1.0 + 8.0 * (double)t)) * 0.5);
    while (jj * (jj - 1) / 2 > t)
        --jj;
    while ((jj + 1) * jj / 2 <= t)
        ++jj;
    j = (uint32_t)jj;
    i = (uint32_t)(t - jj * (jj - 1) / 2);
}

// Bounds of this thread's groups of tile t: groups g0 .. g0 + kScanPerThread - 1
// (contiguous per thread, so a warp reads one 1 KB span with 16-byte loads), the
// kScanPerThread + 1 values gbeg[g0 ..]; past the end they repeat gbeg[u] (empty groups).
__device__ __forceinline__ void scan_load_bounds(const uint32_t *__restrict__ gbeg, uint64_t u, uint64_t t,
                                                 uint32_t (&bnd)[kScanPerThread + 1])
{
    const uint64_t g0 = t * kScanTile + (uint64_t)threadIdx.x * kScanPerThread;
    if (g0 + kScanPerThread <= u) {
        const uint4 *v = reinterpret_cast<const uint4 *>(gbeg + g0);
#pragma unroll
        for (uint32_t j = 0; j < kScanPerThread / 4; ++j) {
            const uint4 w = __ldg(v + j);
            bnd[4 * j] = w.x;
            bnd[4 * j + 1] = w.y;
            bnd[4 * j + 2] = w.z;
            bnd[4 * j + 3] = w.w;
        }
        bnd[kScanPerThread] = __ldg(gbeg + g0 + kScanPerThread);
    } else {
#pragma unroll
        for (uint32_t j = 0; j <= kScanPerThread; ++j)
            bnd[j] = __ldg(gbeg + min(g0 + j, u));
    }
}

// Per tile: every thread holds the bounds of kScanPerThread contiguous groups (loaded
// while the previous tile was joined), one block scan places the tile's shared groups
// in the queue.  PAIRS (a conflict-free index: one object per gid run): the small
// groups' pairs are then dealt out evenly, thread t taking a contiguous range of the
// tile's pair ranks and loading the postings of kScanPairBatch pairs before it credits
// them (2: more costs registers and idle predicated slots at ~2 pairs per lane and
// tile), so every lane runs the same short sequence per pair and no thread walks a
// whole large group while the others wait; with conflicts every thread walks whole
// groups (run cross products).  Groups of more than kScanLaneMax postings are taken by
// the whole CTA.
#ifndef KSSD_SCAN_PAIR_TABLE
#define KSSD_SCAN_PAIR_TABLE 1
#endif
#ifndef KSSD_SCAN_PAIR_BATCH
#define KSSD_SCAN_PAIR_BATCH 2
#endif
constexpr uint32_t kScanPairBatch = KSSD_SCAN_PAIR_BATCH;
static_assert(kScanPerThread % 4 == 0, "contiguous bounds are loaded 4 at a time");

// four CTAs per SM (64 registers): 2,000 genomes 0.112 vs 0.124 ms per join with three
#ifndef KSSD_SCAN_MINB
#define KSSD_SCAN_MINB 4
#endif
template <bool PAIRS>
__global__ void __launch_bounds__(kScanThreads, KSSD_SCAN_MINB) k_self_scan(const uint32_t *__restrict__ gbeg, uint64_t u,
                                                            const uint64_t *__restrict__ post, int ignoreconflict,
                                                            CellTable table,
                                                            unsigned long long *__restrict__ oc,
                                                            unsigned long long *__restrict__ oo)
{
    extern __shared__ __align__(16) unsigned char scan_smem[];
    ScanSmem &S = *reinterpret_cast<ScanSmem *>(scan_smem);
    using Scan = cub::BlockScan<unsigned long long, kScanThreads>;
    __shared__ typename Scan::TempStorage scan_tmp;
    const uint64_t ntiles = (u + kScanTile - 1) / kScanTile;
    bool waited = false;
#if KSSD_SCAN_PAIR_TABLE
    if (PAIRS) {
        for (uint32_t t = threadIdx.x; t < kScanPairRanks; t += kScanThreads) {
            uint32_t i, j;
            pair_of_rank(t, i, j);
            S.pair[t] = (unsigned short)(i | (j << 8));
        }
        // visible to every thread after the first tile's queue barrier
    }
#endif
    uint32_t bnd[kScanPerThread + 1];
    if (blockIdx.x < ntiles)
        scan_load_bounds(gbeg, u, blockIdx.x, bnd);
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        // the next tile's bounds are in flight while this tile is joined
        uint32_t nxt[kScanPerThread + 1];
        if (t + gridDim.x < ntiles)
            scan_load_bounds(gbeg, u, t + gridDim.x, nxt);
        // this thread's small groups (bits 0-15), large groups (bits 16-31) and small
        // pairs (bits 32-63): at most 2,048 x 2 groups and 2,048 x 496 pairs per tile,
        // so one 64-bit scan carries all three without overflow between the fields
        uint32_t cnt[kScanPerThread];
        unsigned long long mine = 0;
#pragma unroll
        for (uint32_t j = 0; j < kScanPerThread; ++j) {
            const uint32_t k = bnd[j + 1] - bnd[j];
            cnt[j] = k;
            const bool small = k >= 2 && k <= kScanLaneMax;
            mine += small ? (1ull | ((unsigned long long)(k * (k - 1) / 2) << 32))
                          : (k > kScanLaneMax ? 0x10000ull : 0ull);
        }
        unsigned long long off, tot;
        Scan(scan_tmp).ExclusiveSum(mine, off, tot);
        uint32_t sl = (uint32_t)off & 0xFFFFu, ll = ((uint32_t)off >> 16) & 0xFFFFu;
        uint32_t poff = (uint32_t)(off >> 32);
#pragma unroll
        for (uint32_t j = 0; j < kScanPerThread; ++j) {
            const uint32_t k = cnt[j];
            const unsigned long long item = (unsigned long long)bnd[j] | ((unsigned long long)k << 32);
            if (k >= 2 && k <= kScanLaneMax) {
                S.queue[sl] = item;
                if (PAIRS) {
                    S.prefix[sl] = poff;
                    poff += k * (k - 1) / 2;
                }
                ++sl;
            } else if (k > kScanLaneMax) {
                S.queue[kScanTile - 1 - ll] = item;
                ++ll;
            }
        }
        __syncthreads();
        const uint32_t nl = (uint32_t)tot & 0xFFFFu, nc = ((uint32_t)tot >> 16) & 0xFFFFu;
        if (!waited) {
            pdl_wait_primary();  // the counters' zero fill has finished (no-op without a dependency)
            waited = true;
        }
        if (PAIRS) {
            const uint32_t total = (uint32_t)(tot >> 32);
            const uint32_t p0 = (uint32_t)((uint64_t)total * threadIdx.x / kScanThreads);
            const uint32_t p1 = (uint32_t)((uint64_t)total * (threadIdx.x + 1) / kScanThreads);
            if (p0 < p1) {
                // the group holding pair rank p0: the last q < nl with prefix[q] <= p0
                uint32_t lo = 0, hi = nl - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (S.prefix[mid] <= p0)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                uint32_t q = lo;
                for (uint32_t pr = p0; pr < p1; pr += kScanPairBatch) {
                    uint64_t pi[kScanPairBatch], pj[kScanPairBatch];
#pragma unroll
                    for (uint32_t x = 0; x < kScanPairBatch; ++x) {
                        if (pr + x < p1) {
                            while (q + 1 < nl && S.prefix[q + 1] <= pr + x)
                                ++q;
                            const unsigned long long item = S.queue[q];
                            uint32_t i, j;
#if KSSD_SCAN_PAIR_TABLE
                            const uint32_t ij = S.pair[pr + x - S.prefix[q]];
                            i = ij & 0xFFu;
                            j = ij >> 8;
#else
                            pair_of_rank(pr + x - S.prefix[q], i, j);
#endif
                            pi[x] = __ldg(post + (uint32_t)item + i);
                            pj[x] = __ldg(post + (uint32_t)item + j);
                        }
                    }
#pragma unroll
                    for (uint32_t x = 0; x < kScanPairBatch; ++x) {
                        if (pr + x < p1) {
                            const int d = min(kMinInit, dna_pop((uint32_t)pi[x] ^ (uint32_t)pj[x]));
                            credit_global(table, oc, oo, (uint32_t)(pj[x] >> 32), (uint32_t)(pi[x] >> 32), d);
                        }
                    }
                }
            }
        } else {
            for (uint32_t i = threadIdx.x; i < nl; i += kScanThreads) {
                const unsigned long long item = S.queue[i];
                join_group_lane(post, (uint32_t)item, (uint32_t)(item >> 32), ignoreconflict, oc, oo);
            }
        }
        for (uint32_t i = 0; i < nc; ++i) {
            const unsigned long long item = S.queue[kScanTile - 1 - i];
            const uint32_t b = (uint32_t)item, k = (uint32_t)(item >> 32);
            if (PAIRS && table.key) {
                // one object per gid: the group's pairs dealt out over the CTA, into the table
                const uint32_t np = (uint32_t)((uint64_t)k * (k - 1) / 2);  // k < 92,682 genomes
                for (uint32_t pr = threadIdx.x; pr < np; pr += kScanThreads) {
                    uint32_t x, y;
                    pair_of_rank_wide(pr, x, y);
                    const uint64_t px = __ldg(post + b + x), py = __ldg(post + b + y);
                    credit_global(table, oc, oo, (uint32_t)(py >> 32), (uint32_t)(px >> 32),
                                  min(kMinInit, dna_pop((uint32_t)px ^ (uint32_t)py)));
                }
            } else {
                join_group_cta(post, b, k, ignoreconflict, oc, oo);
            }
        }
        __syncthreads();  // the queue and the scan storage are reused by the next tile
#pragma unroll
        for (uint32_t j = 0; j <= kScanPerThread; ++j)
            bnd[j] = nxt[j];
    }
}

// Facts of the self join: groups of >= 2 postings, postings in them, their pairs,
// and whether any gid holds several objects of one context (a conflict).
__global__ void k_self_stats(const uint32_t *__restrict__ gbeg, uint64_t u, const uint64_t *__restrict__ post,
                             unsigned long long *__restrict__ tot)
{
    unsigned long long g2 = 0, p2 = 0, pairs = 0, conf = 0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < u; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = gbeg[g];
        const unsigned long long k = gbeg[g + 1] - b;
        if (k >= 2) {
            ++g2;
            p2 += k;
            pairs += k * (k - 1) / 2;
            uint32_t prev = (uint32_t)(post[b] >> 32);
            for (uint32_t i = 1; i < k && !conf; ++i) {
                const uint32_t gid = (uint32_t)(post[b + i] >> 32);
                conf |= gid == prev;
                prev = gid;
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        g2 += __shfl_down_sync(0xffffffffu, g2, o);
        p2 += __shfl_down_sync(0xffffffffu, p2, o);
        pairs += __shfl_down_sync(0xffffffffu, pairs, o);
        conf |= __shfl_down_sync(0xffffffffu, conf, o);
    }
    if ((threadIdx.x & 31) == 0 && (g2 || conf)) {
        atomicAdd(tot + 0, g2);
        atomicAdd(tot + 1, p2);
        atomicAdd(tot + 2, pairs);
        if (conf)
            atomicOr(tot + 3, 1ull);
    }
}

// ------------------------------------------------------------------ dense self join (tensor cores)
//
// For a conflict-free index whose shared contexts are dense (many genomes of one
// species: contexts held by most genomes), the four counters of every pair are one
// exact int8 GEMM.  Rows are the alleles of the shared contexts -- the distinct
// objects u seen at a context c among its postings.  With A'[q][(c,u)] = 1 when genome
// q holds object u at c, and for every genome r holding c with object o_r, d = min(
// dna_popcount(u ^ o_r), NUM_CODENS + 1):
//     F[r][(c,u)] = 1,  F[n+r][(c,u)] = d >= 1,  F[2n+r][(c,u)] = d >= 2,  F[3n+r][(c,u)] = d
// D = A' F^T gives, for q != r over their shared contexts, D[q][r] = num_ctx,
// D[q][n+r] = diff_obj, D[q][2n+r] = num_mut2_ctx and D[q][3n+r] = diff_obj_section:
// the counters of count_lower (src/command_ani.h:694-716; one object per gid run, so
// the minimum over the run cross product is that one difference).

// Alleles of a sample of the shared groups (groups g = i * stride, one warp each):
// tot[0] += distinct objects, tot[1] += postings.  Scales the shared postings to the
// dense join's allele count (its GEMM's K) for the density rule.
__global__ void k_allele_sample(const uint32_t *__restrict__ gbeg, uint64_t u, uint64_t stride, uint32_t samples,
                                const uint64_t *__restrict__ post, unsigned long long *__restrict__ tot)
{
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < samples; i += (gridDim.x * blockDim.x) >> 5) {
        const uint64_t g = (uint64_t)i * stride;
        if (g >= u)
            continue;
        const uint32_t b = gbeg[g], k = gbeg[g + 1] - b;
        if (k < 2)
            continue;
        uint32_t firsts = 0;
        for (uint32_t j = lane; j < k; j += 32) {
            const uint32_t o = (uint32_t)post[b + j];
            bool first = true;
            for (uint32_t t = 0; t < j && first; ++t)
                first = (uint32_t)post[b + t] != o;
            firsts += first;
        }
        for (int o = 16; o; o >>= 1)
            firsts += __shfl_down_sync(0xffffffffu, firsts, o);
        if (lane == 0) {
            atomicAdd(tot + 0, (unsigned long long)firsts);
            atomicAdd(tot + 1, (unsigned long long)k);
        }
    }
}

// Shared groups (>= 2 postings) as (begin | k << 32), appended in any order.
__global__ void k_dense_list(const uint32_t *__restrict__ gbeg, uint64_t u, unsigned long long *__restrict__ list,
                             unsigned int *__restrict__ n_list)
{
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x; g0 < u; g0 += stride) {
        const uint64_t g = g0 + threadIdx.x;
        uint32_t b = 0, k = 0;
        if (g < u) {
            b = gbeg[g];
            k = gbeg[g + 1] - b;
        }
        const bool want = k >= 2;
        const uint32_t at = warp_slot(n_list, want, lane);
        if (want)
            list[at] = (unsigned long long)b | ((unsigned long long)k << 32);
    }
}

// Largest shared group the dense join handles (its postings are held in shared
// memory), which also bounds the references: the dense join needs nref <= this.
constexpr uint32_t kDenseMaxGroup = 4096;
// From this many 128-genome blocks on, the dense join's GEMM runs per block below the
// diagonal instead of over the whole square.
constexpr uint64_t kDenseBlocks = 6;
constexpr int kDenseThreads = 256;

// Shared memory of the allele numbering for groups of at most n postings (n = the
// index's references): a hash of the group's objects (hcap = pow2 >= 2n slots: the
// object with a valid bit) and the allele values by number.
struct DenseGroupSmem {
    unsigned long long *hkey;  // hcap
    uint32_t *aval;            // n: allele values by number
};
__host__ __device__ __forceinline__ uint32_t dense_hcap(uint32_t n)
{
    uint32_t c = 64;
    while (c < 2 * n)
        c <<= 1;
    return c;
}
__host__ __device__ __forceinline__ size_t dense_group_smem(uint32_t n)
{
    return (size_t)dense_hcap(n) * 8 + (size_t)n * 4 + 64;
}
__device__ __forceinline__ DenseGroupSmem dense_group_view(unsigned char *base, uint32_t n)
{
    DenseGroupSmem g;
    g.hkey = reinterpret_cast<unsigned long long *>(base);
    g.aval = reinterpret_cast<uint32_t *>(g.hkey + dense_hcap(n));
    return g;
}

// The alleles of a group [b, b + k) (k <= n postings, one object per gid): its distinct
// objects, numbered 0..m-1 by hash slot order; afterwards aval[a] holds the object of
// allele a.  A few barriers instead of a sort: every posting's object is inserted into
// the hash (CAS on an empty slot, linear probing; 2k slots for at most k objects), each
// thread numbers the occupied slots of its contiguous segment after one block scan of
// their counts.  Returns m (on every thread); ends with a barrier.
__device__ uint32_t dense_group_alleles(const uint64_t *__restrict__ post, uint32_t b, uint32_t k,
                                        const DenseGroupSmem &g)
{
    using Scan = cub::BlockScan<uint32_t, kDenseThreads>;
    __shared__ typename Scan::TempStorage scan_tmp;
    const uint32_t hcap = dense_hcap(k), mask = hcap - 1;
    int lg = 0;
    while ((1u << lg) < hcap)
        ++lg;
    for (uint32_t i = threadIdx.x; i < hcap; i += kDenseThreads)
        g.hkey[i] = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < k; j += kDenseThreads) {
        const uint32_t o = (uint32_t)__ldg(post + b + j);
        const unsigned long long key = (1ull << 32) | o;
        uint32_t h = (o * 2654435761u) >> (32 - lg);
        for (uint32_t probe = 0; probe < hcap; ++probe) {
            const unsigned long long old = atomicCAS(&g.hkey[h], 0ull, key);
            if (old == 0ull || old == key)
                break;
            h = (h + 1) & mask;
        }
    }
    __syncthreads();
    const uint32_t seg = hcap / kDenseThreads, s0 = threadIdx.x * seg;  // hcap >= 64, a multiple of 256 or less
    uint32_t mine = 0;
    for (uint32_t i = 0; i < seg; ++i)
        mine += g.hkey[s0 + i] != 0ull;
    if (hcap < kDenseThreads)
        mine = threadIdx.x < hcap ? (g.hkey[threadIdx.x] != 0ull) : 0u;
    uint32_t first, m;
    Scan(scan_tmp).ExclusiveSum(mine, first, m);
    if (hcap < kDenseThreads) {
        if (threadIdx.x < hcap && g.hkey[threadIdx.x])
            g.aval[first] = (uint32_t)g.hkey[threadIdx.x];
    } else {
        for (uint32_t i = 0; i < seg; ++i) {
            const unsigned long long key = g.hkey[s0 + i];
            if (key)
                g.aval[first++] = (uint32_t)key;
        }
    }
    __syncthreads();
    return m;
}

// Alleles (distinct objects) of every listed shared group: one CTA per group.  The
// count goes to alleles[s]; the values, in allele-number order, to aval[b..b + m) where b
// is the group's first posting (a group has at least as many postings as alleles).
__global__ void __launch_bounds__(kDenseThreads) k_dense_alleles(const unsigned long long *__restrict__ list,
                                                                 uint32_t n_list, const uint64_t *__restrict__ post,
                                                                 uint32_t nref, uint32_t *__restrict__ alleles,
                                                                 uint32_t *__restrict__ aval)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    const DenseGroupSmem g = dense_group_view(dsm, nref);
    for (uint32_t s = blockIdx.x; s < n_list; s += gridDim.x) {
        const unsigned long long item = list[s];
        const uint32_t b = (uint32_t)item;
        const uint32_t m = dense_group_alleles(post, b, (uint32_t)(item >> 32), g);
        if (threadIdx.x == 0)
            alleles[s] = m;
        // g.aval is rewritten only after two barriers of the next group's numbering
        for (uint32_t i = threadIdx.x; i < m; i += kDenseThreads)
            aval[b + i] = g.aval[i];
    }
}

// Genome -> object map of one group for k_dense_rows: the object of genome r as a u32
// word and a presence bit.  The words sit in 16-byte chunks (4 genomes), permuted inside
// blocks of 8 chunks (chunk c at c ^ ((c >> 3) & 7)); the 8 lanes of a quarter warp read
// 8 consecutive chunks, which stay on 8 different bank groups.
__host__ __device__ __forceinline__ uint32_t dense_gobj_words(uint32_t npad) { return (npad + 31) / 32 * 32; }
__host__ __device__ __forceinline__ size_t dense_rows_smem(uint32_t npad)
{
    return (size_t)dense_gobj_words(npad) * 4 + (size_t)dense_gobj_words(npad) / 8;
}
__device__ __forceinline__ uint32_t dense_gobj_slot(uint32_t r)
{
    const uint32_t c = r >> 2;
    return ((c ^ ((c >> 3) & 7u)) << 2) | (r & 3u);
}

// The operand rows of every allele, written whole (allele-major: a row runs over the
// genomes, so the GEMM takes both operands MN-major): A'[a][q] = 1 where genome q holds
// the allele; F[a][4 r + x] for every genome r at the allele's context, x = 0..3:
// 1, d >= 1, d >= 2, d = min(dna_popcount(u ^ o_r), NUM_CODENS + 1) (genome-major, so
// that the columns of a block of genomes are one contiguous range).  One CTA per group:
// the group's alleles come from k_dense_alleles (values at the group's first posting,
// rows from abase[s]); the CTA maps genome -> object from the postings, then every
// thread takes (allele, 4 genomes) pieces, consecutive threads on consecutive genomes
// of one allele, and stores the piece's 4 bytes of A' and 16 bytes of F straight to the
// operands (a warp's stores of one allele are contiguous), zeros included.
__global__ void __launch_bounds__(kDenseThreads) k_dense_rows(const unsigned long long *__restrict__ list,
                                                              uint32_t n_list, const uint32_t *__restrict__ abase,
                                                              const uint32_t *__restrict__ aval,
                                                              const uint64_t *__restrict__ post, uint32_t npad,
                                                              int8_t *__restrict__ A, int8_t *__restrict__ F)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    uint32_t *gobj = reinterpret_cast<uint32_t *>(dsm);
    uint32_t *gbit = gobj + dense_gobj_words(npad);
    const uint32_t nquad = npad / 4, nbit = dense_gobj_words(npad) / 32;
    for (uint32_t s = blockIdx.x; s < n_list; s += gridDim.x) {
        const unsigned long long item = list[s];
        const uint32_t b = (uint32_t)item, k = (uint32_t)(item >> 32);
        const uint32_t a0 = abase[s], m = abase[s + 1] - a0;
        for (uint32_t i = threadIdx.x; i < nbit; i += kDenseThreads)
            gbit[i] = 0u;
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < k; j += kDenseThreads) {
            const uint64_t p = __ldg(post + b + j);
            const uint32_t r = (uint32_t)(p >> 32);
            gobj[dense_gobj_slot(r)] = (uint32_t)p;
            atomicOr(&gbit[r >> 5], 1u << (r & 31u));
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < m * nquad; t += kDenseThreads) {
            const uint32_t a = t / nquad, c = t - a * nquad;  // allele, genomes 4c..4c+3
            const uint32_t u = __ldg(aval + b + a);
            const uint4 o4 = *reinterpret_cast<const uint4 *>(gobj + ((c ^ ((c >> 3) & 7u)) << 2));
            // one byte a genome: d (0..NUM_CODENS + 1, so < 128) of the present genomes,
            // then the thresholds by bytewise adds into bit 7 (no carry leaves a byte);
            // d = 0 exactly when the object is the allele's
            const uint32_t pm = (((gbit[c >> 3] >> ((c & 7u) * 4)) & 0xFu) * 0x204081u) & 0x01010101u;  // bit i -> byte i
            const uint32_t d0 = (uint32_t)min(kMinInit, dna_pop(u ^ o4.x));
            const uint32_t d1 = (uint32_t)min(kMinInit, dna_pop(u ^ o4.y));
            const uint32_t d2 = (uint32_t)min(kMinInit, dna_pop(u ^ o4.z));
            const uint32_t d3 = (uint32_t)min(kMinInit, dna_pop(u ^ o4.w));
            const uint32_t D = __byte_perm(__byte_perm(d0, d1, 0x0040u), __byte_perm(d2, d3, 0x0040u), 0x5410u) &
                               (pm * 0xFFu);
            const uint32_t f1 = ((D + 0x7F7F7F7Fu) >> 7) & 0x01010101u;
            const uint32_t f2 = ((D + 0x7E7E7E7Eu) >> 7) & 0x01010101u;
            const size_t row = (size_t)(a0 + a);
            reinterpret_cast<uint32_t *>(A + row * npad)[c] = pm ^ f1;
            // 4 x 4 byte transpose of (present, d >= 1, d >= 2, d): word e = genome 4c + e
            const uint32_t lo01 = __byte_perm(pm, f1, 0x5140u), hi01 = __byte_perm(pm, f1, 0x7362u);
            const uint32_t lo23 = __byte_perm(f2, D, 0x5140u), hi23 = __byte_perm(f2, D, 0x7362u);
            reinterpret_cast<uint4 *>(F + row * 4 * npad)[c] =
                make_uint4(__byte_perm(lo01, lo23, 0x5410u), __byte_perm(lo01, lo23, 0x7632u),
                           __byte_perm(hi01, hi23, 0x5410u), __byte_perm(hi01, hi23, 0x7632u));
        }
        __syncthreads();  // the map is reused by the next group
    }
}

// Packed lower triangle from D (npad x 4 npad, D[q][4 r + x]; with the blocked GEMM only
// the blocks at or below the diagonal are computed): every cell written (zeros included).
__global__ void k_dense_epilogue(const int32_t *__restrict__ D, uint32_t npad, size_t cells,
                                 unsigned long long *__restrict__ oc, unsigned long long *__restrict__ oo)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
        // row q: the largest q with q (q - 1) / 2 <= c
        uint32_t q = (uint32_t)((1.0 + sqrt(1.0 + 8.0 * (double)c)) * 0.5);
        while ((size_t)q * (q - 1) / 2 > c)
            --q;
        while ((size_t)(q + 1) * q / 2 <= c)
            ++q;
        const uint32_t r = (uint32_t)(c - (size_t)q * (q - 1) / 2);
        const int4 v = *reinterpret_cast<const int4 *>(D + (size_t)q * 4 * npad + 4 * (size_t)r);
        oc[c] = (unsigned long long)(uint32_t)v.x | ((unsigned long long)(uint32_t)v.z << 32);
        oo[c] = (unsigned long long)(uint32_t)v.y | ((unsigned long long)(uint32_t)v.w << 32);
    }
}

// ------------------------------------------------------------------ sparse-scan candidate votes

// Candidate nomination of the indexed sparse scan (src/pairwise_graph.c:1195-1246):
// sample q's keys at positions 0, step, 2*step, ... (qi = position / step) that are
// found in the index, in context groups of at most max_freq postings (0: any), vote
// once for every posting's gid r < q: votes[(q, r)] += 1 and first[(q, r)] =
// min(qi), the order in which the scan first touches r.  One thread per sketch key;
// the key's sample comes from a binary search of the offsets.
__global__ void __launch_bounds__(256) k_self_votes(const Slot *__restrict__ table, uint32_t mask,
                                                    const uint64_t *__restrict__ post,
                                                    const uint64_t *__restrict__ keys,
                                                    const uint64_t *__restrict__ offs, int n, uint64_t nkeys,
                                                    int obj_bits, uint32_t max_freq, uint32_t step,
                                                    uint32_t *__restrict__ votes, uint32_t *__restrict__ first)
{
    const uint64_t base = offs[0];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nkeys;
         i += (uint64_t)gridDim.x * blockDim.x) {
        // the sample holding absolute key base + i: the last q with offs[q] <= base + i
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(offs + mid) <= base + i)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int q = lo;
        const uint64_t pos = base + i - __ldg(offs + q);
        if (q == 0 || pos % step)
            continue;
        const uint32_t qi = (uint32_t)(pos / step);
        const unsigned long long ctx = __ldg(keys + i) >> obj_bits;
        unsigned long long payload;
        bool single;
        if (!table_lookup(table, mask, ctx, payload, single))
            continue;
        uint32_t pb = 0, pc = 1;
        if (!single) {
            pb = (uint32_t)payload;
            pc = (uint32_t)(payload >> 32);
        }
        if (max_freq && pc > max_freq)
            continue;
        for (uint32_t k = 0; k < pc; ++k) {
            const uint32_t gid = single ? (uint32_t)(payload >> 32) : (uint32_t)(__ldg(post + pb + k) >> 32);
            if ((int)gid >= q)
                break;
            const size_t cell = (size_t)q * (q - 1) / 2 + gid;
            atomicAdd(votes + cell, 1u);
            atomicMin(first + cell, qi);
        }
    }
}

// ------------------------------------------------------------------ helpers

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap && p)
            return cudaSuccess;
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess)
            cap = std::max<size_t>(n, 1);
        return e;
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// ------------------------------------------------------------------ sketching (FASTA/FASTQ)
// The reference's sketch of sequence (src/command_sketch.c:3913-3949): every k-mer of a
// record whose bases are all A/C/G/T (either case) takes the canonical context (the
// smaller of the forward and reverse-complement contexts under the context mask, the
// reverse on a tie), is kept when the 32-bit hash of that context is <= UINT32_MAX >>
// drfold, and becomes ctx << obj_bits | obj by extracting the mask's bits of the k-mer
// on the chosen strand.  Per sample: sort, dedup, and without conflict mode the contexts
// holding several objects dropped (src/command_sketch.c:4156-4188, src/kssdlib_sort.c:388-406).
struct SketchGeom {
    unsigned long long ctxmask, tupmask;
    int klen, obj_bits;
    uint32_t filter;
};

// SplitMix64 finalizer (Steele, Lea, Flood 2014): the sketch's context hash (the
// reference's mix64 in src/kssdlib_hash.h, which the sketch files' hash_id names)
__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// bits of x under mask m, packed from the low end (BMI2 pext)
__device__ __forceinline__ unsigned long long extract_bits(unsigned long long x, unsigned long long m)
{
    unsigned long long r = 0;
    int k = 0;
    while (m) {
        const int b = __ffsll((long long)m) - 1;
        r |= ((x >> b) & 1ull) << k++;
        m &= m - 1;
    }
    return r;
}

// 2-bit code of a base, -1 for anything but A/C/G/T in either case
__device__ __forceinline__ int base_code(unsigned char c)
{
    switch (c | 0x20) {
    case 'a': return 0;
    case 'c': return 1;
    case 'g': return 2;
    case 't': return 3;
    default: return -1;
    }
}

constexpr int kSketchThreads = 256;
constexpr int kSketchSpan = 64;                               // k-mer end positions per thread
constexpr int kSketchTile = kSketchThreads * kSketchSpan;     // bytes per CTA
constexpr int kSketchHalo = 32;                               // >= klen - 1 bytes before the tile

// largest i in [0, n) with a[i] <= v (a[0] <= v)
__device__ __forceinline__ uint64_t last_le(const uint64_t *__restrict__ a, uint64_t n, uint64_t v)
{
    uint64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(a + mid) <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Pass 1 (WRITE = false): kept k-mers per thread (counts) and per sample; pass 2: the
// keys, each thread's at out[pos[thread] ...] (byte order, so grouped by sample).
// Records rec_offs[r]..rec_offs[r+1] of seq; sample s = records samp_recs[s]..samp_recs[s+1].
template <bool WRITE>
__global__ void __launch_bounds__(kSketchThreads) k_sketch_scan(
    const unsigned char *__restrict__ seq, uint64_t n, const uint64_t *__restrict__ rec_offs, uint64_t nrec,
    const uint64_t *__restrict__ samp_recs, int nsamples, SketchGeom g, uint32_t *__restrict__ counts,
    uint32_t *__restrict__ samp_counts, const uint32_t *__restrict__ pos, unsigned long long *__restrict__ out)
{
    __shared__ unsigned char tile[kSketchHalo + kSketchTile];
    const uint64_t t0 = (uint64_t)blockIdx.x * kSketchTile;
    // stage the tile and its halo (coalesced bytes; the tile start is 32-byte aligned)
    for (int i = threadIdx.x; i < kSketchHalo + kSketchTile; i += kSketchThreads) {
        const int64_t p = (int64_t)t0 - kSketchHalo + i;
        tile[i] = (p >= 0 && (uint64_t)p < n) ? seq[p] : (unsigned char)'N';
    }
    __syncthreads();
    const uint64_t gt = (uint64_t)blockIdx.x * kSketchThreads + threadIdx.x;
    const uint64_t p0 = gt * kSketchSpan;
    uint32_t kept = 0;
    if (p0 < n && nrec) {
        const uint64_t p1 = min(n, p0 + kSketchSpan);
        const int len_mv = 2 * g.klen - 2;
        uint64_t r = last_le(rec_offs, nrec + 1, p0);   // record holding p0 (or the last empty one before)
        uint64_t rs = __ldg(rec_offs + r), re = r < nrec ? __ldg(rec_offs + r + 1) : rs;
        uint64_t p = p0 >= rs + (uint64_t)(g.klen - 1) ? p0 - (g.klen - 1) : rs;
        unsigned long long tuple = 0, crv = 0;
        int run = 0;
        uint32_t wi = 0;
        const uint32_t wbase = WRITE ? pos[gt] : 0;
        for (; p < p1; ++p) {
            while (p >= re && r < nrec) {  // next record: the k-mer state starts over
                ++r;
                rs = re;
                re = r < nrec ? __ldg(rec_offs + r + 1) : rs;
                run = 0;
                tuple = crv = 0;
            }
            if (r >= nrec)
                break;
            const int v = base_code(tile[kSketchHalo + (int64_t)(p - t0)]);
            if (v < 0) {
                run = 0;
                tuple = crv = 0;
                continue;
            }
            tuple = (tuple << 2) | (unsigned long long)v;
            crv = (crv >> 2) | ((unsigned long long)(v ^ 3) << len_mv);
            if (++run < g.klen || p < p0)
                continue;
            const unsigned long long tc = tuple & g.ctxmask, rc = crv & g.ctxmask;
            const bool fwd = tc < rc;
            const unsigned long long uctx = fwd ? tc : rc;
            if ((uint32_t)splitmix64(uctx) > g.filter)
                continue;
            if (WRITE) {
                const unsigned long long ut = (fwd ? tuple : crv) & g.tupmask;
                out[wbase + wi++] = (extract_bits(ut, g.ctxmask) << g.obj_bits) |
                                    extract_bits(ut, g.tupmask & ~g.ctxmask);
            } else {
                ++kept;
                const int sm = (int)last_le(samp_recs, (uint64_t)nsamples + 1, r);
                atomicAdd(samp_counts + min(sm, nsamples - 1), 1u);
            }
        }
    }
    if (!WRITE && gt < (n + kSketchSpan - 1) / kSketchSpan)
        counts[gt] = kept;
}

// keep[i]: key i of its sample's sorted run is the first of its duplicates and (without
// conflict mode) the only object of its context; kept keys counted per sample
__global__ void k_sketch_keep(const unsigned long long *__restrict__ k, uint64_t n, const uint32_t *__restrict__ seg,
                              int nsamples, int obj_bits, int conflict, uint8_t *__restrict__ keep,
                              uint32_t *__restrict__ kept)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        // sample of key i: the last segment starting at or before i that is not empty
        int lo = 0, hi = nsamples - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (seg[mid] <= i)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint64_t b = seg[lo], e = seg[lo + 1];
        const unsigned long long x = k[i];
        bool ok = i == b || k[i - 1] != x;
        if (ok && !conflict) {
            const unsigned long long c = x >> obj_bits;
            if (i > b && (k[i - 1] >> obj_bits) == c)
                ok = false;
            uint64_t j = i + 1;
            while (ok && j < e && k[j] == x)
                ++j;
            if (ok && j < e && (k[j] >> obj_bits) == c)
                ok = false;
        }
        keep[i] = ok ? 1 : 0;
        if (ok)
            atomicAdd(kept + lo, 1u);
    }
}

int grid_for(uint64_t n, int block = 256)
{
    uint64_t g = (n + block - 1) / block;
    if (g < 1)
        g = 1;
    if (g > 148ull * 64)
        g = 148ull * 64;
    return (int)g;
}

}  // namespace

struct kssdgpu_index {
    int device = 0;
    int nref = 0;
    int obj_bits = 20;
    uint64_t n = 0;
    uint64_t u = 0;
    uint64_t *post = nullptr;
    unsigned long long *gkey = nullptr;
    uint32_t *gbeg = nullptr;
    Slot *table = nullptr;
    uint4 *bloom = nullptr;                 // membership filter of the contexts (see bloom_may_hold)
    uint32_t bloom_mask = 0;                // 32-byte blocks per stripe - 1
    int bloom_stripes = 1;                  // key-range stripes of the filter
    unsigned long long *bloom_bounds = nullptr;  // first context of each stripe (stripes + 1 words)
    DevBuf<uint64_t> s_spos;                // stripe-major count: entry offsets per (query, stripe)
    DevBuf<uint32_t> s_scnt, s_spre;        // stripe-major count: chunks per (stripe, query), their offsets
    DevBuf<WorkItem> s_sitems;              // stripe-major count: the chunks
    bool count_striped = true;              // with several filter stripes, global rows run stripe-major
    bool count_filter = true;               // batched counts consult the filter (kssdgpu_count_tune may turn it off)
    uint32_t mask = 0;
    int *err = nullptr;
    unsigned int *work = nullptr;
    int sms = 148;
    int l2_bytes = 0;
    // host-API staging
    DevBuf<uint64_t> s_keys, s_offs;
    DevBuf<unsigned long long> s_out;
    DevBuf<int> s_order;
    DevBuf<WorkItem> s_items;
    DevBuf<uint32_t> s_prefix, s_counts;    // device-built chunk prefix of a query block
    DevBuf<uint32_t> s_qcnt, s_rcnt, s_dcount;  // detail filter: sketch sizes, candidates per row
    DevBuf<uint64_t> s_dprefix;             // detail filter: candidate offsets per row
    DevBuf<kssdgpu_hit_t> s_hits;           // detail filter: the candidates
    cudaStream_t pipe_st[3] = {nullptr, nullptr, nullptr};  // host-buffer pipeline: H2D, count, D2H
    std::vector<cudaEvent_t> pipe_ev;
    // batched-count setting (kssdgpu_count_tune): shared-memory rows where they fit, or
    // global rows in key-range chunks of count_chunk_keys entries
    bool count_smem = false;
    uint32_t count_chunk_keys = 4096;
    int count_tune_tried = 0;
    float count_tune_ms = 0;
    DevBuf<unsigned char> s_cubtmp;
    // self-join plan: compact small groups (descriptor offset | k << 32 into j_post),
    // big and conflict groups (begin | k << 32 into post)
    DevBuf<unsigned long long> j_small, j_big, j_conf;
    DevBuf<uint64_t> j_post;
    DevBuf<ulonglong2> j_chunks;            // set-major chunks of the small groups
    DevBuf<unsigned long long> j_items;     // (chunk, pair) work items, tile by tile (one warp each)
    DevBuf<uint64_t> j_tile;                // postings of the item chunks, row-interleaved by tile
    bool j_compact_ok = true;               // compact counters allowed (KSSDGPU_JOIN_COMPACT=0: never)
    bool j_compact = false;                 // the plan adds into compact slots of the touched cells
    uint32_t j_ntouched = 0;                // touched lower cells
    DevBuf<uint32_t> j_islot;               // compact slot of every item lane
    DevBuf<unsigned long long> j_touched;   // dense cell of every compact slot
    DevBuf<unsigned long long> j_cacc;      // compact counters, kCompactStride words per slot
    cudaStream_t j_fill_st = nullptr;       // the dense zero fill beside a compact join
    cudaEvent_t j_fill_ev[2] = {nullptr, nullptr};
    uint32_t j_nchunks = 0, j_nitems = 0;
    uint32_t j_chunk_size = 32;             // groups per set-major chunk (1..255)
    bool j_sort_chunks = true;              // chunks ordered by group count, largest first
    uint32_t j_flat_max = 1;                // small groups of up to this many genomes joined flat (1: none)
    FlatClasses j_flat{};                   // the flat classes of the plan
    DevBuf<uint32_t> j_fheads;              // their run heads, one word per 32 groups
    bool j_tuned = false;                   // the autotuner ran for this index
    int j_tune_tried = 0;                   // autotuner candidates timed (0: defaults kept)
    float j_tune_ms = 0;                    // the chosen candidate's join time
    uint32_t j_n[3] = {0, 0, 0};
    unsigned long long j_postings = 0, j_pairs = 0;
    bool j_ready = false;
    int scan_grid = 0;                      // CTAs of the one-pass scan join (resident per SM x SMs)
    DevBuf<double> m_val;                   // self matrix values (kssdgpu_self_lower_metric)
    DevBuf<kssd::RecheckCell> m_recheck;    // cells the host values
    DevBuf<unsigned long long> m_nrecheck;
    DevBuf<uint32_t> c_key;                 // scan join: table of touched cells (empty between calls)
    int c_log = kCellTableLog;              // its 2^c_log slots (KSSDGPU_CELL_TABLE_LOG, read at its allocation)
    DevBuf<unsigned long long> c_acc;       // scan join: its counter words
    // facts of the index, from one pass at build: shared groups (>= 2 postings), their
    // postings and pairs, whether any gid run holds several objects (a conflict)
    unsigned long long f_groups = 0, f_postings = 0, f_pairs = 0;
    unsigned long long f_alleles = 0;       // distinct objects of the shared contexts (sampled estimate)
    bool f_conflict = false;
    // dense self join scratch
    DevBuf<unsigned long long> d_list;
    DevBuf<uint32_t> d_poff, d_allele;
    DevBuf<uint32_t> d_aval;                // alleles of every listed group, at its first posting
    DevBuf<int8_t> d_a, d_f;
    DevBuf<int32_t> d_d;
    DevBuf<unsigned char> d_tmp, d_ws;
    unsigned long long d_alleles = 0;       // alleles of the last dense join (its GEMM's K before padding)
};

namespace {


// The contexts' membership filter: key-range stripes of U / S contexts each, a power of
// two of 32-byte blocks per stripe giving at least 8 bits per context, S the smallest
// power of two (at most kMaxStripes) that keeps a stripe within stripe_bytes.
int build_filter(kssdgpu_index *ix, uint64_t stripe_bytes, cudaStream_t st)
{
    cudaFree(ix->bloom);
    cudaFree(ix->bloom_bounds);
    ix->bloom = nullptr;
    ix->bloom_bounds = nullptr;
    ix->bloom_stripes = 1;
    ix->bloom_mask = 0;
    if (!ix->u)
        return KSSDGPU_OK;
    int stripes = 1;
    uint64_t blocks = 1;
    for (;;) {
        const uint64_t per = (ix->u + stripes - 1) / stripes;
        blocks = 1;
        while (blocks * 256 < per * 8)
            blocks <<= 1;
        if (blocks * 32 <= stripe_bytes || stripes >= kMaxStripes)
            break;
        stripes <<= 1;
    }
    const size_t fbytes = (size_t)stripes * blocks * 32;
    CUDA_TRY(cudaMalloc(&ix->bloom, fbytes));
    CUDA_TRY(cudaMalloc(&ix->bloom_bounds, (size_t)(stripes + 1) * sizeof(unsigned long long)));
    ix->bloom_stripes = stripes;
    ix->bloom_mask = (uint32_t)(blocks - 1);
    CUDA_TRY(cudaMemsetAsync(ix->bloom, 0, fbytes, st));
    k_stripe_bounds<<<1, 256, 0, st>>>(ix->gkey, ix->u, stripes, ix->bloom_bounds);
    k_bloom_insert<<<grid_for(ix->u), 256, 0, st>>>(ix->gkey, ix->u, ix->bloom_mask, stripes, ix->bloom_bounds,
                                                     reinterpret_cast<uint32_t *>(ix->bloom));
    count_launch(2);
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

int finish_build(kssdgpu_index *ix, uint32_t *head, unsigned long long *ctx_of, cudaStream_t st)
{
    const uint64_t n = ix->n;
    uint32_t *gidx = nullptr;
    CUDA_TRY(cudaMalloc(&gidx, std::max<uint64_t>(n, 1) * sizeof(uint32_t)));
    size_t tmp_bytes = 0;
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, head, gidx, (int64_t)n, st));
    void *tmp = nullptr;
    CUDA_TRY(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 1)));
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, head, gidx, (int64_t)n, st));
    count_launch();
    uint32_t last_idx = 0, last_head = 0;
    if (n) {
        CUDA_TRY(cudaMemcpyAsync(&last_idx, gidx + n - 1, 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(&last_head, head + n - 1, 4, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    ix->u = n ? (uint64_t)last_idx + last_head : 0;
    CUDA_TRY(cudaMalloc(&ix->gkey, std::max<uint64_t>(ix->u, 1) * sizeof(unsigned long long)));
    CUDA_TRY(cudaMalloc(&ix->gbeg, (ix->u + 1) * sizeof(uint32_t)));
    k_scatter_groups<<<grid_for(n), 256, 0, st>>>(head, gidx, ctx_of, n, ix->gkey, ix->gbeg, ix->u);
    count_launch();
    uint64_t cap = 1024;
    while (cap < 2 * ix->u)
        cap <<= 1;
    ix->mask = (uint32_t)(cap - 1);
    CUDA_TRY(cudaMalloc(&ix->table, cap * sizeof(Slot)));
    CUDA_TRY(cudaMemsetAsync(ix->table, 0xFF, cap * sizeof(Slot), st));
    k_table_insert<<<grid_for(ix->u), 256, 0, st>>>(ix->gkey, ix->gbeg, ix->u, ix->post, ix->table, ix->mask,
                                                     ix->err);
    count_launch();
    if (ix->u) {
        const int frc = build_filter(ix, kStripeBytes, st);
        if (frc)
            return frc;
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(tmp);
    cudaFree(gidx);
    int herr = 0;
    CUDA_TRY(cudaMemcpy(&herr, ix->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!herr && ix->u) {
        // facts of the shared contexts (sizes of the self joins; the dense path's conditions)
        unsigned long long *d = nullptr, h[4] = {0, 0, 0, 0};
        CUDA_TRY(cudaMalloc(&d, sizeof h));
        cudaError_t e = cudaMemsetAsync(d, 0, sizeof h, st);
        if (e == cudaSuccess) {
            k_self_stats<<<grid_for(ix->u), 256, 0, st>>>(ix->gbeg, ix->u, ix->post, d);
            count_launch();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFree(d);
        if (e != cudaSuccess)
            return fail(KSSDGPU_ERR_CUDA, std::string("index facts: ") + cudaGetErrorString(e));
        ix->f_groups = h[0];
        ix->f_postings = h[1];
        ix->f_pairs = h[2];
        ix->f_conflict = h[3] != 0;
        // the dense join's allele count, estimated from up to 65,536 sampled groups
        ix->f_alleles = ix->f_postings;
        if (ix->f_groups) {
            const uint32_t samples = (uint32_t)std::min<uint64_t>(ix->u, 65536);
            const uint64_t stride = ix->u / samples;
            unsigned long long *d2 = nullptr, h2[2] = {0, 0};
            CUDA_TRY(cudaMalloc(&d2, sizeof h2));
            e = cudaMemsetAsync(d2, 0, sizeof h2, st);
            if (e == cudaSuccess) {
                k_allele_sample<<<(samples * 32 + 255) / 256, 256, 0, st>>>(ix->gbeg, ix->u, stride, samples, ix->post,
                                                                           d2);
                count_launch();
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(h2, d2, sizeof h2, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            cudaFree(d2);
            if (e != cudaSuccess)
                return fail(KSSDGPU_ERR_CUDA, std::string("index facts: ") + cudaGetErrorString(e));
            if (h2[1])
                ix->f_alleles = std::max<unsigned long long>(
                    1, (unsigned long long)((double)ix->f_postings * (double)h2[0] / (double)h2[1]));
        }
    }
    if (herr == kDevUnsorted)
        return fail(KSSDGPU_ERR_UNSORTED, "index records are not sorted by (ctxgid, obj)");
    if (herr == kDevGid)
        return fail(KSSDGPU_ERR_GID, "index record gid is not below the reference count");
    if (herr == kDevProbe)
        return fail(KSSDGPU_ERR_TIMEOUT, "context hash table insert did not terminate");
    return KSSDGPU_OK;
}

int new_index(int nref, int obj_bits, int device, uint64_t n, kssdgpu_index **out)
{
    if (!out)
        return fail(KSSDGPU_ERR_ARG, "null output handle");
    *out = nullptr;
    if (nref <= 0 || nref >= (1 << kGidBits))
        return fail(KSSDGPU_ERR_ARG, "reference count must be in 1..2^20-1");
    if (obj_bits <= 0 || obj_bits > 32)
        return fail(KSSDGPU_ERR_ARG, "object width must be 1..32 bits");
    if (n >= 0xFFFFFFFFull)
        return fail(KSSDGPU_ERR_CAPACITY, "index entries must be below UINT32_MAX");
    CUDA_TRY(cudaSetDevice(device));
    auto *ix = new kssdgpu_index();
    ix->device = device;
    ix->nref = nref;
    ix->obj_bits = obj_bits;
    ix->n = n;
    cudaDeviceGetAttribute(&ix->sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&ix->l2_bytes, cudaDevAttrL2CacheSize, device);
    cudaError_t e = cudaMalloc(&ix->err, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMalloc(&ix->work, sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMemset(ix->err, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMalloc(&ix->post, std::max<uint64_t>(n, 1) * sizeof(uint64_t));
    if (e != cudaSuccess) {
        kssdgpu_index_free(ix);
        return fail(KSSDGPU_ERR_NOMEM, std::string("index allocation: ") + cudaGetErrorString(e));
    }
    *out = ix;
    return KSSDGPU_OK;
}

int check_dev_err(kssdgpu_index *ix, cudaStream_t st)
{
    int herr = 0;
    CUDA_TRY(cudaMemcpyAsync(&herr, ix->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
        cudaMemsetAsync(ix->err, 0, sizeof(int), st);
        if (herr == kDevUnsorted)
            return fail(KSSDGPU_ERR_UNSORTED, "query keys are not sorted ascending within a sample");
        if (herr == kDevGid)
            return fail(KSSDGPU_ERR_GID, "record gid is not below the reference count");
        return fail(KSSDGPU_ERR_TIMEOUT, "device probe loop exceeded its bound");
    }
    return KSSDGPU_OK;
}

uint32_t env_u32(const char *name, uint32_t def, uint32_t lo, uint32_t hi);

// The index's table of touched cells (allocated on first use with 2^KSSDGPU_CELL_TABLE_LOG
// slots, default 2^21; empty between calls: every kernel that fills it is followed by
// k_cell_table_flush on the same stream).
int cell_table(kssdgpu_index *ix, cudaStream_t st, CellTable &t)
{
    if (!ix->c_key.p || !ix->c_acc.p) {
        ix->c_log = (int)env_u32("KSSDGPU_CELL_TABLE_LOG", kCellTableLog, 4, 26);
        const size_t slots = (size_t)1 << ix->c_log;
        CUDA_TRY(ix->c_key.ensure(slots));
        CUDA_TRY(ix->c_acc.ensure(2 * slots));
        CUDA_TRY(cudaMemsetAsync(ix->c_key.p, 0xFF, slots * 4, st));
        CUDA_TRY(cudaMemsetAsync(ix->c_acc.p, 0, slots * 16, st));
    }
    t = CellTable{ix->c_key.p, ix->c_acc.p, ix->c_log};
    return KSSDGPU_OK;
}

template <bool LOWER, bool UNIQUE, bool SMEM>
int launch_batched(kssdgpu_index *ix, const CountParams &P, size_t smem, cudaStream_t st)
{
    auto kern = k_count_batched<LOWER, UNIQUE, SMEM>;
    if (smem > 48 * 1024)
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, smem));
    if (per_sm < 1)
        return fail(KSSDGPU_ERR_CAPACITY, "shared-memory row does not fit one CTA");
    int grid = ix->sms * per_sm;
    // with device-built chunks the count of work units stays on the device
    const int units = (!SMEM && P.items) ? P.nitems : (!SMEM && P.chunk_prefix) ? grid : P.nq;
    if (grid > units)
        grid = std::max(units, 1);
    CUDA_TRY(cudaMemsetAsync(P.work, 0, sizeof(unsigned int), st));
    kern<<<grid, 512, smem, st>>>(P);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

template <bool LOWER, bool UNIQUE>
int launch_striped(kssdgpu_index *ix, const CountParams &P, cudaStream_t st)
{
    auto kern = k_count_striped<LOWER, UNIQUE>;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 512, 0));
    const int grid = ix->sms * std::max(per_sm, 1);  // persistent: the item count stays on the device
    CUDA_TRY(cudaMemsetAsync(P.work, 0, sizeof(unsigned int), st));
    kern<<<grid, 512, 0, st>>>(P);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

template <bool LOWER, bool UNIQUE>
int launch_plain(kssdgpu_index *ix, const CountParams &P, const std::vector<uint64_t> &sizes, cudaStream_t st)
{
    for (int q = 0; q < P.nq; ++q) {
        if (!sizes[q])
            continue;
        const int grid = (int)((sizes[q] + 255) / 256);
        k_count_plain<LOWER, UNIQUE><<<grid, 256, 0, st>>>(P, q);
        count_launch();
    }
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

// shared-memory row budget: four 32-bit counters per reference (eight with unique)
constexpr size_t kSmemRowLimit = 112 * 1024;

bool smem_row_fits(const kssdgpu_index *ix, unsigned flags)
{
    return (size_t)ix->nref * sizeof(unsigned long long) * ((flags & KSSDGPU_UNIQUE) ? 4 : 2) <= kSmemRowLimit;
}

// Accumulator mode of a batched count: global rows in key-range chunks unless the
// caller forces shared-memory rows (KSSDGPU_SMEM_ACC) or the count autotuner chose
// them for this index; shared rows only where a row fits.
bool uses_smem_row(const kssdgpu_index *ix, unsigned flags)
{
    if (flags & (KSSDGPU_PLAIN | KSSDGPU_GLOBAL_ACC))
        return false;
    return smem_row_fits(ix, flags) && ((flags & KSSDGPU_SMEM_ACC) || ix->count_smem);
}

// Key-range chunks of at most `chunk` entries for the global-row kernel, the queries
// taken in the given order (offsets relative or absolute).
void build_chunks(const uint64_t *offs, int nq, const int *order, uint64_t chunk, std::vector<WorkItem> &items)
{
    items.clear();
    for (int k = 0; k < nq; ++k) {
        const int q = order ? order[k] : k;
        const uint64_t b = offs[q] - offs[0], e = offs[q + 1] - offs[0];
        for (uint64_t c = b; c < e; c += chunk)
            items.push_back(WorkItem{(uint32_t)q, 0u, c, std::min(e, c + chunk)});
    }
}

int count_dev_impl(kssdgpu_index *ix, const uint64_t *d_keys, const uint64_t *d_offs, int nq, int qgid_offset, bool lower,
                   unsigned flags, unsigned long long *oc, unsigned long long *oo, unsigned long long *uc,
                   unsigned long long *uo, const int *d_order, const std::vector<uint64_t> *sizes, cudaStream_t st,
                   const WorkItem *d_items = nullptr, int nitems = 0)
{
    const bool unique = (flags & KSSDGPU_UNIQUE) != 0;
    if (lower && unique)
        return fail(KSSDGPU_ERR_ARG, "unique-context counting has no lower-triangle form");
    if (unique && (!uc || !uo))
        return fail(KSSDGPU_ERR_ARG, "unique counters requested without output buffers");
    CountParams P{};
    P.table = ix->table;
    P.mask = ix->mask;
    P.post = ix->post;
    P.qkeys = d_keys;
    P.qoffs = d_offs;
    P.nq = nq;
    P.nref = ix->nref;
    P.qgid_offset = qgid_offset;
    P.obj_bits = ix->obj_bits;
    P.ignoreconflict = (flags & KSSDGPU_IGNORECONFLICT) ? 1 : 0;
    P.out_ctx = oc;
    P.out_obj = oo;
    P.out_uctx = uc;
    P.out_uobj = uo;
    P.work = ix->work;
    P.order = d_order;
    P.err = ix->err;
    P.bloom = ix->count_filter ? ix->bloom : nullptr;
    P.bloom_mask = ix->bloom_mask;
    P.bloom_stripes = ix->bloom_stripes;
    P.bloom_bounds = ix->bloom_bounds;
    const size_t cells = (size_t)nq * ix->nref;
    if (nq == 0)
        return KSSDGPU_OK;
    const size_t smem = (size_t)ix->nref * sizeof(unsigned long long) * (unique ? 4 : 2);
    const bool plain = (flags & KSSDGPU_PLAIN) != 0;
    if ((flags & KSSDGPU_SMEM_ACC) && !plain && !(flags & KSSDGPU_GLOBAL_ACC) && !smem_row_fits(ix, flags))
        return fail(KSSDGPU_ERR_CAPACITY, "shared-memory accumulator rows requested, but a row of " +
                                              std::to_string(ix->nref) + " references does not fit");
    const bool use_smem = uses_smem_row(ix, flags);
    P.chunk_keys = ix->count_chunk_keys;
    // stripe-major items when the filter is on and striped (global rows)
    const bool striped = !use_smem && !plain && !d_items && P.bloom && ix->count_striped && ix->bloom_stripes > 1 &&
                         (uint64_t)nq * (uint64_t)ix->bloom_stripes < (1ull << 30);
    if (striped) {
        // per (query, stripe): entry offsets, chunk counts, their scan, the chunks
        const int S = ix->bloom_stripes;
        const size_t npos = (size_t)nq * (S + 1), nsq = (size_t)nq * S;
        CUDA_TRY(ix->s_spos.ensure(npos));
        CUDA_TRY(ix->s_scnt.ensure(nsq + 1));
        CUDA_TRY(ix->s_spre.ensure(nsq + 1));
        CUDA_TRY(ix->s_sitems.ensure(nsq + kStripeItemsMax));
        size_t tb = 0;
        CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, ix->s_scnt.p, ix->s_spre.p, (int64_t)nsq + 1, st));
        CUDA_TRY(ix->s_cubtmp.ensure(tb));
        k_stripe_pos<<<grid_for(npos), 256, 0, st>>>(d_keys, d_offs, nq, S, ix->bloom_bounds, ix->obj_bits,
                                                      ix->s_spos.p);
        k_stripe_counts<<<grid_for(nsq + 1), 256, 0, st>>>(ix->s_spos.p, d_offs, nq, S, ix->s_scnt.p, ix->err);
        CUDA_TRY(cub::DeviceScan::ExclusiveSum(ix->s_cubtmp.p, tb, ix->s_scnt.p, ix->s_spre.p, (int64_t)nsq + 1, st));
        k_stripe_expand<<<grid_for(nsq), 256, 0, st>>>(ix->s_spos.p, d_offs, nq, S, ix->s_spre.p, ix->s_sitems.p);
        count_launch(4);
        P.items = ix->s_sitems.p;
        P.nitems_dev = ix->s_spre.p + nsq;
        P.order = nullptr;
    } else if (!use_smem && d_items) {
        P.items = d_items;
        P.nitems = nitems;
    } else if (!use_smem && !plain && nq > 0) {
        // device offsets only: chunk counts and their prefix on the device, so that a
        // large query (a read set) spreads over many SMs
        CUDA_TRY(ix->s_prefix.ensure((size_t)nq + 1));
        CUDA_TRY(ix->s_counts.ensure((size_t)nq));
        size_t tb = 0;
        CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tb, ix->s_counts.p, ix->s_prefix.p + 1, nq, st));
        CUDA_TRY(ix->s_cubtmp.ensure(tb));
        k_chunk_counts<<<std::min((nq + 255) / 256, ix->sms * 8), 256, 0, st>>>(d_offs, nq, ix->count_chunk_keys,
                                                                                ix->s_counts.p, ix->s_prefix.p);
        CUDA_TRY(cub::DeviceScan::InclusiveSum(ix->s_cubtmp.p, tb, ix->s_counts.p, ix->s_prefix.p + 1, nq, st));
        count_launch(3);
        P.chunk_prefix = ix->s_prefix.p;
    }
    if (!use_smem && !(flags & KSSDGPU_NO_ZERO)) {
        CUDA_TRY(cudaMemsetAsync(oc, 0, cells * 8, st));
        CUDA_TRY(cudaMemsetAsync(oo, 0, cells * 8, st));
        if (unique) {
            CUDA_TRY(cudaMemsetAsync(uc, 0, cells * 8, st));
            CUDA_TRY(cudaMemsetAsync(uo, 0, cells * 8, st));
        }
    }
    if (plain) {
        if (!sizes)
            return fail(KSSDGPU_ERR_ARG, "plain kernel needs host-side query sizes");
        if (lower)
            return launch_plain<true, false>(ix, P, *sizes, st);
        return unique ? launch_plain<false, true>(ix, P, *sizes, st) : launch_plain<false, false>(ix, P, *sizes, st);
    }
    if (use_smem) {
        if (lower)
            return launch_batched<true, false, true>(ix, P, smem, st);
        return unique ? launch_batched<false, true, true>(ix, P, smem, st)
                      : launch_batched<false, false, true>(ix, P, smem, st);
    }
    if (striped) {
        if (lower)
            return launch_striped<true, false>(ix, P, st);
        return unique ? launch_striped<false, true>(ix, P, st) : launch_striped<false, false>(ix, P, st);
    }
    if (lower)
        return launch_batched<true, false, false>(ix, P, 0, st);
    return unique ? launch_batched<false, true, false>(ix, P, 0, st) : launch_batched<false, false, false>(ix, P, 0, st);
}

// A host-buffer count is split into sub-blocks whose copies overlap the counting when
// the block is large and the host buffers are page-locked (asynchronous copies need it).
bool host_pinned(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

bool pipeline_worthwhile(kssdgpu_index *ix, int nq, uint64_t nkeys, const void *qkeys, const void *ctx)
{
    (void)ix;
    return nq >= 16 && nkeys >= (8ull << 20) && host_pinned(qkeys) && host_pinned(ctx);
}

// Sub-blocks of about equal key counts; per sub-block: keys H2D on one stream, the
// batched count on the compute stream (stream-ordered, so the index's scratch is
// reused safely), counter rows D2H on a third stream.
int count_host_pipelined(kssdgpu_index *ix, const uint64_t *qkeys, const uint64_t *qoffs, int nq, int qgid_offset,
                         bool lower, unsigned flags, void *ctx, void *obj, void *uctx, void *uobj,
                         const std::vector<uint64_t> &sizes)
{
    const bool unique = (flags & KSSDGPU_UNIQUE) != 0;
    const uint64_t nkeys = qoffs[nq] - qoffs[0];
    const int parts = std::min(8, nq / 2);
    std::vector<int> cut(1, 0);
    for (int p = 1; p < parts; ++p) {
        const uint64_t target = qoffs[0] + nkeys * (uint64_t)p / (uint64_t)parts;
        int q = (int)(std::upper_bound(qoffs, qoffs + nq + 1, target) - qoffs) - 1;
        q = std::max(q, cut.back() + 1);
        if (q < nq)
            cut.push_back(q);
    }
    cut.push_back(nq);
    const int np = (int)cut.size() - 1;
    // per sub-block query order (largest first) and key-range chunks, relative to it
    const bool smem = uses_smem_row(ix, flags);
    std::vector<int> order_all(nq);
    std::vector<WorkItem> items_all;
    std::vector<size_t> item_off(np + 1, 0);
    for (int p = 0; p < np; ++p) {
        const int q0 = cut[p], nb = cut[p + 1] - q0;
        int *ord = order_all.data() + q0;
        std::iota(ord, ord + nb, 0);
        std::stable_sort(ord, ord + nb, [&](int a, int b) { return sizes[q0 + a] > sizes[q0 + b]; });
        if (!smem) {
            std::vector<WorkItem> it;
            build_chunks(qoffs + q0, nb, ord, ix->count_chunk_keys, it);
            items_all.insert(items_all.end(), it.begin(), it.end());
        }
        item_off[p + 1] = items_all.size();
    }
    const size_t cells = (size_t)nq * ix->nref;
    const int nout = unique ? 4 : 2;
    CUDA_TRY(ix->s_keys.ensure(nkeys));
    CUDA_TRY(ix->s_offs.ensure((size_t)nq + 1));
    CUDA_TRY(ix->s_out.ensure(cells * nout));
    CUDA_TRY(ix->s_order.ensure((size_t)nq));
    CUDA_TRY(ix->s_items.ensure(items_all.size()));
    for (int i = 0; i < 3; ++i)
        if (!ix->pipe_st[i])
            CUDA_TRY(cudaStreamCreateWithFlags(&ix->pipe_st[i], cudaStreamNonBlocking));
    while ((int)ix->pipe_ev.size() < 2 * np) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ix->pipe_ev.push_back(e);
    }
    cudaStream_t sin = ix->pipe_st[0], scomp = ix->pipe_st[1], sout = ix->pipe_st[2];
    // small tables first, on the compute stream
    CUDA_TRY(cudaMemcpyAsync(ix->s_offs.p, qoffs, ((size_t)nq + 1) * 8, cudaMemcpyHostToDevice, scomp));
    CUDA_TRY(cudaMemcpyAsync(ix->s_order.p, order_all.data(), (size_t)nq * sizeof(int), cudaMemcpyHostToDevice, scomp));
    if (!items_all.empty())
        CUDA_TRY(cudaMemcpyAsync(ix->s_items.p, items_all.data(), items_all.size() * sizeof(WorkItem),
                                 cudaMemcpyHostToDevice, scomp));
    unsigned long long *oc = ix->s_out.p, *oo = oc + cells;
    unsigned long long *uc = unique ? oo + cells : nullptr, *uo = unique ? uc + cells : nullptr;
    void *hout[4] = {ctx, obj, uctx, uobj};
    unsigned long long *dout[4] = {oc, oo, uc, uo};
    for (int p = 0; p < np; ++p) {
        const int q0 = cut[p], nb = cut[p + 1] - q0;
        const uint64_t k0 = qoffs[q0] - qoffs[0], kn = qoffs[q0 + nb] - qoffs[q0];
        if (kn)
            CUDA_TRY(cudaMemcpyAsync(ix->s_keys.p + k0, qkeys + k0, kn * 8, cudaMemcpyHostToDevice, sin));
        CUDA_TRY(cudaEventRecord(ix->pipe_ev[2 * p], sin));
        CUDA_TRY(cudaStreamWaitEvent(scomp, ix->pipe_ev[2 * p], 0));
        const size_t c0 = (size_t)q0 * ix->nref, cn = (size_t)nb * ix->nref;
        std::vector<uint64_t> sub_sizes(sizes.begin() + q0, sizes.begin() + q0 + nb);
        const size_t ni = item_off[p + 1] - item_off[p];
        int rc = count_dev_impl(ix, ix->s_keys.p + k0, ix->s_offs.p + q0, nb, qgid_offset + q0, lower, flags, oc + c0,
                                oo + c0, unique ? uc + c0 : nullptr, unique ? uo + c0 : nullptr, ix->s_order.p + q0,
                                &sub_sizes, scomp, ni ? ix->s_items.p + item_off[p] : nullptr, (int)ni);
        if (rc)
            return rc;
        CUDA_TRY(cudaEventRecord(ix->pipe_ev[2 * p + 1], scomp));
        CUDA_TRY(cudaStreamWaitEvent(sout, ix->pipe_ev[2 * p + 1], 0));
        for (int o = 0; o < nout; ++o)
            CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned long long *>(hout[o]) + c0, dout[o] + c0, cn * 8,
                                     cudaMemcpyDeviceToHost, sout));
    }
    CUDA_TRY(cudaStreamSynchronize(sin));
    CUDA_TRY(cudaStreamSynchronize(scomp));
    return check_dev_err(ix, sout);
}

int count_host_impl(kssdgpu_index *ix, const uint64_t *qkeys, const uint64_t *qoffs, int nq, int qgid_offset, bool lower,
                    unsigned flags, void *ctx, void *obj, void *uctx, void *uobj)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    if (nq < 0 || (nq > 0 && (!qoffs || !ctx || !obj)))
        return fail(KSSDGPU_ERR_ARG, "invalid query block arguments");
    if (nq == 0)
        return KSSDGPU_OK;
    const bool unique = (flags & KSSDGPU_UNIQUE) != 0;
    if (unique && (!uctx || !uobj))
        return fail(KSSDGPU_ERR_ARG, "unique counters requested without output buffers");
    CUDA_TRY(cudaSetDevice(ix->device));
    const uint64_t nkeys = qoffs[nq] - qoffs[0];
    if (nkeys && !qkeys)
        return fail(KSSDGPU_ERR_ARG, "null query keys");
    std::vector<uint64_t> sizes(nq);
    for (int i = 0; i < nq; ++i) {
        if (qoffs[i + 1] < qoffs[i])
            return fail(KSSDGPU_ERR_ARG, "query offsets are not monotone");
        sizes[i] = qoffs[i + 1] - qoffs[i];
    }
    if (!(flags & KSSDGPU_PLAIN) && pipeline_worthwhile(ix, nq, nkeys, qkeys, ctx))
        return count_host_pipelined(ix, qkeys, qoffs, nq, qgid_offset, lower, flags, ctx, obj, uctx, uobj, sizes);
    std::vector<int> order(nq);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sizes[a] > sizes[b]; });
    std::vector<WorkItem> items;
    if (!uses_smem_row(ix, flags) && !(flags & KSSDGPU_PLAIN))
        build_chunks(qoffs, nq, order.data(), ix->count_chunk_keys, items);
    const size_t cells = (size_t)nq * ix->nref;
    const int nout = unique ? 4 : 2;
    CUDA_TRY(ix->s_keys.ensure(nkeys));
    CUDA_TRY(ix->s_offs.ensure((size_t)nq + 1));
    CUDA_TRY(ix->s_out.ensure(cells * nout));
    CUDA_TRY(ix->s_order.ensure((size_t)nq));
    CUDA_TRY(ix->s_items.ensure(items.size()));
    cudaStream_t st = 0;
    if (nkeys)
        CUDA_TRY(cudaMemcpyAsync(ix->s_keys.p, qkeys, nkeys * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_offs.p, qoffs, ((size_t)nq + 1) * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_order.p, order.data(), (size_t)nq * sizeof(int), cudaMemcpyHostToDevice, st));
    if (!items.empty())
        CUDA_TRY(cudaMemcpyAsync(ix->s_items.p, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                 st));
    unsigned long long *oc = ix->s_out.p, *oo = oc + cells;
    unsigned long long *uc = unique ? oo + cells : nullptr, *uo = unique ? uc + cells : nullptr;
    int rc = count_dev_impl(ix, ix->s_keys.p, ix->s_offs.p, nq, qgid_offset, lower, flags, oc, oo, uc, uo, ix->s_order.p,
                            &sizes, st, items.empty() ? nullptr : ix->s_items.p, (int)items.size());
    if (rc)
        return rc;
    CUDA_TRY(cudaMemcpyAsync(ctx, oc, cells * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(obj, oo, cells * 8, cudaMemcpyDeviceToHost, st));
    if (unique) {
        CUDA_TRY(cudaMemcpyAsync(uctx, uc, cells * 8, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(uobj, uo, cells * 8, cudaMemcpyDeviceToHost, st));
    }
    return check_dev_err(ix, st);
}

// ------------------------------------------------------------------ detail-mode candidate filter
//
// The pre-filter of the reference's detail branch (src/command_ani.h:585-609), fused
// behind the count on the device so that only candidate cells cross to the host.
// A cell (i, j) of the dense block is a candidate when num_ctx >= ctxcut, both
// sketch sizes are nonzero, max(num_ctx / qry_size, num_ctx / ref_size) >= afcut (all
// exact: integer and IEEE double division), and its naive ANI reaches anicut minus a
// margin: float 1 - diff_obj / num_ctx / 7 (IEEE float, exact), or with unique
// contexts 1 - naive_dist of the unique or full counters (the 5% rule of
// src/command_ani.h:437-440) in FP64 with the device's pow.  The margin makes the
// device set a superset of the reference's: the host re-applies the exact test (its
// own libm) to the candidates only.
struct DetailFilter {
    const uint32_t *qcnt;   // sketch sizes of the block's queries
    const uint32_t *rcnt;   // sketch sizes of the references
    uint32_t ctxcut;
    double afcut;
    double ani_lo;          // anicut minus the margin
    int unique;
};
constexpr double kDetailMargin = 1e-9;  // far above pow's few-ulp difference, far below a printed digit

// get_naive_dist (src/command_ani.h:202-224) in FP64 on the device
__device__ __forceinline__ double naive_dist_dev(uint32_t xny, uint32_t diff, uint32_t sect)
{
    if (xny == 0)
        return 1.0;
    const double eps = 1e-8;  // EPSILON, src/model_ani.h:224
    const double ratio = ((double)sect + eps) / ((double)diff + eps);
    const double dist0 = (double)diff / (double)(xny + diff);
    const double final_dist = 1.0 - pow(1.0 - dist0, ratio);
    if (final_dist <= 0.0)
        return 0.0;
#if KSSD_NUM_CODENS < 11
    const double scale = 0.1557143, intercept = 9.961e-5;
#else
    const double scale = 0.1544286, intercept = 7.133e-4;
#endif
    const double w = fmin(final_dist / 0.01, 1.0);  // NAIVE_DIST_INTERCEPT_RAMP_TAU
    return final_dist * scale + intercept * w;
}

__device__ __forceinline__ bool detail_candidate(const DetailFilter &F, int i, int j, unsigned long long c,
                                                 unsigned long long o, unsigned long long uc, unsigned long long uo)
{
    const uint32_t shared = (uint32_t)c;
    if (shared < F.ctxcut)
        return false;
    const uint32_t qs = F.qcnt[i], rs = F.rcnt[j];
    if (rs == 0 || qs == 0)
        return false;
    const double afq = (double)shared / (double)qs, afr = (double)shared / (double)rs;
    if ((afq > afr ? afq : afr) < F.afcut)
        return false;
    double ani;
    if (F.unique) {
        const bool use_u = (uint64_t)(uint32_t)uc * 20 >= (uint64_t)rs;  // rs > 0 here
        const unsigned long long xc = use_u ? uc : c, xo = use_u ? uo : o;
        ani = 1.0 - naive_dist_dev((uint32_t)xc, (uint32_t)xo, (uint32_t)(xo >> 32));
    } else {
        const float dist = __fdiv_rn(__fdiv_rn(__uint2float_rn((uint32_t)o), __uint2float_rn(shared)), 7.0f);
        ani = (double)__fsub_rn(1.0f, dist);
    }
    return ani >= F.ani_lo;
}

// Candidates per query row (one CTA per row).
__global__ void __launch_bounds__(256) k_detail_count(const unsigned long long *__restrict__ oc,
                                                      const unsigned long long *__restrict__ oo,
                                                      const unsigned long long *__restrict__ uc,
                                                      const unsigned long long *__restrict__ uo, int nq, int nref,
                                                      DetailFilter F, uint32_t *__restrict__ counts)
{
    __shared__ uint32_t total;
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        if (threadIdx.x == 0)
            total = 0;
        __syncthreads();
        const size_t row = (size_t)q * nref;
        uint32_t mine = 0;
        for (int j = threadIdx.x; j < nref; j += blockDim.x)
            mine += detail_candidate(F, q, j, oc[row + j], oo[row + j], uc ? uc[row + j] : 0ull,
                                     uo ? uo[row + j] : 0ull);
        for (int o = 16; o; o >>= 1)
            mine += __shfl_down_sync(0xffffffffu, mine, o);
        if ((threadIdx.x & 31) == 0 && mine)
            atomicAdd(&total, mine);
        __syncthreads();
        if (threadIdx.x == 0)
            counts[q] = total;
        __syncthreads();
    }
}

// The candidates of each row in ascending reference order at prefix[q] (one CTA per
// row, an ordered compaction 256 cells at a time).
__global__ void __launch_bounds__(256) k_detail_write(const unsigned long long *__restrict__ oc,
                                                      const unsigned long long *__restrict__ oo,
                                                      const unsigned long long *__restrict__ uc,
                                                      const unsigned long long *__restrict__ uo, int nq, int nref,
                                                      DetailFilter F, const uint64_t *__restrict__ prefix,
                                                      kssdgpu_hit_t *__restrict__ hits)
{
    using Scan = cub::BlockScan<uint32_t, 256>;
    __shared__ typename Scan::TempStorage tmp;
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        const size_t row = (size_t)q * nref;
        uint64_t at = prefix[q];
        for (int j0 = 0; j0 < nref; j0 += 256) {
            const int j = j0 + (int)threadIdx.x;
            unsigned long long c = 0, o = 0, u = 0, v = 0;
            bool keep = false;
            if (j < nref) {
                c = oc[row + j];
                o = oo[row + j];
                u = uc ? uc[row + j] : 0ull;
                v = uo ? uo[row + j] : 0ull;
                keep = detail_candidate(F, q, j, c, o, u, v);
            }
            uint32_t pos, sum;
            Scan(tmp).ExclusiveSum(keep ? 1u : 0u, pos, sum);
            if (keep) {
                kssdgpu_hit_t h;
                h.query = (uint32_t)q;
                h.ref = (uint32_t)j;
                h.num_ctx = (uint32_t)c;
                h.num_mut2_ctx = (uint32_t)(c >> 32);
                h.diff_obj = (uint32_t)o;
                h.diff_obj_section = (uint32_t)(o >> 32);
                h.u_num_ctx = (uint32_t)u;
                h.u_num_mut2_ctx = (uint32_t)(u >> 32);
                h.u_diff_obj = (uint32_t)v;
                h.u_diff_obj_section = (uint32_t)(v >> 32);
                hits[at + pos] = h;
            }
            at += sum;
            __syncthreads();  // the scan storage is reused
        }
    }
}

// prefix[0] = 0, prefix[q + 1] = prefix[q] + counts[q] (one CTA)
__global__ void __launch_bounds__(1024) k_detail_prefix(const uint32_t *__restrict__ counts, int nq,
                                                        uint64_t *__restrict__ prefix)
{
    __shared__ unsigned long long part[1024];
    const int per = (nq + 1023) / 1024;
    const int q0 = min(nq, (int)threadIdx.x * per), q1 = min(nq, q0 + per);
    unsigned long long sum = 0;
    for (int q = q0; q < q1; ++q)
        sum += counts[q];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const unsigned long long v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0ull;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0ull;
    if (threadIdx.x == 0)
        prefix[0] = 0;
    for (int q = q0; q < q1; ++q) {
        run += counts[q];
        prefix[q + 1] = run;
    }
}

// Runs of equal gid lists among the n sorted small groups -> chunks -> (chunk, pair)
// items (j_chunks, j_items); the per-group descriptors are released afterwards.
// Plan knobs, overridable for tuning: KSSDGPU_JOIN_CHUNK (groups per chunk, 1..255)
// , KSSDGPU_JOIN_SORT (0: chunks by size only, plan order within a size), KSSDGPU_JOIN_FLAT (largest group
// size joined flat, 1..4; 1: every small group as chunk items) and KSSDGPU_JOIN_COMPACT (0: the
// join always adds into the dense counters; 2: compact slots whenever possible).
uint32_t env_u32(const char *name, uint32_t def, uint32_t lo, uint32_t hi)
{
    const char *v = std::getenv(name);
    if (!v || !*v)
        return def;
    const unsigned long x = std::strtoul(v, nullptr, 10);
    return x < lo ? lo : x > hi ? hi : (uint32_t)x;
}

// One launch of the set-major join: the plan's (chunk, pair) items, then its flat
// classes, largest size first.
cudaError_t launch_sets(kssdgpu_index *ix, unsigned long long *oc, unsigned long long *oo, cudaStream_t st,
                        bool after_zero = false, bool compact = false)
{
    FlatClasses fc = ix->j_flat;
    const uint32_t sb = (ix->j_nitems + 255) / 256;
    uint32_t nb = sb;
    for (uint32_t k = kFlatMax; k >= 2; --k) {
        fc.block0[k] = nb;
        const uint32_t per_block = 256 * kFlatRounds((int)k);  // groups per block
        fc.nblocks[k] = (uint32_t)(((uint64_t)fc.n[k] + per_block - 1) / per_block);
        nb += fc.nblocks[k];
    }
    if (!nb)
        return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    if (after_zero && KSSD_JOIN_PDL) {
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_self_sets, (const unsigned long long *)ix->j_items.p, ix->j_nitems,
                                             sb, (const uint64_t *)ix->j_tile.p,
                                             compact ? (const uint32_t *)ix->j_islot.p : (const uint32_t *)nullptr,
                                             (const uint64_t *)ix->j_post.p, fc, (const uint32_t *)ix->j_fheads.p, oc,
                                             oo);
    count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
}

// One step of the self join on counters oc / oo: zero fill (when `zero`), then the
// set-major launch.  The join launches programmatically after k_zero_pair when the
// fill stays in L2: hiding the join's launch and first loads under a fill of a few
// microseconds shortens the 2,000-genome step by 4 us (of 32); after fills of hundreds
// of microseconds (20,000 genomes: 3.2 GB) it measured 22 us slower, so there the
// launches stay serialized.
cudaError_t join_step(kssdgpu_index *ix, bool zero, unsigned long long *oc, unsigned long long *oo, cudaStream_t st)
{
    const size_t cells = (size_t)ix->nref * (ix->nref - 1) / 2;
    if (ix->j_compact && ix->j_ntouched) {
        // compact counters: the fill (on j_fill_st, after the caller's earlier work)
        // runs beside the join; the scatter waits for both
        const uint32_t T = ix->j_ntouched;
        cudaError_t e = cudaSuccess;
        if (zero) {
            if (!ix->j_fill_st) e = cudaStreamCreateWithFlags(&ix->j_fill_st, cudaStreamNonBlocking);
            for (int i = 0; i < 2 && e == cudaSuccess; ++i)
                if (!ix->j_fill_ev[i]) e = cudaEventCreateWithFlags(&ix->j_fill_ev[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventRecord(ix->j_fill_ev[0], st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(ix->j_fill_st, ix->j_fill_ev[0], 0);
            const size_t words = std::max<size_t>(cells, 1);
            if (e == cudaSuccess) {
                if ((((uintptr_t)oc | (uintptr_t)oo) & 15) == 0) {
                    k_zero_pair<<<ix->sms * 8, 256, 0, ix->j_fill_st>>>(oc, oo, words);
                    count_launch();
                    e = cudaGetLastError();
                } else {
                    e = cudaMemsetAsync(oc, 0, words * 8, ix->j_fill_st);
                    if (e == cudaSuccess) e = cudaMemsetAsync(oo, 0, words * 8, ix->j_fill_st);
                }
            }
            if (e == cudaSuccess) e = cudaEventRecord(ix->j_fill_ev[1], ix->j_fill_st);
        }
        unsigned long long *acc = ix->j_cacc.p;
        if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, (size_t)T * kCompactStride * 8, st);
        if (e == cudaSuccess) e = launch_sets(ix, acc, acc + 1, st, false, true);
        if (e == cudaSuccess && zero) e = cudaStreamWaitEvent(st, ix->j_fill_ev[1], 0);
        if (e == cudaSuccess) {
            k_scatter_touched<<<grid_for(T), 256, 0, st>>>(ix->j_touched.p, T, acc, oc, oo);
            count_launch();
            e = cudaGetLastError();
        }
        return e;
    }
    bool after_fill = false;
    if (zero) {
        const size_t words = std::max<size_t>(cells, 1);
        cudaError_t e;
        if ((((uintptr_t)oc | (uintptr_t)oo) & 15) == 0) {
            // both counter arrays in one launch, 16-byte stores
            k_zero_pair<<<ix->sms * 8, 256, 0, st>>>(oc, oo, words);
            count_launch();
            e = cudaGetLastError();
            after_fill = cells * 16 <= (size_t)ix->l2_bytes;
        } else {
            e = cudaMemsetAsync(oc, 0, words * 8, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(oo, 0, words * 8, st);
        }
        if (e != cudaSuccess)
            return e;
    }
    return launch_sets(ix, oc, oo, st, after_fill);
}

// Compact slots of a plan of items: the item lanes' cells, sorted; one slot per
// distinct cell (T of them); every lane's slot and every slot's cell.
cudaError_t build_compact(kssdgpu_index *ix, uint32_t nitems, uint32_t *ntouched, cudaStream_t st)
{
    unsigned long long *k1 = nullptr, *k2 = nullptr;
    uint32_t *v1 = nullptr, *v2 = nullptr, *hd = nullptr, *inc = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {
        cudaFree(k1); cudaFree(k2); cudaFree(v1); cudaFree(v2); cudaFree(hd); cudaFree(inc); cudaFree(tmp);
    };
    size_t tb1 = 0, tb2 = 0;
    cudaError_t e = cudaMalloc(&k1, (size_t)nitems * 8);
    if (e == cudaSuccess) e = cudaMalloc(&k2, (size_t)nitems * 8);
    if (e == cudaSuccess) e = cudaMalloc(&v1, (size_t)nitems * 4);
    if (e == cudaSuccess) e = cudaMalloc(&v2, (size_t)nitems * 4);
    if (e == cudaSuccess) e = cudaMalloc(&hd, (size_t)nitems * 4);
    if (e == cudaSuccess) e = cudaMalloc(&inc, (size_t)nitems * 4);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb1, k1, k2, v1, v2, nitems, 0, 64, st);
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tb2, hd, inc, nitems, st);
    const size_t tb = std::max<size_t>(std::max(tb1, tb2), 1);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
    if (e == cudaSuccess) {
        k_item_cells<<<grid_for(nitems), 256, 0, st>>>(ix->j_items.p, nitems, ix->j_tile.p, k1, v1);
        count_launch();
        size_t b = tb;
        e = cub::DeviceRadixSort::SortPairs(tmp, b, k1, k2, v1, v2, nitems, 0, 64, st);
        count_launch(8);
    }
    if (e == cudaSuccess) {
        k_touched_heads<<<grid_for(nitems), 256, 0, st>>>(k2, nitems, hd);
        count_launch();
        size_t b = tb;
        e = cub::DeviceScan::InclusiveSum(tmp, b, hd, inc, nitems, st);
        count_launch(2);
    }
    uint32_t T = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&T, inc + nitems - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = ix->j_islot.ensure(nitems);
    if (e == cudaSuccess) e = ix->j_touched.ensure(T);
    if (e == cudaSuccess && (uint64_t)T * kCompactStride >= (1ull << 32))
        e = cudaErrorMemoryAllocation;  // slot word offsets are 32-bit
    if (e == cudaSuccess) e = ix->j_cacc.ensure((size_t)T * kCompactStride);
    if (e == cudaSuccess) {
        k_touched_slots<<<grid_for(nitems), 256, 0, st>>>(k2, v2, hd, inc, nitems, ix->j_islot.p, ix->j_touched.p);
        count_launch();
        e = cudaStreamSynchronize(st);
    }
    cleanup();
    *ntouched = e == cudaSuccess ? T : 0;
    return e;
}

cudaError_t set_major_plan(kssdgpu_index *ix, uint32_t n, cudaStream_t st)
{
    ix->j_chunk_size = env_u32("KSSDGPU_JOIN_CHUNK", ix->j_chunk_size, 1, 255);
    ix->j_sort_chunks = env_u32("KSSDGPU_JOIN_SORT", ix->j_sort_chunks ? 1 : 0, 0, 1) != 0;
    ix->j_flat_max = env_u32("KSSDGPU_JOIN_FLAT", ix->j_flat_max, 1, kFlatMax);
    const uint32_t flat_max = ix->j_flat_max;
    const uint32_t csize = ix->j_chunk_size;
    uint32_t *heads = nullptr, *runs = nullptr, *first = nullptr, *cheads = nullptr, *cpos = nullptr;
    uint32_t *skey = nullptr, *skey2 = nullptr, *sval = nullptr, *sval2 = nullptr, *npairs = nullptr, *ioff = nullptr;
    uint32_t *f2d = nullptr;
    unsigned long long *twords = nullptr, *tword0 = nullptr;
    ulonglong2 *chunks0 = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {
        cudaFree(heads); cudaFree(runs); cudaFree(first); cudaFree(cheads); cudaFree(cpos);
        cudaFree(skey); cudaFree(skey2); cudaFree(sval); cudaFree(sval2); cudaFree(npairs); cudaFree(ioff);
        cudaFree(f2d); cudaFree(twords); cudaFree(tword0); cudaFree(chunks0); cudaFree(tmp);
    };
    size_t tb1 = 0, tb2 = 0, tb3 = 0, tb4 = 0;
    cudaError_t e = cudaMalloc(&heads, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&f2d, (kFlatMax + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&runs, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&first, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&cheads, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&cpos, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&skey, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&skey2, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sval, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sval2, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&npairs, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&ioff, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&chunks0, (size_t)n * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMalloc(&twords, (size_t)n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&tword0, (size_t)n * 8);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb4, twords, tword0, n, st);
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tb1, heads, runs, n, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, cheads, cpos, n, st);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb3, skey, skey2, sval, sval2, n, 0, 16, st);
    const size_t tb = std::max<size_t>(std::max(std::max(tb1, tb2), std::max(tb3, tb4)), 1);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
    if (e == cudaSuccess) {
        k_set_heads<<<grid_for(n), 256, 0, st>>>(ix->j_small.p, n, ix->j_post.p, heads);
        count_launch();
        size_t b = tb;
        e = cub::DeviceScan::InclusiveSum(tmp, b, heads, runs, n, st);
        count_launch(2);
    }
    if (e == cudaSuccess) {
        k_set_run_first<<<grid_for(n), 256, 0, st>>>(heads, runs, n, first);
        k_set_chunk_heads<<<grid_for(n), 256, 0, st>>>(runs, first, n, csize, cheads);
        count_launch(2);
        size_t b = tb;
        e = cub::DeviceScan::ExclusiveSum(tmp, b, cheads, cpos, n, st);
        count_launch(2);
    }
    // flat classes 2..flat_max: where each starts, its first posting, its run heads
    uint32_t fk[kFlatMax + 1];
    unsigned long long dk[kFlatMax + 1] = {};
    FlatClasses fc{};
    if (e == cudaSuccess && flat_max >= 2) {
        e = cudaMemsetAsync(f2d, 0xFF, sizeof fk, st);
        if (e == cudaSuccess) {
            k_flat_firsts<<<grid_for(n), 256, 0, st>>>(ix->j_small.p, n, flat_max, f2d);
            count_launch();
            e = cudaMemcpyAsync(fk, f2d, sizeof fk, cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        uint32_t words = 0;
        for (uint32_t k = 2; e == cudaSuccess && k <= flat_max; ++k) {
            if (fk[k] >= n)
                continue;
            uint32_t end = n;  // the class ends where the next smaller present class starts
            for (uint32_t k2 = 2; k2 < k; ++k2)
                if (fk[k2] < n)
                    end = std::min(end, fk[k2]);
            fc.n[k] = end - fk[k];
            fc.hoff[k] = words;
            words += (fc.n[k] + 31) / 32;
            e = cudaMemcpyAsync(dk + k, ix->j_small.p + fk[k], 8, cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess && words) e = ix->j_fheads.ensure(words);
        for (uint32_t k = 2; e == cudaSuccess && k <= flat_max; ++k) {
            if (!fc.n[k])
                continue;
            k_flat_heads<<<(fc.n[k] + 255) / 256, 256, 0, st>>>(heads, fk[k], fc.n[k], ix->j_fheads.p + fc.hoff[k]);
            count_launch();
        }
    }
    uint32_t last_pos = 0, last_head = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_pos, cpos + n - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_head, cheads + n - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const uint32_t nchunks = last_pos + last_head;
    if (e == cudaSuccess) e = ix->j_chunks.ensure(nchunks);
    if (e == cudaSuccess) {
        k_set_chunks<<<grid_for(n), 256, 0, st>>>(cheads, cpos, n, csize, ix->j_sort_chunks ? 1 : 0, ix->j_small.p,
                                                  chunks0, skey, sval);
        count_launch();
        size_t b = tb;
        e = cub::DeviceRadixSort::SortPairs(tmp, b, skey, skey2, sval, sval2, nchunks, 0, 16, st);
        count_launch(4);
    }
    // Tiles of the item chunks (sizes above flat_max): runs of equal (m, k) in the
    // sorted order are cut into tiles of tile_chunks(k) chunks.  The scratch arrays of
    // the chunk build are free again: heads = class heads, runs = class numbers,
    // first = class starts, cheads = slots, npairs = tile lanes, ioff = first lanes.
    uint32_t *slot = cheads, *tlanes = npairs, *tlane0 = ioff;
    if (e == cudaSuccess) {
        k_set_permute<<<grid_for(nchunks), 256, 0, st>>>(sval2, nchunks, chunks0, ix->j_chunks.p);
        k_tile_class_heads<<<grid_for(nchunks), 256, 0, st>>>(ix->j_chunks.p, nchunks, flat_max, heads);
        count_launch(2);
        size_t b = tb;
        e = cub::DeviceScan::InclusiveSum(tmp, b, heads, runs, nchunks, st);
        count_launch(2);
    }
    if (e == cudaSuccess) {
        k_set_run_first<<<grid_for(nchunks), 256, 0, st>>>(heads, runs, nchunks, first);
        k_tile_slots<<<grid_for(nchunks), 256, 0, st>>>(ix->j_chunks.p, nchunks, flat_max, runs, first, slot, twords,
                                                        tlanes);
        count_launch(2);
        size_t b = tb;
        e = cub::DeviceScan::ExclusiveSum(tmp, b, twords, tword0, nchunks, st);
        count_launch(2);
    }
    if (e == cudaSuccess) {
        size_t b = tb;
        e = cub::DeviceScan::ExclusiveSum(tmp, b, tlanes, tlane0, nchunks, st);
        count_launch(2);
    }
    unsigned long long last_w0 = 0, last_w = 0;
    uint32_t last_l0 = 0, last_l = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_w0, tword0 + nchunks - 1, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_w, twords + nchunks - 1, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_l0, tlane0 + nchunks - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_l, tlanes + nchunks - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const uint64_t nitems = (uint64_t)last_l0 + last_l, tile_words = last_w0 + last_w;
    if (e == cudaSuccess && (nitems >= (1ull << 32) || tile_words >= kSetItemMaxOffset))
        e = cudaErrorMemoryAllocation;  // beyond the 32-bit launch index or the item word's offset field
    if (e == cudaSuccess) e = ix->j_items.ensure(nitems);
    if (e == cudaSuccess) e = ix->j_tile.ensure(tile_words);
    if (e == cudaSuccess && nitems) e = cudaMemsetAsync(ix->j_items.p, 0, nitems * 8, st);  // empty lanes
    if (e == cudaSuccess) {
        k_tile_scatter<<<grid_for(nchunks), 256, 0, st>>>(ix->j_chunks.p, nchunks, flat_max, slot, tword0,
                                                          ix->j_post.p, ix->j_tile.p);
        k_set_items<<<grid_for(nchunks), 256, 0, st>>>(ix->j_chunks.p, nchunks, flat_max, slot, tword0, tlane0,
                                                       ix->j_items.p);
        count_launch(2);
        e = cudaStreamSynchronize(st);
    }
    // Compact counters for plans of items only (the flat path adds into dense cells),
    // while the touched cells are at most half of the lower triangle, and only where
    // the dense counters outgrow L2: there the fill takes hundreds of microseconds and
    // running it beside the join pays (20,000 genomes: step 0.65 vs 0.73 ms); a fill
    // that fits in L2 overlaps the join through the dependent launch instead, and the
    // compact path's extra memset and scatter launches cost more than they save there
    // (2,000 genomes: 34.8 vs 25.6 us).  KSSDGPU_JOIN_COMPACT=2 forces it (tests).
    const uint32_t compact_env = env_u32("KSSDGPU_JOIN_COMPACT", 1, 0, 2);
    ix->j_compact_ok = compact_env != 0;
    const bool big_fill = (uint64_t)ix->nref * (ix->nref - 1) / 2 * 16 > (uint64_t)ix->l2_bytes || compact_env == 2;
    bool compact = false;
    uint32_t ntouched = 0;
    if (e == cudaSuccess && ix->j_compact_ok && big_fill && flat_max < 2 && nitems) {
        e = build_compact(ix, (uint32_t)nitems, &ntouched, st);
        compact = e == cudaSuccess && ntouched && 2 * (uint64_t)ntouched <= (uint64_t)ix->nref * (ix->nref - 1) / 2;
    }
    cleanup();
    if (e == cudaSuccess) {
        ix->j_compact = compact;
        ix->j_ntouched = compact ? ntouched : 0;
        ix->j_nchunks = nchunks;
        ix->j_nitems = (uint32_t)nitems;
        for (uint32_t k = 2; k <= kFlatMax; ++k)
            fc.off[k] = (uint32_t)dk[k];
        ix->j_flat = fc;
    }
    return e;
}

// Autotuner of the set-major join: candidate plans (largest flat group size, then
// groups per chunk and chunk order at the best flat size) are built and each timed
// as a whole step on scratch counters, zero fill and join (CUDA events, best of three
// after one warm-up run, each run after a write of twice the L2 size so that the
// postings come from HBM as in a one-shot call; the fill is timed because the join
// overlaps it); the fastest stays.  Runs once per index, on request
// (kssdgpu_self_plan_tune) or at plan time with KSSDGPU_TUNE=1; keeps the defaults
// when a knob is pinned by its environment variable or when the scratch would take
// more than a quarter of the free device memory.
cudaError_t tune_join(kssdgpu_index *ix, uint32_t n, cudaStream_t st)
{
    ix->j_tuned = true;
    const bool pinned = std::getenv("KSSDGPU_JOIN_CHUNK") || std::getenv("KSSDGPU_JOIN_SORT") ||
                        std::getenv("KSSDGPU_JOIN_FLAT");
    if (pinned || n == 0)
        return n ? set_major_plan(ix, n, st) : cudaSuccess;
    const size_t cells = std::max<size_t>((size_t)ix->nref * (ix->nref - 1) / 2, 1);
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ix->device);
    const size_t flush_b = std::max<size_t>(2 * (size_t)std::max(l2, 0), 64u << 20);
    size_t free_b = 0, total_b = 0;
    cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess || cells * 16 + flush_b > free_b / 4)
        return set_major_plan(ix, n, st);
    unsigned long long *oc = nullptr, *oo = nullptr;
    void *flush = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    e = cudaMalloc(&oc, cells * 8);
    if (e == cudaSuccess) e = cudaMalloc(&oo, cells * 8);
    if (e == cudaSuccess) e = cudaMalloc(&flush, flush_b);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    float best = 1e30f;
    uint32_t best_size = ix->j_chunk_size, best_flat = ix->j_flat_max;
    bool best_sort = ix->j_sort_chunks;
    int tried = 0;
    auto time_plan = [&](uint32_t cs, bool srt, uint32_t flat) {
        ix->j_chunk_size = cs;
        ix->j_sort_chunks = srt;
        ix->j_flat_max = flat;
        e = set_major_plan(ix, n, st);
        float t_min = 1e30f;
        for (int r = 0; r < 4 && e == cudaSuccess; ++r) {
            e = cudaMemsetAsync(flush, r, flush_b, st);
            if (e == cudaSuccess) e = cudaEventRecord(ev0, st);
            if (e == cudaSuccess) e = join_step(ix, true, oc, oo, st);
            if (e == cudaSuccess) e = cudaEventRecord(ev1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev1);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev0, ev1);
            if (e == cudaSuccess && r > 0)
                t_min = std::min(t_min, ms);
        }
        if (e != cudaSuccess)
            return;
        ++tried;
        if (t_min < best) {
            best = t_min;
            best_size = cs;
            best_sort = srt;
            best_flat = flat;
        }
    };
    // the flat size at 32 groups per chunk, largest chunks first; then the chunk
    // size (largest first) and the size-only order at the best flat size
    for (uint32_t flat = kFlatMax; flat >= 1 && e == cudaSuccess; --flat)
        time_plan(32, true, flat);
    static const struct { uint32_t size; bool sorted; } kChunkCands[] = {
        {8, true}, {16, true}, {64, true}, {128, true}, {32, false}};
    const uint32_t flat_at = best_flat;
    for (const auto &cand : kChunkCands)
        if (e == cudaSuccess)
            time_plan(cand.size, cand.sorted, flat_at);
    cudaFree(oc);
    cudaFree(oo);
    cudaFree(flush);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (e != cudaSuccess)
        return e;
    ix->j_chunk_size = best_size;
    ix->j_sort_chunks = best_sort;
    ix->j_flat_max = best_flat;
    ix->j_tune_tried = tried;
    ix->j_tune_ms = best;
    return set_major_plan(ix, n, st);
}

int self_plan(kssdgpu_index *ix, cudaStream_t st)
{
    if (ix->j_ready)
        return KSSDGPU_OK;
    const uint64_t u = ix->u;
    const uint64_t cap = std::max<uint64_t>(ix->n / 2 + 1, 1);  // a listed group holds >= 2 postings
    CUDA_TRY(ix->j_big.ensure(cap));
    CUDA_TRY(ix->j_conf.ensure(cap));
    unsigned long long *skey = nullptr, *skey2 = nullptr;
    uint32_t *sval = nullptr, *sval2 = nullptr, *ks = nullptr, *offs = nullptr;
    unsigned int *cnt = nullptr;
    unsigned long long *tot = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {
        cudaFree(skey); cudaFree(skey2); cudaFree(sval); cudaFree(sval2);
        cudaFree(ks); cudaFree(offs); cudaFree(cnt); cudaFree(tot); cudaFree(tmp);
    };
    cudaError_t e = cudaMalloc(&skey, cap * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sval, cap * 4);
    if (e == cudaSuccess) e = cudaMalloc(&cnt, 3 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&tot, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(tot, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) {
        cleanup();
        return fail(KSSDGPU_ERR_NOMEM, std::string("self-join plan: ") + cudaGetErrorString(e));
    }
    if (u) {
        k_self_classify<<<(unsigned)((u + 255) / 256), 256, 0, st>>>(ix->gbeg, u, ix->post, skey, sval, ix->j_big.p,
                                                                     ix->j_conf.p, cnt, tot);
        count_launch();
    }
    unsigned int hc[3];
    unsigned long long ht[2];
    e = cudaMemcpyAsync(hc, cnt, sizeof hc, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ht, tot, sizeof ht, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const uint32_t n = e == cudaSuccess ? hc[0] : 0;
    // small groups: sort by (size desc, leading gids), then lay their postings out contiguously
    if (e == cudaSuccess && n) {
        e = cudaMalloc(&skey2, (size_t)n * 8);
        if (e == cudaSuccess) e = cudaMalloc(&sval2, (size_t)n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&ks, (size_t)n * 4);
        if (e == cudaSuccess) e = cudaMalloc(&offs, (size_t)n * 4);
        size_t tb = 0, tb2 = 0;
        if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, tb, skey, skey2, sval, sval2, n, 0, 64, st);
        if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, ks, offs, n, st);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(std::max(tb, tb2), 1));
        if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tb, skey, skey2, sval, sval2, n, 0, 64, st);
        count_launch(8);
        if (e == cudaSuccess) {
            k_self_sizes<<<grid_for(n), 256, 0, st>>>(sval2, n, ix->gbeg, ks);
            count_launch();
            e = cub::DeviceScan::ExclusiveSum(tmp, tb2, ks, offs, n, st);
            count_launch(2);
        }
        uint32_t last_off = 0, last_k = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&last_off, offs + n - 1, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&last_k, ks + n - 1, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = ix->j_small.ensure(n);
        if (e == cudaSuccess) e = ix->j_post.ensure((size_t)last_off + last_k);
        if (e == cudaSuccess) {
            k_self_gather<<<grid_for(n), 256, 0, st>>>(sval2, ks, offs, n, ix->gbeg, ix->post, ix->j_small.p,
                                                       ix->j_post.p);
            count_launch();
            e = cudaStreamSynchronize(st);
        }
        if (e == cudaSuccess)
            e = env_u32("KSSDGPU_TUNE", 0, 0, 1) ? tune_join(ix, n, st) : set_major_plan(ix, n, st);
    }
    cleanup();
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? KSSDGPU_ERR_NOMEM : KSSDGPU_ERR_CUDA,
                    std::string("self-join plan: ") + cudaGetErrorString(e));
    ix->j_n[0] = hc[0];
    ix->j_n[1] = hc[1];
    ix->j_n[2] = hc[2];
    ix->j_postings = ht[0];
    ix->j_pairs = ht[1];
    ix->j_ready = true;
    return KSSDGPU_OK;
}

// The one-pass self step: zero fill of the dense lower triangle (unless NO_ZERO), then
// the scan join over the whole index.  When the fill stays in L2 the scan launches
// programmatically after it and waits for it only before its first atomic, so its
// first tiles' gbeg loads overlap the fill.
int self_scan_impl(kssdgpu_index *ix, unsigned flags, unsigned long long *oc, unsigned long long *oo, cudaStream_t st)
{
    const size_t cells = (size_t)ix->nref * (ix->nref - 1) / 2;
    if (!cells)
        return KSSDGPU_OK;
    // a conflict-free index deals out pairs; with conflicts threads walk whole groups
    const bool pairs = !ix->f_conflict;
    // Triangles larger than L2 (and of 32-bit cell numbers: at most 92,681 genomes) add
    // through the table of touched cells (allocated on first use, kept empty between
    // calls); with the counters in L2 the table's probes cost more than they save (2,000
    // genomes: 0.19 vs 0.14 ms per step) and the join adds into the triangle directly.
    const bool big = cells < (size_t)kCellEmpty && cells * 16 > (size_t)ix->l2_bytes;
    CellTable table{nullptr, nullptr, 0};
    if (ix->u && pairs && big) {
        int rc = cell_table(ix, st, table);
        if (rc)
            return rc;
    }
    bool after_fill = false;
    if (!(flags & KSSDGPU_NO_ZERO)) {
        if ((((uintptr_t)oc | (uintptr_t)oo) & 15) == 0) {
            k_zero_pair<<<ix->sms * 8, 256, 0, st>>>(oc, oo, cells);
            count_launch();
            after_fill = cells * 16 <= (size_t)ix->l2_bytes;
            CUDA_TRY(cudaGetLastError());
        } else {
            CUDA_TRY(cudaMemsetAsync(oc, 0, cells * 8, st));
            CUDA_TRY(cudaMemsetAsync(oo, 0, cells * 8, st));
        }
    }
    if (!ix->u)
        return KSSDGPU_OK;
    auto kern = pairs ? k_self_scan<true> : k_self_scan<false>;
    const size_t smem = sizeof(ScanSmem);
    if (!ix->scan_grid) {
        CUDA_TRY(cudaFuncSetAttribute(k_self_scan<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CUDA_TRY(cudaFuncSetAttribute(k_self_scan<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_self_scan<true>, kScanThreads, smem));
        ix->scan_grid = std::max(1, per_sm) * ix->sms;
    }
    const uint64_t ntiles = (ix->u + kScanTile - 1) / kScanTile;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::min<uint64_t>(ntiles, (uint64_t)ix->scan_grid));
    cfg.blockDim = dim3(kScanThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    if (after_fill && KSSD_JOIN_PDL) {
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, (const uint32_t *)ix->gbeg, ix->u, (const uint64_t *)ix->post,
                                (flags & KSSDGPU_IGNORECONFLICT) ? 1 : 0, table, oc, oo));
    count_launch();
    CUDA_TRY(cudaGetLastError());
    if (table.key) {
        k_cell_table_flush<<<ix->sms * 4, 256, 0, st>>>(table.key, table.acc, 1u << table.log, oc, oo);
        count_launch();
        CUDA_TRY(cudaGetLastError());
    }
    return KSSDGPU_OK;
}

// Device bytes of a dense self join with K allele rows (A', F, D).
uint64_t dense_npad(const kssdgpu_index *ix) { return ((uint64_t)ix->nref + 15) / 16 * 16; }
uint64_t dense_bytes(const kssdgpu_index *ix, uint64_t kpad)
{
    const uint64_t np = dense_npad(ix);
    return 5ull * np * kpad + 16ull * np * np;
}

uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Dense self join (see k_dense_list): list the shared groups, count their alleles
// (distinct objects, from a hash of each group's objects in shared memory), build
// every allele's operand rows, the tensor-core GEMM (per block of genomes below the
// diagonal from kDenseBlocks blocks on), and the packed lower triangle
// (every cell written, so no zero fill).  Conflict-free indexes of at most
// kDenseMaxGroup references only; the operands must fit in half of the free memory.
int self_dense_impl(kssdgpu_index *ix, unsigned long long *oc, unsigned long long *oo, cudaStream_t st)
{
    const int n = ix->nref;
    const size_t cells = (size_t)n * (n - 1) / 2;
    if (ix->f_conflict)
        return fail(KSSDGPU_ERR_ARG, "the dense self join needs a conflict-free index (a gid holds several objects "
                                     "of one context)");
    if ((uint32_t)n > kDenseMaxGroup)
        return fail(KSSDGPU_ERR_CAPACITY, "the dense self join takes at most " + std::to_string(kDenseMaxGroup) +
                                              " references");
    if (!cells)
        return KSSDGPU_OK;
    if (ix->f_groups >= (1ull << 31))
        return fail(KSSDGPU_ERR_CAPACITY, "dense self join: too many shared contexts");
    const uint32_t S = (uint32_t)ix->f_groups;
    if (!S) {
        CUDA_TRY(cudaMemsetAsync(oc, 0, cells * 8, st));
        CUDA_TRY(cudaMemsetAsync(oo, 0, cells * 8, st));
        return KSSDGPU_OK;
    }
    const uint32_t npad = (uint32_t)dense_npad(ix);
    const size_t group_smem = dense_group_smem((uint32_t)n);
    const size_t rows_smem = dense_rows_smem(npad);
    CUDA_TRY(cudaFuncSetAttribute(k_dense_alleles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)group_smem));
    CUDA_TRY(cudaFuncSetAttribute(k_dense_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem));
    CUDA_TRY(ix->d_list.ensure(S));
    CUDA_TRY(ix->d_poff.ensure((size_t)S + 1));   // alleles per group, then the fill counter
    CUDA_TRY(ix->d_allele.ensure((size_t)S + 1)); // first allele row of every group
    CUDA_TRY(ix->d_aval.ensure(std::max<uint64_t>(ix->n, 1)));
    unsigned int *d_count = reinterpret_cast<unsigned int *>(ix->d_poff.p + S);
    size_t tb = 0;
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, ix->d_poff.p, ix->d_allele.p, (int)S + 1, st));
    CUDA_TRY(ix->d_tmp.ensure(tb));
    // 1. the shared groups, their allele counts and first allele rows
    CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned int), st));
    k_dense_list<<<grid_for(ix->u), 256, 0, st>>>(ix->gbeg, ix->u, ix->d_list.p, d_count);
    // persistent CTAs over the groups: as many as fit on an SM at once (the group's
    // barriers and dependent loads leave one CTA mostly waiting)
    int per_sm_al = 0, per_sm_rows = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_al, k_dense_alleles, kDenseThreads, group_smem));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_rows, k_dense_rows, kDenseThreads, rows_smem));
    const int grid_al = ix->sms * std::max(1, per_sm_al), grid = ix->sms * std::max(1, per_sm_rows);
    k_dense_alleles<<<grid_al, kDenseThreads, group_smem, st>>>(ix->d_list.p, S, ix->post, (uint32_t)n, ix->d_poff.p,
                                                                ix->d_aval.p);
    CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned int), st));  // poff[S] = 0: the scan's last term
    tb = ix->d_tmp.cap;
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(ix->d_tmp.p, tb, ix->d_poff.p, ix->d_allele.p, (int)S + 1, st));
    count_launch(4);
    uint32_t alleles = 0;
    CUDA_TRY(cudaMemcpyAsync(&alleles, ix->d_allele.p + S, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    ix->d_alleles = alleles;
    const uint64_t kpad = round_up(std::max<uint32_t>(alleles, 1), 128);
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if (dense_bytes(ix, kpad) > free_b / 2)
        return fail(KSSDGPU_ERR_NOMEM, "dense self join: operands of " + std::to_string(dense_bytes(ix, kpad)) +
                                           " bytes exceed half of the free device memory");
    if (kpad > 0x7FFFFFFFull)
        return fail(KSSDGPU_ERR_CAPACITY, "dense self join: allele count beyond the GEMM's 32-bit extent");
    // 2. operands, allele-major; the padding rows past the last allele are zero
    CUDA_TRY(ix->d_a.ensure((size_t)npad * kpad));
    CUDA_TRY(ix->d_f.ensure((size_t)4 * npad * kpad));
    CUDA_TRY(ix->d_d.ensure((size_t)4 * npad * npad));
    if (kpad > alleles) {
        CUDA_TRY(cudaMemsetAsync(ix->d_a.p + (size_t)alleles * npad, 0, (size_t)(kpad - alleles) * npad, st));
        CUDA_TRY(cudaMemsetAsync(ix->d_f.p + (size_t)alleles * 4 * npad, 0, (size_t)(kpad - alleles) * 4 * npad, st));
    }
    k_dense_rows<<<grid, kDenseThreads, rows_smem, st>>>(ix->d_list.p, S, ix->d_allele.p, ix->d_aval.p, ix->post,
                                                         npad, ix->d_a.p, ix->d_f.p);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    // 3. D = A' F^T on the tensor cores (both operands MN-major).  The four counters are
    // symmetric in (q, r) and only cells q > r are kept, so for every block of 128
    // genomes r (512 columns of F) one GEMM covers the rows q >= the block's first:
    // (B + 1) / 2B of the square's work for B blocks, F read once.  Below kDenseBlocks
    // blocks one GEMM over the square is faster (one launch, fewer split-K partials:
    // 512 genomes 0.78 vs 0.86 ms per join; 1,024 genomes 2.53 vs 2.34 ms, 2,048 genomes
    // 11.3 vs 7.8 ms the other way).
    const uint64_t nblk = (npad + 127) / 128;
    const uint64_t bw = nblk >= kDenseBlocks ? 128 : npad;  // genomes r per GEMM
    const uint64_t ngemm = (npad + bw - 1) / bw;
    size_t ws = 0;
    for (uint64_t j = 0; j < ngemm; ++j)
        ws = std::max(ws, kssd::dense_gemm_s8_workspace((int)(npad - bw * j),
                                                        (int)(4 * std::min<uint64_t>(bw, npad - bw * j)), (int)kpad));
    CUDA_TRY(ix->d_ws.ensure(ws));
    for (uint64_t j = 0; j < ngemm; ++j) {
        const uint64_t m = npad - bw * j, nc = 4 * std::min<uint64_t>(bw, npad - bw * j);
        const int grc = kssd::dense_gemm_s8(ix->d_a.p + bw * j, ix->d_f.p + 4 * bw * j,
                                            ix->d_d.p + bw * j * 4 * npad + 4 * bw * j, (int)m, (int)nc, (int)kpad,
                                            (int64_t)npad, (int64_t)(4 * npad), (int64_t)(4 * npad), ix->d_ws.p, st);
        count_launch();
        if (grc)
            return fail(KSSDGPU_ERR_CUDA, grc == 1 ? "dense self join: GEMM shape not supported"
                                                   : "dense self join: GEMM launch failed");
        CUDA_TRY(cudaGetLastError());
    }
    // 4. the packed lower triangle
    k_dense_epilogue<<<grid_for(cells), 256, 0, st>>>(ix->d_d.p, npad, cells, oc, oo);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

// The density rule of the self join: the dense path does at most 4 n^2 K multiply-adds (K
// alleles of the shared contexts), the scan one counter update per pair of postings of
// a shared context.  density = pairs / (n^2 K); the dense join is taken when it is
// above kDenseRatio, on a conflict-free index whose operands fit in half of the free
// device memory.
constexpr double kDenseRatio = 1.0 / 2048.0;

double self_density(const kssdgpu_index *ix)
{
    const double n = (double)ix->nref, k = (double)std::max<unsigned long long>(ix->f_alleles, 1);
    return (double)ix->f_pairs / (n * n * k);
}

bool dense_chosen(const kssdgpu_index *ix)
{
    if (ix->f_conflict || ix->f_pairs == 0 || ix->nref < 2 || (uint32_t)ix->nref > kDenseMaxGroup ||
        self_density(ix) < kDenseRatio)
        return false;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    // the estimate's margin: operands for twice the sampled allele count
    return dense_bytes(ix, round_up(2 * ix->f_alleles, 128)) <= free_b / 2;
}

int self_lower_dev_impl(kssdgpu_index *ix, unsigned flags, unsigned long long *oc, unsigned long long *oo, cudaStream_t st)
{
    if (flags & KSSDGPU_SELF_DENSE)
        return self_dense_impl(ix, oc, oo, st);
    if (!(flags & (KSSDGPU_SELF_PLAN | KSSDGPU_SELF_SCAN)) && !(flags & KSSDGPU_NO_ZERO) && dense_chosen(ix))
        return self_dense_impl(ix, oc, oo, st);
    if (!(flags & KSSDGPU_SELF_PLAN))
        return self_scan_impl(ix, flags, oc, oo, st);
    int rc = self_plan(ix, st);
    if (rc)
        return rc;
    CUDA_TRY(join_step(ix, !(flags & KSSDGPU_NO_ZERO), oc, oo, st));
    if (ix->j_n[1]) {
        k_self_big<<<(unsigned)(((uint64_t)ix->j_n[1] * 32 + 255) / 256), 256, 0, st>>>(ix->j_big.p, ix->j_n[1], ix->post,
                                                                                       oc, oo);
        count_launch();
    }
    if (ix->j_n[2]) {
        k_self_conflict_groups<<<grid_for(ix->j_n[2]), 256, 0, st>>>(ix->j_conf.p, ix->j_n[2], ix->post,
                                                                     (flags & KSSDGPU_IGNORECONFLICT) ? 1 : 0, oc, oo);
        count_launch();
    }
    CUDA_TRY(cudaGetLastError());
    return KSSDGPU_OK;
}

}  // namespace

// ------------------------------------------------------------------ no-allocation counting
//
// Scratch of kssdgpu_count_block_noalloc, in the library's own static device
// memory so that a call needs no cudaMalloc.  Layout (32-bit words):
//   [0]       work counter of the persistent kernel
//   [2, 34)   histogram of query size classes          (shared-memory rows)
//   [34, 66)  scatter cursors of the size classes      (shared-memory rows)
//   [128, ..) query order, largest size class first    (shared-memory rows), or
//   [127, ..) key-range chunk prefix, nq + 1 words      (global rows)
// The first 128 words are cleared at the start of every call; the order or the
// prefix is fully rewritten by every call before it is read.  Errors found on the
// device (query keys out of order) go to the index's own error word, which
// kssdgpu_sync reports.
static __device__ __align__(256) unsigned int g_noalloc_scratch[KSSDGPU_NOALLOC_SCRATCH_BYTES / 4];

namespace {

constexpr int kNoallocHeaderWords = 128;
static_assert(KSSDGPU_NOALLOC_SCRATCH_BYTES == 4 * (kNoallocHeaderWords + KSSDGPU_NOALLOC_MAX_QUERIES),
              "scratch layout and its documented size disagree");

// size class of a query, 0 for the largest: leading zeros of its entry count
__device__ __forceinline__ uint32_t size_class(const uint64_t *__restrict__ offs, int q)
{
    const uint64_t size = offs[q + 1] - offs[q];
    const uint32_t s = size > 0x7FFFFFFFull ? 0x7FFFFFFFu : (uint32_t)size;
    return s ? (uint32_t)__clz(s) : 31u;
}

__global__ void k_noalloc_hist(const uint64_t *__restrict__ offs, int nq, unsigned int *__restrict__ scr)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        atomicAdd(scr + 2 + size_class(offs, q), 1u);
}

__global__ void k_noalloc_scan(unsigned int *__restrict__ scr)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned int run = 0;
        for (int c = 0; c < 32; ++c) {
            scr[34 + c] = run;
            run += scr[2 + c];
        }
    }
}

__global__ void k_noalloc_scatter(const uint64_t *__restrict__ offs, int nq, unsigned int *__restrict__ scr)
{
    int *order = reinterpret_cast<int *>(scr + kNoallocHeaderWords);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        order[atomicAdd(scr + 34 + size_class(offs, q), 1u)] = q;
}

// prefix[0] = 0, prefix[q + 1] = prefix[q] + ceil(size(q) / chunk): the key-range
// chunks of the global-row kernel, in one CTA (nq <= KSSDGPU_NOALLOC_MAX_QUERIES).
__global__ void __launch_bounds__(1024) k_noalloc_prefix(const uint64_t *__restrict__ offs, int nq, uint32_t chunk,
                                                         unsigned int *__restrict__ prefix)
{
    __shared__ unsigned int part[1024];
    const int per = (nq + 1023) / 1024;
    const int q0 = min(nq, (int)threadIdx.x * per), q1 = min(nq, q0 + per);
    unsigned int sum = 0;
    for (int q = q0; q < q1; ++q)
        sum += (unsigned int)((offs[q + 1] - offs[q] + chunk - 1) / chunk);
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const unsigned int v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned int run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    if (threadIdx.x == 0)
        prefix[0] = 0;
    for (int q = q0; q < q1; ++q) {
        run += (unsigned int)((offs[q + 1] - offs[q] + chunk - 1) / chunk);
        prefix[q + 1] = run;
    }
}

std::mutex g_noalloc_mu;
unsigned int *g_noalloc_addr[64] = {};

// Device address of the scratch array on the current device (looked up once per device).
int noalloc_scratch(int device, unsigned int **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= 64)
        return fail(KSSDGPU_ERR_ARG, "device ordinal out of range for the no-allocation scratch");
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(KSSDGPU_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-allocation scratch: ") +
                                              cudaGetErrorString(e));
        g_noalloc_addr[device] = static_cast<unsigned int *>(p);
    }
    *out = g_noalloc_addr[device];
    return KSSDGPU_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

// Device copies of the calibration trees, one per device, replaced when a call passes
// another model.
struct HgbDeviceModel {
    const void *host_nodes = nullptr;
    uint32_t nodes = 0, trees = 0;
    kssd::HgbNode *d_nodes = nullptr;
    uint32_t *d_begin = nullptr;
};
static std::mutex g_hgb_mu;
static std::vector<HgbDeviceModel> g_hgb;

static int metric_params(int device, const kssdgpu_metric_opt_t *o, kssd::MetricParams &P)
{
    if (!o)
        return fail(KSSDGPU_ERR_ARG, "null metric options");
    if (o->hgb_trees && (!o->hgb_nodes || !o->hgb_tree_begin || !o->hgb_nodes_count))
        return fail(KSSDGPU_ERR_ARG, "calibration trees without their nodes");
    P = kssd::MetricParams{};
    P.s = o->s;
    P.e = o->e;
    P.v = o->v;
    P.unassembled = o->unassembled;
    P.unified_metric = o->unified_metric;
    P.raw_output = o->raw_output;
    P.afcut = o->afcut;
    P.drfold = o->drfold;
    P.obj_bits = o->obj_bits;
    P.ctx_bits = o->ctx_bits;
    P.zero_const = o->zero_const;
    P.zero_value = o->zero_value;
    P.baseline = o->hgb_baseline;
    P.ntrees = (int)o->hgb_trees;
    if (!o->hgb_trees)
        return KSSDGPU_OK;
    for (uint32_t t = 0; t < o->hgb_trees; ++t)
        if (o->hgb_tree_begin[t] >= o->hgb_tree_begin[t + 1] || o->hgb_tree_begin[t + 1] > o->hgb_nodes_count)
            return fail(KSSDGPU_ERR_ARG, "calibration tree offsets out of range");
    std::lock_guard<std::mutex> lock(g_hgb_mu);
    if ((int)g_hgb.size() <= device)
        g_hgb.resize(device + 1);
    HgbDeviceModel &m = g_hgb[device];
    if (m.host_nodes != o->hgb_nodes || m.nodes != o->hgb_nodes_count || m.trees != o->hgb_trees) {
        if (m.d_nodes)
            cudaFree(m.d_nodes);
        if (m.d_begin)
            cudaFree(m.d_begin);
        m = HgbDeviceModel{};
        CUDA_TRY(cudaMalloc(&m.d_nodes, (size_t)o->hgb_nodes_count * sizeof(kssd::HgbNode)));
        CUDA_TRY(cudaMalloc(&m.d_begin, ((size_t)o->hgb_trees + 1) * sizeof(uint32_t)));
        CUDA_TRY(cudaMemcpy(m.d_nodes, o->hgb_nodes, (size_t)o->hgb_nodes_count * sizeof(kssd::HgbNode),
                            cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(m.d_begin, o->hgb_tree_begin, ((size_t)o->hgb_trees + 1) * sizeof(uint32_t),
                            cudaMemcpyHostToDevice));
        m.host_nodes = o->hgb_nodes;
        m.nodes = o->hgb_nodes_count;
        m.trees = o->hgb_trees;
    }
    P.nodes = m.d_nodes;
    P.tree_begin = m.d_begin;
    P.nnodes = m.nodes;
    return KSSDGPU_OK;
}

extern "C" {

const char *kssdgpu_last_error(void) { return g_last_error.c_str(); }

int kssdgpu_init(int device)
{
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaFree(nullptr));
    if (device >= 0 && device < 64) {
        // a fresh context (e.g. after the caller's cudaDeviceReset) may hold the
        // no-allocation scratch elsewhere: look its address up again on next use
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        g_noalloc_addr[device] = nullptr;
    }
    return KSSDGPU_OK;
}

uint64_t kssdgpu_launch_count(void) { return g_launches.load(); }

int kssdgpu_sketch_masks(const kssdgpu_sketch_params_t *p, uint64_t *ctxmask, uint64_t *tupmask, int *obj_bits)
{
    if (!p || p->klen < 1 || p->klen > 32)
        return fail(KSSDGPU_ERR_ARG, "sketch k-mer length must be 1..32");
    uint64_t cm = 0;
    int ctx_bits;
    if (p->coden_len > 0) {
        // per coden 4 context bits above 2 object bits; the 11th coden adds a last 4-bit
        // context group (src/sketch_rearrange.h:109-122)
        for (int i = 0; i < p->coden_len; ++i) {
            cm = (cm << 6) | 0x3Cull;
            if (i == 10) {
                cm = (cm << 4) | 0xFull;
                break;
            }
        }
        ctx_bits = 4 * p->coden_len;
    } else {
        const int iolen = p->klen - 2 * (p->hclen + p->holen);
        if (p->hclen < 0 || p->holen < 0 || iolen < 0)
            return fail(KSSDGPU_ERR_ARG, "invalid context/object lengths for the k-mer length");
        const uint64_t hc = p->hclen ? (~0ull >> (64 - 2 * p->hclen)) : 0;
        cm = (hc << (2 * (p->holen + p->hclen + iolen))) | (hc << (2 * p->holen));
        ctx_bits = 4 * p->hclen;
    }
    const uint64_t tm = ~0ull >> (64 - 2 * p->klen);
    if ((cm & ~tm) || 2 * p->klen - ctx_bits < 0)
        return fail(KSSDGPU_ERR_ARG, "context pattern wider than the k-mer");
    if (ctxmask) *ctxmask = cm;
    if (tupmask) *tupmask = tm;
    if (obj_bits) *obj_bits = 2 * p->klen - ctx_bits;
    return KSSDGPU_OK;
}

uint32_t kssdgpu_sketch_hash_id(const kssdgpu_sketch_params_t *p)
{
    // the sketch files' method id (src/command_sketch.h:49-52): hashes of the layout
    // parameters and the filter, xor-folded with that of a fixed tag
    if (!p)
        return 0;
    const uint64_t filter = 0xFFFFFFFFu >> (p->drfold < 0 ? 0 : p->drfold > 31 ? 31 : p->drfold);
    uint64_t v[5];
    if (p->coden_len > 0) {
        v[0] = (uint64_t)p->coden_len; v[1] = 0; v[2] = 0;
    } else {
        v[0] = (uint64_t)p->hclen; v[1] = (uint64_t)p->holen; v[2] = (uint64_t)(p->klen - 2 * (p->hclen + p->holen));
    }
    v[3] = (uint64_t)p->drfold;
    v[4] = filter;
    uint32_t h = (uint32_t)splitmix64(31415926ull);
    for (int i = 0; i < 5; ++i)
        h ^= (uint32_t)splitmix64(v[i]);
    return h;
}

int kssdgpu_sketch(const char *seq, uint64_t seq_len, const uint64_t *rec_offs, uint64_t nrec,
                   const uint64_t *samp_recs, int nsamples, const kssdgpu_sketch_params_t *p, uint64_t *keys,
                   uint64_t keys_cap, uint64_t *offs)
{
    if (!p || !offs || nsamples < 0 || (nrec && !rec_offs) || (nsamples && !samp_recs) || (seq_len && !seq))
        return fail(KSSDGPU_ERR_ARG, "invalid sketch arguments");
    uint64_t cm = 0, tm = 0;
    int ob = 0;
    int rc = kssdgpu_sketch_masks(p, &cm, &tm, &ob);
    if (rc)
        return rc;
    if (p->drfold < 0 || p->drfold > 32)
        return fail(KSSDGPU_ERR_ARG, "sketch drfold must be 0..32");
    if (seq_len >= (1ull << 32))
        return fail(KSSDGPU_ERR_CAPACITY, "sketch at most 4 GiB of sequence per call");
    // records tile the sequence; samples tile the records
    if (nrec && (rec_offs[0] != 0 || rec_offs[nrec] != seq_len))
        return fail(KSSDGPU_ERR_ARG, "record offsets must run from 0 to the sequence length");
    if (!nrec && seq_len)
        return fail(KSSDGPU_ERR_ARG, "sequence bytes without records");
    for (uint64_t r = 0; r < nrec; ++r)
        if (rec_offs[r + 1] < rec_offs[r])
            return fail(KSSDGPU_ERR_ARG, "record offsets must not decrease");
    if (nsamples && (samp_recs[0] != 0 || samp_recs[nsamples] != nrec))
        return fail(KSSDGPU_ERR_ARG, "sample record ranges must run from 0 to the record count");
    for (int s = 0; s < nsamples; ++s)
        if (samp_recs[s + 1] < samp_recs[s])
            return fail(KSSDGPU_ERR_ARG, "sample record ranges must not decrease");
    for (int s = 0; s <= nsamples; ++s)
        offs[s] = 0;
    if (!nsamples || !seq_len)
        return KSSDGPU_OK;
    SketchGeom g;
    g.ctxmask = cm;
    g.tupmask = tm;
    g.klen = p->klen;
    g.obj_bits = ob;
    g.filter = p->drfold >= 32 ? 0u : (0xFFFFFFFFu >> p->drfold);
    cudaStream_t st = nullptr;
    const uint64_t nthreads = (seq_len + kSketchSpan - 1) / kSketchSpan;
    const uint64_t nblocks = (seq_len + kSketchTile - 1) / kSketchTile;
    // device buffers (freed on every path)
    struct Bufs {
        unsigned char *seq = nullptr;
        uint64_t *rec = nullptr, *samp = nullptr;
        uint32_t *counts = nullptr, *pos = nullptr, *scounts = nullptr, *seg = nullptr, *kept = nullptr;
        unsigned long long *k0 = nullptr, *k1 = nullptr;
        uint8_t *keep = nullptr;
        void *tmp = nullptr;
        int *nsel = nullptr;
        ~Bufs()
        {
            cudaFree(seq); cudaFree(rec); cudaFree(samp); cudaFree(counts); cudaFree(pos); cudaFree(scounts);
            cudaFree(seg); cudaFree(kept); cudaFree(k0); cudaFree(k1); cudaFree(keep); cudaFree(tmp); cudaFree(nsel);
        }
    } b;
    CUDA_TRY(cudaMalloc(&b.seq, seq_len));
    CUDA_TRY(cudaMalloc(&b.rec, (nrec + 1) * sizeof(uint64_t)));
    CUDA_TRY(cudaMalloc(&b.samp, ((size_t)nsamples + 1) * sizeof(uint64_t)));
    CUDA_TRY(cudaMalloc(&b.counts, nthreads * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&b.pos, (nthreads + 1) * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&b.scounts, ((size_t)nsamples + 1) * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&b.seg, ((size_t)nsamples + 1) * sizeof(uint32_t)));
    CUDA_TRY(cudaMalloc(&b.kept, ((size_t)nsamples + 1) * sizeof(uint32_t)));
    CUDA_TRY(cudaMemcpyAsync(b.seq, seq, seq_len, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(b.rec, rec_offs, (nrec + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(b.samp, samp_recs, ((size_t)nsamples + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(b.scounts, 0, ((size_t)nsamples + 1) * sizeof(uint32_t), st));
    CUDA_TRY(cudaMemsetAsync(b.kept, 0, ((size_t)nsamples + 1) * sizeof(uint32_t), st));
    k_sketch_scan<false><<<(unsigned)nblocks, kSketchThreads, 0, st>>>(b.seq, seq_len, b.rec, nrec, b.samp, nsamples, g,
                                                                       b.counts, b.scounts, nullptr, nullptr);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    // thread offsets and sample segments: exclusive sums (the totals land in the last word)
    size_t tb0 = 0, tb1 = 0, tb2 = 0, tb3 = 0;
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb0, b.counts, b.pos, (int64_t)nthreads, st));
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb1, b.scounts, b.seg, nsamples + 1, st));
    CUDA_TRY(cudaMalloc(&b.tmp, std::max(tb0, tb1)));
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(b.tmp, tb0, b.counts, b.pos, (int64_t)nthreads, st));
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(b.tmp, tb1, b.scounts, b.seg, nsamples + 1, st));
    count_launch(2);
    uint32_t total = 0;
    CUDA_TRY(cudaMemcpyAsync(&total, b.seg + nsamples, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (total == 0)
        return KSSDGPU_OK;
    CUDA_TRY(cudaMalloc(&b.k0, (size_t)total * sizeof(unsigned long long)));
    CUDA_TRY(cudaMalloc(&b.k1, (size_t)total * sizeof(unsigned long long)));
    CUDA_TRY(cudaMalloc(&b.keep, total));
    CUDA_TRY(cudaMalloc(&b.nsel, sizeof(int)));
    k_sketch_scan<true><<<(unsigned)nblocks, kSketchThreads, 0, st>>>(b.seq, seq_len, b.rec, nrec, b.samp, nsamples, g,
                                                                      nullptr, nullptr, b.pos, b.k0);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    // sort each sample's keys, mark the kept ones, compact
    CUDA_TRY(cub::DeviceSegmentedSort::SortKeys(nullptr, tb2, b.k0, b.k1, (int64_t)total, nsamples, b.seg,
                                                b.seg + 1, st));
    CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, tb3, b.k1, b.keep, b.k0, b.nsel, (int64_t)total, st));
    if (std::max(tb2, tb3) > std::max(tb0, tb1)) {
        cudaFree(b.tmp);
        b.tmp = nullptr;
        CUDA_TRY(cudaMalloc(&b.tmp, std::max(tb2, tb3)));
    }
    CUDA_TRY(cub::DeviceSegmentedSort::SortKeys(b.tmp, tb2, b.k0, b.k1, (int64_t)total, nsamples, b.seg, b.seg + 1,
                                                st));
    k_sketch_keep<<<grid_for(total), 256, 0, st>>>(b.k1, total, b.seg, nsamples, ob, p->conflict ? 1 : 0, b.keep,
                                                   b.kept);
    CUDA_TRY(cub::DeviceSelect::Flagged(b.tmp, tb3, b.k1, b.keep, b.k0, b.nsel, (int64_t)total, st));
    count_launch(3);
    int nsel = 0;
    std::vector<uint32_t> kept((size_t)nsamples);
    CUDA_TRY(cudaMemcpyAsync(&nsel, b.nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(kept.data(), b.kept, (size_t)nsamples * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int s = 0; s < nsamples; ++s)
        offs[s + 1] = offs[s] + kept[s];
    if (offs[nsamples] != (uint64_t)nsel)
        return fail(KSSDGPU_ERR_CUDA, "sketch compaction count mismatch");
    if ((uint64_t)nsel > keys_cap || (nsel && !keys))
        return fail(KSSDGPU_ERR_CAPACITY, "sketch output needs " + std::to_string(nsel) + " keys (offs holds them)");
    if (nsel)
        CUDA_TRY(cudaMemcpy(keys, b.k0, (size_t)nsel * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return KSSDGPU_OK;
}


int kssdgpu_index_from_records(const void *records12, uint64_t n, int nref, int obj_bits, int device,
                               kssdgpu_index_t **out)
{
    if (n && !records12)
        return fail(KSSDGPU_ERR_ARG, "null records");
    kssdgpu_index *ix = nullptr;
    int rc = new_index(nref, obj_bits, device, n, &ix);
    if (rc)
        return rc;
    cudaStream_t st = 0;
    uint32_t *w = nullptr, *head = nullptr;
    unsigned long long *ctx_of = nullptr;
    auto cleanup = [&]() {
        cudaFree(w);
        cudaFree(head);
        cudaFree(ctx_of);
    };
    cudaError_t e = cudaMalloc(&w, std::max<uint64_t>(n, 1) * 12);
    if (e == cudaSuccess)
        e = cudaMalloc(&head, std::max<uint64_t>(n, 1) * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&ctx_of, std::max<uint64_t>(n, 1) * 8);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(w, records12, n * 12, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cleanup();
        kssdgpu_index_free(ix);
        return fail(KSSDGPU_ERR_CUDA, std::string("index upload: ") + cudaGetErrorString(e));
    }
    if (n) {
        k_unpack_records<<<grid_for(n), 256, 0, st>>>(w, n, nref, ix->post, head, ctx_of, ix->err);
        count_launch();
    }
    rc = finish_build(ix, head, ctx_of, st);
    cleanup();
    if (rc) {
        kssdgpu_index_free(ix);
        return rc;
    }
    *out = ix;
    return KSSDGPU_OK;
}

int kssdgpu_index_from_sketch(const uint64_t *keys, const uint64_t *offs, int nref, int obj_bits, int device,
                              kssdgpu_index_t **out)
{
    if (!offs)
        return fail(KSSDGPU_ERR_ARG, "null offsets");
    if (nref <= 0)
        return fail(KSSDGPU_ERR_ARG, "reference count must be positive");
    const uint64_t n = offs[nref] - offs[0];
    if (n && !keys)
        return fail(KSSDGPU_ERR_ARG, "null keys");
    kssdgpu_index *ix = nullptr;
    int rc = new_index(nref, obj_bits, device, n, &ix);
    if (rc)
        return rc;
    cudaStream_t st = 0;
    uint64_t *dk = nullptr, *doffs = nullptr;
    unsigned long long *skey = nullptr, *skey2 = nullptr, *ctx_of = nullptr;
    uint32_t *sval = nullptr, *sval2 = nullptr, *head = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {
        cudaFree(dk);
        cudaFree(doffs);
        cudaFree(skey);
        cudaFree(skey2);
        cudaFree(ctx_of);
        cudaFree(sval);
        cudaFree(sval2);
        cudaFree(head);
        cudaFree(tmp);
    };
    const uint64_t nn = std::max<uint64_t>(n, 1);
    cudaError_t e = cudaMalloc(&dk, nn * 8);
    if (e == cudaSuccess) e = cudaMalloc(&doffs, ((uint64_t)nref + 1) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&skey, nn * 8);
    if (e == cudaSuccess) e = cudaMalloc(&skey2, nn * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sval, nn * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sval2, nn * 4);
    if (e == cudaSuccess) e = cudaMalloc(&head, nn * 4);
    if (e == cudaSuccess) e = cudaMalloc(&ctx_of, nn * 8);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(dk, keys, n * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(doffs, offs, ((uint64_t)nref + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cleanup();
        kssdgpu_index_free(ix);
        return fail(e == cudaErrorMemoryAllocation ? KSSDGPU_ERR_NOMEM : KSSDGPU_ERR_CUDA,
                    std::string("sketch upload: ") + cudaGetErrorString(e));
    }
    if (n) {
        k_sketch_to_sortkeys<<<std::min(nref, 148 * 16), 256, 0, st>>>(dk, doffs, nref, obj_bits, skey, sval, ix->err);
        count_launch();
        // stable LSD radix sort on the 64-bit ctxgid; equal keys keep comblco (obj ascending) order
        int end_bit = 64;
        size_t tb = 0;
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb, skey, skey2, sval, sval2, (int64_t)n, 0, end_bit, st);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max<size_t>(tb, 1));
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(tmp, tb, skey, skey2, sval, sval2, (int64_t)n, 0, end_bit, st);
        count_launch(4);
        if (e != cudaSuccess) {
            cleanup();
            kssdgpu_index_free(ix);
            return fail(KSSDGPU_ERR_CUDA, std::string("device sort: ") + cudaGetErrorString(e));
        }
        k_sorted_to_post<<<grid_for(n), 256, 0, st>>>(skey2, sval2, n, ix->post, head, ctx_of);
        count_launch();
    }
    rc = finish_build(ix, head, ctx_of, st);
    cleanup();
    if (rc) {
        kssdgpu_index_free(ix);
        return rc;
    }
    *out = ix;
    return KSSDGPU_OK;
}

void kssdgpu_index_free(kssdgpu_index_t *ix)
{
    if (!ix)
        return;
    cudaSetDevice(ix->device);
    cudaFree(ix->post);
    cudaFree(ix->gkey);
    cudaFree(ix->gbeg);
    cudaFree(ix->table);
    cudaFree(ix->bloom);
    cudaFree(ix->bloom_bounds);
    cudaFree(ix->err);
    cudaFree(ix->work);
    ix->s_keys.release();
    ix->s_offs.release();
    ix->s_out.release();
    ix->s_order.release();
    ix->s_items.release();
    ix->s_prefix.release();
    ix->s_spos.release();
    ix->s_scnt.release();
    ix->s_spre.release();
    ix->s_sitems.release();
    for (int i = 0; i < 3; ++i)
        if (ix->pipe_st[i])
            cudaStreamDestroy(ix->pipe_st[i]);
    for (cudaEvent_t e : ix->pipe_ev)
        cudaEventDestroy(e);
    ix->pipe_ev.clear();
    ix->s_counts.release();
    ix->s_cubtmp.release();
    ix->j_small.release();
    ix->c_key.release();
    ix->c_acc.release();
    ix->m_val.release();
    ix->m_recheck.release();
    ix->m_nrecheck.release();
    ix->j_post.release();
    ix->j_chunks.release();
    ix->j_items.release();
    ix->j_tile.release();
    ix->j_islot.release();
    ix->j_touched.release();
    ix->j_cacc.release();
    if (ix->j_fill_st)
        cudaStreamDestroy(ix->j_fill_st);
    for (cudaEvent_t e : ix->j_fill_ev)
        if (e)
            cudaEventDestroy(e);
    ix->j_fheads.release();
    ix->j_big.release();
    ix->j_conf.release();
    delete ix;
}

int kssdgpu_index_info(const kssdgpu_index_t *ix, uint64_t *records, uint64_t *contexts, int *nref, int *obj_bits)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    if (records) *records = ix->n;
    if (contexts) *contexts = ix->u;
    if (nref) *nref = ix->nref;
    if (obj_bits) *obj_bits = ix->obj_bits;
    return KSSDGPU_OK;
}

int kssdgpu_index_filter(kssdgpu_index_t *ix, uint64_t max_stripe_bytes, int *stripes, uint64_t *bytes)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    if (max_stripe_bytes && max_stripe_bytes < 32)
        return fail(KSSDGPU_ERR_ARG, "a filter stripe holds at least one 32-byte block");
    CUDA_TRY(cudaSetDevice(ix->device));
    cudaStream_t st = nullptr;
    CUDA_TRY(cudaDeviceSynchronize());
    int rc = build_filter(ix, max_stripe_bytes ? max_stripe_bytes : kStripeBytes, st);
    if (rc)
        return rc;
    CUDA_TRY(cudaStreamSynchronize(st));
    if (stripes)
        *stripes = ix->bloom ? ix->bloom_stripes : 0;
    if (bytes)
        *bytes = ix->bloom ? (uint64_t)ix->bloom_stripes * ((uint64_t)ix->bloom_mask + 1) * 32 : 0;
    return KSSDGPU_OK;
}

int kssdgpu_index_export(const kssdgpu_index_t *cix, void *records12, uint8_t *unique_bits)
{
    kssdgpu_index *ix = const_cast<kssdgpu_index *>(cix);
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    CUDA_TRY(cudaSetDevice(ix->device));
    cudaStream_t st = 0;
    const uint64_t n = ix->n;
    if (records12 && n) {
        uint32_t *w = nullptr;
        CUDA_TRY(cudaMalloc(&w, n * 12));
        k_export_records<<<grid_for(ix->u), 256, 0, st>>>(ix->gkey, ix->gbeg, ix->u, ix->post, w);
        count_launch();
        CUDA_TRY(cudaMemcpyAsync(records12, w, n * 12, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        cudaFree(w);
    }
    if (unique_bits && n) {
        const uint64_t words = (n + 31) / 32;
        uint32_t *b = nullptr;
        CUDA_TRY(cudaMalloc(&b, words * 4));
        CUDA_TRY(cudaMemsetAsync(b, 0, words * 4, st));
        k_unique_bits<<<grid_for(ix->u), 256, 0, st>>>(ix->gbeg, ix->u, ix->post, b);
        count_launch();
        std::vector<uint32_t> hb(words);
        CUDA_TRY(cudaMemcpyAsync(hb.data(), b, words * 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        cudaFree(b);
        std::memcpy(unique_bits, hb.data(), (n + 7) / 8);
    }
    return KSSDGPU_OK;
}

int kssdgpu_index_ref_ctx_counts(const kssdgpu_index_t *cix, int conflict, int ignoreconflict, uint32_t *ctx_count_out,
                                 uint32_t *unique_out)
{
    kssdgpu_index *ix = const_cast<kssdgpu_index *>(cix);
    if (!ix || (!ctx_count_out && !unique_out))
        return fail(KSSDGPU_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(ix->device));
    cudaStream_t st = 0;
    uint32_t *c = nullptr;
    CUDA_TRY(cudaMalloc(&c, (size_t)ix->nref * 2 * sizeof(uint32_t)));
    CUDA_TRY(cudaMemsetAsync(c, 0, (size_t)ix->nref * 2 * sizeof(uint32_t), st));
    k_ref_counts<<<grid_for(ix->u), 256, 0, st>>>(ix->gbeg, ix->u, ix->post, conflict, ignoreconflict, c, c + ix->nref);
    count_launch();
    if (ctx_count_out)
        CUDA_TRY(cudaMemcpyAsync(ctx_count_out, c, (size_t)ix->nref * 4, cudaMemcpyDeviceToHost, st));
    if (unique_out)
        CUDA_TRY(cudaMemcpyAsync(unique_out, c + ix->nref, (size_t)ix->nref * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(c);
    return KSSDGPU_OK;
}

int kssdgpu_count_block(kssdgpu_index_t *ix, const uint64_t *qry_keys, const uint64_t *qry_offs, int nq, unsigned flags,
                        kssdgpu_ctx_mut2_t *ctx, kssdgpu_obj_section_t *obj, kssdgpu_ctx_mut2_t *uctx,
                        kssdgpu_obj_section_t *uobj)
{
    return count_host_impl(ix, qry_keys, qry_offs, nq, 0, false, flags, ctx, obj, uctx, uobj);
}

int kssdgpu_count_lower(kssdgpu_index_t *ix, const uint64_t *qry_keys, const uint64_t *qry_offs, int nq,
                        int qry_gid_offset, unsigned flags, kssdgpu_ctx_mut2_t *ctx, kssdgpu_obj_section_t *obj)
{
    if (flags & KSSDGPU_UNIQUE)
        return fail(KSSDGPU_ERR_ARG, "unique-context counting has no lower-triangle form");
    return count_host_impl(ix, qry_keys, qry_offs, nq, qry_gid_offset, true, flags, ctx, obj, nullptr, nullptr);
}

int kssdgpu_count_block_dev(kssdgpu_index_t *ix, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs, int nq,
                            int qry_gid_offset, int lower, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx,
                            kssdgpu_obj_section_t *d_obj, kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj,
                            void *stream)
{
    if (!ix || nq < 0 || (nq && (!d_qry_offs || !d_ctx || !d_obj)))
        return fail(KSSDGPU_ERR_ARG, "invalid device count arguments");
    if (flags & KSSDGPU_PLAIN)
        return fail(KSSDGPU_ERR_ARG, "the plain kernel needs host offsets; use the host-buffer call");
    CUDA_TRY(cudaSetDevice(ix->device));
    return count_dev_impl(ix, d_qry_keys, d_qry_offs, nq, qry_gid_offset, lower != 0, flags,
                          reinterpret_cast<unsigned long long *>(d_ctx), reinterpret_cast<unsigned long long *>(d_obj),
                          reinterpret_cast<unsigned long long *>(d_uctx), reinterpret_cast<unsigned long long *>(d_uobj),
                          nullptr, nullptr, (cudaStream_t)stream);
}

int kssdgpu_count_tune(kssdgpu_index_t *ix, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs, int nq,
                       int qry_gid_offset, int lower, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx,
                       kssdgpu_obj_section_t *d_obj, kssdgpu_ctx_mut2_t *d_uctx, kssdgpu_obj_section_t *d_uobj,
                       kssdgpu_count_tuning_t *out)
{
    if (!ix || nq < 1 || !d_qry_offs || !d_ctx || !d_obj)
        return fail(KSSDGPU_ERR_ARG, "invalid count-tuning arguments");
    CUDA_TRY(cudaSetDevice(ix->device));
    const unsigned base = flags & (KSSDGPU_UNIQUE | KSSDGPU_IGNORECONFLICT);
    struct Cand {
        bool smem;
        uint32_t chunk;
        bool striped;
    };
    // with the filter on: global rows in key-range chunks, global rows stripe by stripe
    // (several filter stripes), shared rows (where a row fits)
    std::vector<Cand> cands = {{false, 1024, false}, {false, 4096, false}, {false, 16384, false}};
    if (ix->bloom && ix->bloom_stripes > 1)
        cands.push_back({false, 4096, true});
    if (smem_row_fits(ix, base))
        cands.push_back({true, 4096, false});
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(cudaEventCreate(&ev0));
    cudaError_t ce = cudaEventCreate(&ev1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(ev0);
        return fail(KSSDGPU_ERR_CUDA, cudaGetErrorString(ce));
    }
    const bool keep_smem = ix->count_smem, keep_striped = ix->count_striped, keep_filter = ix->count_filter;
    const uint32_t keep_chunk = ix->count_chunk_keys;
    int rc = KSSDGPU_OK, tried = 0;
    // best of three timed runs after a warm-up, CUDA events on the legacy stream
    auto time_setting = [&](const Cand &c, bool filter, float &t_min) {
        ix->count_smem = c.smem;
        ix->count_chunk_keys = c.chunk;
        ix->count_striped = c.striped;
        ix->count_filter = filter;
        const unsigned f = base | (c.smem ? KSSDGPU_SMEM_ACC : KSSDGPU_GLOBAL_ACC);
        t_min = 1e30f;
        for (int r = 0; r < 4 && rc == KSSDGPU_OK; ++r) {
            ce = cudaEventRecord(ev0, 0);
            if (ce == cudaSuccess) {
                rc = count_dev_impl(ix, d_qry_keys, d_qry_offs, nq, qry_gid_offset, lower != 0, f,
                                    reinterpret_cast<unsigned long long *>(d_ctx),
                                    reinterpret_cast<unsigned long long *>(d_obj),
                                    reinterpret_cast<unsigned long long *>(d_uctx),
                                    reinterpret_cast<unsigned long long *>(d_uobj), nullptr, nullptr, 0);
                if (rc)
                    break;
            }
            if (ce == cudaSuccess) ce = cudaEventRecord(ev1, 0);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
            float ms = 0;
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, ev0, ev1);
            if (ce != cudaSuccess) {
                rc = fail(KSSDGPU_ERR_CUDA, cudaGetErrorString(ce));
                break;
            }
            if (r > 0)
                t_min = std::min(t_min, ms);
        }
        if (rc == KSSDGPU_OK)
            ++tried;
    };
    float best = 1e30f;
    Cand pick = {keep_smem, keep_chunk, keep_striped};
    const bool filter_on = ix->bloom != nullptr;
    for (const Cand &c : cands) {
        float t = 0;
        time_setting(c, filter_on, t);
        if (rc)
            break;
        if (t < best) {
            best = t;
            pick = c;
        }
    }
    // then the best setting without the membership filter
    bool filter = filter_on;
    if (rc == KSSDGPU_OK && filter_on) {
        float t = 0;
        time_setting(pick, false, t);
        if (rc == KSSDGPU_OK && t < best) {
            best = t;
            filter = false;
        }
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (rc) {
        ix->count_smem = keep_smem;
        ix->count_chunk_keys = keep_chunk;
        ix->count_striped = keep_striped;
        ix->count_filter = keep_filter;
        return rc;
    }
    ix->count_filter = filter;
    ix->count_striped = pick.striped;
    ix->count_smem = pick.smem;
    ix->count_chunk_keys = pick.chunk;
    ix->count_tune_tried = tried;
    ix->count_tune_ms = best;
    if (out) {
        out->smem_rows = pick.smem ? 1 : 0;
        out->chunk_keys = pick.chunk;
        out->candidates = tried;
        out->ms = best;
        out->filter = ix->count_filter && ix->bloom ? 1 : 0;
        out->striped = out->filter && ix->count_striped && ix->bloom_stripes > 1 && !pick.smem ? 1 : 0;
    }
    return check_dev_err(ix, 0);
}

int kssdgpu_count_plain_dev(kssdgpu_index_t *ix, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs,
                            const uint64_t *h_qry_offs, int nq, int qry_gid_offset, int lower, unsigned flags,
                            kssdgpu_ctx_mut2_t *d_ctx, kssdgpu_obj_section_t *d_obj, kssdgpu_ctx_mut2_t *d_uctx,
                            kssdgpu_obj_section_t *d_uobj, void *stream)
{
    if (!ix || nq < 0 || (nq && (!d_qry_offs || !h_qry_offs || !d_ctx || !d_obj)))
        return fail(KSSDGPU_ERR_ARG, "invalid plain count arguments");
    CUDA_TRY(cudaSetDevice(ix->device));
    std::vector<uint64_t> sizes(nq);
    for (int i = 0; i < nq; ++i)
        sizes[i] = h_qry_offs[i + 1] - h_qry_offs[i];
    return count_dev_impl(ix, d_qry_keys, d_qry_offs, nq, qry_gid_offset, lower != 0, flags | KSSDGPU_PLAIN,
                          reinterpret_cast<unsigned long long *>(d_ctx), reinterpret_cast<unsigned long long *>(d_obj),
                          reinterpret_cast<unsigned long long *>(d_uctx), reinterpret_cast<unsigned long long *>(d_uobj),
                          nullptr, &sizes, (cudaStream_t)stream);
}

int kssdgpu_count_block_noalloc(kssdgpu_index_t *ix, const uint64_t *d_qry_keys, const uint64_t *d_qry_offs,
                                int nq, int qry_gid_offset, int lower, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx,
                                kssdgpu_obj_section_t *d_obj, kssdgpu_ctx_mut2_t *d_uctx,
                                kssdgpu_obj_section_t *d_uobj, void *stream)
{
    if (!ix || nq < 0 || (nq && (!d_qry_offs || !d_ctx || !d_obj)))
        return fail(KSSDGPU_ERR_ARG, "invalid no-allocation count arguments");
    if (nq > KSSDGPU_NOALLOC_MAX_QUERIES)
        return fail(KSSDGPU_ERR_CAPACITY, "no-allocation count: " + std::to_string(nq) +
                                              " queries exceed the maximum of " +
                                              std::to_string(KSSDGPU_NOALLOC_MAX_QUERIES) + " per call");
    if (flags & KSSDGPU_PLAIN)
        return fail(KSSDGPU_ERR_ARG, "the no-allocation count runs the batched kernel only");
    const bool unique = (flags & KSSDGPU_UNIQUE) != 0;
    if (lower && unique)
        return fail(KSSDGPU_ERR_ARG, "unique-context counting has no lower-triangle form");
    if (unique && (!d_uctx || !d_uobj))
        return fail(KSSDGPU_ERR_ARG, "unique counters requested without output buffers");
    CUDA_TRY(cudaSetDevice(ix->device));
    unsigned int *scr = nullptr;
    int rc = noalloc_scratch(ix->device, &scr);
    if (rc)
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(scr, 0, kNoallocHeaderWords * sizeof(unsigned int), st));
    if (nq == 0)
        return KSSDGPU_OK;
    // the accumulator mode of kssdgpu_count_block_dev: global rows in key-range chunks
    // unless shared-memory rows are forced or were chosen by the count autotuner
    if ((flags & KSSDGPU_SMEM_ACC) && !(flags & KSSDGPU_GLOBAL_ACC) && !smem_row_fits(ix, flags))
        return fail(KSSDGPU_ERR_CAPACITY, "shared-memory accumulator rows requested, but a row of " +
                                              std::to_string(ix->nref) + " references does not fit");
    const bool use_smem = uses_smem_row(ix, flags);
    const int grid = std::min((nq + 255) / 256, ix->sms * 8);
    if (use_smem) {
        k_noalloc_hist<<<grid, 256, 0, st>>>(d_qry_offs, nq, scr);
        k_noalloc_scan<<<1, 32, 0, st>>>(scr);
        k_noalloc_scatter<<<grid, 256, 0, st>>>(d_qry_offs, nq, scr);
        count_launch(3);
    } else {
        k_noalloc_prefix<<<1, 1024, 0, st>>>(d_qry_offs, nq, ix->count_chunk_keys, scr + kNoallocHeaderWords - 1);
        count_launch();
    }
    CUDA_TRY(cudaGetLastError());
    CountParams P{};
    P.table = ix->table;
    P.mask = ix->mask;
    P.post = ix->post;
    P.qkeys = d_qry_keys;
    P.qoffs = d_qry_offs;
    P.nq = nq;
    P.nref = ix->nref;
    P.qgid_offset = qry_gid_offset;
    P.obj_bits = ix->obj_bits;
    P.ignoreconflict = (flags & KSSDGPU_IGNORECONFLICT) ? 1 : 0;
    P.out_ctx = reinterpret_cast<unsigned long long *>(d_ctx);
    P.out_obj = reinterpret_cast<unsigned long long *>(d_obj);
    P.out_uctx = reinterpret_cast<unsigned long long *>(d_uctx);
    P.out_uobj = reinterpret_cast<unsigned long long *>(d_uobj);
    P.work = scr;
    P.err = ix->err;
    P.bloom = ix->count_filter ? ix->bloom : nullptr;
    P.bloom_mask = ix->bloom_mask;
    P.bloom_stripes = ix->bloom_stripes;
    P.bloom_bounds = ix->bloom_bounds;
    P.order = use_smem ? reinterpret_cast<const int *>(scr + kNoallocHeaderWords) : nullptr;
    P.chunk_prefix = use_smem ? nullptr : scr + kNoallocHeaderWords - 1;
    P.chunk_keys = ix->count_chunk_keys;
    const size_t cells = (size_t)nq * ix->nref;
    const size_t smem = (size_t)ix->nref * sizeof(unsigned long long) * (unique ? 4 : 2);
    if (!use_smem && !(flags & KSSDGPU_NO_ZERO)) {
        CUDA_TRY(cudaMemsetAsync(d_ctx, 0, cells * 8, st));
        CUDA_TRY(cudaMemsetAsync(d_obj, 0, cells * 8, st));
        if (unique) {
            CUDA_TRY(cudaMemsetAsync(d_uctx, 0, cells * 8, st));
            CUDA_TRY(cudaMemsetAsync(d_uobj, 0, cells * 8, st));
        }
    }
    if (use_smem) {
        if (lower)
            return launch_batched<true, false, true>(ix, P, smem, st);
        return unique ? launch_batched<false, true, true>(ix, P, smem, st)
                      : launch_batched<false, false, true>(ix, P, smem, st);
    }
    if (lower)
        return launch_batched<true, false, false>(ix, P, 0, st);
    return unique ? launch_batched<false, true, false>(ix, P, 0, st) : launch_batched<false, false, false>(ix, P, 0, st);
}

int kssdgpu_count_detail(kssdgpu_index_t *ix, const uint64_t *qry_keys, const uint64_t *qry_offs, int nq,
                         unsigned flags, const uint32_t *qry_ctx_count, const uint32_t *ref_ctx_count, int ctxcut,
                         float afcut, float anicut, kssdgpu_hit_t *hits, uint64_t hits_cap, uint64_t *row_offs)
{
    if (!ix || nq < 0 || !row_offs || (nq > 0 && (!qry_offs || !qry_ctx_count || !ref_ctx_count)))
        return fail(KSSDGPU_ERR_ARG, "invalid detail count arguments");
    if (flags & (KSSDGPU_PLAIN | KSSDGPU_NO_ZERO | KSSDGPU_SELF_PLAN))
        return fail(KSSDGPU_ERR_ARG, "the detail count takes KSSDGPU_IGNORECONFLICT, KSSDGPU_UNIQUE and the "
                                     "accumulator flags only");
    row_offs[0] = 0;
    if (nq == 0)
        return KSSDGPU_OK;
    CUDA_TRY(cudaSetDevice(ix->device));
    const uint64_t nkeys = qry_offs[nq] - qry_offs[0];
    if (nkeys && !qry_keys)
        return fail(KSSDGPU_ERR_ARG, "null query keys");
    std::vector<uint64_t> sizes(nq);
    for (int i = 0; i < nq; ++i) {
        if (qry_offs[i + 1] < qry_offs[i])
            return fail(KSSDGPU_ERR_ARG, "query offsets are not monotone");
        sizes[i] = qry_offs[i + 1] - qry_offs[i];
    }
    const bool unique = (flags & KSSDGPU_UNIQUE) != 0;
    std::vector<int> order(nq);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sizes[a] > sizes[b]; });
    std::vector<WorkItem> items;
    if (!uses_smem_row(ix, flags))
        build_chunks(qry_offs, nq, order.data(), ix->count_chunk_keys, items);
    const int nref = ix->nref;
    const size_t cells = (size_t)nq * nref;
    CUDA_TRY(ix->s_keys.ensure(nkeys));
    CUDA_TRY(ix->s_offs.ensure((size_t)nq + 1));
    CUDA_TRY(ix->s_out.ensure(cells * (unique ? 4 : 2)));
    CUDA_TRY(ix->s_order.ensure((size_t)nq));
    CUDA_TRY(ix->s_items.ensure(items.size()));
    CUDA_TRY(ix->s_qcnt.ensure((size_t)nq));
    CUDA_TRY(ix->s_rcnt.ensure((size_t)nref));
    CUDA_TRY(ix->s_dcount.ensure((size_t)nq));
    CUDA_TRY(ix->s_dprefix.ensure((size_t)nq + 1));
    cudaStream_t st = 0;
    if (nkeys)
        CUDA_TRY(cudaMemcpyAsync(ix->s_keys.p, qry_keys, nkeys * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_offs.p, qry_offs, ((size_t)nq + 1) * 8, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_order.p, order.data(), (size_t)nq * sizeof(int), cudaMemcpyHostToDevice, st));
    if (!items.empty())
        CUDA_TRY(cudaMemcpyAsync(ix->s_items.p, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                 st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_qcnt.p, qry_ctx_count, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_rcnt.p, ref_ctx_count, (size_t)nref * 4, cudaMemcpyHostToDevice, st));
    unsigned long long *oc = ix->s_out.p, *oo = oc + cells;
    unsigned long long *uc = unique ? oo + cells : nullptr, *uo = unique ? uc + cells : nullptr;
    int rc = count_dev_impl(ix, ix->s_keys.p, ix->s_offs.p, nq, 0, false, flags, oc, oo, uc, uo, ix->s_order.p, &sizes,
                            st, items.empty() ? nullptr : ix->s_items.p, (int)items.size());
    if (rc)
        return rc;
    DetailFilter F;
    F.qcnt = ix->s_qcnt.p;
    F.rcnt = ix->s_rcnt.p;
    F.ctxcut = (uint32_t)ctxcut;
    F.afcut = (double)afcut;
    F.ani_lo = (double)anicut - kDetailMargin;
    F.unique = unique ? 1 : 0;
    const int grid = std::min(nq, ix->sms * 8);
    k_detail_count<<<grid, 256, 0, st>>>(oc, oo, uc, uo, nq, nref, F, ix->s_dcount.p);
    k_detail_prefix<<<1, 1024, 0, st>>>(ix->s_dcount.p, nq, ix->s_dprefix.p);
    count_launch(2);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(row_offs, ix->s_dprefix.p, ((size_t)nq + 1) * 8, cudaMemcpyDeviceToHost, st));
    rc = check_dev_err(ix, st);  // synchronizes: row_offs is on the host now
    if (rc)
        return rc;
    const uint64_t total = row_offs[nq];
    if (total > hits_cap)
        return fail(KSSDGPU_ERR_CAPACITY, "detail count: " + std::to_string(total) +
                                              " candidate cells exceed the hit buffer of " + std::to_string(hits_cap) +
                                              " (row_offs holds the sizes)");
    if (!total)
        return KSSDGPU_OK;
    if (!hits)
        return fail(KSSDGPU_ERR_ARG, "null hit buffer");
    CUDA_TRY(ix->s_hits.ensure(total));
    k_detail_write<<<grid, 256, 0, st>>>(oc, oo, uc, uo, nq, nref, F, ix->s_dprefix.p, ix->s_hits.p);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(hits, ix->s_hits.p, total * sizeof(kssdgpu_hit_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return KSSDGPU_OK;
}

int kssdgpu_self_plan_info(kssdgpu_index_t *ix, uint64_t *groups, uint64_t *postings, uint64_t *pairs)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    if (groups) *groups = ix->f_groups;
    if (postings) *postings = ix->f_postings;
    if (pairs) *pairs = ix->f_pairs;
    return KSSDGPU_OK;
}

int kssdgpu_self_dense_alleles(kssdgpu_index_t *ix, uint64_t *alleles)
{
    if (!ix || !alleles)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    *alleles = ix->d_alleles;
    return KSSDGPU_OK;
}

int kssdgpu_self_choice(kssdgpu_index_t *ix, unsigned flags, int *path, double *density)
{
    if (!ix || !path)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(ix->device));
    if (density)
        *density = self_density(ix);
    if (flags & KSSDGPU_SELF_DENSE)
        *path = KSSDGPU_PATH_DENSE;
    else if (flags & KSSDGPU_SELF_PLAN)
        *path = KSSDGPU_PATH_PLAN;
    else if (!(flags & (KSSDGPU_SELF_SCAN | KSSDGPU_NO_ZERO)) && dense_chosen(ix))
        *path = KSSDGPU_PATH_DENSE;
    else
        *path = KSSDGPU_PATH_SCAN;
    return KSSDGPU_OK;
}

int kssdgpu_self_plan_tune(kssdgpu_index_t *ix, uint32_t *chunk_groups, int *sorted, uint32_t *flat_groups,
                           int *candidates, float *step_ms)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    CUDA_TRY(cudaSetDevice(ix->device));
    int rc = self_plan(ix, 0);
    if (rc)
        return rc;
    if (!ix->j_tuned) {
        const cudaError_t e = tune_join(ix, ix->j_n[0], 0);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? KSSDGPU_ERR_NOMEM : KSSDGPU_ERR_CUDA,
                        std::string("self-join autotuner: ") + cudaGetErrorString(e));
    }
    if (chunk_groups) *chunk_groups = ix->j_chunk_size;
    if (sorted) *sorted = ix->j_sort_chunks ? 1 : 0;
    if (flat_groups) *flat_groups = ix->j_flat_max;
    if (candidates) *candidates = ix->j_tune_tried;
    if (step_ms) *step_ms = ix->j_tune_ms;
    return KSSDGPU_OK;
}

int kssdgpu_sync(kssdgpu_index_t *ix, void *stream)
{
    if (!ix)
        return fail(KSSDGPU_ERR_ARG, "null index");
    CUDA_TRY(cudaSetDevice(ix->device));
    CUDA_TRY(cudaGetLastError());
    return check_dev_err(ix, (cudaStream_t)stream);
}

int kssdgpu_self_lower(kssdgpu_index_t *ix, unsigned flags, kssdgpu_ctx_mut2_t *ctx_lower,
                       kssdgpu_obj_section_t *obj_lower)
{
    if (!ix || !ctx_lower || !obj_lower)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(ix->device));
    const size_t cells = (size_t)ix->nref * (ix->nref - 1) / 2;
    CUDA_TRY(ix->s_out.ensure(std::max<size_t>(cells, 1) * 2));
    cudaStream_t st = 0;
    int rc = self_lower_dev_impl(ix, flags, ix->s_out.p, ix->s_out.p + std::max<size_t>(cells, 1), st);
    if (rc)
        return rc;
    if (cells) {
        CUDA_TRY(cudaMemcpyAsync(ctx_lower, ix->s_out.p, cells * 8, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(obj_lower, ix->s_out.p + cells, cells * 8, cudaMemcpyDeviceToHost, st));
    }
    return check_dev_err(ix, st);
}

int kssdgpu_self_votes(kssdgpu_index_t *ix, const uint64_t *keys, const uint64_t *offs, uint32_t max_ctx_freq,
                       uint32_t sample_step, uint32_t *votes, uint32_t *first)
{
    if (!ix || !offs || !votes || !first || sample_step == 0)
        return fail(KSSDGPU_ERR_ARG, "invalid vote arguments");
    CUDA_TRY(cudaSetDevice(ix->device));
    const int n = ix->nref;
    const size_t cells = (size_t)n * (n > 0 ? n - 1 : 0) / 2;
    if (!cells)
        return KSSDGPU_OK;
    const uint64_t nkeys = offs[n] - offs[0];
    if (nkeys && !keys)
        return fail(KSSDGPU_ERR_ARG, "null keys");
    for (int i = 0; i < n; ++i)
        if (offs[i + 1] < offs[i])
            return fail(KSSDGPU_ERR_ARG, "sample offsets are not monotone");
    cudaStream_t st = 0;
    CUDA_TRY(ix->s_keys.ensure(nkeys));
    CUDA_TRY(ix->s_offs.ensure((size_t)n + 1));
    uint32_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, cells * 8);
    if (e != cudaSuccess)
        return fail(KSSDGPU_ERR_NOMEM, std::string("vote counters: ") + cudaGetErrorString(e));
    if (nkeys)
        e = cudaMemcpyAsync(ix->s_keys.p, keys, nkeys * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ix->s_offs.p, offs, ((size_t)n + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, cells * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + cells, 0xFF, cells * 4, st);
    if (e == cudaSuccess && nkeys) {
        k_self_votes<<<grid_for(nkeys), 256, 0, st>>>(ix->table, ix->mask, ix->post, ix->s_keys.p, ix->s_offs.p, n,
                                                      nkeys, ix->obj_bits, max_ctx_freq, sample_step, d, d + cells);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(votes, d, cells * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(first, d + cells, cells * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess)
        return fail(KSSDGPU_ERR_CUDA, cudaGetErrorString(e));
    return check_dev_err(ix, st);
}

int kssdgpu_self_lower_dev(kssdgpu_index_t *ix, unsigned flags, kssdgpu_ctx_mut2_t *d_ctx_lower,
                           kssdgpu_obj_section_t *d_obj_lower, void *stream)
{
    if (!ix || !d_ctx_lower || !d_obj_lower)
        return fail(KSSDGPU_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(ix->device));
    return self_lower_dev_impl(ix, flags, reinterpret_cast<unsigned long long *>(d_ctx_lower),
                               reinterpret_cast<unsigned long long *>(d_obj_lower), (cudaStream_t)stream);
}

int kssdgpu_lower_metric_dev(int device, const kssdgpu_metric_opt_t *opt, int n, const uint32_t *d_qcnt,
                             const uint32_t *d_rcnt, const kssdgpu_ctx_mut2_t *d_ctx_lower,
                             const kssdgpu_obj_section_t *d_obj_lower, double *d_value_lower,
                             kssdgpu_recheck_t *d_recheck, uint64_t recheck_cap, uint64_t *d_nrecheck, void *stream)
{
    if (n < 0 || !d_nrecheck || (n > 1 && (!d_qcnt || !d_rcnt || !d_ctx_lower || !d_obj_lower || !d_value_lower)) ||
        (recheck_cap && !d_recheck))
        return fail(KSSDGPU_ERR_ARG, "null argument or negative size");
    static_assert(sizeof(kssdgpu_recheck_t) == sizeof(kssd::RecheckCell), "recheck records are 24 bytes");
    CUDA_TRY(cudaSetDevice(device));
    kssd::MetricParams P;
    int rc = metric_params(device, opt, P);
    if (rc)
        return rc;
    int sms = 148;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(d_nrecheck, 0, sizeof(uint64_t), st));
    CUDA_TRY(kssd::lower_metric_launch(P, n, reinterpret_cast<const unsigned long long *>(d_ctx_lower),
                                       reinterpret_cast<const unsigned long long *>(d_obj_lower), d_qcnt, d_rcnt,
                                       d_value_lower, reinterpret_cast<kssd::RecheckCell *>(d_recheck), recheck_cap,
                                       reinterpret_cast<unsigned long long *>(d_nrecheck), sms, st));
    count_launch(n > 1 ? 1 : 0);
    return KSSDGPU_OK;
}

int kssdgpu_self_lower_metric(kssdgpu_index_t *ix, unsigned flags, const kssdgpu_metric_opt_t *opt,
                              const uint32_t *qcnt, const uint32_t *rcnt, double *value_lower,
                              kssdgpu_recheck_t *recheck, uint64_t recheck_cap, uint64_t *nrecheck)
{
    if (!ix || !qcnt || !rcnt || !value_lower || !nrecheck || (recheck_cap && !recheck))
        return fail(KSSDGPU_ERR_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(ix->device));
    const int n = ix->nref;
    const size_t cells = (size_t)n * (n - 1) / 2;
    *nrecheck = 0;
    if (!cells)
        return KSSDGPU_OK;
    kssd::MetricParams P;
    int rc = metric_params(ix->device, opt, P);
    if (rc)
        return rc;
    cudaStream_t st = 0;
    CUDA_TRY(ix->s_out.ensure(cells * 2));
    CUDA_TRY(ix->m_val.ensure(cells));
    CUDA_TRY(ix->m_recheck.ensure(std::max<uint64_t>(recheck_cap, 1)));
    CUDA_TRY(ix->m_nrecheck.ensure(1));
    CUDA_TRY(ix->s_qcnt.ensure((size_t)n));
    CUDA_TRY(ix->s_rcnt.ensure((size_t)n));
    CUDA_TRY(cudaMemcpyAsync(ix->s_qcnt.p, qcnt, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(ix->s_rcnt.p, rcnt, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    rc = self_lower_dev_impl(ix, flags, ix->s_out.p, ix->s_out.p + cells, st);
    if (rc)
        return rc;
    CUDA_TRY(cudaMemsetAsync(ix->m_nrecheck.p, 0, sizeof(unsigned long long), st));
    CUDA_TRY(kssd::lower_metric_launch(P, n, ix->s_out.p, ix->s_out.p + cells, ix->s_qcnt.p, ix->s_rcnt.p,
                                       ix->m_val.p, ix->m_recheck.p, recheck_cap, ix->m_nrecheck.p, ix->sms, st));
    count_launch();
    CUDA_TRY(cudaMemcpyAsync(value_lower, ix->m_val.p, cells * 8, cudaMemcpyDeviceToHost, st));
    unsigned long long nre = 0;
    CUDA_TRY(cudaMemcpyAsync(&nre, ix->m_nrecheck.p, sizeof nre, cudaMemcpyDeviceToHost, st));
    rc = check_dev_err(ix, st);  // synchronizes
    if (rc)
        return rc;
    *nrecheck = nre;
    const uint64_t listed = std::min<uint64_t>(nre, recheck_cap);
    if (listed)
        CUDA_TRY(cudaMemcpy(recheck, ix->m_recheck.p, listed * sizeof(kssdgpu_recheck_t), cudaMemcpyDeviceToHost));
    if (nre > recheck_cap)
        return fail(KSSDGPU_ERR_CAPACITY, std::to_string(nre) + " cells to value on the host, more than the " +
                                              std::to_string(recheck_cap) + " the caller's list holds");
    return KSSDGPU_OK;
}

}  // extern "C"

// continuous-batching server (same translation unit: it launches k_count_batched)
#include "kssd_server.cuh"

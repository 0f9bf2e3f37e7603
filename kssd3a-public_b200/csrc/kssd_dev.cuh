// Device-side building blocks shared by the libkssdgpu kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kssd {

constexpr int kGidBits = 20;
// Initial value (and cap) of the per-context minimum object difference: NUM_CODENS + 1
// (src/command_ani.h:287,535,694); the reference's default build has NUM_CODENS = 11,
// its 9- and 10-coden builds (-DNUM_CODENS) cap at 10 and 11.
#ifndef KSSD_NUM_CODENS
#define KSSD_NUM_CODENS 11
#endif
static_assert(KSSD_NUM_CODENS >= 9 && KSSD_NUM_CODENS <= 11, "the reference builds 9, 10 or 11 codens");
constexpr int kMinInit = KSSD_NUM_CODENS + 1;
constexpr unsigned long long kEmptyCtx = ~0ull;      // contexts are at most 44 bits
constexpr unsigned long long kInlineBit = 1ull << 62;  // slot holds its only posting

// Hash-table slot of one unique context: the key, and either its postings range
// or, for a context with a single posting, that posting itself (one random line
// per probe for the common single-owner context).
struct __align__(16) Slot {
    unsigned long long ctx;    // context | kInlineBit when inline; kEmptyCtx when free
    unsigned long long range;  // begin (low 32) | count (high 32), or the inline posting
};

// Error flag values written by kernels (host maps them to status codes).
enum DevErr : int { kDevOk = 0, kDevUnsorted = 1, kDevGid = 2, kDevProbe = 3 };

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Number of differing 2-bit bases between two objects (src/dna_popcount.h:45-49).
__device__ __forceinline__ int dna_pop(uint32_t x) { return __popc((x | (x >> 1)) & 0x55555555u); }

// Probe the open-addressing table; bounded by the table size (load <= 1/2, so an
// empty slot always ends the probe).  Returns the slot's payload and whether it is
// an inline single posting.
__device__ __forceinline__ bool table_lookup(const Slot *__restrict__ t, uint32_t mask, unsigned long long ctx,
                                             unsigned long long &payload, bool &single)
{
    uint32_t i = (uint32_t)mix64(ctx) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        const ulonglong2 s = __ldg(reinterpret_cast<const ulonglong2 *>(t + i));
        if ((s.x & ~kInlineBit) == ctx) {
            payload = s.y;
            single = (s.x & kInlineBit) != 0;
            return true;
        }
        if (s.x == kEmptyCtx)
            return false;
        i = (i + 1) & mask;
    }
    return false;
}

}  // namespace kssd

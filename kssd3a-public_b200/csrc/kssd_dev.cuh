// Device-side building blocks shared by the libkssdgpu kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kssd {

constexpr int kGidBits = 20;
// Initial value of the per-context minimum object difference: NUM_CODENS + 1 with
// the reference's default NUM_CODENS = 11 (src/command_ani.h:547,684).
constexpr int kMinInit = 12;
constexpr unsigned long long kEmptyCtx = ~0ull;  // contexts are at most 44 bits

// Hash-table slot of one unique context: key and its postings range.
struct __align__(16) Slot {
    unsigned long long ctx;    // kEmptyCtx when free
    unsigned long long range;  // begin (low 32) | count (high 32)
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
// empty slot always ends the probe).
__device__ __forceinline__ bool table_lookup(const Slot *__restrict__ t, uint32_t mask, unsigned long long ctx,
                                             uint32_t &begin, uint32_t &count)
{
    uint32_t i = (uint32_t)mix64(ctx) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        const ulonglong2 s = __ldg(reinterpret_cast<const ulonglong2 *>(t + i));
        if (s.x == ctx) {
            begin = (uint32_t)s.y;
            count = (uint32_t)(s.y >> 32);
            return true;
        }
        if (s.x == kEmptyCtx)
            return false;
        i = (i + 1) & mask;
    }
    return false;
}

}  // namespace kssd

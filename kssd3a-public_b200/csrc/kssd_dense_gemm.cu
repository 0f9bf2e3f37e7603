// Exact int8 x int8 -> int32 GEMM on the sm_100a tensor cores (tcgen05.mma with the
// accumulator in TMEM, operands staged into shared memory by TMA), through CUTLASS's
// sm100 collective mainloop and epilogue.  Used by the dense self join of
// libkssdgpu: D[M][N] = sum_k A[k][m] B[k][n] with both operands MN-major (stored
// K x M and K x N, rows contiguous over M and N), int32 D row-major.  One CTA per
// 128 x 128 tile, no thread-block cluster (no multicast loads); split-K when the output
// has fewer tiles than the GPU has SMs, stream-K otherwise.
#include "cutlass/cutlass.h"
#include "cute/tensor.hpp"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/gemm/collective/collective_builder.hpp"
#include "cutlass/gemm/device/gemm_universal_adapter.h"
#include "cutlass/gemm/dispatch_policy.hpp"
#include "cutlass/gemm/kernel/gemm_universal.hpp"
#include "cutlass/util/packed_stride.hpp"

#include <cstdint>

namespace {

using namespace cute;

// Tile width along N.  A 128 x 256 tile (half the tiles, so half the re-streaming of the
// K-long operand slices) was measured against 128 x 128 on the dense join: 5 % faster at
// 2,048 genomes, 7 % slower at 1,024 and even at 512, so 128 stays the default.
#ifndef KSSD_GEMM_TILE_N
#define KSSD_GEMM_TILE_N 128
#endif
// Work decomposition: 0 = the library's heuristic (stream-K here), 1 = split-K when the
// output has fewer tiles than SMs, else the heuristic; 2 = as 1, else data-parallel.
#ifndef KSSD_GEMM_SCHED
#define KSSD_GEMM_SCHED 1
#endif
using TileShape = Shape<_128, Int<KSSD_GEMM_TILE_N>, _128>;
using ClusterShape = Shape<_1, _1, _1>;
using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, TileShape, ClusterShape,
    cutlass::epilogue::collective::EpilogueTileAuto, int32_t, int32_t, int32_t, cutlass::layout::RowMajor, 4,
    int32_t, cutlass::layout::RowMajor, 4, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;
using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, int8_t, cutlass::layout::ColumnMajor, 16, int8_t,
    cutlass::layout::RowMajor, 16, int32_t, TileShape, ClusterShape,
    cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
    cutlass::gemm::KernelTmaWarpSpecialized1SmSm100>::CollectiveOp;
// stream-K scheduler: the output has few 128 x 128 tiles (n x 4n for n of hundreds to
// thousands of genomes) against a deep K, so the K loop of each tile is split across SMs
// (by stream-K, or by an even split-K for the smallest outputs: make_args)
using Kernel =
    cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, cutlass::gemm::StreamKScheduler>;
using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;

// lda / ldb: elements between consecutive k rows of A (K x M) and B (K x N); ldd:
// elements between consecutive rows of D, so that a block of a larger matrix can be
// one GEMM.
typename Gemm::Arguments make_args(const int8_t *A, const int8_t *B, int32_t *D, int M, int N, int K, int64_t lda,
                                   int64_t ldb, int64_t ldd)
{
    using SA = typename Gemm::GemmKernel::StrideA;
    using SB = typename Gemm::GemmKernel::StrideB;
    using SC = typename Gemm::GemmKernel::StrideC;
    using SD = typename Gemm::GemmKernel::StrideD;
    SA sa = cutlass::make_cute_packed_stride(SA{}, cute::make_shape(M, K, 1));
    SB sb = cutlass::make_cute_packed_stride(SB{}, cute::make_shape(N, K, 1));
    SC sc = cutlass::make_cute_packed_stride(SC{}, cute::make_shape(M, N, 1));
    SD sd = cutlass::make_cute_packed_stride(SD{}, cute::make_shape(M, N, 1));
    cute::get<1>(sa) = lda;  // A: (m, k) at m + k lda
    cute::get<1>(sb) = ldb;  // B: (n, k) at n + k ldb
    cute::get<0>(sc) = ldd;  // C (not read: beta = 0) and D: (m, n) at m ldd + n
    cute::get<0>(sd) = ldd;
    typename Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm, {M, N, K, 1}, {A, sa, B, sb},
                                  {{1, 0}, D, sc, D, sd}};
#if KSSD_GEMM_SCHED
    // Fewer output tiles than SMs (up to about 770 genomes): split K evenly over
    // floor(SMs / tiles) CTAs per tile, all resident at once, so the CTAs that share a
    // K range read the same operand slices at about the same time (L2 hits instead of
    // re-streaming); the int32 partial sums are exact in any order.  Measured on the
    // 512-genome dense join: 1.01-1.14 ms per step against 1.15-1.22 ms with stream-K.
    using Sched = typename Gemm::GemmKernel::TileSchedulerArguments;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    const int tiles = ((M + 127) / 128) * ((N + KSSD_GEMM_TILE_N - 1) / KSSD_GEMM_TILE_N);
    if (tiles < sms) {
        args.scheduler.splits = sms / tiles;
        args.scheduler.decomposition_mode = decltype(Sched::decomposition_mode)::SplitK;
        args.scheduler.reduction_mode = decltype(Sched::reduction_mode)::Nondeterministic;
    } else if (KSSD_GEMM_SCHED == 2) {
        args.scheduler.decomposition_mode = decltype(Sched::decomposition_mode)::DataParallel;
    }
#endif
    return args;
}

}  // namespace

namespace kssd {

// Bytes of device workspace the GEMM of this shape needs (0 or more).
size_t dense_gemm_s8_workspace(int M, int N, int K)
{
    return Gemm::get_workspace_size(make_args(nullptr, nullptr, nullptr, M, N, K, M, N, N));
}

// D = A^T B for A stored K x M (row stride lda) and B stored K x N (row stride ldb), D
// row-major with row stride ldd; M, N, lda, ldb multiples of 16 and every base address
// 16-byte aligned.  Returns 0, or 1 when the shape is not supported, 2 when the launch
// failed.
int dense_gemm_s8(const int8_t *A, const int8_t *B, int32_t *D, int M, int N, int K, int64_t lda, int64_t ldb,
                  int64_t ldd, void *workspace, cudaStream_t st)
{
    const auto args = make_args(A, B, D, M, N, K, lda, ldb, ldd);
    Gemm gemm;
    if (gemm.can_implement(args) != cutlass::Status::kSuccess)
        return 1;
    if (gemm.initialize(args, workspace, st) != cutlass::Status::kSuccess)
        return 2;
    if (gemm.run(st) != cutlass::Status::kSuccess)
        return 2;
    return 0;
}

}  // namespace kssd

// pbf_solver.cu — solver iterations, scatter-back, finalize and foam of the
// single-scene PBF step for sm_100a: one thread per sorted slot, the work of
// each slot in pbf_items.cuh.
//
// Replaces densityLambdaSorted (engine/shaders/Constraints.metal:82-131),
// applyDeltaSorted (:140-199), sphereCollision (:262-277),
// scatterPositionsToOriginal (:205-213), finalizeStep (:305-353) and
// computeFoam (:287-299), dispatched by engine/src/Engine.cpp:728-810.
//
//   lambda, first  sorted_a (absolute x, y, z) -> sorted_b (l, lambda), scell
//   delta          sorted_b (l, lambda) -> sorted_a (l')
//   lambda         sorted_a (l) -> sorted_b (l, lambda)
//   last delta     also scatter-back + finalize + foam into original order.
#include "pbf_items.cuh"

namespace mpb {
namespace {

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// Launch shape of the solver kernels, measured on the 1M-particle dam break:
// blocks of 128 threads (slightly ahead of 256 and 512), and a residency
// target that caps registers at 65536 / (256 * N) -- the lambda passes run
// best with N = 4 (64 registers), the middle delta passes with N = 6 (40
// registers and a small spill: 2% ahead of 48 registers, 3% ahead of 32),
// the last one, which also finalizes in FP64, with N = 6 (40 registers, a
// small spill).
#ifndef MPB_SOLVER_BLOCK
#define MPB_SOLVER_BLOCK 128
#endif
constexpr uint32_t kSB = MPB_SOLVER_BLOCK;
#ifndef MPB_LAMBDA_MIN_BLOCKS
#define MPB_LAMBDA_MIN_BLOCKS 4
#endif
#ifndef MPB_DELTA_MIN_BLOCKS
#define MPB_DELTA_MIN_BLOCKS 6
#endif
#ifndef MPB_DELTA_MID_MIN_BLOCKS
#define MPB_DELTA_MID_MIN_BLOCKS 6
#endif

template <bool LAST>
__global__ void __launch_bounds__(kSB, MPB_LAMBDA_MIN_BLOCKS * 256 / kSB)
k_lambda_first(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
               uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
               const uint32_t* __restrict__ sidx, float* __restrict__ lambdas,
               uint32_t* __restrict__ ncount, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < c.n) lambda_first_item<LAST>(c, s, cur, nxt, scell, cstart, sidx, lambdas, ncount, rm);
}

template <bool LAST>
__global__ void __launch_bounds__(kSB, MPB_LAMBDA_MIN_BLOCKS * 256 / kSB)
k_lambda(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
         const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
         const uint32_t* __restrict__ sidx, float* __restrict__ lambdas, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < c.n) lambda_item<LAST>(c, s, cur, nxt, scell, cstart, sidx, lambdas, rm);
}

// SN = 4: the reference's s_corr exponent, fixed at compile time (the host
// launches this instance when scorr_n == 4); SN = 0 reads it from c.
template <bool LAST, uint32_t SN>
__global__ void __launch_bounds__(kSB, (LAST ? MPB_DELTA_MIN_BLOCKS : MPB_DELTA_MID_MIN_BLOCKS) * 256 / kSB)
k_delta(StepConsts c, const float4* __restrict__ src, float4* __restrict__ dst,
        const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
        const uint32_t* __restrict__ sidx, const SphereState* __restrict__ sphere,
        float4* __restrict__ pos, float4* __restrict__ vel, const float4* __restrict__ prev,
        const uint32_t* __restrict__ ncount, float* __restrict__ foam, uint32_t* err, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < c.n)
        delta_item<LAST, SN>(c, s, src, dst, scell, cstart, sidx, sphere, pos, vel, prev, ncount, foam,
                             err, rm, nullptr);
}

template <bool LAST>
void launch_delta(const StepConsts& c, const DevState& d, const RowMasks& rm, cudaStream_t s) {
    const dim3 grid(cdiv(c.n, kSB));
    if (c.scorr_n == 4)
        k_delta<LAST, 4><<<grid, kSB, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx, d.sphere,
                                              d.pos, d.vel, d.prev, d.ncount, d.foam, d.err, rm);
    else
        k_delta<LAST, 0><<<grid, kSB, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx, d.sphere,
                                              d.pos, d.vel, d.prev, d.ncount, d.foam, d.err, rm);
}

__global__ void __launch_bounds__(256)
k_finalize_sorted(StepConsts c, const float4* __restrict__ sorted,
                  const uint32_t* __restrict__ sidx, float4* __restrict__ pos,
                  float4* __restrict__ vel, const float4* __restrict__ prev,
                  const uint32_t* __restrict__ ncount, float* __restrict__ foam, uint32_t* err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < c.n) finalize_sorted_item(c, s, sorted, sidx, pos, vel, prev, ncount, foam, err);
}

}  // namespace

cudaError_t launch_solver(const StepConsts& c, const DevState& d, uint32_t iterations,
                          cudaStream_t s, KernelTimer* t) {
    const uint32_t n = c.n;
    if (n == 0) return cudaSuccess;
    const uint32_t grid = cdiv(n, 256);
    if (iterations == 0) {
        cudaError_t e = launch_count_neighbors(c, d, s, t);
        if (e != cudaSuccess) return e;
        tbegin(t, s);
        k_finalize_sorted<<<grid, 256, 0, s>>>(c, d.sorted_a, d.sidx, d.pos, d.vel, d.prev, d.ncount,
                                               d.foam, d.err);
        tend(t, "finalize", s);
        return cudaGetLastError();
    }
    const RowMasks rm{d.row_masks, d.mask_overflow, d.mask_stride};  // 9 x u32 per slot
    for (uint32_t it = 0; it < iterations; ++it) {
        const bool first = it == 0, last = it + 1 == iterations;
        tbegin(t, s);
        if (first && last)
            k_lambda_first<true><<<cdiv(n, kSB), kSB, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                      d.sidx, d.lambdas, d.ncount, rm);
        else if (first)
            k_lambda_first<false><<<cdiv(n, kSB), kSB, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                       d.sidx, d.lambdas, d.ncount, rm);
        else if (last)
            k_lambda<true><<<cdiv(n, kSB), kSB, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                d.lambdas, rm);
        else
            k_lambda<false><<<cdiv(n, kSB), kSB, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                 d.lambdas, rm);
        tend(t, first ? "lambda_count" : "lambda", s);
        tbegin(t, s);
        if (last)
            launch_delta<true>(c, d, rm, s);
        else
            launch_delta<false>(c, d, rm, s);
        tend(t, last ? "delta_finalize" : "delta", s);
    }
    return cudaGetLastError();
}

uint32_t step_launch_count(uint32_t iterations) {
    // predict+hash, scan, scatter, sort+gather, long segments, then 2 per
    // iteration (or count + finalize for zero iterations).
    return 5u + (iterations ? 2u * iterations : 2u);
}

}  // namespace mpb

// pbf_batch.cu — many independent scenes of uneven particle counts advanced by
// one persistent, cooperative launch per step (no reference counterpart: the
// reference runs one scene per Engine).
//
// Every scene keeps its own parameters (dt, epsilon, box, ...) and its own
// hash grid.  To keep the cell arrays proportional to the particles instead of
// to (scenes x box volume), each step stores only the bounding box of the
// scene's predicted cells: the same dense cell coordinates as a single-scene
// engine, the same x-fastest order inside the box, so a scene's sorted order,
// neighbour sets and arithmetic are exactly those of a single-scene step.
// Scenes' particles and slots are contiguous ranges of the global arrays, and
// each scene's boxes are laid end to end in the global cell arrays.
//
// Phases of one step, separated by a grid-wide barrier (bounded spin: a
// block that gives up sets MP_DEVERR_SPIN_LIMIT and an abort flag, and every
// block leaves the launch at its next barrier, so no phase ever runs on the
// incomplete output of an earlier one):
//   0  per scene: reset the bounding box, advance the sphere
//   1  per particle: predict, dense cell -> scene bounding box (atomics,
//      reduced per warp first)
//   2  one block: per-scene sub-grid dims and cell offsets (exclusive scan)
//   3  per particle: cell id in the scene's box, warp-aggregated count
//   4  exclusive scan of the counts (tile sums, scan of the sums, tile scan)
//   5  scatter, 6 stable re-rank + gather, 7 long segments
//   8+ K x (lambda, delta); the last delta finalizes.
// The per-particle work is the single-scene engine's (pbf_items.cuh).  The
// serial mode launches this same kernel once per scene.
#include <cooperative_groups.h>

#include "pbf_batch.h"
#include "pbf_items.cuh"

namespace mpb {
namespace {

constexpr uint32_t kScanItems = 8;  // per thread and tile in phase 4

// Grid-wide barrier with a generation counter.  Every block calls it the same
// number of times.  The wait is bounded: a block that waits more than
// a.spin_limit polls sets the error bit and the abort flag.  Returns false
// (to every thread of the block) when the launch is aborted, by this block or
// another one; the block must then return.  A barrier only completes once
// every block has arrived, i.e. finished the phase before it, so a block that
// returns true works on complete data; a block that left early never
// arrives at the next barrier, so nobody passes that one.
__device__ __forceinline__ bool grid_barrier(const BatchArgs& a, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = a.bar_gen;
        volatile uint32_t* vabort = a.abort;
        const unsigned g = *vgen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(a.bar_count, 1u) + 1u == gridDim.x + a.bar_extra) {
            atomicExch(a.bar_count, 0u);
            __threadfence();
            atomicAdd(a.bar_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*vgen == g) {
                if (*vabort) {
                    ok = 0;
                    break;
                }
                if (++spins > a.spin_limit) {
                    atomicOr(a.err, kDevErrSpin);
                    atomicExch(a.abort, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (ok && *vabort) ok = 0;
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

template <uint32_t BS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= uint32_t(o)) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < BS / 32 ? s_warp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, wi, o);
            if (lane >= uint32_t(o)) wi += y;
        }
        if (lane < BS / 32) s_warp[lane] = wi - w;
        if (lane == BS / 32 - 1) s_warp[BS / 32] = wi;
    }
    __syncthreads();
    const uint32_t r = s_warp[warp] + incl - v;
    total = s_warp[BS / 32];
    __syncthreads();
    return r;
}

// Resident blocks of BS threads per SM the step kernel is compiled for: its
// registers are capped at 64 per thread (left alone, the compiler takes ~108
// for the inlined phases and fits a single 512-thread block per SM; at 64 the
// ensemble step is ~25% faster despite a small spill).
template <uint32_t BS>
constexpr int batch_min_blocks() {
    return int(65536u / (BS * 64u));
}

// SN: the s_corr exponent fixed at compile time (4, when every scene uses
// the reference's) or read per scene (0); both give the same bits for 4.
template <uint32_t BS, uint32_t SN>
__global__ void __launch_bounds__(BS, batch_min_blocks<BS>()) k_batch_step(BatchArgs a) {
    __shared__ uint32_t s_warp[BS / 32 + 1];
    __shared__ int s_ok;
    const uint32_t gtid = blockIdx.x * BS + threadIdx.x;
    // an earlier launch gave up on a barrier and left the barrier counter
    // mid-count: do nothing until the host has re-armed the batch
    if (*static_cast<volatile uint32_t*>(a.abort)) {
        if (gtid == 0) atomicOr(a.err, kDevErrSpin);
        return;
    }
    const uint32_t gsize = gridDim.x * BS;
    const uint32_t pb = a.p_begin, pe = a.p_end;
    // loops over particles run in whole warps (warp-level operations inside)
    const uint32_t pe_round = pb + ((pe - pb + 31u) & ~31u);
    SceneDev* sc = a.scenes;

    // 0: reset bounding boxes, advance spheres, clear the long-segment queue
    for (uint32_t s = a.scene_begin + gtid; s < a.scene_end; s += gsize) {
        sc[s].bb[0] = sc[s].bb[1] = sc[s].bb[2] = 0xffffffffu;
        sc[s].bb[3] = sc[s].bb[4] = sc[s].bb[5] = 0u;
        if (a.rec.sphere0) a.rec.sphere0[s] = sc[s].sphere;
        if (sc[s].c.sphere) sphere_advance(sc[s].c, &sc[s].sphere);
    }
    if (gtid == 0) *a.long_count = 0;
    if (!grid_barrier(a, &s_ok)) return;

    // 1: predict + dense cell of the predicted position -> scene bounding box
    for (uint32_t i = pb + gtid; i < pe_round; i += gsize) {
        const bool active = i < pe;
        uint32_t scene = 0xffffffffu, dx = 0, dy = 0, dz = 0;
        if (active) {
            scene = a.scene_of[i];
            const StepConsts& c = sc[scene].c;
            const float4 p = predict_item(c, i, a.pos, a.vel, a.prev, a.err);
            dx = uint32_t(cell_axis(p.x, c.g.ox, c.g.inv, c.g.dgx));
            dy = uint32_t(cell_axis(p.y, c.g.oy, c.g.inv, c.g.dgy));
            dz = uint32_t(cell_axis(p.z, c.g.oz, c.g.inv, c.g.dgz));
        }
        const unsigned act = __ballot_sync(kFull, active);
        if (active) {
            const unsigned peers = __match_any_sync(act, scene);
            const uint32_t mnx = __reduce_min_sync(peers, dx), mxx = __reduce_max_sync(peers, dx);
            const uint32_t mny = __reduce_min_sync(peers, dy), mxy = __reduce_max_sync(peers, dy);
            const uint32_t mnz = __reduce_min_sync(peers, dz), mxz = __reduce_max_sync(peers, dz);
            if (int(threadIdx.x & 31) == __ffs(peers) - 1) {
                uint32_t* bb = sc[scene].bb;
                atomicMin(&bb[0], mnx);
                atomicMin(&bb[1], mny);
                atomicMin(&bb[2], mnz);
                atomicMax(&bb[3], mxx);
                atomicMax(&bb[4], mxy);
                atomicMax(&bb[5], mxz);
            }
        }
    }
    if (!grid_barrier(a, &s_ok)) return;

    // 2: sub-grid of every scene and its offset in the cell arrays
    if (blockIdx.x == 0) {
        uint32_t running = 0;
        for (uint32_t s0 = a.scene_begin; s0 < a.scene_end; s0 += BS) {
            const uint32_t s = s0 + threadIdx.x;
            uint32_t cells = 0;
            if (s < a.scene_end) {
                const uint32_t* bb = sc[s].bb;
                GridDev& g = sc[s].c.g;
                if (bb[0] <= bb[3]) {
                    g.lx = int(bb[0]);
                    g.ly = int(bb[1]);
                    g.lz = int(bb[2]);
                    g.gx = int(bb[3] - bb[0]) + 1;
                    g.gy = int(bb[4] - bb[1]) + 1;
                    g.gz = int(bb[5] - bb[2]) + 1;
                } else {  // no particles
                    g.lx = g.ly = g.lz = 0;
                    g.gx = g.gy = g.gz = 0;
                }
                cells = uint32_t(g.gx) * uint32_t(g.gy) * uint32_t(g.gz);
                g.cells = cells;
            }
            uint32_t total = 0;
            const uint32_t excl = block_exclusive_scan<BS>(cells, s_warp, total);
            if (s < a.scene_end) sc[s].c.g.cell0 = running + excl;
            running += total;
        }
        if (threadIdx.x == 0) *a.total_cells = running;
    }
    if (!grid_barrier(a, &s_ok)) return;

    // 3: cell id inside the scene's box + warp-aggregated count
    if (a.rec.scenes)
        for (uint32_t s = a.scene_begin + gtid; s < a.scene_end; s += gsize) a.rec.scenes[s] = sc[s];
    const uint32_t ncells = *a.total_cells;
    if (ncells > a.max_cells && gtid == 0) atomicOr(a.err, kDevErrIndex);
    const bool cells_ok = ncells <= a.max_cells;
    for (uint32_t i = pb + gtid; i < pe_round; i += gsize) {
        const bool active = i < pe && cells_ok;
        uint32_t cell = 0;
        if (active) {
            const StepConsts& c = sc[a.scene_of[i]].c;
            const float4 p = a.pos[i];
            int cx, cy, cz;
            cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
            cell = cell_hash(c.g, cx, cy, cz);
            a.hash[i] = cell;
        }
        uint32_t rank = 0;
        count_cell(active, cell, a.counts, &rank);
        if (active) a.off[i] = rank;
    }
    if (!grid_barrier(a, &s_ok)) return;

    // 4: exclusive scan of counts[0, ncells] into cstart (counts left zero)
    const uint32_t len = cells_ok ? ncells + 1u : 0u;
    const uint32_t tile = BS * kScanItems;
    const uint32_t tiles = (len + tile - 1) / tile;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        uint32_t sum = 0;
        for (uint32_t k = 0; k < kScanItems; ++k) {
            const uint32_t idx = t * tile + k * BS + threadIdx.x;
            if (idx < len) sum += a.counts[idx];
        }
        uint32_t total = 0;
        block_exclusive_scan<BS>(sum, s_warp, total);
        if (threadIdx.x == 0) a.tile_sums[t] = total;
    }
    if (!grid_barrier(a, &s_ok)) return;
    if (blockIdx.x == 0) {
        // slots of this launch start at its first particle (a scene's range
        // in serial mode)
        uint32_t running = pb;
        for (uint32_t t0 = 0; t0 < tiles; t0 += BS) {
            const uint32_t t = t0 + threadIdx.x;
            const uint32_t v = t < tiles ? a.tile_sums[t] : 0u;
            uint32_t total = 0;
            const uint32_t excl = block_exclusive_scan<BS>(v, s_warp, total);
            if (t < tiles) a.tile_sums[t] = running + excl;
            running += total;
        }
    }
    if (!grid_barrier(a, &s_ok)) return;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        // each thread owns kScanItems consecutive items of the tile
        uint32_t v[kScanItems], sum = 0;
        const uint32_t first = t * tile + threadIdx.x * kScanItems;
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k) {
            v[k] = first + k < len ? a.counts[first + k] : 0u;
            sum += v[k];
        }
        uint32_t total = 0;
        uint32_t run = a.tile_sums[t] + block_exclusive_scan<BS>(sum, s_warp, total);
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k)
            if (first + k < len) {
                a.cstart[first + k] = run;
                a.counts[first + k] = 0u;
                run += v[k];
            }
    }
    if (!grid_barrier(a, &s_ok)) return;

    // 5: scatter; 6: stable re-rank + gather; 7: long segments
    if (cells_ok)
        for (uint32_t i = pb + gtid; i < pe; i += gsize) scatter_item(i, a.hash, a.off, a.cstart, a.tmp);
    if (!grid_barrier(a, &s_ok)) return;
    if (cells_ok)
        for (uint32_t s = pb + gtid; s < pe; s += gsize)
            sort_gather_item(s, a.tmp, a.hash, a.cstart, a.pos, a.sidx, a.sorted_a, a.long_list,
                             a.long_count);
    if (!grid_barrier(a, &s_ok)) return;
    {
        const uint32_t nl = cells_ok ? *a.long_count : 0u;
        for (uint32_t li = blockIdx.x; li < nl; li += gridDim.x) {
            const uint32_t cell = a.long_list[li];
            const SceneDev& sd = sc[a.scene_of[a.tmp[a.cstart[cell]]]];
            long_segment(cell, sd.p0, sd.p0 + sd.c.n, a.hash, a.cstart, a.pos, a.sidx, a.sorted_a,
                         s_warp);
        }
    }
    if (!grid_barrier(a, &s_ok)) return;

    // 8+: solver
    const RowMasks rm{a.row_masks, a.mask_overflow, a.mask_stride};
    if (!cells_ok) return;  // every block takes this branch together
    if (a.iterations == 0) {
        for (uint32_t s = pb + gtid; s < pe; s += gsize)
            count_neighbors_item(sc[a.scene_of[s]].c, s, a.sorted_a, a.cstart, a.sidx, a.ncount);
        if (!grid_barrier(a, &s_ok)) return;
        for (uint32_t s = pb + gtid; s < pe; s += gsize)
            finalize_sorted_item(sc[a.scene_of[s]].c, s, a.sorted_a, a.sidx, a.pos, a.vel, a.prev,
                                 a.ncount, a.foam, a.err);
        return;
    }
    // a recorded step keeps every lambda pass's output, row masks and
    // corrections in the record instead of overwriting one buffer
    const bool record = a.rec.lam != nullptr;
    for (uint32_t it = 0; it < a.iterations; ++it) {
        const bool last = it + 1 == a.iterations;
        float4* lam_out = record ? a.rec.lam + size_t(it) * a.rec.stride : a.sorted_b;
        const RowMasks rmi =
            record ? RowMasks{a.rec.masks + size_t(it) * 9 * a.mask_stride,
                              a.rec.overflow + size_t(it) * a.mask_stride, a.mask_stride}
                   : rm;
        float4* drec = record ? a.rec.delta + size_t(it) * a.rec.stride : nullptr;
        for (uint32_t s = pb + gtid; s < pe; s += gsize) {
            const StepConsts& c = sc[a.scene_of[s]].c;
            if (it == 0) {
                if (last)
                    lambda_first_item<true>(c, s, a.sorted_a, lam_out, a.scell, a.cstart, a.sidx,
                                            a.lambdas, a.ncount, rmi);
                else
                    lambda_first_item<false>(c, s, a.sorted_a, lam_out, a.scell, a.cstart, a.sidx,
                                             a.lambdas, a.ncount, rmi);
            } else if (last) {
                lambda_item<true>(c, s, a.sorted_a, lam_out, a.scell, a.cstart, a.sidx, a.lambdas, rmi);
            } else {
                lambda_item<false>(c, s, a.sorted_a, lam_out, a.scell, a.cstart, a.sidx, a.lambdas, rmi);
            }
        }
        if (!grid_barrier(a, &s_ok)) return;
        for (uint32_t s = pb + gtid; s < pe; s += gsize) {
            const SceneDev& sd = sc[a.scene_of[s]];
            if (last)
                delta_item<true, SN>(sd.c, s, lam_out, a.sorted_a, a.scell, a.cstart, a.sidx, &sd.sphere,
                                 a.pos, a.vel, a.prev, a.ncount, a.foam, a.err, rmi, drec);
            else
                delta_item<false, SN>(sd.c, s, lam_out, a.sorted_a, a.scell, a.cstart, a.sidx, &sd.sphere,
                                  a.pos, a.vel, a.prev, a.ncount, a.foam, a.err, rmi, drec);
        }
        if (!last && !grid_barrier(a, &s_ok)) return;
    }
}

template <uint32_t BS>
cudaError_t launch_bs(const BatchArgs& args, uint32_t blocks, cudaStream_t s) {
    void* kargs[] = {const_cast<BatchArgs*>(&args)};
    const void* fn = args.scorr4 ? reinterpret_cast<const void*>(&k_batch_step<BS, 4>)
                                 : reinterpret_cast<const void*>(&k_batch_step<BS, 0>);
    return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(BS), kargs, 0, s);
}

// Blocks of both instances that fit on one SM at once (the smaller count).
template <uint32_t BS>
int occupancy_bs() {
    int n0 = 0, n4 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n0, k_batch_step<BS, 0>, BS, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n4, k_batch_step<BS, 4>, BS, 0) != cudaSuccess)
        return 0;
    return n0 < n4 ? n0 : n4;
}

}  // namespace

int batch_max_blocks_per_sm(uint32_t block) {
    switch (block) {
        case 128: return occupancy_bs<128>();
        case 256: return occupancy_bs<256>();
        case 512: return occupancy_bs<512>();
        default: return 0;
    }
}

cudaError_t launch_batch_step(const BatchArgs& args, uint32_t block, uint32_t blocks, cudaStream_t s) {
    switch (block) {
        case 128: return launch_bs<128>(args, blocks, s);
        case 256: return launch_bs<256>(args, blocks, s);
        case 512: return launch_bs<512>(args, blocks, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mpb

// pbf_hash.cu — spatial hash of the PBF step for sm_100a.
//
// Replaces the reference's hash pipeline (engine/shaders/Spatial.metal:49-243,
// dispatched by engine/src/Engine.cpp:601-679):
//   predict + hash + count  one pass; warp-aggregated atomics (__match_any_sync)
//                           hand each particle its rank among the particles of
//                           its cell that this pass saw
//   exclusive scan          single pass, decoupled look-back, warp shuffles
//                           (replaces scanChunkExclusive/scanChunkSums/
//                           addChunkOffsets and their 1024^2 cap); also zeroes
//                           the counts for the next pass
//   scatter                 slot = cellStart[c] + rank (no second atomic)
//   stable fix-up + gather  re-ranks each particle inside its cell segment by
//                           particle index, so sortedIndex is ascending within a
//                           cell (deterministic, unlike scatterParticles'
//                           atomics), and gathers the sorted positions
//   countNeighbors          only for the standalone buildSpatialHash; the step
//                           fuses the count into its first lambda pass.
#include "pbf_items.cuh"

namespace mpb {
namespace {

// predictPositions (Constraints.metal:54-66) + hashCells (Spatial.metal:49-57)
// + countCells (Spatial.metal:63-70) in one pass.
__global__ void __launch_bounds__(256)
k_predict_hash(StepConsts c, float4* __restrict__ pos, const float4* __restrict__ vel,
               float4* __restrict__ prev, uint32_t* __restrict__ hash, uint32_t* __restrict__ off,
               uint32_t* __restrict__ counts, uint32_t* __restrict__ long_count,
               SphereState* __restrict__ sphere, int predict, uint32_t* __restrict__ err) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *long_count = 0;
        if (predict && c.sphere) sphere_advance(c, sphere);
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < c.n;
    uint32_t cell = 0;
    if (active) {
        const float4 p = predict ? predict_item(c, i, pos, vel, prev, err) : pos[i];
        int cx, cy, cz;
        cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
        cell = cell_hash(c.g, cx, cy, cz);
        hash[i] = cell;
    }
    uint32_t rank = 0;
    count_cell(active, cell, counts, &rank);
    if (active) off[i] = rank;
}

// ---- single-pass exclusive scan (decoupled look-back) -----------------------
//
// Tile = 256 threads x 16 items.  Warp w owns items [w*512, w*512+512) of the
// tile as four 128-item chunks; lane l of chunk k holds items k*128 + 4l ..
// k*128 + 4l + 3, so every load/store instruction is a fully coalesced 512-B
// access.  The tile descriptor is one 64-bit word:
//   [63:33] epoch tag (1..2^31-1), [32] 1 = inclusive prefix / 0 = aggregate,
//   [31:0]  value (mod 2^32).
// Tiles take their index from a monotonic ticket, so predecessors are always
// resident or finished (no deadlock) and the epoch = ticket / tiles tells a
// current descriptor from a stale one without clearing the array.

__device__ __forceinline__ unsigned long long pack_status(uint32_t tag, uint32_t prefix,
                                                          uint32_t v) {
    return (static_cast<unsigned long long>(tag) << 33) |
           (static_cast<unsigned long long>(prefix) << 32) | v;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

template <bool VEC>
__device__ __forceinline__ void load4(const uint32_t* in, uint32_t idx, uint32_t n, uint32_t v[4]) {
    if (VEC && idx + 3 < n) {
        const uint4 q = *reinterpret_cast<const uint4*>(in + idx);
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) v[e] = (idx + e < n) ? in[idx + e] : 0u;
    }
}

template <bool VEC>
__device__ __forceinline__ void store4(uint32_t* out, uint32_t idx, uint32_t n, const uint32_t v[4]) {
    if (VEC && idx + 3 < n) {
        *reinterpret_cast<uint4*>(out + idx) = make_uint4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (idx + e < n) out[idx + e] = v[e];
    }
}

template <bool VEC>
__global__ void __launch_bounds__(kScanThreads)
k_scan(const uint32_t* in, uint32_t* out, uint32_t n, unsigned long long* status,
       unsigned long long* ticket, uint32_t tiles, int zero_input, uint32_t* err, uint32_t spin_limit) {
    constexpr uint32_t kScanWarps = kScanThreads / 32;
    __shared__ uint32_t s_tile, s_tag, s_warp[kScanWarps], s_agg, s_fail;
    __shared__ uint32_t s_has[kScanWarps], s_sum[kScanWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        const unsigned long long t = atomicAdd(ticket, 1ull);
        s_tile = uint32_t(t % tiles);
        s_tag = uint32_t((t / tiles) % 0x7fffffffull) + 1u;
    }
    __syncthreads();
    const uint32_t tile = s_tile, tag = s_tag;
    const uint32_t wbase = tile * kScanTile + warp * 512u;

    uint32_t v[4][4], pre[4];
    // all four loads in flight before the first shuffle
#pragma unroll
    for (int k = 0; k < 4; ++k) load4<VEC>(in, wbase + k * 128u + lane * 4u, n, v[k]);
    uint32_t running = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t t = v[k][0] + v[k][1] + v[k][2] + v[k][3];
        uint32_t incl = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        pre[k] = running + incl - t;
        running += __shfl_sync(kFull, incl, 31);
    }
    if (zero_input) {
        const uint32_t z[4] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 4; ++k) store4<VEC>(const_cast<uint32_t*>(in), wbase + k * 128u + lane * 4u, n, z);
    }
    if (lane == 0) s_warp[warp] = running;
    __syncthreads();

    if (warp == 0) {
        // Block-level scan of the 8 warp totals; publish the tile aggregate
        // (tile 0: its inclusive prefix).
        const uint32_t wt = lane < kScanWarps ? s_warp[lane] : 0u;
        uint32_t wincl = wt;
#pragma unroll
        for (int o = 1; o < int(kScanWarps); o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, wincl, o);
            if (lane >= uint32_t(o)) wincl += y;
        }
        const uint32_t agg = __shfl_sync(kFull, wincl, kScanWarps - 1);
        if (lane < kScanWarps) s_warp[lane] = wincl - wt;
        if (lane == 0) {
            s_agg = agg;
            s_fail = 0;
            *(volatile unsigned long long*)&status[tile] = pack_status(tag, tile == 0 ? 1u : 0u, agg);
        }
    }
    __syncthreads();

    // Look-back by all warps at once: warp w polls the 32 descriptors
    // [base - 32w - 31, base - 32w] until each holds at least an aggregate of
    // this epoch; the nearest inclusive prefix among the 256 ends the walk,
    // else their aggregates are summed and the next 256 follow.  A window
    // that stays stale past the spin limit flags the error word and ends the
    // walk with the prefix summed so far.
    uint32_t excl = 0;
    if (tile > 0) {
        int base = int(tile) - 1;
        uint32_t spins = 0;
        bool done = false;
        while (!done) {
            const int idx = base - int(warp * 32u + lane);
            unsigned long long w;
            bool valid;
            while (true) {
                w = idx >= 0 ? *(volatile unsigned long long*)&status[idx] : pack_status(tag, 1u, 0u);
                valid = uint32_t(w >> 33) == tag;
                if (__all_sync(kFull, valid)) break;
                if (++spins > spin_limit) break;
                __nanosleep(32);
            }
            const bool ok = __all_sync(kFull, valid);
            const unsigned incl = __ballot_sync(kFull, ((w >> 32) & 1ull) != 0ull);
            const uint32_t val = uint32_t(w);
            const int first = incl ? __ffs(incl) - 1 : 32;
            const uint32_t nearest = warp_sum(int(lane) <= first ? val : 0u);
            if (lane == 0) {
                if (!ok) {
                    atomicOr(err, kDevErrSpin);
                    s_fail = 1;
                }
                s_has[warp] = incl != 0u;
                s_sum[warp] = nearest;
            }
            __syncthreads();
            if (s_fail) {
                done = true;
            } else {
                uint32_t acc = 0;
                for (uint32_t q = 0; q < kScanWarps && !done; ++q) {
                    acc += s_sum[q];
                    done = s_has[q] != 0u;
                }
                excl += acc;
                base -= int(kScanThreads);
                done = done || base < 0;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) *(volatile unsigned long long*)&status[tile] = pack_status(tag, 1u, excl + s_agg);
    }

    const uint32_t tile_excl = excl + s_warp[warp];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t o[4];
        uint32_t r = tile_excl + pre[k];
        o[0] = r;
        r += v[k][0];
        o[1] = r;
        r += v[k][1];
        o[2] = r;
        r += v[k][2];
        o[3] = r;
        store4<VEC>(out, wbase + k * 128u + lane * 4u, n, o);
    }
}

__global__ void __launch_bounds__(256)
k_scatter(uint32_t n, const uint32_t* __restrict__ hash, const uint32_t* __restrict__ off,
          const uint32_t* __restrict__ cstart, uint32_t* __restrict__ tmp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) scatter_item(i, hash, off, cstart, tmp);
}

__global__ void __launch_bounds__(256)
k_sort_gather(uint32_t n, const uint32_t* __restrict__ tmp, const uint32_t* __restrict__ hash,
              const uint32_t* __restrict__ cstart, const float4* __restrict__ pos,
              uint32_t* __restrict__ sidx, float4* __restrict__ sorted,
              uint32_t* __restrict__ long_list, uint32_t* __restrict__ long_count) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) sort_gather_item(s, tmp, hash, cstart, pos, sidx, sorted, long_list, long_count);
}

// One block per queued long segment.
__global__ void __launch_bounds__(256)
k_long_segments(uint32_t n, const uint32_t* __restrict__ hash, const uint32_t* __restrict__ cstart,
                const float4* __restrict__ pos, uint32_t* __restrict__ sidx,
                float4* __restrict__ sorted, const uint32_t* __restrict__ long_list,
                const uint32_t* __restrict__ long_count) {
    __shared__ uint32_t s_warp[8];
    const uint32_t total = *long_count;
    for (uint32_t li = blockIdx.x; li < total; li += gridDim.x)
        long_segment(long_list[li], 0u, n, hash, cstart, pos, sidx, sorted, s_warp);
}

__global__ void __launch_bounds__(256)
k_count_neighbors(StepConsts c, const float4* __restrict__ sorted,
                  const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ sidx,
                  uint32_t* __restrict__ ncount) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < c.n) count_neighbors_item(c, s, sorted, cstart, sidx, ncount);
}

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace

cudaError_t launch_scan(const uint32_t* in, uint32_t* out, uint32_t n, unsigned long long* status,
                        unsigned long long* ticket, uint32_t tiles, bool zero_input, uint32_t* err,
                        cudaStream_t s, KernelTimer* t) {
    if (n == 0) return cudaSuccess;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
    const uint32_t spins = scan_spin_limit();
    tbegin(t, s);
    if (vec)
        k_scan<true><<<tiles, kScanThreads, 0, s>>>(in, out, n, status, ticket, tiles, zero_input, err, spins);
    else
        k_scan<false><<<tiles, kScanThreads, 0, s>>>(in, out, n, status, ticket, tiles, zero_input, err, spins);
    tend(t, "scan", s);
    return cudaGetLastError();
}

cudaError_t launch_hash_pass(const StepConsts& c, const DevState& d, bool predict, cudaStream_t s,
                             KernelTimer* t) {
    const uint32_t n = c.n;
    tbegin(t, s);
    k_predict_hash<<<n ? cdiv(n, 256) : 1, 256, 0, s>>>(c, d.pos, d.vel, d.prev, d.hash, d.off,
                                                        d.counts, d.long_count, d.sphere,
                                                        predict ? 1 : 0, d.err);
    tend(t, predict ? "predict_hash" : "hash", s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_scan(d.counts, d.cstart, c.g.cells + 1, d.scan_status, d.scan_ticket, d.scan_tiles,
                    true, d.err, s, t);
    if (e != cudaSuccess || n == 0) return e;
    tbegin(t, s);
    k_scatter<<<cdiv(n, 256), 256, 0, s>>>(n, d.hash, d.off, d.cstart, d.tmp);
    tend(t, "scatter", s);
    tbegin(t, s);
    k_sort_gather<<<cdiv(n, 256), 256, 0, s>>>(n, d.tmp, d.hash, d.cstart, d.pos, d.sidx,
                                                d.sorted_a, d.long_list, d.long_count);
    tend(t, "sort_gather", s);
    tbegin(t, s);
    k_long_segments<<<148, 256, 0, s>>>(n, d.hash, d.cstart, d.pos, d.sidx, d.sorted_a,
                                        d.long_list, d.long_count);
    tend(t, "long_segments", s);
    return cudaGetLastError();
}

cudaError_t launch_count_neighbors(const StepConsts& c, const DevState& d, cudaStream_t s,
                                   KernelTimer* t) {
    if (c.n == 0) return cudaSuccess;
    tbegin(t, s);
    k_count_neighbors<<<cdiv(c.n, 256), 256, 0, s>>>(c, d.sorted_a, d.cstart, d.sidx, d.ncount);
    tend(t, "count_neighbors", s);
    return cudaGetLastError();
}

}  // namespace mpb

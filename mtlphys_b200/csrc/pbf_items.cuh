// pbf_items.cuh — the per-particle and per-slot operations of the PBF step as
// device functions, shared by the single-scene kernels (pbf_hash.cu,
// pbf_solver.cu) and the persistent multi-scene kernel (pbf_batch.cu).
//
//   sphere_advance   Engine.cpp:694-707 (host-side sphere kinematics)
//   predict_item     predictPositions, Constraints.metal:54-66
//   count_cell       hashCells + countCells, Spatial.metal:49-70
//   scatter_item     scatterParticles, Spatial.metal:169-180 (rank from the count)
//   sort_gather_item stable order + gatherPositions, Spatial.metal:190-198
//   long_segment     the same for cells of more than kSegMax particles
//   count_neighbors_item  countNeighbors, Spatial.metal:207-243
//   lambda_*_item    densityLambdaSorted, Constraints.metal:82-131
//   delta_item       applyDeltaSorted + sphereCollision (+ scatter-back,
//                    finalizeStep, computeFoam for the last iteration),
//                    Constraints.metal:140-213, 262-353
//
// Solver state (cell-anchored local coordinates): each particle's position is
// A(c) + l, with c its hash cell (fixed for the step), A(c) = origin +
// c * cellSize per axis in FP32 and l a small FP32 offset.  Neighbour vectors
// are ((A_i - A_cell(k)) + l_i) - l_k with A_i - A_cell(k) exact (Sterbenz:
// neighbouring anchors of one sign are within a factor of two of each other,
// except next to a zero coordinate, where the difference is off by at most
// half an ulp of 0.1 m, ~4e-9 m), so they carry ~1e-8 m of rounding instead of
// the ~5e-7 m of FP32 absolute coordinates at 4-8 m, while each candidate is
// still one 16-byte load.  Box clamps, the sphere push and finalize run in
// FP64 on A + l.  The first lambda pass runs on the absolute FP32 predicted
// positions exactly as the reference does (so the neighbour count it fuses in
// is bit-exact) and converts them to offsets, which is exact for the
// particle's own cell.
#pragma once

#include "pbf_kernels.h"

namespace mpb {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- hash ------------------------------------------------------------------

// Sphere kinematics (Engine.cpp:694-707), in FP32 with one rounding per
// operation, run by one thread before the hash.
__device__ inline void sphere_advance(const StepConsts& c, SphereState* s) {
    float vx = s->v[0], vy = s->v[1], vz = s->v[2];
    vy = __fadd_rn(vy, __fmul_rn(c.sph_gravity, c.dt));
    vx = __fmul_rn(vx, c.sph_drag);
    vy = __fmul_rn(vy, c.sph_drag);
    vz = __fmul_rn(vz, c.sph_drag);
    float p[3] = {__fadd_rn(s->c[0], __fmul_rn(vx, c.dt)), __fadd_rn(s->c[1], __fmul_rn(vy, c.dt)),
                  __fadd_rn(s->c[2], __fmul_rn(vz, c.dt))};
    float v[3] = {vx, vy, vz};
    const float lo[3] = {c.bminx, c.bminy, c.bminz};
    const float hi[3] = {c.bmaxx, c.bmaxy, c.bmaxz};
    const float r = s->r;
    for (int a = 0; a < 3; ++a) {
        if (__fsub_rn(p[a], r) < lo[a]) {
            p[a] = __fadd_rn(lo[a], r);
            v[a] = __fmul_rn(-v[a], c.sph_rest);
        }
        if (__fadd_rn(p[a], r) > hi[a]) {
            p[a] = __fsub_rn(hi[a], r);
            v[a] = __fmul_rn(-v[a], c.sph_rest);
        }
    }
    for (int a = 0; a < 3; ++a) {
        s->c[a] = p[a];
        s->v[a] = v[a];
    }
}

// prev = p; v' = v + g dt; p' = p + v' dt (each one fused multiply-add);
// writes p' over pos[i] and returns it.  A non-finite input would survive as
// a finite clamped position (the reference's clamp semantics), so it is
// flagged here, on entry.
__device__ __forceinline__ float4 predict_item(const StepConsts& c, uint32_t i,
                                               float4* __restrict__ pos,
                                               const float4* __restrict__ vel,
                                               float4* __restrict__ prev, uint32_t* err) {
    float4 p = pos[i];
    const float4 v = vel[i];
    if (!isfinite(p.x + p.y + p.z + v.x + v.y + v.z)) atomicOr(err, kDevErrNaN);
    prev[i] = p;
    const float vx = __fmaf_rn(c.gravx, c.dt, v.x);
    const float vy = __fmaf_rn(c.gravy, c.dt, v.y);
    const float vz = __fmaf_rn(c.gravz, c.dt, v.z);
    p.x = __fmaf_rn(vx, c.dt, p.x);
    p.y = __fmaf_rn(vy, c.dt, p.y);
    p.z = __fmaf_rn(vz, c.dt, p.z);
    pos[i] = p;
    return p;
}

// Warp-aggregated count: every lane of the warp calls it (active or not);
// each active lane gets its rank among the particles of cell `cell` counted
// so far, in *rank.  One atomic per distinct cell in the warp.
__device__ __forceinline__ void count_cell(bool active, uint32_t cell, uint32_t* __restrict__ counts,
                                           uint32_t* rank) {
    const unsigned act = __ballot_sync(kFull, active);
    if (active) {
        const unsigned peers = __match_any_sync(act, cell);
        const int leader = __ffs(peers) - 1;
        const int lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&counts[cell], uint32_t(__popc(peers)));
        base = __shfl_sync(act, base, leader);
        *rank = base + uint32_t(__popc(peers & lanemask_lt()));
    }
}

// scatterParticles without the second atomic: slot = cellStart + rank.
__device__ __forceinline__ void scatter_item(uint32_t i, const uint32_t* __restrict__ hash,
                                             const uint32_t* __restrict__ off,
                                             const uint32_t* __restrict__ cstart,
                                             uint32_t* __restrict__ tmp) {
    tmp[cstart[hash[i]] + off[i]] = i;
}

// Stable re-rank inside the cell segment + gatherPositions: the slot's
// particle j moves to cellStart + (number of particles of its cell with a
// smaller index).  Segments longer than kSegMax are queued instead.
__device__ __forceinline__ void sort_gather_item(uint32_t s, const uint32_t* __restrict__ tmp,
                                                 const uint32_t* __restrict__ hash,
                                                 const uint32_t* __restrict__ cstart,
                                                 const float4* __restrict__ pos,
                                                 uint32_t* __restrict__ sidx,
                                                 float4* __restrict__ sorted,
                                                 uint32_t* __restrict__ long_list,
                                                 uint32_t* __restrict__ long_count) {
    const uint32_t j = tmp[s];
    const uint32_t c = hash[j];
    const uint32_t a = cstart[c], b = cstart[c + 1];
    if (b - a > kSegMax) {
        if (s == a) long_list[atomicAdd(long_count, 1u)] = c;
        return;
    }
    uint32_t rank = 0;
    for (uint32_t k = a; k < b; ++k) rank += (tmp[k] < j) ? 1u : 0u;
    const uint32_t d = a + rank;
    sidx[d] = j;
    sorted[d] = pos[j];
}

// A long segment, by the whole block: rank(j) = number of particles j' < j of
// cell c, from a block-wide scan over the particle indices [p0, p1) that can
// hold the cell's particles.  s_warp: blockDim.x / 32 words of shared memory.
__device__ inline void long_segment(uint32_t c, uint32_t p0, uint32_t p1,
                                    const uint32_t* __restrict__ hash,
                                    const uint32_t* __restrict__ cstart,
                                    const float4* __restrict__ pos, uint32_t* __restrict__ sidx,
                                    float4* __restrict__ sorted, uint32_t* s_warp) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t a = cstart[c], len = cstart[c + 1] - a;
    uint32_t running = 0;
    for (uint32_t base = p0; base < p1 && running < len; base += blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        const bool f = j < p1 && hash[j] == c;
        const unsigned m = __ballot_sync(kFull, f);
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        uint32_t before = 0, blk = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
            if (w < warp) before += s_warp[w];
            blk += s_warp[w];
        }
        if (f) {
            const uint32_t d = a + running + before + __popc(m & lanemask_lt());
            sidx[d] = j;
            sorted[d] = pos[j];
        }
        running += blk;
        __syncthreads();
    }
}

// countNeighbors in sorted order: the 27-cell stencil is 9 contiguous slot
// ranges (x-fastest hash).
__device__ __forceinline__ void count_neighbors_item(const StepConsts& c, uint32_t s,
                                                     const float4* __restrict__ sorted,
                                                     const uint32_t* __restrict__ cstart,
                                                     const uint32_t* __restrict__ sidx,
                                                     uint32_t* __restrict__ ncount) {
    const float4 p = sorted[s];
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    uint32_t cnt = 0;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y) {
            const uint32_t a = cstart[cell_hash(c.g, x0, y, z)];
            const uint32_t b = cstart[cell_hash(c.g, x1, y, z) + 1];
            for (uint32_t k = a; k < b; ++k) {
                const float4 q = __ldg(&sorted[k]);
                const float r2 = dist2(q.x - p.x, q.y - p.y, q.z - p.z);
                cnt += (r2 < c.h2) ? 1u : 0u;
            }
        }
    // the particle itself passed its own distance test unless its position is
    // not finite
    ncount[sidx[s]] = cnt - (dist2(p.x - p.x, p.y - p.y, p.z - p.z) < c.h2 ? 1u : 0u);
}

// ---- solver ------------------------------------------------------------------

// In-range masks of one lambda pass.  For each particle and each of the 9
// stencil rows, bit i is set when candidate slot b0 + i of that row lies
// within h.  The delta pass of the same iteration sees the same positions and
// the same stencil, hence exactly the same in-range pairs, so it walks these
// bits instead of sweeping the 27 cells again.  Row-major layout (row r of
// slot s at r * stride + s): the warp's stores and loads of one row coalesce.
// A row longer than 32 candidates keeps the bits of its first 32 and sets bit
// r of overflow[s]; the delta pass distance-tests that row's remaining
// candidates again.  rows == nullptr disables the masks.
struct RowMasks {
    uint32_t* rows;
    uint32_t* overflow;
    uint32_t stride;
};

// The solver arithmetic below is written with explicit round-to-nearest
// operations (__fmaf_rn, __fmul_rn, __fadd_rn, and their FP64 forms): the
// compiler may not fuse or split them, so every kernel that inlines these
// functions (the single-scene kernels, the persistent batch kernel) rounds
// identically and gives bit-identical results.

// densityLambdaSorted's sums for one particle (Constraints.metal:99-121): the
// density starts at the particle's own W(0) whether or not its slot lies in
// the stencil of its current cell (a particle can drift two cells from its
// hash cell within a step), and add() takes the terms of every other
// in-range candidate at offset r, r2 = |r|^2 < h^2, in slot order.  A
// candidate at the particle's own position (r2 = 0) adds W(0) and no gradient.
struct LambdaAcc {
    float dens = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, gsq = 0.0f;
    // the particle's own W(0)
    __device__ __forceinline__ void self(const StepConsts& c) {
        dens = __fmul_rn(__fmul_rn(__fmul_rn(c.poly6, c.h2), c.h2), c.h2);
    }
    __device__ __forceinline__ void add(const StepConsts& c, float rx, float ry, float rz, float r2) {
        const float d = __fsub_rn(c.h2, r2);
        dens = __fmaf_rn(__fmul_rn(__fmul_rn(c.poly6, d), d), d, dens);
        if (r2 > 1e-12f) {
            const float rinv = rsqrtf(r2);
            const float hd = fmaxf(__fsub_rn(c.h, __fmul_rn(r2, rinv)), 0.0f);
            const float sc = __fmul_rn(__fmul_rn(__fmul_rn(-c.spiky, hd), hd), rinv);
            gx = __fmaf_rn(sc, rx, gx);
            gy = __fmaf_rn(sc, ry, gy);
            gz = __fmaf_rn(sc, rz, gz);
            gsq = __fmaf_rn(__fmul_rn(sc, sc), r2, gsq);
        }
    }
    __device__ __forceinline__ float lambda(const StepConsts& c) const {
        const float C = __fmaf_rn(dens, c.inv_rho0, -1.0f);
        const float g2 = __fmaf_rn(gz, gz, __fmaf_rn(gy, gy, __fmaf_rn(gx, gx, gsq)));
        const float denom = __fmaf_rn(__fmul_rn(c.inv_rho0, c.inv_rho0), g2, c.eps);
        return __fdiv_rn(-C, denom);
    }
};

// ratio^n of s_corr; N = 4 fixes the exponent at compile time (the
// reference's, Constraints.metal:179), N = 0 takes c.scorr_n.  Both give
// the same bits for n = 4.
template <uint32_t N>
__device__ __forceinline__ float scorr_pow(float x, uint32_t n) {
    if (N == 4u || (N == 0u && n == 4u)) {
        const float x2 = __fmul_rn(x, x);
        return __fmul_rn(x2, x2);
    }
    float r = 1.0f;
    for (uint32_t e = 0; e < n; ++e) r = __fmul_rn(r, x);
    return r;
}

// Position-correction term of one in-range candidate (Constraints.metal:
// 170-181) with the common factor -spiky / rho0 left out (delta_item
// applies c.delta_scale once to the sum):
//   (lambda_i + lambda_j - k (W / W(dq))^n) (h - r)^2 / r  r
// W / W(dq) = d^3 poly6 / W(dq) (c.scorr_pq); the sum of lambdas and s_corr is
// one fused multiply-add.
template <uint32_t N = 0>
__device__ __forceinline__ void delta_add(const StepConsts& c, float li, float lj, float rx, float ry,
                                          float rz, float r2, float& dx, float& dy, float& dz) {
    if (r2 > 1e-12f) {
        const float d = __fsub_rn(c.h2, r2);
        const float ratio = __fmul_rn(__fmul_rn(__fmul_rn(d, d), d), c.scorr_pq);
        const float rinv = rsqrtf(r2);
        const float hd = fmaxf(__fsub_rn(c.h, __fmul_rn(r2, rinv)), 0.0f);
        const float coef = __fmul_rn(__fmaf_rn(-c.scorr_k, scorr_pow<N>(ratio, c.scorr_n), __fadd_rn(li, lj)),
                                     __fmul_rn(__fmul_rn(hd, hd), rinv));
        dx = __fmaf_rn(coef, rx, dx);
        dy = __fmaf_rn(coef, ry, dy);
        dz = __fmaf_rn(coef, rz, dz);
    }
}

// Two-phase sweep of the 27-cell stencil around cell (cx, cy, cz).  Each row
// (3 consecutive cells, one contiguous slot range) is taken in chunks of 32
// candidates: phase 1 loads every candidate once, does only the distance test
// and sets a bit for each one within h; phase 2 visits just the set bits and
// calls body(k, q, rx, ry, rz, r2) with k the candidate's slot.  The in-range
// body, about an eighth of the candidates, then runs on most lanes of the warp
// instead of on the few lanes whose candidate happened to be in range.
//
// ANCHORED = false: (px, py, pz) is the absolute FP32 position and r = p - q.
// ANCHORED = true:  (px, py, pz) is the offset l from the anchor of hash cell
// (pcx, pcy, pcz); r = ((A_i - A_cell(k)) + l_i) - l_k, A_i - A_cell(k) exact.
// XW = true: each candidate carries the x anchor of its own hash cell in w
// (the delta pass's output), so its x term is (A_i - q.w) + l_i, the same
// value as the per-cell term the row would otherwise select by slot.
//
// With masks, every row of the stencil stores the bits of its first chunk (the
// particle's own bit cleared) for the delta pass, and a row longer than one
// chunk sets its bit in the overflow word.  Returns the number of in-range
// candidates, the particle itself included.
template <bool ANCHORED, bool XW = false, class Body>
__device__ __forceinline__ uint32_t sweep(const StepConsts& c, const float4* __restrict__ src,
                                          const uint32_t* __restrict__ cstart, int cx, int cy, int cz,
                                          float px, float py, float pz, int pcx, int pcy, int pcz,
                                          uint32_t s, const RowMasks* masks, Body&& body) {
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    const int nx = x1 - x0 + 1;
    uint32_t hits = 0, over = 0;
    if (nx <= 0) {  // drifted more than a cell outside a scene's sub-grid: no candidates
        if (masks) {
            for (int z = z0; z <= z1; ++z)
                for (int y = y0; y <= y1; ++y)
                    masks->rows[uint32_t((z - z0) * 3 + (y - y0)) * masks->stride + s] = 0u;
            masks->overflow[s] = 0u;
        }
        return 0;
    }
#ifndef MPB_NO_XW
    constexpr bool kXW = ANCHORED && XW;
#else
    constexpr bool kXW = false;
#endif
    float ox0 = px, ox1 = px, ox2 = px;
    float aix = 0.0f, aiy = 0.0f, aiz = 0.0f;
    if (ANCHORED) {
        aix = anchor_x(c.g, pcx);
        aiy = anchor_y(c.g, pcy);
        aiz = anchor_z(c.g, pcz);
        ox0 = __fadd_rn(__fsub_rn(aix, anchor_x(c.g, x0)), px);
        ox1 = __fadd_rn(__fsub_rn(aix, anchor_x(c.g, x0 + 1)), px);
        ox2 = __fadd_rn(__fsub_rn(aix, anchor_x(c.g, x0 + 2)), px);
    }
    for (int z = z0; z <= z1; ++z) {
        const float oz = ANCHORED ? __fadd_rn(__fsub_rn(aiz, anchor_z(c.g, z)), pz) : pz;
        for (int y = y0; y <= y1; ++y) {
            const float oy = ANCHORED ? __fadd_rn(__fsub_rn(aiy, anchor_y(c.g, y)), py) : py;
            const uint32_t base = cell_hash(c.g, x0, y, z);
            const uint32_t b0 = cstart[base], b1 = cstart[base + 1];
            const uint32_t b2 = nx > 1 ? cstart[base + 2] : b1;
            const uint32_t b3 = nx > 2 ? cstart[base + 3] : b2;
            uint32_t first = 0;  // bits of the first chunk (the whole row if b3 - b0 <= 32)
            for (uint32_t c0 = b0; c0 < b3; c0 += 32) {
                const uint32_t c1 = min(c0 + 32u, b3);
                uint32_t mask = 0;
                if (!ANCHORED) {
                    // the first pass: a running bit (measured faster here, not in
                    // the anchored passes)
                    uint32_t bit = 1u;
                    for (uint32_t k = c0; k < c1; ++k, bit <<= 1) {
                        const float4 q = __ldg(&src[k]);
                        const float r2 = dist2(__fsub_rn(px, q.x), __fsub_rn(oy, q.y), __fsub_rn(oz, q.z));
                        if (r2 < c.h2) mask |= bit;
                    }
                } else {
                    for (uint32_t k = c0; k < c1; ++k) {
                        const float4 q = __ldg(&src[k]);
                        const float ox =
                            kXW ? __fadd_rn(__fsub_rn(aix, q.w), px) : (k < b1 ? ox0 : (k < b2 ? ox1 : ox2));
                        const float r2 = dist2(__fsub_rn(ox, q.x), __fsub_rn(oy, q.y), __fsub_rn(oz, q.z));
                        mask |= uint32_t(r2 < c.h2) << (k - c0);
                    }
                }
                if (c0 == b0) first = mask;
                hits += __popc(mask);
                // the particle's own slot gets no body (its r is 0)
                if (s - c0 < 32u) mask &= ~(1u << (s - c0));
                while (mask) {
                    const uint32_t k = c0 + uint32_t(__ffs(mask) - 1);
                    mask &= mask - 1;
                    const float4 q = __ldg(&src[k]);
                    const float ox = kXW ? __fadd_rn(__fsub_rn(aix, q.w), px) : (k < b1 ? ox0 : (k < b2 ? ox1 : ox2));
                    const float rx = __fsub_rn(ox, q.x), ry = __fsub_rn(oy, q.y), rz = __fsub_rn(oz, q.z);
                    body(k, q, rx, ry, rz, dist2(rx, ry, rz));
                }
            }
            if (masks) {
                // every row of the stencil is stored, empty ones as 0; a long
                // row stores its first 32 candidates and flags the rest
                const uint32_t row = uint32_t((z - z0) * 3 + (y - y0));
                const uint32_t self = s - b0;
                masks->rows[row * masks->stride + s] = self < 32u ? (first & ~(1u << self)) : first;
                if (b3 - b0 > 32u) over |= 1u << row;
            }
        }
    }
    if (masks) masks->overflow[s] = over;
    return hits;
}

// First lambda pass: absolute FP32 predicted positions (reference arithmetic,
// so the fused neighbour count equals countNeighbors bit for bit); converts
// the state to anchored offsets for the following passes.
template <bool LAST>
__device__ __forceinline__ void lambda_first_item(const StepConsts& c, uint32_t s,
                                                  const float4* __restrict__ cur,
                                                  float4* __restrict__ nxt,
                                                  uint32_t* __restrict__ scell,
                                                  const uint32_t* __restrict__ cstart,
                                                  const uint32_t* __restrict__ sidx,
                                                  float* __restrict__ lambdas,
                                                  uint32_t* __restrict__ ncount, const RowMasks& rm) {
    const float4 p = cur[s];
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    LambdaAcc acc;
    acc.self(c);
    const uint32_t cnt = sweep<false>(c, cur, cstart, cx, cy, cz, p.x, p.y, p.z, cx, cy, cz, s,
                                      rm.rows ? &rm : nullptr,
                                      [&](uint32_t k, const float4&, float rx, float ry, float rz,
                                          float r2) {
                                          acc.add(c, rx, ry, rz, r2);
                                      });
    const float lambda = acc.lambda(c);
    // l = p - A(c): exact for the particle's own cell (Sterbenz) unless the
    // cell reaches a zero coordinate from below, where it rounds once, by at
    // most half an ulp of the cell size; so the anchored state starts equal to
    // the FP32 predicted position.
    nxt[s] = make_float4(__fsub_rn(p.x, anchor_x(c.g, cx)), __fsub_rn(p.y, anchor_y(c.g, cy)),
                         __fsub_rn(p.z, anchor_z(c.g, cz)), lambda);
    scell[s] = cell_local(c.g, cx, cy, cz);
    const uint32_t j = sidx[s];
    // the particle itself was counted iff its own distance test passed
    // (false for a non-finite position)
    const uint32_t self = dist2(p.x - p.x, p.y - p.y, p.z - p.z) < c.h2 ? 1u : 0u;
    ncount[j] = cnt - self;
    if (LAST) lambdas[j] = lambda;
}

// Later lambda passes on the anchored state: cur is the previous delta pass's
// output, (l, x anchor of the hash cell) per slot.
template <bool LAST>
__device__ __forceinline__ void lambda_item(const StepConsts& c, uint32_t s,
                                            const float4* __restrict__ cur, float4* __restrict__ nxt,
                                            const uint32_t* __restrict__ scell,
                                            const uint32_t* __restrict__ cstart,
                                            const uint32_t* __restrict__ sidx,
                                            float* __restrict__ lambdas, const RowMasks& rm) {
    const float4 l = cur[s];
    int pcx, pcy, pcz, cx, cy, cz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    cell_of(c.g, __fadd_rn(anchor_x(c.g, pcx), l.x), __fadd_rn(anchor_y(c.g, pcy), l.y),
            __fadd_rn(anchor_z(c.g, pcz), l.z), cx, cy, cz);
    LambdaAcc acc;
    acc.self(c);
    sweep<true, true>(c, cur, cstart, cx, cy, cz, l.x, l.y, l.z, pcx, pcy, pcz, s, rm.rows ? &rm : nullptr,
                      [&](uint32_t k, const float4&, float rx, float ry, float rz, float r2) {
                          acc.add(c, rx, ry, rz, r2);
                      });
    const float lambda = acc.lambda(c);
    nxt[s] = make_float4(l.x, l.y, l.z, lambda);
    if (LAST) lambdas[sidx[s]] = lambda;
}

// finalizeStep (Constraints.metal:305-353) + computeFoam (:287-299) in FP64
// for particle j at solved position X.
__device__ __forceinline__ void finalize_particle(const StepConsts& c, uint32_t j, double X, double Y,
                                                  double Z, float4* __restrict__ pos,
                                                  float4* __restrict__ vel,
                                                  const float4* __restrict__ prev,
                                                  const uint32_t* __restrict__ ncount,
                                                  float* __restrict__ foam, uint32_t* err) {
    const double bx0 = c.bminx, by0 = c.bminy, bz0 = c.bminz;
    const double bx1 = c.bmaxx, by1 = c.bmaxy, bz1 = c.bmaxz;
    X = fmin(fmax(X, bx0), bx1);
    Y = fmin(fmax(Y, by0), by1);
    Z = fmin(fmax(Z, bz0), bz1);
    const float4 pr = prev[j];
    const double k = __dmul_rn(__drcp_rn(double(c.dt)), double(c.damping));
    double vx = __dmul_rn(__dsub_rn(X, double(pr.x)), k);
    double vy = __dmul_rn(__dsub_rn(Y, double(pr.y)), k);
    double vz = __dmul_rn(__dsub_rn(Z, double(pr.z)), k);
    const double we = c.wall_eps;
    const bool xMin = X <= __dadd_rn(bx0, we), xMax = X >= __dsub_rn(bx1, we);
    const bool yMin = Y <= __dadd_rn(by0, we), yMax = Y >= __dsub_rn(by1, we);
    const bool zMin = Z <= __dadd_rn(bz0, we), zMax = Z >= __dsub_rn(bz1, we);
    if (xMin) vx = fmax(vx, 0.0);
    if (xMax) vx = fmin(vx, 0.0);
    if (yMin) vy = fmax(vy, 0.0);
    if (yMax) vy = fmin(vy, 0.0);
    if (zMin) vz = fmax(vz, 0.0);
    if (zMax) vz = fmin(vz, 0.0);
    if (yMin) {
        vx = __dmul_rn(vx, double(c.floor_fric));
        vz = __dmul_rn(vz, double(c.floor_fric));
    } else if (xMin || xMax || zMin || zMax) {
        vx = __dmul_rn(vx, double(c.wall_fric));
        vy = __dmul_rn(vy, double(c.wall_fric));
        vz = __dmul_rn(vz, double(c.wall_fric));
    }
    const double vmax = __ddiv_rn(__dmul_rn(double(c.vmax_frac), double(c.h)), double(c.dt));
    double vl = __dsqrt_rn(__fma_rn(vz, vz, __fma_rn(vy, vy, __dmul_rn(vx, vx))));
    if (vl > vmax) {
        const double f = __ddiv_rn(vmax, vl);
        vx = __dmul_rn(vx, f);
        vy = __dmul_rn(vy, f);
        vz = __dmul_rn(vz, f);
        vl = __dsqrt_rn(__fma_rn(vz, vz, __fma_rn(vy, vy, __dmul_rn(vx, vx))));
    }
    pos[j] = make_float4(float(X), float(Y), float(Z), 1.0f);
    vel[j] = make_float4(float(vx), float(vy), float(vz), 0.0f);
    const float surface = __fsub_rn(1.0f, fminf(fmaxf(__fdiv_rn(float(ncount[j]), c.foam_maxn), 0.0f), 1.0f));
    foam[j] = __fmul_rn(surface, smoothstep_f(c.foam_lo, c.foam_hi, float(vl)));
    if (!(isfinite(X + Y + Z) && isfinite(vx + vy + vz))) atomicOr(err, kDevErrNaN);
}

// The in-range pairs a lambda pass recorded in its row masks (the particle's
// own bit cleared), walked with the anchored neighbour vector of sweep<true>:
// body(k, q, rx, ry, rz, r2) for each, in sweep<true>'s order (rows in
// stencil order, slots ascending).  The candidates of a long row past its
// first 32 are distance-tested again.  (cx, cy, cz): the stencil cell of the
// particle at offset l from anchor (ax, ay, az).
template <class Body>
__device__ __forceinline__ void masked_pairs(const StepConsts& c, const float4* __restrict__ src,
                                             const uint32_t* __restrict__ cstart, const RowMasks& rm,
                                             uint32_t s, const float4& l, float ax, float ay, float az,
                                             int cx, int cy, int cz, Body&& body) {
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    const int nx = x1 - x0 + 1;
    if (nx <= 0) return;
    const uint32_t longrows = rm.overflow[s];
    const float ox0 = __fadd_rn(__fsub_rn(ax, anchor_x(c.g, x0)), l.x);
    const float ox1 = __fadd_rn(__fsub_rn(ax, anchor_x(c.g, x0 + 1)), l.x);
    const float ox2 = __fadd_rn(__fsub_rn(ax, anchor_x(c.g, x0 + 2)), l.x);
    for (int z = z0; z <= z1; ++z) {
        const float oz = __fadd_rn(__fsub_rn(az, anchor_z(c.g, z)), l.z);
        for (int y = y0; y <= y1; ++y) {
            const uint32_t row = uint32_t((z - z0) * 3 + (y - y0));
            uint32_t mask = rm.rows[row * rm.stride + s];
            const bool long_row = (longrows >> row) & 1u;
            if (mask == 0u && !long_row) continue;
            const float oy = __fadd_rn(__fsub_rn(ay, anchor_y(c.g, y)), l.y);
            const uint32_t base = cell_hash(c.g, x0, y, z);
            const uint32_t b0 = cstart[base], b1 = cstart[base + 1];
            const uint32_t b2 = nx > 1 ? cstart[base + 2] : b1;
            while (mask) {
                const uint32_t k = b0 + uint32_t(__ffs(mask) - 1);
                mask &= mask - 1;
                const float ox = k < b1 ? ox0 : (k < b2 ? ox1 : ox2);
                const float4 q = __ldg(&src[k]);
                const float rx = __fsub_rn(ox, q.x), ry = __fsub_rn(oy, q.y);
                const float rz = __fsub_rn(oz, q.z);
                body(k, q, rx, ry, rz, dist2(rx, ry, rz));
            }
            if (long_row) {
                const uint32_t b3 = nx > 2 ? cstart[base + 3] : b2;
                for (uint32_t k = b0 + 32u; k < b3; ++k) {
                    const float ox = k < b1 ? ox0 : (k < b2 ? ox1 : ox2);
                    const float4 q = __ldg(&src[k]);
                    const float rx = __fsub_rn(ox, q.x), ry = __fsub_rn(oy, q.y);
                    const float rz = __fsub_rn(oz, q.z);
                    const float r2 = dist2(rx, ry, rz);
                    if (r2 < c.h2) body(k, q, rx, ry, rz, r2);
                }
            }
        }
    }
}

// applyDeltaSorted + sphereCollision on the anchored state; the last
// iteration also scatters back, finalizes and writes foam.  drec (may be
// NULL): receives the particle's unclamped correction, for the adjoint.
// SN: the s_corr exponent when fixed at compile time (4), else 0.
template <bool LAST, uint32_t SN = 0>
__device__ __forceinline__ void delta_item(const StepConsts& c, uint32_t s,
                                           const float4* __restrict__ src, float4* __restrict__ dst,
                                           const uint32_t* __restrict__ scell,
                                           const uint32_t* __restrict__ cstart,
                                           const uint32_t* __restrict__ sidx,
                                           const SphereState* __restrict__ sphere,
                                           float4* __restrict__ pos, float4* __restrict__ vel,
                                           const float4* __restrict__ prev,
                                           const uint32_t* __restrict__ ncount,
                                           float* __restrict__ foam, uint32_t* err,
                                           const RowMasks& rm, float4* __restrict__ drec) {
    const float4 l = src[s];
    int pcx, pcy, pcz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    const float ax = anchor_x(c.g, pcx), ay = anchor_y(c.g, pcy), az = anchor_z(c.g, pcz);
    int cx, cy, cz;
    cell_of(c.g, __fadd_rn(ax, l.x), __fadd_rn(ay, l.y), __fadd_rn(az, l.z), cx, cy, cz);
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    auto body = [&](uint32_t, const float4& q, float rx, float ry, float rz, float r2) {
        delta_add<SN>(c, l.w, q.w, rx, ry, rz, r2, dx, dy, dz);
    };
#ifdef MPB_PARTICLE_OVERFLOW
    if (rm.rows != nullptr && rm.overflow[s] == 0u)
#else
    if (rm.rows != nullptr)
#endif
        masked_pairs(c, src, cstart, rm, s, l, ax, ay, az, cx, cy, cz, body);
    else
        sweep<true>(c, src, cstart, cx, cy, cz, l.x, l.y, l.z, pcx, pcy, pcz, s,
                    static_cast<const RowMasks*>(nullptr), body);
    dx = __fmul_rn(dx, c.delta_scale);
    dy = __fmul_rn(dy, c.delta_scale);
    dz = __fmul_rn(dz, c.delta_scale);
    if (drec) drec[s] = make_float4(dx, dy, dz, 0.0f);
    const float dl = __fsqrt_rn(dist2(dx, dy, dz));
    if (dl > c.max_step) {
        const float f = __fdiv_rn(c.max_step, dl);
        dx = __fmul_rn(dx, f);
        dy = __fmul_rn(dy, f);
        dz = __fmul_rn(dz, f);
    }
    // new position A + (l + delta), box clamp (and sphere push) in FP64
    double X = __dadd_rn(double(ax), double(__fadd_rn(l.x, dx)));
    double Y = __dadd_rn(double(ay), double(__fadd_rn(l.y, dy)));
    double Z = __dadd_rn(double(az), double(__fadd_rn(l.z, dz)));
    X = fmin(fmax(X, double(c.bminx)), double(c.bmaxx));
    Y = fmin(fmax(Y, double(c.bminy)), double(c.bmaxy));
    Z = fmin(fmax(Z, double(c.bminz)), double(c.bmaxz));
    if (c.sphere) {
        const double scx = sphere->c[0], scy = sphere->c[1], scz = sphere->c[2], sr = sphere->r;
        const double ex = __dsub_rn(X, scx), ey = __dsub_rn(Y, scy), ez = __dsub_rn(Z, scz);
        const double e2 = __fma_rn(ez, ez, __fma_rn(ey, ey, __dmul_rn(ex, ex)));
        if (e2 < __dmul_rn(sr, sr)) {
            const double inv = __ddiv_rn(sr, __dsqrt_rn(fmax(e2, double(1e-8f))));
            X = __fma_rn(ex, inv, scx);
            Y = __fma_rn(ey, inv, scy);
            Z = __fma_rn(ez, inv, scz);
        }
    }
    if (!LAST) {
        // w: the x anchor of the particle's hash cell, for the next lambda
        // pass's neighbour vectors
        dst[s] = make_float4(float(__dsub_rn(X, double(ax))), float(__dsub_rn(Y, double(ay))),
                             float(__dsub_rn(Z, double(az))), ax);
        return;
    }
    finalize_particle(c, sidx[s], X, Y, Z, pos, vel, prev, ncount, foam, err);
}

// Zero solver iterations: scatter-back + finalize + foam of the predicted
// positions.
__device__ __forceinline__ void finalize_sorted_item(const StepConsts& c, uint32_t s,
                                                     const float4* __restrict__ sorted,
                                                     const uint32_t* __restrict__ sidx,
                                                     float4* __restrict__ pos, float4* __restrict__ vel,
                                                     const float4* __restrict__ prev,
                                                     const uint32_t* __restrict__ ncount,
                                                     float* __restrict__ foam, uint32_t* err) {
    const float4 p = sorted[s];
    finalize_particle(c, sidx[s], p.x, p.y, p.z, pos, vel, prev, ncount, foam, err);
}

}  // namespace mpb

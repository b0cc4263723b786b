// pbf_solver.cu — solver iterations, scatter-back, finalize and foam of the
// PBF step for sm_100a.
//
// Replaces densityLambdaSorted (engine/shaders/Constraints.metal:82-131),
// applyDeltaSorted (:140-199), sphereCollision (:262-277),
// scatterPositionsToOriginal (:205-213), finalizeStep (:305-353) and
// computeFoam (:287-299), dispatched by engine/src/Engine.cpp:728-810.
//
// One thread per sorted slot.  Because the hash is x-fastest, the 27-cell
// stencil is 9 rows of 3 consecutive cells, i.e. 9 contiguous slot ranges,
// read as float4 with neighbouring threads sharing most of their ranges in L1.
//
// Solver state: cell-anchored local coordinates.  Each particle's position is
// A(c) + l, where c is its hash cell (fixed for the step), A(c) =
// origin + c * cellSize per axis in FP32, and l is a small FP32 offset
// (|l| ~ h).  Neighbour vectors are formed as (A_i - A_j + l_i) - l_j, where
// A_i - A_j is exact, so they carry ~1e-8 m of rounding instead of the
// ~5e-7 m of FP32 absolute coordinates at 4-8 m, while each candidate is still
// one 16-byte load.  Box clamps, the sphere push and finalize run in FP64 on
// A + l.  The first lambda pass works on the absolute FP32 predicted
// positions exactly as the reference does (so the neighbour count it fuses in
// is bit-exact) and converts them to the anchored form, which is exact there.
//
//   lambda, first  sorted_a (absolute x, y, z) -> sorted_b (l, lambda), scell
//   delta          sorted_b (l, lambda) -> sorted_a (l')
//   lambda         sorted_a (l) -> sorted_b (l, lambda)
//   last delta     also scatter-back + finalize + foam into original order.
// The particle itself is visited by the stencil loop: it adds W(0) to the
// density (the reference's initial value) and nothing to any gradient.
#include "pbf_kernels.h"

namespace mpb {
namespace {

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// Resident 256-thread blocks per SM the solver kernels are compiled for
// (caps registers at 65536 / (256 * N)).
#ifndef MPB_SOLVER_MIN_BLOCKS
#define MPB_SOLVER_MIN_BLOCKS 6
#endif

__device__ __forceinline__ float anchor(float o, float cs, int c) {
    return __fmaf_rn(float(c), cs, o);
}

__device__ __forceinline__ void decode_cell(const GridDev& g, uint32_t h, int& x, int& y, int& z) {
    const uint32_t gx = uint32_t(g.gx), gy = uint32_t(g.gy);
    x = int(h % gx);
    const uint32_t t = h / gx;
    y = int(t % gy);
    z = int(t / gy);
}

// In-range masks of one lambda pass.  For each particle and each of the 9
// stencil rows, bit i is set when candidate slot b0 + i of that row lies
// within h.  The delta pass of the same iteration sees the same positions and
// the same stencil, hence exactly the same in-range pairs, so it walks these
// bits instead of sweeping the 27 cells again.  Row-major layout (row r of
// slot s at r * stride + s): the warp's stores and loads of one row coalesce.
// A particle with a row longer than 32 candidates gets overflow[s] = 1 and is
// swept in full by the delta pass.  rows == nullptr disables the masks.
struct RowMasks {
    uint32_t* rows;
    uint32_t* overflow;
    uint32_t stride;
};

// Density / gradient terms of one in-range candidate at offset r, r2 = |r|^2
// < h^2 (Constraints.metal:112-118).  The particle itself (r2 = 0) adds W(0).
struct LambdaAcc {
    float dens = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, gsq = 0.0f;
    __device__ __forceinline__ void add(const StepConsts& c, float rx, float ry, float rz, float r2) {
        const float d = c.h2 - r2;
        dens += c.poly6 * d * d * d;
        if (r2 > 1e-12f) {
            const float rinv = rsqrtf(r2);
            const float hd = fmaxf(c.h - r2 * rinv, 0.0f);
            const float sc = -c.spiky * hd * hd * rinv;
            gx += sc * rx;
            gy += sc * ry;
            gz += sc * rz;
            gsq += sc * sc * r2;
        }
    }
    __device__ __forceinline__ float lambda(const StepConsts& c) const {
        const float C = dens * c.inv_rho0 - 1.0f;
        const float denom = c.inv_rho0 * c.inv_rho0 * (gx * gx + gy * gy + gz * gz + gsq) + c.eps;
        return -C / denom;
    }
};

// Position-correction term of one in-range candidate (Constraints.metal:170-181).
__device__ __forceinline__ void delta_add(const StepConsts& c, float li, float lj, float rx, float ry,
                                          float rz, float r2, float& dx, float& dy, float& dz) {
    if (r2 > 1e-12f) {
        const float d = c.h2 - r2;
        const float ratio = c.poly6 * d * d * d * c.inv_wq;
        const float scorr = -c.scorr_k * pow_n(ratio, c.scorr_n);
        const float rinv = rsqrtf(r2);
        const float hd = fmaxf(c.h - r2 * rinv, 0.0f);
        const float coef = (li + lj + scorr) * (-c.spiky * hd * hd * rinv);
        dx += coef * rx;
        dy += coef * ry;
        dz += coef * rz;
    }
}

// Two-phase sweep of the 27-cell stencil around cell (cx, cy, cz).  Each row
// (3 consecutive cells, one contiguous slot range) is taken in chunks of 32
// candidates: phase 1 loads every candidate once, does only the distance test
// and sets a bit for each one within h; phase 2 visits just the set bits and
// calls body(q, rx, ry, rz, r2).  The in-range body, about an eighth of the
// candidates, then runs on most lanes of the warp instead of on the few lanes
// whose candidate happened to be in range.
//
// ANCHORED = false: (px, py, pz) is the absolute FP32 position and r = p - q.
// ANCHORED = true:  (px, py, pz) is the offset l from the anchor of hash cell
// (pcx, pcy, pcz); r = ((A_i - A_cell(k)) + l_i) - l_k, A_i - A_cell(k) exact.
//
// With masks, a row that fits one chunk stores its bits (the particle's own
// bit cleared) for the delta pass; a longer row sets the overflow flag.
// Returns the number of in-range candidates, the particle itself included.
template <bool ANCHORED, class Body>
__device__ __forceinline__ uint32_t sweep(const StepConsts& c, const float4* __restrict__ src,
                                          const uint32_t* __restrict__ cstart, int cx, int cy, int cz,
                                          float px, float py, float pz, int pcx, int pcy, int pcz,
                                          uint32_t s, const RowMasks* masks, Body&& body) {
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    const int nx = x1 - x0 + 1;
    float ox0 = px, ox1 = px, ox2 = px;
    float aiy = 0.0f, aiz = 0.0f;
    if (ANCHORED) {
        const float aix = anchor(c.g.ox, c.g.cs, pcx);
        aiy = anchor(c.g.oy, c.g.cs, pcy);
        aiz = anchor(c.g.oz, c.g.cs, pcz);
        ox0 = (aix - anchor(c.g.ox, c.g.cs, x0)) + px;
        ox1 = (aix - anchor(c.g.ox, c.g.cs, x0 + 1)) + px;
        ox2 = (aix - anchor(c.g.ox, c.g.cs, x0 + 2)) + px;
    }
    uint32_t hits = 0, over = 0;
    for (int z = z0; z <= z1; ++z) {
        const float oz = ANCHORED ? (aiz - anchor(c.g.oz, c.g.cs, z)) + pz : pz;
        for (int y = y0; y <= y1; ++y) {
            const float oy = ANCHORED ? (aiy - anchor(c.g.oy, c.g.cs, y)) + py : py;
            const uint32_t base = cell_hash(c.g, x0, y, z);
            const uint32_t b0 = cstart[base], b1 = cstart[base + 1];
            const uint32_t b2 = nx > 1 ? cstart[base + 2] : b1;
            const uint32_t b3 = nx > 2 ? cstart[base + 3] : b2;
            uint32_t first = 0;  // bits of the first chunk (the whole row if b3 - b0 <= 32)
            for (uint32_t c0 = b0; c0 < b3; c0 += 32) {
                const uint32_t c1 = min(c0 + 32u, b3);
                uint32_t mask = 0;
                for (uint32_t k = c0; k < c1; ++k) {
                    const float ox = k < b1 ? ox0 : (k < b2 ? ox1 : ox2);
                    const float4 q = __ldg(&src[k]);
                    const float r2 = dist2(ox - q.x, oy - q.y, oz - q.z);
                    mask |= uint32_t(r2 < c.h2) << (k - c0);
                }
                if (c0 == b0) first = mask;
                hits += __popc(mask);
                while (mask) {
                    const uint32_t k = c0 + uint32_t(__ffs(mask) - 1);
                    mask &= mask - 1;
                    const float ox = k < b1 ? ox0 : (k < b2 ? ox1 : ox2);
                    const float4 q = __ldg(&src[k]);
                    const float rx = ox - q.x, ry = oy - q.y, rz = oz - q.z;
                    body(q, rx, ry, rz, dist2(rx, ry, rz));
                }
            }
            if (masks) {
                // every row of the stencil is stored, empty ones as 0
                if (b3 - b0 <= 32u) {
                    const uint32_t self = s - b0;
                    masks->rows[uint32_t((z - z0) * 3 + (y - y0)) * masks->stride + s] =
                        self < 32u ? (first & ~(1u << self)) : first;
                } else {
                    over = 1;
                }
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
__global__ void __launch_bounds__(256, MPB_SOLVER_MIN_BLOCKS)
k_lambda_first(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
               uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
               const uint32_t* __restrict__ sidx, float* __restrict__ lambdas,
               uint32_t* __restrict__ ncount, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 p = cur[s];
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    LambdaAcc acc;
    const uint32_t cnt = sweep<false>(c, cur, cstart, cx, cy, cz, p.x, p.y, p.z, cx, cy, cz, s,
                                      rm.rows ? &rm : nullptr,
                                      [&](const float4&, float rx, float ry, float rz, float r2) {
                                          acc.add(c, rx, ry, rz, r2);
                                      });
    const float lambda = acc.lambda(c);
    // l = p - A(c): exact for the particle's own cell (Sterbenz), so the
    // anchored state starts equal to the FP32 predicted position.
    nxt[s] = make_float4(p.x - anchor(c.g.ox, c.g.cs, cx), p.y - anchor(c.g.oy, c.g.cs, cy),
                         p.z - anchor(c.g.oz, c.g.cs, cz), lambda);
    scell[s] = cell_hash(c.g, cx, cy, cz);
    const uint32_t j = sidx[s];
    // the particle itself was counted iff its own distance test passed
    // (false for a non-finite position)
    const uint32_t self = dist2(p.x - p.x, p.y - p.y, p.z - p.z) < c.h2 ? 1u : 0u;
    ncount[j] = cnt - self;
    if (LAST) lambdas[j] = lambda;
}

// Later lambda passes on the anchored state.
template <bool LAST>
__global__ void __launch_bounds__(256, MPB_SOLVER_MIN_BLOCKS)
k_lambda(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
         const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
         const uint32_t* __restrict__ sidx, float* __restrict__ lambdas, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 l = cur[s];
    int pcx, pcy, pcz, cx, cy, cz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    cell_of(c.g, anchor(c.g.ox, c.g.cs, pcx) + l.x, anchor(c.g.oy, c.g.cs, pcy) + l.y,
            anchor(c.g.oz, c.g.cs, pcz) + l.z, cx, cy, cz);
    LambdaAcc acc;
    sweep<true>(c, cur, cstart, cx, cy, cz, l.x, l.y, l.z, pcx, pcy, pcz, s, rm.rows ? &rm : nullptr,
                [&](const float4&, float rx, float ry, float rz, float r2) { acc.add(c, rx, ry, rz, r2); });
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
    const double k = (1.0 / double(c.dt)) * double(c.damping);
    double vx = (X - double(pr.x)) * k, vy = (Y - double(pr.y)) * k, vz = (Z - double(pr.z)) * k;
    const double we = c.wall_eps;
    const bool xMin = X <= bx0 + we, xMax = X >= bx1 - we;
    const bool yMin = Y <= by0 + we, yMax = Y >= by1 - we;
    const bool zMin = Z <= bz0 + we, zMax = Z >= bz1 - we;
    if (xMin) vx = fmax(vx, 0.0);
    if (xMax) vx = fmin(vx, 0.0);
    if (yMin) vy = fmax(vy, 0.0);
    if (yMax) vy = fmin(vy, 0.0);
    if (zMin) vz = fmax(vz, 0.0);
    if (zMax) vz = fmin(vz, 0.0);
    if (yMin) {
        vx *= double(c.floor_fric);
        vz *= double(c.floor_fric);
    } else if (xMin || xMax || zMin || zMax) {
        vx *= double(c.wall_fric);
        vy *= double(c.wall_fric);
        vz *= double(c.wall_fric);
    }
    const double vmax = double(c.vmax_frac) * double(c.h) / double(c.dt);
    double vl = sqrt(vx * vx + vy * vy + vz * vz);
    if (vl > vmax) {
        const double f = vmax / vl;
        vx *= f;
        vy *= f;
        vz *= f;
        vl = sqrt(vx * vx + vy * vy + vz * vz);
    }
    pos[j] = make_float4(float(X), float(Y), float(Z), 1.0f);
    vel[j] = make_float4(float(vx), float(vy), float(vz), 0.0f);
    const float surface = 1.0f - fminf(fmaxf(float(ncount[j]) / c.foam_maxn, 0.0f), 1.0f);
    foam[j] = surface * smoothstep_f(c.foam_lo, c.foam_hi, float(vl));
    if (!(isfinite(X + Y + Z) && isfinite(vx + vy + vz))) atomicOr(err, kDevErrNaN);
}

template <bool LAST>
__global__ void __launch_bounds__(256, MPB_SOLVER_MIN_BLOCKS)
k_delta(StepConsts c, const float4* __restrict__ src, float4* __restrict__ dst,
        const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
        const uint32_t* __restrict__ sidx, const SphereState* __restrict__ sphere,
        float4* __restrict__ pos, float4* __restrict__ vel, const float4* __restrict__ prev,
        const uint32_t* __restrict__ ncount, float* __restrict__ foam, uint32_t* err, RowMasks rm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 l = src[s];
    int pcx, pcy, pcz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    const float ax = anchor(c.g.ox, c.g.cs, pcx), ay = anchor(c.g.oy, c.g.cs, pcy),
                az = anchor(c.g.oz, c.g.cs, pcz);
    int cx, cy, cz;
    cell_of(c.g, ax + l.x, ay + l.y, az + l.z, cx, cy, cz);
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    auto body = [&](const float4& q, float rx, float ry, float rz, float r2) {
        delta_add(c, l.w, q.w, rx, ry, rz, r2, dx, dy, dz);
    };
    if (rm.rows != nullptr && rm.overflow[s] == 0u) {
        // the lambda pass's in-range bits, row by row (rows fit one chunk)
        const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
        const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
        const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
        const int nx = x1 - x0 + 1;
        const float ox0 = (ax - anchor(c.g.ox, c.g.cs, x0)) + l.x;
        const float ox1 = (ax - anchor(c.g.ox, c.g.cs, x0 + 1)) + l.x;
        const float ox2 = (ax - anchor(c.g.ox, c.g.cs, x0 + 2)) + l.x;
        for (int z = z0; z <= z1; ++z) {
            const float oz = (az - anchor(c.g.oz, c.g.cs, z)) + l.z;
            for (int y = y0; y <= y1; ++y) {
                uint32_t mask = rm.rows[uint32_t((z - z0) * 3 + (y - y0)) * rm.stride + s];
                if (mask == 0u) continue;
                const float oy = (ay - anchor(c.g.oy, c.g.cs, y)) + l.y;
                const uint32_t base = cell_hash(c.g, x0, y, z);
                const uint32_t b0 = cstart[base], b1 = cstart[base + 1];
                const uint32_t b2 = nx > 1 ? cstart[base + 2] : b1;
                while (mask) {
                    const uint32_t k = b0 + uint32_t(__ffs(mask) - 1);
                    mask &= mask - 1;
                    const float ox = k < b1 ? ox0 : (k < b2 ? ox1 : ox2);
                    const float4 q = __ldg(&src[k]);
                    const float rx = ox - q.x, ry = oy - q.y, rz = oz - q.z;
                    body(q, rx, ry, rz, dist2(rx, ry, rz));
                }
            }
        }
    } else {
        sweep<true>(c, src, cstart, cx, cy, cz, l.x, l.y, l.z, pcx, pcy, pcz, s,
                    static_cast<const RowMasks*>(nullptr), body);
    }
    dx *= c.inv_rho0;
    dy *= c.inv_rho0;
    dz *= c.inv_rho0;
    const float dl = sqrtf(dx * dx + dy * dy + dz * dz);
    if (dl > c.max_step) {
        const float f = c.max_step / dl;
        dx *= f;
        dy *= f;
        dz *= f;
    }
    // new position A + (l + delta), box clamp (and sphere push) in FP64
    double X = double(ax) + double(l.x + dx);
    double Y = double(ay) + double(l.y + dy);
    double Z = double(az) + double(l.z + dz);
    X = fmin(fmax(X, double(c.bminx)), double(c.bmaxx));
    Y = fmin(fmax(Y, double(c.bminy)), double(c.bmaxy));
    Z = fmin(fmax(Z, double(c.bminz)), double(c.bmaxz));
    if (c.sphere) {
        const double scx = sphere->c[0], scy = sphere->c[1], scz = sphere->c[2], sr = sphere->r;
        const double ex = X - scx, ey = Y - scy, ez = Z - scz;
        const double e2 = ex * ex + ey * ey + ez * ez;
        if (e2 < sr * sr) {
            const double inv = sr / sqrt(fmax(e2, double(1e-8f)));
            X = scx + ex * inv;
            Y = scy + ey * inv;
            Z = scz + ez * inv;
        }
    }
    if (!LAST) {
        dst[s] = make_float4(float(X - double(ax)), float(Y - double(ay)), float(Z - double(az)), 0.0f);
        return;
    }
    finalize_particle(c, sidx[s], X, Y, Z, pos, vel, prev, ncount, foam, err);
}

// Zero solver iterations: scatter-back + finalize + foam of the predicted
// positions; the neighbour count comes from one counting pass.
__global__ void __launch_bounds__(256)
k_finalize_sorted(StepConsts c, const float4* __restrict__ sorted,
                  const uint32_t* __restrict__ sidx, float4* __restrict__ pos,
                  float4* __restrict__ vel, const float4* __restrict__ prev,
                  const uint32_t* __restrict__ ncount, float* __restrict__ foam, uint32_t* err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 p = sorted[s];
    finalize_particle(c, sidx[s], p.x, p.y, p.z, pos, vel, prev, ncount, foam, err);
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
            k_lambda_first<true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                      d.sidx, d.lambdas, d.ncount, rm);
        else if (first)
            k_lambda_first<false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                       d.sidx, d.lambdas, d.ncount, rm);
        else if (last)
            k_lambda<true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                d.lambdas, rm);
        else
            k_lambda<false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                 d.lambdas, rm);
        tend(t, first ? "lambda_count" : "lambda", s);
        tbegin(t, s);
        if (last)
            k_delta<true><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx,
                                               d.sphere, d.pos, d.vel, d.prev, d.ncount, d.foam, d.err, rm);
        else
            k_delta<false><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx,
                                                d.sphere, d.pos, d.vel, d.prev, d.ncount, d.foam, d.err, rm);
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

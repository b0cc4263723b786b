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

// Accumulates density, gradient sum and squared-gradient sum for one
// candidate at offset (rx, ry, rz) (Constraints.metal:112-118).
struct LambdaAcc {
    float dens = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, gsq = 0.0f;
    uint32_t cnt = 0;
    __device__ __forceinline__ void add(const StepConsts& c, float rx, float ry, float rz) {
        const float r2 = dist2(rx, ry, rz);
        if (r2 < c.h2) {
            ++cnt;
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
    }
    __device__ __forceinline__ float lambda(const StepConsts& c) const {
        const float C = dens * c.inv_rho0 - 1.0f;
        const float denom = c.inv_rho0 * c.inv_rho0 * (gx * gx + gy * gy + gz * gz + gsq) + c.eps;
        return -C / denom;
    }
};

// Position correction contribution of one candidate (Constraints.metal:170-181).
__device__ __forceinline__ void delta_add(const StepConsts& c, float li, float lj, float rx, float ry,
                                          float rz, float& dx, float& dy, float& dz) {
    const float r2 = dist2(rx, ry, rz);
    if (r2 < c.h2 && r2 > 1e-12f) {
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

// Visit every candidate of the 27-cell stencil around the cell of the
// particle at absolute FP32 position X (the current iterate), calling
// f(k, ox, oy, oz) with the particle's offset from candidate k's cell anchor:
// candidate vector r = (ox, oy, oz) - l_k.
template <class F>
__device__ __forceinline__ void for_stencil_anchored(const StepConsts& c, const uint32_t* cstart,
                                                     float Xx, float Xy, float Xz, int pcx, int pcy,
                                                     int pcz, float lx, float ly, float lz, F&& f) {
    int cx, cy, cz;
    cell_of(c.g, Xx, Xy, Xz, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    const float aix = anchor(c.g.ox, c.g.cs, pcx), aiy = anchor(c.g.oy, c.g.cs, pcy),
                aiz = anchor(c.g.oz, c.g.cs, pcz);
    // the particle's x offset from the anchors of the (up to) three x cells
    const int nx = x1 - x0 + 1;
    const float ox0 = (aix - anchor(c.g.ox, c.g.cs, x0)) + lx;
    const float ox1 = (aix - anchor(c.g.ox, c.g.cs, x0 + 1)) + lx;
    const float ox2 = (aix - anchor(c.g.ox, c.g.cs, x0 + 2)) + lx;
    for (int z = z0; z <= z1; ++z) {
        const float oz = (aiz - anchor(c.g.oz, c.g.cs, z)) + lz;
        for (int y = y0; y <= y1; ++y) {
            const float oy = (aiy - anchor(c.g.oy, c.g.cs, y)) + ly;
            // all cell boundaries of the row up front (independent loads)
            const uint32_t base = cell_hash(c.g, x0, y, z);
            const uint32_t b0 = cstart[base], b1 = cstart[base + 1];
            const uint32_t b2 = nx > 1 ? cstart[base + 2] : b1;
            const uint32_t b3 = nx > 2 ? cstart[base + 3] : b2;
            for (uint32_t k = b0; k < b1; ++k) f(k, ox0, oy, oz);
            for (uint32_t k = b1; k < b2; ++k) f(k, ox1, oy, oz);
            for (uint32_t k = b2; k < b3; ++k) f(k, ox2, oy, oz);
        }
    }
}

// First lambda pass: absolute FP32 predicted positions (reference arithmetic,
// so the fused neighbour count equals countNeighbors bit for bit); converts
// the state to anchored offsets for the following passes.
template <bool LAST>
__global__ void __launch_bounds__(256)
k_lambda_first(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
               uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
               const uint32_t* __restrict__ sidx, float* __restrict__ lambdas,
               uint32_t* __restrict__ ncount) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 p = cur[s];
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);
    LambdaAcc acc;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y) {
            const uint32_t a = cstart[cell_hash(c.g, x0, y, z)];
            const uint32_t b = cstart[cell_hash(c.g, x1, y, z) + 1];
            for (uint32_t k = a; k < b; ++k) {
                const float4 q = __ldg(&cur[k]);
                acc.add(c, p.x - q.x, p.y - q.y, p.z - q.z);
            }
        }
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
    ncount[j] = acc.cnt - self;
    if (LAST) lambdas[j] = lambda;
}

// Later lambda passes on the anchored state.
template <bool LAST>
__global__ void __launch_bounds__(256)
k_lambda(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
         const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
         const uint32_t* __restrict__ sidx, float* __restrict__ lambdas) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 l = cur[s];
    int pcx, pcy, pcz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    const float Xx = anchor(c.g.ox, c.g.cs, pcx) + l.x;
    const float Xy = anchor(c.g.oy, c.g.cs, pcy) + l.y;
    const float Xz = anchor(c.g.oz, c.g.cs, pcz) + l.z;
    LambdaAcc acc;
    for_stencil_anchored(c, cstart, Xx, Xy, Xz, pcx, pcy, pcz, l.x, l.y, l.z,
                         [&](uint32_t k, float ox, float oy, float oz) {
                             const float4 q = __ldg(&cur[k]);
                             acc.add(c, ox - q.x, oy - q.y, oz - q.z);
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
__global__ void __launch_bounds__(256)
k_delta(StepConsts c, const float4* __restrict__ src, float4* __restrict__ dst,
        const uint32_t* __restrict__ scell, const uint32_t* __restrict__ cstart,
        const uint32_t* __restrict__ sidx, const SphereState* __restrict__ sphere,
        float4* __restrict__ pos, float4* __restrict__ vel, const float4* __restrict__ prev,
        const uint32_t* __restrict__ ncount, float* __restrict__ foam, uint32_t* err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 l = src[s];
    int pcx, pcy, pcz;
    decode_cell(c.g, scell[s], pcx, pcy, pcz);
    const float ax = anchor(c.g.ox, c.g.cs, pcx), ay = anchor(c.g.oy, c.g.cs, pcy),
                az = anchor(c.g.oz, c.g.cs, pcz);
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    for_stencil_anchored(c, cstart, ax + l.x, ay + l.y, az + l.z, pcx, pcy, pcz, l.x, l.y, l.z,
                         [&](uint32_t k, float ox, float oy, float oz) {
                             const float4 q = __ldg(&src[k]);
                             delta_add(c, l.w, q.w, ox - q.x, oy - q.y, oz - q.z, dx, dy, dz);
                         });
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
    for (uint32_t it = 0; it < iterations; ++it) {
        const bool first = it == 0, last = it + 1 == iterations;
        tbegin(t, s);
        if (first && last)
            k_lambda_first<true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                      d.sidx, d.lambdas, d.ncount);
        else if (first)
            k_lambda_first<false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart,
                                                       d.sidx, d.lambdas, d.ncount);
        else if (last)
            k_lambda<true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                d.lambdas);
        else
            k_lambda<false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.scell, d.cstart, d.sidx,
                                                 d.lambdas);
        tend(t, first ? "lambda_count" : "lambda", s);
        tbegin(t, s);
        if (last)
            k_delta<true><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx,
                                               d.sphere, d.pos, d.vel, d.prev, d.ncount, d.foam, d.err);
        else
            k_delta<false><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.scell, d.cstart, d.sidx,
                                                d.sphere, d.pos, d.vel, d.prev, d.ncount, d.foam, d.err);
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

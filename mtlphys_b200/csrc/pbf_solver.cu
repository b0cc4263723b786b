// pbf_solver.cu — solver iterations, scatter-back, finalize and foam of the
// PBF step for sm_100a.
//
// Replaces densityLambdaSorted (engine/shaders/Constraints.metal:82-131),
// applyDeltaSorted (:140-199), sphereCollision (:262-277),
// scatterPositionsToOriginal (:205-213), finalizeStep (:305-353) and
// computeFoam (:287-299), dispatched by engine/src/Engine.cpp:728-810.
//
// Layout: one thread per sorted slot.  Because the hash is x-fastest, the
// 27-cell stencil is 9 contiguous slot ranges (one per (y, z) row), read as
// float4 with neighbouring threads sharing most of their ranges in L1.
//   lambda pass  sorted_a (x, y, z, -) -> sorted_b (x, y, z, lambda); the
//                first pass also writes the neighbour count (it visits
//                exactly countNeighbors' candidates on the same positions)
//   delta pass   sorted_b -> sorted_a (new x, y, z); lambda_j arrives in the
//                same 16-byte load as p_j; the sphere push is fused in
//   last delta   also does scatter-back + finalize + foam, writing the
//                original-order positions, velocities and foam directly.
// The particle itself is visited by the stencil loop: it adds W(0) to the
// density (the reference's initial value) and nothing to any gradient.
#include "pbf_kernels.h"

namespace mpb {
namespace {

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(256)
k_lambda(StepConsts c, const float4* __restrict__ cur, float4* __restrict__ nxt,
         const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ sidx,
         float* __restrict__ lambdas, uint32_t* __restrict__ ncount) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 p = cur[s];
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);

    float dens = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f, gsq = 0.0f;
    uint32_t cnt = 0;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y) {
            const uint32_t a = cstart[cell_hash(c.g, x0, y, z)];
            const uint32_t b = cstart[cell_hash(c.g, x1, y, z) + 1];
            for (uint32_t k = a; k < b; ++k) {
                const float4 q = __ldg(&cur[k]);
                const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
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
        }
    const float C = dens * c.inv_rho0 - 1.0f;
    const float denom = c.inv_rho0 * c.inv_rho0 * (gx * gx + gy * gy + gz * gz + gsq) + c.eps;
    const float lambda = -C / denom;
    nxt[s] = make_float4(p.x, p.y, p.z, lambda);
    if (FIRST || LAST) {
        const uint32_t j = sidx[s];
        if (FIRST) ncount[j] = cnt - 1u;
        if (LAST) lambdas[j] = lambda;
    }
}

// finalizeStep (Constraints.metal:305-353) + computeFoam (:287-299) for the
// particle j whose solved position is (px, py, pz).
__device__ __forceinline__ void finalize_particle(const StepConsts& c, uint32_t j, float px,
                                                  float py, float pz, float4* __restrict__ pos,
                                                  float4* __restrict__ vel,
                                                  const float4* __restrict__ prev,
                                                  const uint32_t* __restrict__ ncount,
                                                  float* __restrict__ foam, uint32_t* err) {
    px = fminf(fmaxf(px, c.bminx), c.bmaxx);
    py = fminf(fmaxf(py, c.bminy), c.bmaxy);
    pz = fminf(fmaxf(pz, c.bminz), c.bmaxz);
    const float4 pr = prev[j];
    float vx = (px - pr.x) * c.inv_dt * c.damping;
    float vy = (py - pr.y) * c.inv_dt * c.damping;
    float vz = (pz - pr.z) * c.inv_dt * c.damping;
    const bool xMin = px <= c.bminx + c.wall_eps, xMax = px >= c.bmaxx - c.wall_eps;
    const bool yMin = py <= c.bminy + c.wall_eps, yMax = py >= c.bmaxy - c.wall_eps;
    const bool zMin = pz <= c.bminz + c.wall_eps, zMax = pz >= c.bmaxz - c.wall_eps;
    if (xMin) vx = fmaxf(vx, 0.0f);
    if (xMax) vx = fminf(vx, 0.0f);
    if (yMin) vy = fmaxf(vy, 0.0f);
    if (yMax) vy = fminf(vy, 0.0f);
    if (zMin) vz = fmaxf(vz, 0.0f);
    if (zMax) vz = fminf(vz, 0.0f);
    if (yMin) {
        vx *= c.floor_fric;
        vz *= c.floor_fric;
    } else if (xMin || xMax || zMin || zMax) {
        vx *= c.wall_fric;
        vy *= c.wall_fric;
        vz *= c.wall_fric;
    }
    float vl = sqrtf(vx * vx + vy * vy + vz * vz);
    if (vl > c.vmax) {
        const float f = c.vmax / vl;
        vx *= f;
        vy *= f;
        vz *= f;
        vl = sqrtf(vx * vx + vy * vy + vz * vz);
    }
    pos[j] = make_float4(px, py, pz, 1.0f);
    vel[j] = make_float4(vx, vy, vz, 0.0f);
    const float surface = 1.0f - fminf(fmaxf(float(ncount[j]) / c.foam_maxn, 0.0f), 1.0f);
    foam[j] = surface * smoothstep_f(c.foam_lo, c.foam_hi, vl);
    if (!(isfinite(px) && isfinite(py) && isfinite(pz))) atomicOr(err, kDevErrNaN);
}

template <bool LAST>
__global__ void __launch_bounds__(256)
k_delta(StepConsts c, const float4* __restrict__ src, float4* __restrict__ dst,
        const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ sidx,
        const SphereState* __restrict__ sphere, float4* __restrict__ pos, float4* __restrict__ vel,
        const float4* __restrict__ prev, const uint32_t* __restrict__ ncount,
        float* __restrict__ foam, uint32_t* err) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= c.n) return;
    const float4 p = src[s];
    const float li = p.w;
    int cx, cy, cz;
    cell_of(c.g, p.x, p.y, p.z, cx, cy, cz);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, c.g.gx - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, c.g.gy - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, c.g.gz - 1);

    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y) {
            const uint32_t a = cstart[cell_hash(c.g, x0, y, z)];
            const uint32_t b = cstart[cell_hash(c.g, x1, y, z) + 1];
            for (uint32_t k = a; k < b; ++k) {
                const float4 q = __ldg(&src[k]);
                const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
                const float r2 = dist2(rx, ry, rz);
                if (r2 < c.h2 && r2 > 1e-12f) {
                    const float d = c.h2 - r2;
                    const float ratio = c.poly6 * d * d * d * c.inv_wq;
                    const float scorr = -c.scorr_k * pow_n(ratio, c.scorr_n);
                    const float rinv = rsqrtf(r2);
                    const float hd = fmaxf(c.h - r2 * rinv, 0.0f);
                    const float coef = (li + q.w + scorr) * (-c.spiky * hd * hd * rinv);
                    dx += coef * rx;
                    dy += coef * ry;
                    dz += coef * rz;
                }
            }
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
    float nx = fminf(fmaxf(p.x + dx, c.bminx), c.bmaxx);
    float ny = fminf(fmaxf(p.y + dy, c.bminy), c.bmaxy);
    float nz = fminf(fmaxf(p.z + dz, c.bminz), c.bmaxz);
    if (c.sphere) {
        const float scx = sphere->c[0], scy = sphere->c[1], scz = sphere->c[2], sr = sphere->r;
        const float ex = nx - scx, ey = ny - scy, ez = nz - scz;
        const float e2 = ex * ex + ey * ey + ez * ez;
        if (e2 < sr * sr) {
            const float inv = sr / sqrtf(fmaxf(e2, 1e-8f));
            nx = scx + ex * inv;
            ny = scy + ey * inv;
            nz = scz + ez * inv;
        }
    }
    if (!LAST) {
        dst[s] = make_float4(nx, ny, nz, 1.0f);
        return;
    }
    finalize_particle(c, sidx[s], nx, ny, nz, pos, vel, prev, ncount, foam, err);
}

// Zero solver iterations: scatter-back + finalize + foam of the predicted
// positions; the neighbour count still comes from one counting pass.
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
            k_lambda<true, true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.cstart, d.sidx, d.lambdas, d.ncount);
        else if (first)
            k_lambda<true, false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.cstart, d.sidx, d.lambdas, d.ncount);
        else if (last)
            k_lambda<false, true><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.cstart, d.sidx, d.lambdas, d.ncount);
        else
            k_lambda<false, false><<<grid, 256, 0, s>>>(c, d.sorted_a, d.sorted_b, d.cstart, d.sidx, d.lambdas, d.ncount);
        tend(t, first ? "lambda_count" : "lambda", s);
        tbegin(t, s);
        if (last)
            k_delta<true><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.cstart, d.sidx, d.sphere,
                                               d.pos, d.vel, d.prev, d.ncount, d.foam, d.err);
        else
            k_delta<false><<<grid, 256, 0, s>>>(c, d.sorted_b, d.sorted_a, d.cstart, d.sidx, d.sphere,
                                                d.pos, d.vel, d.prev, d.ncount, d.foam, d.err);
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

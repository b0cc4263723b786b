// pbf_adjoint.cu — adjoint kernels of the PBF step for sm_100a.  No
// reference counterpart: the reference engine (engine/src/Engine.cpp:685-811)
// is not differentiable.
//
// The reverse of one recorded step of a batch of scenes, every kernel one
// thread per sorted slot of every scene, in this order:
//   finalize   dL/d(solved position) and the prev-position term from dL/dx',
//              dL/dv' (finalizeStep, Constraints.metal:305-353, wall masks,
//              friction and the speed cap held at their forward states)
//   K x, last iteration first:
//     pre      through the sphere push (+ dL/d sphere center, radius), the box
//              clamp and the |delta| clamp: dL/d(delta)
//     delta    pair sweep: dL/d lambda, the direct position terms of
//              applyDelta (Constraints.metal:140-199) and dL/dk of s_corr;
//              recomputes the particle's density sums
//     lbar     dL/d(density, gradient sums) from dL/d lambda
//     lambda   pair sweep: position terms of densityLambda (:82-131)
//   predict    dL/dx, dL/dv of predictPositions (:54-66)
//   sphere     dL/d sphere state through its kinematic advance
//              (Engine.cpp:694-707), one thread per scene
//
// The pair sweeps walk exactly the pairs of the forward iteration: the row
// masks its lambda pass recorded (long rows distance-tested past their first
// 32 candidates, as the forward delta pass does).  The reference's neighbour
// search makes those lists asymmetric once particles leave their predicted
// cells (j is in i's list iff j's predicted cell is next to i's current
// cell), so each pair term of i's list is delivered to j by j's own sweep
// when i is in j's list too (a test on the two cells).  Otherwise (a one-way
// pair, ~0.4% of pairs in a 60-step cube drop) i posts the term to j's inbox
// and a delivery kernel adds j's posts in ascending order of the sender's
// slot.  The scene gradients (dL/dk, the sphere's center and radius) are
// accumulated per slot and summed per scene in a fixed order.  Nothing is
// added with float atomics, so the gradients are the same bytes on every run.
#include "pbf_adjoint.h"
#include "pbf_items.cuh"

namespace mpb {
namespace {

constexpr uint32_t kBlock = 256;

inline uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// Dense cell coordinates packed 11 / 11 / 10 bits (x, y, z); the host checks
// that the dense grid fits.
__device__ __forceinline__ uint32_t pack_cell(int x, int y, int z) {
    return uint32_t(x) | (uint32_t(y) << 11) | (uint32_t(z) << 22);
}

// Whether two packed cells are within one cell of each other on every axis.
__device__ __forceinline__ bool cells_adjacent(uint32_t a, uint32_t b) {
    const int dx = int(a & 0x7ffu) - int(b & 0x7ffu);
    const int dy = int((a >> 11) & 0x7ffu) - int((b >> 11) & 0x7ffu);
    const int dz = int(a >> 22) - int(b >> 22);
    return abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1;
}

// Kernel values of a pair at offset r with 1e-12 < |r|^2 = r2 < h^2:
// spiky gradient g = f r, its Jacobian H v = f v + fp (r . v) r, the poly6
// weight W and d = h^2 - r2 (grad W = -6 poly6 d^2 r).
struct PairTerms {
    float d, f, fp, W;
    __device__ __forceinline__ PairTerms(const StepConsts& c, float r2) {
        d = c.h2 - r2;
        const float rinv = rsqrtf(r2);
        const float hd = fmaxf(c.h - r2 * rinv, 0.0f);
        f = -c.spiky * hd * hd * rinv;
        fp = c.spiky * d * rinv * rinv * rinv;
        W = c.poly6 * d * d * d;
    }
    __device__ __forceinline__ float3 hess(float rx, float ry, float rz, float vx, float vy,
                                           float vz) const {
        const float a = fp * (rx * vx + ry * vy + rz * vz);
        return make_float3(f * vx + a * rx, f * vy + a * ry, f * vz + a * rz);
    }
};

__device__ __forceinline__ float pow_u(float x, uint32_t n) {
    float r = 1.0f;
    for (uint32_t e = 0; e < n; ++e) r *= x;
    return r;
}

// Posts the term v that sender slot `from` owes receiver slot `to` (a
// one-way pair): into one of the receiver's kInbox entries, or a pooled
// entry linked into the receiver's overflow list; a post that finds the pool
// exhausted sets kDevErrIndex.
__device__ __forceinline__ void post(const AdjArgs& a, uint32_t to, uint32_t from, const float4& v) {
    const uint32_t e = atomicAdd(&a.inbox_count[to], 1u);
    if (e < kInbox) {
        a.inbox_src[size_t(e) * a.stride + to] = from;
        a.inbox_val[size_t(e) * a.stride + to] = v;
        return;
    }
    const uint32_t o = atomicAdd(a.ovf_count, 1u);
    if (o < kInboxOverflow) {
        a.ovf_src[o] = from;
        a.ovf_val[o] = v;
        a.ovf_next[o] = atomicExch(&a.ovf_head[to], o);
    } else {
        atomicOr(a.err, kDevErrIndex);
    }
}

// ---- finalize --------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_adj_finalize(AdjArgs a) {
    const uint32_t s = blockIdx.x * kBlock + threadIdx.x;
    if (s >= a.n) return;
    // loads first (in flight together), stores after
    const uint32_t sc = __ldg(&a.scene_of[s]);
    const uint32_t cell = __ldg(&a.t.scell[s]);
    const uint32_t j = __ldg(&a.t.sidx[s]);
    const float4 X4 = __ldg(&a.t.x1[j]), P4 = __ldg(&a.t.x0[j]), xb = a.xbar[j], vb = a.vbar[j];
    const StepConsts& c = a.t.scenes[sc].c;
    int px, py, pz;
    decode_cell(c.g, cell, px, py, pz);
    a.cpred[s] = pack_cell(px + c.g.lx, py + c.g.ly, pz + c.g.lz);
    const double X[3] = {X4.x, X4.y, X4.z}, P[3] = {P4.x, P4.y, P4.z};
    const double lo_b[3] = {c.bminx, c.bminy, c.bminz}, hi_b[3] = {c.bmaxx, c.bmaxy, c.bmaxz};
    const double kd = double(c.damping) / double(c.dt);
    bool lo[3], hi[3], keep[3];
    double b[3];
    for (int k = 0; k < 3; ++k) {
        const double u = (X[k] - P[k]) * kd;
        lo[k] = X[k] <= lo_b[k] + double(c.wall_eps);
        hi[k] = X[k] >= hi_b[k] - double(c.wall_eps);
        keep[k] = !((lo[k] && u < 0.0) || (hi[k] && u > 0.0));
        b[k] = keep[k] ? u : 0.0;
    }
    double fr[3] = {1.0, 1.0, 1.0};
    if (lo[1]) {
        fr[0] = fr[2] = c.floor_fric;
    } else if (lo[0] || hi[0] || lo[2] || hi[2]) {
        fr[0] = fr[1] = fr[2] = c.wall_fric;
    }
    for (int k = 0; k < 3; ++k) b[k] *= fr[k];
    const double vmax = double(c.vmax_frac) * double(c.h) / double(c.dt);
    const double bl = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    double bb[3] = {vb.x, vb.y, vb.z};
    if (bl > vmax) {  // v = b vmax / |b|
        const double dot = (b[0] * bb[0] + b[1] * bb[1] + b[2] * bb[2]) / bl;
        for (int k = 0; k < 3; ++k) bb[k] = (vmax / bl) * (bb[k] - dot * b[k] / bl);
    }
    double ub[3];
    for (int k = 0; k < 3; ++k) ub[k] = keep[k] ? bb[k] * fr[k] * kd : 0.0;
    a.pbar[s] = make_float4(float(xb.x + ub[0]), float(xb.y + ub[1]), float(xb.z + ub[2]), 0.0f);
    a.xbar[j] = make_float4(float(-ub[0]), float(-ub[1]), float(-ub[2]), 0.0f);
}

// ---- one solver iteration ---------------------------------------------------

// Through the sphere push, the box clamp and the |delta| clamp of iteration
// `it`; records the iterate's current cell for the pair sweeps.
__global__ void __launch_bounds__(kBlock) k_adj_pre(AdjArgs a, uint32_t it) {
    const uint32_t s = blockIdx.x * kBlock + threadIdx.x;
    if (s == 0) *a.ovf_count = 0;  // the delta sweep posts into an empty list
    if (s >= a.n) return;
    // every per-slot input first, so their loads are in flight together
    const size_t off = size_t(it) * a.stride;
    const uint32_t sc = __ldg(&a.scene_of[s]);
    const float4 l = __ldg(&a.t.lam[off + s]);
    const float4 dr = __ldg(&a.t.delta[off + s]);
    const uint32_t cell = __ldg(&a.t.scell[s]);
    const float4 pe = a.p_extra[s];
    const float4 pb4 = a.pbar[s];
    const SceneDev& sd = a.t.scenes[sc];
    const StepConsts& c = sd.c;
    int pcx, pcy, pcz;
    decode_cell(c.g, cell, pcx, pcy, pcz);
    const float ax = anchor_x(c.g, pcx), ay = anchor_y(c.g, pcy), az = anchor_z(c.g, pcz);
    int cx, cy, cz;
    cell_of(c.g, __fadd_rn(ax, l.x), __fadd_rn(ay, l.y), __fadd_rn(az, l.z), cx, cy, cz);
    a.ccur[s] = pack_cell(cx + c.g.lx, cy + c.g.ly, cz + c.g.lz);

    // the forward update (delta_item): clamp |delta|, A + (l + delta) in FP64
    const float dl = __fsqrt_rn(dist2(dr.x, dr.y, dr.z));
    const bool big = dl > c.max_step;
    const float f = big ? __fdiv_rn(c.max_step, dl) : 1.0f;
    const float dx = big ? __fmul_rn(dr.x, f) : dr.x;
    const float dy = big ? __fmul_rn(dr.y, f) : dr.y;
    const float dz = big ? __fmul_rn(dr.z, f) : dr.z;
    const double q[3] = {__dadd_rn(double(ax), double(__fadd_rn(l.x, dx))),
                         __dadd_rn(double(ay), double(__fadd_rn(l.y, dy))),
                         __dadd_rn(double(az), double(__fadd_rn(l.z, dz)))};
    const double lo_b[3] = {c.bminx, c.bminy, c.bminz}, hi_b[3] = {c.bmaxx, c.bmaxy, c.bmaxz};
    bool inside[3];
    double qc[3];
    for (int k = 0; k < 3; ++k) {
        inside[k] = q[k] >= lo_b[k] && q[k] <= hi_b[k];
        qc[k] = fmin(fmax(q[k], lo_b[k]), hi_b[k]);
    }

    a.p_extra[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float pb[3] = {pb4.x + pe.x, pb4.y + pe.y, pb4.z + pe.z};
    if (c.sphere) {
        const double ex = qc[0] - sd.sphere.c[0], ey = qc[1] - sd.sphere.c[1], ez = qc[2] - sd.sphere.c[2];
        const double e2 = ex * ex + ey * ey + ez * ez, r = sd.sphere.r;
        if (e2 < r * r) {  // x = center + e r / |e|
            const double el = sqrt(fmax(e2, double(1e-8f)));
            const double e[3] = {ex / el, ey / el, ez / el};
            const double dot = e2 > double(1e-8f) ? e[0] * pb[0] + e[1] * pb[1] + e[2] * pb[2] : 0.0;
            double cb[3], eb[3];
            for (int k = 0; k < 3; ++k) {
                eb[k] = (r / el) * (pb[k] - e[k] * dot);
                cb[k] = pb[k] - eb[k];
            }
            const double rb = e[0] * pb[0] + e[1] * pb[1] + e[2] * pb[2];
            double4 sa = a.sacc[s];  // this slot's share of the step's sphere gradient
            sa.x += cb[0];
            sa.y += cb[1];
            sa.z += cb[2];
            sa.w += rb;
            a.sacc[s] = sa;
            for (int k = 0; k < 3; ++k) pb[k] = float(eb[k]);
        }
    }
    for (int k = 0; k < 3; ++k)
        if (!inside[k]) pb[k] = 0.0f;
    a.qbar[s] = make_float4(pb[0], pb[1], pb[2], 0.0f);
    if (big) {  // delta = d max_step / |d|
        const float ux = dr.x / dl, uy = dr.y / dl, uz = dr.z / dl;
        const float dot = ux * pb[0] + uy * pb[1] + uz * pb[2];
        pb[0] = f * (pb[0] - ux * dot);
        pb[1] = f * (pb[1] - uy * dot);
        pb[2] = f * (pb[2] - uz * dot);
    }
    a.dbar[s] = make_float4(pb[0], pb[1], pb[2], 0.0f);
}

// Pair sweep of applyDelta's adjoint.  With dbar = dL/d delta:
//   lambdabar_i = sum_j g_ij . (dbar_i - dbar_j) / rho0
//   pbar_i     += sum_j ((lambda_i + lambda_j + s_ij) H_ij (dbar_i - dbar_j)
//                        + grad s_ij g_ij . (dbar_i - dbar_j)) / rho0
//   kbar       += sum_j -(W_ij / W(dq))^n g_ij . dbar_i / rho0
// (dbar_j and the j-side terms only for pairs in both lists; the j-side
// terms of a one-way pair are added to j atomically), and the particle's
// density sums for the lambda adjoint.
// The two pair sweeps are compiled for 4 resident blocks per SM (64
// registers): left alone they take ~90 and run 13-16% slower.
#ifndef MPB_ADJ_SWEEP_MIN_BLOCKS
#define MPB_ADJ_SWEEP_MIN_BLOCKS 4
#endif
constexpr int kSweepMinBlocks = MPB_ADJ_SWEEP_MIN_BLOCKS;

__global__ void __launch_bounds__(kBlock, kSweepMinBlocks) k_adj_delta(AdjArgs a, uint32_t it) {
    const uint32_t m = blockIdx.x * kBlock + threadIdx.x;
    float kb = 0.0f;
    if (m < a.n) {
        const StepConsts& c = a.t.scenes[a.scene_of[m]].c;
        const size_t off = size_t(it) * a.stride;
        const float4* src = a.t.lam + off;
        const float4 l = src[m];
        const float4 dm = a.dbar[m];
        const uint32_t pm = a.cpred[m];
        int pcx, pcy, pcz;
        decode_cell(c.g, a.t.scell[m], pcx, pcy, pcz);
        const float ax = anchor_x(c.g, pcx), ay = anchor_y(c.g, pcy), az = anchor_z(c.g, pcz);
        int cx, cy, cz;
        cell_of(c.g, __fadd_rn(ax, l.x), __fadd_rn(ay, l.y), __fadd_rn(az, l.z), cx, cy, cz);
        const float h2 = c.h2;
        float dens = c.poly6 * h2 * h2 * h2;  // the particle itself
        float gx = 0.0f, gy = 0.0f, gz = 0.0f, gsq = 0.0f;
        float lb = 0.0f, px = 0.0f, py = 0.0f, pz = 0.0f;
        const uint32_t n = c.scorr_n;
        const float sgk = n ? 6.0f * c.scorr_k * float(n) * c.inv_wq * c.poly6 : 0.0f;
        auto body = [&](uint32_t k, const float4& q, float rx, float ry, float rz, float r2) {
            if (k == m) return;
            if (!(r2 > 1e-12f)) {
                dens += c.poly6 * (h2 - r2) * (h2 - r2) * (h2 - r2);
                return;
            }
            const PairTerms t(c, r2);
            dens += t.W;
            const float fx = t.f * rx, fy = t.f * ry, fz = t.f * rz;  // g
            gx += fx;
            gy += fy;
            gz += fz;
            gsq += t.f * t.f * r2;
            const float ratio = t.W * c.inv_wq;
            const float rn1 = n ? pow_u(ratio, n - 1) : 0.0f;
            const float rn = n ? rn1 * ratio : 1.0f;
            const float coef = l.w + q.w - c.scorr_k * rn;
            const float sg = sgk * rn1 * t.d * t.d;  // grad s_ij = sg r
            const float gdm = fx * dm.x + fy * dm.y + fz * dm.z;
            kb -= rn * gdm;
            if (cells_adjacent(a.ccur[k], pm)) {
                const float4 di = a.dbar[k];
                const float ex = dm.x - di.x, ey = dm.y - di.y, ez = dm.z - di.z;
                const float gdd = fx * ex + fy * ey + fz * ez;
                lb += gdd;
                const float3 hv = t.hess(rx, ry, rz, ex, ey, ez);
                px += coef * hv.x + sg * gdd * rx;
                py += coef * hv.y + sg * gdd * ry;
                pz += coef * hv.z + sg * gdd * rz;
            } else {
                lb += gdm;
                const float3 hv = t.hess(rx, ry, rz, dm.x, dm.y, dm.z);
                const float vx = coef * hv.x + sg * gdm * rx;
                const float vy = coef * hv.y + sg * gdm * ry;
                const float vz = coef * hv.z + sg * gdm * rz;
                px += vx;
                py += vy;
                pz += vz;
                post(a, k, m,
                     make_float4(-vx * c.inv_rho0, -vy * c.inv_rho0, -vz * c.inv_rho0, gdm * c.inv_rho0));
            }
        };
        const uint32_t ms = a.mask_stride;
        const RowMasks rm{const_cast<uint32_t*>(a.t.masks) + size_t(it) * 9 * ms,
                          const_cast<uint32_t*>(a.t.overflow) + size_t(it) * ms, ms};
        masked_pairs(c, src, a.t.cstart, rm, m, l, ax, ay, az, cx, cy, cz, body);
        const float ir = c.inv_rho0;
        const float4 qb = a.qbar[m];
        a.qbar[m] = make_float4(qb.x + px * ir, qb.y + py * ir, qb.z + pz * ir, 0.0f);
        a.lam_part[m] = lb * ir;
        const float D = ir * ir * (gx * gx + gy * gy + gz * gz + gsq) + c.eps;
        a.gd[m] = make_float4(gx, gy, gz, D);
        kb *= ir;
        a.kacc[m] += double(kb);  // this slot's share of dL/dk
    }
}

// dL/d(density sum, gradient sum, squared-gradient sum) of each particle's
// lambda = -(rho / rho0 - 1) / (|G|^2 + Q) / rho0^2 + eps):
//   rhobar = -lambdabar / (D rho0), Dbar = -lambdabar lambda / D,
//   Gbar = 2 Dbar G / rho0^2, Qbar = Dbar / rho0^2.
__global__ void __launch_bounds__(kBlock) k_adj_lbar(AdjArgs a, uint32_t it) {
    const uint32_t s = blockIdx.x * kBlock + threadIdx.x;
    if (s == 0) *a.ovf_count = 0;  // the lambda sweep posts into an empty list
    if (s >= a.n) return;
    const StepConsts& c = a.t.scenes[a.scene_of[s]].c;
    const float lb = a.lam_part[s] + a.lam_extra[s];
    a.lam_extra[s] = 0.0f;
    const float4 gd = a.gd[s];
    const float lam = a.t.lam[size_t(it) * a.stride + s].w;
    const float ir = c.inv_rho0;
    const float Db = -lb * lam / gd.w;
    const float gG = 2.0f * Db * ir * ir;
    a.lbar[s] = make_float4(gG * gd.x, gG * gd.y, gG * gd.z, -lb * ir / gd.w);
    a.qsc[s] = Db * ir * ir;
}

// Pair sweep of densityLambda's adjoint:
//   pbar_i += sum_j (rhobar_i + rhobar_j) grad W_ij
//             + H_ij (Gbar_i - Gbar_j + 2 (Qbar_i + Qbar_j) g_ij)
// (j-side terms of one-way pairs added to j atomically).
__global__ void __launch_bounds__(kBlock, kSweepMinBlocks) k_adj_lambda(AdjArgs a, uint32_t it) {
    const uint32_t m = blockIdx.x * kBlock + threadIdx.x;
    if (m >= a.n) return;
    const StepConsts& c = a.t.scenes[a.scene_of[m]].c;
    const size_t off = size_t(it) * a.stride;
    const float4* src = a.t.lam + off;
    const float4 l = src[m];
    const float4 lm = a.lbar[m];
    const float qm = a.qsc[m];
    const uint32_t pm = a.cpred[m];
    int pcx, pcy, pcz;
    decode_cell(c.g, a.t.scell[m], pcx, pcy, pcz);
    const float ax = anchor_x(c.g, pcx), ay = anchor_y(c.g, pcy), az = anchor_z(c.g, pcz);
    int cx, cy, cz;
    cell_of(c.g, __fadd_rn(ax, l.x), __fadd_rn(ay, l.y), __fadd_rn(az, l.z), cx, cy, cz);
    const float4 qb = a.qbar[m];
    float px = qb.x, py = qb.y, pz = qb.z;
    const float w6 = -6.0f * c.poly6;
    auto body = [&](uint32_t k, const float4&, float rx, float ry, float rz, float r2) {
        if (k == m || !(r2 > 1e-12f)) return;
        const PairTerms t(c, r2);
        const float gw = w6 * t.d * t.d;  // grad W = gw r
        if (cells_adjacent(a.ccur[k], pm)) {
            const float4 li = a.lbar[k];
            const float qs = 2.0f * (qm + a.qsc[k]) * t.f;
            const float3 hv = t.hess(rx, ry, rz, lm.x - li.x + qs * rx, lm.y - li.y + qs * ry,
                                     lm.z - li.z + qs * rz);
            const float w = (lm.w + li.w) * gw;
            px += w * rx + hv.x;
            py += w * ry + hv.y;
            pz += w * rz + hv.z;
        } else {
            const float qs = 2.0f * qm * t.f;
            const float3 hv = t.hess(rx, ry, rz, lm.x + qs * rx, lm.y + qs * ry, lm.z + qs * rz);
            const float w = lm.w * gw;
            const float vx = w * rx + hv.x, vy = w * ry + hv.y, vz = w * rz + hv.z;
            px += vx;
            py += vy;
            pz += vz;
            post(a, k, m, make_float4(-vx, -vy, -vz, 0.0f));
        }
    };
    const uint32_t ms = a.mask_stride;
    const RowMasks rm{const_cast<uint32_t*>(a.t.masks) + size_t(it) * 9 * ms,
                      const_cast<uint32_t*>(a.t.overflow) + size_t(it) * ms, ms};
    masked_pairs(c, src, a.t.cstart, rm, m, l, ax, ay, az, cx, cy, cz, body);
    a.pbar[m] = make_float4(px, py, pz, 0.0f);
}

// ---- delivery of one-way pair terms, scene sums ----------------------------------

// Adds every post of receiver slot j in ascending order of the sender's slot
// (a sender posts to a receiver at most once per sweep): p_extra += the
// xyz sums, and with LAMBDA lam_extra += the w sum.  Posts beyond the inbox
// are looked up in the overflow list.
template <bool LAMBDA>
__global__ void __launch_bounds__(kBlock) k_adj_deliver(AdjArgs a) {
    const uint32_t j = blockIdx.x * kBlock + threadIdx.x;
    if (j >= a.n) return;
    const uint32_t cnt = a.inbox_count[j];
    if (cnt == 0) return;
    a.inbox_count[j] = 0;
    const uint32_t nin = min(cnt, kInbox);
    const uint32_t head = cnt > kInbox ? a.ovf_head[j] : kNoPost;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, sw = 0.0f;
    uint32_t last = 0;
    for (uint32_t done = 0; done < cnt; ++done) {
        uint32_t best = 0xffffffffu;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (uint32_t e = 0; e < nin; ++e) {
            const uint32_t src = a.inbox_src[size_t(e) * a.stride + j];
            if ((done == 0 || src > last) && src < best) {
                best = src;
                v = a.inbox_val[size_t(e) * a.stride + j];
            }
        }
        for (uint32_t o = head; o != kNoPost; o = a.ovf_next[o]) {
            const uint32_t src = a.ovf_src[o];
            if ((done == 0 || src > last) && src < best) {
                best = src;
                v = a.ovf_val[o];
            }
        }
        if (best == 0xffffffffu) break;  // posts dropped with the pool exhausted
        sx += v.x;
        sy += v.y;
        sz += v.z;
        sw += v.w;
        last = best;
    }
    if (head != kNoPost) a.ovf_head[j] = kNoPost;
    const float4 pe = a.p_extra[j];
    a.p_extra[j] = make_float4(pe.x + sx, pe.y + sy, pe.z + sz, 0.0f);
    if (LAMBDA) a.lam_extra[j] += sw;
}

// Fixed-order block sum of one double per thread (blockDim.x == kBlock).
__device__ __forceinline__ double block_sum(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t w = kBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Block (chunk, scene): the step's sphere gradient summed, in a fixed order,
// over the chunk's kSumChunk slots of a sphere scene into spart; the per-slot
// accumulators are cleared.  k_adj_sphere adds the chunks in order.
__global__ void __launch_bounds__(kBlock) k_adj_sphere_sum(AdjArgs a) {
    __shared__ double sh[kBlock];
    const uint32_t chunk = blockIdx.x, sc = blockIdx.y;
    const SceneDev& sd = a.t.scenes[sc];
    if (!sd.c.sphere) return;  // only sphere scenes accumulate
    const uint32_t first = chunk * kSumChunk, n = sd.c.n;
    const uint32_t end = min(n, first + kSumChunk);
    // kSumChunk / kBlock = 8 entries per thread, loaded 4 at a time before
    // they are added (in index order) and cleared
    static_assert(kSumChunk == 8 * kBlock, "two rounds of four loads per thread");
    double cx = 0.0, cy = 0.0, cz = 0.0, r = 0.0;
    double4* acc = a.sacc + sd.p0;
#pragma unroll
    for (uint32_t round = 0; round < 2; ++round) {
        double4 v[4];
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
            const uint32_t i = first + (round * 4 + u) * kBlock + threadIdx.x;
            v[u] = i < end ? acc[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        }
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
            const uint32_t i = first + (round * 4 + u) * kBlock + threadIdx.x;
            cx += v[u].x;
            cy += v[u].y;
            cz += v[u].z;
            r += v[u].w;
            if (i < end) acc[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        }
    }
    cx = block_sum(cx, sh);
    cy = block_sum(cy, sh);
    cz = block_sum(cz, sh);
    r = block_sum(r, sh);
    if (threadIdx.x == 0) a.spart[size_t(sc) * a.sum_chunks + chunk] = make_double4(cx, cy, cz, r);
}

// One block per scene: dL/dk = the sum of the per-slot accumulators over the
// scene's slots (fixed order), which are cleared.
__global__ void __launch_bounds__(kBlock) k_adj_k_sum(AdjArgs a) {
    __shared__ double sh[kBlock];
    const SceneDev& sd = a.t.scenes[blockIdx.x];
    const uint32_t p0 = sd.p0, n = sd.c.n;
    double k = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += kBlock) {
        k += a.kacc[p0 + i];
        a.kacc[p0 + i] = 0.0;
    }
    k = block_sum(k, sh);
    if (threadIdx.x == 0) a.grads[size_t(blockIdx.x) * kGradStride + kGradK] = k;
}

// ---- predict, sphere ----------------------------------------------------------

__global__ void __launch_bounds__(kBlock) k_adj_predict(AdjArgs a) {
    const uint32_t s = blockIdx.x * kBlock + threadIdx.x;
    if (s >= a.n) return;
    // loads first (in flight together), stores after
    const uint32_t sc = __ldg(&a.scene_of[s]);
    const uint32_t j = __ldg(&a.t.sidx[s]);
    const float4 pb = a.pbar[s], pe = a.p_extra[s];
    const float4 xb = a.xbar[j];
    const float dt = a.t.scenes[sc].c.dt;
    a.p_extra[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float bx = pb.x + pe.x, by = pb.y + pe.y, bz = pb.z + pe.z;
    a.xbar[j] = make_float4(xb.x + bx, xb.y + by, xb.z + bz, 0.0f);
    a.vbar[j] = make_float4(bx * dt, by * dt, bz * dt, 0.0f);
}

// The sphere's kinematic advance of this step (sphere_advance) reversed:
// the adjoint of the advanced state -> the adjoint of the state before it.
__global__ void __launch_bounds__(128) k_adj_sphere(AdjArgs a) {
    const uint32_t sc = blockIdx.x * 128 + threadIdx.x;
    if (sc >= a.nscenes) return;
    const StepConsts& c = a.t.scenes[sc].c;
    if (!c.sphere) return;
    {  // this step's push terms, chunk by chunk in order (k_adj_sphere_sum)
        // added in chunk order in registers (the same sums as adding each
        // chunk into g), loads four chunks ahead
        double* g = a.grads + size_t(sc) * kGradStride;
        const uint32_t chunks = (c.n + kSumChunk - 1) / kSumChunk;
        const double4* part = a.spart + size_t(sc) * a.sum_chunks;
        double gx = g[kGradCenter], gy = g[kGradCenter + 1], gz = g[kGradCenter + 2], gr = g[kGradRadius];
        for (uint32_t k0 = 0; k0 < chunks; k0 += 4) {
            double4 v[4];
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u)
                v[u] = k0 + u < chunks ? part[k0 + u] : make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u) {
                if (k0 + u >= chunks) break;
                gx += v[u].x;
                gy += v[u].y;
                gz += v[u].z;
                gr += v[u].w;
            }
        }
        g[kGradCenter] = gx;
        g[kGradCenter + 1] = gy;
        g[kGradCenter + 2] = gz;
        g[kGradRadius] = gr;
    }
    const SphereState s0 = a.t.sphere0[sc];
    // forward branch decisions, as sphere_advance computes them
    float v[3] = {s0.v[0], __fadd_rn(s0.v[1], __fmul_rn(c.sph_gravity, c.dt)), s0.v[2]};
    float p[3];
    const float lo_b[3] = {c.bminx, c.bminy, c.bminz}, hi_b[3] = {c.bmaxx, c.bmaxy, c.bmaxz};
    bool lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        v[k] = __fmul_rn(v[k], c.sph_drag);
        p[k] = __fadd_rn(s0.c[k], __fmul_rn(v[k], c.dt));
        lo[k] = __fsub_rn(p[k], s0.r) < lo_b[k];
        if (lo[k]) p[k] = __fadd_rn(lo_b[k], s0.r);
        hi[k] = __fadd_rn(p[k], s0.r) > hi_b[k];
    }
    double* g = a.grads + size_t(sc) * kGradStride;
    double cb[3] = {g[kGradCenter], g[kGradCenter + 1], g[kGradCenter + 2]};
    double vb[3] = {g[kGradVel], g[kGradVel + 1], g[kGradVel + 2]};
    double rb = g[kGradRadius];
    const double rest = c.sph_rest;
    for (int k = 2; k >= 0; --k) {
        if (hi[k]) {  // p = hi - r, v = -v rest
            rb -= cb[k];
            cb[k] = 0.0;
            vb[k] *= -rest;
        }
        if (lo[k]) {  // p = lo + r, v = -v rest
            rb += cb[k];
            cb[k] = 0.0;
            vb[k] *= -rest;
        }
    }
    for (int k = 0; k < 3; ++k) {
        vb[k] = (vb[k] + cb[k] * double(c.dt)) * double(c.sph_drag);  // p = c + v dt, v = v drag
        g[kGradCenter + k] = cb[k];
        g[kGradVel + k] = vb[k];
    }
    g[kGradRadius] = rb;
}

}  // namespace

cudaError_t launch_adjoint_step(const AdjArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    const uint32_t grid = cdiv(a.n, kBlock);
    k_adj_finalize<<<grid, kBlock, 0, s>>>(a);
    for (uint32_t it = a.iterations; it-- > 0;) {
        k_adj_pre<<<grid, kBlock, 0, s>>>(a, it);
        k_adj_delta<<<grid, kBlock, 0, s>>>(a, it);
        k_adj_deliver<true><<<grid, kBlock, 0, s>>>(a);
        k_adj_lbar<<<grid, kBlock, 0, s>>>(a, it);
        k_adj_lambda<<<grid, kBlock, 0, s>>>(a, it);
        k_adj_deliver<false><<<grid, kBlock, 0, s>>>(a);
    }
    k_adj_predict<<<grid, kBlock, 0, s>>>(a);
    if (a.nscenes && a.sum_chunks) k_adj_sphere_sum<<<dim3(a.sum_chunks, a.nscenes), kBlock, 0, s>>>(a);
    k_adj_sphere<<<cdiv(a.nscenes, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_finish(const AdjArgs& a, cudaStream_t s) {
    if (a.n == 0 || a.nscenes == 0) return cudaSuccess;
    k_adj_k_sum<<<a.nscenes, kBlock, 0, s>>>(a);
    return cudaGetLastError();
}

uint32_t adjoint_launch_count(uint32_t iterations) { return 4u + 6u * iterations; }

}  // namespace mpb

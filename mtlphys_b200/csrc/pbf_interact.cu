// pbf_interact.cu — the interactive and legacy per-particle passes of the
// engine for sm_100a, one thread per particle in original order:
//
//   k_integrate     Engine::integrate (engine/src/Engine.cpp:578-596),
//                   kernel integrate (engine/shaders/Integrate.metal:11-42)
//   k_mouse_pulse   Engine::applyMousePulse (Engine.cpp:813-841),
//                   kernel applyMousePulse (Constraints.metal:231-253)
//
// Both are streaming (32 B read + 32 B written per particle for integrate,
// 32 B read and up to 16 B written for the pulse).  The arithmetic is written
// with explicit round-to-nearest operations in the shaders' order, so the
// results equal the reference's FP32 arithmetic without contraction (the
// pulse's exp is CUDA's expf).
#include "pbf_kernels.h"

namespace mpb {
namespace {

constexpr uint32_t kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_integrate(IntegrateConsts c, float4* __restrict__ pos,
                                                      float4* __restrict__ vel) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= c.n) return;
    const float4 p4 = pos[i], v4 = vel[i];
    float p[3] = {p4.x, p4.y, p4.z}, v[3] = {v4.x, v4.y, v4.z};
    const float g[3] = {c.gx, c.gy, c.gz};
    // symplectic Euler: velocity first, then position
    for (int a = 0; a < 3; ++a) {
        v[a] = __fmul_rn(__fadd_rn(v[a], __fmul_rn(g[a], c.dt)), c.damping);
        p[a] = __fadd_rn(p[a], __fmul_rn(v[a], c.dt));
    }
    // box: all lower faces, then all upper faces, as the shader orders them
    const float lo[3] = {c.bminx, c.bminy, c.bminz}, hi[3] = {c.bmaxx, c.bmaxy, c.bmaxz};
    for (int a = 0; a < 3; ++a)
        if (p[a] < lo[a]) {
            p[a] = lo[a];
            v[a] = __fmul_rn(-v[a], c.restitution);
        }
    for (int a = 0; a < 3; ++a)
        if (p[a] > hi[a]) {
            p[a] = hi[a];
            v[a] = __fmul_rn(-v[a], c.restitution);
        }
    pos[i] = make_float4(p[0], p[1], p[2], 1.0f);
    vel[i] = make_float4(v[0], v[1], v[2], 0.0f);
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

__global__ void __launch_bounds__(kBlock) k_mouse_pulse(MouseConsts c, float4* __restrict__ vel,
                                                        const float4* __restrict__ pos) {
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= c.n) return;
    const float4 p = pos[i];
    // distance from the particle to the nearest point of the ray
    const float tx = __fsub_rn(p.x, c.ox), ty = __fsub_rn(p.y, c.oy), tz = __fsub_rn(p.z, c.oz);
    const float t = dot3(tx, ty, tz, c.dx, c.dy, c.dz);
    if (t <= 0.0f) return;  // behind the ray origin
    const float cx = __fadd_rn(c.ox, __fmul_rn(c.dx, t));
    const float cy = __fadd_rn(c.oy, __fmul_rn(c.dy, t));
    const float cz = __fadd_rn(c.oz, __fmul_rn(c.dz, t));
    const float ex = __fsub_rn(p.x, cx), ey = __fsub_rn(p.y, cy), ez = __fsub_rn(p.z, cz);
    const float r2 = dot3(ex, ey, ez, ex, ey, ez);
    const float R2 = __fmul_rn(c.radius, c.radius);
    if (r2 < R2) {
        const float intensity = expf(__fdiv_rn(-r2, __fmul_rn(R2, c.falloff)));
        const float4 v = vel[i];
        vel[i] = make_float4(__fadd_rn(v.x, __fmul_rn(c.fx, intensity)),
                             __fadd_rn(v.y, __fmul_rn(c.fy, intensity)),
                             __fadd_rn(v.z, __fmul_rn(c.fz, intensity)), 0.0f);
    }
}

}  // namespace

cudaError_t launch_integrate(const IntegrateConsts& c, float4* pos, float4* vel, cudaStream_t s) {
    if (c.n == 0) return cudaSuccess;
    k_integrate<<<(c.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(c, pos, vel);
    return cudaGetLastError();
}

cudaError_t launch_mouse_pulse(const MouseConsts& c, float4* vel, const float4* pos, cudaStream_t s) {
    if (c.n == 0) return cudaSuccess;
    k_mouse_pulse<<<(c.n + kBlock - 1) / kBlock, kBlock, 0, s>>>(c, vel, pos);
    return cudaGetLastError();
}

}  // namespace mpb

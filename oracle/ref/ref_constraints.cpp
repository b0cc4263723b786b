// ref_constraints.cpp — compiles the reference's engine/shaders/
// Constraints.metal unchanged as host C++ (through the metal_stdlib shim in
// this folder) and exposes one loop per kernel: call k runs GPU thread k.
//
// TEST INFRASTRUCTURE ONLY (the "_ref" cross-check of the oracle).
#include "Constraints.metal"

#include "ref_harness.h"

extern "C" {

size_t ref_sizeof_pbf_params(void) { return sizeof(PBFParams); }

void ref_fill_pbf_params(void* out, const float gravity[3], float dt, const float bmin[3],
                         const float bmax[3], float h, float h2, float poly6_norm,
                         float spiky_norm, float rest_density, float epsilon, float damping,
                         uint32_t n) {
    auto& pp = *static_cast<PBFParams*>(out);
    pp.gravity = float3(gravity[0], gravity[1], gravity[2]);
    pp.dt = dt;
    pp.boundsMin = float3(bmin[0], bmin[1], bmin[2]);
    pp.invDt = 1.0f / dt;
    pp.boundsMax = float3(bmax[0], bmax[1], bmax[2]);
    pp.h = h;
    pp.h2 = h2;
    pp.poly6Norm = poly6_norm;
    pp.spikyGradNorm = spiky_norm;
    pp.restDensity = rest_density;
    pp.invRestDensity = 1.0f / rest_density;
    pp.epsilon = epsilon;
    pp.damping = damping;
    pp.particleCount = n;
}

void ref_k_predict(float* pos4, const float* vel4, float* prev4, const void* pp, uint32_t threads) {
    const auto& p = *static_cast<const PBFParams*>(pp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        predictPositions(reinterpret_cast<float4*>(pos4), reinterpret_cast<const float4*>(vel4),
                         reinterpret_cast<float4*>(prev4), p, uint(g));
}

void ref_k_density_lambda(const float* sorted4, const uint32_t* cell_start,
                          const uint32_t* sorted_index, float* sorted_lambda, float* lambdas,
                          const void* sp, const void* pp, uint32_t threads) {
    const auto& s = *static_cast<const SpatialParams*>(sp);
    const auto& p = *static_cast<const PBFParams*>(pp);
#pragma omp parallel for schedule(dynamic, 1024) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        densityLambdaSorted(reinterpret_cast<const float4*>(sorted4), cell_start, sorted_index,
                            sorted_lambda, lambdas, s, p, uint(g));
}

void ref_k_apply_delta(const float* sorted4, const uint32_t* cell_start,
                       const float* sorted_lambda, float* next4, const void* sp, const void* pp,
                       uint32_t threads) {
    const auto& s = *static_cast<const SpatialParams*>(sp);
    const auto& p = *static_cast<const PBFParams*>(pp);
#pragma omp parallel for schedule(dynamic, 1024) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        applyDeltaSorted(reinterpret_cast<const float4*>(sorted4), cell_start, sorted_lambda,
                         reinterpret_cast<float4*>(next4), s, p, uint(g));
}

void ref_k_sphere_collision(float* buf4, const void* sp, const float center[3], float radius,
                            uint32_t threads) {
    const auto& s = *static_cast<const SpatialParams*>(sp);
    SphereParams sph;
    sph.center = float3(center[0], center[1], center[2]);
    sph.radius = radius;
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        sphereCollision(reinterpret_cast<float4*>(buf4), s, sph, uint(g));
}

void ref_k_scatter_to_original(const float* sorted4, const uint32_t* sorted_index, float* pos4,
                               const void* sp, uint32_t threads) {
    const auto& s = *static_cast<const SpatialParams*>(sp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        scatterPositionsToOriginal(reinterpret_cast<const float4*>(sorted4), sorted_index,
                                   reinterpret_cast<float4*>(pos4), s, uint(g));
}

void ref_k_finalize(float* pos4, float* vel4, const float* prev4, const void* pp, uint32_t threads) {
    const auto& p = *static_cast<const PBFParams*>(pp);
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        finalizeStep(reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4),
                     reinterpret_cast<const float4*>(prev4), p, uint(g));
}

void ref_k_compute_foam(const float* vel4, const uint32_t* ncount, float* foam, uint32_t count,
                        float max_neighbors, uint32_t threads) {
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        computeFoam(reinterpret_cast<const float4*>(vel4), ncount, foam, count, max_neighbors,
                    uint(g));
}

void ref_k_mouse_pulse(float* vel4, const float* pos4, const float origin[3], const float dir[3],
                       const float force[3], float radius, uint32_t count, uint32_t threads) {
    MousePulseUniforms u{};
    u.rayOrigin = float3(origin[0], origin[1], origin[2]);
    u.rayDir = float3(dir[0], dir[1], dir[2]);
    u.force = float3(force[0], force[1], force[2]);
    u.radius = radius;
#pragma omp parallel for schedule(static) if (ref_parallel())
    for (int64_t g = 0; g < int64_t(threads); ++g)
        applyMousePulse(reinterpret_cast<float4*>(vel4), reinterpret_cast<const float4*>(pos4), u,
                        count, uint(g));
}

}  // extern "C"

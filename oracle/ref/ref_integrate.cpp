// ref_integrate.cpp — compiles the reference's engine/shaders/
// Integrate.metal unchanged as host C++ (legacy integrator).
//
// TEST INFRASTRUCTURE ONLY (the "_ref" cross-check of the oracle).
#include "Integrate.metal"

#include "ref_harness.h"

extern "C" void ref_integrate(float* pos4, float* vel4, const float gravity[3], float dt,
                              const float bmin[3], const float bmax[3], float damping,
                              uint32_t n) {
    SimParams p{};
    p.gravity = float3(gravity[0], gravity[1], gravity[2]);
    p.dt = dt;
    p.boundsMin = float3(bmin[0], bmin[1], bmin[2]);
    p.boundsMax = float3(bmax[0], bmax[1], bmax[2]);
    p.damping = damping;
    p.particleCount = n;
    for (uint32_t g = 0; g < n; ++g)
        integrate(reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4), p, g);
}

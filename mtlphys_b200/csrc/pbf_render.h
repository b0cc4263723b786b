// pbf_render.h — headless screen-space fluid rendering (pbf_render.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pbf_device.cuh"

namespace mpb {

constexpr uint32_t kRenderBox = 1u, kRenderSphere = 2u, kRenderFoam = 4u;

// Per-frame constants (RenderUniforms, engine/shaders/Shared.h:83-91, plus
// the box and the pass switches).  view: rows 0-2 of the 4x4 view matrix
// (view position = view[4r..4r+2] . p + view[4r+3]); p00, p11, p22, p23:
// the perspective matrix's non-trivial entries.
struct RenderConsts {
    uint32_t W, H, n, flags;
    float view[12];
    float p00, p11, p22, p23;
    float znear, zfar, radius, foam_scale, tan_half, aspect;
    float bmin[3], bmax[3];
};

struct RenderBuffers {
    uint32_t* depth;   // W*H: closest sphere-surface view distance (float bits), 0x7f7f7f7f = none
    float* thick;      // W*H: summed thickness
    float* smoothed;   // W*H: smoothed view distance, 0 = no fluid
    float* ndc;        // W*H: NDC depth of the final image (1 = far)
    float4* rgba;      // W*H: linear colour in [0, 1]
};

}  // namespace mpb

struct mp_render_params;
struct mp_pbf_params;

namespace mpb {

// Host: the camera (column-major 4x4 view and projection) and the frame
// constants of a render.
int render_camera(const mp_render_params& rp, float view[16], float proj[16]);
int make_render_consts(const mp_render_params& rp, const mp_pbf_params& p, uint32_t n, bool sphere_scene,
                       RenderConsts& c);

cudaError_t launch_render(const RenderConsts& c, const RenderBuffers& b, const float4* pos, const float* foam,
                          const SphereState* sphere, cudaStream_t s);

}  // namespace mpb

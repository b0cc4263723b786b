// pbf_render.cu — headless screen-space fluid rendering for sm_100a: the
// reference's Metal render pipeline (engine/src/Engine.cpp:884-1020,
// engine/shaders/Render.metal) as CUDA passes over device image buffers.
// There is no rasteriser here, so each pass finds its own pixels:
//
//   k_splat      fluidDepth* + fluidThicknessFragment (Render.metal:37-103):
//                one thread per particle walks the pixels of its
//                camera-facing disc; the closest sphere-surface view distance
//                wins (atomicMin on the float bits of a positive distance, the
//                same order as the reference's Less depth test on NDC z) and
//                0.05 exp(-4 r^2) is summed into the thickness (FP32; the
//                reference blends into an R16Float target).
//   k_smooth     fluidSmoothFragment (:128-157): masked 9x9 Gaussian.
//   k_composite  fluidCompositeFragment (:164-293), one thread per pixel; the
//                surface normal's screen derivatives are differences within
//                the pixel's 2x2 quad, as a fragment quad computes them.
//   k_wire_box   wireBox* (:296-335): 12 edges, LessEqual against the fluid
//                depth, alpha blend 0.85; one block, edges in order.
//   k_sphere     sphereDraw* (:394-458): opaque, Less, writes depth.
//   k_foam       foam* (:337-389): additive sprites, LessEqual, no depth write.
//   k_saturate   the [0, 1] clamp of the unorm colour target.
// Image layout: row-major, y = 0 on the top row, pixel centres at +0.5.
#include "pbf_render.h"

namespace mpb {
namespace {

constexpr uint32_t kNone = 0x7f7f7f7fu;  // "no fluid" in the splat buffer (memset byte 0x7f)

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ V3 mix(V3 a, V3 b, float t) { return a + (b - a) * t; }

// The unorm target's store: clamp to [0, 1], NaN (the normal of a lone fluid
// pixel whose quad neighbours are all sky) to 0.
__device__ __forceinline__ float unorm(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// The geometry below (view transform, pixel centres, billboard bounds, disc
// coordinates, sphere-surface distance) is written with explicit
// round-to-nearest operations in a fixed order, so which pixels a particle
// covers and the depth it leaves are reproducible exactly.
__device__ __forceinline__ float view_row(const float* v, float4 p) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(v[0], p.x), __fmul_rn(v[1], p.y)), __fmul_rn(v[2], p.z)), v[3]);
}
__device__ __forceinline__ V3 to_view(const RenderConsts& c, float4 p) {
    return v3(view_row(c.view, p), view_row(c.view + 4, p), view_row(c.view + 8, p));
}
__device__ __forceinline__ float ndc_z(const RenderConsts& c, float vz) {
    return __fdiv_rn(__fadd_rn(__fmul_rn(c.p22, vz), c.p23), -vz);
}
__device__ __forceinline__ float pixel_ndc_x(const RenderConsts& c, int x) {
    return __fsub_rn(__fmul_rn(__fdiv_rn(__fadd_rn(float(x), 0.5f), float(c.W)), 2.0f), 1.0f);
}
__device__ __forceinline__ float pixel_ndc_y(const RenderConsts& c, int y) {
    return __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(__fadd_rn(float(y), 0.5f), float(c.H)), 2.0f));
}

// Pixel rectangle covered by the square billboard of view-space centre vc
// and half-size r (camera-facing, so screen-linear); false if empty.
__device__ __forceinline__ bool billboard_pixels(const RenderConsts& c, V3 vc, float r, int& x0, int& x1,
                                                 int& y0, int& y1) {
    const float w = -vc.z, W = float(c.W), H = float(c.H);
    auto sx = [&](float vx) {
        return __fsub_rn(__fmul_rn(__fmul_rn(__fadd_rn(__fdiv_rn(__fmul_rn(c.p00, vx), w), 1.0f), 0.5f), W), 0.5f);
    };
    auto sy = [&](float vy) {
        return __fsub_rn(__fmul_rn(__fmul_rn(__fsub_rn(1.0f, __fdiv_rn(__fmul_rn(c.p11, vy), w)), 0.5f), H), 0.5f);
    };
    x0 = max(int(floorf(sx(__fsub_rn(vc.x, r)))), 0);
    x1 = min(int(ceilf(sx(__fadd_rn(vc.x, r)))), int(c.W) - 1);
    y0 = max(int(floorf(sy(__fadd_rn(vc.y, r)))), 0);
    y1 = min(int(ceilf(sy(__fsub_rn(vc.y, r)))), int(c.H) - 1);
    return x0 <= x1 && y0 <= y1;
}

// Disc coordinate (u, v) in [-1, 1]^2 of pixel (x, y) on the billboard.
__device__ __forceinline__ float disc_u(const RenderConsts& c, V3 vc, float r, int x) {
    return __fdiv_rn(__fsub_rn(__fdiv_rn(__fmul_rn(pixel_ndc_x(c, x), -vc.z), c.p00), vc.x), r);
}
__device__ __forceinline__ float disc_v(const RenderConsts& c, V3 vc, float r, int y) {
    return __fdiv_rn(__fsub_rn(__fdiv_rn(__fmul_rn(pixel_ndc_y(c, y), -vc.z), c.p11), vc.y), r);
}
__device__ __forceinline__ float disc_r2(const RenderConsts& c, V3 vc, float r, int x, int y) {
    const float u = disc_u(c, vc, r, x), v = disc_v(c, vc, r, y);
    return __fadd_rn(__fmul_rn(v, v), __fmul_rn(u, u));
}

__global__ void __launch_bounds__(128) k_splat(RenderConsts c, const float4* __restrict__ pos,
                                               uint32_t* __restrict__ depth, float* __restrict__ thick) {
    const uint32_t i = blockIdx.x * 128 + threadIdx.x;
    if (i >= c.n) return;
    const V3 vc = to_view(c, pos[i]);
    const float w = -vc.z;
    if (!(w > c.znear && w < c.zfar)) return;  // billboard clipped
    int x0, x1, y0, y1;
    if (!billboard_pixels(c, vc, c.radius, x0, x1, y0, y1)) return;
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const float r2 = disc_r2(c, vc, c.radius, x, y);
            if (r2 > 1.0f) continue;
            const float dist = -__fadd_rn(vc.z, __fmul_rn(c.radius, __fsqrt_rn(__fsub_rn(1.0f, r2))));
            const size_t k = size_t(y) * c.W + x;
            atomicMin(&depth[k], __float_as_uint(dist));
            atomicAdd(&thick[k], 0.05f * expf(-r2 * 4.0f));
        }
}

__global__ void __launch_bounds__(256) k_smooth(RenderConsts c, const uint32_t* __restrict__ depth,
                                                float* __restrict__ smoothed) {
    const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
    if (x >= int(c.W) || y >= int(c.H)) return;
    const uint32_t center = depth[size_t(y) * c.W + x];
    if (center == kNone) {
        smoothed[size_t(y) * c.W + x] = 0.0f;
        return;
    }
    const float two_sigma2 = 2.0f * 2.8f * 2.8f;
    float sum = 0.0f, weight = 0.0f;
    for (int dy = -4; dy <= 4; ++dy) {
        const int yy = min(max(y + dy, 0), int(c.H) - 1);
        for (int dx = -4; dx <= 4; ++dx) {
            const int xx = min(max(x + dx, 0), int(c.W) - 1);
            const uint32_t b = depth[size_t(yy) * c.W + xx];
            if (b != kNone) {
                const float w = expf(-float(dx * dx + dy * dy) / two_sigma2);
                sum += __uint_as_float(b) * w;
                weight += w;
            }
        }
    }
    smoothed[size_t(y) * c.W + x] = sum / fmaxf(weight, 1e-6f);
}

__device__ __forceinline__ V3 sun_dir() { return normalize(v3(0.45f, 0.75f, 0.50f)); }

// Procedural sky (Render.metal:183-198).
__device__ V3 sky(V3 d) {
    const V3 zenith = v3(0.18f, 0.42f, 0.78f), horizon = v3(0.85f, 0.91f, 0.97f);
    const V3 ground = v3(0.08f, 0.09f, 0.11f);
    V3 col = d.y >= 0.0f ? mix(horizon, zenith, powf(d.y, 0.55f)) : mix(horizon, ground, powf(-d.y, 0.45f));
    const float sd = fmaxf(dot(d, sun_dir()), 0.0f);
    col = col + v3(1.0f, 0.96f, 0.86f) * (powf(sd, 380.0f) + powf(sd, 6.0f) * 0.18f);
    return col;
}

__device__ __forceinline__ V3 view_pos(const RenderConsts& c, const float* sd, int x, int y) {
    const float d = sd[size_t(y) * c.W + x];
    return v3(pixel_ndc_x(c, x) * c.tan_half * c.aspect * d, pixel_ndc_y(c, y) * c.tan_half * d, -d);
}

__global__ void __launch_bounds__(256) k_composite(RenderConsts c, const float* __restrict__ sdepth,
                                                   const float* __restrict__ thick,
                                                   float4* __restrict__ rgba, float* __restrict__ ndc) {
    const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
    if (x >= int(c.W) || y >= int(c.H)) return;
    const size_t k = size_t(y) * c.W + x;
    const V3 right = v3(c.view[0], c.view[1], c.view[2]), up = v3(c.view[4], c.view[5], c.view[6]);
    const V3 fwd = v3(-c.view[8], -c.view[9], -c.view[10]);
    const float nx = pixel_ndc_x(c, x), ny = pixel_ndc_y(c, y);
    const V3 ray = normalize(fwd + right * (nx * c.tan_half * c.aspect) + up * (ny * c.tan_half));
    const float d = sdepth[k];
    if (d <= 0.0f) {
        const V3 s = sky(ray);
        rgba[k] = make_float4(s.x, s.y, s.z, 1.0f);
        ndc[k] = 1.0f;
        return;
    }
    // screen derivatives within the 2x2 quad (x per row, y per column)
    const int qx = x & ~1, qy = y & ~1;
    const int qx1 = min(qx + 1, int(c.W) - 1), qy1 = min(qy + 1, int(c.H) - 1);
    const V3 vp = view_pos(c, sdepth, x, y);
    const V3 ddx = view_pos(c, sdepth, qx1, y) - view_pos(c, sdepth, qx, y);
    const V3 ddy = view_pos(c, sdepth, x, qy1) - view_pos(c, sdepth, x, qy);
    const V3 nv = normalize(cross(ddy, ddx));
    const V3 n = normalize(right * nv.x + up * nv.y + fwd * (-nv.z));
    const float dn = dot(n, ray);
    const V3 refl = ray - n * (2.0f * dn);
    const float eta = 1.0f / 1.33f;
    const float kk = 1.0f - eta * eta * (1.0f - dn * dn);
    const V3 refr = kk < 0.0f ? v3(0, 0, 0) : ray * eta - n * (eta * dn + sqrtf(kk));
    const V3 refr_sky = sky(sqrtf(dot(refr, refr)) < 1e-4f ? refl : refr);
    const float t = thick[k];
    const V3 transmitted = refr_sky * v3(expf(-2.5f * t), expf(-0.55f * t), expf(-0.25f * t));
    const float cos_i = fmaxf(-dn, 0.0f);
    const float schlick = 0.02f + 0.98f * powf(1.0f - cos_i, 5.0f);
    const V3 fill = sky(n) * (0.18f * (1.0f - schlick));
    const float align = fmaxf(dot(refl, sun_dir()), 0.0f);
    const V3 glint = v3(1.0f, 0.96f, 0.84f) * (powf(align, 320.0f) * 2.5f);
    const V3 col = mix(transmitted, sky(refl), schlick) + fill + glint;
    rgba[k] = make_float4(col.x, col.y, col.z, 1.0f);
    ndc[k] = ndc_z(c, vp.z);
}

__global__ void __launch_bounds__(256) k_saturate(uint32_t n, float4* __restrict__ rgba) {
    const uint32_t k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const float4 v = rgba[k];
    rgba[k] = make_float4(unorm(v.x), unorm(v.y), unorm(v.z), unorm(v.w));
}

// Bounding box: 12 edges (corner bit 0 = x, 1 = y, 2 = z), each rasterised by
// stepping the major axis through pixel centres.  Edges run in order, one
// block, so the blending of shared pixels is deterministic.
__global__ void __launch_bounds__(256) k_wire_box(RenderConsts c, const float* __restrict__ ndc,
                                                  float4* __restrict__ rgba) {
    const uint8_t edges[24] = {0, 1, 1, 3, 3, 2, 2, 0, 4, 5, 5, 7, 7, 6, 6, 4, 0, 4, 1, 5, 2, 6, 3, 7};
    for (int e = 0; e < 12; ++e) {
        float sx[2], sy[2], sz[2];
        V3 pv[2];
        for (int j = 0; j < 2; ++j) {
            const int cn = edges[2 * e + j];
            const float4 p = make_float4((cn & 1) ? c.bmax[0] : c.bmin[0], (cn & 2) ? c.bmax[1] : c.bmin[1],
                                         (cn & 4) ? c.bmax[2] : c.bmin[2], 1.0f);
            pv[j] = to_view(c, p);
        }
        // clip to the near plane in view space
        const float zn = -c.znear;
        bool visible = !(pv[0].z > zn && pv[1].z > zn);
        if (visible) {
            for (int j = 0; j < 2; ++j)
                if (pv[j].z > zn) {
                    const V3 o = pv[1 - j];
                    const float t = (zn - o.z) / (pv[j].z - o.z);
                    pv[j] = o + (pv[j] - o) * t;
                }
            for (int j = 0; j < 2; ++j) {
                const float w = -pv[j].z;
                sx[j] = (c.p00 * pv[j].x / w + 1.0f) * 0.5f * float(c.W);
                sy[j] = (1.0f - c.p11 * pv[j].y / w) * 0.5f * float(c.H);
                sz[j] = ndc_z(c, pv[j].z);
            }
            const bool xmajor = fabsf(sx[1] - sx[0]) >= fabsf(sy[1] - sy[0]);
            const float a0 = xmajor ? sx[0] : sy[0], a1 = xmajor ? sx[1] : sy[1];
            const float lo = fminf(a0, a1), hi = fmaxf(a0, a1);
            const int m0 = int(ceilf(lo - 0.5f)), m1 = int(floorf(hi - 0.5f));
            for (int m = m0 + int(threadIdx.x); m <= m1; m += blockDim.x) {
                const float t = (a1 != a0) ? ((float(m) + 0.5f) - a0) / (a1 - a0) : 0.0f;
                const float other = xmajor ? sy[0] + t * (sy[1] - sy[0]) : sx[0] + t * (sx[1] - sx[0]);
                const int px = xmajor ? m : int(floorf(other)), py = xmajor ? int(floorf(other)) : m;
                if (px < 0 || py < 0 || px >= int(c.W) || py >= int(c.H)) continue;
                const float z = sz[0] + t * (sz[1] - sz[0]);
                const size_t k = size_t(py) * c.W + px;
                if (z <= ndc[k]) {
                    const float4 d = rgba[k];
                    const float a = 0.85f;
                    rgba[k] = make_float4(0.62f * a + d.x * (1.0f - a), 0.72f * a + d.y * (1.0f - a),
                                          0.86f * a + d.z * (1.0f - a), a * a + d.w * (1.0f - a));
                }
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_sphere(RenderConsts c, const SphereState* __restrict__ sphere,
                                                float* __restrict__ ndc, float4* __restrict__ rgba) {
    const SphereState s = *sphere;
    const V3 vc = to_view(c, make_float4(s.c[0], s.c[1], s.c[2], 1.0f));
    if (!(-vc.z > c.znear && -vc.z < c.zfar)) return;
    int x0, x1, y0, y1;
    if (!billboard_pixels(c, vc, s.r, x0, x1, y0, y1)) return;
    const int x = x0 + int(blockIdx.x * 16 + threadIdx.x), y = y0 + int(blockIdx.y * 16 + threadIdx.y);
    if (x > x1 || y > y1) return;
    const float r2 = disc_r2(c, vc, s.r, x, y);
    if (r2 > 1.0f) return;
    const float u = disc_u(c, vc, s.r, x), v = disc_v(c, vc, s.r, y);
    const V3 vp = vc + v3(u * s.r, v * s.r, s.r * sqrtf(1.0f - r2));
    const size_t k = size_t(y) * c.W + x;
    const float z = ndc_z(c, vp.z);
    if (!(z < ndc[k])) return;
    const V3 N = normalize(vp - vc);
    const V3 sw = sun_dir();
    const V3 sunv = normalize(v3(c.view[0] * sw.x + c.view[1] * sw.y + c.view[2] * sw.z,
                                 c.view[4] * sw.x + c.view[5] * sw.y + c.view[6] * sw.z,
                                 c.view[8] * sw.x + c.view[9] * sw.y + c.view[10] * sw.z));
    const V3 V = v3(0, 0, 1);
    const V3 Hh = normalize(sunv + V);
    const float diff = fmaxf(dot(N, sunv), 0.0f);
    const float spec = powf(fmaxf(dot(N, Hh), 0.0f), 80.0f);
    const float fres = powf(1.0f - fmaxf(dot(N, V), 0.0f), 3.0f);
    const V3 col = v3(0.85f, 0.32f, 0.22f) * (0.25f + 0.75f * diff) + v3(1, 1, 1) * (spec * 0.7f) +
                   v3(1.0f, 0.95f, 0.88f) * (fres * 0.18f);
    rgba[k] = make_float4(unorm(col.x), unorm(col.y), unorm(col.z), 1.0f);
    ndc[k] = z;
}

__global__ void __launch_bounds__(128) k_foam(RenderConsts c, const float4* __restrict__ pos,
                                              const float* __restrict__ foam, const float* __restrict__ ndc,
                                              float4* __restrict__ rgba) {
    const uint32_t i = blockIdx.x * 128 + threadIdx.x;
    if (i >= c.n) return;
    const float intensity = foam[i];
    if (intensity < 0.05f) return;
    const V3 vc = to_view(c, pos[i]);
    const float w = -vc.z;
    if (!(w > c.znear && w < c.zfar)) return;
    const float r = c.radius * c.foam_scale;
    int x0, x1, y0, y1;
    if (!billboard_pixels(c, vc, r, x0, x1, y0, y1)) return;
    const float z = ndc_z(c, vc.z);  // flat sprite
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x) {
            const float r2 = disc_r2(c, vc, r, x, y);
            if (r2 > 1.0f) continue;
            const size_t k = size_t(y) * c.W + x;
            if (!(z <= ndc[k])) continue;
            const float f = expf(-r2 * 7.0f) * intensity * 0.65f;
            atomicAdd(&rgba[k].x, f);
            atomicAdd(&rgba[k].y, f);
            atomicAdd(&rgba[k].z, f);
            atomicAdd(&rgba[k].w, f);
        }
}

}  // namespace

cudaError_t launch_render(const RenderConsts& c, const RenderBuffers& b, const float4* pos, const float* foam,
                          const SphereState* sphere, cudaStream_t s) {
    const size_t px = size_t(c.W) * c.H;
    if (px == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(b.depth, 0x7f, px * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.thick, 0, px * 4, s);
    if (e != cudaSuccess) return e;
    if (c.n) k_splat<<<(c.n + 127) / 128, 128, 0, s>>>(c, pos, b.depth, b.thick);
    const dim3 blk(16, 16), grd((c.W + 15) / 16, (c.H + 15) / 16);
    k_smooth<<<grd, blk, 0, s>>>(c, b.depth, b.smoothed);
    k_composite<<<grd, blk, 0, s>>>(c, b.smoothed, b.thick, b.rgba, b.ndc);
    k_saturate<<<uint32_t((px + 255) / 256), 256, 0, s>>>(uint32_t(px), b.rgba);
    if (c.flags & kRenderBox) k_wire_box<<<1, 256, 0, s>>>(c, b.ndc, b.rgba);
    if ((c.flags & kRenderSphere) && sphere) {
        // the sphere's screen rectangle is found on the device; cover the
        // largest it can be (the whole image) with early-exit blocks
        k_sphere<<<grd, blk, 0, s>>>(c, sphere, b.ndc, b.rgba);
    }
    if ((c.flags & kRenderFoam) && foam && c.n) {
        k_foam<<<(c.n + 127) / 128, 128, 0, s>>>(c, pos, foam, b.ndc, b.rgba);
        k_saturate<<<uint32_t((px + 255) / 256), 256, 0, s>>>(uint32_t(px), b.rgba);
    }
    return cudaGetLastError();
}

}  // namespace mpb

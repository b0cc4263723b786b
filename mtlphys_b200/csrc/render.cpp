// render.cpp — host side of the headless renderer: default parameters, the
// camera of Engine::render (engine/src/Engine.cpp:45-67, 893-905) and the
// per-frame constants of pbf_render.cu.
#include <cmath>
#include <cstring>

#include "../../include/mtlphys_b200.h"
#include "host_common.h"
#include "pbf_render.h"

namespace mpb {

namespace {

struct F3 {
    float x, y, z;
};
F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
F3 normalize(F3 a) {
    const float l = std::sqrt(dot(a, a));
    return {a.x / l, a.y / l, a.z / l};
}

}  // namespace

// lookAt(eye, target, up = +y) and perspective(fovY, W / H, near, far) as
// column-major 4x4 matrices (the reference's simd::float4x4 layout).
int render_camera(const mp_render_params& rp, float view[16], float proj[16]) {
    if (rp.size != sizeof(mp_render_params))
        return fail(MP_ERR_INVALID_ARGUMENT, "mp_render_params.size is %u, expected %zu", rp.size,
                    sizeof(mp_render_params));
    if (rp.width == 0 || rp.height == 0 || rp.width > 16384 || rp.height > 16384)
        return fail(MP_ERR_INVALID_ARGUMENT, "image size %ux%u out of range", rp.width, rp.height);
    if (!(rp.z_near > 0.0f && rp.z_far > rp.z_near && rp.fov_y > 0.0f && rp.fov_y < 3.14f &&
          rp.particle_radius > 0.0f))
        return fail(MP_ERR_INVALID_ARGUMENT, "bad camera parameters");
    const F3 eye{rp.eye[0], rp.eye[1], rp.eye[2]}, ctr{rp.target[0], rp.target[1], rp.target[2]};
    const F3 f = normalize(sub(ctr, eye));
    const F3 s = normalize(cross(f, F3{0.0f, 1.0f, 0.0f}));
    const F3 u = cross(s, f);
    if (!std::isfinite(s.x + s.y + s.z + f.x + f.y + f.z))
        return fail(MP_ERR_INVALID_ARGUMENT, "eye and target must differ and not look straight up or down");
    std::memset(view, 0, 16 * sizeof(float));
    view[0] = s.x, view[1] = u.x, view[2] = -f.x;
    view[4] = s.y, view[5] = u.y, view[6] = -f.y;
    view[8] = s.z, view[9] = u.z, view[10] = -f.z;
    view[12] = -dot(s, eye), view[13] = -dot(u, eye), view[14] = dot(f, eye), view[15] = 1.0f;
    const float aspect = float(rp.width) / float(rp.height);
    const float ys = 1.0f / std::tan(rp.fov_y * 0.5f);
    const float xs = ys / aspect;
    const float zs = rp.z_far / (rp.z_near - rp.z_far);
    std::memset(proj, 0, 16 * sizeof(float));
    proj[0] = xs;
    proj[5] = ys;
    proj[10] = zs;
    proj[11] = -1.0f;
    proj[14] = rp.z_near * zs;
    return MP_OK;
}

int make_render_consts(const mp_render_params& rp, const mp_pbf_params& p, uint32_t n, bool sphere_scene,
                       RenderConsts& c) {
    float view[16], proj[16];
    const int rc = render_camera(rp, view, proj);
    if (rc != MP_OK) return rc;
    std::memset(&c, 0, sizeof(c));
    c.W = rp.width;
    c.H = rp.height;
    c.n = n;
    c.flags = rp.flags & (kRenderBox | kRenderFoam);
    if (sphere_scene) c.flags |= rp.flags & kRenderSphere;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 4; ++k) c.view[4 * r + k] = view[4 * k + r];  // column-major -> rows
    c.p00 = proj[0];
    c.p11 = proj[5];
    c.p22 = proj[10];
    c.p23 = proj[14];
    c.znear = rp.z_near;
    c.zfar = rp.z_far;
    c.radius = rp.particle_radius;
    c.foam_scale = rp.foam_radius_scale;
    c.tan_half = std::tan(rp.fov_y * 0.5f);
    c.aspect = float(rp.width) / float(rp.height);
    for (int a = 0; a < 3; ++a) {
        c.bmin[a] = p.bounds_min[a];
        c.bmax[a] = p.bounds_max[a];
    }
    return MP_OK;
}

}  // namespace mpb

extern "C" {

int mp_default_render_params(mp_render_params* rp) {
    if (!rp) return mpb::fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(rp, 0, sizeof(*rp));
    rp->size = sizeof(mp_render_params);
    rp->width = 1280;
    rp->height = 720;
    rp->flags = MP_RENDER_BOX | MP_RENDER_SPHERE | MP_RENDER_FOAM;
    // the app's orbit camera at start-up (app/MetalView.swift:93-96, 218-224):
    // target (0, 1.5, 0), distance 13, azimuth pi/4, elevation 0.40
    const float az = 0.78539816f, el = 0.40f, dist = 13.0f;
    rp->target[1] = 1.5f;
    rp->eye[0] = rp->target[0] + dist * std::cos(el) * std::cos(az);
    rp->eye[1] = rp->target[1] + dist * std::sin(el);
    rp->eye[2] = rp->target[2] + dist * std::cos(el) * std::sin(az);
    rp->fov_y = 1.0f;             // Engine.cpp:893
    rp->z_near = 0.1f;            // Engine.cpp:900
    rp->z_far = 100.0f;
    rp->particle_radius = 0.022f * 1.3f;  // kParticleRadius * 1.3 (Engine.cpp:26, 902)
    rp->foam_radius_scale = 0.25f;        // Render.metal:363
    return MP_OK;
}

int mp_render_camera(const mp_render_params* rp, float view[16], float proj[16]) {
    if (!rp || !view || !proj) return mpb::fail(MP_ERR_INVALID_ARGUMENT, "NULL argument");
    return mpb::render_camera(*rp, view, proj);
}

}  // extern "C"

"""CPU restatement of the reference's screen-space fluid renderer.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA render passes
(mtlphys_b200/csrc/pbf_render.cu); the product never imports it.

It restates Engine::render (engine/src/Engine.cpp:884-1020) and the shader
math of engine/shaders/Render.metal in numpy FP32 (FP64 only where noted),
rasterising the way the CUDA passes do, since there is no graphics pipeline
here (the reference's passes are Metal render pipelines):

  camera            the matrices of mp_render_camera (lookAt / perspective,
                    Engine.cpp:45-67; fovY 1, near 0.1, far 100), billboard
                    radius 1.3 x 0.022 (:893-905)
  depth + thickness fluidDepthVertex/Fragment and fluidThicknessFragment
                    (Render.metal:37-103): every pixel centre inside a
                    particle's camera-facing disc gets the sphere-surface
                    view distance (closest wins) and 0.05 exp(-4 r^2) of
                    thickness (summed; FP32 here, R16Float in the reference)
  smooth            fluidSmoothFragment (:128-157): masked 9x9 Gaussian,
                    sigma 2.8, clamp-to-edge, nearest
  composite         fluidCompositeFragment (:164-293): view position from
                    depth, normal from 2x2-quad finite differences, reflected
                    and refracted sky (:199-217), Beer-Lambert, Schlick
                    Fresnel, sky fill, sun glint; sky where there is no fluid
  box, sphere, foam wireBox (:296-329), sphereDraw (:394-458), foam (:337-389)
                    with the reference's depth tests and blend modes, on an
                    RGBA target clamped to [0, 1] (BGRA8Unorm_sRGB stores
                    linear colour clamped; sRGB encoding is left to output)

Pixel (x, y) has y = 0 on the top row; its centre is (x + 0.5, y + 0.5).
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32
KERNEL_RADIUS, SIGMA = 4, 2.8


def normalize(v):
    v = np.asarray(v, f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        return (v / f32(np.sqrt(np.sum(v * v, axis=-1, keepdims=True, dtype=f32)))).astype(f32)


def unorm(x):
    """The unorm target's store: clamp to [0, 1], NaN to 0."""
    return np.fmin(np.fmax(np.asarray(x, f32), f32(0)), f32(1)).astype(f32)


class Camera:
    """Frame constants of a render.  view, proj: row-major 4x4 (from
    mp_render_camera, so the oracle and the CUDA passes share the camera)."""

    def __init__(self, rp, view, proj, bounds_min=(-3, -3, -3), bounds_max=(3, 6, 3)):
        self.W, self.H = int(rp.width), int(rp.height)
        self.aspect = f32(self.W) / f32(self.H)
        self.view, self.proj = np.asarray(view, f32), np.asarray(proj, f32)
        self.near, self.far = f32(rp.z_near), f32(rp.z_far)
        self.radius = f32(rp.particle_radius)
        self.foam_scale = f32(rp.foam_radius_scale)
        self.tan_half = f32(math.tan(f32(rp.fov_y) * f32(0.5)))
        self.bmin, self.bmax = np.asarray(bounds_min, f32), np.asarray(bounds_max, f32)

    def to_view(self, p):
        p = np.asarray(p, f32)[..., :3]
        V = self.view
        return np.stack([((V[r, 0] * p[..., 0] + V[r, 1] * p[..., 1]) + V[r, 2] * p[..., 2]) + V[r, 3]
                         for r in range(3)], axis=-1).astype(f32)

    def ndc_z(self, vz):
        """clip.z / clip.w of a view-space depth vz (< 0)."""
        P = self.proj
        with np.errstate(divide="ignore", invalid="ignore"):
            return ((P[2, 2] * vz + P[2, 3]) / (-vz)).astype(f32)

    def pixel_ndc(self):
        xs = ((np.arange(self.W, dtype=f32) + f32(0.5)) / f32(self.W)) * f32(2) - f32(1)
        ys = f32(1) - ((np.arange(self.H, dtype=f32) + f32(0.5)) / f32(self.H)) * f32(2)
        return xs, ys


def _discs(cam, centers, radius):
    """For every particle whose billboard plane lies between the near and
    far planes: the pixels whose centres fall inside its disc, with the
    disc coordinate r^2 = |uv|^2.  Yields (index, ys, xs, r2, view centre)."""
    vc = cam.to_view(centers)
    nx, ny = cam.pixel_ndc()
    p00, p11 = cam.proj[0, 0], cam.proj[1, 1]
    W, H = f32(cam.W), f32(cam.H)
    radius = f32(radius)
    for i, c in enumerate(vc):
        cx, cy, cz = c
        w = -cz
        if not (w > cam.near and w < cam.far):
            continue
        x0 = (((p00 * (cx - radius)) / w + f32(1)) * f32(0.5)) * W - f32(0.5)
        x1 = (((p00 * (cx + radius)) / w + f32(1)) * f32(0.5)) * W - f32(0.5)
        y0 = ((f32(1) - (p11 * (cy + radius)) / w) * f32(0.5)) * H - f32(0.5)
        y1 = ((f32(1) - (p11 * (cy - radius)) / w) * f32(0.5)) * H - f32(0.5)
        ia, ib = max(int(math.floor(x0)), 0), min(int(math.ceil(x1)), cam.W - 1)
        ja, jb = max(int(math.floor(y0)), 0), min(int(math.ceil(y1)), cam.H - 1)
        if ia > ib or ja > jb:
            continue
        u = (((nx[ia:ib + 1] * w) / p00 - cx) / radius).astype(f32)
        v = (((ny[ja:jb + 1] * w) / p11 - cy) / radius).astype(f32)
        r2 = (v[:, None] * v[:, None] + u[None, :] * u[None, :]).astype(f32)
        yy, xx = np.nonzero(r2 <= 1)
        if len(yy):
            yield i, yy + ja, xx + ia, r2[yy, xx], c, u[xx], v[yy]


def depth_thickness(cam, centers):
    depth = np.full((cam.H, cam.W), np.inf, f32)
    thick = np.zeros((cam.H, cam.W), f32)
    R = cam.radius
    for _, ys, xs, r2, c, _u, _v in _discs(cam, centers, R):
        z = (-(c[2] + R * np.sqrt(f32(1) - r2))).astype(f32)
        np.minimum.at(depth, (ys, xs), z)
        np.add.at(thick, (ys, xs), (f32(0.05) * np.exp(-r2 * f32(4))).astype(f32))
    depth[np.isinf(depth)] = 0
    return depth, thick


def smooth(depth):
    H, W = depth.shape
    out = np.zeros_like(depth)
    two_s2 = f32(2) * f32(SIGMA) * f32(SIGMA)
    num = np.zeros_like(depth)
    den = np.zeros_like(depth)
    for dy in range(-KERNEL_RADIUS, KERNEL_RADIUS + 1):
        for dx in range(-KERNEL_RADIUS, KERNEL_RADIUS + 1):
            yi = np.clip(np.arange(H) + dy, 0, H - 1)
            xi = np.clip(np.arange(W) + dx, 0, W - 1)
            d = depth[yi][:, xi]
            w = f32(np.exp(-f32(dx * dx + dy * dy) / two_s2))
            m = d > 0
            num = np.where(m, num + d * w, num).astype(f32)
            den = np.where(m, den + w, den).astype(f32)
    out = np.where(depth > 0, num / np.maximum(den, f32(1e-6)), f32(0)).astype(f32)
    return out


def sun_dir():
    return normalize([0.45, 0.75, 0.50])


def sky(d):
    d = np.asarray(d, f32)
    zen, hor, gnd = (np.array(c, f32) for c in ((0.18, 0.42, 0.78), (0.85, 0.91, 0.97), (0.08, 0.09, 0.11)))
    h = d[..., 1:2]
    up = hor + (zen - hor) * np.power(np.maximum(h, 0), f32(0.55))
    dn = hor + (gnd - hor) * np.power(np.maximum(-h, 0), f32(0.45))
    col = np.where(h >= 0, up, dn).astype(f32)
    sd = np.maximum(np.sum(d * sun_dir(), axis=-1, keepdims=True), 0).astype(f32)
    glow = (np.power(sd, f32(380)) + np.power(sd, f32(6)) * f32(0.18)).astype(f32)
    return (col + np.array((1.0, 0.96, 0.86), f32) * glow).astype(f32)


def composite(cam, sdepth, thick):
    """Returns (rgba (H, W, 4) clamped to [0, 1], ndc depth (H, W))."""
    H, W = sdepth.shape
    V = cam.view
    right, up, fwd = V[0, :3].copy(), V[1, :3].copy(), -V[2, :3]
    nx, ny = cam.pixel_ndc()
    NX, NY = np.meshgrid(nx, ny)
    ta = cam.tan_half * cam.aspect
    ray = normalize(fwd + right * (NX * ta)[..., None] + up * (NY * cam.tan_half)[..., None])
    d = sdepth
    vp = np.stack([NX * ta * d, NY * cam.tan_half * d, -d], axis=-1).astype(f32)
    # derivatives on 2x2 quads (per row for x, per column for y)
    qx = np.arange(W) & ~1
    qy = np.arange(H) & ~1
    qx1 = np.minimum(qx + 1, W - 1)
    qy1 = np.minimum(qy + 1, H - 1)
    ddx = (vp[:, qx1] - vp[:, qx]).astype(f32)
    ddy = (vp[qy1, :] - vp[qy, :]).astype(f32)
    n_view = normalize(np.cross(ddy, ddx).astype(f32))
    n = normalize(right * n_view[..., 0:1] + up * n_view[..., 1:2] + fwd * (-n_view[..., 2:3]))
    dn = np.sum(n * ray, axis=-1, keepdims=True).astype(f32)
    refl = (ray - f32(2) * dn * n).astype(f32)
    eta = f32(1.0) / f32(1.33)
    k = (f32(1) - eta * eta * (f32(1) - dn * dn)).astype(f32)
    refr = np.where(k < 0, f32(0), eta * ray - (eta * dn + np.sqrt(np.maximum(k, 0))) * n).astype(f32)
    refr_len = np.sqrt(np.sum(refr * refr, axis=-1, keepdims=True))
    refr_sky = sky(np.where(refr_len < 1e-4, refl, refr))
    alpha = np.array((2.5, 0.55, 0.25), f32)
    transmitted = (refr_sky * np.exp(-alpha * thick[..., None])).astype(f32)
    cos_i = np.maximum(-dn, 0).astype(f32)
    schlick = (f32(0.02) + f32(0.98) * np.power(f32(1) - cos_i, f32(5))).astype(f32)
    refl_sky = sky(refl)
    fill = (sky(n) * f32(0.18) * (f32(1) - schlick)).astype(f32)
    align = np.maximum(np.sum(refl * sun_dir(), axis=-1, keepdims=True), 0).astype(f32)
    glint = (np.array((1.0, 0.96, 0.84), f32) * np.power(align, f32(320)) * f32(2.5)).astype(f32)
    col = (transmitted + (refl_sky - transmitted) * schlick + fill + glint).astype(f32)
    fluid = (d > 0)[..., None]
    rgb = np.where(fluid, col, sky(ray))
    rgba = np.concatenate([unorm(rgb), np.ones((H, W, 1), f32)], axis=-1).astype(f32)
    ndc = np.where(d > 0, cam.ndc_z(-d), f32(1)).astype(f32)
    return rgba, ndc


def wire_box(cam, rgba, ndc):
    """The 12 box edges in order (corner bit 0 = x, 1 = y, 2 = z), clipped at
    the near plane, rasterised by stepping the major axis through pixel
    centres; LessEqual against ndc, alpha blend 0.85 (Render.metal:296-335)."""
    edges = [0, 1, 1, 3, 3, 2, 2, 0, 4, 5, 5, 7, 7, 6, 6, 4, 0, 4, 1, 5, 2, 6, 3, 7]
    P = cam.proj
    for e in range(12):
        pv = []
        for j in range(2):
            cn = edges[2 * e + j]
            p = np.array([cam.bmax[0] if cn & 1 else cam.bmin[0], cam.bmax[1] if cn & 2 else cam.bmin[1],
                          cam.bmax[2] if cn & 4 else cam.bmin[2]], f32)
            pv.append(cam.to_view(p))
        zn = -cam.near
        if pv[0][2] > zn and pv[1][2] > zn:
            continue
        for j in range(2):
            if pv[j][2] > zn:
                o = pv[1 - j]
                t = (zn - o[2]) / (pv[j][2] - o[2])
                pv[j] = (o + (pv[j] - o) * f32(t)).astype(f32)
        sx = [(P[0, 0] * v[0] / (-v[2]) + f32(1)) * f32(0.5) * f32(cam.W) for v in pv]
        sy = [(f32(1) - P[1, 1] * v[1] / (-v[2])) * f32(0.5) * f32(cam.H) for v in pv]
        sz = [cam.ndc_z(v[2]) for v in pv]
        xmajor = abs(sx[1] - sx[0]) >= abs(sy[1] - sy[0])
        a0, a1 = (sx if xmajor else sy)
        lo, hi = min(a0, a1), max(a0, a1)
        for m in range(int(math.ceil(lo - 0.5)), int(math.floor(hi - 0.5)) + 1):
            t = f32(((f32(m) + f32(0.5)) - a0) / (a1 - a0)) if a1 != a0 else f32(0)
            other = (sy[0] + t * (sy[1] - sy[0])) if xmajor else (sx[0] + t * (sx[1] - sx[0]))
            px, py = (m, int(math.floor(other))) if xmajor else (int(math.floor(other)), m)
            if px < 0 or py < 0 or px >= cam.W or py >= cam.H:
                continue
            z = sz[0] + t * (sz[1] - sz[0])
            if z <= ndc[py, px]:
                d = rgba[py, px].copy()
                a = f32(0.85)
                rgba[py, px] = [f32(0.62) * a + d[0] * (1 - a), f32(0.72) * a + d[1] * (1 - a),
                                f32(0.86) * a + d[2] * (1 - a), a * a + d[3] * (1 - a)]


def sphere_pass(cam, rgba, ndc, sphere):
    """Opaque Phong sphere (Render.metal:394-458), Less, writes depth."""
    c = np.asarray(sphere[:3], f32)
    r = f32(sphere[6])
    sw = sun_dir()
    V = cam.view
    sunv = normalize(np.array([np.dot(V[k, :3], sw) for k in range(3)], f32))
    Hh = normalize(sunv + np.array([0, 0, 1], f32))
    for _, ys, xs, r2, vc, u, v in _discs(cam, c[None, :], r):
        vp = np.stack([vc[0] + u * r, vc[1] + v * r, vc[2] + r * np.sqrt(f32(1) - r2)], -1).astype(f32)
        z = cam.ndc_z(vp[:, 2])
        ok = z < ndc[ys, xs]
        N = normalize(vp - vc)
        diff = np.maximum(N @ sunv, 0)
        spec = np.power(np.maximum(N @ Hh, 0), f32(80))
        fres = np.power(f32(1) - np.maximum(N[:, 2], 0), f32(3))
        col = (np.array((0.85, 0.32, 0.22), f32) * (f32(0.25) + f32(0.75) * diff)[:, None]
               + (spec * f32(0.7))[:, None] + np.array((1.0, 0.95, 0.88), f32) * (fres * f32(0.18))[:, None])
        rgba[ys[ok], xs[ok], :3] = unorm(col[ok])
        rgba[ys[ok], xs[ok], 3] = 1
        ndc[ys[ok], xs[ok]] = z[ok]


def foam_pass(cam, rgba, ndc, centers, foam):
    """Additive foam sprites (Render.metal:337-389): quarter-size flat
    billboards of particles with intensity >= 0.05, LessEqual, no depth
    write; the target clamps to [0, 1]."""
    keep = np.nonzero(np.asarray(foam, f32) >= f32(0.05))[0]
    r = cam.radius * cam.foam_scale
    for j, ys, xs, r2, vc, _u, _v in _discs(cam, np.asarray(centers, f32)[keep], r):
        z = cam.ndc_z(vc[2])
        ok = z <= ndc[ys, xs]
        f = (np.exp(-r2 * f32(7)) * f32(foam[keep[j]]) * f32(0.65)).astype(f32)
        np.add.at(rgba, (ys[ok], xs[ok]), f[ok][:, None])
    rgba[...] = unorm(rgba)


def render(cam, positions, foam=None, sphere=None, flags=7):
    """All passes; returns dict of rgba, ndc, depth, smoothed, thickness."""
    depth, thick = depth_thickness(cam, positions)
    sm = smooth(depth)
    rgba, ndc = composite(cam, sm, thick)
    if flags & 1:
        wire_box(cam, rgba, ndc)
    if (flags & 2) and sphere is not None:
        sphere_pass(cam, rgba, ndc, sphere)
    if (flags & 4) and foam is not None:
        foam_pass(cam, rgba, ndc, positions, foam)
    return {"rgba": rgba, "ndc": ndc, "depth": depth, "smoothed": sm, "thickness": thick}

"""Known answers for the render oracle (oracle/render_ref.py), derived by hand
from the shader formulas of the reference's engine/shaders/Render.metal.

The render passes cannot be run from the reference's own code here (its
fragment shaders need Metal's rasteriser, samplers and screen derivatives),
so each pass of the restatement is pinned instead against values worked out
in this file with plain float64 math: a single particle's depth and
thickness profile (Render.metal:37-103), the masked 9x9 Gaussian with
sigma 2.8 and clamp-to-edge sampling (:128-157), the procedural sky at the
zenith, nadir, horizon and sun (:190-209), the composite of a flat sheet of
fluid facing the camera and of a tilted one (refraction, Beer-Lambert,
Schlick, sky fill, glint; :217-293) and the foam sprite falloff
(:337-389).  Runs without a GPU."""
import math
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import render_ref as R

f32 = np.float32


def camera(W=41, H=31, fov=1.0, near=0.1, far=100.0, radius=0.05, foam_scale=0.25):
    """Camera at the origin looking down -z (view = identity), Metal-style
    perspective with depth in [0, 1]."""
    rp = SimpleNamespace(width=W, height=H, z_near=near, z_far=far, particle_radius=radius,
                         foam_radius_scale=foam_scale, fov_y=fov)
    t = math.tan(0.5 * fov)
    aspect = W / H
    P = np.zeros((4, 4), f32)
    P[0, 0] = 1.0 / (aspect * t)
    P[1, 1] = 1.0 / t
    P[2, 2] = far / (near - far)
    P[2, 3] = near * far / (near - far)
    P[3, 2] = -1.0
    return R.Camera(rp, np.eye(4, dtype=f32), P), P


def pixel_ndc(i, n):
    return (i + 0.5) / n * 2.0 - 1.0


# ---- depth and thickness: fluidDepthFragment / fluidThicknessFragment -------------

def test_single_particle_depth_and_thickness_profile():
    d, rad = 2.0, 0.05
    cam, P = camera(radius=rad)
    depth, thick = R.depth_thickness(cam, np.array([[0.0, 0.0, -d, 1.0]], f32))
    W, H = cam.W, cam.H
    cx, cy = W // 2, H // 2  # odd sizes: the centre pixel looks straight down -z
    # disc centre: the sphere's front surface, d - R; thickness 0.05 exp(0)
    assert depth[cy, cx] == pytest.approx(d - rad, rel=1e-6)
    assert thick[cy, cx] == pytest.approx(0.05, rel=1e-6)
    # along the row through the centre: u = ndc_x w / P00 / R, depth
    # d - R sqrt(1 - u^2), thickness 0.05 exp(-4 u^2); nothing outside the disc
    for x in range(W):
        u = pixel_ndc(x, W) * d / float(P[0, 0]) / rad
        if u * u <= 1.0:
            assert depth[cy, x] == pytest.approx(d - rad * math.sqrt(1.0 - u * u), rel=1e-6)
            assert thick[cy, x] == pytest.approx(0.05 * math.exp(-4.0 * u * u), rel=1e-5)
        else:
            assert depth[cy, x] == 0.0 and thick[cy, x] == 0.0
    # the covered pixels form the projected disc: |uv| <= 1 for every pixel centre
    ys, xs = np.nonzero(depth > 0)
    u = np.array([pixel_ndc(x, W) for x in xs]) * d / float(P[0, 0]) / rad
    v = np.array([-pixel_ndc(y, H) for y in ys]) * d / float(P[1, 1]) / rad
    assert (u * u + v * v <= 1.0 + 1e-6).all()
    inside = sum(1 for y in range(H) for x in range(W)
                 if (pixel_ndc(x, W) * d / float(P[0, 0]) / rad) ** 2
                 + (pixel_ndc(y, H) * d / float(P[1, 1]) / rad) ** 2 <= 1.0 - 1e-6)
    assert len(ys) >= inside


def test_closest_particle_wins_and_thickness_adds():
    cam, _ = camera()
    depth, thick = R.depth_thickness(cam, np.array([[0, 0, -3.0, 1], [0, 0, -2.0, 1]], f32))
    cy, cx = cam.H // 2, cam.W // 2
    assert depth[cy, cx] == pytest.approx(2.0 - 0.05, rel=1e-6)
    assert thick[cy, cx] == pytest.approx(0.10, rel=1e-6)


def test_particles_outside_the_depth_range_are_dropped():
    cam, _ = camera()
    depth, thick = R.depth_thickness(cam, np.array([[0, 0, 1.0, 1], [0, 0, -0.05, 1], [0, 0, -200.0, 1]], f32))
    assert not depth.any() and not thick.any()


# ---- masked 9x9 Gaussian, sigma 2.8: fluidSmoothFragment ------------------------------

def gauss(dx, dy):
    return math.exp(-(dx * dx + dy * dy) / (2.0 * 2.8 * 2.8))


def test_smooth_keeps_a_lone_pixel_and_a_constant_image():
    img = np.zeros((15, 17), f32)
    img[7, 8] = 3.25
    out = R.smooth(img)
    assert out[7, 8] == pytest.approx(3.25, rel=1e-6)
    assert np.count_nonzero(out) == 1  # sky stays sky
    const = np.full((9, 9), 1.5, f32)
    np.testing.assert_allclose(R.smooth(const), 1.5, rtol=1e-6)


def test_smooth_weights_two_pixels_by_the_gaussian():
    img = np.zeros((20, 20), f32)
    a, b = 2.0, 5.0
    img[10, 10], img[12, 13] = a, b  # offset (dx, dy) = (3, 2): inside the 9x9 window
    out = R.smooth(img)
    w = gauss(3, 2)
    assert out[10, 10] == pytest.approx((a + b * w) / (1.0 + w), rel=1e-6)
    assert out[12, 13] == pytest.approx((b + a * w) / (1.0 + w), rel=1e-6)
    img[12, 13], img[10, 15] = 0.0, b  # offset (5, 0): outside the window, no influence
    out = R.smooth(img)
    assert out[10, 10] == pytest.approx(a, rel=1e-6)


def test_smooth_clamps_samples_at_the_edge():
    """One row: every vertical offset and every offset left of x = 0 samples
    the edge pixels again (clamp to edge)."""
    img = np.zeros((1, 12), f32)
    a, b = 1.0, 4.0
    img[0, 0], img[0, 1] = a, b
    out = R.smooth(img)
    wa = sum(gauss(dx, dy) for dx in range(-4, 1) for dy in range(-4, 5))
    wb = sum(gauss(1, dy) for dy in range(-4, 5))
    assert out[0, 0] == pytest.approx((a * wa + b * wb) / (wa + wb), rel=1e-5)


# ---- procedural sky: skyColor ------------------------------------------------------------

ZEN, HOR, GND = (0.18, 0.42, 0.78), (0.85, 0.91, 0.97), (0.08, 0.09, 0.11)
SUN = np.array([0.45, 0.75, 0.50]) / math.sqrt(0.45 ** 2 + 0.75 ** 2 + 0.50 ** 2)


def sky_by_hand(d):
    d = np.asarray(d, float) / np.linalg.norm(d)
    h = d[1]
    base = [hz + (z - hz) * max(h, 0.0) ** 0.55 if h >= 0 else hz + (g - hz) * (-h) ** 0.45
            for z, hz, g in zip(ZEN, HOR, GND)]
    sd = max(float(d @ SUN), 0.0)
    glow = sd ** 380 + sd ** 6 * 0.18
    return np.array(base) + np.array((1.0, 0.96, 0.86)) * glow


@pytest.mark.parametrize("d", [(0, 1, 0), (0, -1, 0), (1, 0, 0), (0, 0, 1), (0, 0, -1), tuple(SUN),
                               (0.3, 0.2, -0.9), (-0.5, -0.4, 0.2)])
def test_sky_colour(d):
    got = R.sky(R.normalize(np.array(d, f32)))
    # pow(sd, 380) near the sun multiplies the FP32 rounding of sd (~6e-8) by 380
    sd = max(float(np.asarray(d) @ SUN) / float(np.linalg.norm(d)), 0.0)
    rtol = 2e-5 + 380 * 1.2e-7 * sd ** 379
    np.testing.assert_allclose(got, sky_by_hand(d), rtol=rtol, atol=2e-6)


def test_sky_at_known_directions():
    np.testing.assert_allclose(R.sky(np.array([0, -1, 0], f32)), GND, rtol=1e-6)  # nadir: ground, no sun
    z = R.sky(np.array([0, 1, 0], f32))  # zenith: sun halo only (0.744^380 ~ 1e-49)
    np.testing.assert_allclose(z, np.array(ZEN) + np.array((1, 0.96, 0.86)) * 0.18 * SUN[1] ** 6, rtol=1e-5)
    s = R.sky(SUN.astype(f32))  # looking at the sun: core 1 + halo 0.18 (core to 380 ulps)
    assert s[0] == pytest.approx(HOR[0] + (ZEN[0] - HOR[0]) * SUN[1] ** 0.55 + 1.18, rel=6e-5)


# ---- composite: fluidCompositeFragment ---------------------------------------------------

@pytest.mark.parametrize("t", [0.0, 0.4, 3.0])
def test_composite_of_a_flat_sheet_facing_the_camera(t):
    """A constant depth image is a plane facing the camera: at the centre pixel
    the view ray is -z and the normal +z, so cos_i = 1, Schlick = F0 = 0.02,
    the reflected ray is +z, the refracted ray (eta = 1/1.33) goes on along
    -z, the transmitted sky is attenuated by exp(-(2.5, 0.55, 0.25) t), the
    sky fill is sky(+z) 0.18 (1 - 0.02) and the glint pow(max(refl.sun, 0),
    320) 2.5 is negligible."""
    cam, _ = camera()
    H, W = cam.H, cam.W
    depth = np.full((H, W), 2.0, f32)
    thick = np.full((H, W), t, f32)
    rgba, ndc = R.composite(cam, depth, thick)
    cy, cx = H // 2, W // 2
    refl_sky = sky_by_hand((0, 0, 1))
    trans = sky_by_hand((0, 0, -1)) * np.exp(-np.array((2.5, 0.55, 0.25)) * t)
    schlick = 0.02
    glint = np.array((1.0, 0.96, 0.84)) * max(SUN[2], 0.0) ** 320 * 2.5
    want = trans + (refl_sky - trans) * schlick + refl_sky * 0.18 * (1 - schlick) + glint
    np.testing.assert_allclose(rgba[cy, cx, :3], np.clip(want, 0, 1), rtol=1e-5, atol=1e-6)
    assert rgba[cy, cx, 3] == 1.0
    # NDC depth of the sheet: (P22 (-d) + P23) / d
    P = cam.proj
    assert ndc[cy, cx] == pytest.approx((-float(P[2, 2]) * 2.0 + float(P[2, 3])) / 2.0, rel=1e-6)


def test_composite_shows_sky_where_there_is_no_fluid():
    cam, _ = camera()
    rgba, ndc = R.composite(cam, np.zeros((cam.H, cam.W), f32), np.zeros((cam.H, cam.W), f32))
    cy, cx = cam.H // 2, cam.W // 2
    np.testing.assert_allclose(rgba[cy, cx, :3], np.clip(sky_by_hand((0, 0, -1)), 0, 1), rtol=1e-5)
    assert (ndc == 1.0).all()


def test_schlick_at_oblique_incidence():
    """Fresnel term 0.02 + 0.98 (1 - cos_i)^5 (Render.metal:266) on a plane
    tilted about the x axis, read back from the composite: a sheet thick
    enough to transmit nothing leaves the reflected sky, the fill and the
    glint; a thin sheet adds the transmitted sky times (1 - Schlick)."""
    cam, _ = camera(W=41, H=41)
    H, W = cam.H, cam.W
    k = 0.8
    ys = np.array([-pixel_ndc(y, H) for y in range(H)]) * math.tan(0.5)
    depth = np.repeat((2.0 / (1.0 + k * ys))[:, None], W, axis=1).astype(f32)
    a, _ = R.composite(cam, depth, np.zeros((H, W), f32))
    b, _ = R.composite(cam, depth, np.full((H, W), 50.0, f32))
    cy, cx = H // 2, W // 2
    # the view point (ny tan d, -d) with d (1 + k ny tan) = 2 lies on the plane
    # z = k y - 2, whose normal towards the camera is (0, -k, 1)/|.|; the view
    # ray at the centre is -z
    n = np.array([0.0, -k, 1.0]) / math.hypot(1.0, k)
    cos_i = n[2]
    schlick = 0.02 + 0.98 * (1.0 - cos_i) ** 5
    refl = np.array([0.0, 0.0, -1.0]) + 2.0 * cos_i * n
    refl_sky = sky_by_hand(refl)
    fill = sky_by_hand(n) * 0.18 * (1 - schlick)
    glint = np.array((1.0, 0.96, 0.84)) * max(float(refl @ SUN), 0.0) ** 320 * 2.5
    # thick sheet (t = 50): exp(-alpha t) < 4e-6, nothing transmitted
    for ch in range(3):
        want_b = refl_sky[ch] * schlick + fill[ch] + glint[ch]
        assert abs(b[cy, cx, ch] - want_b) < 1e-5 + 1e-5 * abs(want_b) + math.exp(-0.25 * 50.0)
    # thin sheet minus thick sheet = transmitted (1 - schlick)
    d_ab = a[cy, cx, :3] - b[cy, cx, :3]
    eta = 1.0 / 1.33
    ray = np.array([0.0, 0.0, -1.0])
    dn = float(n @ ray)
    kk = 1.0 - eta * eta * (1.0 - dn * dn)
    refr = eta * ray - (eta * dn + math.sqrt(kk)) * n
    trans = sky_by_hand(refr) * (1.0 - schlick)
    np.testing.assert_allclose(d_ab, trans - sky_by_hand(refr) * np.exp(-np.array((2.5, 0.55, 0.25)) * 50.0)
                               * (1.0 - schlick), rtol=1e-4, atol=1e-5)


# ---- foam sprites: foamVertex / foamFragment ------------------------------------------------

def test_foam_sprite_falloff_and_depth_test():
    cam, P = camera(radius=0.2, foam_scale=0.25)
    rad = 0.2 * 0.25
    d = 2.0
    W, H = cam.W, cam.H
    rgba = np.zeros((H, W, 4), f32)
    ndc = np.ones((H, W), f32)
    f = 0.8
    R.foam_pass(cam, rgba, ndc, np.array([[0, 0, -d, 1]], f32), np.array([f], f32))
    cy, cx = H // 2, W // 2
    assert rgba[cy, cx, 0] == pytest.approx(0.65 * f, rel=1e-6)  # exp(0) f 0.65, added to every channel
    assert rgba[cy, cx, 3] == pytest.approx(0.65 * f, rel=1e-6)
    for x in range(W):
        u = pixel_ndc(x, W) * d / float(P[0, 0]) / rad
        want = 0.65 * f * math.exp(-7.0 * u * u) if u * u <= 1.0 else 0.0
        assert rgba[cy, x, 1] == pytest.approx(want, rel=1e-5, abs=1e-7)
    # below the 0.05 intensity threshold nothing is drawn; behind a nearer surface neither
    rgba2 = np.zeros((H, W, 4), f32)
    R.foam_pass(cam, rgba2, ndc, np.array([[0, 0, -d, 1]], f32), np.array([0.049], f32))
    assert not rgba2.any()
    near = np.full((H, W), cam.ndc_z(f32(-1.0)), f32)
    rgba3 = np.zeros((H, W, 4), f32)
    R.foam_pass(cam, rgba3, near, np.array([[0, 0, -d, 1]], f32), np.array([f], f32))
    assert not rgba3.any()

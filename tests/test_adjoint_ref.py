"""The FP64 numpy adjoint restatement (oracle/adjoint_ref.py) on CPU: its
forward step equals the C++ FP64 oracle, and its vector-Jacobian product
equals central finite differences of that forward step."""
import numpy as np
import pytest

from mtlphys_b200 import configs
from oracle import adjoint_ref as A
from oracle import oracle as O

DT = 1.0 / 120.0


def scene(side, origin, k=0.1, eps=100.0, jitter=0.01, vel=0.0, seed=1, sphere_radius=None,
          spacing=0.5):
    p = configs.base_params(3)
    p.scorr_k = k
    p.epsilon = eps
    if sphere_radius is not None:
        p.sphere_radius = sphere_radius
    d = configs.lattice((side,) * 3, origin, seed, spacing=spacing * configs.H,
                        jitter=jitter * configs.H)
    x = O.seed_scene(p, 0, side ** 3, d)[:, :3].astype(np.float64)
    v = np.random.default_rng(seed).normal(0.0, vel, size=x.shape)
    return p, x, v


CASES = {
    # name: (scene kwargs, sphere state before the advance or None)
    "floor_friction": (dict(side=6, origin=(2.0, 0.03, 2.0), vel=0.5), None),
    "corner_walls": (dict(side=6, origin=(0.03, 0.03, 2.0), vel=0.5, jitter=0.1), None),
    "violent_capped": (dict(side=6, origin=(2.0, 3.0, 2.0), vel=3.0, jitter=0.3), None),
    "sphere_push": (dict(side=6, origin=(2.0, 0.03, 2.0), vel=0.2, sphere_radius=0.12),
                    [2.12, 0.15, 2.12, 0.0, -1.0, 0.0, 0.12]),
    "gentle": (dict(side=6, origin=(2.0, 3.0, 2.0), k=1e-4, eps=1e4, vel=0.1), None),
    # ~110 candidates per stencil row: rows longer than 32 candidates
    "crowded": (dict(side=9, origin=(2.0, 3.0, 2.0), k=1e-4, eps=1e5, vel=0.1, spacing=0.3), None),
}


def _advanced(p, sphere):
    if sphere is None:
        return None
    s = np.array(sphere, np.float64)
    A.sphere_advance(p, DT, s)
    return s


@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_equals_the_fp64_oracle(name):
    kw, sphere = CASES[name]
    p, x, v = scene(**kw)
    c = A.consts(p, DT)
    X, V, _ = A.forward(c, x, v, _advanced(p, sphere))
    xo, vo = x.copy(), v.copy()
    if sphere is None:
        O.step_f64(p, DT, xo, vo)
    else:
        O.step_f64(p, DT, xo, vo, np.array(sphere, np.float64))
    np.testing.assert_allclose(X, xo, rtol=0, atol=1e-12)
    np.testing.assert_allclose(V, vo, rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", sorted(CASES))
def test_vjp_equals_central_differences(name):
    kw, sphere = CASES[name]
    p, x, v = scene(**kw)
    c = A.consts(p, DT)
    s7 = _advanced(p, sphere)
    rng = np.random.default_rng(9)
    X, V, tape = A.forward(c, x, v, s7)
    wx, wv = rng.normal(size=X.shape), rng.normal(size=X.shape)
    loss = lambda XV: float(np.sum(wx * XV[0]) + np.sum(wv * XV[1]))
    xb, vb, kb, cb, rb = A.adjoint(c, tape, wx, wv)
    ux, uv = rng.normal(size=X.shape), rng.normal(size=X.shape)
    e = 1e-7
    fd = (loss(A.forward(c, x + e * ux, v + e * uv, s7)) - loss(A.forward(c, x - e * ux, v - e * uv, s7))) / (2 * e)
    an = float(np.sum(xb * ux) + np.sum(vb * uv))
    assert abs(fd - an) <= 1e-4 * abs(fd)
    ek = e * max(abs(c["k"]), 1e-3)
    fdk = (loss(A.forward(c, x, v, s7, k=c["k"] + ek)) - loss(A.forward(c, x, v, s7, k=c["k"] - ek))) / (2 * ek)
    assert abs(fdk - kb) <= 1e-4 * abs(fdk)
    if s7 is not None:
        for a, an_s in ((1, cb[1]), (6, rb)):
            sp, sm = s7.copy(), s7.copy()
            sp[a] += e
            sm[a] -= e
            fds = (loss(A.forward(c, x, v, sp)) - loss(A.forward(c, x, v, sm))) / (2 * e)
            assert abs(fds - an_s) <= 1e-4 * abs(fds)


def test_sphere_kinematics_adjoint_equals_central_differences():
    p = configs.base_params(3)
    p.set(bounds_min=(0.0, 0.0, 0.0), bounds_max=(1.0, 1.0, 1.0))
    rng = np.random.default_rng(4)
    w = rng.normal(size=7)
    for s0 in ([0.5, 0.5, 0.5, 0.3, -2.0, 0.1, 0.2],    # free flight
               [0.5, 0.205, 0.81, 0.0, -3.0, 2.0, 0.2]):  # floor and wall bounces
        s0 = np.array(s0)

        def run(s):
            s = s.copy()
            recs = [A.sphere_advance(p, DT, s) for _ in range(5)]
            return s, recs

        s1, recs = run(s0)
        g = w.copy()
        for rec in reversed(recs):
            g = A.sphere_advance_adjoint(p, DT, rec, g)
        for a in range(7):
            e = 1e-7
            sp, sm = s0.copy(), s0.copy()
            sp[a] += e
            sm[a] -= e
            fd = (np.dot(w, run(sp)[0]) - np.dot(w, run(sm)[0])) / (2 * e)
            assert abs(fd - g[a]) <= 1e-6 * max(1.0, abs(fd)), (s0, a, fd, g[a])

"""Adjoint of the PBF step on the GPU (mp_batch_rollout_*, the
torch.autograd.Function in mtlphys_b200.autograd).

  * one step: the CUDA adjoint equals the FP64 numpy adjoint restatement
    (oracle/adjoint_ref.py, itself pinned to the C++ oracle and to finite
    differences by test_adjoint_ref.py) on the same FP32 input state;
  * rollouts: gradients through 60 checkpointed steps equal central finite
    differences of FP64 oracle rollouts within 1e-3 relative (directional
    derivative for the per-particle initial velocities, dL/dk for s_corr k,
    dL/d v0 for the sphere's initial speed), and equal the FP64 numpy
    adjoint chained over the same steps;
  * the checkpoint interval does not change the gradients; the state after
    the backward pass is the state the forward pass ended in.

Conditioning.  The benchmark parameters (s_corr k = 0.1, CFM epsilon = 100)
make these scenes explode within a few steps; finite differences of the FP64
oracle itself then do not converge beyond one step, so the rollout checks
run the same geometry at k = 1e-4 and a softer constraint (epsilon 1e4 or
1e5), where they converge to six or more digits.  Single steps are also
checked at k = 0.1.
"""
import numpy as np
import pytest

from mtlphys_b200 import _abi, configs

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def _torch():
    import torch

    return torch


def make_batch(params, descs, counts, scenes=None, dts=None):
    from mtlphys_b200.batch import Batch

    b = Batch(0)
    b.reset(counts, params, dts or [DT] * len(counts), scenes, descs)
    return b


# ---- one step against the numpy restatement ---------------------------------------

from test_adjoint_ref import CASES, scene  # noqa: E402


@pytest.mark.parametrize("name", sorted(CASES))
def test_one_step_adjoint_matches_the_fp64_restatement(cuda, name):
    one_step_check(name)


@pytest.mark.parametrize("name,iterations", [("floor_friction", 0), ("floor_friction", 1),
                                             ("sphere_push", 0), ("sphere_push", 1)])
def test_one_step_adjoint_with_zero_and_one_solver_iterations(cuda, name, iterations):
    """No solver pass (predict + finalize only) and a single one."""
    one_step_check(name, iterations)


def one_step_check(name, iterations=None):
    from oracle import adjoint_ref as A

    torch = _torch()
    kw, sphere = CASES[name]
    p, x, v = scene(**kw)
    if iterations is not None:
        p.solver_iterations = iterations
    n = len(x)
    d = configs.lattice((kw["side"],) * 3, kw["origin"], 1)
    sid = _abi.MP_SCENE_SPHERE_DROP if sphere is not None else _abi.MP_SCENE_CUBE_DROP
    b = make_batch([p], [d], [n], [sid])
    dev = torch.device("cuda", 0)
    pos0 = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    vel0 = torch.zeros_like(pos0)
    pos0[:, :3] = torch.tensor(x, dtype=torch.float32)
    vel0[:, :3] = torch.tensor(v, dtype=torch.float32)
    b.tensor(_abi.MP_BUF_POSITIONS).copy_(pos0)
    b.tensor(_abi.MP_BUF_VELOCITIES).copy_(vel0)
    if sphere is not None:
        b.set_sphere(0, sphere[:3], sphere[3:6], sphere[6])
    b.rollout_forward(1, 1)
    rng = np.random.default_rng(9)
    wx, wv = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    gp = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    gv = torch.zeros_like(gp)
    gp[:, :3] = torch.tensor(wx, dtype=torch.float32)
    gv[:, :3] = torch.tensor(wv, dtype=torch.float32)
    dp, dv, ds = b.rollout_backward(gp, gv)
    torch.cuda.synchronize()
    assert b.check_errors() == 0
    # the same step in FP64 from the same FP32 state
    c = A.consts(p, DT)
    s7 = None
    if sphere is not None:
        s7 = np.array(sphere, np.float64)
        A.sphere_advance(p, DT, s7)
    xin = pos0[:, :3].double().cpu().numpy()
    vin = vel0[:, :3].double().cpu().numpy()
    _, _, tape = A.forward(c, xin, vin, s7)
    xb, vb, kb, cb, rb = A.adjoint(c, tape, wx, wv)
    rel = lambda a, r: np.linalg.norm(a - r) / np.linalg.norm(r)
    assert rel(dp[:, :3].double().cpu().numpy(), xb) < 1e-3
    assert rel(dv[:, :3].double().cpu().numpy(), vb) < 1e-3
    g = ds.cpu().numpy()[0]
    # At k = 0.1 these steps move particles by up to 0.3h per iteration and
    # the FP32 step itself differs from the FP64 one by up to ~6e-4 relative;
    # dL/dk, a sum over all pairs with cancellation, inherits a few times that.
    k_tol = 1e-3 if kw.get("k", 0.1) < 1e-3 else 5e-3
    assert abs(g[_abi.MP_GRAD_SCORR_K] - kb) <= k_tol * abs(kb)
    if p.solver_iterations == 0:
        assert g[_abi.MP_GRAD_SCORR_K] == 0.0
    if sphere is not None:
        # through this step's push and the kinematic advance before it
        sb = np.zeros(7)
        sb[:3] = cb
        sb[6] = rb
        s0 = np.array(sphere, np.float64)
        rec = A.sphere_advance(p, DT, s0.copy())
        want = A.sphere_advance_adjoint(p, DT, rec, sb)
        np.testing.assert_allclose(g[1:8], want, rtol=1e-3, atol=1e-3 * np.abs(want).max())
    b.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_one_step_adjoint_on_random_clouds(cuda, seed):
    """One step of a seeded random cloud (tight clumps, points outside the
    grid and clamped by the hash and the box, random velocities) at the
    reference engine's parameters: the CUDA VJP equals the FP64 numpy VJP on
    the same FP32 input state."""
    from oracle import adjoint_ref as A
    from parity import random_scene

    torch = _torch()
    p = _abi.default_params()
    p.solver_iterations = 3
    pos4, vel4 = random_scene(seed, 600)
    n = len(pos4)
    b = make_batch([p], None, [n], [_abi.MP_SCENE_CUBE_DROP])
    dev = torch.device("cuda", 0)
    pos0 = torch.tensor(pos4, device=dev)
    vel0 = torch.tensor(vel4, device=dev)
    b.tensor(_abi.MP_BUF_POSITIONS).copy_(pos0)
    b.tensor(_abi.MP_BUF_VELOCITIES).copy_(vel0)
    b.rollout_forward(1, 1)
    rng = np.random.default_rng(seed + 10)
    wx, wv = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    gp = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    gv = torch.zeros_like(gp)
    gp[:, :3] = torch.tensor(wx, dtype=torch.float32)
    gv[:, :3] = torch.tensor(wv, dtype=torch.float32)
    dp, dv, ds = b.rollout_backward(gp, gv)
    torch.cuda.synchronize()
    assert b.check_errors() == 0
    c = A.consts(p, DT)
    _, _, tape = A.forward(c, pos4[:, :3].astype(np.float64), vel4[:, :3].astype(np.float64), None)
    xb, vb, kb, _, _ = A.adjoint(c, tape, wx, wv)
    rel = lambda a, r: np.linalg.norm(a - r) / np.linalg.norm(r)
    assert rel(dp[:, :3].double().cpu().numpy(), xb) < 1e-3
    assert rel(dv[:, :3].double().cpu().numpy(), vb) < 1e-3
    assert abs(ds.cpu().numpy()[0][_abi.MP_GRAD_SCORR_K] - kb) <= 1e-3 * abs(kb)
    b.close()


# ---- rollouts against finite differences of the FP64 oracle ------------------------

def cube_params(cfm=1e4):
    p = configs.base_params(3)
    p.scorr_k = 1e-4
    p.epsilon = cfm
    return p


def oracle_rollout(p, pos0, vel0, steps, sphere=None):
    from oracle import oracle as O

    x = np.array(pos0[:, :3], dtype=np.float64)  # copies: the oracle steps in place
    v = np.array(vel0[:, :3], dtype=np.float64)
    s = None if sphere is None else np.array(sphere, np.float64)
    for _ in range(steps):
        O.step_f64(p, DT, x, v, s)
    return x


_CUBE_CASES = {}


def cube_case(cfm, steps):
    """The 20^3 differentiable cube drop, its FP64 target run (initial
    velocities N(0, 0.5 m/s)) and central differences of the FP64 oracle's
    loss along a random velocity direction u and along k.  k is stored in
    FP32, so its difference quotient uses the two FP32 values the oracle
    actually ran with."""
    key = (cfm, steps)
    if key in _CUBE_CASES:
        return _CUBE_CASES[key]
    from oracle import oracle as O

    w = configs.diff_cube(side=20, steps=steps)
    p = cube_params(cfm)
    pos0 = O.seed_scene(p, w.scene, w.n, w.desc)
    rng = np.random.default_rng(5)
    target = oracle_rollout(p, pos0, rng.normal(0.0, 0.5, size=(w.n, 3)), steps)
    u = rng.normal(size=(w.n, 3))
    zero = np.zeros((w.n, 3))

    def loss(v0, k=None):
        q = cube_params(cfm)
        if k is not None:
            q.scorr_k = k
        return float(np.mean(np.sum((oracle_rollout(q, pos0, v0, steps) - target) ** 2, axis=1)))

    e = 1e-6
    fd_u = (loss(e * u) - loss(-e * u)) / (2 * e)
    kp, km = float(np.float32(p.scorr_k * (1 + 1e-5))), float(np.float32(p.scorr_k * (1 - 1e-5)))
    fd_k = (loss(zero, kp) - loss(zero, km)) / (kp - km)
    c = {"w": w, "p": p, "steps": steps, "pos0": pos0, "target": target, "u": u, "fd_u": fd_u,
         "fd_k": fd_k, "loss0": loss(zero)}
    _CUBE_CASES[key] = c
    return c


def gpu_cube_gradients(case, every):
    torch = _torch()
    from mtlphys_b200.autograd import rollout

    w, p = case["w"], case["p"]
    b = make_batch([p], [w.desc], [w.n])
    dev = torch.device("cuda", 0)
    pos0 = torch.tensor(case["pos0"], dtype=torch.float32, device=dev)
    vel0 = torch.zeros((w.n, 4), dtype=torch.float32, device=dev, requires_grad=True)
    k = torch.tensor([p.scorr_k], dtype=torch.float64, requires_grad=True)
    pos, _ = rollout(b, case["steps"], pos0, vel0, scorr_k=k, checkpoint_every=every)
    target = torch.tensor(case["target"], dtype=torch.float64, device=dev)
    loss = ((pos[:, :3].double() - target) ** 2).sum(1).mean()
    loss.backward()
    torch.cuda.synchronize()
    assert b.check_errors() == 0
    final = pos.detach().clone()
    after = b.tensor(_abi.MP_BUF_POSITIONS).clone()
    b.close()
    return {"loss": float(loss.detach()), "gv": vel0.grad[:, :3].double().cpu().numpy(),
            "gk": float(k.grad[0]), "final": final, "after": after}


@pytest.mark.parametrize("cfm,steps", [(1e5, 60), (1e4, 20)])
def test_rollout_gradients_match_fp64_finite_differences(cuda, cfm, steps):
    """60 checkpointed steps (every 10) at CFM epsilon 1e5 and 20 steps at
    1e4.  At epsilon 1e4 over 60 steps the FP32 trajectory drifts ~3e-4 m
    from the FP64 one and the velocity gradient differs from the FP64 one by
    tens of percent: a property of the scene, not of the adjoint (which
    matches the FP64 adjoint chain to 5e-7 per step, below)."""
    case = cube_case(cfm, steps)
    g = gpu_cube_gradients(case, every=10)
    assert abs(g["loss"] - case["loss0"]) <= 1e-4 * case["loss0"]
    an_u = float(np.sum(g["gv"] * case["u"]))
    assert abs(an_u - case["fd_u"]) <= 1e-3 * abs(case["fd_u"]), (an_u, case["fd_u"])
    assert abs(g["gk"] - case["fd_k"]) <= 1e-3 * abs(case["fd_k"]), (g["gk"], case["fd_k"])
    # the backward pass leaves the state where the forward pass ended
    torch = _torch()
    assert torch.equal(g["final"], g["after"])


def test_checkpoint_interval_does_not_change_gradients(cuda):
    case = cube_case(1e4, 20)
    ref = gpu_cube_gradients(case, every=10)
    for every in (1, 7, 20):
        g = gpu_cube_gradients(case, every=every)
        assert g["loss"] == ref["loss"]
        np.testing.assert_allclose(g["gv"], ref["gv"], rtol=0, atol=1e-6 * np.abs(ref["gv"]).max())
        assert abs(g["gk"] - ref["gk"]) <= 1e-6 * abs(ref["gk"])


def test_rollout_adjoint_matches_the_fp64_adjoint_chain(cuda):
    """A 6^3 cube, 5 steps, checkpoint every 2: the CUDA gradients equal the
    FP64 numpy adjoint chained over the FP64 steps to 1e-4 relative (the FP32
    and FP64 trajectories are 1.6e-6 m apart at the end)."""
    torch = _torch()
    from oracle import adjoint_ref as A
    from oracle import oracle as O

    side, steps = 6, 5
    p = cube_params()
    d = configs.lattice((side,) * 3, (2.0, 3.0, 2.0), 11)
    n = side ** 3
    pos0 = O.seed_scene(p, _abi.MP_SCENE_CUBE_DROP, n, d)
    rng = np.random.default_rng(3)
    v0 = rng.normal(0.0, 0.1, size=(n, 3))
    c = A.consts(p, DT)
    x, v, tapes = pos0[:, :3].astype(np.float64), v0.copy(), []
    for _ in range(steps):
        x, v, t = A.forward(c, x, v)
        tapes.append(t)
    wx, wv = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    xb, vb, kb = wx.copy(), wv.copy(), 0.0
    for t in reversed(tapes):
        xb, vb, k1, _, _ = A.adjoint(c, t, xb, vb)
        kb += k1
    b = make_batch([p], [d], [n])
    dev = torch.device("cuda", 0)
    V = torch.zeros((n, 4), device=dev)
    V[:, :3] = torch.tensor(v0, dtype=torch.float32)
    b.tensor(_abi.MP_BUF_POSITIONS).copy_(torch.tensor(pos0, device=dev))
    b.tensor(_abi.MP_BUF_VELOCITIES).copy_(V)
    b.rollout_forward(steps, 2)
    gx, gv = torch.zeros((n, 4), device=dev), torch.zeros((n, 4), device=dev)
    gx[:, :3] = torch.tensor(wx, dtype=torch.float32)
    gv[:, :3] = torch.tensor(wv, dtype=torch.float32)
    dp, dv, ds = b.rollout_backward(gx, gv)
    rel = lambda a, r: np.linalg.norm(a - r) / np.linalg.norm(r)
    assert rel(dp[:, :3].double().cpu().numpy(), xb) < 1e-4
    assert rel(dv[:, :3].double().cpu().numpy(), vb) < 1e-4
    assert abs(float(ds[0, _abi.MP_GRAD_SCORR_K]) - kb) <= 1e-4 * abs(kb)
    b.close()


def test_sphere_drop_gradients_match_fp64_finite_differences(cuda):
    """A sphere pushed into a small lake: dL/d(initial vertical speed) and
    dL/d(radius) of the mean squared height of the 200 highest particles of
    a target run, 15 steps, against FD of FP64 oracle rollouts.  FD of the
    radius is itself only good to ~0.2% here (particles crossing the sphere
    surface switch cells), hence its looser bound."""
    torch = _torch()
    from oracle import oracle as O
    from mtlphys_b200.autograd import rollout

    H = configs.H
    side, layers, steps, r0 = 9, 20, 15, 0.12
    width = (side - 1) * 0.5 * H + H
    p = cube_params()
    p.set(bounds_min=(0.0, 0.0, 0.0), bounds_max=(width, 40 * H, width))
    p.sphere_radius = r0
    d = configs.lattice((side, layers, side), (0.5 * H, 0.5 * H, 0.5 * H), 77)
    n = side * side * layers
    pos0 = O.seed_scene(p, _abi.MP_SCENE_SPHERE_DROP, n, d)
    top = float(pos0[:, 1].max())
    sphere = lambda vy, r: [width / 2, top + r + 0.02, width / 2, 0.0, vy, 0.0, r]
    target = oracle_rollout(p, pos0, np.zeros((n, 3)), steps, sphere(-1.5, r0))
    surf = np.argsort(-target[:, 1])[:200]

    def loss(vy, r):
        x = oracle_rollout(p, pos0, np.zeros((n, 3)), steps, sphere(vy, r))
        return float(np.mean((x[surf, 1] - target[surf, 1]) ** 2))

    e = 1e-5
    fd_v = (loss(-1.0 + e, r0) - loss(-1.0 - e, r0)) / (2 * e)
    fd_r = (loss(-1.0, r0 + e) - loss(-1.0, r0 - e)) / (2 * e)

    b = make_batch([p], [d], [n], [_abi.MP_SCENE_SPHERE_DROP])
    dev = torch.device("cuda", 0)
    s0 = sphere(-1.0, r0)
    c = torch.tensor([s0[:3]], dtype=torch.float64, requires_grad=True)
    v = torch.tensor([s0[3:6]], dtype=torch.float64, requires_grad=True)
    r = torch.tensor([r0], dtype=torch.float64, requires_grad=True)
    pos, _ = rollout(b, steps, torch.tensor(pos0, device=dev), torch.zeros((n, 4), device=dev),
                     sphere=(c, v, r), checkpoint_every=5)
    idx = torch.tensor(surf, device=dev)
    tgt = torch.tensor(target[surf, 1], dtype=torch.float64, device=dev)
    L = ((pos[idx, 1].double() - tgt) ** 2).mean()
    L.backward()
    assert b.check_errors() == 0
    assert abs(float(v.grad[0, 1]) - fd_v) <= 1e-3 * abs(fd_v), (float(v.grad[0, 1]), fd_v)
    # the FD moves the sphere's start (top + r + gap) with its radius
    an_r = float(r.grad[0]) + float(c.grad[0, 1])
    assert abs(an_r - fd_r) <= 1e-2 * abs(fd_r), (an_r, fd_r)
    b.close()


def test_batched_scenes_get_their_single_scene_gradients(cuda):
    """Three uneven scenes in one batch: each scene's gradients equal those
    of the same scene alone (the scenes do not interact)."""
    torch = _torch()
    from mtlphys_b200.autograd import rollout

    w = configs.batch_cubes(num=3, lo=300, hi=3000, steps=8)
    for p in w.params:
        p.scorr_k = 1e-4
        p.epsilon = 1e4
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(2)

    def run(idx):
        b = make_batch([w.params[i] for i in idx], [w.descs[i] for i in idx], [w.counts[i] for i in idx],
                       dts=[w.dts[i] for i in idx])
        n = b.particle_count()
        pos0 = b.tensor(_abi.MP_BUF_POSITIONS).clone()
        vel0 = torch.zeros((n, 4), device=dev, requires_grad=True)
        k = torch.tensor([w.params[i].scorr_k for i in idx], dtype=torch.float64, requires_grad=True)
        pos, vel = rollout(b, w.steps, pos0, vel0, scorr_k=k, checkpoint_every=3)
        wts = torch.tensor(rng_weights[np.concatenate([np.arange(offs[i], offs[i] + w.counts[i]) for i in idx])],
                           dtype=torch.float64, device=dev)
        (pos[:, :3].double() * wts).sum().backward()
        out = (vel0.grad[:, :3].cpu().numpy(), k.grad.numpy())
        b.close()
        return out

    offs = np.concatenate([[0], np.cumsum(w.counts)])
    rng_weights = rng.normal(size=(int(offs[-1]), 3))
    gv_all, gk_all = run([0, 1, 2])
    for s in range(3):
        gv, gk = run([s])
        np.testing.assert_allclose(gv_all[offs[s]:offs[s + 1]], gv, rtol=0, atol=1e-6 * np.abs(gv).max())
        assert abs(gk_all[s] - gk[0]) <= 1e-9 * abs(gk[0])


def test_empty_scene_in_a_differentiable_batch(cuda):
    """A scene with no particles next to a real one: the rollout and its
    gradient run, the empty scene's parameter gradients are zero and the
    other scene gets its single-scene gradients."""
    torch = _torch()
    w = configs.diff_cube(side=8, steps=6)
    p = cube_params()
    dev = torch.device("cuda", 0)

    def run(counts):
        b = make_batch([p] * len(counts), [w.desc] * len(counts), counts)
        n = b.particle_count()
        g = torch.zeros((n, 4), device=dev)
        g[:, 1] = 1.0
        b.rollout_forward(w.steps, 4)
        dp, dv, ds = b.rollout_backward(g, None)
        assert b.check_errors() == 0
        out = dv.cpu().numpy(), ds.cpu().numpy()
        b.close()
        return out

    dv_pair, ds_pair = run([0, w.n])
    dv_one, ds_one = run([w.n])
    assert not ds_pair[0].any()
    np.testing.assert_allclose(dv_pair, dv_one, rtol=0, atol=1e-6 * np.abs(dv_one).max())
    assert abs(ds_pair[1, _abi.MP_GRAD_SCORR_K] - ds_one[0, _abi.MP_GRAD_SCORR_K]) <= 1e-9 * abs(
        ds_one[0, _abi.MP_GRAD_SCORR_K])


def test_backward_after_a_state_change_is_refused(cuda):
    w = configs.diff_cube(side=6, steps=3)
    b = make_batch([cube_params()], [w.desc], [w.n])
    b.rollout_forward(3, 2)
    b.rollout_backward()
    b.step()
    with pytest.raises(_abi.MPError):
        b.rollout_backward()
    b.close()


@pytest.mark.parametrize("case", ["cube_k01", "clumps", "spheres"])
def test_backward_passes_are_byte_identical(cuda, case):
    """The gradients do not depend on the order in which threads run: pair
    terms owed to a particle whose own sweep does not see the pair are posted
    to it and added in sender order, and the scene gradients are summed per
    slot and then per scene in a fixed order.  Two forward + backward passes
    from the same state give the same bytes: per-particle dL/dx0, dL/dv0 and
    every scene's parameter gradients.  Cases: the cube drop at the
    benchmark parameters (k = 0.1, exploding), tight clumps of particles
    (long drifts, many one-way pairs, inbox overflow) and two sphere drops
    (sphere-push gradients)."""
    torch = _torch()
    from parity import random_scene

    dev = torch.device("cuda", 0)
    if case == "cube_k01":
        w = configs.diff_cube(side=20, steps=12)
        b = make_batch([w.params], [w.desc], [w.n])
        steps, every = 12, 5
    elif case == "clumps":
        p = _abi.default_params()
        pos, vel = random_scene(9, 6000)
        b = make_batch([p], None, [len(pos)], dts=[1.0 / 240.0])
        b.write(_abi.MP_BUF_POSITIONS, pos)
        b.write(_abi.MP_BUF_VELOCITIES, vel)
        steps, every = 4, 2
    else:
        ws = configs.batch_spheres(num=2, lo=3000, hi=6000, steps=6)
        b = make_batch(ws.params, ws.descs, ws.counts, ws.scenes, ws.dts)
        steps, every = 6, 3
    n = b.particle_count()
    pos0 = b.tensor(_abi.MP_BUF_POSITIONS).clone()
    vel0 = b.tensor(_abi.MP_BUF_VELOCITIES).clone()
    spheres = [b.sphere(s) for s in range(b.scene_count())]
    g = torch.zeros((n, 4), device=dev)
    g[:, :3] = torch.from_numpy(np.random.default_rng(3).normal(size=(n, 3)).astype(np.float32)).to(dev)
    outs = []
    for _ in range(2):
        b.tensor(_abi.MP_BUF_POSITIONS).copy_(pos0)
        b.tensor(_abi.MP_BUF_VELOCITIES).copy_(vel0)
        for s, sph in enumerate(spheres):
            b.set_sphere(s, sph[:3], sph[3:6], sph[6])
        b.rollout_forward(steps, every)
        dp, dv, ds = b.rollout_backward(g, g)
        torch.cuda.synchronize()
        assert b.check_errors() == 0
        outs.append((dp.cpu().numpy().copy(), dv.cpu().numpy().copy(), ds.cpu().numpy().copy()))
    b.close()
    for x, y in zip(*outs):
        assert x.tobytes() == y.tobytes()
    assert np.isfinite(outs[0][0]).all() and np.abs(outs[0][1]).max() > 0

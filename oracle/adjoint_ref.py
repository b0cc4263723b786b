"""FP64 restatement of one PBF step and of its adjoint, for small systems.

TEST INFRASTRUCTURE ONLY: the tests use it to check the CUDA adjoint kernels
(mtlphys_b200/csrc/pbf_adjoint.cu) on systems small enough for all-pairs
numpy arithmetic.  The product never imports it.

The forward step follows the FP64 oracle (oracle/pbf_oracle.cpp, step_core),
which restates engine/src/Engine.cpp:685-811 and the shaders
engine/shaders/Constraints.metal:54-353: predict, K x (densityLambda,
applyDelta with s_corr, |delta| <= max_delta h, box clamp, sphere push),
finalize (wall absorption, friction, speed cap).  Neighbour lists follow the
reference's search: the hash is built once per step on the predicted
positions, and every solver iteration looks, from the cell of particle i's
current position (FP32 cellCoordOf, Constraints.metal:94, 152), through the
27 cells around it.  So j is in i's list (M_ij) when |p_i - p_j| < h and j's
predicted cell is within one cell of i's current cell on every axis; once
particles have moved off their predicted cells the lists are not symmetric.

The adjoint is the vector-Jacobian product of that map with the neighbour
topology, the clamp states and the wall masks held fixed.  Notation, per
solver iteration, with r_ij = p_i - p_j, rho = |r_ij|:
  W(r)   = poly6 (h^2 - rho^2)^3                 (density kernel)
  g(r)   = f(rho) r, f = -spiky (h - rho)^2 / rho  (spiky gradient)
  H(r)   = dg/dr = f I + (s (h^2 - rho^2) / rho^3) r r^T,  s = spiky
  rho_i  = sum_j W(r_ij) (self included), G_i = sum_j g_ij, Q_i = sum_j |g_ij|^2
  lambda_i = -(rho_i / rho0 - 1) / ((|G_i|^2 + Q_i) / rho0^2 + eps)
  s_ij   = -k (W(r_ij) / W(dq))^n
  delta_i = (1 / rho0) sum_j (lambda_i + lambda_j + s_ij) g_ij
Every sum over j runs over i's list (M_ij).  The adjoint is written in
scatter form: a pair term of i's list adds to i's adjoint and subtracts from
j's (or adds, for lambda), whether or not i is in j's list.  Given the
adjoint dbar_i of delta_i, with u_ij = ((lambda_i + lambda_j + s_ij) H_ij dbar_i
+ grad s_ij (g_ij . dbar_i)) / rho0:
  lambdabar_i += g_ij . dbar_i / rho0,  lambdabar_j += g_ij . dbar_i / rho0
  pbar_i += u_ij,  pbar_j -= u_ij
  kbar   += -(W_ij / W(dq))^n g_ij . dbar_i / rho0
and from lambdabar: rhobar_i = -lambdabar_i / (D_i rho0), Dbar_i = -lambdabar_i lambda_i / D_i,
  Gbar_i = 2 Dbar_i G_i / rho0^2, Qbar_i = Dbar_i / rho0^2; with
  v_ij = rhobar_i grad W(r_ij) + H_ij Gbar_i + 2 Qbar_i H_ij g_ij:
  pbar_i += v_ij,  pbar_j -= v_ij.
"""
from __future__ import annotations

import math

import numpy as np

F32_EPS6 = float(np.float32(1e-6))
F32_EPS8 = float(np.float32(1e-8))


def consts(p, dt: float) -> dict:
    """The step constants of parameter set `p` (an mp_pbf_params)."""
    h = float(p.h)
    c = {
        "h": h, "h2": h * h, "poly6": 315.0 / (64.0 * math.pi * h ** 9),
        "spiky": 45.0 / (math.pi * h ** 6), "rho0": float(p.rest_density), "eps": float(p.epsilon),
        "damping": float(p.damping), "g": np.array([float(x) for x in p.gravity]),
        "bmin": np.array([float(x) for x in p.bounds_min]), "bmax": np.array([float(x) for x in p.bounds_max]),
        "k": float(p.scorr_k), "n": int(p.scorr_n), "max_step": float(p.max_delta) * h,
        "wall_eps": float(p.wall_eps), "floor_fric": float(p.floor_friction),
        "wall_fric": float(p.wall_friction), "dt": float(dt), "vmax": float(p.vmax) * h / float(dt),
        "iters": int(p.solver_iterations),
    }
    dq = float(p.scorr_dq) * h
    wq = c["poly6"] * (c["h2"] - dq * dq) ** 3
    c["inv_wq"] = 1.0 / wq
    # hash grid (Engine.cpp:398-452): origin = bounds_min, FP32 1/cell,
    # dims = ceil(extent / cell) in FP32
    cell = np.float32(p.cell_size)
    c["origin"] = np.array([np.float32(x) for x in p.bounds_min], np.float32)
    c["inv_cell"] = np.float32(1.0) / cell
    ext = np.array([np.float32(b) - np.float32(a) for a, b in zip(p.bounds_min, p.bounds_max)], np.float32)
    c["dims"] = np.maximum(np.ceil(ext / cell).astype(np.int64), 1)
    return c


def cells_f32(c, p):
    """cellCoordOf (Spatial.metal:35-39) of FP64 positions rounded to FP32."""
    q = (p.astype(np.float32) - c["origin"]) * c["inv_cell"]
    return np.clip(np.floor(q).astype(np.int64), 0, c["dims"] - 1)


def _pairs(c, p, pred_cells):
    """Pair arrays of one iteration: M[i, j] = j is in i's list."""
    r = p[:, None, :] - p[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", r, r)
    cur = cells_f32(c, p)
    near = np.all(np.abs(cur[:, None, :] - pred_cells[None, :, :]) <= 1, axis=2)
    M = near & (r2 < c["h2"])
    np.fill_diagonal(M, False)
    rl = np.sqrt(r2)
    d = np.where(M, c["h2"] - r2, 0.0)
    W = c["poly6"] * d ** 3
    gm = M & (rl > F32_EPS6)
    safe = np.where(gm, rl, 1.0)
    f = np.where(gm, -c["spiky"] * (c["h"] - safe) ** 2 / safe, 0.0)
    fp = np.where(gm, c["spiky"] * (c["h2"] - safe ** 2) / safe ** 3, 0.0)  # f'(rho) / rho
    gW = (-6.0 * c["poly6"] * d ** 2)[..., None] * r                      # grad W (zero off the list)
    return {"r": r, "M": M, "gm": gm, "W": W, "f": f, "fp": fp, "g": f[..., None] * r, "gW": gW}


def _hess_apply(P, d):
    """H_ij d_ij for pair arrays: f d + fp (r . d) r."""
    rd = np.einsum("ijk,ijk->ij", P["r"], d)
    return P["f"][..., None] * d + (P["fp"] * rd)[..., None] * P["r"]


def forward(c, x, v, sphere=None, k=None):
    """One step from FP64 state x, v (n x 3).  sphere: None or 7 floats
    (center, velocity, radius) AFTER this step's kinematic advance.  Returns
    (x', v', tape)."""
    k = c["k"] if k is None else k
    x = np.asarray(x, np.float64)
    v = np.asarray(v, np.float64)
    pred = x + c["dt"] * (v + c["g"] * c["dt"])
    pred_cells = cells_f32(c, pred)
    cur = pred.copy()
    tape = {"x": x, "iters": [], "k": k, "sphere": None if sphere is None else np.array(sphere, np.float64)}
    for _ in range(c["iters"]):
        P = _pairs(c, cur, pred_cells)
        dens = c["poly6"] * c["h2"] ** 3 + P["W"].sum(1)
        G = P["g"].sum(1)
        Q = np.einsum("ijk,ijk->i", P["g"], P["g"])
        C = dens / c["rho0"] - 1.0
        D = (np.einsum("ik,ik->i", G, G) + Q) / c["rho0"] ** 2 + c["eps"]
        lam = -C / D
        ratio = P["W"] * c["inv_wq"]
        s = np.where(P["gm"], -k * ratio ** c["n"], 0.0)
        coef = lam[:, None] + lam[None, :] + s
        delta = (coef[..., None] * P["g"]).sum(1) / c["rho0"]
        dl = np.sqrt(np.einsum("ik,ik->i", delta, delta))
        big = dl > c["max_step"]
        scale = np.where(big, c["max_step"] / np.where(big, dl, 1.0), 1.0)
        q = cur + scale[:, None] * delta
        qc = np.minimum(np.maximum(q, c["bmin"]), c["bmax"])
        nxt = qc.copy()
        push = np.zeros(len(cur), bool)
        if sphere is not None:
            ctr, rad = np.asarray(sphere[:3], np.float64), float(sphere[6])
            e = qc - ctr
            e2 = np.einsum("ik,ik->i", e, e)
            push = e2 < rad * rad
            el = np.sqrt(np.maximum(e2, F32_EPS8))
            nxt = np.where(push[:, None], ctr + (rad / el)[:, None] * e, qc)
        tape["iters"].append({"p": cur, "P": P, "G": G, "D": D, "lam": lam, "s": s, "delta": delta,
                              "dl": dl, "big": big, "scale": scale, "q": q, "qc": qc, "push": push})
        cur = nxt
    X = np.minimum(np.maximum(cur, c["bmin"]), c["bmax"])
    kd = c["damping"] / c["dt"]
    u = (X - x) * kd
    lo = X <= c["bmin"] + c["wall_eps"]
    hi = X >= c["bmax"] - c["wall_eps"]
    keep = ~((lo & (u < 0)) | (hi & (u > 0)))
    a = np.where(keep, u, 0.0)
    ymin = lo[:, 1]
    wall = lo[:, 0] | hi[:, 0] | lo[:, 2] | hi[:, 2]
    fr = np.ones_like(a)
    fr[ymin] = [c["floor_fric"], 1.0, c["floor_fric"]]
    fr[~ymin & wall] = c["wall_fric"]
    b = a * fr
    bl = np.sqrt(np.einsum("ik,ik->i", b, b))
    cap = bl > c["vmax"]
    vout = np.where(cap[:, None], (c["vmax"] / np.where(cap, bl, 1.0))[:, None] * b, b)
    tape.update({"X": X, "kd": kd, "keep": keep, "fr": fr, "b": b, "bl": bl, "cap": cap})
    return X, vout, tape


def adjoint(c, tape, xbar, vbar):
    """Vector-Jacobian product of forward(): given dL/dx', dL/dv', returns
    (dL/dx, dL/dv, dL/dk, dL/d sphere center (3), dL/d sphere radius)."""
    xbar = np.asarray(xbar, np.float64)
    vbar = np.asarray(vbar, np.float64)
    # finalize: cap, friction, absorption masks, v = (X - x) kd
    b, bl = tape["b"], tape["bl"]
    bbar = vbar.copy()
    cap = tape["cap"]
    if cap.any():
        bh = b[cap] / bl[cap, None]
        vb = vbar[cap]
        bbar[cap] = (c["vmax"] / bl[cap])[:, None] * (vb - bh * np.einsum("ik,ik->i", bh, vb)[:, None])
    ubar = bbar * tape["fr"] * tape["keep"]
    Xbar = xbar + ubar * tape["kd"]
    x_bar = -ubar * tape["kd"]
    # the finalize clamp is the identity on a solver output inside the box
    pbar = Xbar
    kbar, cbar, rbar = 0.0, np.zeros(3), 0.0
    sph = tape["sphere"]
    rho0 = c["rho0"]
    for T in reversed(tape["iters"]):
        # sphere push
        qcbar = pbar.copy()
        if sph is not None and T["push"].any():
            ctr, rad = sph[:3], float(sph[6])
            m = T["push"]
            e = T["qc"][m] - ctr
            e2 = np.einsum("ik,ik->i", e, e)
            el = np.sqrt(np.maximum(e2, F32_EPS8))
            pb = pbar[m]
            eh = e / el[:, None]
            full = e2 > F32_EPS8
            ebar = np.where(full[:, None],
                            (rad / el)[:, None] * (pb - eh * np.einsum("ik,ik->i", eh, pb)[:, None]),
                            (rad / el)[:, None] * pb)
            cbar += (pb - ebar).sum(0)
            rbar += np.einsum("ik,ik->", e / el[:, None], pb)
            qcbar[m] = ebar
        # box clamp
        inside = (T["q"] >= c["bmin"]) & (T["q"] <= c["bmax"])
        qbar = qcbar * inside
        # |delta| clamp
        dbar = qbar.copy()
        big = T["big"]
        if big.any():
            dh = T["delta"][big] / T["dl"][big, None]
            qb = qbar[big]
            dbar[big] = T["scale"][big, None] * (qb - dh * np.einsum("ik,ik->i", dh, qb)[:, None])
        P = T["P"]
        lam, s = T["lam"], T["s"]
        gd = np.einsum("ijk,ik->ij", P["g"], dbar)                       # g_ij . dbar_i
        lambar = (gd.sum(1) + gd.sum(0)) / rho0
        coef = lam[:, None] + lam[None, :] + s
        ratio = P["W"] * c["inv_wq"]
        n = c["n"]
        ds_dr = np.where(P["gm"], -tape["k"] * n * ratio ** (n - 1) * c["inv_wq"], 0.0)[..., None] * P["gW"]
        di = np.broadcast_to(dbar[:, None, :], P["r"].shape)
        u = (coef[..., None] * _hess_apply(P, di) + ds_dr * gd[..., None]) / rho0
        pd = u.sum(1) - u.sum(0)
        dsdk = np.where(P["gm"], -(ratio ** n), 0.0)
        kbar += np.einsum("ij,ij->", dsdk, gd) / rho0
        # lambda
        D, G = T["D"], T["G"]
        rhobar = -lambar / (D * rho0)
        Dbar = -lambar * lam / D
        Gbar = (2.0 * Dbar / rho0 ** 2)[:, None] * G
        Qbar = Dbar / rho0 ** 2
        vv = (rhobar[:, None, None] * P["gW"]
              + _hess_apply(P, np.broadcast_to(Gbar[:, None, :], P["r"].shape))
              + (2.0 * Qbar)[:, None, None] * _hess_apply(P, P["g"]))
        pl = vv.sum(1) - vv.sum(0)
        pbar = qbar + pd + pl
    # predict
    x_bar = x_bar + pbar
    v_bar = pbar * c["dt"]
    return x_bar, v_bar, kbar, cbar, rbar


def sphere_advance(p, dt: float, s):
    """Kinematic sphere advance (Engine.cpp:694-707) in FP64, in place on
    s = [cx, cy, cz, vx, vy, vz, r]; returns the bounce record."""
    bmin = [float(x) for x in p.bounds_min]
    bmax = [float(x) for x in p.bounds_max]
    s[4] += float(p.sphere_gravity) * dt
    for a in range(3):
        s[3 + a] *= float(p.sphere_drag)
    for a in range(3):
        s[a] += s[3 + a] * dt
    rec = []
    r = s[6]
    for a in range(3):
        lo = s[a] - r < bmin[a]
        if lo:
            s[a] = bmin[a] + r
            s[3 + a] = -s[3 + a] * float(p.sphere_restitution)
        hi = s[a] + r > bmax[a]
        if hi:
            s[a] = bmax[a] - r
            s[3 + a] = -s[3 + a] * float(p.sphere_restitution)
        rec.append((lo, hi))
    return rec


def sphere_advance_adjoint(p, dt: float, rec, sbar):
    """Reverse of sphere_advance given its bounce record: sbar = adjoint of
    the advanced state [c(3), v(3), r] -> adjoint of the state before."""
    out = np.array(sbar, np.float64)
    rest = float(p.sphere_restitution)
    for a in reversed(range(3)):
        lo, hi = rec[a]
        if hi:
            out[6] -= out[a]
            out[a] = 0.0
            out[3 + a] = -rest * out[3 + a]
        if lo:
            out[6] += out[a]
            out[a] = 0.0
            out[3 + a] = -rest * out[3 + a]
    # c' = c + v' dt
    for a in range(3):
        out[3 + a] += out[a] * dt
    # v' = (v + g dt e_y) drag
    for a in range(3):
        out[3 + a] *= float(p.sphere_drag)
    return out

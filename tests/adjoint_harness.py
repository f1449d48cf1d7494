"""Test harness of the differentiable rollout (no counterpart in the reference).

* ``Rollout`` -- an autograd-style function (``torch.autograd.Function``) over the C ABI:
  forward = PHYSIK_Step repeated ``steps`` times from (x0, v0) with per-tet Young's moduli
  E = exp(theta), keeping a checkpoint of the state every ``k`` steps; backward = the
  adjoint steps (PHYSIK_B200_AdjointStep), segment by segment from the last checkpoint
  back, recomputing each segment's states from its checkpoint.  Returns x_T; gradients
  flow to theta (per tet) and v0 (per node).
* ``cpu_adjoint`` -- an FP64 CPU reference gradient written independently in numpy: the
  forward steps and their assembled systems (A, delta-v) come from the FP64 oracle (the
  reference's CPU solve run in double), the adjoint systems are solved directly
  (scipy), and the element terms are evaluated in numpy, the rotation by the reference's
  polar iteration and its derivative in reverse mode through that iteration.
* ``rollout_loss`` -- L = 1/2 |x_T - x_target|^2 of a plain forward rollout (for finite
  differences).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from oracle import pyoracle as po


def set_young(world, young32):
    world.set_tet_young(0, np.asarray(young32, np.float32))


def forward(world, young32, x0, v0, steps):
    set_young(world, young32)
    world.set_state(x0, v0, f64=True)
    for _ in range(steps):
        world.step()
    return world.state(f64=True)


def trajectory(world, young32, x0, v0, steps):
    """The rollout's states (x_t, v_t), t < steps, and x_T."""
    set_young(world, young32)
    world.set_state(x0, v0, f64=True)
    states = []
    for _ in range(steps):
        states.append(world.state(f64=True))
        world.step()
    return states, world.state(f64=True)[0]


def rollout_loss(world, young32, x0, v0, steps, x_target):
    xT, _ = forward(world, young32, x0, v0, steps)
    return 0.5 * float(np.sum((xT - x_target) ** 2))


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, v0, world, x0, steps, k):
        young = np.exp(theta.detach().numpy()).astype(np.float32)
        set_young(world, young)
        world.set_state(x0, v0.detach().numpy(), f64=True)
        checkpoints = []
        for t in range(steps):
            if t % k == 0:
                checkpoints.append(world.state(f64=True))
            world.step()
        xT, _ = world.state(f64=True)
        ctx.world, ctx.checkpoints, ctx.steps, ctx.k = world, checkpoints, steps, k
        ctx.tets = theta.shape[0]
        return torch.from_numpy(xT)

    @staticmethod
    def backward(ctx, grad_xT):
        world, steps, k = ctx.world, ctx.steps, ctx.k
        xbar = np.ascontiguousarray(grad_xT.detach().numpy(), np.float64)
        vbar = np.zeros_like(xbar)
        theta_bar = np.zeros(ctx.tets, np.float64)
        for seg in reversed(range(len(ctx.checkpoints))):
            t0, t1 = seg * k, min(steps, (seg + 1) * k)
            states = [ctx.checkpoints[seg]]
            world.set_state(*states[0], f64=True)
            for _ in range(t0, t1 - 1):
                world.step()
                states.append(world.state(f64=True))
            for t in reversed(range(t0, t1)):
                world.set_state(*states[t - t0], f64=True)
                xbar, vbar = world.adjoint_step(xbar, vbar, theta_bar)
        return torch.from_numpy(theta_bar), torch.from_numpy(vbar), None, None, None, None


# ---------------------------------------------------------------------- CPU reference
def _sym(m):
    return 0.5 * (m + np.swapaxes(m, -1, -2))


def _inv_t(m):
    """inverse(m^T) as the reference's Mat3::Inverse: the identity when |det| <= 1e-6."""
    d = np.linalg.det(m)
    small = ~(np.abs(d) > 1e-6)
    out = np.empty_like(m)
    ok = ~small
    out[ok] = np.linalg.inv(np.swapaxes(m[ok], 1, 2))
    out[small] = np.eye(3)
    return out, small


def _newton_polar(F):
    """The reference's polar iteration (FEMModel.cpp:115-163) per tet, keeping every
    iterate: R_0 = F, R_k+1 = (R_k + R_k^-T) / 2, at most 12 steps, stopped when the
    squared step <= 1e-10, identity when F or an inverse is singular (|det| <= 1e-8) or
    non-finite, column 2 negated when det R < 0."""
    t = F.shape[0]
    iters = np.zeros((13, t, 3, 3))
    iters[0] = F
    n = np.zeros(t, int)
    fallback = ~np.isfinite(F).all(axis=(1, 2)) | ~(np.abs(np.linalg.det(F)) > 1e-8)
    active = ~fallback
    for it in range(12):
        if not active.any():
            break
        ti, _ = _inv_t(iters[it])
        bad = active & (~np.isfinite(ti).all(axis=(1, 2)) | ~(np.abs(np.linalg.det(ti)) > 1e-8))
        fallback |= bad
        active &= ~bad
        nxt = 0.5 * (iters[it] + ti)
        bad = active & ~np.isfinite(nxt).all(axis=(1, 2))
        fallback |= bad
        active &= ~bad
        iters[it + 1] = np.where(active[:, None, None], nxt, iters[it])
        n[active] = it + 1
        diff = np.sum((nxt - iters[it]) ** 2, axis=(1, 2))
        active &= ~(diff <= 1e-10)
    R = iters[n, np.arange(t)].copy()
    R[fallback] = np.eye(3)
    reflect = ~fallback & (np.linalg.det(R) < 0)
    R[reflect, :, 2] *= -1.0
    return R, iters, n, reflect, fallback


def _newton_polar_backward(GR, iters, n, reflect, fallback):
    """dL/dF through the iteration of _newton_polar, given dL/dR: with G = dL/dR_k+1,
    dL/dR_k = (G - R_k^-T G^T R_k^-T) / 2 (G / 2 where the inverse was the identity)."""
    G = GR.copy()
    G[reflect, :, 2] *= -1.0
    for k in range(11, -1, -1):
        live = (k < n) & ~fallback
        if not live.any():
            continue
        xt, small = _inv_t(iters[k])
        back = 0.5 * (G - xt @ np.swapaxes(G, 1, 2) @ xt)
        back[small] = 0.5 * G[small]
        G = np.where(live[:, None, None], back, G)
    G[fallback] = 0.0
    return G


def _full_matrix(sys_):
    """Scipy CSR of the symmetric matrix from the upper BSR (values[k, c, r] = B[r][c])."""
    rs, col, val = sys_.row_start, sys_.col, sys_.values
    n = len(rs) - 1
    rows = np.repeat(np.arange(n), np.diff(rs))
    B = np.transpose(val, (0, 2, 1))  # row-major blocks
    I, J, V = [], [], []
    for i in range(3):
        for j in range(3):
            I.append(3 * rows + i)
            J.append(3 * col + j)
            V.append(B[:, i, j])
            off = col != rows
            I.append(3 * col[off] + j)
            J.append(3 * rows[off] + i)
            V.append(B[off, i, j])
    return sp.csr_matrix((np.concatenate(V), (np.concatenate(I), np.concatenate(J))), shape=(3 * n, 3 * n))


def cpu_adjoint(scene, young32, x0, v0, steps, x_target, trajectory=None, with_xbar=False):
    """FP64 CPU gradient of L = 1/2 |x_T - x_target|^2 w.r.t. log E (per tet) and v0.

    trajectory: optional (states, x_T) of a rollout to differentiate along -- states[t] =
    (x_t, v_t) for t < steps.  Without it the rollout is the FP64 oracle's own.  (Two
    rollouts that agree to the CG tolerance can still seed noticeably different
    gradients when x_T - x_target is small, so comparisons use one trajectory.)"""
    body = scene.bodies[0]
    ora = po.Oracle(scene, "f64", float_inputs=True)
    ora.set_tet_young(np.asarray(young32, np.float64))
    dt = ora.dt
    E = np.asarray(young32, np.float32).astype(np.float64)
    nu = min(0.49, max(-0.99, float(np.float32(body.poisson))))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    damp = np.full(E.shape, float(np.float32(body.damping)))
    vol, _, grads = ora.tet_rest()
    tets = np.asarray(body.tets, np.int64)
    if trajectory is None:
        x, v = np.array(x0, np.float64), np.array(v0, np.float64)
        states = []
        for _ in range(steps):
            states.append((x.copy(), v.copy()))
            ora.set_state(x, v)
            ora.step()
            x, v = ora.x.copy(), ora.v.copy()
    else:
        states, x = trajectory
    xbar = np.asarray(x, np.float64) - x_target
    vbar = np.zeros_like(xbar)
    theta_bar = np.zeros(len(E))
    for t in reversed(range(steps)):
        xt, vt = states[t]
        ora.set_state(xt.copy(), vt.copy())
        ora.step()
        s = ora.last_system()
        dyn_nodes = np.nonzero(s.node_to_dyn >= 0)[0]
        A = _full_matrix(s)
        g = (vbar[dyn_nodes] + dt * xbar[dyn_nodes]).reshape(-1)
        w_rows = spla.spsolve(A.tocsc(), g).reshape(-1, 3)
        aw = (A @ w_rows.reshape(-1)).reshape(-1, 3)
        w = np.zeros_like(xt)
        w[dyn_nodes] = w_rows
        z = vt.copy()
        z[dyn_nodes] += s.dv
        # element terms
        X, W, Z = xt[tets], w[tets], z[tets]
        F = np.einsum("tai,taj->tij", X, grads)
        R, iters, nsteps, reflect, fallback = _newton_polar(F)
        Rt = np.swapaxes(R, 1, 2)
        Wg = np.einsum("tai,taj->tij", W, grads)
        Zg = np.einsum("tai,taj->tij", Z, grads)
        eye = np.eye(3)[None]
        eps = _sym(Rt @ F) - eye
        tr = np.trace(eps, axis1=1, axis2=2)
        sigma = lam[:, None, None] * tr[:, None, None] * eye + 2.0 * mu[:, None, None] * eps
        Aw, Az = Rt @ Wg, Rt @ Zg
        rw, rz = np.sum(R * Wg, axis=(1, 2)), np.sum(R * Zg, axis=(1, 2))
        T1 = -dt * vol * np.sum((R @ sigma) * Wg, axis=(1, 2))
        T2 = -dt * dt * vol * (lam * rw * rz + mu * np.trace(Aw @ Az, axis1=1, axis2=2) + mu * np.sum(Aw * Az, axis=(1, 2)))
        theta_bar += T1 + T2
        Sbar = lam[:, None, None] * np.trace(Aw, axis1=1, axis2=2)[:, None, None] * eye + 2.0 * mu[:, None, None] * _sym(Aw)
        GF = -dt * vol[:, None, None] * (R @ Sbar)
        GR = -dt * vol[:, None, None] * (Wg @ sigma + F @ Sbar)
        GR -= dt * dt * vol[:, None, None] * (
            lam[:, None, None] * (rz[:, None, None] * Wg + rw[:, None, None] * Zg)
            + mu[:, None, None] * (Wg @ Az + Zg @ Aw)
            + mu[:, None, None] * ((Wg @ np.swapaxes(Zg, 1, 2) + Zg @ np.swapaxes(Wg, 1, 2)) @ R))
        GF += _newton_polar_backward(GR, iters, nsteps, reflect, fallback)
        node_grad = np.einsum("tij,taj->tai", GF, grads)
        xbar_new = xbar.copy()
        contrib = np.zeros_like(xbar)
        np.add.at(contrib, tets.reshape(-1), node_grad.reshape(-1, 3))
        xbar_new[dyn_nodes] += contrib[dyn_nodes]
        csum = np.zeros(len(xt))
        np.add.at(csum, tets.reshape(-1), np.repeat(damp, 4))
        vbar_new = vbar.copy()
        m = s.mass[dyn_nodes][:, None]
        vbar_new[dyn_nodes] = g.reshape(-1, 3) - aw + m * w_rows - dt * csum[dyn_nodes][:, None] * w_rows
        xbar, vbar = xbar_new, vbar_new
    if with_xbar:
        return theta_bar, vbar, xbar
    return theta_bar, vbar


def oracle_rollout_loss(scene, young32, x0, v0, steps, x_target):
    """L of a forward rollout on the FP64 oracle (CPU)."""
    ora = po.Oracle(scene, "f64", float_inputs=True)
    ora.set_tet_young(np.asarray(young32, np.float64))
    x, v = np.array(x0, np.float64), np.array(v0, np.float64)
    for _ in range(steps):
        ora.set_state(x, v)
        ora.step()
        x, v = ora.x.copy(), ora.v.copy()
    return 0.5 * float(np.sum((x - x_target) ** 2)), x

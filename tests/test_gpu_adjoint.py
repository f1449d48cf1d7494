"""Adjoint of the implicit rollout (PHYSIK_B200_AdjointStep) -- no counterpart in the
reference, checked three ways:

* against central finite differences of the loss L = 1/2 |x_T - x_target|^2 computed
  with FP64 forward rollouts (the FP64 GPU path, itself checked against the FP64 oracle
  to 1e-14 per step), epsilon = 1e-3 (on the rollout workload Richardson-extrapolated
  from 1e-3 and 5e-4), each coordinate relative to its own finite difference: 1e-4 (the
  most sensitive coordinate of the 60-step rollout, where elements are crushed nearly flat
  and the loss is far from quadratic at 1e-3, with epsilon = 1e-5); on the rollout
  workload's random coordinates 1e-4 |fd| plus the CG tolerance times the gradient's
  scale, the gap between differentiating exact solves and differencing CG-stopped ones;
* against an FP64 CPU reference gradient written independently in numpy on top of the
  FP64 oracle's assembled systems (tests/adjoint_harness.py), all coordinates, along the
  same trajectory (relative 1e-6);
* on the differentiable-rollout workload: 32x8x8 beam, log E ~ N(ln 1e5, 0.3^2) (seed 3),
  x_target from a rollout with log E of seed 4, 60 steps, checkpoints every 10 steps,
  16 random coordinates of (log E, v0).

The CG tolerance is tightened to 1e-8 (the ABI's minimum) with up to 1024 iterations so
that the solves, which the adjoint treats as exact, are.
"""
import numpy as np
import pytest
import torch

from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

from tests.adjoint_harness import Rollout, cpu_adjoint, rollout_loss, trajectory  # noqa: E402


def tight(scene):
    scene.tolerance = 1e-8
    scene.max_iterations = 1024
    return scene


def gradients(scene, young32, x0, v0, steps, k, x_target):
    world = SimWorld(scene, precision="fp64")
    theta = torch.tensor(np.log(young32.astype(np.float64)), requires_grad=True)
    v0_t = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    xT = Rollout.apply(theta, v0_t, world, x0, steps, k)
    loss = 0.5 * torch.sum((xT - torch.from_numpy(x_target)) ** 2)
    loss.backward()
    return world, float(loss.detach()), theta.grad.numpy().copy(), v0_t.grad.numpy().copy()


def fd_theta(world, young32, x0, v0, steps, x_target, i, eps=1e-3):
    # The ABI takes float32 moduli: difference over the exactly represented log E values.
    yp, ym = young32.copy(), young32.copy()
    yp[i] = np.float32(young32[i] * np.exp(eps))
    ym[i] = np.float32(young32[i] * np.exp(-eps))
    lp = rollout_loss(world, yp, x0, v0, steps, x_target)
    lm = rollout_loss(world, ym, x0, v0, steps, x_target)
    return (lp - lm) / (np.log(np.float64(yp[i])) - np.log(np.float64(ym[i])))


def fd_v0(world, young32, x0, v0, steps, x_target, node, comp, eps=1e-3):
    vp, vm = v0.copy(), v0.copy()
    vp[node, comp] += eps
    vm[node, comp] -= eps
    lp = rollout_loss(world, young32, x0, vp, steps, x_target)
    lm = rollout_loss(world, young32, x0, vm, steps, x_target)
    return (lp - lm) / (2 * eps)


def target_for(scene, young_target, x0, v0, steps):
    w = SimWorld(scene, precision="fp64")
    w.set_tet_young(0, young_target)
    w.set_state(x0, v0, f64=True)
    for _ in range(steps):
        w.step()
    return w.state(f64=True)[0]


def test_adjoint_small_box_against_fd_and_cpu():
    scene = tight(meshes.small_box(3, 2, 2, young=2e4))
    body = scene.bodies[0]
    T = body.tets.shape[0]
    rng = np.random.default_rng(0)
    young = (2e4 * np.exp(rng.normal(0.0, 0.3, T))).astype(np.float32)
    young_t = (2e4 * np.exp(rng.normal(0.0, 0.3, T))).astype(np.float32)
    x0 = body.positions.astype(np.float64)
    v0 = np.zeros_like(x0)
    v0[~body.pinned] = rng.normal(0.0, 0.2, size=(int((~body.pinned).sum()), 3))
    steps, k = 6, 2
    x_target = target_for(scene, young_t, x0, v0, steps)
    world, loss, g_theta, g_v0 = gradients(scene, young, x0, v0, steps, k, x_target)
    assert loss > 0
    c_theta, c_v0 = cpu_adjoint(scene, young, x0, v0, steps, x_target,
                                trajectory=trajectory(world, young, x0, v0, steps))
    free = ~body.pinned
    assert np.linalg.norm(g_theta - c_theta) <= 1e-6 * np.linalg.norm(c_theta)
    assert np.linalg.norm(g_v0[free] - c_v0[free]) <= 1e-6 * np.linalg.norm(c_v0[free])
    # Relative to each coordinate's own finite difference (no floor).
    for i in range(0, T, max(1, T // 8)):
        fd = fd_theta(world, young, x0, v0, steps, x_target, i)
        assert abs(g_theta[i] - fd) <= 1e-4 * abs(fd), (i, g_theta[i], fd)
    nodes = np.nonzero(free)[0]
    for node in nodes[:: max(1, len(nodes) // 4)]:
        fd = fd_v0(world, young, x0, v0, steps, x_target, node, 2)
        assert abs(g_v0[node, 2] - fd) <= 1e-4 * abs(fd), (node, g_v0[node, 2], fd)


def test_adjoint_beam32_rollout_workload():
    scene = tight(meshes.config5(theta_seed=3))
    body = scene.bodies[0]
    T = body.tets.shape[0]
    young = body.tet_young.astype(np.float32)
    young_target = np.exp(meshes.config5_theta(4, T)).astype(np.float32)
    x0 = body.positions.astype(np.float64)
    v0 = np.zeros_like(x0)
    steps, k = scene.steps, 10
    x_target = target_for(scene, young_target, x0, v0, steps)
    world, loss, g_theta, g_v0 = gradients(scene, young, x0, v0, steps, k, x_target)
    assert loss > 0 and np.all(np.isfinite(g_theta)) and np.all(np.isfinite(g_v0))
    # FP64 CPU reference gradient, every coordinate, along the GPU rollout's trajectory.
    c_theta, c_v0 = cpu_adjoint(scene, young, x0, v0, steps, x_target,
                                trajectory=trajectory(world, young, x0, v0, steps))
    free = ~body.pinned
    assert np.linalg.norm(g_theta - c_theta) <= 1e-6 * np.linalg.norm(c_theta)
    assert np.linalg.norm(g_v0[free] - c_v0[free]) <= 1e-6 * np.linalg.norm(c_v0[free])
    # Central differences on 16 random coordinates of (log E, v0).
    rng = np.random.default_rng(16)
    free_nodes = np.nonzero(free)[0]
    # Each coordinate against its own central difference, Richardson-extrapolated from eps
    # and eps/2 ((4 D(eps/2) - D(eps)) / 3: truncation error O(eps^4) instead of O(eps^2)):
    # |adjoint - fd| <= 1e-4 |fd| + tol_cg |g|.  The second term is the one the method
    # itself leaves: the adjoint differentiates steps whose solves are exact, the
    # differences a rollout whose CG stops at relative residual tol_cg = 1e-8, and the two
    # derivatives differ by about tol_cg times the gradient's scale (measured: a coordinate
    # of 7.2e-6 whose differences agree to 5 digits from eps 2e-3 to 1e-4 sits 2.1e-9 from
    # the adjoint, with |g| = 0.33).
    gscale = float(np.sqrt(np.sum(g_theta ** 2) + np.sum(g_v0[free] ** 2)))
    errors = []
    for c in range(16):
        if c % 2 == 0:
            i = int(rng.integers(0, T))
            d1 = fd_theta(world, young, x0, v0, steps, x_target, i)
            d2 = fd_theta(world, young, x0, v0, steps, x_target, i, eps=5e-4)
            ad = g_theta[i]
        else:
            node, comp = int(rng.choice(free_nodes)), int(rng.integers(0, 3))
            d1 = fd_v0(world, young, x0, v0, steps, x_target, node, comp)
            d2 = fd_v0(world, young, x0, v0, steps, x_target, node, comp, eps=5e-4)
            ad = g_v0[node, comp]
        fd = (4.0 * d2 - d1) / 3.0
        errors.append((abs(ad - fd) / (1e-4 * abs(fd) + scene.tolerance * gscale), ad, fd, d1))
    assert max(e[0] for e in errors) <= 1.0, errors
    # The most sensitive coordinate (a tet at the clamped end that is nearly crushed flat,
    # where the rollout is strongly nonlinear): central differences converge to the
    # adjoint as the step shrinks; at 1e-5 they agree to 1e-4.
    i = int(np.argmax(np.abs(g_theta)))
    fd = fd_theta(world, young, x0, v0, steps, x_target, i, eps=1e-5)
    assert abs(g_theta[i] - fd) <= 1e-4 * abs(fd), (i, g_theta[i], fd)

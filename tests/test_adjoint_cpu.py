"""The FP64 CPU reference gradient of the rollout (tests/adjoint_harness.py), itself
checked without a GPU: central finite differences (epsilon 1e-3 on log E and on v0) of
L = 1/2 |x_T - x_target|^2 over FP64 oracle rollouts agree with it to 1e-4 relative.
This pins the adjoint derivation (element terms, polar-factor derivative, velocity and
position propagation) that the GPU kernel implements and is compared against."""
import numpy as np

from physik_b200 import meshes

from tests.adjoint_harness import cpu_adjoint, oracle_rollout_loss


def test_cpu_adjoint_matches_oracle_finite_differences():
    scene = meshes.small_box(3, 2, 2, young=2e4)
    scene.tolerance, scene.max_iterations = 1e-8, 1024
    body = scene.bodies[0]
    T = body.tets.shape[0]
    rng = np.random.default_rng(1)
    young = (2e4 * np.exp(rng.normal(0.0, 0.3, T))).astype(np.float32)
    young_t = (2e4 * np.exp(rng.normal(0.0, 0.3, T))).astype(np.float32)
    x0 = body.positions.astype(np.float64)
    v0 = np.zeros_like(x0)
    free = ~body.pinned
    v0[free] = rng.normal(0.0, 0.2, size=(int(free.sum()), 3))
    steps = 4
    _, x_target = oracle_rollout_loss(scene, young_t, x0, v0, steps, np.zeros_like(x0))
    g_theta, g_v0 = cpu_adjoint(scene, young, x0, v0, steps, x_target)
    scale_t, scale_v = np.abs(g_theta).max(), np.abs(g_v0[free]).max()
    for i in range(0, T, 5):
        yp, ym = young.copy(), young.copy()
        yp[i] = np.float32(young[i] * np.exp(1e-3))
        ym[i] = np.float32(young[i] * np.exp(-1e-3))
        lp, _ = oracle_rollout_loss(scene, yp, x0, v0, steps, x_target)
        lm, _ = oracle_rollout_loss(scene, ym, x0, v0, steps, x_target)
        fd = (lp - lm) / (np.log(np.float64(yp[i])) - np.log(np.float64(ym[i])))
        assert abs(g_theta[i] - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale_t), (i, g_theta[i], fd)
    for node in np.nonzero(free)[0][::7]:
        for comp in range(3):
            vp, vm = v0.copy(), v0.copy()
            vp[node, comp] += 1e-3
            vm[node, comp] -= 1e-3
            lp, _ = oracle_rollout_loss(scene, young, x0, vp, steps, x_target)
            lm, _ = oracle_rollout_loss(scene, young, x0, vm, steps, x_target)
            fd = (lp - lm) / 2e-3
            assert abs(g_v0[node, comp] - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale_v), (node, comp, g_v0[node, comp], fd)

"""FP64 outer true-residual refinement of the mixed-precision solve (PHYSIK_B200_SetRefinement).

No counterpart in the reference (it solves once, in FP32).  Checked here, on the GPU:

* when the refined step reports convergence, the true residual of its delta-v, recomputed
  here in FP64 from the assembled system (SparseBlockMatrix::Multiply semantics,
  src/Math/SparseBlockMatrix.cpp:209-268), meets the reference's stopping target
  r^T M^-1 r <= tol^2 b^T M^-1 b (ConjugateGradientSolver.cpp:114-241), the total CG
  iterations stay within the step's budget, and positions match the FP64 oracle to 3e-7
  (ten times the mixed step's measured position error);
* at the iteration cap (the 64x16x16 beam) no budget is left: the refined step equals
  the plain one;
* FP64 worlds ignore it, and a world with graph capture on still steps (refined steps
  are never captured) and equals a plain refined world bit for bit.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

from tests.test_ring_tiling import sym_upper_spmv  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def true_residual(world):
    g = world.system()
    rs, col = g["row_start"].astype(np.int64), g["col"].astype(np.int64)
    vals = np.asarray(g["values"], np.float64).reshape(-1)
    b, minv, dv = g["rhs"], g["minv"], g["dv"]
    r = b - sym_upper_spmv(rs, col, vals, dv)
    M = minv.transpose(0, 2, 1)  # column-major blocks -> matrices
    rho = float(np.einsum("ni,nij,nj->", r, M, r))
    rho0 = float(np.einsum("ni,nij,nj->", b, M, b))
    return rho, rho0


def test_refined_step_meets_the_true_residual_target():
    scene = meshes.config1()
    tol = scene.tolerance
    gpu = SimWorld(scene, precision="mixed")
    gpu.set_refinement(4)
    ora = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(3):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        assert st["iterations"] <= scene.max_iterations
        x, _ = gpu.state(f64=True)
        assert rel(x, ora.x) <= 3e-7
        if st["converged"]:
            rho, rho0 = true_residual(gpu)
            assert rho <= tol * tol * rho0 * (1 + 1e-3), (rho, tol * tol * rho0)


def test_refinement_without_budget_equals_the_plain_step():
    scene = meshes.config2()  # 100-iteration cap reached by the first solve
    plain = SimWorld(scene, precision="mixed")
    refined = SimWorld(scene, precision="mixed")
    refined.set_refinement(4)
    for _ in range(2):
        plain.step()
        refined.step()
    xp, vp = plain.state(f64=True)
    xr, vr = refined.state(f64=True)
    assert refined.cg_stats()["iterations"] == plain.cg_stats()["iterations"] == scene.max_iterations
    assert rel(xr, xp) <= 1e-12 and rel(vr, vp) <= 1e-10


def test_fp64_ignores_refinement_and_graph_steps_stay_plain():
    scene = meshes.small_box(5, 4, 3)
    a = SimWorld(scene, precision="fp64")
    b = SimWorld(scene, precision="fp64")
    b.set_refinement(3)
    for _ in range(3):
        a.step()
        b.step()
    np.testing.assert_array_equal(a.state(f64=True)[0], b.state(f64=True)[0])
    g = SimWorld(scene, precision="mixed")
    p = SimWorld(scene, precision="mixed")
    for w in (g, p):
        w.set_refinement(2)
    g.set_graph(True)
    for _ in range(4):
        g.step()
        p.step()
    assert g.cg_stats()["flags"] & L.FLAG_INTEGRATED
    np.testing.assert_array_equal(g.state(f64=True)[0], p.state(f64=True)[0])
    np.testing.assert_array_equal(g.state(f64=True)[1], p.state(f64=True)[1])

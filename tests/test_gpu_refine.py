"""FP64 outer true-residual refinement of the mixed-precision solve (PHYSIK_B200_SetRefinement).

No counterpart in the reference (it solves once, in FP32).  The refinement measures the
residual of the FP64 system -- recomputed element by element from the tets in FP64
(FP64 rest data, FP64 polar rotation and stress), not from the FP32-stored blocks -- and
corrects the solution until that residual meets the reference's stopping target.
Checked here, on the GPU:

* when the refined step reports convergence, the residual of its delta-v in the FP64
  system the FP64 oracle assembles from the same inputs (SparseBlockMatrix::Multiply
  semantics, src/Math/SparseBlockMatrix.cpp:209-268) meets the target
  r^T M^-1 r <= tol^2 b^T M^-1 b (ConjugateGradientSolver.cpp:114-241), the total CG
  iterations stay within the step's budget, and positions match the FP64 oracle to 3e-7;
* on a converging configuration with a tight tolerance the refined step's velocity error
  against the FP64 oracle is far below the plain mixed step's (the plain step is limited
  by the FP32 assembly and recursion, the refined one by the tolerance);
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


def fp64_residual(world, oracle_system):
    """r^T M^-1 r of the world's delta-v in the FP64 oracle's system, and b^T M^-1 b."""
    g = world.system()
    o = oracle_system
    np.testing.assert_array_equal(g["row_start"], o.row_start)
    np.testing.assert_array_equal(g["col"], o.col)
    rs, col = o.row_start.astype(np.int64), o.col.astype(np.int64)
    vals = np.asarray(o.values, np.float64).reshape(-1)
    b, dv = o.rhs, g["dv"]
    r = b - sym_upper_spmv(rs, col, vals, dv)
    M = np.asarray(g["minv"], np.float64).transpose(0, 2, 1)  # column-major blocks -> matrices
    rho = float(np.einsum("ni,nij,nj->", r, M, r))
    rho0 = float(np.einsum("ni,nij,nj->", b, M, b))
    return rho, rho0


def float_state(ora):
    """The oracle's state rounded to float32 -- what an FP32-stored world holds -- set back
    into the oracle, so both step from the same numbers."""
    x = ora.x.astype(np.float32).astype(np.float64)
    v = ora.v.astype(np.float32).astype(np.float64)
    ora.set_state(x, v)
    return x, v


def test_refined_step_meets_the_fp64_residual_target():
    scene = meshes.config1()
    tol = scene.tolerance
    gpu = SimWorld(scene, precision="mixed")
    gpu.set_refinement(4)
    ora = po.Oracle(scene, "f64", float_inputs=True)
    converged = 0
    for _ in range(3):
        x0, v0 = float_state(ora)
        gpu.set_state(x0, v0, f64=True)
        gpu.step()
        ora.step()
        assert gpu.cg_stats()["flags"] & L.FLAG_REFINED_FP64
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        assert st["iterations"] <= scene.max_iterations
        x, _ = gpu.state(f64=True)
        assert rel(x, ora.x) <= 3e-7
        if st["converged"]:
            converged += 1
            rho, rho0 = fp64_residual(gpu, ora.last_system())
            # the oracle's FP64 system and the element-wise one differ by rounding only
            assert rho <= tol * tol * rho0 * 1.01, (rho, tol * tol * rho0)
    assert converged > 0


def test_refinement_lowers_the_velocity_error_on_a_converging_config():
    scene = meshes.config1()
    scene.tolerance = 1e-8  # the ABI's minimum
    scene.max_iterations = 1024
    ora = po.Oracle(scene, "f64", float_inputs=True)
    plain = SimWorld(scene, precision="mixed")
    refined = SimWorld(scene, precision="mixed")
    refined.set_refinement(8)
    errs = []
    for _ in range(3):
        x0, v0 = float_state(ora)
        for w in (plain, refined):
            w.set_state(x0, v0, f64=True)
            w.step()
        ora.step()
        ep = rel(plain.state(f64=True)[1], ora.v)
        er = rel(refined.state(f64=True)[1], ora.v)
        errs.append((ep, er))
        assert refined.cg_stats()["flags"] & L.FLAG_INTEGRATED
        assert refined.cg_stats()["converged"]
    # refined: limited by the tolerance (1e-8); plain: by the FP32 assembly and recursion
    for ep, er in errs:
        assert er < 0.1 * ep, errs


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

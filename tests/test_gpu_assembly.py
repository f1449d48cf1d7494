"""The assembly kernels' variants agree (TetMeshPhysicsComponent::UpdateSystem +
SolverData::AssembleImplicitMatrixAndRhs, TetMeshPhysicsComponent.cpp:293-354,
SolverData.cpp:308-465).

* The four-lanes-per-row kernel (default) and the one-thread-per-row kernel
  (PK_ROW_KERNEL=thread) produce the same blocks, right-hand side and block-Jacobi inverse
  bit for bit: every slot receives its tets' blocks in tet order in both.
* The folded right-hand side (the tet kernel's T g_a term, default) and the long form
  (PK_ASSEMBLY_FOLD=0: all 16 blocks per tet and sum_b K_ab v_b in the row kernel) give
  the same blocks bit for bit, and right-hand sides that differ only by rounding
  (measured: relative 2e-16 in FP64).
* Both equal the FP64 oracle's assembled system (the reference restated in C) to the
  FP64 tolerances of the world tests.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402


def scenes():
    two = meshes.small_box(9, 6, 5)
    two.bodies += meshes.small_box(7, 8, 4, young=5e4, seed=11).bodies
    two.bodies[1].initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32),
                                               (two.bodies[1].positions.shape[0], 1))
    moving = meshes.config1()
    rng = np.random.default_rng(5)
    moving.bodies[0].initial_velocities = rng.normal(0, 0.3, moving.bodies[0].positions.shape).astype(np.float32)
    moving.bodies[0].initial_velocities[moving.bodies[0].pinned] = 0.0
    return {"cube8_moving": moving, "two_bodies": two}


def assembled(scene, precision, monkeypatch, **env):
    for k in ("PK_ROW_KERNEL", "PK_ASSEMBLY_FOLD"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    w = SimWorld(scene, precision=precision)
    w.step()  # from a moving state (the scenes start with velocities)
    return w.system()


@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("name", ["cube8_moving", "two_bodies"])
def test_lanes_and_thread_rows_are_bit_identical(name, precision, monkeypatch):
    scene = scenes()[name]
    a = assembled(scene, precision, monkeypatch)
    b = assembled(scene, precision, monkeypatch, PK_ROW_KERNEL="thread")
    for key in ("values", "rhs", "minv"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_folded_rhs_matches_the_long_form(precision, monkeypatch):
    scene = scenes()["cube8_moving"]
    a = assembled(scene, precision, monkeypatch)
    b = assembled(scene, precision, monkeypatch, PK_ASSEMBLY_FOLD="0")
    np.testing.assert_array_equal(a["values"], b["values"])
    np.testing.assert_array_equal(a["minv"], b["minv"])
    scale = np.abs(b["rhs"]).max()
    tol = 2e-6 if precision == "fp32" else 2e-15
    assert np.abs(a["rhs"] - b["rhs"]).max() <= tol * scale


@pytest.mark.parametrize("env", [{}, {"PK_ROW_KERNEL": "thread"}, {"PK_ASSEMBLY_FOLD": "0"}],
                         ids=["lanes_folded", "thread_folded", "long_form"])
def test_assembly_variants_match_fp64_oracle(env, monkeypatch):
    scene = scenes()["cube8_moving"]
    for k in ("PK_ROW_KERNEL", "PK_ASSEMBLY_FOLD"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    w = SimWorld(scene, precision="fp64")
    ora = po.Oracle(scene, "f64", float_inputs=True)
    w.set_state(ora.x, ora.v, f64=True)
    w.step()
    ora.step()
    g = w.system()
    o = ora.last_system()
    np.testing.assert_array_equal(g["row_start"], o.row_start)
    np.testing.assert_array_equal(g["col"], o.col)
    vs = np.abs(o.values).max()
    assert np.abs(g["values"] - o.values).max() <= 1e-13 * vs
    rs = np.abs(o.rhs).max()
    assert np.abs(g["rhs"] - o.rhs).max() <= 1e-13 * rs
    ms = np.abs(o.minv).max()
    assert np.abs(g["minv"] - o.minv).max() <= 1e-13 * ms

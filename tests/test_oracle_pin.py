"""Pins the oracle (the C restatement in oracle/pk_oracle.c) to the reference.

* Against the committed fixtures made by tests/golden/make_golden.py from the
  reference's own code: bit-exact in FP32 and in the float->double build.
* Against the reference compiled here (oracle/_ref) when it is present: bit-exact
  on further scenes, including per-element Young's modulus and multi-body worlds.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes


def _two_bodies():
    two = meshes.small_box(2, 2, 2)
    two.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    return two


def _check_steps(scene, fixture, precision, steps, with_system):
    o = po.Oracle(scene, precision)
    if with_system:
        o_sys = None
    for s in range(steps):
        o.step()
        if s == 0 and with_system:
            o_sys = o.last_system()
        np.testing.assert_array_equal(o.x.astype(np.float64), fixture[f"{precision}_x"][s])
        np.testing.assert_array_equal(o.v.astype(np.float64), fixture[f"{precision}_v"][s])
        st = o.last_stats()
        assert st["iterations"] == int(fixture[f"{precision}_cg"][s][0])
        assert st["converged"] == int(fixture[f"{precision}_cg"][s][1])
        assert st["residual"] == fixture[f"{precision}_cg"][s][2]
    if with_system:
        p = precision
        np.testing.assert_array_equal(o_sys.row_start, fixture[f"{p}_sys_row_start"])
        np.testing.assert_array_equal(o_sys.col, fixture[f"{p}_sys_col"])
        for name in ("values", "rhs", "minv", "dv", "mass", "force"):
            np.testing.assert_array_equal(getattr(o_sys, name).astype(np.float64), fixture[f"{p}_sys_{name}"])
        np.testing.assert_array_equal(o_sys.node_to_dyn, fixture[f"{p}_sys_node_to_dyn"])


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_oracle_matches_reference_fixture_box(golden_dir, precision):
    fx = np.load(f"{golden_dir}/box_steps.npz")
    _check_steps(meshes.small_box(2, 2, 2), fx, precision, 3, True)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_oracle_matches_reference_fixture_cube8(golden_dir, precision):
    fx = np.load(f"{golden_dir}/cube8_steps.npz")
    _check_steps(meshes.config1(), fx, precision, 2, False)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_oracle_matches_reference_fixture_two_bodies(golden_dir, precision):
    fx = np.load(f"{golden_dir}/two_bodies.npz")
    _check_steps(_two_bodies(), fx, precision, 2, True)


def test_oracle_matches_reference_fixture_tet_young(golden_dir):
    fx = np.load(f"{golden_dir}/beam32_tet_young.npz")
    _check_steps(meshes.config5(), fx, "f64", 1, False)


def test_kat_spmv_and_patterns(golden_dir):
    k = np.load(f"{golden_dir}/kat_bsr.npz")
    # Values stated by the reference's tests (PointConnectionTests.cpp:1983-2050).
    np.testing.assert_allclose(k["a_y"], [[14, 19, 24], [19, 26, 33]])
    np.testing.assert_allclose(k["b_y"], [[34, 81, 128], [42, 51, 60]])
    for p in ("f32", "f64"):
        np.testing.assert_array_equal(po.oracle_bsr_multiply(k["a_row_start"], k["a_col"], k["a_values"], k["a_x"], p),
                                      k["a_y"])
        np.testing.assert_array_equal(po.oracle_bsr_multiply(k["b_row_start"], k["b_col"], k["b_values"], k["b_x"], p),
                                      k["b_y"])
    # Single tet: 10 canonical blocks, row lengths 4,3,2,1; two adjacent tets: 14 blocks.
    np.testing.assert_array_equal(k["tet1_row_start"], [0, 4, 7, 9, 10])
    assert k["tet2_row_start"][-1] == 14
    pairs = [(a, b) for a in range(4) for b in range(4)]
    rs, col = po.oracle_build_pattern(4, [p[0] for p in pairs], [p[1] for p in pairs])
    np.testing.assert_array_equal(rs, k["tet1_row_start"])
    np.testing.assert_array_equal(col, k["tet1_col"])


@pytest.mark.parametrize("case", ["c", "d", "e"])
def test_kat_pcg(golden_dir, case):
    k = np.load(f"{golden_dir}/kat_bsr.npz")
    minv = k[f"{case}_minv"] if f"{case}_minv" in k else np.stack([np.eye(3)] * (len(k[f"{case}_row_start"]) - 1))
    max_it = {"c": 16, "d": 32, "e": 8}[case]
    x, st = po.oracle_pcg(k[f"{case}_row_start"], k[f"{case}_col"], k[f"{case}_values"], k[f"{case}_b"], minv,
                          max_it, 1e-6, "f32")
    np.testing.assert_array_equal(x.astype(np.float64), k[f"{case}_x"])
    assert st["iterations"] == int(k[f"{case}_it"])
    assert st["converged"] == int(k[f"{case}_conv"])


def test_kat_pcg_stated_answers(golden_dir):
    k = np.load(f"{golden_dir}/kat_bsr.npz")
    np.testing.assert_allclose(k["c_x"], [[1, 2, 3]], atol=1e-4)
    np.testing.assert_allclose(k["d_x"], [[1, 2, 3], [4, 5, 6]], atol=1e-4)
    np.testing.assert_array_equal(k["e_x"], [[0, 0, 0]])  # d.q <= 0 breakdown: x stays 0
    assert int(k["e_conv"]) == 0


def test_pcg_invalid_settings_clear_output():
    rs, col = np.array([0, 1], np.int32), np.array([0], np.int32)
    vals = np.eye(3)[None]
    b = np.array([[1.0, 0, 0]])
    for max_it, tol in ((0, 1e-6), (8, 0.0), (8, np.inf)):
        x, st = po.oracle_pcg(rs, col, vals, b, np.eye(3)[None], max_it, tol, "f32")
        assert x is None and st["converged"] == 0


def test_polar_rigid_rotation_and_fallback():
    rz = np.array([[0.0, -1, 0], [1, 0, 0], [0, 0, 1]])
    r, it = po.oracle_polar(rz.T, "f64")  # column-major in, column-major out
    np.testing.assert_allclose(r.T, rz, atol=1e-12)
    r, it = po.oracle_polar(np.zeros(9), "f64")  # |det| <= 1e-8 -> identity, no iterations
    np.testing.assert_array_equal(r, np.eye(3))
    assert it == 0
    refl = np.diag([1.0, 1.0, -1.0])  # reflection: column 2 is negated to a rotation
    r, _ = po.oracle_polar(refl.T, "f64")
    assert np.linalg.det(r.T) > 0


@pytest.mark.skipif(not po.reference_available("f32") or not po.reference_available("f64"),
                    reason="reference not built here (make -C oracle ref)")
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_oracle_matches_live_reference_multibody_and_edge_cases(precision):
    """Live pin: a jittered two-body world (one coupled PCG) with an initial velocity
    on the second body, four steps -- bit-exact against the reference."""
    scene = _two_bodies()
    scene.bodies[1].initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32),
                                                 (scene.bodies[1].positions.shape[0], 1))
    o = po.Oracle(scene, precision)
    r = po.Reference(scene, precision)
    for s in range(4):
        o.step()
        sr = r.system()
        r.step()
        x, v = r.state()
        np.testing.assert_array_equal(o.x.astype(np.float64), x)
        np.testing.assert_array_equal(o.v.astype(np.float64), v)
        osys = o.last_system()
        np.testing.assert_array_equal(osys.row_start, sr.row_start)
        np.testing.assert_array_equal(osys.col, sr.col)
        np.testing.assert_array_equal(osys.values.astype(np.float64), sr.values)
        np.testing.assert_array_equal(osys.dv.astype(np.float64), sr.dv)
        assert o.last_stats()["iterations"] == r.cg_stats()["iterations"]

"""Step-level parity of the drop-in C ABI (PHYSIK_Step on the GPU) against the oracle.

Comparisons are teacher-forced: both sides start every checked step from the same
state, so the error is that of one step.  Tolerances (relative, 2-norm) are about ten
times the largest error measured on a B200 over these scenes:
* FP64 GPU vs FP64 oracle fed the same float32 inputs the C ABI passes (dt, gravity,
  material): positions 1e-15, velocities 1e-13 (measured 8e-17 / 4e-15: summation order
  only).
* FP32 GPU vs FP32 reference restatement: positions 3e-7, velocities 2.5e-5 (measured
  3.5e-8 / 2.3e-6).
* mixed GPU vs FP64 oracle: positions 3e-7, velocities 5e-5 (measured 3e-8 / 4.5e-6; the
  FP32 reference itself is 2.8e-8 / 4.9e-6 from FP64 on these steps).
CG iteration counts may differ by one when the residual sits at the tolerance.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

TOL = {"fp64": (1e-15, 1e-13, 1), "fp32": (3e-7, 2.5e-5, 1), "mixed": (3e-7, 5e-5, 1)}
ORACLE = {"fp64": "f64", "fp32": "f32", "mixed": "f64"}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def two_bodies():
    s = meshes.small_box(2, 2, 2)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    s.bodies[1].initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32),
                                             (s.bodies[1].positions.shape[0], 1))
    return s


SCENES = {
    "box3x2x2": lambda: meshes.small_box(3, 2, 2),
    "cube8": meshes.config1,
    "two_bodies": two_bodies,
    "beam32_tet_young": meshes.config5,
}


def teacher_forced(scene, precision, steps):
    gpu = SimWorld(scene, precision=precision)
    ora = po.Oracle(scene, ORACLE[precision], float_inputs=precision == "fp64")
    worst = [0.0, 0.0, 0]
    for _ in range(steps):
        gpu.set_state(ora.x, ora.v, f64=True)
        x_prev = ora.x.copy()
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        worst[0] = max(worst[0], rel(x, ora.x))
        worst[1] = max(worst[1], rel(v, ora.v))
        worst[2] = max(worst[2], abs(st["iterations"] - ora.last_stats()["iterations"]))
        assert np.linalg.norm(ora.x - x_prev) > 0
    return worst


@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("name", list(SCENES))
def test_step_parity(name, precision):
    tx, tv, ti = TOL[precision]
    ex, ev, di = teacher_forced(SCENES[name](), precision, 3)
    assert ex <= tx, (ex, ev, di)
    assert ev <= tv, (ex, ev, di)
    assert di <= ti, (ex, ev, di)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_assembled_system_matches_oracle(precision):
    scene = two_bodies()
    gpu = SimWorld(scene, precision=precision)
    ora = po.Oracle(scene, ORACLE[precision], float_inputs=precision == "fp64")
    gpu.step()
    ora.step()
    g = gpu.system()
    o = ora.last_system()
    np.testing.assert_array_equal(g["row_start"], o.row_start)
    np.testing.assert_array_equal(g["col"], o.col)
    tol = 1e-12 if precision == "fp64" else 2e-5
    scale = np.abs(o.values).max()
    np.testing.assert_allclose(g["values"], o.values, rtol=0, atol=tol * scale)
    np.testing.assert_allclose(g["rhs"], o.rhs, rtol=0, atol=tol * np.abs(o.rhs).max() * 10)
    np.testing.assert_allclose(g["minv"], o.minv, rtol=0, atol=tol * np.abs(o.minv).max() * 10)
    assert rel(g["dv"], o.dv) < (1e-12 if precision == "fp64" else 2e-4)


def test_rollout_matches_fp32_reference_cube8():
    """Free 20-step rollout, FP32 GPU vs the FP32 reference: drift stays small."""
    scene = meshes.config1()
    gpu = SimWorld(scene, precision="fp32")
    ref = po.Oracle(scene, "f32")
    for _ in range(20):
        gpu.step()
        ref.step()
    x, v = gpu.state(f64=True)
    assert rel(x, ref.x) < 1e-5
    assert rel(v, ref.v) < 5e-3


def test_mixed_beats_position_bar_on_beam():
    """64x16x16 beam (CG capped at 100 iterations): mixed vs FP64 oracle, teacher-forced."""
    scene = meshes.config2()
    gpu = SimWorld(scene, precision="mixed")
    ora = po.Oracle(scene, "f64")
    gpu.set_state(ora.x, ora.v, f64=True)
    gpu.step()
    ora.step()
    x, v = gpu.state(f64=True)
    assert rel(x, ora.x) <= 2e-7  # measured 1.6e-8
    assert rel(v, ora.v) <= 2e-4  # measured 1.9e-5; the FP32 reference itself: 2.3e-5
    assert gpu.cg_stats()["iterations"] == ora.last_stats()["iterations"] == 100


def test_nan_velocity_leaves_state_unchanged():
    scene = meshes.small_box(2, 2, 2)
    gpu = SimWorld(scene, precision="fp32")
    x0, v0 = gpu.state()
    v0 = v0.copy()
    free = np.nonzero(~scene.bodies[0].pinned)[0]
    v0[free[0]] = np.nan
    gpu.set_state(x0, v0)
    gpu.step()
    x1, v1 = gpu.state()
    st = gpu.cg_stats()
    assert st["flags"] & L.FLAG_PRECOMPUTE_FAILED
    assert not st["flags"] & L.FLAG_INTEGRATED
    np.testing.assert_array_equal(x1, x0)
    assert st["iterations"] == 0 and st["converged"] == 0


def test_deactivated_tets_match_oracle():
    """PHYSIK_SetTetActive removes tets from forces and mass; nodes no tet references become inactive."""
    import ctypes as C
    scene = meshes.small_box(3, 2, 2)
    gpu = SimWorld(scene, precision="fp64")
    comp = gpu.components[0]
    off = [0, 1, 2, 3, 4, 5, 30]
    for t in off:
        L.PX.PHYSIK_SetTetActive(gpu.h, comp, t, 0)
    ora = po.Oracle(scene, "f64", float_inputs=True)
    active = np.ones(scene.tet_count, np.uint8)
    active[off] = 0
    ora.set_tet_active(active)
    tets = scene.bodies[0].tets
    node_active = np.zeros(scene.vertex_count, np.uint8)
    node_active[np.unique(tets[active.astype(bool)])] = 1
    ora.set_node_flags(active=node_active)
    ora.v[node_active == 0] = 0.0
    for _ in range(2):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        assert rel(x, ora.x) < 1e-14
        assert rel(v, ora.v) < 1e-12


def test_explicit_mode_matches_reference():
    scene = meshes.small_box(2, 2, 2, young=1e3)
    gpu = SimWorld(scene, precision="fp32", implicit=False)
    if not po.reference_available("f32"):
        pytest.skip("reference build not present")
    ref = po.Reference(scene, "f32")
    ref.lib.ref_world_settings.argtypes  # noqa: B018
    import ctypes as C
    g = np.array(scene.gravity, np.float64)
    ref.lib.ref_world_settings(ref.h, 0, g.ctypes.data_as(C.c_void_p), scene.max_iterations, scene.tolerance, 1)
    for _ in range(3):
        gpu.step(1e-3)
        ref.step(1e-3)
    x, v = gpu.state(f64=True)
    xr, vr = ref.state()
    assert rel(x, xr) < 1e-6
    assert rel(v, vr) < 1e-4


def test_unstaged_spmv_fallback_matches_oracle(monkeypatch):
    """The PCG kernel without shared-memory tiles (used when a row does not fit a
    tile) gives the same step as the staged one."""
    monkeypatch.setenv("PK_PCG_STAGED", "0")
    ex, ev, di = teacher_forced(two_bodies(), "fp64", 2)
    assert ex <= 1e-14 and ev <= 1e-12 and di <= 1, (ex, ev, di)


def test_staged_and_unstaged_agree_on_beam():
    """Staged and unstaged SpMV on the 64x16x16 beam: same iterations, same state to rounding."""
    import os
    scene = meshes.config2()
    out = []
    for flag in ("1", "0"):
        os.environ["PK_PCG_STAGED"] = flag
        try:
            w = SimWorld(scene, precision="fp64")
            for _ in range(2):
                w.step()
            out.append((w.state(f64=True), w.cg_stats()["iterations"]))
        finally:
            os.environ.pop("PK_PCG_STAGED", None)
    (xa, va), ia = out[0]
    (xb, vb), ib = out[1]
    assert ia == ib
    assert rel(xa, xb) < 1e-13 and rel(va, vb) < 1e-9


def test_deactivation_between_steps_keeps_device_state():
    """Tets deactivated between steps while their nodes stay in other tets: the pattern is
    unchanged, so only masses and tet data go to the device again and its FP64 state carries
    over exactly; the following free steps match the oracle with the same tets off."""
    scene = meshes.small_box(3, 2, 2)
    gpu = SimWorld(scene, precision="fp64")
    ora = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(2):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
    off = [30, 40]
    active = np.ones(scene.tet_count, np.uint8)
    active[off] = 0
    tets = scene.bodies[0].tets
    assert len(np.unique(tets[active.astype(bool)])) == scene.vertex_count  # every node stays in a tet
    for t in off:
        L.PX.PHYSIK_SetTetActive(gpu.h, gpu.components[0], t, 0)
    ora.set_tet_active(active)
    for _ in range(2):
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        assert rel(x, ora.x) < 1e-14, rel(x, ora.x)
        assert rel(v, ora.v) < 1e-12, rel(v, ora.v)

"""The FEM model switch (TetMeshPhysicsComponent::SetFemModel through
PHYSIK_B200_SetTetMeshFemModel) on the GPU against the reference.

* Linear FEM (FemModel::Linear -> FEMModel::ComputeElasticForces, FEMModel.cpp:580-612:
  R = I, K = Ke): FP64 GPU vs the FP64 oracle run with the linear model (positions 1e-14,
  velocities 1e-12), FP32 GPU vs the FP32 reference itself with its
  component switched to the linear model, in implicit and explicit mode.
* NeoHookean (not implemented by the reference: ComputeForces returns false and the
  component emits masses only, TetMeshPhysicsComponent.cpp:322-353): the body falls
  under gravity alone, as in the reference.
* Mixed models in one world: one body linear, one corotated.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

needs_ref = pytest.mark.skipif(not po.reference_available("f32"), reason="reference not built (make -C oracle ref)")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def bent_box():
    """A box that starts deformed (rotated half, moving) so linear and corotated differ."""
    s = meshes.small_box(4, 2, 2, young=2e4, seed=3)
    b = s.bodies[0]
    p = b.positions.astype(np.float64)
    ang = 0.4 * p[:, 0] / p[:, 0].max()
    c, sn = np.cos(ang), np.sin(ang)
    q = p.copy()
    q[:, 1] = c * p[:, 1] - sn * p[:, 2]
    q[:, 2] = sn * p[:, 1] + c * p[:, 2]
    b.initial_positions = q.astype(np.float32)
    b.initial_velocities = np.tile(np.array([0.0, 0.2, -0.1], np.float32), (p.shape[0], 1))
    b.initial_velocities[b.pinned] = 0.0
    return s


def set_model(w, body, model):
    assert w.X.PHYSIK_B200_SetTetMeshFemModel(w.h, w.components[body], model) == 1


def test_linear_fp64_matches_oracle():
    scene = bent_box()
    gpu = SimWorld(scene, precision="fp64")
    set_model(gpu, 0, 0)
    ora = po.Oracle(scene, "f64", linear=True, float_inputs=True)
    cor = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(3):
        gpu.set_state(ora.x, ora.v, f64=True)
        cor.set_state(ora.x, ora.v)
        gpu.step()
        ora.step()
        cor.step()
        x, v = gpu.state(f64=True)
        assert gpu.cg_stats()["flags"] & L.FLAG_INTEGRATED
        # measured 4e-17 / 9e-16
        assert rel(x, ora.x) <= 1e-14 and rel(v, ora.v) <= 1e-12, (rel(x, ora.x), rel(v, ora.v))
        assert abs(gpu.cg_stats()["iterations"] - ora.last_stats()["iterations"]) <= 1
        assert rel(cor.v, ora.v) > 1e-3  # the models really differ on this motion


@needs_ref
@pytest.mark.parametrize("implicit", [True, False], ids=["implicit", "explicit"])
def test_linear_fp32_matches_reference(implicit):
    scene = bent_box()
    gpu = SimWorld(scene, precision="fp32", implicit=implicit)
    set_model(gpu, 0, 0)
    ref = po.Reference(scene, "f32")
    ref.set_fem_model(0, 0)
    if not implicit:
        g = np.array(scene.gravity, np.float64)
        ref.lib.ref_world_settings(ref.h, 0, g.ctypes.data, scene.max_iterations, scene.tolerance, 1)
    dt = scene.dt if implicit else 1e-4
    for _ in range(3):
        x0, v0 = ref.state()
        gpu.set_state(x0, v0, f64=True)
        gpu.step(dt)
        ref.step(dt)
        x, v = gpu.state(f64=True)
        xr, vr = ref.state()
        assert rel(x, xr) <= 1e-6, rel(x, xr)
        assert rel(v, vr) <= (5e-5 if implicit else 1e-5), rel(v, vr)


@needs_ref
def test_neohookean_emits_masses_only_as_the_reference():
    scene = bent_box()
    scene.dt, scene.gravity = 1.0 / 64.0, (0.0, 0.0, -9.8125)  # float-exact: the double reference sees the same
    gpu = SimWorld(scene, precision="fp64")
    set_model(gpu, 0, 2)
    ref = po.Reference(scene, "f64")
    ref.set_fem_model(0, 2)
    for _ in range(2):
        gpu.step()
        ref.step()
    x, v = gpu.state(f64=True)
    xr, vr = ref.state()
    assert rel(x, xr) <= 1e-9 and rel(v, vr) <= 1e-9, (rel(x, xr), rel(v, vr))


def test_mixed_models_in_one_world():
    s = bent_box()
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    s.bodies[1].positions = s.bodies[1].positions + np.float32(2.0)
    # one coupled CG solves both bodies here, two separate ones in the oracles: solve tightly
    # (the C ABI's smallest tolerance) so every solve is close to the exact one
    s.tolerance, s.max_iterations = 1e-8, 1000
    gpu = SimWorld(s, precision="fp64")
    set_model(gpu, 0, 0)
    one = lambda b: meshes.Scene("one", [b], dt=s.dt, steps=1, tolerance=s.tolerance,  # noqa: E731
                                 max_iterations=s.max_iterations)
    lin = po.Oracle(one(s.bodies[0]), "f64", linear=True, float_inputs=True)
    cor = po.Oracle(one(s.bodies[1]), "f64", float_inputs=True)
    gpu.step()
    lin.step()
    cor.step()
    x, v = gpu.state(f64=True)
    n0 = s.bodies[0].positions.shape[0]
    assert rel(x[:n0], lin.x) <= 1e-8 and rel(x[n0:], cor.x) <= 1e-8

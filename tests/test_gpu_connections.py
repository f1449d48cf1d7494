"""Transient point connections on the device (PHYSIK_AddPointConnection) against the reference.

The reference's PointConnection::UpdateSystem (src/Core/PhysicsConnections/PointConnection.cpp:
55-140) adds, per connection, its spring-and-damper force times each corner's weight and the
blocks stiffness * w_i * w_j * I between its corners to SolverData, which assembles them with
the FEM contributions (SolverData.cpp:308-465); World::Step clears the connections when the
frame ends (World.cpp:32-73, 727-746).  The checker is the reference itself compiled with
float -> double (oracle/_ref/libphysik_ref_f64.so).  Every input is a float32 value (the C
ABI takes floats): dt 1/64, gravity -9.8125, Poisson's ratio 0.25, CG tolerance 2^-20.

Tolerances (relative, 2-norm): FP64 system blocks and rhs 1e-12 of their largest entry,
delta-v 1e-8; FP64 steps positions 1e-14, velocities 1e-12; mixed steps positions 3e-7,
velocities 2e-4 (about ten times the step errors measured without connections).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

needs_ref = pytest.mark.skipif(not po.reference_available("f64"), reason="reference not built (make -C oracle ref)")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def exact_scene():
    s = meshes.small_box(2, 2, 2, poisson=0.25)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, poisson=0.25, seed=11).bodies
    s.dt = 1.0 / 64.0
    s.gravity = (0.0, 0.0, -9.8125)
    s.tolerance = 2.0 ** -20
    return s


def f32(values):
    return tuple(float(np.float32(v)) for v in values)


def connections(scene):
    """Inside body 0 (with damping), across the bodies, with a pinned corner, without
    stiffness (force only), and with repeated nodes."""
    n0 = scene.bodies[0].positions.shape[0]
    pinned0 = int(np.nonzero(scene.bodies[0].pinned)[0][0])
    return [
        ((1, 4, 6, 7), (0.25, 0.25, 0.25, 0.25), f32((0.05, 0.12, 0.3)), 40.0, 0.5),
        ((5, n0 + 7, 0, 0), (0.5, 0.5, 0.0, 0.0), f32((0.1, 0.1, 0.1)), 80.0, 0.0),
        ((pinned0, 8, 2, 3), f32((0.4, 0.3, 0.2, 0.1)), f32((0.0, -0.1, 0.2)), 25.0, 0.25),
        ((n0 + 2, n0 + 3, n0 + 9, n0 + 10), f32((0.1, 0.2, 0.3, 0.4)), f32((0.3, 0.0, 0.0)), 0.0, 1.0),
        ((n0 + 5, n0 + 5, n0 + 6, n0 + 6), f32((0.3, 0.2, 0.25, 0.25)), f32((0.2, 0.2, 0.0)), 15.0, 0.0),
    ]


def random_state(scene, seed=3):
    """The scene's positions and a float32 velocity field, zero on the pinned nodes."""
    rng = np.random.default_rng(seed)
    x = np.concatenate([b.positions for b in scene.bodies]).astype(np.float32).astype(np.float64)
    v = rng.normal(0.0, 0.2, x.shape).astype(np.float32).astype(np.float64)
    v[np.concatenate([b.pinned for b in scene.bodies])] = 0.0
    return x, v


def add_all(scene, *worlds):
    for c in connections(scene):
        for w in worlds:
            w.add_point_connection(*c)


@needs_ref
def test_connection_system_matches_reference_fp64():
    scene = exact_scene()
    gpu = SimWorld(scene, precision="fp64")
    ref = po.Reference(scene, "f64")
    x, v = random_state(scene)
    gpu.set_state(x, v, f64=True)
    ref.set_state(x, v)
    add_all(scene, gpu, ref)
    assert gpu.point_connection_count() == ref.point_connection_count() == len(connections(scene))
    o = ref.system()
    gpu.step()
    assert gpu.point_connection_count() == 0
    g = gpu.system()
    np.testing.assert_array_equal(g["row_start"], o.row_start)
    np.testing.assert_array_equal(g["col"], o.col)
    tol = 1e-12
    np.testing.assert_allclose(g["values"], o.values, rtol=0, atol=tol * np.abs(o.values).max())
    np.testing.assert_allclose(g["rhs"], o.rhs, rtol=0, atol=tol * np.abs(o.rhs).max() * 10)
    np.testing.assert_allclose(g["minv"], o.minv, rtol=0, atol=tol * np.abs(o.minv).max() * 10)
    assert rel(g["dv"], o.dv) < 1e-8


@needs_ref
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_connection_steps_match_reference(precision):
    """Teacher-forced steps, the connections added again before each (frame lifetime)."""
    tx, tv, ti = {"fp64": (1e-14, 1e-12, 1), "mixed": (3e-7, 2e-4, 1)}[precision]
    scene = exact_scene()
    gpu = SimWorld(scene, precision=precision)
    ref = po.Reference(scene, "f64")
    x, v = random_state(scene)
    ref.set_state(x, v)
    for _ in range(3):
        xr, vr = ref.state()
        gpu.set_state(xr, vr, f64=True)
        add_all(scene, gpu, ref)
        gpu.step()
        assert ref.step() == 0
        xg, vg = gpu.state(f64=True)
        xr, vr = ref.state()
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        assert rel(xg, xr) <= tx, rel(xg, xr)
        assert rel(vg, vr) <= tv, rel(vg, vr)
        assert abs(st["iterations"] - ref.cg_stats()["iterations"]) <= ti
        assert gpu.point_connection_count() == ref.point_connection_count() == 0


def test_step_after_connections_equals_a_world_without_them():
    """The pattern returns to the bodies' own once the connections are gone."""
    scene = exact_scene()
    a = SimWorld(scene, precision="fp64")
    b = SimWorld(scene, precision="fp64")
    x, v = random_state(scene)
    a.set_state(x, v, f64=True)
    add_all(scene, a)
    a.step()
    x1, v1 = a.state(f64=True)
    assert np.linalg.norm(x1 - x) > 0
    b.prepare(upload=True)  # FP64 state goes to the device only once it holds the scene
    b.set_state(x1, v1, f64=True)
    a.step()
    b.step()
    np.testing.assert_array_equal(a.state(f64=True)[0], b.state(f64=True)[0])
    np.testing.assert_array_equal(a.state(f64=True)[1], b.state(f64=True)[1])
    assert len(a.system()["col"]) == len(b.system()["col"])


@needs_ref
def test_connection_forces_in_explicit_mode_match_reference():
    scene = exact_scene()
    gpu = SimWorld(scene, precision="fp64", implicit=False)
    ref = po.Reference(scene, "f64")
    import ctypes as C
    g = np.array(scene.gravity, np.float64)
    ref.lib.ref_world_settings(ref.h, 0, g.ctypes.data_as(C.c_void_p), scene.max_iterations, scene.tolerance, 1)
    x, v = random_state(scene)
    gpu.set_state(x, v, f64=True)
    ref.set_state(x, v)
    for _ in range(3):
        add_all(scene, gpu, ref)
        gpu.step(2.0 ** -10)
        ref.step(2.0 ** -10)
    xg, vg = gpu.state(f64=True)
    xr, vr = ref.state()
    assert rel(xg, xr) < 1e-12
    assert rel(vg, vr) < 1e-10


def test_batched_and_graph_worlds_solve_connections_coupled():
    """A connection across two bodies couples them: a batched world and a world with CUDA
    graphs on step exactly as the plain coupled world, and batching resumes after."""
    scene = exact_scene()
    worlds = [SimWorld(scene, precision="mixed") for _ in range(3)]
    worlds[1].set_batched(True)
    worlds[2].set_graph(True)
    x, v = random_state(scene)
    for w in worlds:
        w.set_state(x, v, f64=True)
    for step in range(3):
        if step < 2:
            add_all(scene, *worlds)
        for w in worlds:
            w.step()
            assert w.cg_stats()["flags"] & L.FLAG_INTEGRATED
        if step < 2:
            for w in worlds[1:]:
                np.testing.assert_array_equal(w.state(f64=True)[0], worlds[0].state(f64=True)[0])
                np.testing.assert_array_equal(w.state(f64=True)[1], worlds[0].state(f64=True)[1])
    # Batched again (per-body statistics available) once the connections are gone.
    assert worlds[1].body_stats(0)["iterations"] >= 1

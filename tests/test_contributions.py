"""Host-emitted SolverData contributions (SolverData::AddNodeMass / AddNodeForce /
AddStiffnessBlock, SolverData.h:41-54) from custom components, against the reference.

The reference's soft bodies, point connections and any custom C++ component feed the
implicit system through these calls; the drop-in's device step computes the soft bodies
and connections itself and takes the rest as host-emitted extras: masses join the lumped
masses in emission order (before or after the body's own, by execution priority) and may
make a node dynamic, forces join the rhs, blocks join the pattern and the matrix (the
upper triangle; a lower block whose upper twin is emitted too is dropped, as
SolverData.cpp:407-450 does) and add -dt^2 B v_column to the rhs of their row.  Here the
custom component is a contribution component (PHYSIK_B200_CreateContributionComponent)
whose callback emits through the C ABI; the reference runs the same callback from a C++
component of its own (oracle/ref_harness.cpp).

Without a GPU: the host scene -- masses, dynamic mapping and the pattern joined with the
emitted blocks -- equals the reference's bit for bit.  With a GPU (marked): the assembled
FP64 system and three FP64 steps against the reference compiled in double, and FP32 steps
against the FP32 reference; a non-finite block skips the step.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

needs_ref = pytest.mark.skipif(not po.reference_available("f64"), reason="reference not built (make -C oracle ref)")

OURS = C.CFUNCTYPE(None, C.c_void_p, C.c_float, C.c_void_p)
THEIRS = C.CFUNCTYPE(None, C.c_void_p, C.c_double, C.c_void_p)


def exact_scene():
    """Two bodies with every input exactly a float32 value (the double reference then sees
    the same numbers)."""
    s = meshes.small_box(2, 2, 2, poisson=0.25)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, poisson=0.25, seed=11).bodies
    s.dt = 1.0 / 64.0
    s.gravity = (0.0, 0.0, -9.8125)
    s.tolerance = 2.0 ** -20
    return s


def emissions(scene, bad_block=False):
    """Two emitters: (priority, [(kind, args)]): one before the soft bodies, one after."""
    n0 = scene.bodies[0].positions.shape[0]
    pinned = int(np.nonzero(scene.bodies[0].pinned)[0][0])
    B = np.array([[3.0, 0.5, 0.25], [0.5, 2.0, 0.0], [0.25, 0.0, 1.5]])  # symmetric
    Cb = np.array([[1.0, 0.25, 0.0], [0.125, 1.0, 0.5], [0.0, 0.5, 2.0]])  # not symmetric
    early = [("mass", (3, 0.015625)), ("force", (4, (0.125, 0.0, 0.25))), ("mass", (n0 + 5, 0.03125)),
             ("mass", (7, -1.0)), ("force", (5, (float("nan"), 0.0, 0.0))), ("mass", (10 ** 6, 1.0))]
    late = [("block", (2, n0 + 3, B)), ("block", (n0 + 3, 2, B.T)),       # both orientations
            ("block", (n0 + 7, 6, Cb)),                                   # lower one only
            ("block", (3, 3, 0.5 * np.eye(3))), ("block", (8, pinned, Cb)),  # column fixed: rhs only
            ("block", (4, 10 ** 6, B)), ("mass", (3, 0.0078125)), ("force", (n0 + 2, (0.0, -0.5, 0.0)))]
    if bad_block:
        late.append(("block", (1, 2, np.full((3, 3), np.inf))))
    return [(100, early), (1000, late)]


def attach_ours(w, emitters):
    X = L.PX
    keep = []
    for priority, items in emitters:
        def cb(sd, dt, user, items=items):
            for kind, args in items:
                if kind == "mass":
                    X.PHYSIK_B200_SolverDataAddNodeMass(sd, args[0], args[1])
                elif kind == "force":
                    X.PHYSIK_B200_SolverDataAddNodeForce(sd, args[0], *args[1])
                else:
                    blk = (C.c_float * 9)(*np.asarray(args[2], np.float64).T.reshape(-1))  # column-major
                    X.PHYSIK_B200_SolverDataAddStiffnessBlock(sd, args[0], args[1], blk)
        fn = OURS(cb)
        h = X.PHYSIK_B200_CreateContributionComponent(w.h, priority)
        X.PHYSIK_B200_SetContributionCallback(w.h, h, C.cast(fn, C.c_void_p), None)
        keep.append(fn)
    return keep


def attach_theirs(ref, emitters):
    R = ref.lib
    for priority, items in emitters:
        def cb(sd, dt, user, items=items):
            for kind, args in items:
                if kind == "mass":
                    R.ref_solverdata_add_mass(sd, args[0], args[1])
                elif kind == "force":
                    R.ref_solverdata_add_force(sd, args[0], *args[1])
                else:
                    blk = np.ascontiguousarray(np.asarray(args[2], np.float64).T.reshape(-1))
                    R.ref_solverdata_add_block(sd, args[0], args[1], blk.ctypes.data_as(C.c_void_p))
        assert ref.add_contribution(priority, THEIRS(cb)) == 1


@needs_ref
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_host_scene_with_emitted_masses_and_blocks_matches_reference(precision):
    scene = exact_scene()
    em = emissions(scene)
    w = SimWorld(scene, precision=precision)
    keep = attach_ours(w, em)  # noqa: F841  (callbacks stay alive)
    ref = po.Reference(scene, "f32" if precision == "fp32" else "f64")
    attach_theirs(ref, em)
    w.prepare(upload=False)
    rs, col, n2d, mass = w.pattern()
    s = ref.system()
    np.testing.assert_array_equal(n2d, s.node_to_dyn)
    np.testing.assert_array_equal(mass, s.mass)  # emission order kept: bit for bit
    np.testing.assert_array_equal(rs, s.row_start)
    np.testing.assert_array_equal(col, s.col)
    plain = SimWorld(scene, precision=precision)
    plain.prepare(upload=False)
    assert len(col) > len(plain.pattern()[1])  # the block joining the bodies is in


@pytest.mark.gpu
@needs_ref
def test_fp64_system_and_steps_follow_reference():
    scene = exact_scene()
    em = emissions(scene)
    w = SimWorld(scene, precision="fp64")
    keep = attach_ours(w, em)  # noqa: F841
    ref = po.Reference(scene, "f64")
    attach_theirs(ref, em)
    g_first = True
    for _ in range(3):
        if g_first:
            s = ref.system()  # the system of the coming step, from the same state
        w.step()
        ref.step()
        if g_first:
            g = w.system()
            np.testing.assert_array_equal(g["row_start"], s.row_start)
            np.testing.assert_array_equal(g["col"], s.col)
            scale = np.abs(s.values).max()
            np.testing.assert_allclose(g["values"], s.values, rtol=0, atol=1e-12 * scale)
            np.testing.assert_allclose(g["rhs"], s.rhs, rtol=0, atol=1e-12 * np.abs(s.rhs).max())
            g_first = False
        x, v = w.state(f64=True)
        xr, vr = ref.state()
        assert w.cg_stats()["flags"] & L.FLAG_INTEGRATED
        assert np.linalg.norm(x - xr) <= 1e-14 * np.linalg.norm(xr)
        assert np.linalg.norm(v - vr) <= 1e-12 * np.linalg.norm(vr)


@pytest.mark.gpu
@needs_ref
def test_fp32_steps_follow_fp32_reference():
    scene = exact_scene()
    em = emissions(scene)
    w = SimWorld(scene, precision="fp32")
    keep = attach_ours(w, em)  # noqa: F841
    ref = po.Reference(scene, "f32")
    attach_theirs(ref, em)
    for _ in range(3):
        x0, v0 = ref.state()
        w.set_state(x0, v0, f64=True)
        w.step()
        ref.step()
        x, v = w.state(f64=True)
        xr, vr = ref.state()
        assert np.linalg.norm(x - xr) <= 3e-7 * np.linalg.norm(xr)
        assert np.linalg.norm(v - vr) <= 2.5e-5 * np.linalg.norm(vr)


@pytest.mark.gpu
def test_non_finite_block_skips_the_step():
    scene = exact_scene()
    w = SimWorld(scene, precision="fp64")
    keep = attach_ours(w, emissions(scene, bad_block=True))  # noqa: F841
    x0, v0 = w.state(f64=True)
    w.step()
    x, v = w.state(f64=True)
    np.testing.assert_array_equal(x, x0)
    np.testing.assert_array_equal(v, v0)
    assert w.cg_stats()["flags"] & L.FLAG_PRECOMPUTE_FAILED

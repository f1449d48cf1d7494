"""PHYSIK_GetTetMeshLocalCurrentPosition / PHYSIK_SetTetMeshLocalCurrentPosition
(PhysiKAPI.h:236-251, PhysiKAPI.cpp:992-1053) against the reference.

A tet mesh keeps its own copy of its node positions (TetMeshComponent::nodePositions).
A physics mesh refreshes it from the world in every substep it takes part in and again
at the end of the frame (TetMeshPhysicsComponent::UpdateSystem and PostUpdate ->
SyncCurrentPositionsFromWorld, TetMeshPhysicsComponent.cpp:234-252, 293-300, 356-363), so
after a step it holds the positions the step ended with; before the first step it holds
the generated mesh's positions.  Set writes that copy only (not the world's node) until
the next step overwrites it.

Without a GPU: creation positions, Set / Get round trips and the argument checks.  With a
GPU (marked): the copies after steps, against the reference driven through the same calls.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

needs_ref = pytest.mark.skipif(not po.reference_available("f32"), reason="reference not built (make -C oracle ref)")


def two_bodies():
    s = meshes.small_box(2, 2, 2)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    b = s.bodies[1]
    b.initial_positions = b.positions + np.float32(0.25)
    b.initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32), (b.positions.shape[0], 1))
    return s


@needs_ref
def test_creation_positions_and_set_get_match_reference():
    scene = two_bodies()
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    for body, b in enumerate(scene.bodies):
        count = b.positions.shape[0]
        got = w.local_positions(body)
        want = ref.local_positions(body, count)
        # the generated mesh's positions, not the world's initial state (body 1 starts moved)
        np.testing.assert_array_equal(got.astype(np.float64), want)
        np.testing.assert_array_equal(got, b.positions)
    assert w.set_local_position(1, 3, (1.0, 2.0, 3.0)) == 1
    ref.set_local_position(1, 3, (1.0, 2.0, 3.0))
    np.testing.assert_array_equal(w.local_positions(1).astype(np.float64),
                                  ref.local_positions(1, scene.bodies[1].positions.shape[0]))
    # Set does not move the world's node
    x, _ = w.state()
    begin = w.X.PHYSIK_GetTetMeshGlobalNodeBeginIndex(w.h, w.components[1])
    np.testing.assert_array_equal(x[begin + 3], scene.bodies[1].initial_positions[3])


def test_argument_checks():
    w = SimWorld(meshes.small_box(2, 2, 2))
    c = w.components[0]
    fx, fy, fz = C.c_float(7.0), C.c_float(), C.c_float()
    X = L.PX
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(w.h, c, -1, C.byref(fx), C.byref(fy), C.byref(fz)) == 0
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(w.h, c, 27, C.byref(fx), C.byref(fy), C.byref(fz)) == 0
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(w.h, c, 0, None, C.byref(fy), C.byref(fz)) == 0
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(None, c, 0, C.byref(fx), C.byref(fy), C.byref(fz)) == 0
    assert fx.value == 7.0  # out-pointers untouched on failure
    bad = L.ComponentHandle(0xFFFFFFFF, 0)
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(w.h, bad, 0, C.byref(fx), C.byref(fy), C.byref(fz)) == 0
    assert X.PHYSIK_SetTetMeshLocalCurrentPosition(w.h, c, 27, 1.0, 1.0, 1.0) == 0
    assert X.PHYSIK_SetTetMeshLocalCurrentPosition(None, c, 0, 1.0, 1.0, 1.0) == 0
    assert X.PHYSIK_GetTetMeshLocalCurrentPosition(w.h, c, 26, C.byref(fx), C.byref(fy), C.byref(fz)) == 1


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_copies_after_steps_match_reference(precision):
    scene = two_bodies()
    w = SimWorld(scene, precision=precision)
    ref = po.Reference(scene, "f32")
    sizes = [b.positions.shape[0] for b in scene.bodies]
    begins = [w.X.PHYSIK_GetTetMeshGlobalNodeBeginIndex(w.h, c) for c in w.components]
    for step in range(3):
        w.step()
        ref.step()
        x_end, _ = w.state()  # the state this step ended with
        xr, _ = ref.state()
        for body, count in enumerate(sizes):
            got = w.local_positions(body)
            # exactly the world's positions after the step (float32 copies of the state)
            np.testing.assert_array_equal(got, x_end[begins[body]:begins[body] + count])
            want = ref.local_positions(body, count)
            np.testing.assert_array_equal(want, xr[begins[body]:begins[body] + count])  # the reference's rule
            assert np.abs(got - want).max() <= 3e-7 * np.abs(want).max() + 1e-9
        # a Set lasts until the next step overwrites the copy, and does not move the node
        assert w.set_local_position(0, 2, (9.0, 9.0, 9.0)) == 1
        ref.set_local_position(0, 2, (9.0, 9.0, 9.0))
        assert tuple(w.local_positions(0)[2]) == (9.0, 9.0, 9.0)
        np.testing.assert_array_equal(w.local_positions(0)[2].astype(np.float64), ref.local_positions(0, sizes[0])[2])
        np.testing.assert_array_equal(w.state()[0][begins[0] + 2], x_end[begins[0] + 2])


@pytest.mark.gpu
@needs_ref
def test_copy_with_substeps_is_the_end_of_the_frame():
    """Two substeps per step: the copy holds the positions after the second substep."""
    scene = two_bodies()
    w = SimWorld(scene, precision="fp32")
    ref = po.Reference(scene, "f32", substeps=2)
    w.X.PHYSIK_SetSubstepCount(w.h, 2)
    w.step()
    ref.step()
    x_end, _ = w.state()
    begin = w.X.PHYSIK_GetTetMeshGlobalNodeBeginIndex(w.h, w.components[1])
    count = scene.bodies[1].positions.shape[0]
    got = w.local_positions(1)
    np.testing.assert_array_equal(got, x_end[begin:begin + count])
    want = ref.local_positions(1, count)
    assert np.abs(got - want).max() <= 3e-7 * np.abs(want).max() + 1e-9


@pytest.mark.gpu
def test_state_written_after_a_step_does_not_change_the_copy():
    scene = two_bodies()
    w = SimWorld(scene, precision="mixed")
    w.step()
    x_end, v_end = w.state()
    before = w.local_positions(0).copy()
    w.set_state(x_end + np.float32(1.0), v_end)  # moves every node; the copy keeps the frame's end
    np.testing.assert_array_equal(w.local_positions(0), before)
    w.step(0.0)  # a zero step runs no PostUpdate sync either
    np.testing.assert_array_equal(w.local_positions(0), before)

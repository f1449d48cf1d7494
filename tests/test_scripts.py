"""Script components (PHYSIK_CreateScriptComponent / PHYSIK_SetScriptComponentCallback /
PHYSIK_ClearScriptComponentCallback; PhysiKAPI.cpp:719-765, ScriptComponent.cpp).

A script's callback runs once per PHYSIK_Step, before the substeps (PreUpdate), with the
world handle, so it can drive the world through the C ABI -- here it pulls two bodies
together with a point connection whose target moves every frame.

Without a GPU: the callback runs once per frame (PHYSIK_Step with dt = 0 runs PreUpdate
and nothing else), receives the world handle and its user data, stops after it is
cleared, and invalid handles are ignored.  With a GPU (marked): three frames of a script
that adds a connection every frame, FP64 device step against the reference compiled in
double driven by the same script through its own C ABI (positions 1e-14, velocities 1e-12).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

CALLBACK = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)


def two_bodies():
    s = meshes.small_box(2, 2, 2)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    s.bodies[1].positions = s.bodies[1].positions + np.float32(0.05)
    return s


def test_callback_runs_once_per_frame_with_the_world_and_stops_when_cleared():
    w = SimWorld(meshes.small_box(2, 2, 2))
    X = L.PX
    calls = []

    def cb(world, user):
        calls.append((world, user))

    fn = CALLBACK(cb)
    h = X.PHYSIK_CreateScriptComponent(w.h)
    assert h.valid() and X.PHYSIK_IsComponentHandleValid(w.h, h) == 1
    X.PHYSIK_SetScriptComponentCallback(w.h, h, C.cast(fn, C.c_void_p), C.c_void_p(1234))
    for _ in range(3):
        X.PHYSIK_Step(w.h, 0.0)
    assert len(calls) == 3 and all(c == (w.h, 1234) for c in calls)
    X.PHYSIK_ClearScriptComponentCallback(w.h, h)
    X.PHYSIK_Step(w.h, 0.0)
    assert len(calls) == 3
    # invalid handles and worlds are ignored
    bad = L.ComponentHandle(0xFFFFFFFF, 0)
    X.PHYSIK_SetScriptComponentCallback(w.h, bad, C.cast(fn, C.c_void_p), None)
    X.PHYSIK_SetScriptComponentCallback(w.h, w.components[0], C.cast(fn, C.c_void_p), None)  # not a script
    X.PHYSIK_SetScriptComponentCallback(None, h, C.cast(fn, C.c_void_p), None)
    X.PHYSIK_Step(w.h, 0.0)
    assert len(calls) == 3
    assert not X.PHYSIK_CreateScriptComponent(None).valid()
    X.PHYSIK_DestroyComponent(w.h, h)
    assert X.PHYSIK_IsComponentHandleValid(w.h, h) == 0


def _puller(add, n0):
    """A script: every frame a connection from node 5 of body 0 and node 7 of body 1 to a
    target that moves with the frame number (float32 values, as the C ABI passes them)."""
    frame = [0]

    def cb(world, user):
        t = np.float32(0.02) * np.float32(frame[0])
        target = [float(np.float32(0.3) + t), float(np.float32(0.1)), float(np.float32(0.2) - t)]
        add(world, 5, n0 + 7, 9, n0 + 12, [0.25, 0.25, 0.25, 0.25], target, 40.0, 0.5)
        frame[0] += 1

    return CALLBACK(cb)


@pytest.mark.gpu
@pytest.mark.skipif(not po.reference_available("f64"), reason="reference not built (make -C oracle ref)")
def test_script_driven_connections_follow_the_reference():
    from tests.test_gpu_connections import exact_scene  # every input exactly a float32 value

    scene = exact_scene()
    n0 = scene.bodies[0].positions.shape[0]
    gpu = SimWorld(scene, precision="fp64")
    ref = po.Reference(scene, "f64")
    X = L.PX

    def add_gpu(world, a, b, c, d, wts, tgt, k, damp):
        X.PHYSIK_AddPointConnection(world, a, b, c, d, *wts, *tgt, k, damp)

    rl = ref.lib
    rl.PHYSIK_AddPointConnection.argtypes = [C.c_void_p] + [C.c_int] * 4 + [C.c_double] * 9
    rl.PHYSIK_AddPointConnection.restype = None

    def add_ref(world, a, b, c, d, wts, tgt, k, damp):
        rl.PHYSIK_AddPointConnection(world, a, b, c, d, *wts, *tgt, k, damp)

    fg, fr = _puller(add_gpu, n0), _puller(add_ref, n0)
    h = X.PHYSIK_CreateScriptComponent(gpu.h)
    X.PHYSIK_SetScriptComponentCallback(gpu.h, h, C.cast(fg, C.c_void_p), None)
    assert ref.add_script(fr) == 1
    for _ in range(3):
        gpu.step()
        ref.step()
        x, v = gpu.state(f64=True)
        xr, vr = ref.state()
        assert np.linalg.norm(x - xr) <= 1e-14 * np.linalg.norm(xr)
        assert np.linalg.norm(v - vr) <= 1e-12 * np.linalg.norm(vr)
        assert gpu.cg_stats()["flags"] & L.FLAG_INTEGRATED
    assert gpu.point_connection_count() == 0  # frame lifetime: gone after the step

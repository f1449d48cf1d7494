"""Collision spheres (PHYSIK_CreateCollisionSphereComponent, connection settings,
kinematic targets; CollisionSphereComponent.cpp:112-190, CollisionComponent.cpp,
PhysiKAPI.cpp:685-701, 1180-1218, 1407-1429) against the reference.

Every substep each active tet whose centroid ((x0/4 + x1/4) + x2/4) + x3/4 lies strictly
inside the sphere becomes a point connection pulling the centroid to the sphere's surface.
The contacts are found on the GPU (pk_system_sphere_contacts) with every operation rounded
once, as the reference's float code, so the set of contacts must equal the reference's.

Without a GPU: settings, their sanitising (negative or non-finite -> 0), defaults and
handle checks.  With a GPU (marked): the contact list of pk_system_sphere_contacts equals
a float32 recomputation of the reference's test; and three frames of a soft box pressed
by a sphere that moves (kinematic target) follow the reference in FP32 (positions 1e-6,
velocities 1e-4) and in FP64 against the reference compiled in double (positions 2e-8,
velocities 2e-6: the connection targets are stored as floats, as in the reference's float
API).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

needs_ref = pytest.mark.skipif(not po.reference_available("f32"), reason="reference not built (make -C oracle ref)")


def settings(w, h):
    k, c = C.c_float(-1.0), C.c_float(-1.0)
    L.PX.PHYSIK_GetCollisionSphereConnectionSettings(w.h, h, C.byref(k), C.byref(c))
    return k.value, c.value


def test_settings_defaults_and_handles():
    w = SimWorld(meshes.small_box(2, 2, 2))
    X = L.PX
    h = w.add_sphere((0.5, 0.5, 1.2), 0.3)
    assert settings(w, h) == (1000.0, 10.0)
    X.PHYSIK_SetCollisionSphereConnectionSettings(w.h, h, 250.0, 2.5)
    assert settings(w, h) == (250.0, 2.5)
    X.PHYSIK_SetCollisionSphereConnectionSettings(w.h, h, -3.0, float("nan"))
    assert settings(w, h) == (0.0, 0.0)
    X.PHYSIK_SetCollisionSphereConnectionSettings(w.h, h, float("inf"), 4.0)
    assert settings(w, h) == (0.0, 4.0)
    # invalid handles: ignored, out-pointers untouched
    bad = L.ComponentHandle(0xFFFFFFFF, 0)
    X.PHYSIK_SetCollisionSphereConnectionSettings(w.h, bad, 1.0, 1.0)
    assert settings(w, bad) == (-1.0, -1.0)
    assert settings(w, w.components[0]) == (-1.0, -1.0)  # a tet mesh is not a sphere
    X.PHYSIK_SetCollisionComponentKinematicTarget(w.h, w.components[0], 1.0, 2.0, 3.0)  # ignored
    assert not X.PHYSIK_CreateCollisionSphereComponent(None, 0.0, 0.0, 0.0, 1.0).valid()
    neg = w.add_sphere((0.0, 0.0, 0.0), -2.0)  # radius clamped at 0: never any contact
    assert X.PHYSIK_IsComponentHandleValid(w.h, neg) == 1


def pressed_box():
    """A 4x3x3 box over 0.4 x 0.3 x 0.3 (x=0 pinned) whose free end sits inside a sphere
    (14 tet centroids inside at rest).  Every input is exact in float (dt 1/64, gravity
    -9.8125, Poisson 0.3125, the sphere's centre and radius), so the FP64 run and the
    reference compiled in double see the same numbers."""
    s = meshes.small_box(4, 3, 3, young=2e4, poisson=0.3125, seed=4)
    s.dt = 1.0 / 64.0
    s.gravity = (0.0, 0.0, -9.8125)
    return s, (0.4375, 0.15625, 0.15625), 0.125


def reference_contacts(x, tets, center, radius):
    """The reference's test in float32, operation by operation (numpy rounds each)."""
    x = x.astype(np.float32)
    w = np.float32(0.25)
    p = ((x[tets[:, 0]] * w + x[tets[:, 1]] * w) + x[tets[:, 2]] * w) + x[tets[:, 3]] * w
    d = p - np.asarray(center, np.float32)
    dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    return np.nonzero(dist < np.float32(radius))[0], p


@pytest.mark.gpu
def test_device_contact_list_equals_the_float_test():
    scene, center, radius = pressed_box()
    w = SimWorld(scene, precision="fp32")
    w.step()  # uploads the scene; positions now moved by one step
    x, _ = w.state()
    X = L.PK
    tets = scene.bodies[0].tets
    want, p = reference_contacts(x, tets, center, radius)
    assert 0 < len(want) < len(tets)
    sys_ptr = w.X.PHYSIK_B200_GetDeviceSystem(w.h)
    assert sys_ptr
    n = X.pk_system_sphere_contacts(sys_ptr, (C.c_double * 3)(*center), radius, 0, None, None)
    assert n == len(want)
    got = np.zeros(n, np.int32)
    pts = np.zeros((n, 3))
    assert X.pk_system_sphere_contacts(sys_ptr, (C.c_double * 3)(*center), radius, n,
                                       got.ctypes.data_as(C.c_void_p), pts.ctypes.data_as(C.c_void_p)) == n
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(pts.astype(np.float32), p[want])


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_pressed_box_with_moving_sphere_follows_reference(precision):
    scene, center, radius = pressed_box()
    gpu = SimWorld(scene, precision=precision)
    ref = po.Reference(scene, "f32" if precision == "fp32" else "f64")
    h = gpu.add_sphere(center, radius, 300.0, 1.0)
    s = ref.add_sphere(center, radius, 300.0, 1.0)
    # FP64: the contacts' targets pass through the host's float PointConnection (as they
    # would through the reference's float API), so the FP64 run differs from the reference
    # compiled in double by those roundings (measured 1.6e-9 in positions after 3 frames).
    tx, tv = (1e-6, 1e-4) if precision == "fp32" else (2e-8, 2e-6)
    for frame in range(3):
        c = (center[0] - 0.015625 * frame, center[1], center[2])
        L.PX.PHYSIK_SetCollisionComponentKinematicTarget(gpu.h, h, *c)
        ref.set_sphere_target(s, c)
        gpu.step()
        ref.step()
        x, v = gpu.state(f64=True)
        xr, vr = ref.state()
        assert np.linalg.norm(x - xr) <= tx * np.linalg.norm(xr), (frame, np.linalg.norm(x - xr) / np.linalg.norm(xr))
        assert np.linalg.norm(v - vr) <= tv * np.linalg.norm(vr), (frame, np.linalg.norm(v - vr) / np.linalg.norm(vr))
        assert gpu.cg_stats()["flags"] & L.FLAG_INTEGRATED
    # the sphere really pushed: the same box without it moves differently
    free = SimWorld(scene, precision=precision)
    for _ in range(3):
        free.step()
    assert np.linalg.norm(free.state(f64=True)[1] - v) > 1e-3 * np.linalg.norm(v)

"""ctypes wrappers for the CPU checkers of the CUDA path.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``    -- the C restatement in ``pk_oracle.c`` (``liboracle_f32.so`` / ``liboracle_f64.so``).
* ``Reference`` -- the reference compiled from its own sources plus ``ref_harness.cpp``
  (``_ref/libphysik_ref.so`` FP32, ``_ref/libphysik_ref_f64.so`` float->double).

Both take a ``physik_b200.meshes.Scene`` and advance it with one ``World::Step`` per
call, exposing the assembled system of the last step for kernel-level parity checks.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_i = C.c_int
_p = C.c_void_p
_d = C.c_double


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def oracle_library_path(precision: str) -> str:
    return os.path.join(HERE, f"liboracle_{precision}.so")


def reference_library_path(precision: str) -> str:
    name = "libphysik_ref.so" if precision == "f32" else "libphysik_ref_f64.so"
    return os.path.join(HERE, "_ref", name)


def reference_available(precision: str = "f32") -> bool:
    return os.path.exists(reference_library_path(precision))


@dataclass
class System:
    """The implicit system of one substep, as SolverData holds it."""

    row_start: np.ndarray
    col: np.ndarray
    values: np.ndarray  # (nnz, 3, 3) column-major: values[k, c, r] = B[r][c]
    rhs: np.ndarray  # (n, 3)
    minv: Optional[np.ndarray]  # (n, 3, 3) column-major
    dv: Optional[np.ndarray]  # (n, 3)
    node_to_dyn: np.ndarray
    mass: np.ndarray
    force: np.ndarray
    cg_iterations: int
    cg_residual: float
    cg_converged: int
    solved: int


def scene_arrays(scene):
    """Concatenate the bodies of a scene into world arrays (world node order)."""
    pos, rest, vel, tets, fixed = [], [], [], [], []
    body_tet_start, body_node_start, density = [0], [0], []
    young, poisson, damping = [], [], []
    off = 0
    for b in scene.bodies:
        V, T = b.positions.shape[0], b.tets.shape[0]
        rest.append(b.positions.astype(np.float32))
        pos.append((b.initial_positions if b.initial_positions is not None else b.positions).astype(np.float32))
        vel.append(b.initial_velocities.astype(np.float32) if b.initial_velocities is not None
                   else np.zeros((V, 3), np.float32))
        tets.append(b.tets.astype(np.int32) + off)
        fixed.append(b.pinned.astype(np.uint8))
        density.append(b.density)
        ty = b.tet_young if b.tet_young is not None else np.full(T, b.young)
        young.append(np.asarray(ty, dtype=np.float64))
        poisson.append(np.full(T, b.poisson, np.float64))
        damping.append(np.full(T, b.damping, np.float64))
        off += V
        body_tet_start.append(body_tet_start[-1] + T)
        body_node_start.append(off)
    return dict(
        rest=np.concatenate(rest), x=np.concatenate(pos), v=np.concatenate(vel),
        tets=np.concatenate(tets), fixed=np.concatenate(fixed),
        body_tet_start=np.array(body_tet_start, np.int32), body_node_start=np.array(body_node_start, np.int32),
        density=np.array(density, np.float64), young=np.concatenate(young),
        poisson=np.concatenate(poisson), damping=np.concatenate(damping),
    )


class Oracle:
    """The C restatement.  precision 'f32' reproduces the FP32 reference; 'f64' is the FP64 oracle."""

    def __init__(self, scene, precision: str = "f64", linear: bool = False, use_jacobi: bool = True,
                 float_inputs: bool = False):
        """float_inputs: round dt, gravity, material and tolerance to float32 first -- the
        values a caller of the float C ABI (PHYSIK_Step(float dt), PhysikMaterialDesc)
        actually passes -- so an FP64 device run can be checked against identical inputs."""
        self.precision = precision
        self.float_inputs = float_inputs
        self.dtype = np.float32 if precision == "f32" else np.float64
        self.lib = C.CDLL(oracle_library_path(precision))
        pre = f"pko_{precision}_"
        self._f = lambda name: getattr(self.lib, pre + name)
        self._f("create").restype = _p
        for n in ("destroy", "set_settings", "set_node_flags", "set_tet_active", "set_tet_young", "last_sizes",
                  "last_system", "tet_rest"):
            self._f(n).restype = None
        self._f("step").restype = _i
        a = scene_arrays(scene)
        if float_inputs:
            for key in ("density", "young", "poisson", "damping"):
                a[key] = a[key].astype(np.float32).astype(np.float64)
        self.arrays = a
        dt_ = self.dtype
        self.node_count = a["rest"].shape[0]
        self.tet_count = a["tets"].shape[0]
        self._keep = [a["rest"].astype(dt_), a["tets"], a["body_tet_start"], a["body_node_start"],
                      a["density"].astype(dt_), a["young"].astype(dt_), a["poisson"].astype(dt_),
                      a["damping"].astype(dt_)]
        k = self._keep
        self.h = self._f("create")(
            _i(self.node_count), _ptr(k[0]), _i(self.tet_count), _ptr(k[1]), _i(len(scene.bodies)), _ptr(k[2]),
            _ptr(k[3]), _ptr(k[4]), _ptr(k[5]), _ptr(k[6]), _ptr(k[7]))
        g = np.array(scene.gravity, np.float32 if float_inputs else np.float64).astype(dt_)
        tol = float(np.float32(scene.tolerance)) if float_inputs else scene.tolerance
        self._f("set_settings")(_p(self.h), _ptr(g), _i(scene.max_iterations),
                                (C.c_float if precision == "f32" else C.c_double)(tol),
                                _i(1 if use_jacobi else 0), _i(1 if linear else 0))
        self._fixed = a["fixed"].copy()
        self._active = np.ones(self.node_count, np.uint8)
        self._f("set_node_flags")(_p(self.h), _ptr(self._fixed), _ptr(self._active))
        self.x = a["x"].astype(dt_)
        self.v = a["v"].astype(dt_)
        self.v[self._fixed.astype(bool)] = 0.0
        self.dt = float(np.float32(scene.dt)) if float_inputs else scene.dt

    def __del__(self):
        if getattr(self, "h", None):
            self._f("destroy")(_p(self.h))
            self.h = None

    def set_state(self, x, v):
        # copies: step() updates the state in place, so it must not alias a caller's array
        self.x = np.array(x, dtype=self.dtype, order="C", copy=True)
        self.v = np.array(v, dtype=self.dtype, order="C", copy=True)

    def set_tet_young(self, young):
        y = np.ascontiguousarray(young, dtype=self.dtype)
        self._f("set_tet_young")(_p(self.h), _ptr(y))

    def set_tet_active(self, active):
        a = np.ascontiguousarray(active, dtype=np.uint8)
        self._f("set_tet_active")(_p(self.h), _ptr(a))

    def set_node_flags(self, fixed=None, active=None):
        if fixed is not None:
            self._fixed = np.ascontiguousarray(fixed, np.uint8)
        if active is not None:
            self._active = np.ascontiguousarray(active, np.uint8)
        self._f("set_node_flags")(_p(self.h), _ptr(self._fixed), _ptr(self._active))

    def step(self, dt: Optional[float] = None) -> int:
        dt = self.dt if dt is None else dt
        if self.float_inputs:
            dt = float(np.float32(dt))
        ctype = C.c_float if self.precision == "f32" else C.c_double
        self._f("step").argtypes = [_p, _p, _p, ctype]
        return self._f("step")(_p(self.h), _ptr(self.x), _ptr(self.v), ctype(dt))

    def last_stats(self):
        dyn, nnz, it, conv, flags = _i(), _i(), _i(), _i(), _i()
        res = _d()
        self._f("last_sizes")(_p(self.h), C.byref(dyn), C.byref(nnz), C.byref(it), C.byref(res), C.byref(conv),
                              C.byref(flags))
        return dict(dyn=dyn.value, nnz=nnz.value, iterations=it.value, residual=res.value,
                    converged=conv.value, flags=flags.value)

    def last_system(self) -> System:
        s = self.last_stats()
        n, nnz = s["dyn"], s["nnz"]
        dt_ = self.dtype
        rs = np.zeros(n + 1, np.int32)
        col = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros((max(nnz, 1), 3, 3), dt_)
        rhs = np.zeros((max(n, 1), 3), dt_)
        minv = np.zeros((max(n, 1), 3, 3), dt_)
        dv = np.zeros((max(n, 1), 3), dt_)
        n2d = np.zeros(self.node_count, np.int32)
        mass = np.zeros(self.node_count, dt_)
        force = np.zeros((self.node_count, 3), dt_)
        self._f("last_system")(_p(self.h), _ptr(rs), _ptr(col), _ptr(val), _ptr(rhs), _ptr(minv), _ptr(dv),
                               _ptr(n2d), _ptr(mass), _ptr(force))
        return System(rs, col[:nnz], val[:nnz], rhs[:n], minv[:n], dv[:n], n2d, mass, force,
                      s["iterations"], s["residual"], s["converged"], (s["flags"] >> 1) & 1)

    def tet_rest(self):
        vol = np.zeros(self.tet_count, self.dtype)
        dminv = np.zeros((self.tet_count, 3, 3), self.dtype)
        grads = np.zeros((self.tet_count, 4, 3), self.dtype)
        self._f("tet_rest")(_p(self.h), _ptr(vol), _ptr(dminv), _ptr(grads))
        return vol, dminv, grads


def _oracle_fn(precision, name, restype, argtypes):
    lib = C.CDLL(oracle_library_path(precision))
    f = getattr(lib, f"pko_{precision}_{name}")
    f.restype = restype
    f.argtypes = argtypes
    return f


def oracle_bsr_multiply(row_start, col, values, x, precision="f64"):
    dt_ = np.float32 if precision == "f32" else np.float64
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, dt_)
    xx = np.ascontiguousarray(x, dt_)
    y = np.zeros((n, 3), dt_)
    f = _oracle_fn(precision, "bsr_multiply", None, [_i, _p, _p, _p, _p, _p])
    f(n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(xx), _ptr(y))
    return y


def oracle_pcg(row_start, col, values, b, minv, max_iterations, tolerance, precision="f64"):
    dt_ = np.float32 if precision == "f32" else np.float64
    ctype = C.c_float if precision == "f32" else C.c_double
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, dt_)
    bb = np.ascontiguousarray(b, dt_)
    mm = np.ascontiguousarray(minv, dt_)
    x = np.zeros((max(n, 1), 3), dt_)
    it, conv = _i(), _i()
    res = _d()
    f = _oracle_fn(precision, "pcg", _i, [_i, _p, _p, _p, _p, _p, _i, _i, ctype, _p, _p, _p, _p])
    have = f(n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(bb), _ptr(mm), len(mm) if minv is not None else 0,
             max_iterations, ctype(tolerance), _ptr(x), C.byref(it), C.byref(res), C.byref(conv))
    return (x[:n] if have else None), dict(iterations=it.value, residual=res.value, converged=conv.value)


def oracle_build_pattern(n, rows, cols, precision="f64"):
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    f = _oracle_fn(precision, "build_pattern", _i, [_i, _p, _p, C.c_long, _p, _p, _i])
    rs = np.zeros(n + 1, np.int32)
    nnz = f(n, _ptr(rows), _ptr(cols), len(rows), _ptr(rs), None, 0)
    col = np.zeros(max(nnz, 1), np.int32)
    f(n, _ptr(rows), _ptr(cols), len(rows), _ptr(rs), _ptr(col), nnz)
    return rs, col[:nnz]


def oracle_polar(f9, precision="f64"):
    dt_ = np.float32 if precision == "f32" else np.float64
    fin = np.ascontiguousarray(f9, dt_).reshape(9)
    out = np.zeros(9, dt_)
    it = _i()
    fn = _oracle_fn(precision, "polar", None, [_p, _p, _p])
    fn(_ptr(fin), _ptr(out), C.byref(it))
    return out.reshape(3, 3), it.value


class RefHandle(C.Structure):
    """PhysiK::ComponentHandle (Handles.h:10-19)."""
    _fields_ = [("index", C.c_uint32), ("generation", C.c_uint32)]


class Reference:
    """The reference itself (compiled from its sources), driven through ref_harness.cpp."""

    def __init__(self, scene, precision: str = "f32", substeps: int = 1):
        path = reference_library_path(precision)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_world_create.restype = _p
        L.ref_world_destroy.argtypes = [_p]
        L.ref_world_settings.argtypes = [_p, _i, _p, _i, _d, _i]
        L.ref_add_body.argtypes = [_p, _p, _i, _p, _i, _d, _d, _d, _d]
        L.ref_add_body.restype = _i
        L.ref_set_tet_young.argtypes = [_p, _i, _p]
        L.ref_set_fixed.argtypes = [_p, _p, _i]
        L.ref_node_count.argtypes = [_p]
        L.ref_set_state.argtypes = [_p, _p, _p]
        L.ref_get_state.argtypes = [_p, _p, _p]
        L.ref_step.argtypes = [_p, _d]
        L.ref_step.restype = _i
        L.ref_cg_stats.argtypes = [_p, _p, _p, _p]
        L.ref_dump_begin.argtypes = [_p, _d, _p, _p]
        L.ref_dump_begin.restype = _i
        L.ref_dump_copy.argtypes = [_p] + [_p] * 9
        L.ref_dump_cg.argtypes = [_p, _p, _p, _p]
        L.ref_add_point_connection.argtypes = [_p, _p, _p, _p, _d, _d]
        L.ref_point_connection_count.argtypes = [_p]
        L.ref_point_connection_count.restype = _i
        self.h = L.ref_world_create()
        self.precision = precision
        self.dt = scene.dt
        g = np.array(scene.gravity, np.float64)
        L.ref_world_settings(self.h, 1, _ptr(g), scene.max_iterations, scene.tolerance, substeps)
        for bi, b in enumerate(scene.bodies):
            pos = np.ascontiguousarray(b.positions, np.float64)
            tets = np.ascontiguousarray(b.tets, np.int32)
            begin = L.ref_add_body(self.h, _ptr(pos), pos.shape[0], _ptr(tets), tets.shape[0], b.density,
                                   b.young, b.poisson, b.damping)
            if begin < 0:
                raise RuntimeError("reference rejected body")
            if b.tet_young is not None:
                ty = np.ascontiguousarray(b.tet_young, np.float64)
                L.ref_set_tet_young(self.h, bi, _ptr(ty))
        a = scene_arrays(scene)
        self.node_count = L.ref_node_count(self.h)
        fixed = np.ascontiguousarray(a["fixed"], np.uint8)
        L.ref_set_fixed(self.h, _ptr(fixed), self.node_count)
        v = a["v"].astype(np.float64)
        v[fixed.astype(bool)] = 0.0
        self.set_state(a["x"].astype(np.float64), v)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_world_destroy(self.h)
            self.h = None

    def set_tet_young(self, body, young):
        y = np.ascontiguousarray(young, np.float64)
        self.lib.ref_set_tet_young(self.h, body, _ptr(y))

    def add_sphere(self, center, radius, stiffness=1000.0, damping=10.0) -> int:
        """A CollisionSphereComponent with its connection settings; returns its index."""
        self.lib.ref_add_sphere.argtypes = [_p, _d, _d, _d, _d, _d, _d]
        self.lib.ref_add_sphere.restype = _i
        return self.lib.ref_add_sphere(self.h, *[float(c) for c in center], float(radius), float(stiffness),
                                       float(damping))

    def set_sphere_target(self, sphere, center):
        self.lib.ref_sphere_target.argtypes = [_p, _i, _d, _d, _d]
        self.lib.ref_sphere_target(self.h, sphere, *[float(c) for c in center])

    def add_contribution(self, priority, callback) -> int:
        """A component whose UpdateSystem calls `callback(solverData, dt, user)` (a ctypes
        CFUNCTYPE(None, c_void_p, c_double, c_void_p)); emit with solverdata_add_*."""
        L = self.lib
        L.ref_add_contribution.argtypes = [_p, _i, _p, _p]
        L.ref_add_contribution.restype = _i
        L.ref_solverdata_add_force.argtypes = [_p, _i, _d, _d, _d]
        L.ref_solverdata_add_mass.argtypes = [_p, _i, _d]
        L.ref_solverdata_add_block.argtypes = [_p, _i, _i, _p]
        self._contrib = getattr(self, "_contrib", []) + [callback]
        return L.ref_add_contribution(self.h, priority, C.cast(callback, C.c_void_p), None)

    def add_script(self, callback) -> int:
        """A ScriptComponent calling `callback` (a ctypes CFUNCTYPE(None, c_void_p, c_void_p))
        once per frame with the reference world's handle."""
        self.lib.ref_add_script.argtypes = [_p, _p, _p]
        self.lib.ref_add_script.restype = _i
        self._script = callback  # keep the callback alive as long as the world
        return self.lib.ref_add_script(self.h, C.cast(callback, C.c_void_p), None)

    def set_fem_model(self, body, model):
        """TetMeshPhysicsComponent::SetFemModel: 0 linear, 1 corotated, 2 NeoHookean."""
        self.lib.ref_set_fem_model.argtypes = [_p, _i, _i]
        self.lib.ref_set_fem_model(self.h, body, model)

    def local_positions(self, body, count):
        """TetMeshComponent::GetLocalCurrentPosition for every node of a body."""
        out = np.zeros((count, 3))
        self.lib.ref_get_local_positions.argtypes = [_p, _i, _p]
        self.lib.ref_get_local_positions(self.h, body, _ptr(out))
        return out

    def body_handle(self, body):
        """The reference's ComponentHandle of a body (for its own C ABI)."""
        out = np.zeros(2, np.uint32)
        self.lib.ref_body_handle.argtypes = [_p, _i, _p]
        self.lib.ref_body_handle(self.h, body, _ptr(out))
        return RefHandle(int(out[0]), int(out[1]))

    def world_handle(self):
        self.lib.ref_world_handle.restype = _p
        self.lib.ref_world_handle.argtypes = [_p]
        return self.lib.ref_world_handle(self.h)

    def api(self, name, restype, argtypes):
        """One of the reference's own PHYSIK_* C functions (its float arguments are double
        in the float->double build: use `self.real`)."""
        f = getattr(self.lib, name)
        f.restype = restype
        f.argtypes = argtypes
        return f

    @property
    def real(self):
        return C.c_float if self.precision == "f32" else C.c_double

    def set_local_position(self, body, node, p):
        self.lib.ref_set_local_position.argtypes = [_p, _i, _i, _d, _d, _d]
        self.lib.ref_set_local_position(self.h, body, node, *[float(c) for c in p])

    def add_point_connection(self, nodes, weights, target, stiffness, damping=0.0):
        """World::AddPointConnection (kept until the end of the next step)."""
        n = np.ascontiguousarray(nodes, np.int32)
        w = np.ascontiguousarray(weights, np.float64)
        t = np.ascontiguousarray(target, np.float64)
        self.lib.ref_add_point_connection(self.h, _ptr(n), _ptr(w), _ptr(t), float(stiffness), float(damping))

    def point_connection_count(self) -> int:
        return int(self.lib.ref_point_connection_count(self.h))

    def set_state(self, x, v):
        x = np.ascontiguousarray(x, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        self.lib.ref_set_state(self.h, _ptr(x), _ptr(v))

    def state(self):
        x = np.zeros((self.node_count, 3))
        v = np.zeros((self.node_count, 3))
        self.lib.ref_get_state(self.h, _ptr(x), _ptr(v))
        return x, v

    def step(self, dt: Optional[float] = None) -> int:
        return self.lib.ref_step(self.h, self.dt if dt is None else dt)

    def cg_stats(self):
        it, conv = _i(), _i()
        res = _d()
        self.lib.ref_cg_stats(self.h, C.byref(it), C.byref(res), C.byref(conv))
        return dict(iterations=it.value, residual=res.value, converged=conv.value)

    def system(self, dt: Optional[float] = None) -> System:
        dyn, nnz = _i(), _i()
        solved = self.lib.ref_dump_begin(self.h, self.dt if dt is None else dt, C.byref(dyn), C.byref(nnz))
        n, m = dyn.value, nnz.value
        rs = np.zeros(n + 1, np.int32)
        col = np.zeros(max(m, 1), np.int32)
        val = np.zeros((max(m, 1), 3, 3))
        rhs = np.zeros((max(n, 1), 3))
        minv = np.zeros((max(n, 1), 3, 3))
        dv = np.zeros((max(n, 1), 3))
        n2d = np.zeros(self.node_count, np.int32)
        mass = np.zeros(self.node_count)
        force = np.zeros((self.node_count, 3))
        self.lib.ref_dump_copy(self.h, _ptr(rs), _ptr(col), _ptr(val), _ptr(rhs), _ptr(minv), _ptr(dv), _ptr(n2d),
                               _ptr(mass), _ptr(force))
        it, conv = _i(), _i()
        res = _d()
        self.lib.ref_dump_cg(self.h, C.byref(it), C.byref(res), C.byref(conv))
        return System(rs, col[:m], val[:m], rhs[:n], minv[:n], dv[:n], n2d, mass, force, it.value, res.value,
                      conv.value, solved)


def _ref_lib(precision="f32"):
    return C.CDLL(reference_library_path(precision))


def reference_bsr_multiply(row_start, col, values, x, precision="f32"):
    L = _ref_lib(precision)
    L.ref_bsr_multiply.argtypes = [_i, _p, _p, _p, _p, _p]
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, np.float64)
    xx = np.ascontiguousarray(x, np.float64)
    y = np.zeros((n, 3))
    L.ref_bsr_multiply(n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(xx), _ptr(y))
    return y


def reference_pcg(row_start, col, values, b, minv, max_iterations, tolerance, precision="f32"):
    L = _ref_lib(precision)
    L.ref_pcg.argtypes = [_i, _p, _p, _p, _p, _p, _i, _d, _p, _p, _p, _p]
    L.ref_pcg.restype = _i
    n = len(row_start) - 1
    rs = np.ascontiguousarray(row_start, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    vv = np.ascontiguousarray(values, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    mm = np.ascontiguousarray(minv, np.float64)
    x = np.zeros((max(n, 1), 3))
    it, conv = _i(), _i()
    res = _d()
    have = L.ref_pcg(n, _ptr(rs), _ptr(cl), _ptr(vv), _ptr(bb), _ptr(mm), max_iterations, tolerance, _ptr(x),
                     C.byref(it), C.byref(res), C.byref(conv))
    return (x[:n] if have else None), dict(iterations=it.value, residual=res.value, converged=conv.value)


def reference_build_pattern(n, rows, cols, precision="f32"):
    L = _ref_lib(precision)
    L.ref_bsr_pattern.argtypes = [_i, _p, _p, _i, _p, _p, _i]
    L.ref_bsr_pattern.restype = _i
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    rs = np.zeros(n + 1, np.int32)
    nnz = L.ref_bsr_pattern(n, _ptr(rows), _ptr(cols), len(rows), _ptr(rs), None, 0)
    col = np.zeros(max(nnz, 1), np.int32)
    L.ref_bsr_pattern(n, _ptr(rows), _ptr(cols), len(rows), _ptr(rs), _ptr(col), nnz)
    return rs, col[:nnz]

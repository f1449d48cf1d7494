"""Python view of the drop-in C ABI (``include/physik_b200.h``), for tests and the bench.

``SimWorld`` builds a world from a ``physik_b200.meshes.Scene`` exactly as a reference
user would through the ``PHYSIK_*`` calls (``PHYSIK_GenerateTetMesh``,
``PHYSIK_CreateTetMeshPhysicsComponent``, ``PHYSIK_SetNodeFixed``, ...), then steps it
with ``PHYSIK_Step``.  Every call goes through the C ABI; nothing here computes physics.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib as L

PRECISIONS = {"fp32": 0, "mixed": 1, "fp64": 2}


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class PhysikError(RuntimeError):
    pass


class SimWorld:
    def __init__(self, scene, precision: str = "fp32", device: int = 0, implicit: bool = True):
        self.X = L.PX
        self.h = self.X.PHYSIK_CreateWorld()
        if not self.h:
            raise PhysikError("PHYSIK_CreateWorld failed")
        X, h = self.X, self.h
        X.PHYSIK_B200_SetPrecision(h, PRECISIONS[precision])
        X.PHYSIK_B200_SetDevice(h, device)
        X.PHYSIK_SetSolverMode(h, 1 if implicit else 0)
        X.PHYSIK_SetGravity(h, *[float(g) for g in scene.gravity])
        X.PHYSIK_SetConjugateGradientMaxIterations(h, scene.max_iterations)
        X.PHYSIK_SetConjugateGradientTolerance(h, scene.tolerance)
        self.dt = scene.dt
        self.components = []
        fixed_all, x0, v0 = [], [], []
        for b in scene.bodies:
            pos = np.ascontiguousarray(b.positions, np.float32)
            tets = np.ascontiguousarray(b.tets, np.int32)
            mesh = X.PHYSIK_GenerateTetMesh(_ptr(pos), pos.shape[0], _ptr(tets), tets.shape[0])
            mat = L.MaterialDesc(b.density, b.young, b.poisson, b.damping)
            comp = X.PHYSIK_CreateTetMeshPhysicsComponent(h, mesh, C.byref(mat))
            X.PHYSIK_DestroyGeneratedTetMesh(mesh)
            if not comp.valid():
                raise PhysikError("PHYSIK_CreateTetMeshPhysicsComponent failed: " + self.error())
            if b.tet_young is not None:
                ty = np.ascontiguousarray(b.tet_young, np.float32)
                if not X.PHYSIK_B200_SetTetMeshYoungModulus(h, comp, _ptr(ty), ty.shape[0]):
                    raise PhysikError("per-tet Young's modulus rejected")
            self.components.append(comp)
            fixed_all.append(b.pinned)
            x0.append(b.initial_positions if b.initial_positions is not None else b.positions)
            v0.append(b.initial_velocities if b.initial_velocities is not None else np.zeros_like(b.positions))
        self.node_count = X.PHYSIK_B200_GetNodeCount(h)
        fixed = np.concatenate(fixed_all)
        for i in np.nonzero(fixed)[0]:
            X.PHYSIK_SetNodeFixed(h, int(i), 1)
        x0 = np.ascontiguousarray(np.concatenate(x0), np.float32)
        v0 = np.ascontiguousarray(np.concatenate(v0), np.float32)
        v0[fixed] = 0.0
        self.set_state(x0, v0)

    def __del__(self):
        if getattr(self, "h", None):
            self.X.PHYSIK_DestroyWorld(self.h)
            self.h = None

    @staticmethod
    def error() -> str:
        return (L.PX.PHYSIK_B200_GetLastError() or b"").decode()

    def step(self, dt: Optional[float] = None):
        self.X.PHYSIK_Step(self.h, self.dt if dt is None else dt)

    def state(self, f64: bool = False):
        x = np.zeros((self.node_count, 3), np.float64 if f64 else np.float32)
        v = np.zeros_like(x)
        fn = self.X.PHYSIK_B200_GetNodeStatesF64 if f64 else self.X.PHYSIK_B200_GetNodeStates
        if fn(self.h, _ptr(x), _ptr(v), self.node_count) < 0:
            raise PhysikError("GetNodeStates failed: " + self.error())
        return x, v

    def set_state(self, x, v, f64: bool = False):
        dt_ = np.float64 if f64 else np.float32
        x = np.ascontiguousarray(x, dt_)
        v = np.ascontiguousarray(v, dt_)
        fn = self.X.PHYSIK_B200_SetNodeStatesF64 if f64 else self.X.PHYSIK_B200_SetNodeStates
        if fn(self.h, _ptr(x), _ptr(v), self.node_count) < 0:
            raise PhysikError("SetNodeStates failed: " + self.error())

    def local_positions(self, body: int):
        """PHYSIK_GetTetMeshLocalCurrentPosition for every node of a mesh: the mesh's own
        copy of its positions (float32, (count, 3))."""
        comp = self.components[body]
        count = self.X.PHYSIK_GetTetMeshNodeCount(self.h, comp)
        out = np.zeros((max(count, 0), 3), np.float32)
        fx, fy, fz = C.c_float(), C.c_float(), C.c_float()
        for i in range(count):
            if not self.X.PHYSIK_GetTetMeshLocalCurrentPosition(self.h, comp, i, C.byref(fx), C.byref(fy),
                                                                C.byref(fz)):
                raise PhysikError("GetTetMeshLocalCurrentPosition failed: " + self.error())
            out[i] = (fx.value, fy.value, fz.value)
        return out

    def set_local_position(self, body: int, node: int, p) -> int:
        return int(self.X.PHYSIK_SetTetMeshLocalCurrentPosition(self.h, self.components[body], int(node),
                                                                *[float(c) for c in p]))

    def add_sphere(self, center, radius, stiffness=None, damping=None):
        """PHYSIK_CreateCollisionSphereComponent (+ its connection settings when given)."""
        h = self.X.PHYSIK_CreateCollisionSphereComponent(self.h, *[float(c) for c in center], float(radius))
        if not h.valid():
            raise PhysikError("PHYSIK_CreateCollisionSphereComponent failed: " + self.error())
        if stiffness is not None:
            self.X.PHYSIK_SetCollisionSphereConnectionSettings(self.h, h, float(stiffness), float(damping))
        return h

    def add_point_connection(self, nodes, weights, target, stiffness: float, damping: float = 0.0):
        """PHYSIK_AddPointConnection: a spring from sum_i weights[i] x(nodes[i]) to `target`,
        kept until the end of the next step."""
        n = [int(i) for i in nodes]
        w = [float(x) for x in weights]
        t = [float(x) for x in target]
        self.X.PHYSIK_AddPointConnection(self.h, *n, *w, *t, float(stiffness), float(damping))

    def point_connection_count(self) -> int:
        return int(self.X.PHYSIK_GetPointConnectionCount(self.h))

    def set_batched(self, on: bool = True):
        self.X.PHYSIK_B200_SetBatchedSolve(self.h, 1 if on else 0)

    def tet_count(self) -> int:
        return int(self.X.PHYSIK_B200_GetTetCount(self.h))

    def set_tet_young(self, body: int, young):
        ty = np.ascontiguousarray(young, np.float32)
        if not self.X.PHYSIK_B200_SetTetMeshYoungModulus(self.h, self.components[body], _ptr(ty), ty.shape[0]):
            raise PhysikError("per-tet Young's modulus rejected: " + self.error())

    def adjoint_step(self, xbar_next, vbar_next, theta_bar, dt: Optional[float] = None):
        """Sensitivities to the current state, given those to the state after one step;
        adds the log-Young's-modulus sensitivities to theta_bar (float64, one per tet)."""
        xbar_next = np.ascontiguousarray(xbar_next, np.float64)
        vbar_next = np.ascontiguousarray(vbar_next, np.float64)
        xbar = np.zeros_like(xbar_next)
        vbar = np.zeros_like(vbar_next)
        if self.X.PHYSIK_B200_AdjointStep(self.h, self.dt if dt is None else dt, _ptr(xbar_next), _ptr(vbar_next),
                                          _ptr(xbar), _ptr(vbar), _ptr(theta_bar)) != 0:
            raise PhysikError("adjoint step failed: " + self.error())
        return xbar, vbar

    def set_graph(self, on: bool = True):
        self.X.PHYSIK_B200_SetGraphCapture(self.h, 1 if on else 0)

    def autotune(self, repeats: int = 3):
        ms = C.c_double()
        chosen = self.X.PHYSIK_B200_Autotune(self.h, repeats, C.byref(ms))
        if chosen < 0:
            raise PhysikError("autotune failed: " + self.error())
        return chosen, ms.value

    def set_refinement(self, passes: int):
        """FP64 outer true-residual refinement passes (FP32 / mixed precision); 0: off."""
        if self.X.PHYSIK_B200_SetRefinement(self.h, passes) != 0:
            raise PhysikError("bad refinement pass count")

    PCG_KERNELS = {0: "ring", 1: "staged", 2: "plain", 3: "slab", 4: "batched", 5: "slab-batched"}

    def pcg_kernel(self):
        """(name, blocks) of the PCG kernel the last step's solve ran on."""
        blocks = C.c_int()
        k = self.X.PHYSIK_B200_GetPcgKernel(self.h, C.byref(blocks))
        return self.PCG_KERNELS.get(k, "none"), blocks.value

    def pcg_stream_form(self) -> str:
        """Stream form of the part-resident kernel in the last solve: "full", "sym" or "none"."""
        return {0: "full", 1: "sym"}.get(self.X.PHYSIK_B200_GetPcgStreamForm(self.h), "none")

    def body_stats(self, i: int):
        it, conv, res, fl = C.c_int(), C.c_int(), C.c_float(), C.c_uint()
        if self.X.PHYSIK_B200_GetBodyConjugateGradientStats(self.h, self.components[i], C.byref(it), C.byref(conv),
                                                           C.byref(res), C.byref(fl)) != 0:
            raise PhysikError("no batched statistics: " + self.error())
        return dict(iterations=it.value, converged=conv.value, residual=res.value, flags=fl.value)

    def cg_stats(self):
        X, h = self.X, self.h
        return dict(iterations=X.PHYSIK_GetLastConjugateGradientIterations(h),
                    residual=X.PHYSIK_GetLastConjugateGradientResidualNorm(h),
                    converged=X.PHYSIK_DidLastConjugateGradientSolveConverge(h),
                    flags=X.PHYSIK_B200_GetLastStepFlags(h))

    def prepare(self, upload: bool = False) -> int:
        n = self.X.PHYSIK_B200_PrepareScene(self.h, 1 if upload else 0)
        if n < 0:
            raise PhysikError("PrepareScene failed: " + self.error())
        return n

    def pattern(self):
        dyn, nnz = C.c_int(), C.c_int()
        if self.X.PHYSIK_B200_GetSolverSizes(self.h, C.byref(dyn), C.byref(nnz)) < 0:
            raise PhysikError("no prepared scene")
        rs = np.zeros(dyn.value + 1, np.int32)
        col = np.zeros(max(nnz.value, 1), np.int32)
        n2d = np.zeros(self.node_count, np.int32)
        self.X.PHYSIK_B200_GetSolverPattern(self.h, _ptr(rs), _ptr(col), _ptr(n2d))
        mass = np.zeros(self.node_count, np.float64)
        self.X.PHYSIK_B200_GetSolverMasses(self.h, _ptr(mass))
        return rs, col[:nnz.value], n2d, mass

    def system(self):
        """The last substep's assembled system (values column-major per block)."""
        rs, col, n2d, _ = self.pattern()
        n, nnz = len(rs) - 1, len(col)
        vals = np.zeros((max(nnz, 1), 3, 3))
        rhs = np.zeros((max(n, 1), 3))
        minv = np.zeros((max(n, 1), 3, 3))
        dv = np.zeros((max(n, 1), 3))
        if self.X.PHYSIK_B200_GetSolverSystem(self.h, _ptr(vals), _ptr(rhs), _ptr(minv), _ptr(dv)) != 0:
            raise PhysikError("GetSolverSystem failed: " + self.error())
        return dict(row_start=rs, col=col, values=vals[:nnz], rhs=rhs[:n], minv=minv[:n], dv=dv[:n], node_to_dyn=n2d)

    def enable_timing(self, on=True):
        return self.X.PHYSIK_B200_EnableTiming(self.h, 1 if on else 0)

    def timings(self):
        a, s, k = C.c_double(), C.c_double(), C.c_int()
        launches = C.c_longlong()
        self.X.PHYSIK_B200_GetTimings(self.h, C.byref(a), C.byref(s), C.byref(k), C.byref(launches))
        return dict(assemble_ms=a.value, solve_ms=s.value, steps=k.value, launches=launches.value)

    def synchronize(self):
        return self.X.PHYSIK_B200_Synchronize(self.h)

    def stream(self) -> int:
        return self.X.PHYSIK_B200_GetStream(self.h) or 0

    def set_pcg_grid(self, grid: int) -> int:
        return self.X.PHYSIK_B200_SetPcgGrid(self.h, grid)

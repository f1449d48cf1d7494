"""Loader for the in-tree shared libraries (built by ``physik_b200/csrc/Makefile``).

The CUDA path has no CPU fallback: if ``lib/libphysik_b200.so`` or ``lib/libpkcuda.so``
is missing, importing this module raises ``ImportError`` naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "lib")
PKCUDA_PATH = os.path.join(LIB_DIR, "libpkcuda.so")
PHYSIK_PATH = os.path.join(LIB_DIR, "libphysik_b200.so")
HEADERS = [os.path.join(ROOT, "include", "pkcuda.h"), os.path.join(ROOT, "include", "physik_b200.h")]

for _p in (PKCUDA_PATH, PHYSIK_PATH):
    if not os.path.exists(_p):
        raise ImportError(f"{_p} is missing: build it with `make -C physik_b200/csrc` "
                          "(or `python -c 'import __graft_entry__ as g; g.build()'`)")

pkcuda = C.CDLL(PKCUDA_PATH, mode=C.RTLD_GLOBAL)
physik = C.CDLL(PHYSIK_PATH)


def declared_symbols(header: str):
    """Names of the functions a public header declares (PHYSIK_*, pk_*)."""
    text = open(header).read()
    return sorted(set(re.findall(r"\b((?:PHYSIK_\w+|pk_\w+))\s*\(", text)) - {"PHYSIK_B200_API", "PKCUDA_API"})


class PkStepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double * 3), ("max_iterations", C.c_int),
                ("tolerance", C.c_double), ("use_jacobi", C.c_int), ("linear", C.c_int),
                ("explicit_mode", C.c_int), ("integrate", C.c_int)]


class PkStepStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("residual_norm", C.c_double),
                ("flags", C.c_uint), ("polar_fp64_count", C.c_int), ("polar_identity_count", C.c_int)]


class PkCgResult(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("residual_norm", C.c_double),
                ("have_solution", C.c_int)]


class ComponentHandle(C.Structure):
    _fields_ = [("index", C.c_uint32), ("generation", C.c_uint32)]

    def valid(self) -> bool:
        return self.index != 0xFFFFFFFF and self.generation != 0


class MaterialDesc(C.Structure):
    _fields_ = [("density", C.c_float), ("youngModulus", C.c_float), ("poissonRatio", C.c_float),
                ("damping", C.c_float)]


_v, _i, _f, _d, _p, _u = None, C.c_int, C.c_float, C.c_double, C.c_void_p, C.c_uint
_H = ComponentHandle
_SIGS = {
    # pkcuda.h
    "pk_last_error": (C.c_char_p, []),
    "pk_device_count": (_i, []),
    "pk_system_create": (_i, [_i, _i, C.POINTER(_p)]),
    "pk_system_destroy": (_i, [_p]),
    "pk_system_stream": (_p, [_p]),
    "pk_system_set_nodes": (_i, [_p, _i, _p, _p]),
    "pk_system_set_state_f32": (_i, [_p, _p, _p]),
    "pk_system_set_state_f64": (_i, [_p, _p, _p]),
    "pk_system_get_state_f32": (_i, [_p, _p, _p]),
    "pk_system_get_state_f64": (_i, [_p, _p, _p]),
    "pk_system_set_tets": (_i, [_p, _i, _p, _p, _p, _p, _p, _p, _p]),
    "pk_system_set_pattern": (_i, [_p, _i, _p, _p, _p, _p, _p]),
    "pk_system_step": (_i, [_p, C.POINTER(PkStepParams)]),
    "pk_system_stats": (_i, [_p, C.POINTER(PkStepStats)]),
    "pk_system_get_system_f64": (_i, [_p, _p, _p, _p, _p]),
    "pk_system_solve_given_f64": (_i, [_p, _p, _p, _p, C.POINTER(PkStepParams)]),
    "pk_system_enable_timing": (_i, [_p, _i]),
    "pk_system_timings": (_i, [_p, _p, _p, _p, _p]),
    "pk_system_set_pcg_grid": (_i, [_p, _i]),
    "pk_bsr_multiply": (_i, [_i, _i, _i, _p, _p, _p, _p, _p]),
    "pk_pcg": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _i, _i, _d, _p, C.POINTER(PkCgResult)]),
    "pk_bsr_transpose_index": (_i, [_i, _p, _p, _p, _p, _p]),
    "pk_pcg_noalloc": (_i, [_i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _i, _d, _p, C.POINTER(PkCgResult), _p]),
    "pk_pcg_noalloc_last_error": (C.c_char_p, []),
    "pk_system_set_segments": (_i, [_p, _i, _p]),
    "pk_system_set_batched": (_i, [_p, _i]),
    "pk_system_segment_stats": (_i, [_p, _i, _p, _p, _p, _p]),
    "pk_ring_tiling_selfcheck": (_i, [_i, _i, _p, _p, _p, _p, _p, _p, _p]),
    "pk_slab_plan_selfcheck": (_i, [_i, _p, _p, _p, _p, _p, _i, _i, _p, _p]),
    "pk_slab_plan_batched_selfcheck": (_i, [_i, _p, _p, _p, _p, _p, _p, _i, _i, _i, _p, _p]),
    "pk_system_set_graph": (_i, [_p, _i]),
    "pk_system_adjoint_step": (_i, [_p, C.POINTER(PkStepParams), _p, _p, _p, _p, _p]),
    "pk_system_autotune": (_i, [_p, C.POINTER(PkStepParams), _i, _p, _p]),
    "pk_system_pcg_kernel": (_i, [_p, _p]),
    "pk_system_set_refinement": (_i, [_p, _i]),
    "pk_system_set_connections": (_i, [_p, _i, _p, _p, _p, _p]),
    "pk_system_set_masses": (_i, [_p, _p]),
    # physik_b200.h
    "PHYSIK_CreateWorld": (_p, []),
    "PHYSIK_DestroyWorld": (_v, [_p]),
    "PHYSIK_Step": (_v, [_p, _f]),
    "PHYSIK_SetSubstepCount": (_v, [_p, _i]),
    "PHYSIK_SetSolverMode": (_v, [_p, _i]),
    "PHYSIK_SetConjugateGradientTolerance": (_v, [_p, _f]),
    "PHYSIK_GetConjugateGradientTolerance": (_f, [_p]),
    "PHYSIK_SetConjugateGradientMaxIterations": (_v, [_p, _i]),
    "PHYSIK_GetConjugateGradientMaxIterations": (_i, [_p]),
    "PHYSIK_GetLastConjugateGradientIterations": (_i, [_p]),
    "PHYSIK_GetLastConjugateGradientResidualNorm": (_f, [_p]),
    "PHYSIK_DidLastConjugateGradientSolveConverge": (_i, [_p]),
    "PHYSIK_SetGravity": (_v, [_p, _f, _f, _f]),
    "PHYSIK_AddNode": (_i, [_p, _f, _f, _f]),
    "PHYSIK_SetNodeFixed": (_v, [_p, _i, _i]),
    "PHYSIK_IsNodeFixed": (_i, [_p, _i]),
    "pk_exchange_wait_selftest": (_i, [_i, _i, _i, C.c_ulonglong, _p]),
    "PHYSIK_GenerateTetMesh": (_p, [_p, _i, _p, _i]),
    "PHYSIK_IsGeneratedTetMeshHandleValid": (_i, [_p]),
    "PHYSIK_DestroyGeneratedTetMesh": (_v, [_p]),
    "PHYSIK_GetGeneratedTetMeshVertexCount": (_i, [_p]),
    "PHYSIK_GetGeneratedTetMeshTetCount": (_i, [_p]),
    "PHYSIK_GetGeneratedTetMeshTetIndexCount": (_i, [_p]),
    "PHYSIK_GetGeneratedTetMeshVertex": (_i, [_p, _i, _p, _p, _p]),
    "PHYSIK_GetGeneratedTetMeshTetNodeIndex": (_i, [_p, _i, _p]),
    "PHYSIK_CreateTetMeshComponent": (_H, [_p, _p]),
    "PHYSIK_CreateTetMeshPhysicsComponent": (_H, [_p, _p, C.POINTER(MaterialDesc)]),
    "PHYSIK_GetTetMeshGlobalNodeBeginIndex": (_i, [_p, _H]),
    "PHYSIK_GetTetMeshGlobalNodeCount": (_i, [_p, _H]),
    "PHYSIK_GetTetMeshGlobalNodeIndex": (_i, [_p, _H, _i]),
    "PHYSIK_CreateCollisionSphereComponent": (_H, [_p, _f, _f, _f, _f]),
    "PHYSIK_SetCollisionSphereConnectionSettings": (_v, [_p, _H, _f, _f]),
    "PHYSIK_GetCollisionSphereConnectionSettings": (_v, [_p, _H, _p, _p]),
    "PHYSIK_SetCollisionComponentKinematicTarget": (_v, [_p, _H, _f, _f, _f]),
    "PHYSIK_B200_CreateContributionComponent": (_H, [_p, _i]),
    "PHYSIK_B200_SetContributionCallback": (_v, [_p, _H, _p, _p]),
    "PHYSIK_B200_SolverDataAddNodeForce": (_v, [_p, _i, _f, _f, _f]),
    "PHYSIK_B200_SolverDataAddNodeMass": (_v, [_p, _i, _f]),
    "PHYSIK_B200_SolverDataAddStiffnessBlock": (_v, [_p, _i, _i, _p]),
    "PHYSIK_CreateScriptComponent": (_H, [_p]),
    "PHYSIK_SetScriptComponentCallback": (_v, [_p, _H, _p, _p]),
    "PHYSIK_ClearScriptComponentCallback": (_v, [_p, _H]),
    "PHYSIK_SetTetMeshLocalCurrentPosition": (_i, [_p, _H, _i, _f, _f, _f]),
    "PHYSIK_GetTetMeshLocalCurrentPosition": (_i, [_p, _H, _i, _p, _p, _p]),
    "PHYSIK_SetTetMeshMaterial": (_v, [_p, _H, C.POINTER(MaterialDesc)]),
    "PHYSIK_DestroyComponent": (_v, [_p, _H]),
    "PHYSIK_IsComponentHandleValid": (_i, [_p, _H]),
    "PHYSIK_GetTetMeshTetCount": (_i, [_p, _H]),
    "PHYSIK_GetTetMeshNodeCount": (_i, [_p, _H]),
    "PHYSIK_IsTetActive": (_i, [_p, _H, _i]),
    "PHYSIK_SetTetActive": (_v, [_p, _H, _i, _i]),
    "PHYSIK_DeactivateTet": (_v, [_p, _H, _i]),
    "PHYSIK_GetActiveTetCount": (_i, [_p, _H]),
    "PHYSIK_GetNodePosition": (_v, [_p, _i, _p, _p, _p]),
    "PHYSIK_GetNodeVelocity": (_v, [_p, _i, _p, _p, _p]),
    "PHYSIK_SetNodePosition": (_v, [_p, _i, _f, _f, _f]),
    "PHYSIK_SetNodeVelocity": (_v, [_p, _i, _f, _f, _f]),
    "PHYSIK_GetPointConnectionCount": (_i, [_p]),
    "PHYSIK_AddPointConnection": (_v, [_p, _i, _i, _i, _i] + [_f] * 9),
    "PHYSIK_B200_SetPrecision": (_v, [_p, _i]),
    "PHYSIK_B200_GetPrecision": (_i, [_p]),
    "PHYSIK_B200_SetDevice": (_v, [_p, _i]),
    "PHYSIK_B200_GetNodeCount": (_i, [_p]),
    "PHYSIK_B200_GetNodeStates": (_i, [_p, _p, _p, _i]),
    "PHYSIK_B200_SetNodeStates": (_i, [_p, _p, _p, _i]),
    "PHYSIK_B200_GetNodeStatesF64": (_i, [_p, _p, _p, _i]),
    "PHYSIK_B200_SetNodeStatesF64": (_i, [_p, _p, _p, _i]),
    "PHYSIK_B200_SetTetMeshYoungModulus": (_i, [_p, _H, _p, _i]),
    "PHYSIK_B200_SetTetMeshFemModel": (_i, [_p, _H, _i]),
    "PHYSIK_B200_GetLastStepFlags": (_u, [_p]),
    "PHYSIK_B200_GetLastError": (C.c_char_p, []),
    "PHYSIK_B200_PrepareScene": (_i, [_p, _i]),
    "PHYSIK_B200_GetSolverSizes": (_i, [_p, _p, _p]),
    "PHYSIK_B200_GetSolverPattern": (_i, [_p, _p, _p, _p]),
    "PHYSIK_B200_GetSolverMasses": (_i, [_p, _p]),
    "PHYSIK_B200_GetSolverSystem": (_i, [_p, _p, _p, _p, _p]),
    "PHYSIK_B200_EnableTiming": (_i, [_p, _i]),
    "PHYSIK_B200_GetTimings": (_i, [_p, _p, _p, _p, _p]),
    "PHYSIK_B200_SetPcgGrid": (_i, [_p, _i]),
    "PHYSIK_B200_SetBatchedSolve": (_v, [_p, _i]),
    "PHYSIK_B200_SetGraphCapture": (_v, [_p, _i]),
    "PHYSIK_B200_AdjointStep": (_i, [_p, _f, _p, _p, _p, _p, _p]),
    "PHYSIK_B200_GetTetCount": (_i, [_p]),
    "PHYSIK_B200_Autotune": (_i, [_p, _i, _p]),
    "PHYSIK_B200_GetPcgKernel": (_i, [_p, _p]),
    "PHYSIK_B200_GetPcgStreamForm": (_i, [_p]),
    "PHYSIK_B200_GetDeviceSystem": (_p, [_p]),
    "pk_system_sphere_contacts": (_i, [_p, _p, C.c_double, _i, _p, _p]),
    "PHYSIK_B200_SetRefinement": (_i, [_p, _i]),
    "PHYSIK_B200_GetBodyConjugateGradientStats": (_i, [_p, _H, _p, _p, _p, _p]),
    "PHYSIK_B200_GetStream": (_p, [_p]),
    "PHYSIK_CreateSurfaceExtractionComponent": (_H, [_p, _H]),
    "PHYSIK_GetSurfaceTriangleIndexCount": (_i, [_p, _H]),
    "PHYSIK_CopySurfaceTriangleIndices": (_i, [_p, _H, _p, _i]),
    "PHYSIK_CreateSurfaceVisualComponent": (_H, [_p, _H]),
    "PHYSIK_GetSurfaceVisualVertexCount": (_i, [_p, _H]),
    "PHYSIK_GetSurfaceVisualTriangleIndexCount": (_i, [_p, _H]),
    "PHYSIK_GetSurfaceVisualNormalCount": (_i, [_p, _H]),
    "PHYSIK_GetSurfaceVisualVertex": (_i, [_p, _H, _i, _p, _p, _p]),
    "PHYSIK_GetSurfaceVisualTriangleIndex": (_i, [_p, _H, _i, _p]),
    "PHYSIK_GetSurfaceVisualNormal": (_i, [_p, _H, _i, _p, _p, _p]),
    "PHYSIK_CreateVisualMeshComponent": (_H, [_p, _H]),
    "PHYSIK_SetVisualMeshData": (_v, [_p, _H, _p, _i, _p, _i]),
    "PHYSIK_BuildVisualMeshEmbedding": (_i, [_p, _H]),
    "PHYSIK_GetVisualMeshVertexCount": (_i, [_p, _H]),
    "PHYSIK_GetVisualMeshTriangleIndexCount": (_i, [_p, _H]),
    "PHYSIK_CopyVisualMeshVertices": (_i, [_p, _H, _p, _i]),
    "PHYSIK_CopyVisualMeshTriangleIndices": (_i, [_p, _H, _p, _i]),
    "PHYSIK_B200_GetVisualUpdateOnDevice": (_i, [_p, _H]),
    "PHYSIK_B200_Synchronize": (_i, [_p]),
}

for _name, (_res, _args) in _SIGS.items():
    _lib = pkcuda if _name.startswith("pk_") else physik
    _fn = getattr(_lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

PK = pkcuda
PX = physik

# include/pkcuda.h constants
PK_PREC_FP32, PK_PREC_MIXED, PK_PREC_FP64 = 0, 1, 2
PK_ERR_UNSUPPORTED = -5
FLAG_PRECOMPUTE_FAILED = 0x1
FLAG_SINGULAR_DIAG = 0x2
FLAG_INVALID_RHS = 0x4
FLAG_BREAKDOWN = 0x8
FLAG_NONFINITE_DV = 0x10
FLAG_INTEGRATE_ABORT = 0x20
FLAG_POLAR_IDENTITY = 0x40
FLAG_POLAR_FP64 = 0x80
FLAG_BARRIER_TIMEOUT = 0x100
FLAG_SOLVED = 0x1000
FLAG_INTEGRATED = 0x2000
FLAG_CONVERGED = 0x4000
FLAG_REFINED_FP64 = 0x8000


def last_error() -> str:
    return (PK.pk_last_error() or b"").decode()


def device_count() -> int:
    return PK.pk_device_count()

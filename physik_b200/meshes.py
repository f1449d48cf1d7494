"""Synthetic soft-body scenes: Kuhn-split hex grids and the five benchmark workloads.

Every workload is a box of ``nx x ny x nz`` hexahedral cells.  Vertex ``(i, j, k)``
gets id ``i + (nx+1) * (j + (ny+1) * k)``; cells are visited with ``i`` fastest,
then ``j``, then ``k``, and each cell is split into six tetrahedra around its main
diagonal (corner 0 to corner 6), in the order

    {0,1,2,6} {0,2,3,6} {0,3,7,6} {0,7,4,6} {0,4,5,6} {0,5,1,6}

with corners c0..c7 = (i,j,k) (i+1,j,k) (i+1,j+1,k) (i,j+1,k) and the same at k+1.

Conventions fixed here (the reference's own tests pin none of them):

* Jitter: every vertex, boundary included, moves by U(-a*h, +a*h) per axis, drawn
  from ``numpy.random.default_rng(seed)`` as one ``(V, 3)`` array in vertex-id order.
* Positions are rounded to float32 once; the same float32 values feed the GPU path,
  the FP32 reference and the FP64 oracle, so precision is the only difference.
* Faces are pinned by grid index (``i == 0`` for "x=0", ``k == 0`` for "bottom"),
  never by coordinate, because jitter moves coordinates.
* Unstated parameters: damping 0, gravity (0, 0, -9.81), CG tolerance 1e-6,
  at most 100 CG iterations, one substep.

Node ordering matches ``TetMeshGenerator::Generate`` (TetMeshGenerator.cpp:153-282):
at these spacings nothing welds and no tet is degenerate, so the generator keeps
ids and tet order unchanged.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

KUHN_TETS = np.array(
    [[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]],
    dtype=np.int64,
)
CORNER_OFFSETS = np.array(
    [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
    dtype=np.int64,
)


@dataclasses.dataclass
class Body:
    """One tet-mesh soft body (one TetMeshPhysicsComponent)."""

    positions: np.ndarray  # (V, 3) float32 rest = initial positions
    tets: np.ndarray  # (T, 4) int32 local node ids
    pinned: np.ndarray  # (V,) bool, nodes to fix
    density: float
    young: float
    poisson: float
    damping: float = 0.0
    tet_young: Optional[np.ndarray] = None  # (T,) per-element E overriding `young`
    initial_positions: Optional[np.ndarray] = None  # (V, 3) float32, defaults to rest
    initial_velocities: Optional[np.ndarray] = None  # (V, 3) float32, defaults to 0
    cells: tuple = (0, 0, 0)


@dataclasses.dataclass
class Scene:
    """A world of bodies plus the step settings of a workload."""

    name: str
    bodies: List[Body]
    dt: float
    steps: int
    gravity: tuple = (0.0, 0.0, -9.81)
    tolerance: float = 1e-6
    max_iterations: int = 100

    @property
    def vertex_count(self) -> int:
        return int(sum(b.positions.shape[0] for b in self.bodies))

    @property
    def tet_count(self) -> int:
        return int(sum(b.tets.shape[0] for b in self.bodies))


def kuhn_grid(nx: int, ny: int, nz: int, size=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Return (positions float64 (V,3), tets int32 (T,4), grid index (V,3))."""
    i = np.arange(nx + 1)
    j = np.arange(ny + 1)
    k = np.arange(nz + 1)
    kk, jj, ii = np.meshgrid(k, j, i, indexing="ij")
    idx = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)  # vertex id order
    h = np.array([size[0] / nx, size[1] / ny, size[2] / nz])
    pos = np.asarray(origin, dtype=np.float64) + idx * h

    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cell = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)  # (C,3), i fastest
    corners = cell[:, None, :] + CORNER_OFFSETS[None, :, :]  # (C,8,3)
    corner_ids = corners[..., 0] + (nx + 1) * (corners[..., 1] + (ny + 1) * corners[..., 2])
    tets = corner_ids[:, KUHN_TETS].reshape(-1, 4)  # (C*6, 4)
    return pos, tets.astype(np.int32), idx, h


def jittered_box(nx, ny, nz, size, jitter, seed, pin_axis, pin_value=0):
    pos, tets, idx, h = kuhn_grid(nx, ny, nz, size)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        pos = pos + rng.uniform(-1.0, 1.0, size=pos.shape) * (jitter * h)
    pinned = idx[:, pin_axis] == pin_value
    return pos.astype(np.float32), tets, pinned


def config1() -> Scene:
    """8x8x8 unit cube, jitter 0.1h (seed 0), E=1e5, nu=0.3, x=0 pinned, dt=1/60, 200 steps."""
    pos, tets, pinned = jittered_box(8, 8, 8, (1.0, 1.0, 1.0), 0.1, 0, 0)
    body = Body(pos, tets, pinned, density=1000.0, young=1e5, poisson=0.3, cells=(8, 8, 8))
    return Scene("cube8_plain", [body], dt=1.0 / 60.0, steps=200)


def config2() -> Scene:
    """64x16x16 beam over 4x1x1 m, E=1e6, nu=0.45, x=0 pinned, dt=1/120, 500 steps."""
    pos, tets, pinned = jittered_box(64, 16, 16, (4.0, 1.0, 1.0), 0.0, 0, 0)
    body = Body(pos, tets, pinned, density=1000.0, young=1e6, poisson=0.45, cells=(64, 16, 16))
    return Scene("beam64x16x16_mixed", [body], dt=1.0 / 120.0, steps=500)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
        ]
    )


def config3(body_count: int = 256, seed: int = 1, h: float = 0.05) -> Scene:
    """Batched uneven bodies: cells per axis U{4..24}, E log-uniform [1e4,1e6],
    nu U[0.25,0.45], random rigid rotation of the initial pose about the centroid,
    rigid initial velocity N(0, 0.5^2), x=0 face pinned, dt=1/60, 300 steps.

    Draw order from ``default_rng(seed)``: all cell counts first ((body_count, 3)
    integers), then per body: log E, nu, rotation quaternion (4 normals), velocity (3)."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(4, 25, size=(body_count, 3))
    bodies = []
    for b in range(body_count):
        nx, ny, nz = (int(c) for c in cells[b])
        log_e = rng.uniform(math.log(1e4), math.log(1e6))
        nu = rng.uniform(0.25, 0.45)
        rot = random_rotation(rng)
        vel = rng.normal(0.0, 0.5, size=3)
        pos, tets, idx, _ = kuhn_grid(nx, ny, nz, (nx * h, ny * h, nz * h))
        rest = pos.astype(np.float32)
        centroid = pos.mean(axis=0)
        init = ((pos - centroid) @ rot.T + centroid).astype(np.float32)
        pinned = idx[:, 0] == 0
        v0 = np.tile(vel, (pos.shape[0], 1)).astype(np.float32)
        v0[pinned] = 0.0
        bodies.append(
            Body(rest, tets, pinned, density=1000.0, young=float(math.exp(log_e)), poisson=float(nu),
                 initial_positions=init, initial_velocities=v0, cells=(nx, ny, nz))
        )
    return Scene("batched256_uneven", bodies, dt=1.0 / 60.0, steps=300)


def config4() -> Scene:
    """128x64x64 over 2x1x1 m, jitter 0.05h (seed 2), E=5e5, nu=0.4, bottom pinned, dt=1/60, 50 steps."""
    pos, tets, pinned = jittered_box(128, 64, 64, (2.0, 1.0, 1.0), 0.05, 2, 2)
    body = Body(pos, tets, pinned, density=1000.0, young=5e5, poisson=0.4, cells=(128, 64, 64))
    return Scene("block128x64x64", [body], dt=1.0 / 60.0, steps=50)


def config5_theta(seed: int, tet_count: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.normal(math.log(1e5), 0.3, size=tet_count)


def config5(theta_seed: int = 3) -> Scene:
    """32x8x8 beam over 1x0.25x0.25 m, per-element log E ~ N(ln 1e5, 0.3^2), nu=0.3,
    x=0 pinned, dt=1/60, 60 steps."""
    pos, tets, pinned = jittered_box(32, 8, 8, (1.0, 0.25, 0.25), 0.0, 0, 0)
    theta = config5_theta(theta_seed, tets.shape[0])
    body = Body(pos, tets, pinned, density=1000.0, young=1e5, poisson=0.3,
                tet_young=np.exp(theta).astype(np.float32), cells=(32, 8, 8))
    return Scene("beam32x8x8_adjoint", [body], dt=1.0 / 60.0, steps=60)


def small_box(nx=2, ny=2, nz=2, young=1e4, poisson=0.3, jitter=0.1, seed=7, size=None) -> Scene:
    """A few-cell box for fast unit tests."""
    size = size or (nx * 0.1, ny * 0.1, nz * 0.1)
    pos, tets, pinned = jittered_box(nx, ny, nz, size, jitter, seed, 0)
    body = Body(pos, tets, pinned, density=1000.0, young=young, poisson=poisson, cells=(nx, ny, nz))
    return Scene(f"box{nx}x{ny}x{nz}", [body], dt=1.0 / 60.0, steps=10)


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}

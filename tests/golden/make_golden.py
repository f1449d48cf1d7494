"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root after ``make -C oracle ref`` (which compiles the
reference from its own sources into ``oracle/_ref``):

    python tests/golden/make_golden.py

Each fixture records inputs and the reference's outputs:

* ``kat_bsr.npz``   -- the known-answer SparseBlockMatrix / PCG cases that the
  reference's tests state (tests/PointConnectionTests.cpp:1983-2113, 2155-2390),
  re-derived here from their maths and run through the reference's own code.
* ``box_steps.npz`` -- a jittered 2x2x2 Kuhn box, three World::Step calls in FP32
  and in the float->double build, with the assembled system of the first step.
* ``cube8_steps.npz`` -- the 8x8x8 cube workload, two steps, FP32 and FP64.
* ``two_bodies.npz`` -- two boxes in one World (one coupled PCG), two steps.
* ``beam32_tet_young.npz`` -- the 32x8x8 beam with per-element Young's modulus, one step in FP64.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from physik_b200 import meshes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def diag_block(s):
    return (np.eye(3) * s).T  # column-major storage of s*I


def colmajor(m):
    """Column-major storage (values[c, r] = M[r][c]) of a row-major 3x3."""
    return np.asarray(m, dtype=np.float64).T.copy()


def kat_cases():
    out = {}
    # SparseBlockMatrixStoresAndMultipliesBlocks: blocks 2I, 3I, 4I on pattern {(0,0),(0,1),(1,1)}.
    rs, col = po.reference_build_pattern(2, [0, 0, 1], [0, 1, 1])
    vals = np.stack([diag_block(2.0), diag_block(3.0), diag_block(4.0)])
    x = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
    out.update(a_row_start=rs, a_col=col, a_values=vals, a_x=x, a_y=po.reference_bsr_multiply(rs, col, vals, x))
    # SparseBlockMatrixMultipliesCanonicalOffDiagonalBlocks: the off-diagonal block is added
    # at (1,0) as M^T, so the canonical (0,1) slot stores M.
    m = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]])
    rs, col = po.reference_build_pattern(2, [0, 1, 0, 1], [0, 0, 1, 1])
    vals = np.stack([diag_block(2.0), colmajor(m), diag_block(3.0)])
    out.update(b_row_start=rs, b_col=col, b_values=vals, b_x=x, b_y=po.reference_bsr_multiply(rs, col, vals, x))
    # Single-tet and two-adjacent-tet patterns.
    pairs = [(a, b) for a in range(4) for b in range(4)]
    rs, col = po.reference_build_pattern(4, [p[0] for p in pairs], [p[1] for p in pairs])
    out.update(tet1_row_start=rs, tet1_col=col)
    t2 = [[0, 1, 2, 3], [1, 2, 3, 4]]
    pr = [(t[a], t[b]) for t in t2 for a in range(4) for b in range(4)]
    rs, col = po.reference_build_pattern(5, [p[0] for p in pr], [p[1] for p in pr])
    out.update(tet2_row_start=rs, tet2_col=col)
    # ConjugateGradientSolvesDiagonalSparseSystem.
    rs, col = np.array([0, 1], np.int32), np.array([0], np.int32)
    vals = colmajor(np.diag([4.0, 9.0, 16.0]))[None]
    b = np.array([[4.0, 18.0, 48.0]])
    minv = colmajor(np.diag([0.25, 1.0 / 9.0, 1.0 / 16.0]))[None]
    xs, st = po.reference_pcg(rs, col, vals, b, minv, 16, 1e-6)
    out.update(c_row_start=rs, c_col=col, c_values=vals, c_b=b, c_minv=minv, c_x=xs, c_it=st["iterations"],
               c_conv=st["converged"])
    # ConjugateGradientSolvesCoupledSparseSystem: 4I, -I, 3I with x* = (1,2,3),(4,5,6).
    rs, col = po.reference_build_pattern(2, [0, 0, 1, 1], [0, 1, 0, 1])
    vals = np.stack([diag_block(4.0), diag_block(-1.0), diag_block(3.0)])
    b = po.reference_bsr_multiply(rs, col, vals, x)
    minv = np.stack([diag_block(0.25), diag_block(1.0 / 3.0)])
    xs, st = po.reference_pcg(rs, col, vals, b, minv, 32, 1e-6)
    out.update(d_row_start=rs, d_col=col, d_values=vals, d_b=b, d_minv=minv, d_x=xs, d_it=st["iterations"],
               d_conv=st["converged"])
    # ConjugateGradientFailsOnNonPositiveDenominator: A = -I, M^-1 = I.
    rs, col = np.array([0, 1], np.int32), np.array([0], np.int32)
    vals = diag_block(-1.0)[None]
    b = np.array([[1.0, 0.0, 0.0]])
    xs, st = po.reference_pcg(rs, col, vals, b, diag_block(1.0)[None], 8, 1e-6)
    out.update(e_row_start=rs, e_col=col, e_values=vals, e_b=b, e_x=xs, e_it=st["iterations"],
               e_conv=st["converged"])
    return out


def run_steps(scene, precision, steps, with_system=True):
    ref = po.Reference(scene, precision)
    rec = {}
    if with_system:
        s = ref.system()
        rec.update(sys_row_start=s.row_start, sys_col=s.col, sys_values=s.values, sys_rhs=s.rhs, sys_minv=s.minv,
                   sys_dv=s.dv, sys_node_to_dyn=s.node_to_dyn, sys_mass=s.mass, sys_force=s.force)
    xs, vs, its = [], [], []
    for _ in range(steps):
        if ref.step() != 0:
            raise RuntimeError("reference step failed")
        x, v = ref.state()
        xs.append(x)
        vs.append(v)
        st = ref.cg_stats()
        its.append([st["iterations"], st["converged"], st["residual"]])
    rec.update(x=np.stack(xs), v=np.stack(vs), cg=np.array(its))
    return {f"{precision}_{k}": val for k, val in rec.items()}


def main():
    if not po.reference_available("f32") or not po.reference_available("f64"):
        raise SystemExit("build the reference first: make -C oracle ref")
    np.savez_compressed(os.path.join(OUT, "kat_bsr.npz"), **kat_cases())

    box = meshes.small_box(2, 2, 2)
    rec = {}
    for p in ("f32", "f64"):
        rec.update(run_steps(box, p, 3))
    np.savez_compressed(os.path.join(OUT, "box_steps.npz"), **rec)

    cube = meshes.config1()
    rec = {}
    for p in ("f32", "f64"):
        rec.update(run_steps(cube, p, 2, with_system=False))
    np.savez_compressed(os.path.join(OUT, "cube8_steps.npz"), **rec)

    two = meshes.small_box(2, 2, 2)
    other = meshes.small_box(3, 2, 2, young=5e4, seed=11)
    two.bodies += other.bodies
    rec = {}
    for p in ("f32", "f64"):
        rec.update(run_steps(two, p, 2))
    np.savez_compressed(os.path.join(OUT, "two_bodies.npz"), **rec)

    beam = meshes.config5()
    np.savez_compressed(os.path.join(OUT, "beam32_tet_young.npz"), **run_steps(beam, "f64", 1, with_system=False))
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()

"""Tiling of the ring-staged PCG kernel, checked on the CPU (no GPU needed).

``pk_ring_tiling_selfcheck`` builds the kernel's tiles for a pattern, replays the
producer's bulk copies into a stage buffer byte for byte (widened spans, stage offsets,
the device allocations' slack) and evaluates every row through the staged data as the
consumer lanes index it.  Here it must report no index or span violation, and its
product must equal the symmetric upper-BSR product (SparseBlockMatrix::Multiply,
src/Math/SparseBlockMatrix.cpp:209-268) computed with numpy, for patterns built by the
drop-in host layer: structured Kuhn boxes, a body whose vertices are numbered at random
(long, scattered rows), and a multi-body world.
"""
import ctypes as C

import numpy as np
import pytest

from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def sym_upper_spmv(rs, col, vals, x):
    n = len(rs) - 1
    rows = np.repeat(np.arange(n), np.diff(rs))
    B = vals.reshape(-1, 3, 3).transpose(0, 2, 1)  # column-major blocks -> row-major matrices
    y = np.zeros((n, 3))
    np.add.at(y, rows, np.einsum("kij,kj->ki", B, x[col]))
    off = col != rows
    np.add.at(y, col[off], np.einsum("kji,kj->ki", B[off], x[rows[off]]))
    return y


def _pattern(scene):
    w = SimWorld(scene)
    w.prepare(upload=False)
    rs, col, _, _ = w.pattern()
    return rs.astype(np.int32), col.astype(np.int32)


def _check(rs, col, precision, seed=0):
    n = len(rs) - 1
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(9 * len(col))
    x = rng.standard_normal((n, 3))
    if precision != L.PK_PREC_FP64:
        vals = vals.astype(np.float32).astype(np.float64)
        x = x.astype(np.float32).astype(np.float64)
    y = np.zeros((n, 3))
    tiles, max_span = C.c_int(), C.c_int()
    bad = L.PK.pk_ring_tiling_selfcheck(precision, n, _ptr(rs), _ptr(col), _ptr(vals), _ptr(x), _ptr(y),
                                        C.byref(tiles), C.byref(max_span))
    assert bad == 0, (bad, L.last_error())
    ref = sym_upper_spmv(rs, col, vals, x)
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-10)
    return tiles.value, max_span.value




@pytest.mark.parametrize("precision", [L.PK_PREC_MIXED, L.PK_PREC_FP64])
def test_ring_tiling_structured_boxes(precision):
    for scene in (meshes.config1(), meshes.small_box(7, 3, 5), meshes.config5()):
        rs, col = _pattern(scene)
        tiles, max_span = _check(rs, col, precision)
        assert tiles > 0 and max_span > 0


@pytest.mark.parametrize("precision", [L.PK_PREC_MIXED, L.PK_PREC_FP64])
def test_ring_tiling_beam64(precision):
    rs, col = _pattern(meshes.config2())
    n = len(rs) - 1
    tiles, _ = _check(rs, col, precision, seed=1)
    rows = 32 if precision != L.PK_PREC_FP64 else 16
    assert tiles <= 2 * (n + rows - 1) // rows  # structured rows fill most tiles


def test_ring_tiling_randomly_numbered_body():
    scene = meshes.small_box(6, 5, 4)
    body = scene.bodies[0]
    rng = np.random.default_rng(3)
    perm = rng.permutation(body.positions.shape[0])  # new id -> old id
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    body.positions = body.positions[perm]
    body.tets = inv[body.tets].astype(np.int32)
    body.pinned = body.pinned[perm]
    if body.initial_positions is not None:
        body.initial_positions = body.initial_positions[perm]
    rs, col = _pattern(scene)
    for precision in (L.PK_PREC_MIXED, L.PK_PREC_FP64):
        _check(rs, col, precision, seed=2)


def test_ring_tiling_two_bodies():
    scene = meshes.small_box(4, 3, 3)
    scene.bodies.append(meshes.small_box(3, 5, 2, seed=9).bodies[0])
    rs, col = _pattern(scene)
    _check(rs, col, L.PK_PREC_MIXED, seed=4)

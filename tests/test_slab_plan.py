"""Layout of the part-resident PCG kernel, checked on the CPU (no GPU needed).

``pk_slab_plan_selfcheck`` cuts the rows into parts by their node positions, builds each
part's window (its rows, then the halo rows of other parts it couples to) and its stream
of tiles with 16-bit window columns, fills the stream from the upper blocks as the device
fill does, and evaluates y = A x by decoding the tiles exactly as the kernel's lanes read
them.  Both stream forms are checked: full symmetric rows (each block and the transpose
of each off-diagonal one), and the symmetric form that streams each block inside a part's
sub-part once and sends its transposed product through the consumer group's ring of
slots (decoded with the ring's wrap-around, so a slot reused too early would show).  The product must equal the symmetric upper-BSR product
(SparseBlockMatrix::Multiply, src/Math/SparseBlockMatrix.cpp:209-268) computed with
numpy, for patterns built by the drop-in host layer: structured boxes, the 128x64x64
block cut into 148 parts (the B200's SM count), a randomly numbered body, several
bodies, and parts cut without positions.  In the full form the self-check also requires
every part's interior rows (no halo column) ahead of its other rows and each tile's halo
flag to match its columns: the kernel streams the interior tiles before the halo exists.
"""
import ctypes as C

import numpy as np
import pytest

from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

from tests.test_ring_tiling import sym_upper_spmv


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _pattern_and_coords(scene):
    w = SimWorld(scene)
    w.prepare(upload=False)
    rs, col, n2d, _ = w.pattern()
    pos = np.concatenate([(b.initial_positions if b.initial_positions is not None else b.positions)
                          for b in scene.bodies]).astype(np.float64)
    n = len(rs) - 1
    coords = np.zeros((n, 3))
    dyn = n2d >= 0
    coords[n2d[dyn]] = pos[dyn]
    return rs.astype(np.int32), col.astype(np.int32), coords


FULL, SYM, AUTO = 0, 1, 2


def _check(rs, col, coords, parts, seed=0, form=FULL):
    n = len(rs) - 1
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(9 * len(col)).astype(np.float32).astype(np.float64)
    x = rng.standard_normal((n, 3)).astype(np.float32).astype(np.float64)
    y = np.full((n, 3), np.nan)
    info = np.zeros(5, np.int32)
    cp = _ptr(coords) if coords is not None else None
    rc = L.PK.pk_slab_plan_selfcheck(n, _ptr(rs), _ptr(col), _ptr(vals), _ptr(x), cp, parts, form, _ptr(y),
                                     _ptr(info))
    assert rc == 0, L.last_error()
    assert info[4] == (1 if form == SYM else 0 if form == FULL else info[4])
    ref = sym_upper_spmv(rs, col, vals, x)
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-10)
    return info


@pytest.mark.parametrize("form", [FULL, SYM])
@pytest.mark.parametrize("parts", [1, 3, 16])
def test_slab_plan_structured_boxes(parts, form):
    for scene in (meshes.config1(), meshes.small_box(7, 3, 5), meshes.config5()):
        rs, col, coords = _pattern_and_coords(scene)
        info = _check(rs, col, coords, parts, form=form)
        assert info[0] == min(parts, len(rs) - 1)
        assert 0 < info[1] <= 6144


@pytest.mark.parametrize("form", [FULL, SYM])
def test_slab_plan_block128_at_148_parts_fits_shared_memory(form):
    scene = meshes.config4()
    rs, col, coords = _pattern_and_coords(scene)
    info = _check(rs, col, coords, 148, seed=5, form=form)
    n = len(rs) - 1
    assert info[0] == 148
    assert info[1] <= 6144  # window of every part inside the kernel's shared-memory window
    assert info[2] <= 128
    assert info[1] < 2 * (n // 148)  # coordinate cuts keep halos well below the part size
    if form == SYM:  # each in-part block streamed about once: well under the full rows' stream
        full = _check(rs, col, coords, 148, seed=5, form=FULL)
        assert info[3] < 0.7 * full[3], (info[3], full[3])


def test_slab_plan_randomly_numbered_body():
    scene = meshes.small_box(6, 5, 4)
    body = scene.bodies[0]
    rng = np.random.default_rng(3)
    perm = rng.permutation(body.positions.shape[0])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    body.positions = body.positions[perm]
    body.tets = inv[body.tets].astype(np.int32)
    body.pinned = body.pinned[perm]
    rs, col, coords = _pattern_and_coords(scene)
    for form in (FULL, AUTO):
        _check(rs, col, coords, 5, seed=2, form=form)
        _check(rs, col, None, 5, seed=2, form=form)  # contiguous parts of the scattered numbering


def test_slab_plan_bodies_and_rows_without_positions():
    scene = meshes.small_box(4, 3, 3)
    scene.bodies.append(meshes.small_box(3, 5, 2, seed=9).bodies[0])
    rs, col, coords = _pattern_and_coords(scene)
    for form in (FULL, SYM):
        for parts in (1, 2, 7):
            _check(rs, col, coords, parts, seed=4, form=form)
            _check(rs, col, None, parts, seed=4, form=form)
        # every row in one spot: the cuts fall back to row order and still cover every row
        _check(rs, col, np.zeros_like(coords), 4, seed=6, form=form)


def _reject(rs, col, coords, parts, form=FULL):
    n = len(rs) - 1
    vals = np.zeros(9 * len(col))
    x = np.zeros((n, 3))
    y = np.zeros((n, 3))
    cp = _ptr(coords) if coords is not None else None
    rc = L.PK.pk_slab_plan_selfcheck(n, _ptr(rs), _ptr(col), _ptr(vals), _ptr(x), cp, parts, form, _ptr(y), None)
    assert rc == L.PK_ERR_UNSUPPORTED
    return L.last_error()


def test_slab_plan_rejects_parts_that_do_not_fit():
    # one part for the whole 18k-row beam: more rows than tensor memory holds
    rs, col, coords = _pattern_and_coords(meshes.config2())
    assert "tensor memory" in _reject(rs, col, coords, 1)
    assert "tensor memory" in _reject(rs, col, coords, 1, SYM)
    # randomly numbered beam cut into contiguous id ranges: every part touches most rows
    scene = meshes.config2()
    body = scene.bodies[0]
    perm = np.random.default_rng(5).permutation(body.positions.shape[0])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    body.positions = body.positions[perm]
    body.tets = inv[body.tets].astype(np.int32)
    body.pinned = body.pinned[perm]
    rs, col, _ = _pattern_and_coords(scene)
    assert "window" in _reject(rs, col, None, 6)
    assert "window" in _reject(rs, col, None, 6, SYM)


def test_symmetric_form_rejects_a_ring_too_small():
    # every row coupled to the next 45 rows: every sub-part is a dense band whose
    # transposed products in flight exceed the ring, so only the full rows apply
    n, band = 600, 45
    rows = np.repeat(np.arange(n), band + 1)
    cols = rows + np.tile(np.arange(band + 1), n)
    keep = cols < n
    rs = np.zeros(n + 1, np.int32)
    np.add.at(rs, rows[keep] + 1, 1)
    rs = np.cumsum(rs).astype(np.int32)
    col = cols[keep].astype(np.int32)
    assert "ring" in _reject(rs, col, None, 1, SYM)
    info = _check(rs, col, None, 1, seed=3, form=AUTO)  # falls back to the full rows
    assert info[4] == 0


def _segments(scene, n2d):
    """Dynamic-row ranges of the bodies (rows are numbered body by body)."""
    seg, base = [0], 0
    for b in scene.bodies:
        nodes = b.positions.shape[0]
        seg.append(seg[-1] + int(np.count_nonzero(n2d[base:base + nodes] >= 0)))
        base += nodes
    return np.asarray(seg, np.int32)


def _check_batched(scene, max_blocks, coords_on=True, seed=0, form=SYM):
    w = SimWorld(scene)
    w.prepare(upload=False)
    rs, col, n2d, _ = w.pattern()
    rs, col = rs.astype(np.int32), col.astype(np.int32)
    n = len(rs) - 1
    pos = np.concatenate([(b.initial_positions if b.initial_positions is not None else b.positions)
                          for b in scene.bodies]).astype(np.float64)
    coords = np.zeros((n, 3))
    coords[n2d[n2d >= 0]] = pos[n2d >= 0]
    seg = _segments(scene, n2d)
    rng = np.random.default_rng(seed)
    vals = rng.standard_normal(9 * len(col)).astype(np.float32).astype(np.float64)
    x = rng.standard_normal((n, 3)).astype(np.float32).astype(np.float64)
    y = np.full((n, 3), np.nan)
    info = np.zeros(6, np.int32)
    cp = _ptr(coords) if coords_on else None
    rc = L.PK.pk_slab_plan_batched_selfcheck(n, _ptr(rs), _ptr(col), _ptr(vals), _ptr(x), cp, _ptr(seg),
                                             len(seg) - 1, max_blocks, form, _ptr(y), _ptr(info))
    assert rc == 0, L.last_error()
    assert info[5] == (1 if form == SYM else 0)
    np.testing.assert_allclose(y, sym_upper_spmv(rs, col, vals, x), rtol=1e-12, atol=1e-10)
    return info


def test_batched_plan_small_worlds():
    scene = meshes.small_box(4, 3, 3)
    scene.bodies += meshes.small_box(3, 5, 2, seed=9).bodies + meshes.small_box(2, 2, 2, seed=5).bodies
    for form in (FULL, SYM):
        for max_blocks, coords_on in ((1, True), (2, True), (148, True), (3, False)):
            info = _check_batched(scene, max_blocks, coords_on, form=form)
            assert info[0] == 3 and info[4] == -(-3 // max_blocks)  # one part per small body


@pytest.mark.parametrize("form", [FULL, SYM])
def test_batched_plan_256_uneven_bodies(form):
    scene = meshes.config3()
    info = _check_batched(scene, 148, seed=3, form=form)
    parts, launches = int(info[0]), int(info[4])
    assert parts >= 256 and launches == -(-parts // 148) or launches == -(-parts // 148) + 1
    assert info[1] <= 6144 and info[2] <= 128


def test_slab_plan_pattern_joined_with_point_connections():
    """The pattern with point-connection blocks (two bodies joined, PHYSIK_AddPointConnection)
    through the part-resident layout: the blocks coupling the bodies cross parts."""
    scene = meshes.small_box(4, 3, 3)
    scene.bodies.append(meshes.small_box(3, 5, 2, seed=9).bodies[0])
    n0 = scene.bodies[0].positions.shape[0]
    w = SimWorld(scene)
    w.add_point_connection((5, n0 + 7, 9, n0 + 12), (0.25, 0.25, 0.25, 0.25), (0.1, 0.1, 0.1), 50.0)
    w.add_point_connection((20, 21, n0 + 30, n0 + 31), (0.4, 0.1, 0.3, 0.2), (0.0, 0.2, 0.1), 10.0)
    w.prepare(upload=False)
    rs, col, n2d, _ = w.pattern()
    rs, col = rs.astype(np.int32), col.astype(np.int32)
    plain = SimWorld(scene)
    plain.prepare(upload=False)
    assert len(col) > len(plain.pattern()[1])
    pos = np.concatenate([b.positions for b in scene.bodies]).astype(np.float64)
    coords = np.zeros((len(rs) - 1, 3))
    dyn = n2d >= 0
    coords[n2d[dyn]] = pos[dyn]
    for form in (FULL, SYM):
        for parts in (2, 5):
            _check(rs, col, coords, parts, seed=7, form=form)

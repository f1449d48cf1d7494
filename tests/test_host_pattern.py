"""Host-side logic of the drop-in library, no GPU needed.

* The shared libraries load and export every function the public headers declare.
* The solver scene the host builds before any upload -- lumped masses, dynamic-node
  mapping, canonical upper BSR pattern -- equals the reference's SolverData bit for bit
  (reference compiled here from its sources), including deactivated tets, freed and
  fixed nodes and multi-body worlds.
* World settings clamps and defaults (World.cpp:24-27, 157-205; World.h:131-134).
* TetMeshGenerator welding and degenerate-tet removal (TetMeshGenerator.cpp:153-282).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

needs_ref = pytest.mark.skipif(not po.reference_available("f32"), reason="reference not built (make -C oracle ref)")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def test_libraries_export_every_declared_symbol():
    for header in L.HEADERS:
        names = L.declared_symbols(header)
        assert names, header
        for name in names:
            lib = L.pkcuda if name.startswith("pk_") else L.physik
            assert hasattr(lib, name), f"{name} declared in {header} but not exported"


def _compare_with_reference(scene, mutate=None):
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    if mutate:
        mutate(w, ref)
    w.prepare(upload=False)
    rs, col, n2d, mass = w.pattern()
    s = ref.system()
    np.testing.assert_array_equal(rs, s.row_start)
    np.testing.assert_array_equal(col, s.col)
    np.testing.assert_array_equal(n2d, s.node_to_dyn)
    np.testing.assert_array_equal(mass, s.mass)  # float32 sums in the reference's order


@needs_ref
def test_pattern_mass_mapping_cube8():
    _compare_with_reference(meshes.config1())


@needs_ref
def test_pattern_mass_mapping_beam32_per_tet_young():
    _compare_with_reference(meshes.config5())


@needs_ref
def test_pattern_mass_mapping_block128():
    """The 128x64x64 block of the roofline workload (545,025 nodes, 3.1 M tets, 4.2 M
    upper blocks): the whole host scene against the reference's, bit for bit."""
    _compare_with_reference(meshes.config4())


@needs_ref
def test_pattern_mass_mapping_batched256():
    """The 256 uneven bodies of the batched workload, one world (bodies never couple)."""
    _compare_with_reference(meshes.config3())


@needs_ref
def test_pattern_mass_mapping_two_bodies():
    s = meshes.small_box(2, 2, 2)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    _compare_with_reference(s)


@needs_ref
def test_pattern_after_fixing_nodes():
    scene = meshes.small_box(3, 2, 2)

    # The harness can only fix nodes, so compare a world where nodes 5 and 7 were
    # additionally fixed through PHYSIK_SetNodeFixed.
    def mutate_fix_only(w, ref):
        for node in (5, 7):
            L.PX.PHYSIK_SetNodeFixed(w.h, node, 1)
        flags = scene.bodies[0].pinned.astype(np.uint8).copy()
        flags[[5, 7]] = 1
        ref.lib.ref_set_fixed.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        ref.lib.ref_set_fixed(ref.h, _ptr(np.ascontiguousarray(flags)), len(flags))

    _compare_with_reference(scene, mutate_fix_only)


def test_pattern_with_deactivated_tets_matches_oracle():
    """Deactivated tets leave the pattern (their blocks stay, as zero blocks, while their
    nodes stay active) but lose their mass; nodes no active tet references leave it."""
    scene = meshes.small_box(3, 2, 2)
    w = SimWorld(scene)
    off = [0, 1, 2, 3, 4, 5, 30]
    for t in off:
        L.PX.PHYSIK_SetTetActive(w.h, w.components[0], t, 0)
    w.prepare(upload=False)
    rs, col, n2d, mass = w.pattern()
    o = po.Oracle(scene, "f32")
    active = np.ones(scene.tet_count, np.uint8)
    active[off] = 0
    o.set_tet_active(active)
    node_active = np.zeros(scene.vertex_count, np.uint8)
    node_active[np.unique(scene.bodies[0].tets[active.astype(bool)])] = 1
    o.set_node_flags(active=node_active)
    o.step()
    s = o.last_system()
    np.testing.assert_array_equal(rs, s.row_start)
    np.testing.assert_array_equal(col, s.col)
    np.testing.assert_array_equal(n2d, s.node_to_dyn)
    np.testing.assert_array_equal(mass.astype(np.float32), s.mass)


def test_world_settings_defaults_and_clamps():
    X = L.PX
    h = X.PHYSIK_CreateWorld()
    try:
        assert abs(X.PHYSIK_GetConjugateGradientTolerance(h) - 1e-4) < 1e-10
        assert X.PHYSIK_GetConjugateGradientMaxIterations(h) == 128
        X.PHYSIK_SetConjugateGradientTolerance(h, float("inf"))
        assert abs(X.PHYSIK_GetConjugateGradientTolerance(h) - 1e-4) < 1e-10
        X.PHYSIK_SetConjugateGradientTolerance(h, 0.0)
        assert abs(X.PHYSIK_GetConjugateGradientTolerance(h) - 1e-8) < 1e-14
        X.PHYSIK_SetConjugateGradientTolerance(h, 1.0)
        assert abs(X.PHYSIK_GetConjugateGradientTolerance(h) - 0.1) < 1e-7
        X.PHYSIK_SetConjugateGradientMaxIterations(h, 0)
        assert X.PHYSIK_GetConjugateGradientMaxIterations(h) == 1
        X.PHYSIK_SetConjugateGradientMaxIterations(h, 4096)
        assert X.PHYSIK_GetConjugateGradientMaxIterations(h) == 1024
        assert X.PHYSIK_GetLastConjugateGradientIterations(h) == 0
        assert X.PHYSIK_DidLastConjugateGradientSolveConverge(h) == 0
    finally:
        X.PHYSIK_DestroyWorld(h)
    # NULL world: silent no-ops and zero getters, as in the reference.
    assert X.PHYSIK_GetConjugateGradientMaxIterations(None) == 0
    assert X.PHYSIK_GetLastConjugateGradientIterations(None) == 0
    assert X.PHYSIK_DidLastConjugateGradientSolveConverge(None) == 0
    X.PHYSIK_Step(None, 0.1)


def test_generator_welds_and_drops_degenerate_tets():
    X = L.PX
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1e-6, 0, 0], [1, 0, 0]], np.float32)
    tets = np.array([[0, 1, 2, 3], [4, 1, 2, 3], [0, 5, 2, 3], [0, 1, 2, 9]], np.int32)
    m = X.PHYSIK_GenerateTetMesh(_ptr(pos), 6, _ptr(tets), 4)
    try:
        assert X.PHYSIK_IsGeneratedTetMeshHandleValid(m) == 1
        # node 4 welds to node 0, node 5 to node 1: 4 distinct nodes
        assert X.PHYSIK_GetGeneratedTetMeshVertexCount(m) == 4
        # tet 1 becomes a duplicate of tet 0 (kept), tet 2 too (kept), tet 3 is out of range (dropped)
        assert X.PHYSIK_GetGeneratedTetMeshTetCount(m) == 3
        out = C.c_int()
        assert X.PHYSIK_GetGeneratedTetMeshTetNodeIndex(m, 4, C.byref(out)) == 1 and out.value == 0
    finally:
        X.PHYSIK_DestroyGeneratedTetMesh(m)
    assert X.PHYSIK_IsGeneratedTetMeshHandleValid(m) == 0
    flat = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32)
    m = X.PHYSIK_GenerateTetMesh(_ptr(flat), 4, _ptr(np.array([0, 1, 2, 3], np.int32)), 1)
    assert X.PHYSIK_GetGeneratedTetMeshTetCount(m) == 0  # zero volume
    X.PHYSIK_DestroyGeneratedTetMesh(m)


def test_massless_dynamic_node_is_reported_not_thrown():
    X = L.PX
    scene = meshes.small_box(2, 2, 2)
    w = SimWorld(scene)
    X.PHYSIK_AddNode(w.h, 5.0, 5.0, 5.0)  # active, not fixed, no tet: no mass
    assert X.PHYSIK_B200_PrepareScene(w.h, 0) == -1
    assert "no physical mass" in w.error()


def _connection_scene():
    s = meshes.small_box(2, 2, 2)
    s.bodies += meshes.small_box(3, 2, 2, young=5e4, seed=11).bodies
    return s


def _connections(scene):
    """Point connections of the checks below: inside body 0, across the two bodies, one with
    a pinned corner, one without stiffness (forces only), one with repeated nodes, one
    naming a node that does not exist (never added), and one with a non-finite target (kept,
    but it adds no block)."""
    n0 = scene.bodies[0].positions.shape[0]
    n1 = scene.bodies[1].positions.shape[0]
    pinned0 = int(np.nonzero(scene.bodies[0].pinned)[0][0])
    return [
        ((1, 4, 6, 7), (0.25, 0.25, 0.25, 0.25), (0.05, 0.12, 0.3), 40.0, 0.5),
        ((5, n0 + 7, 0, 0), (0.5, 0.5, 0.0, 0.0), (0.1, 0.1, 0.1), 80.0, 0.0),
        ((pinned0, 8, 2, 3), (0.4, 0.3, 0.2, 0.1), (0.0, -0.1, 0.2), 25.0, 0.1),
        ((n0 + 2, n0 + 3, n0 + 9, n0 + 10), (0.1, 0.2, 0.3, 0.4), (0.3, 0.0, 0.0), 0.0, 1.0),
        ((n0 + 5, n0 + 5, n0 + 6, n0 + 6), (0.3, 0.2, 0.25, 0.25), (0.2, 0.2, 0.0), 15.0, 0.0),
        ((0, 1, 2, n0 + n1 + 3), (0.25, 0.25, 0.25, 0.25), (0.0, 0.0, 0.0), 10.0, 0.0),
        ((2, n0 + 11, 3, 4), (0.5, 0.5, 0.0, 0.0), (float("nan"), 0.0, 0.0), 30.0, 0.0),
    ]


@needs_ref
def test_point_connection_pattern_matches_reference():
    """PHYSIK_AddPointConnection (PhysiKAPI.h:353-369): the connections' blocks join the
    pattern as SolverData::AssembleImplicitMatrixAndRhs builds it (SolverData.cpp:308-393),
    and only connections whose nodes exist are kept (World.cpp:126-131, 748-759)."""
    scene = _connection_scene()
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    for c in _connections(scene):
        w.add_point_connection(*c)
        ref.add_point_connection(*c)
    assert w.point_connection_count() == ref.point_connection_count() == len(_connections(scene)) - 1
    w.prepare(upload=False)
    rs, col, n2d, mass = w.pattern()
    s = ref.system()
    np.testing.assert_array_equal(rs, s.row_start)
    np.testing.assert_array_equal(col, s.col)
    np.testing.assert_array_equal(n2d, s.node_to_dyn)
    np.testing.assert_array_equal(mass, s.mass)
    # The blocks across the two bodies are new.
    plain = SimWorld(scene)
    plain.prepare(upload=False)
    assert len(col) > len(plain.pattern()[1])


def test_point_connection_needs_active_nodes():
    """World::AddPointConnection keeps a connection only if its four nodes exist and are
    active (World.cpp:126-131, 748-759): a node whose tets are all deactivated is inactive."""
    scene = meshes.small_box(2, 2, 2)
    w = SimWorld(scene)
    tets = scene.bodies[0].tets
    node = 0
    around = np.nonzero((tets == node).any(axis=1))[0]
    for t in around:
        L.PX.PHYSIK_SetTetActive(w.h, w.components[0], int(t), 0)
    w.add_point_connection((node, 1, 2, 3), (0.25, 0.25, 0.25, 0.25), (0.0, 0.0, 0.0), 10.0)
    assert w.point_connection_count() == 0
    other = int(tets[np.setdiff1d(np.arange(len(tets)), around)[0], 0])
    w.add_point_connection((other, other, other, other), (1.0, 0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 10.0)
    w.add_point_connection((-1, 1, 2, 3), (0.25, 0.25, 0.25, 0.25), (0.0, 0.0, 0.0), 10.0)
    assert w.point_connection_count() == 1

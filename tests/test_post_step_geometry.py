"""Post-step geometry (SurfaceExtractionComponent.cpp, SurfaceVisualComponent.cpp,
VisualMeshComponent.cpp; C ABI PhysiKAPI.cpp:703-717, 767-980, 1055-1170) against the
reference driven through its own C ABI.

Without a GPU: PHYSIK_Step(world, 0) runs the components' PostUpdate with no substep, so
the host route builds everything from the creation positions, local-position edits,
node moves and tet deactivation.  The index buffers (boundary faces in the reference's
hash-map order, filtered triangles), vertices, normals and embedding must equal the
FP32 reference bit for bit.

With a GPU (marked): after real steps the per-frame updates run on the device (skinning
and flat normals from the device state).  Their output must equal, bit for bit, the
reference's float formulas evaluated in float32 on this world's own positions, and the
index buffers must equal the reference's after the same steps.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import _lib as L
from physik_b200 import meshes
from physik_b200.world import SimWorld

needs_ref = pytest.mark.skipif(not po.reference_available("f32"), reason="reference not built (make -C oracle ref)")
_p, _i = C.c_void_p, C.c_int
H = po.RefHandle


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def scene_two_bodies():
    s = meshes.small_box(3, 2, 2)
    s.bodies += meshes.small_box(2, 3, 2, young=5e4, seed=11).bodies
    b = s.bodies[1]
    b.initial_positions = b.positions + np.float32(0.25)
    return s


# ---------------------------------------------------------------- our side
class Ours:
    def __init__(self, w: SimWorld, body: int):
        self.w, self.X, self.h = w, w.X, w.h
        self.body = w.components[body]
        self.ex = self.X.PHYSIK_CreateSurfaceExtractionComponent(self.h, self.body)
        self.sv = self.X.PHYSIK_CreateSurfaceVisualComponent(self.h, self.ex)
        self.vm = self.X.PHYSIK_CreateVisualMeshComponent(self.h, self.body)
        assert self.ex.valid() and self.sv.valid() and self.vm.valid()

    def surface(self):
        n = self.X.PHYSIK_GetSurfaceTriangleIndexCount(self.h, self.ex)
        out = np.zeros(max(n, 1), np.int32)
        got = self.X.PHYSIK_CopySurfaceTriangleIndices(self.h, self.ex, _ptr(out), n)
        assert got == n
        return out[:n]

    def visual(self):
        X, h, sv = self.X, self.h, self.sv
        nv = X.PHYSIK_GetSurfaceVisualVertexCount(h, sv)
        nn = X.PHYSIK_GetSurfaceVisualNormalCount(h, sv)
        ni = X.PHYSIK_GetSurfaceVisualTriangleIndexCount(h, sv)
        verts, normals = np.zeros((nv, 3), np.float32), np.zeros((nn, 3), np.float32)
        idx = np.zeros(ni, np.int32)
        fx, fy, fz, fi = C.c_float(), C.c_float(), C.c_float(), C.c_int()
        for i in range(nv):
            assert X.PHYSIK_GetSurfaceVisualVertex(h, sv, i, C.byref(fx), C.byref(fy), C.byref(fz)) == 1
            verts[i] = (fx.value, fy.value, fz.value)
        for i in range(nn):
            assert X.PHYSIK_GetSurfaceVisualNormal(h, sv, i, C.byref(fx), C.byref(fy), C.byref(fz)) == 1
            normals[i] = (fx.value, fy.value, fz.value)
        for i in range(ni):
            assert X.PHYSIK_GetSurfaceVisualTriangleIndex(h, sv, i, C.byref(fi)) == 1
            idx[i] = fi.value
        return verts, normals, idx

    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32)
        t = np.ascontiguousarray(tris, np.int32)
        self.X.PHYSIK_SetVisualMeshData(self.h, self.vm, _ptr(v), v.shape[0], _ptr(t), t.size)

    def embed(self):
        return self.X.PHYSIK_BuildVisualMeshEmbedding(self.h, self.vm)

    def mesh(self):
        X, h, vm = self.X, self.h, self.vm
        nv = X.PHYSIK_GetVisualMeshVertexCount(h, vm)
        ni = X.PHYSIK_GetVisualMeshTriangleIndexCount(h, vm)
        v = np.zeros((max(nv, 1), 3), np.float32)
        t = np.zeros(max(ni, 1), np.int32)
        assert X.PHYSIK_CopyVisualMeshVertices(h, vm, _ptr(v), nv) == nv
        assert X.PHYSIK_CopyVisualMeshTriangleIndices(h, vm, _ptr(t), ni) == ni
        return v[:nv], t[:ni]

    def set_tet_active(self, tet, on):
        self.X.PHYSIK_SetTetActive(self.h, self.body, int(tet), int(on))

    def on_device(self):
        return (self.X.PHYSIK_B200_GetVisualUpdateOnDevice(self.h, self.sv),
                self.X.PHYSIK_B200_GetVisualUpdateOnDevice(self.h, self.vm))


# ---------------------------------------------------------------- the reference
class Theirs:
    def __init__(self, ref: po.Reference, body: int):
        self.ref, self.w = ref, ref.world_handle()
        self.R = ref.real
        api = ref.api
        self.body = ref.body_handle(body)
        self.ex = api("PHYSIK_CreateSurfaceExtractionComponent", H, [_p, H])(self.w, self.body)
        self.sv = api("PHYSIK_CreateSurfaceVisualComponent", H, [_p, H])(self.w, self.ex)
        self.vm = api("PHYSIK_CreateVisualMeshComponent", H, [_p, H])(self.w, self.body)

    def surface(self):
        api = self.ref.api
        n = api("PHYSIK_GetSurfaceTriangleIndexCount", _i, [_p, H])(self.w, self.ex)
        out = np.zeros(max(n, 1), np.int32)
        assert api("PHYSIK_CopySurfaceTriangleIndices", _i, [_p, H, _p, _i])(self.w, self.ex, _ptr(out), n) == n
        return out[:n]

    def visual(self):
        api, w, sv, R = self.ref.api, self.w, self.sv, self.R
        nv = api("PHYSIK_GetSurfaceVisualVertexCount", _i, [_p, H])(w, sv)
        nn = api("PHYSIK_GetSurfaceVisualNormalCount", _i, [_p, H])(w, sv)
        ni = api("PHYSIK_GetSurfaceVisualTriangleIndexCount", _i, [_p, H])(w, sv)
        gv = api("PHYSIK_GetSurfaceVisualVertex", _i, [_p, H, _i, _p, _p, _p])
        gn = api("PHYSIK_GetSurfaceVisualNormal", _i, [_p, H, _i, _p, _p, _p])
        gi = api("PHYSIK_GetSurfaceVisualTriangleIndex", _i, [_p, H, _i, _p])
        verts, normals, idx = np.zeros((nv, 3)), np.zeros((nn, 3)), np.zeros(ni, np.int32)
        fx, fy, fz, fi = R(), R(), R(), C.c_int()
        for i in range(nv):
            assert gv(w, sv, i, C.byref(fx), C.byref(fy), C.byref(fz)) == 1
            verts[i] = (fx.value, fy.value, fz.value)
        for i in range(nn):
            assert gn(w, sv, i, C.byref(fx), C.byref(fy), C.byref(fz)) == 1
            normals[i] = (fx.value, fy.value, fz.value)
        for i in range(ni):
            assert gi(w, sv, i, C.byref(fi)) == 1
            idx[i] = fi.value
        return verts, normals, idx

    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32 if self.R is C.c_float else np.float64)
        t = np.ascontiguousarray(tris, np.int32)
        self.ref.api("PHYSIK_SetVisualMeshData", None, [_p, H, _p, _i, _p, _i])(self.w, self.vm, _ptr(v), v.shape[0],
                                                                              _ptr(t), t.size)

    def embed(self):
        return self.ref.api("PHYSIK_BuildVisualMeshEmbedding", _i, [_p, H])(self.w, self.vm)

    def mesh(self):
        api, w, vm = self.ref.api, self.w, self.vm
        nv = api("PHYSIK_GetVisualMeshVertexCount", _i, [_p, H])(w, vm)
        ni = api("PHYSIK_GetVisualMeshTriangleIndexCount", _i, [_p, H])(w, vm)
        v = np.zeros((max(nv, 1), 3), np.float32 if self.R is C.c_float else np.float64)
        t = np.zeros(max(ni, 1), np.int32)
        assert api("PHYSIK_CopyVisualMeshVertices", _i, [_p, H, _p, _i])(w, vm, _ptr(v), nv) == nv
        assert api("PHYSIK_CopyVisualMeshTriangleIndices", _i, [_p, H, _p, _i])(w, vm, _ptr(t), ni) == ni
        return v[:nv].astype(np.float64), t[:ni]

    def set_tet_active(self, tet, on):
        self.ref.api("PHYSIK_SetTetActive", None, [_p, H, _i, _i])(self.w, self.body, int(tet), int(on))

    def set_node_position(self, node, p):
        R = self.R
        self.ref.api("PHYSIK_SetNodePosition", None, [_p, _i, R, R, R])(self.w, int(node), *[float(c) for c in p])


def visual_mesh_input(body, seed=3, count=60):
    """Points spread over (and a little beyond) the body's bounding box, and triangles
    over them, some of which reference vertices outside every tet."""
    rng = np.random.default_rng(seed)
    lo, hi = body.positions.min(0), body.positions.max(0)
    pad = 0.1 * (hi - lo)
    pts = rng.uniform(lo - pad, hi + pad, size=(count, 3)).astype(np.float32)
    pts[:4] = body.positions[[0, 1, 5, 9]]  # exactly on nodes
    tris = rng.integers(0, count, size=(count, 3)).astype(np.int32)
    tris[-1] = (0, count + 3, 1)  # an index out of range: always filtered
    return pts, tris


def assert_same_visuals(ours: Ours, theirs: Theirs):
    np.testing.assert_array_equal(ours.surface(), theirs.surface())
    v, n, i = ours.visual()
    rv, rn, ri = theirs.visual()
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_array_equal(v.astype(np.float64), rv)
    np.testing.assert_array_equal(n.astype(np.float64), rn)
    mv, mt = ours.mesh()
    rmv, rmt = theirs.mesh()
    np.testing.assert_array_equal(mt, rmt)
    np.testing.assert_array_equal(mv.astype(np.float64), rmv)


# ---------------------------------------------------------------- CPU: host route
@needs_ref
def test_host_route_matches_reference_through_edits_and_deactivation():
    scene = scene_two_bodies()
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    for body in (0, 1):
        pts, tris = visual_mesh_input(scene.bodies[body], seed=3 + body)
        a, b = Ours(w, body), Theirs(ref, body)
        a.set_mesh(pts, tris)
        b.set_mesh(pts, tris)
        assert a.embed() == b.embed() == 1
        # before any frame: the extraction waits for PostUpdate, the visual mesh shows its rest vertices
        assert a.surface().size == 0 and b.surface().size == 0
        assert_same_visuals(a, b)
        w.step(0.0)
        assert ref.step(0.0) == 0
        assert a.surface().size > 0
        assert_same_visuals(a, b)
        assert a.on_device() == (0, 0)
        # local copies edited: the surface visual follows them (and a face flips when its
        # node crosses the opposite corner, once the surface is rebuilt by a topology event)
        tets = scene.bodies[body].tets
        moved = int(tets[0][0])
        for node, p in ((moved, scene.bodies[body].positions[int(tets[0][3])] * np.float32(1.5)),
                        (int(tets[3][1]), (0.05, -0.02, 0.3))):
            assert w.set_local_position(body, node, p) == 1
            ref.set_local_position(body, node, p)
        w.step(0.0)
        ref.step(0.0)
        assert_same_visuals(a, b)
        # tets deactivated: topology event -> new boundary, re-filtered triangles; the
        # vertices embedded in them keep their last skinned value
        for t in (0, 2, 5, 7):
            a.set_tet_active(t, False)
            b.set_tet_active(t, False)
        w.step(0.0)
        ref.step(0.0)
        assert_same_visuals(a, b)
        # world nodes moved: the visual mesh follows the world positions
        x, _ = w.state()
        begin = w.X.PHYSIK_GetTetMeshGlobalNodeBeginIndex(w.h, w.components[body])
        for k, node in enumerate((begin, begin + 4, begin + 7)):
            p = x[node] + np.float32(0.01 * (k + 1))
            w.X.PHYSIK_SetNodePosition(w.h, node, *[float(c) for c in p])
            b.set_node_position(node, p)
        w.step(0.0)
        ref.step(0.0)
        assert_same_visuals(a, b)
        # reactivation
        a.set_tet_active(2, True)
        b.set_tet_active(2, True)
        w.step(0.0)
        ref.step(0.0)
        assert_same_visuals(a, b)


@needs_ref
def test_degenerate_triangles_get_the_fallback_normal():
    scene = meshes.small_box(2, 2, 2)
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    a, b = Ours(w, 0), Theirs(ref, 0)
    w.step(0.0)
    ref.step(0.0)
    tris = a.surface().reshape(-1, 3)
    # collapse one surface triangle onto a point
    p = scene.bodies[0].positions[tris[0][0]]
    for node in tris[0]:
        assert w.set_local_position(0, int(node), p) == 1
        ref.set_local_position(0, int(node), p)
    w.step(0.0)
    ref.step(0.0)
    assert_same_visuals(a, b)
    _, n, _ = a.visual()
    np.testing.assert_array_equal(n[:3], np.tile(np.float32([0, 1, 0]), (3, 1)))


def test_argument_checks():
    w = SimWorld(meshes.small_box(2, 2, 2))
    X, h = w.X, w.h
    bad = L.ComponentHandle(0xFFFFFFFF, 0)
    assert not X.PHYSIK_CreateSurfaceExtractionComponent(h, bad).valid()
    assert not X.PHYSIK_CreateSurfaceExtractionComponent(None, w.components[0]).valid()
    assert not X.PHYSIK_CreateVisualMeshComponent(h, bad).valid()
    # a surface visual needs a surface extraction, not a tet mesh
    assert not X.PHYSIK_CreateSurfaceVisualComponent(h, w.components[0]).valid()
    a = Ours(w, 0)
    w.step(0.0)
    n = X.PHYSIK_GetSurfaceTriangleIndexCount(h, a.ex)
    assert n > 0 and n % 3 == 0
    out = np.full(n, -7, np.int32)
    assert X.PHYSIK_CopySurfaceTriangleIndices(h, a.ex, _ptr(out), 5) == 5
    assert (out[5:] == -7).all()
    assert X.PHYSIK_CopySurfaceTriangleIndices(h, a.ex, None, n) == 0
    assert X.PHYSIK_CopySurfaceTriangleIndices(h, a.ex, _ptr(out), 0) == 0
    assert X.PHYSIK_GetSurfaceTriangleIndexCount(h, a.sv) == 0  # wrong component kind
    fx = C.c_float()
    nv = X.PHYSIK_GetSurfaceVisualVertexCount(h, a.sv)
    assert nv == n
    assert X.PHYSIK_GetSurfaceVisualVertex(h, a.sv, nv, C.byref(fx), C.byref(fx), C.byref(fx)) == 0
    assert X.PHYSIK_GetSurfaceVisualVertex(h, a.sv, -1, C.byref(fx), C.byref(fx), C.byref(fx)) == 0
    assert X.PHYSIK_GetSurfaceVisualNormal(h, a.sv, 0, None, C.byref(fx), C.byref(fx)) == 0
    assert X.PHYSIK_GetSurfaceVisualTriangleIndex(h, a.sv, 0, None) == 0
    assert X.PHYSIK_GetSurfaceVisualVertexCount(h, a.ex) == 0
    # visual mesh: no data, no embedding
    assert X.PHYSIK_BuildVisualMeshEmbedding(h, a.vm) == 0
    assert X.PHYSIK_GetVisualMeshVertexCount(h, a.vm) == 0
    assert X.PHYSIK_BuildVisualMeshEmbedding(h, bad) == 0
    # vertices all outside: valid data, no vertex embedded, every triangle filtered out
    pts = np.float32([[10, 10, 10], [11, 10, 10], [10, 11, 10]])
    a.set_mesh(pts, np.int32([0, 1, 2]))
    assert X.PHYSIK_GetVisualMeshTriangleIndexCount(h, a.vm) == 3
    assert a.embed() == 0
    assert X.PHYSIK_GetVisualMeshTriangleIndexCount(h, a.vm) == 0
    v = np.zeros((3, 3), np.float32)
    assert X.PHYSIK_CopyVisualMeshVertices(h, a.vm, _ptr(v), 2) == 2
    np.testing.assert_array_equal(v[:2], pts[:2])
    X.PHYSIK_SetVisualMeshData(h, a.vm, None, 0, None, 0)
    assert X.PHYSIK_GetVisualMeshVertexCount(h, a.vm) == 0
    assert X.PHYSIK_B200_GetVisualUpdateOnDevice(h, a.ex) == -1


# ---------------------------------------------------------------- GPU: device route
def f32_normal(p0, p1, p2):
    """Cross(p1 - p0, p2 - p0) / length in float32, one rounding per operation (numpy's
    float32 arithmetic and sqrt are IEEE single operations)."""
    f = np.float32
    e1, e2 = (p1 - p0).astype(f), (p2 - p0).astype(f)
    c = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1], e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1).astype(f)
    length = np.sqrt((c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2]).astype(f)
    out = np.tile(f([0, 1, 0]), (c.shape[0], 1))
    ok = length > f(0.000001)
    out[ok] = c[ok] / length[ok, None]
    return out


def expected_visual(local, surface):
    tri = surface.reshape(-1, 3)
    p = local[tri]  # (T, 3, 3)
    n = f32_normal(p[:, 0], p[:, 1], p[:, 2])
    return p.reshape(-1, 3), np.repeat(n, 3, axis=0)


def expected_skinning(x, body_begin, tets, embedding, last, live):
    out = last.copy()
    f = np.float32
    for v, (tet, w) in enumerate(embedding):
        if tet < 0 or not live[v]:
            continue
        p = x[body_begin + tets[tet]].astype(f)
        acc = p[0] * f(w[0])
        for k in range(1, 4):
            acc = (acc + p[k] * f(w[k])).astype(f)
        out[v] = acc
    return out


def host_embedding(body, pts):
    """ComputeTetBarycentric + the first-active-tet scan, in float32 (the reference's
    float formula: every product and sum rounded once)."""
    f = np.float32
    rest = body.positions.astype(f)
    res = []

    def cross(a, b):
        return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], f)

    def dot(a, b):
        return f((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2])

    for p in pts:
        found = (-1, None)
        for t, n in enumerate(body.tets):
            a, b, c, d = rest[n]
            ab, ac, ad, ap = (b - a).astype(f), (c - a).astype(f), (d - a).astype(f), (p - a).astype(f)
            det = dot(ab, cross(ac, ad))
            if abs(det) <= f(0.00000001):
                continue
            inv = f(f(1.0) / det)
            wb = f(dot(ap, cross(ac, ad)) * inv)
            wc = f(dot(ab, cross(ap, ad)) * inv)
            wd = f(dot(ab, cross(ac, ap)) * inv)
            wa = f(f(f(f(1.0) - wb) - wc) - wd)
            w = (wa, wb, wc, wd)
            if all(x >= f(-0.0001) for x in w):
                found = (t, w)
                break
        res.append(found)
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp64"])
def test_device_route_is_bit_exact_and_topology_matches_reference(precision):
    scene = scene_two_bodies()
    w = SimWorld(scene, precision=precision)
    w.X.PHYSIK_SetSubstepCount(w.h, 2)
    ref = po.Reference(scene, "f32", substeps=2)
    body = 1
    pts, tris = visual_mesh_input(scene.bodies[body], seed=5)
    a, b = Ours(w, body), Theirs(ref, body)
    a.set_mesh(pts, tris)
    b.set_mesh(pts, tris)
    assert a.embed() == b.embed() == 1
    embedding = host_embedding(scene.bodies[body], pts)
    begin = w.X.PHYSIK_GetTetMeshGlobalNodeBeginIndex(w.h, w.components[body])
    live = np.array([t >= 0 for t, _ in embedding])
    last = pts.copy()
    for frame in range(4):
        w.step()
        assert ref.step() == 0
        assert a.on_device() == (1, 1)
        surface = a.surface()
        np.testing.assert_array_equal(surface, b.surface())
        local = w.local_positions(body)
        ev, en = expected_visual(local, surface)
        v, n, idx = a.visual()
        np.testing.assert_array_equal(idx, np.arange(surface.size))
        np.testing.assert_array_equal(v, ev)
        np.testing.assert_array_equal(n, en)
        x, _ = w.state()
        last = expected_skinning(x, begin, scene.bodies[body].tets, embedding, last, live)
        mv, mt = a.mesh()
        np.testing.assert_array_equal(mv, last)
        np.testing.assert_array_equal(mt, b.mesh()[1])
        if frame == 1:
            # deactivation between frames: the surface is rebuilt, the vertices embedded in
            # the deactivated tets stop following
            for t in (1, 4, 6):
                a.set_tet_active(t, False)
                b.set_tet_active(t, False)
            live = np.array([t >= 0 and t not in (1, 4, 6) for t, _ in embedding])


@pytest.mark.gpu
def test_local_edit_after_a_step_switches_to_the_host_route():
    scene = meshes.small_box(3, 2, 2)
    w = SimWorld(scene)
    ref = po.Reference(scene, "f32")
    a, b = Ours(w, 0), Theirs(ref, 0)
    w.step()
    ref.step()
    assert a.on_device()[0] == 1
    surface = a.surface()
    node = int(surface[0])
    assert w.set_local_position(0, node, (0.5, 0.5, 0.5)) == 1
    w.step(0.0)  # PostUpdate only: the edited copy is what the visual shows
    assert a.on_device()[0] == 0
    local = w.local_positions(0)
    assert tuple(local[node]) == (0.5, 0.5, 0.5)
    ev, en = expected_visual(local, a.surface())
    v, n, _ = a.visual()
    np.testing.assert_array_equal(v, ev)
    np.testing.assert_array_equal(n, en)
    w.step()  # the next frame overwrites the copy from the device again
    assert a.on_device()[0] == 1
    ev, en = expected_visual(w.local_positions(0), a.surface())
    v, n, _ = a.visual()
    np.testing.assert_array_equal(v, ev)
    np.testing.assert_array_equal(n, en)


@pytest.mark.gpu
def test_results_survive_a_precision_change():
    scene = meshes.small_box(3, 2, 2)
    w = SimWorld(scene, precision="fp32")
    a = Ours(w, 0)
    pts, tris = visual_mesh_input(scene.bodies[0], seed=9)
    a.set_mesh(pts, tris)
    assert a.embed() == 1
    w.step()
    assert a.on_device() == (1, 1)
    # the scene is rebuilt on the next step: the pending device results are fetched first
    w.X.PHYSIK_B200_SetPrecision(w.h, L.PK_PREC_FP64)
    before_v, _, _ = a.visual()
    before_m, _ = a.mesh()
    w.step(0.0)  # no substep: host route, same positions
    v, _, _ = a.visual()
    m, _ = a.mesh()
    np.testing.assert_array_equal(v, before_v)
    np.testing.assert_array_equal(m, before_m)
    w.step()
    assert a.on_device() == (1, 1)
    ev, en = expected_visual(w.local_positions(0), a.surface())
    v, n, _ = a.visual()
    np.testing.assert_array_equal(v, ev)
    np.testing.assert_array_equal(n, en)

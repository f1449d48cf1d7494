"""The part-resident ("slab") PCG kernel on the GPU, against the oracle and the other kernels.

The kernel keeps each part's search directions in shared memory and streams the matrix as
full symmetric rows or, by default where the layout fits, in the symmetric form (each
block inside a sub-part once); it runs wherever the storage is FP32 (FP32 and mixed
precision) and the parts' windows fit.  Tolerances are about ten times the errors measured
on a B200.  Checked here:

* it is the kernel the automatic choice picks for FP32-storage worlds, with one block per
  part, and not for FP64;
* one mixed-precision step equals the FP64 oracle's step (the reference's CPU solve in
  double, teacher-forced from the same state) to positions 3e-7 and velocities 2e-4
  (measured 3e-8 / 1.9e-5), on a box cut into a few parts, on the 64x16x16 beam cut into one part
  per SM (halos on every side), and on a two-body world;
* FP32 steps follow the FP32 reference restatement (positions 3e-7, velocities 2.5e-5);
* it agrees with the ring-staged kernel on the same step (both FP32 storage; they differ
  only in the order of sums);
* the solve is deterministic: two worlds stepped alike are bit-identical, and a graph
  replay equals plain launches.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def two_bodies():
    s = meshes.small_box(9, 6, 5)
    s.bodies += meshes.small_box(7, 8, 4, young=5e4, seed=11).bodies
    s.bodies[1].initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32),
                                             (s.bodies[1].positions.shape[0], 1))
    return s


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_slab_is_the_default_for_fp32_storage(precision):
    w = SimWorld(meshes.config1(), precision=precision)
    w.step()
    name, blocks = w.pcg_kernel()
    assert name == "slab" and blocks >= 1, (name, blocks, w.error())
    assert w.cg_stats()["flags"] & L.FLAG_INTEGRATED
    w64 = SimWorld(meshes.config1(), precision="fp64")
    w64.step()
    assert w64.pcg_kernel()[0] == "ring"


@pytest.mark.parametrize("make", [meshes.config1, meshes.config2, two_bodies], ids=["cube8", "beam64", "two_bodies"])
def test_slab_mixed_matches_fp64_oracle(make):
    scene = make()
    gpu = SimWorld(scene, precision="mixed")
    ora = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(2):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        assert gpu.pcg_kernel()[0] == "slab"
        x, v = gpu.state(f64=True)
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        assert rel(x, ora.x) <= 3e-7
        assert rel(v, ora.v) <= 2e-4
        assert abs(st["iterations"] - ora.last_stats()["iterations"]) <= 1


def test_slab_beam64_uses_one_block_per_part():
    w = SimWorld(meshes.config2(), precision="mixed")
    w.step()
    name, blocks = w.pcg_kernel()
    assert name == "slab" and blocks > 64, (name, blocks)


def test_slab_fp32_follows_fp32_reference():
    scene = meshes.config1()
    gpu = SimWorld(scene, precision="fp32")
    ora = po.Oracle(scene, "f32")
    for _ in range(3):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        assert gpu.pcg_kernel()[0] == "slab"
        assert rel(x, ora.x) <= 3e-7
        assert rel(v, ora.v) <= 2.5e-5
        assert abs(gpu.cg_stats()["iterations"] - ora.last_stats()["iterations"]) <= 1


def test_slab_agrees_with_ring_kernel(monkeypatch):
    scene = meshes.config2()
    slab = SimWorld(scene, precision="mixed")
    slab.step()
    assert slab.pcg_kernel()[0] == "slab"
    monkeypatch.setenv("PK_PCG_KERNEL", "ring")
    ring = SimWorld(scene, precision="mixed")
    ring.step()
    assert ring.pcg_kernel()[0] == "ring"
    xs, vs = slab.state(f64=True)
    xr, vr = ring.state(f64=True)
    assert rel(xs, xr) <= 3e-7
    assert rel(vs, vr) <= 2e-4
    assert abs(slab.cg_stats()["iterations"] - ring.cg_stats()["iterations"]) <= 2


def test_slab_is_deterministic_and_graph_replay_is_bit_identical():
    scene = two_bodies()
    a = SimWorld(scene, precision="mixed")
    b = SimWorld(scene, precision="mixed")
    g = SimWorld(scene, precision="mixed")
    g.set_graph(True)
    for _ in range(5):
        a.step()
        b.step()
        g.step()
    xa, va = a.state(f64=True)
    for w in (b, g):
        x, v = w.state(f64=True)
        np.testing.assert_array_equal(x, xa)
        np.testing.assert_array_equal(v, va)
    assert g.pcg_kernel()[0] == "slab"


# ---------------------------------------------------------------- stream forms
# The part-resident kernel streams full symmetric rows (the default) or, where the layout
# fits and PK_SLAB_FORM asks for it, the symmetric form (each block inside a sub-part
# streamed once, its transposed product sent through the consumer group's ring of slots in
# shared memory).  Both must follow the FP64 oracle, agree with each other to summation
# order, and repeat bit for bit (also under CUDA-graph replay).


def _world(scene, form, monkeypatch, precision="mixed", graph=False):
    monkeypatch.setenv("PK_SLAB_FORM", form)
    w = SimWorld(scene, precision=precision)
    if graph:
        w.set_graph(True)
    return w


@pytest.mark.parametrize("form", ["full", "sym"])
@pytest.mark.parametrize("make", [meshes.config1, meshes.config2, two_bodies], ids=["cube8", "beam64", "two_bodies"])
def test_stream_forms_follow_fp64_oracle(make, form, monkeypatch):
    scene = make()
    gpu = _world(scene, form, monkeypatch)
    ora = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(2):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        assert gpu.pcg_kernel()[0] == "slab" and gpu.pcg_stream_form() == form, (gpu.pcg_stream_form(), gpu.error())
        x, v = gpu.state(f64=True)
        st = gpu.cg_stats()
        assert st["flags"] & L.FLAG_INTEGRATED, hex(st["flags"])
        assert rel(x, ora.x) <= 3e-7
        assert rel(v, ora.v) <= 2e-4
        assert abs(st["iterations"] - ora.last_stats()["iterations"]) <= 1


def test_stream_forms_agree_and_full_is_the_default(monkeypatch):
    scene = meshes.config2()
    monkeypatch.delenv("PK_SLAB_FORM", raising=False)
    default = SimWorld(scene, precision="mixed")
    default.step()
    assert default.pcg_stream_form() == "full"
    auto = _world(scene, "auto", monkeypatch)  # the symmetric form where it fits
    auto.step()
    assert auto.pcg_stream_form() == "sym"
    full = _world(scene, "full", monkeypatch)
    full.step()
    np.testing.assert_array_equal(default.state(f64=True)[0], full.state(f64=True)[0])
    xa, va = auto.state(f64=True)
    xf, vf = full.state(f64=True)
    assert rel(xa, xf) <= 3e-7
    assert rel(va, vf) <= 2e-4
    assert abs(auto.cg_stats()["iterations"] - full.cg_stats()["iterations"]) <= 2


def test_sym_form_repeats_bit_for_bit_and_under_graph_replay(monkeypatch):
    scene = two_bodies()
    a = _world(scene, "sym", monkeypatch)
    b = _world(scene, "sym", monkeypatch)
    g = _world(scene, "sym", monkeypatch, graph=True)
    for _ in range(5):
        a.step()
        b.step()
        g.step()
    xa, va = a.state(f64=True)
    for w in (b, g):
        x, v = w.state(f64=True)
        np.testing.assert_array_equal(x, xa)
        np.testing.assert_array_equal(v, va)
    assert g.pcg_stream_form() == "sym"


def test_sym_form_fp32_follows_fp32_reference(monkeypatch):
    scene = meshes.config1()
    gpu = _world(scene, "sym", monkeypatch, precision="fp32")
    ora = po.Oracle(scene, "f32")
    for _ in range(3):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        assert gpu.pcg_stream_form() == "sym"
        assert rel(x, ora.x) <= 3e-7
        assert rel(v, ora.v) <= 2.5e-5


"""Batched per-body solve (PHYSIK_B200_SetBatchedSolve) against one-body worlds.

A reference World holding only one body runs that body's PCG with its own scalars and
stopping test.  The batched step must reproduce, for every body of a many-body world, the
step of a one-body world: here against the FP64 oracle run on each body alone (fed the
same float32 inputs the C ABI passes) and against the unbatched GPU path on each body
alone.  Bodies differ in size (some are split over several blocks), stiffness, rotation
and initial velocity, as in the batched uneven-bodies workload.  With FP32 storage the
batched solve runs on the part-resident kernel with one group of parts per body in one
persistent launch (checked also when the bodies need several rounds of it, and with the
round table the device rebuilds before every solve from the previous iteration counts);
the per-body batch kernel serves FP64.  Tolerances as in the
step parity tests: FP64 positions 1e-14 / velocities 1e-12, mixed positions 3e-7 against
the FP64 oracle; CG iterations within one.
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


def uneven_bodies(count=5, seed=5):
    """Small Kuhn boxes of different sizes / materials / motions, each pinned on i == 0."""
    rng = np.random.default_rng(seed)
    bodies = []
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(2, 7, size=3))
        young = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        sub = meshes.small_box(nx, ny, nz, young=young, poisson=float(rng.uniform(0.25, 0.45)), seed=100 + b)
        body = sub.bodies[0]
        body.positions = body.positions + np.float32(0.5 * b)  # keep bodies apart
        vel = rng.normal(0.0, 0.5, size=3).astype(np.float32)
        body.initial_velocities = np.tile(vel, (body.positions.shape[0], 1))
        body.initial_velocities[body.pinned] = 0.0
        bodies.append(body)
    scene = meshes.small_box(2, 2, 2)
    scene.bodies = bodies
    return scene


def one_body_scene(scene, i):
    s = meshes.small_box(2, 2, 2)
    s.bodies = [scene.bodies[i]]
    s.gravity, s.tolerance, s.max_iterations, s.dt = scene.gravity, scene.tolerance, scene.max_iterations, scene.dt
    return s


def body_slices(scene):
    out, base = [], 0
    for b in scene.bodies:
        n = b.positions.shape[0]
        out.append(slice(base, base + n))
        base += n
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_step_matches_one_body_worlds(precision):
    scene = uneven_bodies()
    gpu = SimWorld(scene, precision=precision)
    gpu.set_batched(True)
    oracles = [po.Oracle(one_body_scene(scene, i), "f64", float_inputs=precision == "fp64")
               for i in range(len(scene.bodies))]
    sl = body_slices(scene)
    tx, tv = (1e-14, 1e-12) if precision == "fp64" else (3e-7, 2e-4)
    for step in range(3):
        # teacher forcing: every body starts the step from its oracle's state
        gpu.set_state(np.concatenate([o.x for o in oracles]), np.concatenate([o.v for o in oracles]), f64=True)
        gpu.step()
        for o in oracles:
            o.step()
        x, v = gpu.state(f64=True)
        for i, o in enumerate(oracles):
            assert rel(x[sl[i]], o.x) <= tx, (step, i, rel(x[sl[i]], o.x))
            assert rel(v[sl[i]], o.v) <= tv, (step, i, rel(v[sl[i]], o.v))
            bs = gpu.body_stats(i)
            assert bs["flags"] & L.FLAG_INTEGRATED, hex(bs["flags"])
            assert abs(bs["iterations"] - o.last_stats()["iterations"]) <= 1, (bs, o.last_stats())
        st = gpu.cg_stats()
        assert st["iterations"] == max(gpu.body_stats(i)["iterations"] for i in range(len(oracles)))
        assert st["flags"] & L.FLAG_INTEGRATED


def test_batched_matches_unbatched_single_bodies():
    scene = uneven_bodies(count=4, seed=9)
    batched = SimWorld(scene, precision="fp64")
    batched.set_batched(True)
    singles = [SimWorld(one_body_scene(scene, i), precision="fp64") for i in range(len(scene.bodies))]
    sl = body_slices(scene)
    for _ in range(4):
        batched.step()
        for w in singles:
            w.step()
    x, v = batched.state(f64=True)
    for i, w in enumerate(singles):
        xs, vs = w.state(f64=True)
        assert rel(x[sl[i]], xs) <= 1e-11
        assert rel(v[sl[i]], vs) <= 1e-7
        assert batched.body_stats(i)["iterations"] == w.cg_stats()["iterations"]


def test_batched_with_a_fully_pinned_body():
    scene = uneven_bodies(count=3, seed=2)
    scene.bodies[1].pinned[:] = True
    scene.bodies[1].initial_velocities[:] = 0.0
    gpu = SimWorld(scene, precision="fp64")
    gpu.set_batched(True)
    x0, _ = gpu.state(f64=True)
    gpu.step()
    x, _ = gpu.state(f64=True)
    sl = body_slices(scene)
    np.testing.assert_array_equal(x[sl[1]], x0[sl[1]])
    for i in (0, 2):
        assert np.linalg.norm(x[sl[i]] - x0[sl[i]]) > 0
        assert gpu.body_stats(i)["flags"] & L.FLAG_INTEGRATED


def test_batched_toggle_back_to_coupled():
    scene = uneven_bodies(count=3, seed=4)
    a = SimWorld(scene, precision="fp64")
    b = SimWorld(scene, precision="fp64")
    a.set_batched(True)
    a.step()
    a.set_batched(False)
    b.step()
    a.set_state(*b.state(f64=True), f64=True)
    a.step()
    b.step()
    xa, _ = a.state(f64=True)
    xb, _ = b.state(f64=True)
    assert rel(xa, xb) <= 1e-13


@pytest.mark.parametrize("blocks", [0, 2])
def test_batched_part_resident_kernel_matches_one_body_worlds(blocks):
    """Mixed precision, batched: the part-resident kernel with a group of parts per body.
    blocks = 2 caps the launch at two blocks, so the five bodies take several rounds."""
    scene = uneven_bodies(count=5, seed=7)
    gpu = SimWorld(scene, precision="mixed")
    gpu.set_batched(True)
    if blocks:
        gpu.step()
        gpu.set_pcg_grid(blocks)
    oracles = [po.Oracle(one_body_scene(scene, i), "f64") for i in range(len(scene.bodies))]
    sl = body_slices(scene)
    for step in range(2):
        gpu.set_state(np.concatenate([o.x for o in oracles]), np.concatenate([o.v for o in oracles]), f64=True)
        gpu.step()
        for o in oracles:
            o.step()
        assert gpu.pcg_kernel()[0] == "slab-batched", gpu.pcg_kernel()
        x, v = gpu.state(f64=True)
        for i, o in enumerate(oracles):
            assert rel(x[sl[i]], o.x) <= 3e-7, (step, i, rel(x[sl[i]], o.x))
            assert rel(v[sl[i]], o.v) <= 2e-4, (step, i, rel(v[sl[i]], o.v))
            bs = gpu.body_stats(i)
            assert bs["flags"] & L.FLAG_INTEGRATED, hex(bs["flags"])
            assert abs(bs["iterations"] - o.last_stats()["iterations"]) <= 3, (bs, o.last_stats())
        st = gpu.cg_stats()
        assert st["iterations"] == max(gpu.body_stats(i)["iterations"] for i in range(len(oracles)))
        assert st["flags"] & L.FLAG_INTEGRATED


def test_batched_part_resident_agrees_with_batch_kernel(monkeypatch):
    scene = uneven_bodies(count=4, seed=11)
    slab = SimWorld(scene, precision="mixed")
    slab.set_batched(True)
    slab.step()
    assert slab.pcg_kernel()[0] == "slab-batched"
    monkeypatch.setenv("PK_PCG_KERNEL", "ring")  # no part-resident layout: the batch kernel
    other = SimWorld(scene, precision="mixed")
    other.set_batched(True)
    other.step()
    assert other.pcg_kernel()[0] == "batched"
    xs, _ = slab.state(f64=True)
    xo, _ = other.state(f64=True)
    assert rel(xs, xo) <= 1e-6
    for i in range(len(scene.bodies)):
        assert abs(slab.body_stats(i)["iterations"] - other.body_stats(i)["iterations"]) <= 2


def test_batched_round_table_does_not_change_results():
    """The device rebuilds the round table before every solve from the previous solve's
    per-body iteration counts; a body's solve must not depend on where it is placed.  A
    world that has stepped before (its table follows those counts) and a fresh world (its
    first table assumes the iteration cap) step from the same state bit for bit alike."""
    scene = uneven_bodies(count=6, seed=5)
    warm = SimWorld(scene, precision="mixed")
    warm.set_batched(True)
    warm.step()
    warm.set_pcg_grid(3)  # a new layout of three blocks
    for _ in range(2):
        warm.step()
    x0, v0 = warm.state(f64=True)
    fresh = SimWorld(scene, precision="mixed")
    fresh.set_batched(True)
    fresh.step()
    fresh.set_pcg_grid(3)  # the layout is rebuilt at the next solve, with no counts yet
    fresh.set_state(x0, v0, f64=True)
    fresh.step()
    warm.set_state(x0, v0, f64=True)
    warm.step()
    assert warm.pcg_kernel()[0] == "slab-batched" and fresh.pcg_kernel()[0] == "slab-batched"
    xw, vw = warm.state(f64=True)
    xf, vf = fresh.state(f64=True)
    np.testing.assert_array_equal(xw, xf)
    np.testing.assert_array_equal(vw, vf)
    for i in range(len(scene.bodies)):
        assert warm.body_stats(i)["iterations"] == fresh.body_stats(i)["iterations"]

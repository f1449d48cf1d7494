"""Step runtime options on the GPU: CUDA-graph replay, the autotuner, and each PCG kernel
variant the autotuner chooses from, checked against the oracle.

* A world stepped through a captured CUDA graph equals, bit for bit, the same world
  stepped with plain launches (same kernels in the same order; every kernel here is
  deterministic), unbatched and batched.
* Every PCG kernel variant (ring-staged, TMA-staged with 16/32/64-row tiles, unstaged)
  reproduces the FP64 oracle's step (the reference's CPU solve run in double) within
  the step-parity tolerances, and the autotuner's pick does too.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def scene_two_bodies():
    s = meshes.small_box(4, 3, 3)
    s.bodies += meshes.small_box(3, 5, 2, young=5e4, seed=11).bodies
    s.bodies[1].initial_velocities = np.tile(np.array([0.3, -0.2, 0.1], np.float32),
                                             (s.bodies[1].positions.shape[0], 1))
    return s


@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_graph_replay_is_bit_identical(precision, batched):
    scene = scene_two_bodies()
    plain = SimWorld(scene, precision=precision)
    graph = SimWorld(scene, precision=precision)
    for w in (plain, graph):
        w.set_batched(batched)
    graph.set_graph(True)
    for _ in range(6):
        plain.step()
        graph.step()
    xp, vp = plain.state(f64=True)
    xg, vg = graph.state(f64=True)
    np.testing.assert_array_equal(xp, xg)
    np.testing.assert_array_equal(vp, vg)
    assert plain.cg_stats()["iterations"] == graph.cg_stats()["iterations"]
    assert graph.cg_stats()["flags"] & L.FLAG_INTEGRATED


@pytest.mark.parametrize("kernel", ["ring", "staged", "plain"])
def test_each_pcg_kernel_matches_oracle(kernel, monkeypatch):
    if kernel != "ring":
        monkeypatch.setenv("PK_PCG_KERNEL", kernel)
    scene = meshes.config1()
    gpu = SimWorld(scene, precision="fp64")
    ora = po.Oracle(scene, "f64", float_inputs=True)
    for _ in range(2):
        gpu.set_state(ora.x, ora.v, f64=True)
        gpu.step()
        ora.step()
        x, v = gpu.state(f64=True)
        assert rel(x, ora.x) <= 1e-14 and rel(v, ora.v) <= 1e-12
        assert abs(gpu.cg_stats()["iterations"] - ora.last_stats()["iterations"]) <= 1


def test_autotuned_choice_matches_oracle():
    scene = scene_two_bodies()
    gpu = SimWorld(scene, precision="fp64")
    gpu.step()
    chosen, ms = gpu.autotune(2)
    assert 0 <= chosen <= 4 and ms > 0
    ora = po.Oracle(scene, "f64", float_inputs=True)
    gpu.set_state(ora.x, ora.v, f64=True)
    gpu.step()
    ora.step()
    x, v = gpu.state(f64=True)
    assert rel(x, ora.x) <= 1e-14 and rel(v, ora.v) <= 1e-12


def test_autotuned_batched_matches_untuned():
    scene = scene_two_bodies()
    tuned = SimWorld(scene, precision="fp64")
    plain = SimWorld(scene, precision="fp64")
    for w in (tuned, plain):
        w.set_batched(True)
        w.step()
    chosen, ms = tuned.autotune(2)
    assert 0 <= chosen <= 6 and ms > 0
    for _ in range(3):
        tuned.step()
        plain.step()
    xt, vt = tuned.state(f64=True)
    xp, vp = plain.state(f64=True)
    assert rel(xt, xp) <= 1e-12 and rel(vt, vp) <= 1e-8


def test_graph_after_autotune_batched_matches_plain():
    """The autotuner rebuilds the batched part table; the next graph capture must see it."""
    scene = scene_two_bodies()
    tuned = SimWorld(scene, precision="fp64")
    plain = SimWorld(scene, precision="fp64")
    for w in (tuned, plain):
        w.set_batched(True)
        w.step()
    tuned.autotune(2)
    tuned.set_graph(True)
    for _ in range(4):
        tuned.step()
        plain.step()
    st = tuned.cg_stats()
    assert st["flags"] & L.FLAG_INTEGRATED, (hex(st["flags"]), tuned.error())
    xt, _ = tuned.state(f64=True)
    xp, _ = plain.state(f64=True)
    assert rel(xt, xp) <= 1e-12

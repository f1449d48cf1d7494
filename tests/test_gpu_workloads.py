"""The benchmarked workloads themselves against the FP64 oracle, on the GPU.

* The 128x64x64 block (545,025 nodes, 3,145,728 tets, 536,640 dynamic rows, 4.2 M upper
  blocks; bench.py's default workload): the pattern of the device system equals the
  oracle's bit for bit, and two teacher-forced steps (each starting from the oracle's
  state) of the mixed, the FP32 and the FP64 device step follow the FP64 oracle (the
  reference's solve in double: SolverData.cpp:126-212, ConjugateGradientSolver.cpp:114-241)
  with the same 100 CG iterations.
* The 256 uneven bodies (batched per-body solve, CUDA graph): twelve bodies -- the two
  smallest, the two largest, the median and every 37th -- each against the FP64 oracle
  run on that body alone, two teacher-forced steps, iterations equal within one.

Each block step starts from the oracle's state rounded to float32 (what an FP32-stored
world holds), set back into the oracle, so the comparison sees the solver and the
assembly, not the storage of the state.  Tolerances are about ten times the errors
measured on a B200 (block: mixed and FP32 positions 2.3e-8 and velocities 1.4e-6, FP64
7e-17 / 4e-14; bodies: mixed 3.3e-8 / 9.5e-6, FP64 1.4e-16 / 1.5e-14).  For comparison,
the FP32 reference itself differs from the FP64 oracle on a block step from the same
float32 state by 3.3e-8 in positions and 1.4e-5 in velocities.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from physik_b200 import meshes

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

BLOCK_TOL = {"mixed": (3e-7, 2e-5), "fp32": (3e-7, 2e-5), "fp64": (1e-15, 1e-12)}
BODY_TOL = {"mixed": (3e-7, 1e-4), "fp64": (1e-15, 1e-12)}


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def block128():
    scene = meshes.config4()
    return scene, po.Oracle(scene, "f64", float_inputs=True)


def test_block128_pattern_and_steps_follow_fp64_oracle(block128):
    scene, ora = block128
    worlds = {p: SimWorld(scene, precision=p) for p in ("mixed", "fp32", "fp64")}
    for step in range(2):
        x0 = ora.x.astype(np.float32).astype(np.float64)
        v0 = ora.v.astype(np.float32).astype(np.float64)
        ora.set_state(x0, v0)
        for w in worlds.values():
            w.set_state(x0, v0, f64=True)
        ora.step()
        for p, w in worlds.items():
            w.step()
            x, v = w.state(f64=True)
            st = w.cg_stats()
            assert st["flags"] & L.FLAG_INTEGRATED, (p, hex(st["flags"]))
            tx, tv = BLOCK_TOL[p]
            assert rel(x, ora.x) <= tx, (p, step, rel(x, ora.x))
            assert rel(v, ora.v) <= tv, (p, step, rel(v, ora.v))
            assert st["iterations"] == ora.last_stats()["iterations"] == 100, (p, st)
            if step == 0 and p == "mixed":
                g, o = w.system(), ora.last_system()
                np.testing.assert_array_equal(g["row_start"], o.row_start)
                np.testing.assert_array_equal(g["col"], o.col)
                np.testing.assert_array_equal(g["node_to_dyn"], o.node_to_dyn)
                assert len(g["col"]) == 4210431


def _pick(sizes):
    order = np.argsort(sizes, kind="stable")
    pick = {int(order[0]), int(order[1]), int(order[-1]), int(order[-2]), int(order[len(order) // 2])}
    pick |= set(range(0, len(sizes), 37))
    return sorted(pick)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched256_bodies_follow_their_own_fp64_oracle(precision):
    scene = meshes.config3()
    sizes = [b.positions.shape[0] for b in scene.bodies]
    base = np.cumsum([0] + sizes)
    gpu = SimWorld(scene, precision=precision)
    gpu.set_batched(True)
    gpu.step()
    gpu.set_graph(True)
    x, v = gpu.state(f64=True)
    oracles = {}
    for i in _pick(sizes):
        one = meshes.Scene(f"body{i}", [scene.bodies[i]], dt=scene.dt, steps=1, gravity=scene.gravity,
                           tolerance=scene.tolerance, max_iterations=scene.max_iterations)
        o = po.Oracle(one, "f64", float_inputs=True)
        o.set_state(x[base[i]:base[i + 1]], v[base[i]:base[i + 1]])
        oracles[i] = o
    assert len(oracles) >= 8
    tx, tv = BODY_TOL[precision]
    for step in range(2):
        x, v = gpu.state(f64=True)
        for i, o in oracles.items():
            x[base[i]:base[i + 1]] = o.x
            v[base[i]:base[i + 1]] = o.v
        gpu.set_state(x, v, f64=True)
        gpu.step()
        xg, vg = gpu.state(f64=True)
        for i, o in oracles.items():
            o.step()
            bs = gpu.body_stats(i)
            assert bs["flags"] & L.FLAG_INTEGRATED, (i, hex(bs["flags"]))
            assert rel(xg[base[i]:base[i + 1]], o.x) <= tx, (i, step, rel(xg[base[i]:base[i + 1]], o.x))
            assert rel(vg[base[i]:base[i + 1]], o.v) <= tv, (i, step, rel(vg[base[i]:base[i + 1]], o.v))
            assert abs(bs["iterations"] - o.last_stats()["iterations"]) <= 1, (i, bs, o.last_stats())
    assert gpu.pcg_kernel()[0] in ("slab-batched", "batched")

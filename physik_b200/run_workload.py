"""Steps one of the benchmark workloads through the drop-in world and reports what ran.

    python -m physik_b200.run_workload block128 [--steps 3] [--precision mixed] [--batched]
    python -m physik_b200.run_workload cube8 --steps 5 --against-fp64

Builds the scene (synthetic meshes, physik_b200.meshes), steps it, and prints the PCG
kernel and block count of the last solve, CG iterations, flags and the step's device
time split (assembly / solve).  A small, fixed launch sequence -- per step one tet, one
row and one PCG launch -- for profilers.  With --against-fp64 it instead steps an FP64
world (one coupled solve) alongside, starts every step of the world under test from the
FP64 world's state, and prints each step's relative position and velocity differences.
"""
from __future__ import annotations

import argparse

from physik_b200 import meshes
from physik_b200.world import SimWorld

WORKLOADS = {"cube8": 1, "beam64": 2, "batched256": 3, "block128": 4, "beam32": 5}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", choices=["mixed", "fp32", "fp64"], default="mixed")
    ap.add_argument("--batched", action="store_true", help="one PCG per body")
    ap.add_argument("--against-fp64", action="store_true",
                    help="per-step position / velocity differences against an FP64 world")
    args = ap.parse_args(argv)
    scene = meshes.CONFIGS[WORKLOADS[args.workload]]()
    w = SimWorld(scene, precision=args.precision)
    w.set_batched(args.batched)
    if args.against_fp64:
        compare_fp64(args, scene, w)
        return
    w.step()  # builds and uploads the scene; timing starts with the next step
    w.enable_timing(True)
    for _ in range(max(0, args.steps - 1)):
        w.step()
    w.synchronize()
    st = w.cg_stats()
    tm = w.timings()
    kernel, blocks = w.pcg_kernel()
    n = max(1, tm["steps"])
    print(f"{args.workload} {args.precision}: {args.steps} steps, PCG kernel {kernel} on {blocks} blocks, "
          f"CG iterations {st['iterations']}, flags {st['flags']:#x}, assembly {tm['assemble_ms'] / n:.3f} ms, "
          f"solve {tm['solve_ms'] / n:.3f} ms per step")


def compare_fp64(args, scene, w):
    import numpy as np

    ref = SimWorld(scene, precision="fp64")
    for k in range(args.steps):
        x, v = ref.state(f64=True)
        w.set_state(x, v, f64=True)
        ref.step()
        w.step()
        xr, vr = ref.state(f64=True)
        xw, vw = w.state(f64=True)
        ex = np.linalg.norm(xw - xr) / max(np.linalg.norm(xr), 1e-300)
        ev = np.linalg.norm(vw - vr) / max(np.linalg.norm(vr), 1e-300)
        print(f"{args.workload} {args.precision} step {k + 1}: positions {ex:.2e}, velocities {ev:.2e} "
              f"(relative to FP64); CG iterations {w.cg_stats()['iterations']} (FP64 {ref.cg_stats()['iterations']})")


if __name__ == "__main__":
    main()

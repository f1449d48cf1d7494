"""Steps one of the benchmark workloads through the drop-in world and reports what ran.

    python -m physik_b200.run_workload block128 [--steps 3] [--precision mixed] [--batched]

Builds the scene (synthetic meshes, physik_b200.meshes), steps it, and prints the PCG
kernel and block count of the last solve, CG iterations, flags and the step's device
time split (assembly / solve).  A small, fixed launch sequence -- per step one tet, one
row and one PCG launch -- for profilers.
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
    args = ap.parse_args(argv)
    scene = meshes.CONFIGS[WORKLOADS[args.workload]]()
    w = SimWorld(scene, precision=args.precision)
    w.set_batched(args.batched)
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


if __name__ == "__main__":
    main()

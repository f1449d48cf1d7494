"""Benchmark of the implicit soft-body step (PhysiK's World::Step on the GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload block128|beam64|cube8|beam32|batched256] [--precision mixed|fp32|fp64]
    python bench.py --workload block128 --profile-steps 3 [--against-fp64]   (profiling runs)

One JSON line on rank 0.  A "step" is one PHYSIK_Step (one implicit-Euler substep:
per-tet corotated FEM, assembly of M + dt^2 K and its rhs, block-Jacobi PCG,
integration) of the whole workload.  The PCG kernel (and its tile or part size) is the
one the library's autotuner picks for the scene after the first step.

* value   -- steps/s with the state resident on the GPU, K steps timed with CUDA
             events on the world's stream (max over ranks).
* e2e     -- the same steps through the C ABI with host buffers: every step uploads
             positions and velocities from pinned host memory (PHYSIK_B200_SetNodeStates),
             steps, and reads them back (PHYSIK_B200_GetNodeStates); wall clock.
* roofline-- the PCG kernel: algorithmic bytes per solve (CG iterations x
             (40U + 4(n+1) + 24n + 132n) in FP32 storage, (76U + 4(n+1) + 48n + 264n) in
             FP64; per body for the batched solve) over its mean device time.
* config.fp64_gpu -- the plain FP64 GPU step (one coupled PCG, FP64 everywhere) on the
             same workload, and the mixed step's relative position error against it
             from one shared state.
* cpu_baseline -- the reference compiled from its own sources (oracle/_ref, FP32,
             one thread: the reference is single-threaded), bounded sample of the same
             workload (for the batched workload: a sample of bodies, each in its own
             reference World, scaled to the batch).

batched256 runs one PCG per body in one launch, replayed as a CUDA graph.

--impl reference times that reference CPU path alone on the same workload and prints
the same line with "impl": "reference".  Multi-GPU (torchrun): a single body does not
shard, so each rank runs an independent replica ("scaling": "weak"); the batched bodies
are independent, so rank r steps bodies r, r + N, ... ("scaling": "strong", no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "implicit steps/s & PCG SpMV HBM GB/s, mixed vs FP64 GPU at ≤1e-5 rel err"

WORKLOADS = {
    "block128": (4, "block128x64x64: 545,025 vertices, 3,145,728 Kuhn tets, bottom pinned, E=5e5 nu=0.4, "
                    "dt=1/60, CG tol 1e-6 / 100 iterations"),
    "beam64": (2, "beam64x16x16: 18,785 vertices, 98,304 Kuhn tets, x=0 pinned, E=1e6 nu=0.45, dt=1/120, "
                  "CG tol 1e-6 / 100 iterations"),
    "cube8": (1, "cube8: 729 vertices, 3,072 Kuhn tets, jitter 0.1h, x=0 pinned, E=1e5 nu=0.3, dt=1/60"),
    "beam32": (5, "beam32x8x8: 2,673 vertices, 12,288 Kuhn tets, per-element E, x=0 pinned, dt=1/60"),
    "batched256": (3, "batched256: 256 independent Kuhn boxes, cells per axis U{4..24} (seed 1), E log-uniform "
                      "[1e4,1e6], nu U[0.25,0.45], random rotation and rigid velocity N(0,0.5^2), x=0 face pinned, "
                      "dt=1/60, CG tol 1e-6 / 100 iterations, one PCG per body"),
}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


KERNEL_NAMES = {
    "slab": "pcg_slab_kernel (cooperative, one block per part: search directions resident in shared memory, "
            "full symmetric rows streamed by TMA, block-Jacobi, dots, integrate)",
    "ring": "pcg_ring_kernel (cooperative: TMA-staged upper BSR rows, L2 gathers of lower blocks and records, "
            "block-Jacobi, dots, integrate)",
    "staged": "pcg_kernel (cooperative, TMA-staged tiles)",
    "plain": "pcg_kernel (cooperative, unstaged)",
    "batched": "pcg_batch_kernel (cooperative per-body PCG: symmetric BSR SpMV + block-Jacobi + dots + integrate)",
    "slab-batched": "pcg_slab_kernel with one group of parts per body (per-body CG scalars and exchanges; "
                    "bodies packed into a few cooperative launches)",
}


def traffic_per_iteration():
    """DRAM bytes per PCG iteration from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "pcg_dram_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


class ClockSampler:
    """nvidia-smi clock / throttle sampling around the timed region.  The sampler starts
    before the warm-up and waits until it is writing; mark() records the wall-clock window
    of the timed region and summary() keeps only the samples taken inside it."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device, period_ms=20):
        self.device = device
        self.period_ms = period_ms
        self.proc = None
        self.file = None
        self.window = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.period_ms)], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        deadline = time.time() + 10.0  # wait until the sampler writes (its start-up takes a moment)
        while time.time() < deadline and self.proc.poll() is None:
            self.file.flush()
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.02)
        return self

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    @staticmethod
    def _stamp(text):
        import datetime

        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(text.strip(), fmt).timestamp()
            except ValueError:
                continue
        return None

    def summary(self):
        if self.proc is None or self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                try:
                    rows.append((self._stamp(parts[0]), float(parts[2]), float(parts[3]), float(parts[4]), parts[5:]))
                except ValueError:
                    continue
        os.unlink(self.file.name)
        if self.window is not None:
            t0, t1 = self.window
            rows = [r for r in rows if r[0] is not None and t0 <= r[0] <= t1]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples in the timed region"],
                    "period_ms": self.period_ms}
        sm = np.array([r[1] for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[4][1:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(r[2] for r in rows)),
                "power_w_max": float(max(r[3] for r in rows)), "samples": len(rows), "period_ms": self.period_ms,
                "window_s": round(self.window[1] - self.window[0], 4) if self.window else None,
                "reasons": sorted(reasons)}


def pcg_bytes_per_iteration(n, nnz, precision):
    if precision == "fp64":
        return 76 * nnz + 4 * (n + 1) + 48 * n + 264 * n
    return 40 * nnz + 4 * (n + 1) + 24 * n + 132 * n


def cpu_reference_sample(scene, budget_s=45.0, max_steps=None):
    """Time the reference (FP32 build of its own sources) on the same workload.
    One untimed step (it builds the component pattern), then timed steps until the
    budget is spent (at least one)."""
    from oracle import pyoracle as po

    if not po.reference_available("f32"):
        return None
    t0 = time.perf_counter()
    ref = po.Reference(scene, "f32")
    setup = time.perf_counter() - t0
    ref.step()
    times = []
    while True:
        t = time.perf_counter()
        if ref.step() != 0:
            raise RuntimeError("reference step failed")
        times.append(time.perf_counter() - t)
        if sum(times) >= budget_s or (max_steps and len(times) >= max_steps):
            break
    stats = ref.cg_stats()
    return dict(steps=len(times), seconds=float(sum(times)), steps_per_s=len(times) / sum(times),
                setup_s=setup, cg_iterations=stats["iterations"])


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def dist_setup(gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value, local):
    """The largest value over the ranks (a CUDA tensor with NCCL, a host tensor with gloo)."""
    if pg is None:
        return value
    import torch

    device = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def shard_scene(scene, rank, world):
    """Independent bodies split over ranks: rank r keeps bodies r, r + world, ..."""
    from physik_b200 import meshes

    if world <= 1:
        return scene
    return meshes.Scene(scene.name, scene.bodies[rank::world], dt=scene.dt, steps=scene.steps,
                        gravity=scene.gravity, tolerance=scene.tolerance, max_iterations=scene.max_iterations)


def batched_bytes(rs, col, n2d, scene, body_iters, precision):
    """Algorithmic PCG bytes of one batched solve: per body, its iterations times the
    per-iteration bytes of its own diagonal block of the matrix."""
    total, base, row0 = 0, 0, 0
    for b, body in enumerate(scene.bodies):
        nodes = body.positions.shape[0]
        dyn = n2d[base:base + nodes]
        rows = int(np.count_nonzero(dyn >= 0))
        if rows:
            nnz = int(rs[row0 + rows] - rs[row0])
            total += body_iters[b] * pcg_bytes_per_iteration(rows, nnz, precision)
        base += nodes
        row0 += rows
    return total


def time_steps(w, stream, steps):
    import torch

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(steps):
        w.step()
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop)


def run_ours(args, scene, rank, world, local, pg):
    import torch

    from physik_b200 import _lib
    from physik_b200.world import SimWorld

    torch.cuda.set_device(local)
    batched = args.workload == "batched256"
    w = SimWorld(scene, precision=args.precision, device=local)
    n_nodes = w.node_count
    w.set_batched(batched)
    w.step()  # builds and uploads the scene
    w.synchronize()
    tuned = w.autotune(3)  # picks the PCG kernel / tile or part size for this scene
    w.set_graph(batched)   # the batched step (many small bodies) is replayed as one CUDA graph
    rs, col, n2d, _ = w.pattern()
    n, nnz = len(rs) - 1, len(col)
    stream = torch.cuda.ExternalStream(w.stream(), device=f"cuda:{local}")

    # The clock sampler starts before the warm-up (its start-up takes a moment) and keeps
    # the samples of the timed region only.
    with ClockSampler(local) as clocks:
        for _ in range(args.warmup):
            w.step()
        w.synchronize()
        pcg_kernel, pcg_blocks = w.pcg_kernel()

        # --- device-resident timed region ---------------------------------
        w.enable_timing(True)
        barrier(pg)
        torch.cuda.synchronize()
        t_begin = time.time()
        elapsed_ms = time_steps(w, stream, args.steps)
        torch.cuda.synchronize()
        clocks.mark(t_begin, time.time())
    barrier(pg)
    elapsed_ms = max_over_ranks(pg, elapsed_ms, local)
    tm = w.timings()
    stats = w.cg_stats()
    clock = clocks.summary()
    if not (stats["flags"] & _lib.FLAG_INTEGRATED) or tm["steps"] != args.steps:
        raise RuntimeError(f"timed steps did not all run: flags {stats['flags']:#x}, {tm['steps']} timed steps, "
                           f"last error: {w.error()}")

    # PCG kernel time for the roofline: graph steps time as a whole, so a few extra steps
    # run with plain launches to split assembly and solve.
    if batched:
        w.set_graph(False)
        w.enable_timing(True)
        w.step()
        w.step()
        w.synchronize()
        tm_split = w.timings()
        w.set_graph(True)
        body_iters = [w.body_stats(i)["iterations"] for i in range(len(scene.bodies))]
        bytes_per_solve = batched_bytes(rs, col, n2d, scene, body_iters, args.precision)
    else:
        tm_split = tm
        bytes_per_solve = pcg_bytes_per_iteration(n, nnz, args.precision) * stats["iterations"]
    solve_ms = tm_split["solve_ms"] / max(1, tm_split["steps"])
    assemble_ms = tm_split["assemble_ms"] / max(1, tm_split["steps"])

    # --- end to end through the C ABI with pinned host buffers ------------
    hx = torch.empty((n_nodes, 3), dtype=torch.float32, pin_memory=True).numpy()
    hv = torch.empty((n_nodes, 3), dtype=torch.float32, pin_memory=True).numpy()
    x0, v0 = w.state()
    hx[:] = x0
    hv[:] = v0
    X = _lib.PX
    ptr = lambda a: a.ctypes.data_as(__import__("ctypes").c_void_p)  # noqa: E731
    for _ in range(max(1, args.warmup)):
        X.PHYSIK_B200_SetNodeStates(w.h, ptr(hx), ptr(hv), n_nodes)
        w.step()
        X.PHYSIK_B200_GetNodeStates(w.h, ptr(hx), ptr(hv), n_nodes)
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        X.PHYSIK_B200_SetNodeStates(w.h, ptr(hx), ptr(hv), n_nodes)
        w.step()
        X.PHYSIK_B200_GetNodeStates(w.h, ptr(hx), ptr(hv), n_nodes)
    e2e_s = time.perf_counter() - t0
    barrier(pg)
    e2e_s = max_over_ranks(pg, e2e_s, local)
    if not np.all(np.isfinite(hx)):
        raise RuntimeError("non-finite state after the e2e steps")

    # --- the plain FP64 GPU step on the same workload (one coupled solve), and the
    # mixed step's position error against it from one shared state ---------------
    fp64 = None
    if world == 1 and args.precision != "fp64" and not args.no_fp64:
        ref = SimWorld(scene, precision="fp64", device=local)
        ref.step()
        ref.synchronize()
        ref_stream = torch.cuda.ExternalStream(ref.stream(), device=f"cuda:{local}")
        for _ in range(2):
            ref.step()
        k = max(2, min(args.steps, 10))
        ref.enable_timing(True)
        ref_ms = time_steps(ref, ref_stream, k)
        ref_tm = ref.timings()
        ref_stats = ref.cg_stats()
        ref_kernel, ref_blocks = ref.pcg_kernel()
        ref_solve_ms = ref_tm["solve_ms"] / max(1, ref_tm["steps"])
        ref_bytes = pcg_bytes_per_iteration(n, nnz, "fp64") * ref_stats["iterations"]
        ref_achieved = ref_bytes / (ref_solve_ms / 1e3) / 1e9 if ref_solve_ms > 0 else None
        peak64, _ = measured_peaks()
        xs, vs = w.state(f64=True)
        ref.set_state(xs, vs, f64=True)
        w.set_state(xs, vs, f64=True)
        ref.step()
        w.step()
        xr, vr = ref.state(f64=True)
        xm, vm = w.state(f64=True)
        err = float(np.linalg.norm(xm - xr) / np.linalg.norm(xr))
        verr = float(np.linalg.norm(vm - vr) / max(np.linalg.norm(vr), 1e-300))
        fp64 = {"steps_per_s": k / (ref_ms / 1e3), "ms_per_step": ref_ms / k, "steps": k,
                "solve": "one coupled PCG over all bodies, FP64 storage and arithmetic",
                "pcg_kernel": ref_kernel, "pcg_blocks": ref_blocks, "cg_iterations": ref_stats["iterations"],
                "pcg_ms": ref_solve_ms, "assemble_ms": ref_tm["assemble_ms"] / max(1, ref_tm["steps"]),
                "algorithmic_bytes_per_solve": ref_bytes,
                "spmv_gbs": ref_achieved,
                "frac": (ref_achieved / peak64) if ref_achieved else None,
                "bytes_formula": "per CG iteration 76U + 4(n+1) + 48n + 264n (FP64 storage)",
                "mixed_position_rel_err_vs_fp64_one_step": err,
                "mixed_velocity_rel_err_vs_fp64_one_step": verr}
        del ref

    steps_total = args.steps * world if not batched else args.steps
    value = steps_total / (elapsed_ms / 1e3)
    achieved = bytes_per_solve / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else None
    peak, peak_kind = measured_peaks()
    traffic = None
    tpi = traffic_per_iteration()
    if (tpi and tpi.get("workload") == args.workload and tpi.get("precision") == args.precision
            and tpi.get("kernel") == pcg_kernel and not batched):
        traffic = float(tpi["dram_bytes_per_iteration"]) * stats["iterations"]
    return dict(
        value=value, ms_per_step=elapsed_ms / args.steps, e2e_s=e2e_s, n=n, nnz=nnz, nodes=n_nodes,
        iters=stats["iterations"], converged=stats["converged"], flags=stats["flags"], assemble_ms=assemble_ms,
        solve_ms=solve_ms, launches=tm["launches"], achieved=achieved, peak=peak, peak_kind=peak_kind,
        traffic=traffic, clocks=clock, bytes_per_solve=bytes_per_solve, h2d=2 * 12 * n_nodes, d2h=2 * 12 * n_nodes,
        tuned=tuned, fp64=fp64, batched=batched, pcg_kernel=pcg_kernel, pcg_blocks=pcg_blocks)


def reference_sample(args, scene):
    """The reference on the host cores.  One body: its PHYSIK_Step, one thread (the
    reference is single-threaded).  Batched bodies: each body stepped in a reference World
    of its own (what the batched solve computes per body), a sample of bodies timed and
    scaled to the whole batch."""
    if args.workload != "batched256":
        s = cpu_reference_sample(scene, budget_s=args.cpu_budget)
        if s is None:
            return None
        s["sample"] = (f"{s['steps']} timed PHYSIK_Step of {args.workload} ({s['seconds']:.1f} s) after 1 untimed "
                       f"step, FP32 reference compiled from its sources, 1 thread ({cpu_model()})")
        return s
    from physik_b200 import meshes

    sample = list(range(0, len(scene.bodies), 16))  # 16 of the 256 bodies, every 16th
    total, steps = 0.0, 0
    for i in sample:
        sub = meshes.Scene(f"body{i}", [scene.bodies[i]], dt=scene.dt, steps=scene.steps)
        s = cpu_reference_sample(sub, budget_s=args.cpu_budget / len(sample), max_steps=3)
        if s is None:
            return None
        total += s["seconds"] / s["steps"]
        steps = s["steps"]
    per_batch_step = total * len(scene.bodies) / len(sample)
    return {"steps_per_s": 1.0 / per_batch_step, "steps": steps, "seconds": total,
            "sample": (f"{len(sample)} of {len(scene.bodies)} bodies (every 16th), each in its own reference World, "
                       f"{steps} timed PHYSIK_Step each after 1 untimed step, scaled to the whole batch; FP32 "
                       f"reference compiled from its sources, 1 thread ({cpu_model()})")}


def profile_run(args, scene):
    """A small, fixed launch sequence for profilers: build the world, step it
    --profile-steps times (per step one tet, one row, one fill and one PCG launch), print
    the PCG kernel, CG iterations and the step's device time split.  No autotuning, no
    FP64 comparison, no CPU baseline.  With --against-fp64 every step of the world under
    test instead starts from an FP64 world's state and its position / velocity
    differences are printed."""
    from physik_b200.world import SimWorld

    w = SimWorld(scene, precision=args.precision)
    w.set_batched(args.workload == "batched256")
    if args.against_fp64:
        ref = SimWorld(scene, precision="fp64")
        for k in range(args.profile_steps):
            x, v = ref.state(f64=True)
            w.set_state(x, v, f64=True)
            ref.step()
            w.step()
            xr, vr = ref.state(f64=True)
            xw, vw = w.state(f64=True)
            ex = np.linalg.norm(xw - xr) / max(np.linalg.norm(xr), 1e-300)
            ev = np.linalg.norm(vw - vr) / max(np.linalg.norm(vr), 1e-300)
            print(f"{args.workload} {args.precision} step {k + 1}: positions {ex:.2e}, velocities {ev:.2e} "
                  f"(relative to FP64); CG iterations {w.cg_stats()['iterations']} "
                  f"(FP64 {ref.cg_stats()['iterations']})")
        return
    w.step()  # builds and uploads the scene; timing starts with the next step
    w.enable_timing(True)
    for _ in range(max(0, args.profile_steps - 1)):
        w.step()
    w.synchronize()
    st = w.cg_stats()
    tm = w.timings()
    kernel, blocks = w.pcg_kernel()
    k = max(1, tm["steps"])
    print(f"{args.workload} {args.precision}: {args.profile_steps} steps, PCG kernel {kernel} on {blocks} blocks, "
          f"CG iterations {st['iterations']}, flags {st['flags']:#x}, assembly {tm['assemble_ms'] / k:.3f} ms, "
          f"solve {tm['solve_ms'] / k:.3f} ms per step")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="block128")
    ap.add_argument("--precision", choices=["mixed", "fp32", "fp64"], default="mixed")
    ap.add_argument("--cpu-budget", type=float, default=45.0, help="seconds of reference CPU time to sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 GPU comparison")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling mode: step the workload this many times, print what ran, no JSON line")
    ap.add_argument("--against-fp64", action="store_true",
                    help="with --profile-steps: per-step differences against an FP64 world")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched256 side measurement of a single-GPU block128 run")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    from physik_b200 import meshes

    cfg, desc = WORKLOADS[args.workload]
    if args.profile_steps > 0:
        profile_run(args, meshes.CONFIGS[cfg]())
        return
    rank, world, local, pg = dist_setup(args.gpus)
    scene = meshes.CONFIGS[cfg]()
    batched = args.workload == "batched256"
    if batched and world > 1:
        # Bodies are independent: rank r steps bodies r, r + N, ... (no collective).
        scene = shard_scene(scene, rank, world)
    if batched:
        parallelism = "single GPU" if world == 1 else f"{world} GPUs, bodies sharded by rank, no collective"
    else:
        parallelism = "single GPU" if world == 1 else f"{world} independent replicas (a body does not shard)"
    base_config = {"workload": desc, "precision": args.precision, "gpus": world, "parallelism": parallelism,
                   "l2": "working set larger than the 126 MB L2; no flush between steps"}

    if args.impl == "reference":
        if rank != 0:
            return
        s = reference_sample(args, scene)
        if s is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": s["steps_per_s"], "unit": "steps/s",
                "n_gpus": 0, "steps": s["steps"], "warmup": 1, "ms_per_step": 1e3 / s["steps_per_s"],
                "higher_is_better": True, "scaling": "strong" if batched else "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": dict(base_config, precision="fp32 (reference)"),
                "cpu_baseline": {"value": s["steps_per_s"], "unit": "steps/s", "cores": 1, "kind": "reference",
                                 "sample": s["sample"]},
                "e2e": {"value": s["steps_per_s"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    r = run_ours(args, scene, rank, world, local, pg)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu_baseline:
        s = reference_sample(args, scene)
        if s is not None:
            cpu = {"value": s["steps_per_s"], "unit": "steps/s", "cores": 1, "kind": "reference",
                   "sample": s["sample"]}
    roof = None
    if r["achieved"] is not None:
        traffic_src = ("profiles/pcg_dram_traffic.json: DRAM bytes per CG iteration of an ncu capture of this "
                       "kernel on this workload, times this run's iterations" if r["traffic"] is not None else
                       "no ncu capture of this kernel and workload committed")
        kernel = KERNEL_NAMES.get(r["pcg_kernel"], r["pcg_kernel"]) + f", {r['pcg_blocks']} blocks"
        roof = {"bound": "hbm", "achieved": r["achieved"], "peak": r["peak"], "unit": "GB/s",
                "frac": r["achieved"] / r["peak"], "traffic": r["traffic"], "traffic_source": traffic_src,
                "kernel": kernel,
                "peak_source": f"{r['peak_kind']} hbm_gbs (MEASURED_PEAKS.json)",
                "algorithmic_bytes_per_solve": r["bytes_per_solve"],
                "bytes_formula": "per CG iteration 40U + 4(n+1) + 24n + 132n (FP32 storage), "
                                 "76U + 4(n+1) + 48n + 264n (FP64)"}
    cfg_out = dict(base_config, dynamic_rows=r["n"], upper_blocks=r["nnz"], cg_iterations=r["iters"],
                   converged=r["converged"], assemble_ms=r["assemble_ms"], pcg_ms=r["solve_ms"],
                   autotuned_candidate=r["tuned"][0], pcg_kernel=r["pcg_kernel"], pcg_blocks=r["pcg_blocks"],
                   batched_per_body_solve=r["batched"],
                   cuda_graph=r["batched"])
    if r["fp64"] is not None:
        cfg_out["fp64_gpu"] = r["fp64"]
    if world == 1 and args.workload == "block128" and not args.no_batched:
        # The batched workload (256 uneven bodies, one PCG per body) measured in the same run.
        side = argparse.Namespace(**vars(args))
        side.workload, side.no_fp64 = "batched256", True
        bcfg, bdesc = WORKLOADS["batched256"]
        b = run_ours(side, meshes.CONFIGS[bcfg](), rank, world, local, pg)
        cfg_out["batched256"] = {
            "workload": bdesc, "steps_per_s": b["value"], "ms_per_step": b["ms_per_step"],
            "e2e_steps_per_s": args.steps / b["e2e_s"], "pcg_ms": b["solve_ms"], "assemble_ms": b["assemble_ms"],
            "pcg_kernel": b["pcg_kernel"], "pcg_blocks": b["pcg_blocks"], "max_body_cg_iterations": b["iters"],
            "algorithmic_bytes_per_solve": b["bytes_per_solve"], "spmv_gbs": b["achieved"],
            "frac": (b["achieved"] / b["peak"]) if b["achieved"] else None, "cuda_graph": True,
            "gpu_launches": b["launches"], "clocks": b["clocks"]}
    line = {
        "metric": METRIC, "value": r["value"], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "strong" if r["batched"] else "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision != "fp64" else "f64", "data": "synthetic",
        "config": cfg_out, "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": (args.steps * (1 if r["batched"] else world)) / r["e2e_s"], "unit": "steps/s",
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
        "gpu_launches": r["launches"], "clocks": r["clocks"],
    }
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()

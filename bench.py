"""Benchmark of the vlp4d hot path on B200: Landau damping at 128^4.

Workload (one "step" = one Strang time step, timestep.hpp:14-67 of the
reference, as three fused passes + the FP64 field solve and diagnostic):
Landau damping with the sum-form initial condition
(1 + 0.05 cos(0.5x) + 0.05 cos(0.5y)) M(vx) M(vy) on x, y in [0, 4pi),
v in [-6, 6), 128^4 cells, dt = 0.1.  f is stored in FP32 (the headline)
and, for the FP32-vs-FP64 error and the FP64 throughput, also in FP64.
Inputs are synthetic (the initial condition); f (1.07 GB FP32) is larger
than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One process per GPU.  N > 1 cuts the same 128^4 run into N vy slabs
(distrib.SlabRun: NCCL send/recv of the halo planes and an all-reduce of
rho per step; strong scaling, timed as the max over ranks), and splits the
batched ensemble's members over the ranks (no communication); `--replicas`
runs N independent copies of the single-GPU workload instead.
`--impl reference` times the reference's own OpenMP CPU build (oracle/_ref)
on the host cores instead.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
N_GRID = 128
DT = 0.1
L_BOX = 4 * math.pi
VMAX = 6.0
METRIC = "Gcell-updates/s"
WORKLOAD = "Landau damping 128^4, dt 0.1, sum-form IC (amp 0.05, k 0.5), Strang step"


def headline_config(n, world, slabs=False, halo=4, rank=0):
    """The `config` of the headline line: the same dict for this library's
    arm and the reference arm at the same N.  With vy slabs, `rank`'s
    planes (rank 0 prints the line): nvy // world planes, one more on the
    first nvy % world ranks."""
    cells = n ** 4
    cfg = {"workload": WORKLOAD, "grid": [n] * 4, "dt": DT, "storage": "f32 f, f64 fields/diagnostics"}
    if slabs:
        nloc = n // world + (1 if rank < n % world else 0)
        cfg["parallelism"] = (f"vy slabs x{world}: {nloc} planes on rank {rank}, halo {halo} planes per side "
                              f"(NCCL send/recv), rho all-reduce (NCCL)")
        cfg["l2"] = "f slab (%.2f GB per GPU) larger than L2, no flush" % (cells / world * 4 / 1e9)
    else:
        cfg["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
        cfg["l2"] = "f (%.2f GB) larger than L2, no flush" % (cells * 4 / 1e9)
    return cfg


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=N_GRID, help="cells per dimension (default 128)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end runs")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip timing the reference CPU build")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own CUDA build (baseline/_ref) on this GPU")
    ap.add_argument("--only-f32", action="store_true", help="FP32 storage only (no FP64 run, no e2e): profiling")
    ap.add_argument("--only-f64", action="store_true",
                    help="the FP64 time loop and stage timings only (one JSON line): profiling")
    ap.add_argument("--case", choices=["main", "adjoint", "ensemble", "mpi", "stage"], default="main",
                    help="profiling cases: the reverse-mode, the ensemble or the vlp4d_mpi arm alone "
                         "(--steps steps, --members members, default tiles; --n for mpi), or one stage entry "
                         "point (--stage, --dtype, --n; --steps calls after one field solve), one JSON line")
    ap.add_argument("--stage", default="advect_xyxy",
                    choices=["advect_x", "advect_y", "advect_vx", "advect_vy", "advect_xy", "advect_vxvy",
                             "advect_xyxy", "field_rho", "field_poisson"], help="stage entry point for --case stage")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32", help="storage for --case stage")
    ap.add_argument("--members", type=int, default=256, help="ensemble members for --case ensemble")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent copies of the single-GPU workload instead of one run cut into vy slabs")
    ap.add_argument("--halo", type=int, default=4, help="vy halo planes per side of a slab (N > 1)")
    ap.add_argument("--slab", action="store_true",
                    help="run the vy-slab path even on one GPU (one slab, its halos filled from itself)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- ranks
class Ranks:
    """torch.distributed plumbing for barriers and max-over-ranks timing only."""

    def __init__(self, world: int, backend: str = "nccl"):
        self.world = world
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        if world > 1:
            import datetime

            import torch.distributed as dist

            if backend == "nccl":
                import torch

                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
            self.dist = dist
        self.backend = backend

    def _tensor(self, x):
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def aggregate(seconds_max: float, cells: int, steps: int, world: int) -> dict:
    """Whole-job throughput: all replicas' cell updates over the slowest rank's time."""
    return {
        "value": cells * steps * world / seconds_max / 1e9,
        "ms_per_step": seconds_max * 1e3 / steps,
    }


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timed regions."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"vlp4d_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------- GPU arm
def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_calls(torch, stream, fn, reps):
    """Mean device time (s) of `fn()` over `reps` calls, events on `stream`."""
    e0, e1 = _events(torch)
    fn()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def dram_traffic(n: int, kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    summary of the n^4 FP32 workload (lines "<kernel> <bytes>"), or None."""
    path = ROOT / "profiles" / f"dram_traffic_landau{n}_f32.txt"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0] == kernel and not line.startswith("#"):
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def gpu_arm(args, ranks):
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    v = pkg.vlp4d
    torch.cuda.set_device(ranks.local_rank)
    dev = torch.device("cuda", ranks.local_rank)
    stream = torch.cuda.current_stream(dev)
    K, W = args.steps, max(args.warmup, 3)
    n = args.n
    dom = pkg.landau_domain(n, dt=DT, nbiter=W + K + 2, L=L_BOX, vmax=VMAX)
    cells = dom.cells
    sampler = ClockSampler(ranks.local_rank)
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        sampler.index = "GPU-" + uuid if not uuid.startswith("GPU-") else uuid
    except Exception:
        pass
    out = {"stages": {}}
    sampler.start()

    per_dtype = {}
    for dtype in (("f32",) if args.only_f32 else ("f64",) if args.only_f64 else ("f32", "f64")):
        with pkg.Context(dom, dtype) as ctx:
            fa, fb = ctx.empty_f(), ctx.empty_f()
            ctx.init_case(fa, v.IC_LANDAU_SUM, 0.05, 0.5)
            ctx.field_rho(fa)
            ctx.field_poisson()
            ctx.diags_compute(0)
            cur, nxt = fa, fb
            for it in range(1, W + 1):
                ctx.step(cur, nxt, it)
                cur, nxt = nxt, cur
            torch.cuda.synchronize()
            ranks.barrier()
            torch.cuda.synchronize()
            # Headline: the time loop (vlp4d_steps), K steps in one call.
            launches0 = v.kernel_launches()
            e0, e1 = _events(torch)
            e0.record(stream)
            ctx.steps(cur, nxt, W + 1, K)
            e1.record(stream)
            torch.cuda.synchronize()
            cur, nxt = nxt, cur
            ranks.barrier()
            secs = e0.elapsed_time(e1) / 1e3
            launches = v.kernel_launches() - launches0
            ctx.check()
            tmax = ranks.max(secs)
            rec = aggregate(tmax, cells, K, ranks.world)
            rec["launches"] = launches
            # The same K steps as K calls of vlp4d_step (three passes each).
            ranks.barrier()
            e0.record(stream)
            for it in range(1, K + 1):
                ctx.step(cur, nxt, it)
                cur, nxt = nxt, cur
            e1.record(stream)
            torch.cuda.synchronize()
            rec["per_step_api"] = aggregate(ranks.max(e0.elapsed_time(e1) / 1e3), cells, K, ranks.world)
            # Stage timings: the reference's timer labels (timer.hpp:51-59) plus the fused passes.
            reps = 10
            st = {}
            st["advec1D_x"] = time_calls(torch, stream, lambda: ctx.advect_x(cur, nxt, 0.5 * DT), reps)
            st["advec1D_y"] = time_calls(torch, stream, lambda: ctx.advect_y(cur, nxt, 0.5 * DT), reps)
            st["advec1D_vx"] = time_calls(torch, stream, lambda: ctx.advect_vx(cur, nxt, DT), reps)
            st["advec1D_vy"] = time_calls(torch, stream, lambda: ctx.advect_vy(cur, nxt, DT), reps)
            st["advect_xy"] = time_calls(torch, stream, lambda: ctx.advect_xy(cur, nxt, 0.5 * DT), reps)
            st["advect_vxvy"] = time_calls(torch, stream, lambda: ctx.advect_vxvy(cur, nxt, DT), reps)
            st["advect_xyxy"] = time_calls(torch, stream, lambda: ctx.advect_xyxy(cur, nxt, 0.5 * DT), reps)
            st["field"] = time_calls(torch, stream, lambda: ctx.field_rho(cur), reps)
            st["Fourier"] = time_calls(torch, stream, lambda: ctx.field_poisson(), reps)
            st["diag"] = time_calls(torch, stream, lambda: ctx.diags_compute(1), reps)
            ctx.check()
            elem = 4 if dtype == "f32" else 8
            rw = 2.0 * cells * elem
            rec["stages"] = {
                k: {"ms": t * 1e3,
                    "gbs": ((cells * elem if k == "field" else rw) / t / 1e9) if k not in ("Fourier", "diag") else None}
                for k, t in st.items()}
            per_dtype[dtype] = rec
            del fa, fb, cur, nxt
            torch.cuda.empty_cache()

    clocks = sampler.stop()
    if args.only_f64:
        rec = per_dtype["f64"]
        return {"metric": METRIC, "value": rec["value"], "unit": METRIC, "n_gpus": ranks.world, "steps": K,
                "warmup": W, "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "dtype": "f64",
                "profiling": "FP64 arm only", "config": {"workload": WORKLOAD, "grid": [n] * 4, "dt": DT},
                "stages": rec["stages"], "gpu_launches": rec["launches"], "clocks": clocks}

    # Roofline of the dominant kernel of the time loop.  Each step between
    # the first and the last runs one k_plane_xyxy pass (two x/y half steps)
    # and one k_vslab pass (vx then vy); both read f once and write it once,
    # so the algorithmic bytes per launch are 2 * cells * 4 (FP32).
    peak, peak_kind = measured_hbm_peak()
    f32 = per_dtype["f32"]
    t_xx = f32["stages"]["advect_xyxy"]["ms"] / 1e3
    t_vv = f32["stages"]["advect_vxvy"]["ms"] / 1e3
    dominant = "advect_xyxy (k_plane_xyxy, two x/y half steps)" if t_xx >= t_vv else "advect_vxvy (k_vslab)"
    t_dom = max(t_xx, t_vv)
    achieved = 2.0 * cells * 4 / t_dom / 1e9
    traffic = dram_traffic(n, "k_plane_xyxy" if "xy" in dominant else "k_vslab")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": dominant, "peak_kind": peak_kind,
                "bytes_per_launch": 2 * cells * 4,
                # Whole-step fractions: f is read and written once per pass;
                # vlp4d_steps runs 2 passes per step, vlp4d_step 3.
                "step_frac_3pass": (6.0 * cells * 4 / (f32["per_step_api"]["ms_per_step"] / 1e3) / 1e9) / peak,
                "step_frac_2pass": (4.0 * cells * 4 / (f32["ms_per_step"] / 1e3) / 1e9) / peak}

    # End to end through the C ABI with host buffers (vlp4d_run): H2D of the
    # initial f from pinned memory, the initial solve, K steps, D2H of the
    # diagnostic history and of the final f.
    e2e = None
    err = {}
    if not args.no_e2e and not args.only_f32:
        e2e_vals = {}
        for dtype in ("f32", "f64"):
            tdt = torch.float32 if dtype == "f32" else torch.float64
            with pkg.Context(dom, dtype) as ctx:
                fa, fb = ctx.empty_f(), ctx.empty_f()
                ctx.init_case(fa, v.IC_LANDAU_SUM, 0.05, 0.5)
                h0 = torch.empty(dom.shape4, dtype=tdt, pin_memory=True)
                h0.copy_(fa)
                hout = torch.empty(dom.shape4, dtype=tdt, pin_memory=True)
                torch.cuda.synchronize()
                ranks.barrier()
                e0, e1 = _events(torch)
                e0.record(stream)
                ctx.run(h0, K, fa, fb, f_out_host=hout)
                e1.record(stream)
                torch.cuda.synchronize()
                secs = ranks.max(e0.elapsed_time(e1) / 1e3)
                e2e_vals[dtype] = cells * K * ranks.world / secs / 1e9
                fbytes = cells * h0.element_size()
                if dtype == "f32":
                    e2e = {"value": e2e_vals["f32"], "unit": METRIC,
                           "h2d_bytes_per_step": fbytes / K, "d2h_bytes_per_step": (fbytes + 16 * (K + 1)) / K,
                           "seconds": secs, "api": "vlp4d_run (C ABI, pinned host buffers)"}
                del fa, fb, h0, hout
                torch.cuda.empty_cache()
        err = error_arm(pkg, torch, n)
        err["e2e_f64"] = e2e_vals["f64"]

    adjoint = None if args.only_f32 else adjoint_arm(pkg, torch, stream)
    ensemble = None if args.only_f32 else ensemble_arm(pkg, torch, stream, peak)

    rec = per_dtype["f32"]
    line = {
        "metric": METRIC, "value": rec["value"], "unit": METRIC, "n_gpus": ranks.world, "steps": K, "warmup": W,
        "ms_per_step": rec["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "api": "vlp4d_steps (time loop, K steps per call)",
        "per_step_api": rec["per_step_api"],
        "dtype": "f32", "data": "synthetic (Landau initial condition computed on the device)",
        "config": headline_config(n, ranks.world),
        "roofline": roofline, "e2e": e2e, "gpu_launches": rec["launches"], "clocks": clocks,
        "f64": ({"value": per_dtype["f64"]["value"], "ms_per_step": per_dtype["f64"]["ms_per_step"],
                 "per_step_api": per_dtype["f64"]["per_step_api"],
                 "speedup_f32_over_f64": rec["value"] / per_dtype["f64"]["value"],
                 "published_a100_stdpar_f64": 7.19,
                 "stages": per_dtype["f64"]["stages"]} if "f64" in per_dtype else None),
        "stages": rec["stages"], "error_f32_vs_f64": err,
        "adjoint": adjoint,
        "ensemble": ensemble,
    }
    return line


def slab_arm(args, ranks):
    """N > 1: the 128^4 FP32 run cut into N vy slabs, one per GPU
    (distrib.SlabRun on slab contexts; per step an NCCL all-reduce of the
    nx*ny FP64 rho and NCCL send/recv of `--halo` vy planes on each side).
    Strong scaling: the whole job advances N^4 cells per step.  `value` is
    device-timed with CUDA events over K steps on buffers already on the
    GPUs (max over ranks); `e2e` adds, per rank, the H2D copy of its owned
    planes of f0 from pinned memory, the initial solve, and the D2H copy of
    its final planes and of the diagnostic history."""
    import importlib

    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    v = pkg.vlp4d
    d = importlib.import_module(pkg.__name__ + ".distrib")
    torch.cuda.set_device(ranks.local_rank)
    dev = torch.device("cuda", ranks.local_rank)
    stream = torch.cuda.current_stream(dev)
    K, W = args.steps, max(args.warmup, 3)
    n = args.n
    dom = pkg.landau_domain(n, dt=DT, nbiter=W + 2 * K + 2, L=L_BOX, vmax=VMAX)
    ivy0, nloc = d.partition_vy(n, ranks.world)[ranks.rank]
    ctx = pkg.Context(dom, "f32", slab=(ivy0, nloc, args.halo))
    run = d.SlabRun(ctx, DT)
    comm = d.TorchComm()
    sampler = ClockSampler(ranks.local_rank)
    sampler.start()
    ctx.init_case(run.state, v.IC_LANDAU_SUM, 0.05, 0.5)
    d.run_distributed(run, comm, W, iter0=1)  # initial field + warm-up steps
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    launches0 = v.kernel_launches()
    halo0 = comm.halo_bytes
    e0, e1 = _events(torch)
    e0.record(stream)
    d.run_distributed(run, comm, K, iter0=W + 1, start=False)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = v.kernel_launches() - launches0
    halo_bytes = (comm.halo_bytes - halo0) / K
    ctx.check()
    secs = ranks.max(e0.elapsed_time(e1) / 1e3)
    ranks.barrier()
    # End to end: this rank's planes of f0 from pinned host memory in, the
    # final planes and the diagnostic history out.
    own = ctx.owned(run.state)
    h0 = torch.empty(own.shape, dtype=torch.float32, pin_memory=True)
    h0.copy_(own)
    hout = torch.empty_like(h0, pin_memory=True)
    torch.cuda.synchronize()
    ranks.barrier()
    e0.record(stream)
    ctx.owned(run.state).copy_(h0, non_blocking=True)
    d.run_distributed(run, comm, K, iter0=1)
    hout.copy_(ctx.owned(run.state), non_blocking=True)
    nrj, _ = ctx.diags_read(K + 1)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_secs = ranks.max(e0.elapsed_time(e1) / 1e3)
    clocks = sampler.stop()
    cells = dom.cells
    fbytes = h0.numel() * 4
    ensemble = ensemble_arm(pkg, torch, stream, measured_hbm_peak()[0], ranks=ranks, autotune=False)
    line = {
        "metric": METRIC, "value": cells * K / secs / 1e9, "unit": METRIC, "n_gpus": ranks.world, "steps": K,
        "warmup": W, "ms_per_step": secs * 1e3 / K, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "api": "distrib.SlabRun over vlp4d slab contexts (C ABI), NCCL exchanges",
        "dtype": "f32", "data": "synthetic (Landau initial condition computed on the device)",
        "config": headline_config(n, ranks.world, slabs=True, halo=args.halo, rank=ranks.rank),
        "halo_bytes_per_step_per_rank": halo_bytes,
        "e2e": {"value": cells * K / e2e_secs / 1e9, "unit": METRIC, "h2d_bytes_per_step": fbytes / K,
                "d2h_bytes_per_step": (fbytes + 8 * (K + 1)) / K, "seconds": e2e_secs,
                "api": "distrib.SlabRun (C ABI, pinned host buffers, per rank)"},
        "gpu_launches": launches, "clocks": clocks,
        "energy_first_last": [float(nrj[0]), float(nrj[-1])],
        "ensemble": ensemble,
    }
    del own, h0, hout
    ctx.close()
    return line


def stage_arm(pkg, torch, stream, stage, dtype, n, calls):
    """One stage entry point on the Landau n^4 state after one field solve
    (the x/y shifts by dt/2, the v shifts by dt, as in a step), `calls`
    calls: a short, self-contained command for profiling one kernel."""
    v = pkg.vlp4d
    dom = pkg.landau_domain(n, dt=DT, nbiter=4, L=L_BOX, vmax=VMAX)
    with pkg.Context(dom, dtype) as ctx:
        a, b = ctx.empty_f(), ctx.empty_f()
        ctx.init_case(a, v.IC_LANDAU_SUM, 0.05, 0.5)
        ctx.field_rho(a)
        ctx.field_poisson()
        fn = getattr(ctx, stage)
        dt = DT if stage in ("advect_vx", "advect_vy", "advect_vxvy") else 0.5 * DT
        if stage == "field_poisson":
            call = fn
        elif stage == "field_rho":
            call = lambda: fn(a)
        else:
            call = lambda: fn(a, b, dt)
        t = time_calls(torch, stream, call, max(calls, 1))
        ctx.check()
    elem = 4 if dtype == "f32" else 8
    if stage == "field_poisson":  # rho in; phi, Ex, Ey out (FP64 planes)
        moved = 4 * n * n * 8
    else:
        moved = (1 if stage == "field_rho" else 2) * dom.cells * elem
    return {"stage": stage, "dtype": dtype, "grid": [n] * 4, "calls": calls, "ms": t * 1e3,
            "gbs": moved / t / 1e9}


ERROR_STEPS = 100


def error_arm(pkg, torch, n, nsteps=ERROR_STEPS):
    """FP32-storage error against the FP64 path over the configuration's own
    100 steps, whatever --steps is: the same initial condition and solve,
    then vlp4d_steps (the timed time loop; in FP32 its joined k_plane_xyxy
    passes) for nsteps steps in each precision, untimed.  Relative
    electric-energy error max_t |W32 - W64| / W64 (W = exp(2 nrj), the
    history of Diags::compute) and the max-norm difference of the final f."""
    import numpy as np

    v = pkg.vlp4d
    dom = pkg.landau_domain(n, dt=DT, nbiter=nsteps, L=L_BOX, vmax=VMAX)
    hist, final = {}, {}
    for dtype in ("f64", "f32"):
        with pkg.Context(dom, dtype) as ctx:
            fa, fb = ctx.empty_f(), ctx.empty_f()
            ctx.init_case(fa, v.IC_LANDAU_SUM, 0.05, 0.5)
            ctx.field_rho(fa)
            ctx.field_poisson()
            ctx.diags_compute(0)
            ctx.steps(fa, fb, 1, nsteps)
            hist[dtype] = ctx.diags_read(nsteps + 1)[0]
            final[dtype] = fb.double()
            del fa, fb
        torch.cuda.empty_cache()
    w32, w64 = np.exp(2 * hist["f32"]), np.exp(2 * hist["f64"])
    rel = np.abs(w32 - w64) / w64
    df = (final["f32"] - final["f64"]).abs().max().item()
    out = {"steps": nsteps, "api": "vlp4d_steps in both precisions",
           "energy_rel_max": float(rel.max()), "energy_rel_argmax_step": int(rel.argmax()),
           "energy_rel_final": float(rel[-1]),
           "energy_abs_max_over_wmax": float(np.abs(w32 - w64).max() / w64.max()),
           "f_maxabs": df, "f_max": final["f64"].abs().max().item()}
    del final
    torch.cuda.empty_cache()
    out["two_stream"] = two_stream_error(pkg, torch)
    return out


def two_stream_error(pkg, torch, nsteps=400):
    """The two-stream configuration (64 x 64 x 128 x 128, x, y in
    [0, 10 pi), v in [-8, 8), dt 0.05, 400 steps, f0 = (1 + 0.001 cos 0.2x +
    0.001 cos 0.2y) 1/2 [M(vx - 2.4) + M(vx + 2.4)] M(vy)): FP32 f against
    FP64 f over the whole run, vlp4d_steps in both, untimed."""
    import numpy as np

    v = pkg.vlp4d
    L = 10 * math.pi
    dom = pkg.Domain([64, 64, 128, 128], [0.0, 0.0, -8.0, -8.0], [L, L, 8.0, 8.0], 0.05, nsteps, 120)
    hist, final = {}, {}
    for dtype in ("f64", "f32"):
        with pkg.Context(dom, dtype) as ctx:
            fa, fb = ctx.empty_f(), ctx.empty_f()
            ctx.init_case(fa, v.IC_TWO_STREAM, 0.001, 0.2, 2.4)
            ctx.field_rho(fa)
            ctx.field_poisson()
            ctx.diags_compute(0)
            ctx.steps(fa, fb, 1, nsteps)
            hist[dtype] = ctx.diags_read(nsteps + 1)[0]
            final[dtype] = fb.double()
            del fa, fb
    w32, w64 = np.exp(2 * hist["f32"]), np.exp(2 * hist["f64"])
    rel = np.abs(w32 - w64) / w64
    out = {"grid": [64, 64, 128, 128], "steps": nsteps, "dt": 0.05,
           "energy_rel_max": float(rel.max()), "energy_rel_final": float(rel[-1]),
           "energy_growth": float(w64[-1] / w64[0]),
           "f_maxabs_over_fmax": float((final["f32"] - final["f64"]).abs().max() / final["f64"].abs().max())}
    del final
    torch.cuda.empty_cache()
    return out


def ensemble_arm(pkg, torch, stream, peak, nruns=256, nsteps=50, autotune=True, ranks=None):
    """The batched-ensemble configuration: 256 Landau members, N per dimension
    drawn from {16, 24, 32, 48}, amp ~ U[0.01, 0.1], k in {0.3, 0.5}, 50 steps
    of dt 0.1, FP32 f, in one persistent launch replayed from a CUDA graph.
    Tiles from the autotuner (3 steps per configuration).  Algorithmic bytes
    per cell of a run: the moment of f0 reads f once (4 B), each step's x/y
    pass (the first one alone, later ones joined with the previous step's
    closing half step) and vx/vy pass read and write it (16 B per step), and
    the closing x/y pass of the last step reads and writes it (8 B).

    With ranks over several GPUs the members are split over them
    (distrib.partition_members, no communication); the time is the slowest
    rank's and the cells are summed over the ranks."""
    import importlib

    v = pkg.vlp4d
    members = v.landau_ensemble_members(nruns)
    world = ranks.world if ranks is not None else 1
    if world > 1:
        d = importlib.import_module(pkg.__name__ + ".distrib")
        mine = d.partition_members([m.n for m in members], world)[ranks.rank]
        members = [members[i] for i in mine]
    with v.Ensemble(members, nsteps) as ens:
        tiles = ens.autotune(3) if autotune else ens.tiles()
        ens.run()  # capture
        ens.check()
        if world > 1:
            ranks.barrier()
        t = time_calls(torch, stream, lambda: ens.run(stream), 3)
        ens.check()
        cells = ens.cells
        if world > 1:
            t = ranks.max(t)
            cells = int(ranks.sum(cells))
        run_bytes = (16.0 * nsteps + 12.0) * cells
        gbs = run_bytes / t / 1e9
        return {"config": {"members": nruns, "sizes": [16, 24, 32, 48], "steps": nsteps, "dt": 0.1,
                           "amp": [0.01, 0.1], "k": [0.3, 0.5], "storage": "f32 f, f64 fields",
                           "ranks": world, "members_this_rank": len(members)},
                "cells": cells, "ms": t * 1e3, "value": cells * nsteps / t / 1e9, "unit": METRIC,
                "tiles": {"threads": tiles[0], "cols_per_tile": tiles[1], "ctas_per_sm": tiles[2]},
                "hbm": {"achieved_gbs": gbs, "frac": gbs / (peak * world), "bytes_per_run": run_bytes},
                "launches_per_run": 3}


def adjoint_arm(pkg, torch, stream, n=64, nsteps=200, every=8):
    """Reverse mode on the adjoint configuration: Landau 64^4, dt 0.1, T = 20
    (200 steps), FP32 f / FP64 fields, a checkpoint every 8 steps.  Times the
    forward run with checkpoints, the reverse run (segment recomputation
    included) and, as the forward reference, the same steps through
    vlp4d_steps; device time with CUDA events.  `store_all`: the same with
    every = 0 (the forward run keeps every step's stage input and field,
    200 x 67 MB, and the reverse run recomputes nothing)."""
    v = pkg.vlp4d
    dom = pkg.landau_domain(n, dt=0.1, nbiter=nsteps + 1, idcase=110)
    out = {"config": {"grid": [n] * 4, "dt": 0.1, "steps": nsteps, "checkpoint_every": every,
                      "storage": "f32 f, f64 fields", "objective": "dx dy sum |E(T)|^2"}}
    with pkg.Context(dom, "f32") as ctx:
        f0 = ctx.empty_f()
        ctx.init_case(f0, v.IC_LANDAU_SUM, 0.05, 0.5)
        a, b = f0.clone(), ctx.empty_f()
        ctx.field_rho(a)
        ctx.field_poisson()
        ctx.diags_compute(0)
        grad = ctx.empty_f()
        fwd_steps = time_calls(torch, stream, lambda: ctx.steps(a.clone(), b, 1, nsteps), 3)
        out["forward_steps_ms_per_step"] = fwd_steps * 1e3 / nsteps
        for ev, key in ((every, None), (0, "store_all")):
            with v.Adjoint(ctx, nsteps, ev) as adj:
                adj.forward(f0)  # warm-up (allocations, tables, graph capture)
                adj.backward(grad)
                t_fwd = time_calls(torch, stream, lambda: adj.forward(f0), 3)
                t_bwd = time_calls(torch, stream, lambda: adj.backward(grad), 3)
                J = adj.forward(f0)
            res = {
                "J": J,
                ("forward_with_checkpoints_ms_per_step" if key is None else "forward_storing_ms_per_step"):
                    t_fwd * 1e3 / nsteps,
                "backward_ms_per_step": t_bwd * 1e3 / nsteps,
                "ratio_backward_to_forward_steps": t_bwd / fwd_steps,
                ("ratio_backward_to_forward_checkpointed" if key is None else "ratio_backward_to_forward_storing"):
                    t_bwd / t_fwd,
                "grad_finite": bool(torch.isfinite(grad).all().item()),
            }
            if key is None:
                out.update(res)
            else:
                out[key] = res
            torch.cuda.empty_cache()
        del a, b, grad, f0
    torch.cuda.empty_cache()
    return out


MPI_L = 12.56637112  # wk/SLD10.dat: x, y in [0, 12.56637112), v in [-9, 9), dt 0.01


def mpi_reference_cpu(n, budget_s=20.0):
    """The reference's own OpenMP vlp4d_mpi (oracle/_ref/libvlp4d_mpi_ref.so,
    one process) on an n^4 SLD10 grid: one untimed step, then steps while
    the total stays within budget_s."""
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import MpiReference

    if not MpiReference.available():
        return None
    ref = MpiReference((n,) * 4, (0.0, 0.0, -9.0, -9.0), (MPI_L, MPI_L, 9.0, 9.0), 0.01, nbiter=64, idcase=10)
    threads = int(ref.L.refm_max_threads())
    ref.onetimestep(1)
    times = []
    for it in range(60):
        t0 = time.perf_counter()
        ref.onetimestep(2 + it)
        times.append(time.perf_counter() - t0)
        if sum(times) > budget_s:
            break
    ref.close()
    secs = sum(times)
    return {"value": n ** 4 * len(times) / secs / 1e9, "unit": METRIC, "cores": threads, "kind": "reference",
            "sample": f"{len(times)} onetimestep calls of the {n}^4 SLD10 grid (after 1 untimed), reference "
                      f"OpenMP build miniapps/vlp4d_mpi/openmp as one process, FP64, OMP_NUM_THREADS={threads}"}


def mpi_arm(pkg, torch, stream, peak, n=128, nsteps=10, warmup=3):
    """The vlp4d_mpi step (cubic splines, 4D advection) for one process on the
    geometry of its reference deck wk/SLD10.dat (128^4, x, y in
    [0, 12.566), v in [-9, 9), dt 0.01, SLD10 initial condition), FP64
    halo-extended arrays.  Times vlp4d_mpi_step (fused: four passes over f)
    and the reference-order sequence of the separate entry points (halo
    fill, spline_xy, advect_2d, field, spline_vxvy, advect_4d, field,
    diagnostics) with CUDA events."""
    dom = pkg.Domain([n] * 4, [0.0, 0.0, -9.0, -9.0], [MPI_L, MPI_L, 9.0, 9.0], 0.01, nsteps + warmup + 8, 10)
    cells = n ** 4
    with pkg.Context(dom, "f64") as ctx:
        fn, fnp1 = ctx.mpi_empty(), ctx.mpi_empty()
        ctx.mpi_init_case(fn)  # SLD10 (Init.cpp:228-247) on the device
        ctx.mpi_field(fn)
        ctx.diags_compute(0)
        ctx.mpi_l2norm(fn, 0)
        bufs = [fn, fnp1]
        it = [1]

        def one():
            ctx.mpi_step(bufs[0], bufs[1], min(it[0], dom.nbiter), stream)
            bufs.reverse()
            it[0] += 1

        for _ in range(warmup):
            one()
        torch.cuda.synchronize()
        e0, e1 = _events(torch)
        e0.record(stream)
        for _ in range(nsteps):
            one()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.check()
        t = e0.elapsed_time(e1) / 1e3 / nsteps
        finite = bool(torch.isfinite(bufs[0][3:-3, 3:-3, 3:-3, 3:-3]).all().item())
        _, _, l2 = ctx.diags_read_ext(it[0])
        # The separate entry points in the reference's order.
        tmp = ctx.mpi_empty()

        def seq():
            a = bufs[0]
            ctx.mpi_halo_fill(a, stream)
            ctx.mpi_spline_xy(a, stream)
            bufs[1].copy_(a)
            ctx.mpi_advect_2d(a, tmp, 0.005, stream)
            ctx.mpi_field(a, stream)
            ctx.mpi_spline_vxvy(bufs[1], stream)
            ctx.mpi_advect_4d(bufs[1], a, 0.01, stream)
            ctx.mpi_field(bufs[1], stream)
            ctx.diags_compute(1, stream)
            ctx.mpi_l2norm(bufs[1], 1, stream)
            bufs.reverse()

        t_seq = time_calls(torch, stream, seq, 2)
        ctx.check()
        del tmp
    torch.cuda.empty_cache()
    # FP64 bytes the four fused passes read and write once each (E = n + 6):
    # x/y: n^4 -> E^2 n^2; vx: E^2 n^2 -> E^3 n; vy: E^3 n -> E^4;
    # 4D: E^4 -> n^4.
    e = n + 6
    bytes_step = 8.0 * 2 * (n ** 4 + e * e * n * n + e ** 3 * n + e ** 4)
    return {"config": {"workload": "vlp4d_mpi one process, SLD10 deck geometry", "grid": [n] * 4, "dt": 0.01,
                       "x": [0, MPI_L], "v": [-9, 9], "storage": "f64 halo-extended (n+6)^4"},
            "ms_per_step": t * 1e3, "value": cells / t / 1e9, "unit": METRIC,
            "reference_order_entry_points_ms_per_step": t_seq * 1e3,
            "hbm_bytes_per_step_model": bytes_step, "hbm_gbs_model": bytes_step / t / 1e9,
            "finite": finite, "l2norm_first_last": [float(l2[0]), float(l2[-1])],
            "launches_per_step": 9}


# ---------------------------------------------------------------- CPU reference
def landau_f0_numpy(n):
    """The benchmark initial condition on the host, FP64, layout_left order."""
    import numpy as np

    dx = L_BOX / n
    dv = 2 * VMAX / n
    x = np.arange(n) * dx
    v = -VMAX + np.arange(n) * dv
    s = 1.0 + 0.05 * np.cos(0.5 * x)[None, :] + 0.05 * np.cos(0.5 * x)[:, None]  # (iy, ix)
    m = np.exp(-0.5 * v * v) / math.sqrt(2 * math.pi)
    out = np.empty((n, n, n, n))
    for ivy in range(n):
        out[ivy] = (m[ivy] * m)[:, None, None] * s[None, :, :]
    return out


def reference_cpu(n, max_steps, budget_s, warmup=1):
    """Times the reference's own OpenMP build (oracle/_ref) on this host:
    full Strang steps on the whole grid, `warmup` untimed steps first (at
    least one), then up to max_steps timed steps while the total stays
    within budget_s."""
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Reference

    if not Reference.available():
        return None
    warmup = max(int(warmup), 1)
    ref = Reference((n, n, n, n), (0.0, 0.0, -VMAX, -VMAX), (L_BOX, L_BOX, VMAX, VMAX), DT,
                    nbiter=max_steps + warmup + 1, idcase=10)
    f0 = landau_f0_numpy(n)
    ref.set_f(0, f0)
    del f0
    threads = int(ref.L.ref_max_threads())
    for w in range(warmup):  # the first one touches fnp1 and the FFT buffers
        ref.onetimestep(1 + w)
    times = []
    for it in range(max_steps):
        t0 = time.perf_counter()
        ref.onetimestep(1 + warmup + it)
        times.append(time.perf_counter() - t0)
        if sum(times) > budget_s:
            break
    ref.close()
    secs = sum(times)
    return {"value": n ** 4 * len(times) / secs / 1e9, "unit": METRIC, "cores": threads, "kind": "reference",
            "steps": len(times), "warmup": warmup, "seconds": secs,
            "sample": f"{len(times)} full Strang steps of the {n}^4 grid (after {warmup} untimed), "
                      f"reference OpenMP build miniapps/vlp4d/openmp, FP64, OMP_NUM_THREADS={threads}"}


REF_DECK = """grid points along x : {n}
grid points along y : {n}
grid points along vx : {n}
grid points along vy : {n}
lower bound of x : 0.
upper bound of x : {L!r}
lower bound of y : 0.
upper bound of y : {L!r}
lower bound of vx : {vmin!r}
upper bound of vx : {vmax!r}
lower bound of vy : {vmin!r}
upper bound of vy : {vmax!r}
test case : 10
time step : {dt!r}
number of steps : {steps}
diagnostic frequency : 1
write fxvx slices : 0
"""


def reference_gpu(n, steps, timeout_s=240):
    """The reference's own CUDA variant (miniapps/vlp4d/thrust, built for
    sm_100a by baseline/Makefile) on this GPU: its main() on an n^4 deck of
    the benchmark geometry (x, y in [0, 4 pi), v in [-6, 6), dt 0.1, its
    SLD10 initial condition, `steps` steps, FP64).  Throughput from its own
    MainLoop timer (host clock around each onetimestep, which synchronises
    after every stage), as the reference measures itself; its stage timers
    as ms per call."""
    import tempfile

    exe = ROOT / "baseline" / "_ref" / "vlp4d_ref_cuda"
    if not exe.exists():
        return {"unavailable": "baseline/_ref/vlp4d_ref_cuda (the reference's CUDA build) is absent"}
    with tempfile.TemporaryDirectory() as tmp:
        deck = Path(tmp) / "landau.dat"
        deck.write_text(REF_DECK.format(n=n, L=L_BOX, vmin=-VMAX, vmax=VMAX, dt=DT, steps=steps))
        try:
            out = subprocess.run([str(exe), str(deck)], cwd=tmp, capture_output=True, text=True, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"the reference's CUDA build did not finish {steps} steps within {timeout_s} s"}
        if out.returncode != 0:
            return {"unavailable": f"the reference's CUDA build exited with {out.returncode}: {out.stderr[-300:]}"}
        timers = {}
        for line in out.stdout.splitlines():
            parts = line.split()
            if len(parts) >= 5 and parts[2] == "[s]," and parts[4] == "calls":
                timers[parts[0]] = (float(parts[1]), int(parts[3]))
        nrj = []
        nrj_path = Path(tmp) / "nrj.out"
        if nrj_path.exists():
            nrj = [float(l.split()[1]) for l in nrj_path.read_text().splitlines() if l.strip()]
    if "MainLoop" not in timers or timers["MainLoop"][1] == 0:
        return {"unavailable": "the reference's CUDA build printed no MainLoop timer"}
    secs, calls = timers["MainLoop"]
    return {"value": n ** 4 * calls / secs / 1e9, "unit": METRIC, "ms_per_step": secs * 1e3 / calls,
            "steps": calls, "dtype": "f64",
            "kind": "reference CUDA variant miniapps/vlp4d/thrust (ENABLE_CUDA, Impl::for_each kernels, "
                    "thrust reductions, cuFFT), compiled from its sources for sm_100a",
            "timing": "the reference's own MainLoop timer (host clock, cudaDeviceSynchronize after each stage)",
            "stages_ms_per_call": {k: v[0] * 1e3 / v[1] for k, v in timers.items() if v[1] > 0},
            "nrj_first_last": [nrj[0], nrj[-1]] if nrj else None}


def _set_omp_env():
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_PROC_BIND", "true")


def reference_arm(args):
    _set_omp_env()
    budget = 150.0
    res = reference_cpu(args.n, max(args.steps, 1), budget, warmup=max(args.warmup, 1))
    if res is None:
        return {"impl": "reference", "unavailable": "oracle/_ref/libvlp4d_ref.so (the reference's OpenMP build) is absent"}
    ms = res["seconds"] * 1e3 / res["steps"]
    world = args.gpus
    slabs = (world > 1 and not args.replicas) or args.slab
    return {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": METRIC, "n_gpus": args.gpus,
        "steps": res["steps"], "warmup": res["warmup"], "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if slabs else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (Landau initial condition)",
        # The same config as this library's arm at the same N (the reference
        # itself is one FP64 process on the host cores: `dtype`, `cpu_baseline`).
        "config": headline_config(args.n, world, slabs=slabs, halo=args.halo),
        "requested_steps": args.steps,
        "cpu_baseline": res,
        "e2e": {"value": res["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    args = parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return 0
    if args.case != "main":
        import torch

        import __graft_entry__ as ge

        pkg = ge.load_package()
        stream = torch.cuda.current_stream()
        peak, _ = measured_hbm_peak()
        if args.case == "adjoint":
            out = adjoint_arm(pkg, torch, stream, nsteps=args.steps)
        elif args.case == "mpi":
            out = mpi_arm(pkg, torch, stream, peak, n=args.n, nsteps=args.steps, warmup=max(args.warmup, 1))
            if not args.no_cpu_baseline:
                _set_omp_env()
                out["cpu_baseline"] = mpi_reference_cpu(32)
        elif args.case == "stage":
            out = stage_arm(pkg, torch, stream, args.stage, args.dtype, args.n, args.steps)
        else:
            out = ensemble_arm(pkg, torch, stream, peak, nruns=args.members, nsteps=args.steps, autotune=False)
        print(json.dumps({"case": args.case, **out}), flush=True)
        return 0
    ranks = Ranks(world)
    try:
        use_slabs = (world > 1 and not args.replicas) or args.slab
        line = slab_arm(args, ranks) if use_slabs else gpu_arm(args, ranks)
        if rank == 0 and world == 1 and not args.no_cpu_baseline and not use_slabs:
            _set_omp_env()
            line["cpu_baseline"] = reference_cpu(args.n, 3, 20.0) or {
                "value": None, "unit": METRIC, "cores": 0, "kind": "reference", "sample": "oracle/_ref absent"}
        if rank == 0 and world == 1 and not args.no_reference_gpu and not use_slabs:
            ref = reference_gpu(args.n, 10)
            if "value" in ref:
                ref["f64_over_reference"] = line["f64"]["value"] / ref["value"] if line.get("f64") else None
                ref["f32_over_reference"] = line["value"] / ref["value"]
            line["reference_gpu"] = ref
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

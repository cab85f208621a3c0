"""Benchmark of the fused Euler step on B200.

Workload (the headline configuration): 2D Kelvin-Helmholtz, 2048^2 interior
cells, periodic, WENO5-Z + HLLC, SSPRK3, CFL 0.4, FP64, seeded synthetic
initial conditions. One bench step = one full SSPRK3 step of the grid
(3 fused stage kernels + a one-thread clock kernel), driven on the device
(mc_advance: dt, the clock and the output clamp never leave the GPU).

Prints one JSON line (rank 0). Metric: zone-updates/s = interior cells x
steps / time. With --gpus N (one process per GPU under torchrun) the problem
is a 2048 x 2048N stack of the KH layer split along y, 2048^2 cells per
rank (weak scaling), in the device-driven loop: after every stage each rank
exchanges its 3 edge rows with its neighbours and every step's dt is the
global CFL minimum, both issued by the library in the stream (NCCL
send/recv and all-reduce MIN, mc_set_slab_decomposition); --decomp
replicas runs an independent 2048^2 problem per rank instead. The timed region is
bracketed by a barrier and device synchronisation and the time is the
maximum over ranks.

--impl reference times the reference's own CPU implementation of the same
step (the reference's hot-path sources compiled against the host shim,
oracle/_ref; the C restatement oracle/liboracle_port.so if that build is
absent) with every host thread, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s"
UNIT = "zone-updates/s"
N_CELLS_SIDE = 2048
WORKLOAD = "kelvin_helmholtz_2d_2048x2048_weno5z_hllc_ssprk3_fp64"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_CELLS_SIDE, help="cells per side (default 2048)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--workload", default="kh2d", choices=["kh2d", "sedov3d", "batch", "adjoint"],
                    help="kh2d: the headline line; sedov3d and batch print their own lines")
    ap.add_argument("--solver", default="hllc", choices=["hllc", "rusanov"], help="batch workload solver")
    ap.add_argument("--fd-directions", type=int, default=64, help="adjoint workload: finite-difference checks")
    ap.add_argument("--problems", type=int, default=4096, help="batch workload: number of problems (half 1D, half 2D)")
    ap.add_argument("--decomp", default="auto", choices=["auto", "slab", "replicas"],
                    help="kh2d: one problem split along y with halo exchange (slab; auto = slab when --gpus > 1) "
                         "or an independent problem per GPU (replicas)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="batch workload: keep the default schedule (no autotuner)")
    ap.add_argument("--no-extras", action="store_true",
                    help="kh2d at N=1: skip the FP32 form, Sedov 512^3, batch and adjoint measurements "
                         "that the default run adds to the line under 'forms'")
    return ap.parse_args()


def config(n, precision, world, decomp="auto"):
    c = {"workload": WORKLOAD if (n == N_CELLS_SIDE and precision == "fp64") else
         f"kelvin_helmholtz_2d_{n}x{n}_weno5z_hllc_ssprk3_{precision}",
         "grid": f"{n}x{n}", "ghost_cells": 3, "vars": 4, "reconstruction": "weno5z",
         "riemann_solver": "hllc", "time_stepper": "ssprk3", "cfl": 0.4, "gamma": 5.0 / 3.0,
         "boundaries": "periodic", "per_rank_problem": f"{n}x{n} cells per GPU",
         "parallelism": "one GPU",
         "l2": "inputs larger than L2 (state 135 MB; each step streams ~400 MB), no flush"}
    if decomp == "slab" or (decomp == "auto" and world > 1):
        c["grid"] = f"{n}x{n * world} (KH layer stacked {world}x in y)"
        c["parallelism"] = (f"slab decomposition along y over {world} GPUs, device-driven loop: ghost-row exchange "
                            f"after every stage (NCCL send/recv) and global CFL minimum (NCCL all-reduce MIN) "
                            f"issued by the library in the stream")
    elif world > 1:
        c["parallelism"] = f"independent {n}x{n} problems x{world}"
    return c


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_profile_value(key):
    """A figure of the committed ncu summary of the headline stage kernel
    (a line `key: value ...`)."""
    path = os.path.join(ROOT, "profiles", "stage2d_weno5z_hllc_kh2048_ncu.md")
    try:
        for ln in open(path):
            if ln.startswith(key + ":"):
                return float(ln.split(":")[1].split()[0])
    except OSError:
        pass
    return None


def ncu_traffic_per_launch():
    """DRAM bytes per stage-kernel launch from the committed ncu summary."""
    return ncu_profile_value("traffic_bytes_per_launch")


# ---------------------------------------------------------------------------
# CPU side: the reference's own implementation
# ---------------------------------------------------------------------------
def cpu_oracle_kind():
    from oracle import oracle as O
    return "reference" if os.path.exists(O.LIB_PATHS["reference"]) else "port"


def cpu_run(n, steps, warmup, budget_s=None):
    """Time SSPRK3 steps of the KH problem on the host; returns (cells*steps/s, steps, seconds, kind, cores)."""
    from oracle import oracle as O
    from mosscap_b200 import problems as P
    kind = cpu_oracle_kind()
    cores = os.cpu_count() or 1
    p = P.kelvin_helmholtz_2d(n, seed=0)
    s = O.OracleSim(O.OracleConfig(**p.scheme_fields()), kind, threads=cores)
    s.set_Q(p.Q)
    s.fill_bcs()
    for _ in range(warmup):
        s.run(1)
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        s.run(1)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return n * n * done / dt, done, dt, kind, cores


def cpu_baseline_subprocess(n, budget_s):
    """The CPU baseline timed in a process of its own (no CUDA context, no
    clock sampler beside it), so that its OpenMP threads have the host cores
    to themselves; returns the cpu_baseline object."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "v, done, secs, kind, cores = bench.cpu_run(%d, 1000, 1, budget_s=%r); "
            "print(json.dumps([v, done, secs, kind, cores]))") % (ROOT, n, float(budget_s))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return {"error": r.stderr.strip().splitlines()[-1] if r.stderr.strip() else f"rc {r.returncode}"}
    v, done, secs, kind, cores = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{done} full SSPRK3 steps of the {n}x{n} problem ({secs:.1f} s, {cores} threads, "
                      f"in a CPU-only child process after the GPU work)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.n
    # a bounded sample: at most K steps and at most ~2 minutes of CPU work
    value, done, secs, kind, cores = cpu_run(n, args.steps, min(args.warmup, 2), budget_s=120.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * secs / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(n, "fp64", 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"{done} full SSPRK3 steps of the {n}x{n} problem on {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    from mosscap_b200 import problems as P
    from mosscap_b200.hydro import HydroSim

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.n
    p = P.kelvin_helmholtz_2d(n, seed=rank)
    cells = n * n
    slab = None
    use_slab = args.decomp == "slab" or (args.decomp == "auto" and world > 1)
    if use_slab:
        # one n x (n * world) periodic layer stack split along y: rank r owns
        # rows [r n, (r + 1) n), a unit-square copy of the KH layer (continuous
        # across slabs, since the layer is periodic in y); ghost rows come from
        # the neighbours after every stage and dt is the global CFL minimum,
        # both by the library's own NCCL calls in the stream
        from mosscap_b200.distributed import SlabSim
        slab = SlabSim(p, rank, world, precision=args.precision, device=dev, is_slab=True, transport="library")
        sim = slab.sim
        slab.fill_bcs()

        def advance(k):
            # device-driven loop: ghost rows and the global CFL minimum are
            # exchanged in-stream by the library
            return len(slab.advance(k)) if k else 0
    else:
        sim = HydroSim(p, precision=args.precision, device=dev)
        sim.fill_bcs()

        def advance(k):
            return len(sim.advance(k, log_dt=False)) if k else 0
    if args.warmup:
        advance(args.warmup)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # ---- timed region: K device-driven steps -----------------------------
    phys = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    gpu_index = int(phys[local]) if len(phys) > local and phys[local].strip().isdigit() else local
    sampler = ClockSampler(gpu_index)
    barrier()
    sampler.start()
    time.sleep(0.3)
    launches0 = sim.launch_count()
    sim.profile_stages(True)
    e0.record(stream)
    steps_done = advance(args.steps)
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    stage_ms, stage_n = sim.stage_time(0)
    sim.profile_stages(False)
    launches = sim.launch_count() - launches0
    ms_max = max_over_ranks(ms)
    assert steps_done == args.steps, "the device loop stopped early"
    value = world * cells * args.steps / (ms_max / 1e3)
    flags = sim.status()

    # roofline of the dominant kernel (the fused stage kernel): algorithmic
    # bytes per launch = the stage's state reads and writes, (3s-1) n_var 8 B
    # per cell per step spread over s = 3 launches
    nvar = 4
    alg_bytes_per_launch = cells * (3 * 3 - 1) * nvar * 8 / 3.0
    avg_launch_ms = stage_ms / max(stage_n, 1)
    achieved = alg_bytes_per_launch / (avg_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    # the committed ncu traffic figure is that of the FP64 kernel
    traffic = ncu_traffic_per_launch() if args.precision == "fp64" else None
    kname = "stage2d_kernel<WENO5Z,HLLC,f64>" if args.precision == "fp64" else "stage2d_kernel<WENO5Z,HLLC,f32>"
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind, "kernel": kname,
                "alg_bytes_per_launch": alg_bytes_per_launch, "avg_launch_ms": avg_launch_ms,
                "launches_timed": stage_n}
    if args.precision == "fp64":
        # the bound the exact FP64 kernel actually meets: the FP64 pipe
        # (IEEE divisions and square roots in the reference's order); its
        # activity from the committed ncu capture of the same kernel
        fp64_active = ncu_profile_value("fp64_pipe_active_frac")
        roofline["compute"] = {"bound": "fp64 pipe", "active_frac_ncu": fp64_active,
                               "source": "profiles/stage2d_weno5z_hllc_kh2048_ncu.md"}

    # the density after warmup + K steps, for the FP32 form's error
    rho64 = None
    if rank == 0 and world == 1 and not args.no_extras and args.precision == "fp64":
        ng = p.ng
        rho64 = sim.Q[0, 0, ng:-ng, ng:-ng].clone()

    # ---- end to end through the C ABI with host buffers --------------------
    e2e = None
    if not args.no_e2e:
        import ctypes
        K = min(args.steps, 20) or 1
        host = torch.empty(sim.Q.shape, dtype=torch.float64, pin_memory=True)
        host.copy_(sim.Q)
        qbytes = host.numel() * 8

        def serial_step():
            sim.Q.copy_(host, non_blocking=True)
            if slab is not None:
                slab.step()                # global dt read back on the host, then the step
            else:
                dt = sim.compute_dt()      # dt back on the host, like the reference hook
                sim.time_step(dt)
            host.copy_(sim.Q, non_blocking=True)
            torch.cuda.synchronize(dev)

        def timed(step):
            # warm-up calls first: the first call of an entry point loads its
            # kernels' module and creates its streams
            for _ in range(2):
                step()
            barrier()
            t0 = time.perf_counter()
            for _ in range(K):
                step()
            barrier()
            return max_over_ranks(time.perf_counter() - t0)

        secs_serial = timed(serial_step)
        if slab is None:
            # mc_step_host: the same copies and step in one call, the copies
            # overlapping the step
            secs = timed(lambda: sim.step_host(host))
            how = ("per step: mc_step_host on a pinned-host state (state -> device band by band with stage 0's "
                   "fluxes computed behind it, dt on the device, the step, the last stage band by band with each "
                   "band's rows copied back behind it), dt read back, synchronize")
        else:
            secs = secs_serial
            how = ("per step: pinned-host state -> device, global dt (mc_compute_dt with the slab all-reduce, read "
                   "back), mc_time_step, state -> pinned host, synchronize")
        e2e = {"value": world * cells * K / secs, "unit": UNIT, "h2d_bytes_per_step": qbytes,
               "d2h_bytes_per_step": qbytes + 8, "how": how,
               "serial_calls_value": world * cells * K / secs_serial,
               "serial_calls_how": "per step: pinned-host state -> device, mc_compute_dt (dt read back), "
                                   "mc_time_step, state -> pinned host, synchronize"}

    # ---- the other forms, measured in this run (rank 0, N = 1) ------------
    extras = None
    if rank == 0 and world == 1 and not args.no_extras and args.precision == "fp64":
        extras = run_extras(args, rho64, value)
        rho64 = None

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_subprocess(n, budget_s=15.0)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
                "data": "synthetic", "config": config(n, args.precision, world, args.decomp), "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
                "status_flags": int(flags)}
        if extras is not None:
            line["forms"] = extras
        print(json.dumps(line), flush=True)
    if slab is not None:
        # the library's own NCCL communicator goes first, on every rank, with
        # no work in flight, and only then torch's process group
        torch.cuda.synchronize(dev)
        slab.sim.close()
    del sim
    if world > 1:
        dist.destroy_process_group()


def measure_sedov(n, precision, steps, warmup):
    """3D Sedov blast n^3 (5 vars, PPM + HLL, SSPRK3, CFL 0.8/3): K
    device-driven steps with inputs resident; returns a dict."""
    import torch
    from mosscap_b200 import problems as P
    from mosscap_b200.hydro import HydroSim
    p = P.sedov_3d(n).with_scheme(max_time=1e30, output_delta=1e30)
    sim = HydroSim(p, precision=precision)
    p.Q = None
    sim.fill_bcs()
    sim.advance(warmup, log_dt=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    sim.profile_stages(True)
    e0.record()
    done = len(sim.advance(steps, log_dt=False))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    plane_ms, plane_n = sim.stage_time(0)
    z_ms, z_n = sim.stage_time(1)
    sim.profile_stages(False)
    flags = sim.status()
    sim.close()
    del sim
    torch.cuda.empty_cache()
    cells = n ** 3
    alg = cells * (3 * 3 - 1) * 5 * 8 / 3.0  # per stage, both passes together
    peak, kind = measured_peak_hbm()
    stage_ms = (plane_ms + z_ms) / max(plane_n, 1)
    achieved = alg / (stage_ms / 1e3) / 1e9
    return {"workload": f"sedov_3d_{n}^3_ppm_mc_hll_ssprk3_cfl0.267_{precision}", "value": cells * done / (ms / 1e3),
            "unit": UNIT, "steps": done, "warmup": warmup, "ms_per_step": ms / max(done, 1),
            "dtype": "f64" if precision == "fp64" else "f32+f64",
            "kernels": {"plane_pass_ms_avg": plane_ms / max(plane_n, 1), "z_pass_ms_avg": z_ms / max(z_n, 1)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": kind,
                         "alg_bytes_per_stage": alg,
                         "note": "algorithmic state bytes per stage / (plane pass + z pass) time"},
            "status_flags": int(flags)}


def run_sedov(args):
    """3D Sedov blast, 512^3 (5 vars, PPM + HLL, SSPRK3): K device-driven steps."""
    n = args.n if args.n != N_CELLS_SIDE else 512
    r = measure_sedov(n, args.precision, args.steps, args.warmup)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["steps"],
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "dtype": r["dtype"], "data": "synthetic", "config": {"workload": r["workload"]},
            "kernels": r["kernels"], "roofline": r["roofline"], "status_flags": r["status_flags"]}
    print(json.dumps(line), flush=True)


def measure_batch(problems, precision, steps, warmup, tune=True):
    """Batched independent problems (one persistent launch per stage, or
    the split form where the autotuner measures it faster; graph-replayed
    steps, autotuned schedule); returns a dict."""
    import torch
    from mosscap_b200.hydro import BatchSim
    cells = sum(p.interior_cells for p in problems)
    b = BatchSim(problems, precision=precision)
    b.fill_bcs()
    t0 = time.perf_counter()
    sched = b.tune() if tune else b.schedule()
    tune_s = time.perf_counter() - t0
    b.advance(warmup)
    _, k0, _ = b.clocks()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    b.advance(steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    _, nsteps, status = b.clocks()
    updates = sum(p.interior_cells * int(k - k_) for p, k, k_ in zip(problems, nsteps, k0))
    b.close()
    del b
    torch.cuda.empty_cache()
    return {"value": updates / (ms / 1e3), "unit": UNIT, "steps": steps, "warmup": warmup,
            "ms_per_step": ms / max(steps, 1), "dtype": "f64" if precision == "fp64" else "f32+f64",
            "problems": len(problems), "interior_cells": cells, "schedule": sched, "tune_s": tune_s,
            "problems_flagged": int((status != 0).sum())}


def run_batch(args):
    """Batched independent Riemann problems: 2048 1D (64..4096 cells) and 2048
    2D quadrant problems (64^2..512^2), MUSCL / minmod, rk2, own dt each.
    With N ranks the problems are split by cost (interior cells) over the
    ranks, which share no data; the value is all ranks' zone updates over
    the slowest rank's time (strong scaling: the batch is fixed)."""
    import torch
    from mosscap_b200 import problems as P
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    half = max(args.problems // 2, 1)
    probs = P.riemann_batch(seed=0, n1d=half, n2d=half, riemann_solver=args.solver)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        from mosscap_b200.distributed import partition_by_cost
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        mine = partition_by_cost([p.interior_cells for p in probs], world)[rank]
        probs = [probs[k] for k in mine]
        dist.barrier()
    r = measure_batch(probs, args.precision, args.steps, args.warmup, tune=not args.no_tune)
    if world > 1:
        t = torch.tensor([r["ms_per_step"], r["value"] * r["ms_per_step"]], dtype=torch.float64, device="cuda")
        tm = t[:1].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        # all ranks' updates per step over the slowest rank's step time
        r["value"] = float(t[1].item()) / float(tm.item())
        r["ms_per_step"] = float(tm.item())
        r["problems"] = args.problems
        dist.destroy_process_group()
        if rank != 0:
            return
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
            "dtype": r["dtype"], "data": "synthetic",
            "scaling": "strong",
            "config": {"workload": f"riemann_batch_{half}x1d_{half}x2d_muscl_minmod_{args.solver}_rk2_{args.precision}",
                       "problems": r["problems"], "interior_cells": r["interior_cells"], "schedule": r["schedule"],
                       "parallelism": "one GPU" if world == 1 else
                       f"problems split by cost (interior cells) over {world} GPUs, no data exchange"},
            "problems_flagged": r["problems_flagged"]}
    print(json.dumps(line), flush=True)


def measure_adjoint(n, steps, fd_directions, warmup=3, checkpoint_every=20, tlm_directions=0, eps_ladder=False):
    """Adjoint of KH n^2 (WENO5-Z + HLLC, SSPRK3, FP64): the gradient of
    J = 1/2 |rho - rho_target|^2 with respect to the initial vy field and
    gamma through the autograd wrapper, the adjoint : forward cost ratio of
    the C ABI calls (CUDA events on the launching stream, mean of 3
    repetitions after warm-up), the gradient against the tangent-linear model
    on tlm_directions random directions and against central finite
    differences on the first fd_directions of them (with eps_ladder, the
    finite-difference misses re-run over a ladder of steps). Returns a dict."""
    import ctypes
    import torch
    from mosscap_b200 import problems as P
    from mosscap_b200 import capi
    from mosscap_b200.adjoint import EulerSteps, _Runner, kh_initial_state, kh_vy, pad_periodic
    p = P.kelvin_helmholtz_2d(n, seed=0)
    pt = P.kelvin_helmholtz_2d(n, seed=1)
    dev = torch.device("cuda")
    with torch.no_grad():
        gt = torch.tensor(pt.gamma, dtype=torch.float64, device=dev)
        vyt = torch.tensor(kh_vy(pt), device=dev)
        rho_t = EulerSteps.apply(kh_initial_state(vyt, gt, pt), gt, pt, steps, 1 << 30)[0].clone()
    # gradient through the autograd wrapper (the user-facing call)
    vy = torch.tensor(kh_vy(p), device=dev, requires_grad=True)
    g = torch.tensor(p.gamma, dtype=torch.float64, device=dev, requires_grad=True)
    q = EulerSteps.apply(kh_initial_state(vy, g, p), g, p, steps, checkpoint_every)
    J = 0.5 * ((q[0] - rho_t) ** 2).sum()
    J.backward()
    # cost: the C ABI calls on one mc_adjoint whose buffers a warm-up pass
    # allocated; forward = mc_adjoint_forward (K steps with checkpoints),
    # adjoint = mc_adjoint_backward (segment recompute + reverse sweep)
    runner = _Runner(p, p.gamma, checkpoint_every)
    ng = p.ng
    with torch.no_grad():
        q0 = pad_periodic(kh_initial_state(vy.detach(), g.detach(), p), ng)
    stream = runner.stream()

    def one(rec=None):
        qq = q0.clone()
        if rec:
            rec[0].record()
        runner.forward(qq, steps)
        if rec:
            rec[1].record()
        lam = torch.zeros_like(qq)
        lam[0, 0, ng:-ng, ng:-ng] = qq[0, 0, ng:-ng, ng:-ng] - rho_t
        if rec:
            rec[2].record()
        capi.check(runner.lib.mc_adjoint_backward(runner.h, ctypes.c_void_p(lam.data_ptr()), None, stream),
                   "mc_adjoint_backward")
        if rec:
            rec[3].record()

    for _ in range(max(warmup, 3)):
        one()
    reps = 3
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(reps)]
    torch.cuda.synchronize()
    for r in range(reps):
        one(ev[r])
    torch.cuda.synchronize()
    fwd = sum(x[0].elapsed_time(x[1]) for x in ev) / reps
    bwd = sum(x[2].elapsed_time(x[3]) for x in ev) / reps
    # random unit directions of (vy, gamma): the adjoint gradient against the
    # tangent-linear model (mc_tangent_linear, forward-mode dual numbers
    # through the forward arithmetic) on every direction, and against
    # central finite differences on the first fd_directions of them
    from mosscap_b200.adjoint import kh_directional_derivatives
    gvy, gg = vy.grad.detach(), g.grad.item()
    rng = np.random.default_rng(2)
    ndir = max(fd_directions, tlm_directions)
    dirs, dgs = [], []
    for _ in range(ndir):
        dvy = torch.tensor(rng.standard_normal((n, n)), device=dev)
        dirs.append(dvy / dvy.norm())
        dgs.append(float(rng.standard_normal()) * 1e-2)
    ads = np.array([float((gvy * d).sum()) + gg * dg for d, dg in zip(dirs, dgs)])

    def rel(a, b):
        return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)

    tlm_check = None
    tls = None
    if tlm_directions:
        t0 = time.perf_counter()
        tls = []
        for c0 in range(0, tlm_directions, 16):
            c1 = min(c0 + 16, tlm_directions)
            Jt, dJ = kh_directional_derivatives(p, vy.detach(), p.gamma, torch.stack(dirs[c0:c1]), dgs[c0:c1],
                                                rho_t, steps)
            tls.extend(dJ)
        tls = np.array(tls)
        r = rel(ads[:tlm_directions], tls)
        tlm_check = {"directions": tlm_directions, "max_rel_err": float(r.max()), "median_rel_err": float(np.median(r)),
                     "n_within_1e-5": int((r <= 1e-5).sum()), "n_within_1e-8": int((r <= 1e-8).sum()),
                     "loss_rel_diff": abs(Jt - J.item()) / J.item(), "seconds": time.perf_counter() - t0,
                     "how": "mc_tangent_linear: dual numbers (4 directions per pass) through the forward arithmetic, "
                            "branches as the forward run takes them"}

    def final_rho(vy_, g_):
        with torch.no_grad():
            gt_ = torch.tensor(g_, dtype=torch.float64, device=dev)
            return EulerSteps.apply(kh_initial_state(vy_, gt_, p), gt_, p, steps, 1 << 30)[0]

    def cdiff(dvy, dg, eps):
        rp = final_rho(vy.detach() + eps * dvy, p.gamma + eps * dg)
        rm = final_rho(vy.detach() - eps * dvy, p.gamma - eps * dg)
        return float((0.5 * (rp - rm) * (rp + rm - 2.0 * rho_t)).sum()) / (2 * eps)

    fds = np.array([cdiff(dirs[k], 0.0, 1e-7) + cdiff(0.0 * dirs[k], dgs[k], 1e-6) for k in range(fd_directions)])
    fd_check = {"directions": fd_directions, "eps": {"vy": 1e-7, "gamma": 1e-6},
                "direction": "unit vy field, gamma 1e-2 N(0,1)"}
    if fd_directions:
        r = rel(fds, ads[:fd_directions])
        fd_check.update({"max_rel_err": float(r.max()), "median_rel_err": float(np.median(r)),
                         "n_within_1e-5": int((r <= 1e-5).sum()),
                         "aggregate_rel_err": float(np.linalg.norm(fds - ads[:fd_directions]) /
                                                    np.linalg.norm(ads[:fd_directions])),
                         "max_abs_err": float(np.abs(fds - ads[:fd_directions]).max())})
        if tls is not None and tlm_directions >= fd_directions:
            fd_check["max_abs_err_vs_tlm"] = float(np.abs(fds - tls[:fd_directions]).max())
        if eps_ladder:
            # the directions FD misses by more than 1e-5: the vy part's
            # absolute error against the tangent-linear value over a ladder of
            # steps, which shows the FD noise floor (roundoff below ~1e-7,
            # kinks of the CFL arg-min and of the branches above)
            ladder = []
            ref = tls if tls is not None else ads
            for k in np.nonzero(r > 1e-5)[0]:
                dg_part = cdiff(0.0 * dirs[k], dgs[k], 1e-6)
                errs = {f"{e:g}": abs(cdiff(dirs[k], 0.0, e) + dg_part - float(ref[k]))
                        for e in (1e-8, 1e-7, 1e-6, 1e-5, 1e-4)}
                ladder.append({"direction": int(k), "derivative": float(ref[k]), "abs_err_by_eps": errs,
                               "min_abs_err": min(errs.values()),
                               "min_rel_err": min(errs.values()) / max(abs(float(ref[k])), 1e-300)})
            fd_check["eps_ladder"] = ladder
    out = {"workload": f"kh_2d_{n}x{n}_weno5z_hllc_ssprk3_adjoint_ckpt{checkpoint_every}", "steps": steps,
           "adjoint_forward_ratio": bwd / fwd, "forward_ms": fwd, "backward_ms": bwd,
           "forward_zone_updates_per_s": n * n * steps / (fwd / 1e3),
           "loss": J.item(), "dgamma": g.grad.item(), "grad_vy_norm": vy.grad.norm().item(),
           "fd_check": fd_check, "tlm_check": tlm_check}
    del runner
    torch.cuda.empty_cache()
    return out


def run_adjoint(args):
    """Adjoint of KH 512^2 (WENO5-Z + HLLC, SSPRK3, FP64): forward run of K
    steps with checkpoints every 20, then the reverse sweep; reports the
    adjoint : forward cost ratio and a finite-difference check of the
    gradient along --fd-directions random directions."""
    n = args.n if args.n != N_CELLS_SIDE else 512
    r = measure_adjoint(n, args.steps, args.fd_directions, args.warmup, tlm_directions=args.fd_directions,
                        eps_ladder=True)
    line = {"metric": "adjoint:forward cost", "value": r["adjoint_forward_ratio"], "unit": "ratio", "n_gpus": 1,
            "steps": args.steps, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": r["workload"], "loss": "1/2 |rho - rho_target|^2",
                       "gradient": "initial vy field and gamma"}}
    line.update({k: v for k, v in r.items() if k not in ("workload", "steps", "adjoint_forward_ratio")})
    print(json.dumps(line), flush=True)


def measure_kh_form(n, precision, steps, warmup, rho_ref=None):
    """KH n^2 in the given precision form, device-driven loop with inputs
    resident; the density after warmup + steps steps is compared with
    rho_ref (the FP64 run's after the same number of steps), if given."""
    import torch
    from mosscap_b200 import problems as P
    from mosscap_b200.hydro import HydroSim
    p = P.kelvin_helmholtz_2d(n, seed=0)
    sim = HydroSim(p, precision=precision)
    sim.fill_bcs()
    sim.advance(warmup, log_dt=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    sim.profile_stages(True)
    e0.record()
    done = len(sim.advance(steps, log_dt=False))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    stage_ms, stage_n = sim.stage_time(0)
    sim.profile_stages(False)
    out = {"value": n * n * done / (ms / 1e3), "unit": UNIT, "steps": done, "warmup": warmup,
           "ms_per_step": ms / max(done, 1), "stage_ms_avg": stage_ms / max(stage_n, 1),
           "status_flags": int(sim.status())}
    if rho_ref is not None:
        ng = p.ng
        rho = sim.Q[0, 0, ng:-ng, ng:-ng]
        d = (rho - rho_ref).abs()
        out["density_rel_l1_vs_fp64"] = float(d.sum() / rho_ref.abs().sum())
        out["density_rel_linf_vs_fp64"] = float(d.max() / rho_ref.abs().max())
        out["error_after_steps"] = warmup + done
    sim.close()
    return out


def run_extras(args, rho64, value64):
    """The forms beside the headline, measured in the same run (1 GPU):
    the FP32 compute form on the headline problem, Sedov 512^3 in FP64 and
    FP32, the 4096-problem batch in FP64 and FP32, and the adjoint at 512^2
    for a reduced step count. Each failure is recorded, not raised."""
    import torch
    from mosscap_b200 import problems as P
    ex = {}

    def guarded(name, fn):
        t0 = time.perf_counter()
        try:
            ex[name] = fn()
        except Exception as e:  # recorded in the line; the headline stands
            ex[name] = {"error": f"{type(e).__name__}: {e}"}
        ex[name]["wall_s"] = round(time.perf_counter() - t0, 2)
        torch.cuda.empty_cache()

    def fp32():
        r = measure_kh_form(args.n, "fp32", args.steps, args.warmup, rho_ref=rho64)
        r["speedup_vs_fp64"] = r["value"] / value64
        r["workload"] = f"kelvin_helmholtz_2d_{args.n}x{args.n}_weno5z_hllc_ssprk3_fp32_form"
        return r

    guarded("fp32_form", fp32)

    def sedov():
        steps = max(2, min(args.steps, 5))
        r64 = measure_sedov(512, "fp64", steps, 1)
        r32 = measure_sedov(512, "fp32", steps, 1)
        r64["fp32_form"] = {"value": r32["value"], "ms_per_step": r32["ms_per_step"],
                            "kernels": r32["kernels"], "status_flags": r32["status_flags"],
                            "speedup_vs_fp64": r32["value"] / r64["value"]}
        return r64

    guarded("sedov3d", sedov)

    def batch():
        probs = P.riemann_batch(seed=0, n1d=2048, n2d=2048, riemann_solver="hllc")
        steps = max(3, min(args.steps, 10))
        r = {"workload": "riemann_batch_2048x1d_2048x2d_muscl_minmod_hllc_rk2",
             "fp64": measure_batch(probs, "fp64", steps, 2),
             "fp32": measure_batch(probs, "fp32", steps, 2)}
        r["fp32_speedup"] = r["fp32"]["value"] / r["fp64"]["value"]
        return r

    guarded("batch", batch)

    def adjoint():
        # the full configuration: 512^2, 400 steps, checkpoints every 20;
        # the gradient against the tangent-linear model on 64 directions
        # and against finite differences on 8 of them
        return measure_adjoint(512, 400, 8, tlm_directions=64)

    guarded("adjoint", adjoint)
    return ex


def main():
    args = parse()
    if args.impl != "reference" and args.workload == "adjoint":
        run_adjoint(args)
        return
    if args.impl != "reference" and args.workload == "sedov3d":
        run_sedov(args)
        return
    if args.impl != "reference" and args.workload == "batch":
        run_batch(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

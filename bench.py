#!/usr/bin/env python
"""Benchmark of the Parareal T2S4 CC-CFV solver on B200.

Workload (default): periodic unit square, solid-body rotation
u = -2 pi (y - 1/2), v = 2 pi (x - 1/2), nu = 1e-3, Gaussian hump sigma 0.05
at (0.5, 0.75), T = 1 (one revolution), N^2 = 2048^2 cells, fine dt at
CFL ~0.8 (Nt = 4N), 64 time slices, coarse dt = 8 x fine, Parareal iterated
to a relative update < 1e-10 (or the iteration cap).  One benchmark step is
one full Parareal solve; the metric is the effective rate N^2 * Nt / time
(cell-updates/s of the serial fine solve that Parareal replaces).

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank solves its own instance
(instances are independent: weak scaling, no collective on the data path);
the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "parareal-cc-cfv-split-gpu_b200"
sys.path.insert(0, str(PKG))

BYTES_PER_FINE_CELL_SWEEP = 16  # FP64: 8 B read + 8 B written per cell per sweep


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-device", default="cpu", choices=["cpu", "gpu"],
                    help="reference arm: the oracle port on the host cores (cpu) or the "
                         "reference binary's own GPU step (gpu)")
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--nu", type=float, default=1e-3,
                    help="diffusivity of the plain / step workload (1e-3: the benchmark)")
    ap.add_argument("--slices", type=int, default=64)
    ap.add_argument("--ratio", type=int, default=8)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--kmax", type=int, default=24)
    ap.add_argument("--coarse", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--form", default="delta", choices=["standard", "delta"])
    ap.add_argument("--cpu-sample-s", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="plain",
                    choices=["plain", "batch", "serve", "step", "split", "dist"],
                    help="plain: one instance (default workload); batch: a mixed batch of "
                         "instances in shared launches; serve: Poisson arrivals through the "
                         "continuous-batching server; step: serial fine time-stepping of the "
                         "workload's field (the sweep kernels alone); split: the precision-split "
                         "case (swirl, 128 slices): FP32 vs FP64 coarse against the serial "
                         "fine; dist: the slice-distributed solve (the default for N > 1) "
                         "also on one GPU")
    ap.add_argument("--inner", type=int, default=16,
                    help="step mode: fine steps per timed step")
    ap.add_argument("--vel", default="rotation", choices=["rotation", "swirl", "compat"],
                    help="step mode: the workload's rotation field, the swirling deformation "
                         "(per-cell feet), or the reference's own setting (compat boundaries)")
    ap.add_argument("--noalloc", action="store_true",
                    help="step mode: through the allocation-free entry point")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--serve-nmax", type=int, default=1024,
                    help="serve: largest grid side of the requests (log-uniform from 128)")
    ap.add_argument("--multi", default="dist", choices=["dist", "instances"],
                    help="N > 1 GPUs: dist = one Parareal solve with its time slices spread "
                         "over the ranks (ccfv.dist, NCCL; strong scaling); instances = an "
                         "independent solve per rank (weak scaling)")
    ap.add_argument("--no-batch-serve", action="store_true",
                    help="plain mode: leave out the batched and served sub-measurements")
    ap.add_argument("--seed", type=int, default=20261206)
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="instances solved one at a time (FP64 coarse) for the plain rate "
                         "(0: all; the solve times are heavy-tailed, so a sample is noisy)")
    ap.add_argument("--coarse-theta", default="auto",
                    help="batch/serve: diffusion weight of the coarse steps ('auto': the "
                         "damping rule, 'cn': Crank-Nicolson as the reference, or a value "
                         "in [0.5, 1]); the plain rate always uses Crank-Nicolson")
    return ap.parse_args()


def coarse_theta_arg(a):
    import ccfv
    if a.coarse_theta == "auto":
        return ccfv.COARSE_THETA_AUTO
    if a.coarse_theta == "cn":
        return 0.5
    return float(a.coarse_theta)


def workload(a):
    N = a.n
    nt = 4 * N
    return dict(N=N, T=1.0, nt=nt, slices=a.slices, ratio=a.ratio, tol=a.tol, kmax=a.kmax,
                nu=a.nu, omega=2 * np.pi, center=(0.5, 0.5), hump=(0.5, 0.75), sigma=0.05)


def workload_name(w, a):
    return (f"periodic unit square {w['N']}^2, solid-body rotation (one revolution, T=1), "
            f"nu={w['nu']}, Gaussian sigma={w['sigma']} at {w['hump']}, Nt={w['nt']} fine steps, "
            f"{w['slices']} slices, coarse dt = {w['ratio']} x fine ({a.coarse} coarse, {a.form} "
            f"form), Parareal to relative update < {w['tol']:g} (cap {w['kmax']})")


def initial_field(w, solver, device):
    """Cell averages (3x3 Simpson, as T2S4_Parareal.cu:118-140) of the
    Gaussian hump with its periodic images, computed on the device by
    ccfv_gaussians; synthetic input data."""
    import torch
    N = w["N"]
    C = torch.empty(N, N, dtype=torch.float64, device=device)
    solver.gaussians(C, [[w["hump"][0], w["hump"][1], 2.0 * w["sigma"] ** 2, 1.0]], images=1)
    return C


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines: list[str] = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons, pw = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                pw.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(mx),
                "power_w_max": max(pw) if pw else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def spawn_ranks(a):
    """--gpus N > 1 without a launcher: start N ranks on this node through
    torch.distributed.run (rendezvous on 127.0.0.1) and return its exit
    code; NCCL's initialisation log stays on, so the communicator's ranks
    show in the output."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    env.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={a.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd, env=env)


def dist_setup(a):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if "WORLD_SIZE" in os.environ and ws != a.gpus:
        raise SystemExit(f"bench.py: WORLD_SIZE={ws} but --gpus {a.gpus}")
    if ws > 1 or (a.mode == "dist" and a.impl == "ours"):
        import datetime
        import torch.distributed as dist
        backend = "nccl"
        try:
            import torch
            if not torch.cuda.is_available():
                backend = "gloo"
        except Exception:
            backend = "gloo"
        if ws > 1:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        else:  # --mode dist on one GPU: a one-rank group
            import socket
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                port = sk.getsockname()[1]
            dist.init_process_group(backend, init_method=f"tcp://127.0.0.1:{port}", rank=0,
                                    world_size=1, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def reduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# DRAM bytes per cell per sweep of the fine sweep kernel, from one-launch ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum / cells) of a 4096^2
# FP64 sweep of each kernel form (warm-up form: the rotation field at
# nu = 1e-3; cluster form: nu = 0.02).
NCU_BYTES_PER_CELL_SWEEP = {"filter": 13.28, "filter_exact": 13.27}


def ncu_traffic(N, variants=()):
    """Measured DRAM bytes per cell per sweep of the kernel form the fine
    sweeps run (the exact cluster form when any sub-step runs it); scaled by
    the caller to a launch.  None for forms without a capture."""
    if "filter_exact" in variants:
        return NCU_BYTES_PER_CELL_SWEEP["filter_exact"]
    if variants and all(v == "filter" for v in variants):
        return NCU_BYTES_PER_CELL_SWEEP["filter"]
    return None


def cpu_baseline(w, sample_s):
    """The oracle (CPU restatement of the reference step) on all host cores:
    serial fine steps of the same workload, bounded to ~sample_s seconds."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    cores = O.cpu_count()
    N = w["N"]
    g = O.grid(N, bc=O.BC_PERIODIC, vel=O.VEL_ROTATION, vp=(w["omega"], 0.5, 0.5), K=w["nu"],
               threads=cores, scheme=O.SCHEME_CONSISTENT)
    den = 2 * w["sigma"] ** 2
    x = (np.arange(N) + 0.5) / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    C = np.exp(-((X - w["hump"][0]) ** 2 + (Y - w["hump"][1]) ** 2) / den)
    dt = w["T"] / w["nt"]
    t0 = time.perf_counter()
    C = O.run(g, C, 0.0, dt, 1)
    t1 = time.perf_counter() - t0
    n = max(1, min(200, int(sample_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    O.run(g, C, dt, dt, n)
    el = time.perf_counter() - t0
    return {"value": N * N * n / el, "unit": "cell-updates/s", "cores": cores, "kind": "port",
            "sample": f"{n} serial fine steps of the {N}^2 workload (oracle, OpenMP over lines)"}


def run_reference(a, w, ws, rank):
    """Reference arm: the reference path's serial fine time-stepping, on the
    host cores (oracle port: the reference has no CPU implementation of its
    own) or, with --ref-device gpu, the reference binary's GpuOneStep on the
    GPU (oracle/_ref).  Rank 0 only."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    N = w["N"]
    dt = w["T"] / w["nt"]
    if a.ref_device == "gpu":
        if not O.ref_available():
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference binary not built (make -C oracle ref)"}))
            return
        x = -1.0 + (np.arange(N) + 0.5) * (2.0 / N)
        X, Y = np.meshgrid(x, x, indexing="ij")
        C0 = np.exp(-((X + 0.35) ** 2 + Y ** 2) / 0.005)
        nst = max(2, int(2e8 / (N * N)))
        vals = []
        for i in range(a.warmup + a.steps):
            _, ms = O.ref_time_run(N, w["nu"], 0.0, dt, nst, C0)
            if i >= a.warmup:
                vals.append(N * N * nst / (ms * 1e-3))
        v = statistics.median(vals)
        line = dict(metric="parareal_cell_updates_per_s", value=v, unit="cell-updates/s",
                    impl="reference", n_gpus=1, steps=a.steps, warmup=a.warmup,
                    ms_per_step=N * N * nst / v * 1e3, higher_is_better=True, scaling="weak",
                    vs_baseline=None, dtype="f64", data="synthetic",
                    config={"workload": f"reference binary GpuOneStep, {N}^2, {nst} serial fine "
                                        "steps per sample (reference domain and velocity)"},
                    cpu_baseline=None,
                    e2e={"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line))
        return
    cores = O.cpu_count()
    g = O.grid(N, bc=O.BC_PERIODIC, vel=O.VEL_ROTATION, vp=(w["omega"], 0.5, 0.5), K=w["nu"],
               threads=cores, scheme=O.SCHEME_CONSISTENT)
    den = 2 * w["sigma"] ** 2
    x = (np.arange(N) + 0.5) / N
    X, Y = np.meshgrid(x, x, indexing="ij")
    C = np.exp(-((X - w["hump"][0]) ** 2 + (Y - w["hump"][1]) ** 2) / den)
    t0 = time.perf_counter()
    O.run(g, C, 0.0, dt, 1)
    t1 = time.perf_counter() - t0
    nst = max(1, int(min(a.cpu_sample_s, 20.0) / max(t1, 1e-6)))
    vals = []
    for i in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        C = O.run(g, C, 0.0, dt, nst)
        el = time.perf_counter() - t0
        if i >= a.warmup:
            vals.append(N * N * nst / el)
    v = statistics.median(vals)
    sample = f"{nst} serial fine steps of the {N}^2 workload per step (oracle port, OpenMP)"
    line = dict(metric="parareal_cell_updates_per_s", value=v, unit="cell-updates/s",
                impl="reference", n_gpus=ws, steps=a.steps, warmup=a.warmup,
                ms_per_step=N * N * nst / v * 1e3, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic",
                config={"workload": workload_name(w, a) + "; reference arm: serial fine "
                                                          "time-stepping on the host cores"},
                cpu_baseline={"value": v, "unit": "cell-updates/s", "cores": cores,
                              "kind": "port", "sample": sample},
                e2e={"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": 0})
    print(json.dumps(line))


def run_ours(a, w, ws, rank, local):
    import torch
    import ccfv
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, nt = w["N"], w["nt"]
    grid = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_ROTATION,
                          vel_params=(w["omega"], *w["center"]), K=w["nu"],
                          scheme=ccfv.SCHEME_CONSISTENT)
    solver = ccfv.Solver(grid, local)
    C0 = initial_field(w, solver, dev)
    out = torch.empty_like(C0)
    prec = ccfv.FP32 if a.coarse == "fp32" else ccfv.FP64
    form = ccfv.FORM_DELTA if a.form == "delta" else ccfv.FORM_STANDARD
    kw = dict(t0=0.0, t1=w["T"], nt_fine=nt, n_slices=w["slices"], coarse_ratio=w["ratio"],
              tol=w["tol"], kmax=w["kmax"], coarse_precision=prec, form=form)
    stream = torch.cuda.current_stream()

    for _ in range(a.warmup):
        solver.parareal(C0, out, **kw)
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ccfv.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    ev0.record(stream)
    for _ in range(a.steps):
        _, st = solver.parareal(C0, out, **kw)
        stats.append(st)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = ccfv.kernel_launches() - l0
    ck = clocks.stop()
    barrier(ws)
    ms = ev0.elapsed_time(ev1)
    ms_max = reduce_max(ms, ws)
    value = ws * (N * N * nt) * a.steps / (ms_max * 1e-3)

    # e2e: the same solve through the C ABI with pinned host buffers (H2D of
    # the initial field and D2H of the result inside every timed step)
    h_in = torch.empty(N, N, dtype=torch.float64, pin_memory=True)
    h_in.copy_(C0.cpu())
    h_out = torch.empty(N, N, dtype=torch.float64, pin_memory=True)
    hin_np, hout_np = h_in.numpy(), h_out.numpy()
    solver.parareal(hin_np, hout_np, **kw)
    torch.cuda.synchronize()
    barrier(ws)
    e0 = time.perf_counter()
    for _ in range(a.steps):
        solver.parareal(hin_np, hout_np, **kw)
    torch.cuda.synchronize()
    e_s = reduce_max(time.perf_counter() - e0, ws)
    e2e_value = ws * (N * N * nt) * a.steps / e_s

    # live roofline of the dominant kernel (the fine sweep) from the F-phase
    # device time of the timed solves
    f_ms = sum(s["fine_ms"] for s in stats)
    f_launch = sum(s["fine_sweep_launches"] for s in stats)
    f_cells = sum(s["fine_sweep_cells"] for s in stats)
    peak, peak_kind = measured_peak()
    achieved = f_cells * BYTES_PER_FINE_CELL_SWEEP / (f_ms * 1e-3) / 1e9 if f_ms > 0 else None
    tpc = ncu_traffic(N, [v for v, _ in solver.sweep_plan(w["T"] / nt)])
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": (tpc * f_cells / f_launch) if (tpc and f_launch) else None,
            "kernel": "F phase: " + solver.variant_names(w["T"] / nt),
            "bytes_per_launch": f_cells * BYTES_PER_FINE_CELL_SWEEP / max(f_launch, 1),
            "avg_launch_us": f_ms * 1e3 / max(f_launch, 1), "peak_source": peak_kind}

    # accuracy of the benchmarked solve against the serial fine solve (untimed)
    err = None
    plain = None
    if rank == 0:
        fine = C0.clone()
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        solver.run(fine, 0.0, w["T"] / nt, nt)
        e_b.record(stream)
        torch.cuda.synchronize()
        plain = N * N * nt / (e_a.elapsed_time(e_b) * 1e-3)
        err = float(torch.linalg.norm(out - fine) / torch.linalg.norm(fine))

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(w, a.cpu_sample_s)

    if rank == 0:
        st = stats[-1]
        line = dict(
            metric="parareal_cell_updates_per_s", value=value, unit="cell-updates/s",
            n_gpus=ws, steps=a.steps, warmup=a.warmup, ms_per_step=ms_max / a.steps,
            higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
            data="synthetic",
            config={"workload": workload_name(w, a), "N": N, "nt_fine": nt,
                    "n_slices": w["slices"], "coarse_ratio": w["ratio"],
                    "coarse_precision": a.coarse, "form": a.form,
                    "l2_flush": "working set (slice states) > L2: "
                                f"{(2 * w['slices'] + 2) * N * N * 8 / 1e9:.1f} GB",
                    "parallelism": f"{ws} independent instance(s), one per GPU"},
            iterations=st["iterations"], converged=st["converged"],
            final_update=st["update"][-1] if st["update"] else None,
            l2_err_vs_serial_fine=err,
            executed_cell_updates_per_s=ws * (st["fine_cell_updates"] +
                                              st["coarse_cell_updates"]) * a.steps /
            (ms_max * 1e-3),
            plain_serial_fine_cell_updates_per_s=plain,
            e2e={"value": e2e_value, "unit": "cell-updates/s",
                 "h2d_bytes_per_step": 8 * N * N, "d2h_bytes_per_step": 8 * N * N},
            roofline=roof, cpu_baseline=cpu, clocks=ck, gpu_launches=launches)
        if ws == 1 and not a.no_batch_serve:
            # the batched and served forms of the metric on the same GPU (one
            # timed batch solve after one warm-up; one served request stream)
            line["batch"] = measure_batch(a, ws, rank, local, 1, 1)
            line["serve"] = measure_serve(a, ws, rank, local)
            line["batched_vs_plain"] = line["batch"].get("batched_vs_plain_same_coarse_theta")
            line["served_vs_plain"] = line["serve"].get("served_vs_plain_same_coarse_theta")
        print(json.dumps(line))


def batch_problems(a, rng, n, nmin=64, nmax=1024, mixed_velocity=False):
    """Mixed instances: N log-uniform, velocity, diffusivity log-uniform, 1-8
    Gaussians, T = 1, slices scaled with N, coarse dt = 8 x fine, FP32 coarse
    (synthetic, seeded)."""
    import ccfv
    probs = []
    for _ in range(n):
        N = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        T = 1.0
        if mixed_velocity:
            kind = int(rng.integers(0, 3))
            nu = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
            T = float(rng.uniform(0.25, 2.0))
            tol = float(rng.choice([1e-8, 1e-10]))
        else:
            kind = 0
            nu = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-1))))
            tol = 1e-10
        if kind == 0:
            V = rng.uniform(-2, 2, 2)
            vel, vp, vmax = ccfv.VEL_CONST, (float(V[0]), float(V[1])), float(np.abs(V).max())
        elif kind == 1:
            vel, vp, vmax = ccfv.VEL_ROTATION, (2 * np.pi, 0.5, 0.5), np.pi
        else:
            vel, vp, vmax = ccfv.VEL_SWIRL, (T,), 1.0
        S = int(min(64, max(16, 16 * 2 ** round(np.log2(N / 64)))))
        ratio = 8
        dt = 0.8 / (N * max(vmax, 1e-3))
        nt = int(np.ceil(T / dt / (S * ratio))) * S * ratio
        ng = int(rng.integers(1, 9))
        par = [[float(rng.uniform(0.2, 0.8)), float(rng.uniform(0.2, 0.8)),
                2.0 * float(rng.uniform(0.03, 0.1)) ** 2, float(rng.uniform(0.5, 1.0))]
               for _ in range(ng)]
        g = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=vel, vel_params=vp, K=nu,
                           scheme=ccfv.SCHEME_CONSISTENT)
        probs.append(dict(grid=g, gauss=par, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                          coarse_ratio=ratio, tol=tol, kmax=S, coarse_precision=ccfv.FP32,
                          form=ccfv.FORM_DELTA, N=N, coarse_theta=coarse_theta_arg(a)))
    return probs


def _fields(probs, device, host=False):
    import torch
    import ccfv
    for p in probs:
        s = ccfv.Solver(p["grid"], device)
        C0 = torch.empty(p["N"], p["N"], dtype=torch.float64, device=f"cuda:{device}")
        s.gaussians(C0, p["gauss"], images=1)
        if host:
            p["C0"] = C0.cpu().numpy()
            p["C_T"] = np.empty_like(p["C0"])
        else:
            p["C0"] = C0
            p["C_T"] = torch.empty_like(C0)
        s.close()


def plain_sample(probs, n):
    """Every problem (n <= 0) or n of them, evenly strided."""
    if n <= 0 or n >= len(probs):
        return list(probs)
    return probs[:: max(1, len(probs) // n)][:n]


def plain_rate(probs, device, theta=0.5):
    """Plain single-instance FP64 form: each problem alone, FP64 coarse
    (Crank-Nicolson coarse steps unless `theta` says otherwise)."""
    import torch
    import ccfv
    cells, ms = 0.0, 0.0
    for p in probs:
        s = ccfv.Solver(p["grid"], device)
        kw = {k: p[k] for k in ("t0", "t1", "nt_fine", "n_slices", "coarse_ratio", "tol", "kmax")}
        kw["coarse_theta"] = theta
        s.parareal(p["C0"], p["C_T"], coarse_precision=ccfv.FP64, form=ccfv.FORM_DELTA, **kw)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.parareal(p["C0"], p["C_T"], coarse_precision=ccfv.FP64, form=ccfv.FORM_DELTA, **kw)
        b.record()
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
        cells += p["N"] ** 2 * p["nt_fine"]
        s.close()
    return cells / (ms * 1e-3)


def run_dist(a, w, ws, rank, local):
    """One Parareal solve of the workload with its time slices spread over
    the ranks (ccfv.dist.parareal_dist on the CudaSlices backend: the F
    phases of all ranks run concurrently, the coarse sweep is pipelined rank
    to rank with one N^2 boundary state per rank boundary over NCCL).  The
    whole job solves one problem: strong scaling.  Rank 0 checks the result
    against the single-GPU engine (ccfv_parareal) on its own GPU."""
    import torch
    import ccfv
    from ccfv.dist import CudaSlices, parareal_dist
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, nt = w["N"], w["nt"]
    grid = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_ROTATION,
                          vel_params=(w["omega"], *w["center"]), K=w["nu"],
                          scheme=ccfv.SCHEME_CONSISTENT)
    solver = ccfv.Solver(grid, local)
    C0 = initial_field(w, solver, dev)
    be = CudaSlices(solver, timed=True)
    kw = dict(t0=0.0, t1=w["T"], nt_fine=nt, n_slices=w["slices"], coarse_ratio=w["ratio"],
              tol=w["tol"], kmax=w["kmax"], form=ccfv.FORM_DELTA)
    for _ in range(a.warmup):
        out, st = parareal_dist(be, C0, **kw)
    torch.cuda.synchronize()
    be.reset_timers()
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ccfv.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(a.steps):
        out, st = parareal_dist(be, C0, **kw)
    ev1.record()
    torch.cuda.synchronize()
    launches = ccfv.kernel_launches() - l0
    ck = clocks.stop()
    barrier(ws)
    ms_max = reduce_max(ev0.elapsed_time(ev1), ws)
    value = (N * N * nt) * a.steps / (ms_max * 1e-3)
    f_ms = be.fine_phase_ms()
    peak, peak_kind = measured_peak()
    achieved = be.fine_cells * BYTES_PER_FINE_CELL_SWEEP / (f_ms * 1e-3) / 1e9 if f_ms else 0.0
    achieved_min = -reduce_max(-achieved, ws)  # the slowest rank's F phase
    # e2e: initial field from pinned host memory on rank 0 (passed on to the
    # other ranks by the pipeline), result read back to the host on rank 0
    h_in = torch.empty(N, N, dtype=torch.float64, pin_memory=True)
    h_in.copy_(C0.cpu())
    h_out = torch.empty(N, N, dtype=torch.float64, pin_memory=True)
    barrier(ws)
    e0 = time.perf_counter()
    for _ in range(a.steps):
        c0 = h_in.to(dev, non_blocking=True) if rank == 0 else C0
        o, _ = parareal_dist(be, c0, **kw)
        if rank == 0:
            h_out.copy_(o)
    torch.cuda.synchronize()
    e_s = reduce_max(time.perf_counter() - e0, ws)
    err = None
    if rank == 0:
        ref, _ = solver.parareal(C0, t0=0.0, t1=w["T"], nt_fine=nt, n_slices=w["slices"],
                                 coarse_ratio=w["ratio"], tol=w["tol"], kmax=w["kmax"],
                                 coarse_precision=ccfv.FP64, form=ccfv.FORM_DELTA)
        err = float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref))
    barrier(ws)
    if rank == 0:
        line = dict(
            metric="parareal_cell_updates_per_s", value=value, unit="cell-updates/s",
            n_gpus=ws, steps=a.steps, warmup=a.warmup, ms_per_step=ms_max / a.steps,
            higher_is_better=True, scaling="strong", vs_baseline=None, dtype="f64",
            data="synthetic",
            config={"workload": workload_name(w, a), "N": N, "nt_fine": nt,
                    "n_slices": w["slices"], "coarse_ratio": w["ratio"],
                    "coarse_precision": "fp64", "form": "delta",
                    "l2_flush": "working set (slice states) > L2",
                    "parallelism": f"time slices over {ws} rank(s) (ccfv.dist: NCCL send/recv "
                                   "of boundary states, max all-reduce of updates)"},
            iterations=st["iterations"], converged=st["converged"],
            final_update=st["update"][-1] if st["update"] else None,
            l2_err_vs_single_gpu_parareal=err,
            e2e={"value": (N * N * nt) * a.steps / e_s, "unit": "cell-updates/s",
                 "h2d_bytes_per_step": 8 * N * N, "d2h_bytes_per_step": 8 * N * N},
            roofline={"bound": "hbm", "achieved": achieved_min, "peak": peak, "unit": "GB/s",
                      "frac": achieved_min / peak if achieved_min else None, "traffic": None,
                      "kernel": "F phase (slowest rank, in-place sweeps): " +
                                solver.variant_names(w["T"] / nt),
                      "peak_source": peak_kind},
            cpu_baseline=None, clocks=ck, gpu_launches=launches)
        print(json.dumps(line))


def fine_errors(probs, device):
    """Relative L2 of every problem's Parareal result against its own serial
    fine solve on the GPU (same fine steps, untimed)."""
    import torch
    import ccfv
    errs = []
    for p in probs:
        s = ccfv.Solver(p["grid"], device)
        c0 = p["C0"]
        fine = (torch.from_numpy(c0).cuda(device) if isinstance(c0, np.ndarray)
                else c0.clone())
        s.run(fine, p["t0"], (p["t1"] - p["t0"]) / p["nt_fine"], p["nt_fine"])
        out = p["C_T"]
        out = torch.from_numpy(out).cuda(device) if isinstance(out, np.ndarray) else out
        errs.append(float(torch.linalg.norm(out - fine) / torch.linalg.norm(fine)))
        s.close()
    return errs


def measure_batch(a, ws, rank, local, steps, warmup):
    """The batched form on `a.instances` mixed instances: rate of the whole
    batch, every instance's error against its serial fine solve, and the
    plain single-instance FP64 rate of the same instances (with the batch's
    coarse weight, and with Crank-Nicolson coarse steps)."""
    import torch
    import ccfv
    torch.cuda.set_device(local)
    rng = np.random.default_rng(a.seed + rank)
    probs = batch_problems(a, rng, a.instances)
    _fields(probs, local)
    cells = [p["N"] ** 2 * p["nt_fine"] for p in probs]
    for _ in range(warmup):
        st = ccfv.batch_solve(probs, device=local)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ccfv.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        st = ccfv.batch_solve(probs, device=local)
    ev1.record()
    torch.cuda.synchronize()
    launches = ccfv.kernel_launches() - l0
    ck = clocks.stop()
    ms = reduce_max(ev0.elapsed_time(ev1), ws)
    value = ws * sum(cells) * steps / (ms * 1e-3)
    res = dict(value=value, unit="cell-updates/s", ms_per_step=ms / steps, steps=steps,
               warmup=warmup, clocks=ck, gpu_launches=launches, instances=len(probs))
    if rank != 0:
        return res
    errs = fine_errors(probs, local)
    ok = [e <= 1e-10 for e in errs]
    its = [x["iterations"] for x in st]
    sample = plain_sample(probs, a.plain_sample)
    th = coarse_theta_arg(a)
    plain = plain_rate(sample, local)
    plain_th = plain_rate(sample, local, th) if th != 0.5 else plain
    # the batch's shared F phases: 48 algorithmic bytes per executed fine
    # cell-update (3 FP64 sweeps, read + write)
    fine_cu = float(sum(x["fine_cell_updates"] for x in st))
    peak, peak_kind = measured_peak()
    f_gbs = 48.0 * fine_cu / (st[0]["fine_ms"] * 1e-3) / 1e9 if st[0]["fine_ms"] else None
    res.update(
        # the instances whose result meets 1e-10 against the serial fine solve:
        # their share of the cell-updates over the whole batch time
        value_meeting_1e10=ws * sum(c for c, g in zip(cells, ok) if g) * steps / (ms * 1e-3),
        max_l2_err_vs_serial_fine=max(errs), instances_meeting_1e10=int(sum(ok)),
        all_meet_1e10=all(ok), all_converged=all(x["converged"] for x in st),
        converged=int(sum(1 for x in st if x["converged"])),
        not_converged=[dict(instance=i, N=p["N"], iterations=x["iterations"],
                            slices=p["n_slices"],
                            last_update=x["update"][-1] if x["update"] else None,
                            l2_err_vs_serial_fine=errs[i])
                       for i, (p, x) in enumerate(zip(probs, st)) if not x["converged"]],
        iterations_mean=float(np.mean(its)), fine_ms=st[0]["fine_ms"],
        coarse_ms=st[0]["coarse_ms"],
        fine_phase={"executed_fine_cell_updates": fine_cu, "achieved_gbs": f_gbs,
                    "peak_gbs": peak, "frac": (f_gbs / peak) if f_gbs else None,
                    "peak_source": peak_kind},
        plain_fp64_same_coarse_theta_cell_updates_per_s=plain_th,
        batched_vs_plain_same_coarse_theta=(value / ws / plain_th) if plain_th else None,
        plain_fp64_crank_nicolson_cell_updates_per_s=plain,
        batched_vs_plain_crank_nicolson=(value / ws / plain) if plain else None,
        config={"workload": f"{a.instances} periodic instances per GPU, N log-uniform "
                            "64..1024, constant velocity U[-2,2]^2, nu log-uniform "
                            "1e-4..1e-1, 1-8 Gaussians, T=1, fine dt at CFL 0.8, 16-64 "
                            "slices, coarse dt = 8 x fine, FP32 coarse / FP64 fine, "
                            f"coarse diffusion weight {a.coarse_theta}, "
                            "tol 1e-10 (cap = slices)", "seed": a.seed,
                "plain": "each instance alone, FP64 coarse steps, with the batch's coarse "
                         "weight (headline ratio) and with Crank-Nicolson "
                         f"({len(sample)} instances)"})
    return res


def run_batch(a, ws, rank, local):
    r = measure_batch(a, ws, rank, local, a.steps, a.warmup)
    if rank == 0:
        line = dict(metric="parareal_cell_updates_per_s", value=r.pop("value"),
                    unit=r.pop("unit"), mode="batch", n_gpus=ws, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f64", data="synthetic")
        line.update(r)
        print(json.dumps(line))


def measure_serve(a, ws, rank, local):
    """The served form: `a.requests` mixed requests, first all at once
    (closed-loop capacity), then as Poisson arrivals at 80% of that capacity
    through the continuous-batching server; latency percentiles, every
    request's error against its serial fine solve, and the plain
    single-instance FP64 rate of the same requests."""
    import torch
    import ccfv
    torch.cuda.set_device(local)
    rng = np.random.default_rng(a.seed + 1000 + rank)
    probs = batch_problems(a, rng, a.requests, nmin=128, nmax=a.serve_nmax, mixed_velocity=True)
    _fields(probs, local, host=True)
    cells = [p["N"] ** 2 * p["nt_fine"] for p in probs]
    budget = int(96e9)
    # capacity: the same requests all at once (closed loop)
    srv = ccfv.Server(budget, device=local)
    t0 = time.perf_counter()
    tk = [srv.submit(p) for p in probs]
    for t in tk:
        srv.wait(t)
    cap = sum(cells) / (time.perf_counter() - t0)
    srv.close()
    # open loop: Poisson arrivals at 80% of capacity
    rate = 0.8 * cap / float(np.mean(cells))
    gaps = rng.exponential(1.0 / rate, len(probs))
    srv = ccfv.Server(budget, device=local)
    lat, tickets = [], []
    t_start = time.perf_counter()
    t_next = t_start
    for p, gap in zip(probs, gaps):
        t_next += gap
        while time.perf_counter() < t_next:
            time.sleep(0.0002)
        tickets.append(srv.submit(p))
    its, conv = [], []
    for t in tickets:
        st, l_ms = srv.wait(t)
        lat.append(l_ms)
        its.append(st["iterations"])
        conv.append(st["converged"])
    span = time.perf_counter() - t_start
    srv.close()
    value = sum(cells) / span
    res = dict(value=value, unit="cell-updates/s", requests=len(probs))
    if rank != 0:
        return res
    errs = fine_errors(probs, local)
    ok10 = [e <= 1e-10 for e in errs]
    ok_tol = [e <= p["tol"] for e, p in zip(errs, probs)]
    sample = plain_sample(probs, a.plain_sample)
    for p in sample:
        p["C0"] = torch.from_numpy(p["C0"]).cuda(local)
        p["C_T"] = torch.empty_like(p["C0"])
    th = coarse_theta_arg(a)
    plain = plain_rate(sample, local)
    plain_th = plain_rate(sample, local, th) if th != 0.5 else plain
    res.update(
        latency_ms_p50=float(np.percentile(lat, 50)),
        latency_ms_p99=float(np.percentile(lat, 99)),
        capacity_cell_updates_per_s=cap, arrival_rate_per_s=rate,
        iterations_mean=float(np.mean(its)), all_converged=all(conv),
        max_l2_err_vs_serial_fine=max(errs), requests_meeting_1e10=int(sum(ok10)),
        requests_meeting_own_tol=int(sum(ok_tol)),
        value_meeting_1e10=sum(c for c, g in zip(cells, ok10) if g) / span,
        plain_fp64_same_coarse_theta_cell_updates_per_s=plain_th,
        served_vs_plain_same_coarse_theta=(value / plain_th) if plain_th else None,
        plain_fp64_crank_nicolson_cell_updates_per_s=plain,
        served_vs_plain_crank_nicolson=(value / plain) if plain else None,
        capacity_vs_plain_same_coarse_theta=(cap / plain_th) if plain_th else None,
        config={"workload": f"{a.requests} requests, Poisson arrivals at 80% of measured "
                            f"capacity, N log-uniform 128..{a.serve_nmax}, velocity from "
                            "{constant, rotation, swirl}, nu log-uniform 1e-4..1e-2, T "
                            "U[0.25,2], tol in {1e-8,1e-10}, HBM budget 96 GB, FP32 coarse, "
                            f"coarse diffusion weight {a.coarse_theta}", "seed": a.seed,
                "plain": "each request alone, FP64 coarse steps, with the served coarse "
                         "weight (headline ratio) and with Crank-Nicolson "
                         f"({len(sample)} requests)"})
    return res


def run_serve(a, ws, rank, local):
    r = measure_serve(a, ws, rank, local)
    if rank == 0:
        line = dict(metric="parareal_cell_updates_per_s", value=r.pop("value"),
                    unit=r.pop("unit"), mode="serve", n_gpus=ws, higher_is_better=True,
                    scaling="weak", vs_baseline=None, dtype="f64", data="synthetic")
        line.update(r)
        print(json.dumps(line))


def run_step(a, w, ws, rank, local):
    """Serial fine time-stepping of the workload's field: the fused sweep
    kernels alone (three launches per fine step), no Parareal around them."""
    import torch
    import ccfv
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, nt = w["N"], w["nt"]
    dt = w["T"] / nt
    t0 = 0.0
    if a.vel == "swirl":  # swirling deformation (T = 1.5), fine dt at CFL 0.8
        grid = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_SWIRL,
                              vel_params=(1.5,), K=w["nu"], scheme=ccfv.SCHEME_CONSISTENT)
        dt, t0 = 0.8 / N, 0.2
        desc = f"periodic {N}^2 swirling-deformation field, nu={w['nu']}, dt=0.8/N"
    elif a.vel == "compat":  # the reference's domain, velocity, boundaries and scheme
        grid = ccfv.make_grid(N, K=w["nu"])
        dt = 0.8 * (2.0 / N) / 4.0
        desc = (f"{N}^2 field on the reference's domain [-1,1]^2, velocity (-4y, 4x), "
                f"compat boundaries, reference scheme, K={w['nu']}, dt at CFL 0.8")
    else:
        grid = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_ROTATION,
                              vel_params=(w["omega"], *w["center"]), K=w["nu"],
                              scheme=ccfv.SCHEME_CONSISTENT)
        desc = f"periodic {N}^2 rotation field, nu={w['nu']}, dt=T/{nt}"
    solver = ccfv.Solver(grid, local)
    C = initial_field(w, solver, dev)
    n = a.inner
    stream = torch.cuda.current_stream()

    def advance(field, t):
        if a.noalloc:  # the allocation-free entry point (its scan kernels)
            import ctypes
            sp = ctypes.c_void_p(stream.cuda_stream)
            for k in range(n):
                rc = ccfv.lib().ccfv_step_noalloc(ctypes.byref(grid),
                                                  ctypes.c_void_p(field.data_ptr()),
                                                  t + k * dt, dt, sp)
                if rc:
                    raise ccfv.CcfvError(rc, "ccfv_step_noalloc")
        else:
            solver.run(field, t, dt, n)

    for i in range(a.warmup):
        advance(C, t0 + i * n * dt)
    solver.check()
    torch.cuda.synchronize()
    barrier(ws)
    clocks = ClockSampler(local)
    clocks.start()
    l0 = ccfv.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(a.steps):
        advance(C, t0 + i * n * dt)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = ccfv.kernel_launches() - l0
    ck = clocks.stop()
    solver.check()
    ms = reduce_max(ev0.elapsed_time(ev1), ws)
    cells = N * N * n * a.steps
    value = ws * cells / (ms * 1e-3)
    # e2e: host field in, host field out, through the C ABI, every step
    h = torch.empty(N, N, dtype=torch.float64, pin_memory=True)
    h.copy_(C.cpu())
    hn = h.numpy()
    solver.run(hn, 0.0, dt, n)
    barrier(ws)
    e0 = time.perf_counter()
    for i in range(a.steps):
        hn = solver.run(hn, i * n * dt, dt, n)
    e_s = reduce_max(time.perf_counter() - e0, ws)
    peak, peak_kind = measured_peak()
    sweeps = 3 * n * a.steps
    achieved = N * N * sweeps * BYTES_PER_FINE_CELL_SWEEP / (ms * 1e-3) / 1e9
    tpc = ncu_traffic(N, [v for v, _ in solver.sweep_plan(dt)])
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(w, a.cpu_sample_s)
    if rank == 0:
        print(json.dumps(dict(
            metric="fine_cell_updates_per_s", value=value, unit="cell-updates/s", mode="step",
            n_gpus=ws, steps=a.steps, warmup=a.warmup, ms_per_step=ms / a.steps,
            higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
            data="synthetic",
            config={"workload": f"serial fine split steps of the {desc}, {n} steps per timed "
                                "step" + (" (ccfv_step_noalloc)" if a.noalloc else ""),
                    "l2_flush": f"field {N * N * 8 / 1e6:.0f} MB per sweep (read + write "
                                "stream; L2 not flushed)"},
            e2e={"value": ws * cells / e_s, "unit": "cell-updates/s",
                 "h2d_bytes_per_step": 8 * N * N, "d2h_bytes_per_step": 8 * N * N},
            roofline={"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                      "frac": achieved / peak, "traffic": tpc * N * N if tpc else None,
                      "kernel": ("sweep_kernel / sweep_fast_kernel (ccfv_step_noalloc)"
                                 if a.noalloc else solver.variant_names(dt)),
                      "bytes_per_launch": 16 * N * N, "avg_launch_us": ms * 1e3 / sweeps,
                      "peak_source": peak_kind},
            cpu_baseline=cpu, clocks=ck, gpu_launches=launches)))


def run_split(a, ws, rank, local):
    """Precision split: swirling deformation (T = 1.5), nu = 1e-4, four seeded
    Gaussians, 128 slices, coarse dt = 8 x fine; Parareal with FP32 and with
    FP64 coarse steps against the serial fine solve (iterations to the
    tolerance, final error, rate).  Grid side from --n."""
    import torch
    import ccfv
    torch.cuda.set_device(local)
    N, S, ratio, T, nu = a.n, 128, 8, 1.5, 1e-4
    dt = 0.8 / N  # swirl speed <= 1
    nt = int(np.ceil(T / dt / (S * ratio))) * S * ratio
    rng = np.random.default_rng(a.seed)
    gs = [[float(rng.uniform(0.25, 0.75)), float(rng.uniform(0.25, 0.75)),
           2.0 * float(rng.uniform(0.03, 0.1)) ** 2, 1.0] for _ in range(4)]
    g = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_SWIRL, vel_params=(T,), K=nu,
                       scheme=ccfv.SCHEME_CONSISTENT)
    s = ccfv.Solver(g, local)
    C0 = torch.empty(N, N, dtype=torch.float64, device=f"cuda:{local}")
    s.gaussians(C0, gs, images=1)
    fine = C0.clone()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s.run(fine, 0.0, T / nt, nt)
    e1.record()
    torch.cuda.synchronize()
    serial_ms = e0.elapsed_time(e1)
    res = {}
    out = torch.empty_like(C0)
    for name, prec in (("fp64", ccfv.FP64), ("fp32", ccfv.FP32)):
        e0.record()
        _, st = s.parareal(C0, out, t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                           tol=1e-10, kmax=a.kmax, coarse_precision=prec, form=ccfv.FORM_DELTA)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[name] = dict(iterations=st["iterations"], converged=st["converged"],
                         final_update=st["update"][-1] if st["update"] else None,
                         l2_err_vs_serial_fine=float(torch.linalg.norm(out - fine) /
                                                     torch.linalg.norm(fine)),
                         cell_updates_per_s=N * N * nt / (ms * 1e-3), ms=ms,
                         update=[float("%.3g" % u) for u in st["update"]])
    if rank == 0:
        print(json.dumps(dict(
            metric="parareal_cell_updates_per_s", value=res["fp32"]["cell_updates_per_s"],
            unit="cell-updates/s", mode="split", n_gpus=ws, steps=1, warmup=0,
            higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64+f32",
            data="synthetic",
            config={"workload": f"precision split: periodic {N}^2, swirling deformation T=1.5, "
                                f"nu=1e-4, 4 seeded Gaussians, Nt={nt}, 128 slices, coarse dt = "
                                f"8 x fine, delta form, tol 1e-10 (cap {a.kmax})",
                    "seed": a.seed},
            serial_fine_cell_updates_per_s=N * N * nt / (serial_ms * 1e-3),
            fp32_coarse=res["fp32"], fp64_coarse=res["fp64"])))


def main():
    a = parse()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(a))
    w = workload(a)
    ws, rank, local = dist_setup(a)
    try:
        if a.impl == "reference":
            run_reference(a, w, ws, rank)
        elif a.mode == "batch":
            run_batch(a, ws, rank, local)
        elif a.mode == "serve":
            run_serve(a, ws, rank, local)
        elif a.mode == "step":
            run_step(a, w, ws, rank, local)
        elif a.mode == "split":
            run_split(a, ws, rank, local)
        elif (ws > 1 and a.multi == "dist") or a.mode == "dist":
            run_dist(a, w, ws, rank, local)
        else:
            run_ours(a, w, ws, rank, local)
    finally:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

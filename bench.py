#!/usr/bin/env python
"""Benchmark of the LBM time step: D3Q19 256^3 square duct on B200.

Workload (the configuration the headline metric is quoted on): D3Q19 TRT,
tau = 0.9, Lambda = 3/16, 256 x 256 x 256 nodes, solid layers at y = 0, 255
and z = 0, 255, periodic in x, Guo body force Fx = 1e-6, float32 storage.
One bench "step" is one LBM time step over the whole lattice: one launch of
the bulk kernel (the duct has no link rules, so no boundary launch); runs of
32 steps replay a CUDA graph captured before the warm-up. The lattice
(2 x 1.27 GB) is ~20x the 126 MB L2, so every step streams from HBM; no L2
flush is needed. Timing: exactly W warm-up steps, then timed regions of
exactly K steps (CUDA events between barriers, max over ranks), repeated
until they span 2 s so that the nvidia-smi clock samples (every 50 ms) see
the GPU under load; ``ms_per_step`` is the median region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--variant pull|aa]
                    [--storage float32|float16|bfloat16|float64] [--impl reference]

Prints one JSON line (rank 0). ``value`` is whole-job MLUPS (all GPUs; each
GPU runs its own replica of the duct: the step has no inter-GPU exchange in
this build, so scaling is weak, replicas only). ``e2e`` is MLUPS through the
public API with host buffers: per e2e step, ``initialize`` from pinned host
rho/u (float64), ``run`` of a chunk of time steps, ``macroscopic`` back to the
host. ``roofline.achieved`` = 152 B per update (2 Q float32, the reference's
count, benchmarks/bench_mlups.py:9-10) x the nodes of one launch over the
CUDA-event time per step (one launch per step, so an upper bound on the
launch duration). ``cpu_baseline`` times the reference's own CPU solver
(``ReferenceSolver(params, xp=numpy)``, the unmodified package in
baseline/_ref; the NumPy oracle port where that is absent) on a bounded slab
of the same duct on this host; ``--impl reference`` times the same.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "D3Q19 256\u00b3 MLUPS, %HBM peak: fp32 vs fp16-store at \u22641e-3 u err; adj/fwd time"
BYTES = {"float32": 4, "float64": 8, "float16": 2, "bfloat16": 2}
DTYPE_TAG = {"float32": "f32", "float64": "f64", "float16": "f16-store/f32", "bfloat16": "bf16-store/f32"}
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
MIN_TIMED_SECONDS = 2.0
MIN_REPEATS, MAX_REPEATS = 3, 100000
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--variant", choices=("pull", "aa"), default="pull")
    ap.add_argument("--storage", choices=tuple(BYTES), default="float32")
    ap.add_argument("--launch", choices=("split", "fused"), default="split")
    ap.add_argument("--block", default="32x4", help="bulk tile, e.g. 32x4")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--e2e-iters", type=int, default=3)
    ap.add_argument("--e2e-chunk", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the batched-cavities study (aggregate MLUPS against separate launches)")
    ap.add_argument("--study", choices=("tgv", "cylinder", "batched", "adjoint", "precision", "setup", "kernels"),
                    default=None,
                    help="run one configuration study alone and print its JSON (no duct line)")
    ap.add_argument("--study-steps", type=int, default=None, help="steps of --study (default: the study's own)")
    ap.add_argument("--cylinder-method", choices=("both", "bouzidi", "ibm"), default="both",
                    help="body of --study cylinder")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the Taylor-Green and cylinder configuration studies")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the adjoint-configuration study (forward/backward cost and finite differences)")
    ap.add_argument("--precision-steps", type=int, default=5000,
                    help="steps of the storage-precision study (0 = skip)")
    ap.add_argument("--repeat-seconds", type=float, default=MIN_TIMED_SECONDS,
                    help="repeat the timed region of exactly --steps steps until the repeats span this long "
                         "(at least 3 repeats); 0 for three repeats (profiling)")
    ap.add_argument("--no-run-loop", dest="run_loop", action="store_false",
                    help="skip the public run-loop measurement (fused state checks)")
    return ap.parse_args()


def duct_params(lbm, n, nx=None, nz=None, storage="float32"):
    nx = n if nx is None else nx
    nz = n if nz is None else nz
    solid = np.zeros((nz, n, nx), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    return lbm.SimulationParams(nx=nx, ny=n, nz=nz, tau=0.9, collision="trt", force=(1e-6, 0.0, 0.0),
                                solid=solid, dtype=storage)


# --------------------------------------------------------------------- CPU side
def duct_slab_solid(n: int, nz: int) -> np.ndarray:
    solid = np.zeros((nz, n, n), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    return solid


def _time_steps(step, steps: int, warmup: int, budget: float | None):
    """Call ``step()`` `warmup` times, then time at least `steps` calls (more, up to 10x, while under
    `budget` seconds; at least 3): (calls timed, seconds)."""
    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    done = 0
    while done < steps or (budget is not None and time.perf_counter() - t0 < budget and done < 10 * steps):
        step()
        done += 1
        if budget is not None and time.perf_counter() - t0 >= budget and done >= 3:
            break
    return done, time.perf_counter() - t0


def oracle_mlups(n: int, nz: int, steps: int, warmup: int, budget: float | None = None):
    """NumPy oracle on an n x n x nz slab of the duct: (MLUPS, steps timed, seconds)."""
    import lbm_b200 as lbm
    from oracle import OracleSolver

    s = OracleSolver(duct_params(lbm, n, nz=nz))
    done, dt = _time_steps(s.step, steps, warmup, budget)
    return n * n * nz * done / dt / 1e6, done, dt


def cpu_reference_mlups(n: int, nz: int, steps: int, warmup: int, budget: float | None = None):
    """The reference's own CPU solver, ``ReferenceSolver(params, xp=numpy)`` from the unmodified
    package in baseline/_ref (``make_solver(params, backend="numpy")``), one ``_advance(1)`` per step,
    on an n x n x nz slab of the duct: (MLUPS, steps timed, seconds, kind). Without baseline/_ref
    the NumPy oracle port stands in (kind "port")."""
    from oracle import reference_package

    ref = reference_package.modules()
    if ref is None:
        mlups, done, dt = oracle_mlups(n, nz, steps, warmup, budget)
        return mlups, done, dt, "port"
    params = ref.params.SimulationParams(nx=n, ny=n, nz=nz, tau=0.9, collision="trt", force=(1e-6, 0.0, 0.0),
                                         solid=duct_slab_solid(n, nz), dtype="float32")
    s = ref.backends.make_solver(params, backend="numpy")
    s.initialize()
    done, dt = _time_steps(lambda: s._advance(1), steps, warmup, budget)
    return n * n * nz * done / dt / 1e6, done, dt, "reference"


CPU_KIND_NOTE = {
    "reference": "the unmodified reference ReferenceSolver(params, xp=numpy) from baseline/_ref",
    "port": "the NumPy oracle port of the reference ReferenceSolver (baseline/_ref not installed)",
}


def _reference_worker(job):
    """One host core's share of the reference arm (a spawned process): the reference's CPU solver
    on its own slab of the duct; (node updates, seconds, steps, kind)."""
    n, nz, steps, warmup, budget = job
    mlups, done, dt, kind = cpu_reference_mlups(n, nz, steps, warmup, budget=budget)
    return n * n * nz * done, dt, done, kind


def run_reference(args, rank):
    """Reference arm: the reference's own CPU solver (NumPy), rank 0 only, on every host core.

    NumPy's element-wise work runs on one thread, so the arm runs one solver per core, each in a
    process of its own (spawned before any GPU work) on its own slab of the duct, and reports their
    aggregate: all node updates over the slowest process's time."""
    if rank != 0:
        return
    import multiprocessing

    n = args.n
    # the cores this process may run on (at most 64 processes, to bound host memory)
    workers = max(1, min(64, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1))
    # size each slab so that K steps take about a minute (a larger K is cut off at a 60 s budget);
    # with many processes the slabs stay thin to bound host memory
    per_node = 1.0 / 1.4e6
    nz = int(min(16, max(3, round(60.0 / (max(args.steps, 1) * n * n * per_node)))))
    if workers > 4:
        nz = 3
    warm = min(args.warmup, 3)
    with multiprocessing.get_context("spawn").Pool(workers) as pool:
        results = pool.map(_reference_worker, [(n, nz, args.steps, warm, 60.0)] * workers)
    updates = sum(r[0] for r in results)
    dt = max(r[1] for r in results)
    done = min(r[2] for r in results)
    ms_step = max(1e3 * r[1] / r[2] for r in results)  # the slowest process's time per step
    kind = results[0][3]
    mlups = updates / dt / 1e6
    sample = (f"{workers} processes, each a {n}x{n}x{nz} slab of the duct (same walls, force, tau), at least "
              f"{done} steps timed per process ({args.steps} asked; up to 10x as many while under a 60 s budget) "
              f"after {warm} warm-up; all node updates over the slowest process's time")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(mlups, 4), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": round(mlups, 4), "unit": "MLUPS", "cores": workers, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(mlups, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": f"{CPU_KIND_NOTE[kind]}; NumPy element-wise work runs on one thread, so one process per core "
                f"(host has {os.cpu_count()} cores)",
    }
    gpu = reference_gpu_kernels(args)
    if gpu is not None:
        line["reference_gpu_kernels"] = gpu
    print(json.dumps(line), flush=True)


def reference_gpu_kernels(args):
    """For information beside the CPU value: the reference's own CUDA kernels (compiled unmodified
    for sm_100a into oracle/_ref) on the same duct, float32, timed with CUDA events; None when the
    libraries or a GPU are missing."""
    try:
        import torch

        from oracle import ref_kernels

        if not torch.cuda.is_available() or not ref_kernels.available():
            return None
        import lbm_b200 as lbm

        torch.cuda.set_device(0)
        params = duct_params(lbm, args.n, storage="float32")
        out = {v: round(ref_kernels.time_reference(params, v, 100), 1) for v in ("naive", "aa")}
        out |= {"unit": "MLUPS", "workload": f"D3Q19 duct {args.n}^3 float32, 100 steps after 100 untimed",
                "kernels": "stream_collide_naive; aa_odd + aa_even (reference src/lbm/backends/kernels)"}
        return out
    except Exception as exc:  # noqa: BLE001 -- informational only; the CPU value stands
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def workload_config(args):
    n = args.n
    return {
        "workload": f"D3Q19 TRT square duct {n}x{n}x{n}, tau=0.9, Fx=1e-6, walls y/z, periodic x",
        "variant": {"pull": "two-lattice fused pull", "aa": "in-place AA pair"}[args.variant],
        "launch": args.launch, "block": args.block,
        "storage": args.storage, "nodes": n**3, "bytes_per_update": 2 * 19 * BYTES[args.storage],
        "l2": "inputs larger than L2 (lattice %.2f GB vs 126 MB)" % (19 * n**3 * BYTES[args.storage] / 1e9),
        "parallelism": f"replicas x{args.gpus}",
    }


# --------------------------------------------------------------------- GPU side
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every `interval_ms` while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid: str | None, interval_ms: int = 50):
        self.uuid = device_uuid
        self.interval_ms = int(interval_ms)
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms",
               str(self.interval_ms)]
        if self.uuid:
            cmd.insert(1, f"--id={self.uuid}")
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        rows = [r.split(", ") for r in self.lines if r and r[0].isdigit()]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 4 + i and r[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][1]), "samples": len(rows),
                "power_w_max": max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit()) if rows else None,
                "reasons": reasons}


def measured_peak():
    try:
        peaks = json.loads(PEAKS_FILE.read_text())
        return float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, torch copy_ of 1 Gi bf16)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def step_kernel_name(args) -> str:
    """The kernel that carries the duct step (one launch per step)."""
    if args.storage in ("float16", "bfloat16") and args.launch == "split":
        if args.variant == "pull":
            return f"lbm_tma_pull_kernel<D3Q19, {args.storage}>"
        return f"lbm_tma_aa_kernel<D3Q19, {args.storage}, aa_odd + aa_even>"
    return f"lbm_bulk_kernel<D3Q19, {args.storage}, {args.variant}>"


def profile_traffic(variant: str, storage: str):
    """DRAM bytes per launch from the committed ncu summary, if one exists for this kernel/workload."""
    path = ROOT / "profiles" / f"step_{variant}_d3q19_{storage}_duct.md"
    if not path.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", path.read_text())
    return float(m.group(1)) if m else None


def copy_peak_gbs(torch, device, nbytes=512 * 2**20, repeats=20):
    """Device copy bandwidth (read + write), as the reference measures it (bench_mlups.py:66-79)."""
    src = torch.ones(nbytes // 4, dtype=torch.float32, device=device)
    dst = torch.empty_like(src)
    dst.copy_(src)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(repeats):
        dst.copy_(src)
    b.record()
    b.synchronize()
    del src, dst
    return 2 * nbytes * repeats / (a.elapsed_time(b) / 1e3) / 1e9


def precision_study(lbm, torch, n: int, steps: int, variant: str):
    """Duct after `steps` steps in float64, float32, float16 and bfloat16 storage.

    Returns per storage: MLUPS of the run and the velocity error against the
    float64 run (relative L2 over fluid nodes, and max |du| / max |u64|).
    """
    out = {}
    ref = None
    backend = "cuda-aa" if variant == "aa" else "cuda-naive"
    for storage in ("float64", "float32", "float16", "bfloat16"):
        s = lbm.make_solver(duct_params(lbm, n, storage=storage), backend=backend)
        s._advance(2)
        s.initialize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s._advance(steps)
        b.record()
        b.synchronize()
        s.time_step = steps
        s._check_health()
        m = s.macroscopic()
        u = np.stack([c.astype(np.float64) for c in m.u])
        fluid = ~m.solid
        entry = {"mlups": round(n**3 * steps / (a.elapsed_time(b) / 1e3) / 1e6, 1)}
        if ref is None:
            ref = u
        else:
            du = u[:, fluid] - ref[:, fluid]
            entry["u_rel_l2_vs_f64"] = float(np.linalg.norm(du) / np.linalg.norm(ref[:, fluid]))
            entry["u_rel_max_vs_f64"] = float(np.abs(du).max() / np.abs(ref[:, fluid]).max())
        out[storage] = entry
        del s
        torch.cuda.empty_cache()
    out["steps"] = steps
    out["u_max_f64"] = float(np.abs(ref[0]).max())
    return out


def adjoint_study(lbm, torch, steps: int = 2000, window: int = 500, checkpoint: int = 100, fd: bool = True):
    """Adjoint configuration: D3Q19 channel 128 x 64 x 64, Bouzidi sphere r = 8, Zou-He inlet U = 0.04,
    pressure outlet, tau = 0.6, loss = drag averaged over the last `window` of `steps` steps,
    gradients w.r.t. the inlet-speed scale U and a per-node Guo force field G ~ N(0, 1e-7^2).

    float32: forward and backward (recompute + adjoint kernels) timed with CUDA events, host-driven
    as a user calls them; the median of three runs. float64: adjoint dL/dU and dL/dG.v against central differences (h = 1e-4
    relative).
    """
    from lbm_b200.adjoint import AdjointRun, aligned_rules

    lat = lbm.D3Q19
    nx, ny, nz = 128, 64, 64
    solid = lbm.duct_walls(nx, ny, nz)
    body = lbm.sphere(nx / 4.0, (ny - 1) / 2.0, (nz - 1) / 2.0, 8.0)
    solid |= lbm.voxelize(body, solid.shape)
    inflow = np.zeros((3, nz, ny))
    inflow[0, 1:-1, 1:-1] = 0.04

    def case(dtype):
        def make(scale):
            s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
            links = lbm.wall_links(lat, body, s2)
            all_rules, all_d = aligned_rules(rules, d_rules, lbm.bouzidi_rules(lat, links, s2))
            p = lbm.SimulationParams(nx=nx, ny=ny, nz=nz, tau=0.6, collision="trt", solid=s2, dtype=dtype,
                                     link_rules=all_rules)
            return p, all_d
        p, _ = make(1.0)
        return make, lbm.wall_links(lat, body, p.solid), p

    out = {"config": f"D3Q19 {nx}x{ny}x{nz} sphere r=8 (Bouzidi), Zou-He U=0.04, tau=0.6, {steps} steps, "
                     f"drag mean over last {window}, checkpoint every {checkpoint}"}
    make, links, p = case("float32")
    rng = np.random.default_rng(0)
    G = 1e-7 * rng.standard_normal((3, *p.shape)) * p.fluid
    run = AdjointRun(make, links, steps=steps, window=window, checkpoint=checkpoint)
    run.forward(1.0, G)  # warm-up: set-up and tables (later forwards at the same U reuse them)
    run.backward()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwds, bwds = [], []
    for _ in range(3):  # the median of three forward + backward runs
        torch.cuda.synchronize()
        ev[0].record()
        loss = run.forward(1.0, G)
        ev[1].record()
        dU, dG = run.backward()
        ev[2].record()
        ev[2].synchronize()
        fwds.append(ev[0].elapsed_time(ev[1]))
        bwds.append(ev[1].elapsed_time(ev[2]))
    fwd, bwd = statistics.median(fwds), statistics.median(bwds)
    out["float32"] = {"loss": loss, "dL_dU": dU, "forward_ms_per_step": round(fwd / steps, 5),
                      "backward_ms_per_step": round(bwd / steps, 5), "backward_over_forward": round(bwd / fwd, 3),
                      "runs_ms": {"forward": [round(v, 2) for v in fwds], "backward": [round(v, 2) for v in bwds]}}
    if not fd:
        return out
    make64, links64, p64 = case("float64")
    run = AdjointRun(make64, links64, steps=steps, window=window, checkpoint=checkpoint)
    run.forward(1.0, G)
    dU, dG = run.backward()
    h = 1e-4
    fd_u = (run.forward(1.0 + h, G) - run.forward(1.0 - h, G)) / (2 * h)
    v = rng.standard_normal(G.shape) * p64.fluid
    eps = h * np.abs(G).max()
    fd_g = (run.forward(1.0, G + eps * v) - run.forward(1.0, G - eps * v)) / (2 * eps)
    out["float64"] = {"dL_dU": dU, "fd_dL_dU": fd_u, "rel_err_U": abs(dU - fd_u) / abs(fd_u),
                      "dL_dG_dot_v": float((dG * v).sum()), "fd_dL_dG_dot_v": fd_g,
                      "rel_err_G": abs(float((dG * v).sum()) - fd_g) / abs(fd_g)}
    out["float32_vs_float64_dU"] = abs(out["float32"]["dL_dU"] - dU) / abs(dU)
    return out


def tgv_study(lbm, torch, n: int = 512, steps: int = 1000):
    """Taylor-Green configuration: D2Q9 TRT n x n periodic, tau = 0.8, float32, u0 = 0.01 (sin kx cos ky,
    -cos kx sin ky), k = 2 pi / n. MLUPS of `steps` steps (CUDA events; the 2 x 19 MB lattice stays in L2)
    and the decay of the velocity amplitude against exp(-2 nu k^2 t), nu = (tau - 1/2)/3.
    """
    tau = 0.8
    k = 2 * math.pi / n
    y, x = np.mgrid[0:n, 0:n]
    ux = 0.01 * np.sin(k * x) * np.cos(k * y)
    uy = -0.01 * np.cos(k * x) * np.sin(k * y)
    params = lbm.SimulationParams(nx=n, ny=n, tau=tau, collision="trt", dtype="float32")
    s = lbm.make_solver(params, backend="cuda-naive")
    s.initialize(1.0, ux, uy)
    s._advance(s.GRAPH_CHUNK)  # graph capture
    s.initialize(1.0, ux, uy)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    s._advance(steps)
    b.record()
    b.synchronize()
    s.time_step = steps
    s._check_health()
    f = s.macroscopic()
    amp = float((f.u[0] * ux).sum() / (ux * ux).sum())
    exact = math.exp(-2 * (tau - 0.5) / 3 * k * k * steps)
    return {"config": f"D2Q9 TRT {n}x{n} periodic, tau={tau}, float32, {steps} steps",
            "mlups": round(n * n * steps / (a.elapsed_time(b) / 1e3) / 1e6, 1),
            "amplitude": amp, "amplitude_exact": exact, "amplitude_rel_err": abs(amp - exact) / exact}


def cylinder_params(lbm, method: str, nx: int = 880, ny: int = 164, u_max: float = 0.05, iterations: int = 3):
    """Cylinder configuration: D2Q9 channel nx x ny, walls at y = 0 and ny - 1, circle D = 40 at (200, 82),
    parabolic Zou-He inflow (U_max 0.05, profile as the reference's 2D-2 builder), outlet rho = 1, Re = 100
    (tau from nu = U_mean D / Re), float32; the body as Bouzidi links or as an immersed boundary."""
    lattice = lbm.D2Q9
    height = ny - 2
    yc = np.arange(ny) - 0.5
    profile = np.where((yc > 0) & (yc < height), 4.0 * u_max * yc * (height - yc) / height**2, 0.0)
    inflow = np.stack([profile, np.zeros(ny)])
    solid = np.zeros((ny, nx), dtype=bool)
    solid[0, :] = solid[-1, :] = True
    body = lbm.circle(200.0, 82.0, 20.0)
    immersed = links = None
    if method == "ibm":
        immersed = lbm.ImmersedBoundary.from_ball(body, spacing=1.0, iterations=iterations)
    else:
        solid |= lbm.voxelize(body, solid.shape)
    solid, rules = lbm.open_channel(lattice, solid, inflow)
    if method == "bouzidi":
        links = lbm.wall_links(lattice, body, solid)
        rules = lbm.LinkRules.concat(rules, lbm.bouzidi_rules(lattice, links, solid))
    u_mean = 2.0 * u_max / 3.0
    tau = 3.0 * (u_mean * 40.0 / 100.0) + 0.5
    params = lbm.SimulationParams(nx=nx, ny=ny, tau=tau, collision="trt", solid=solid, dtype="float32",
                                  link_rules=rules, immersed=immersed)
    return params, links, u_mean


def cylinder_study(lbm, torch, steps: int = 40000, every: int = 100, methods=("bouzidi", "ibm")):
    """Cylinder configuration, Bouzidi and immersed boundary: `steps` steps from rest through the public run
    loop, drag and lift sampled every `every` steps in float64 (force probe / immersed-body force), as
    C = F / (0.5 U_mean^2 D). MLUPS of the whole run (wall clock, samples included) and of the steps alone
    (CUDA events, no sampling); C_D mean and C_L range over the last quarter of the run.
    """
    out = {}
    for method in methods:
        params, links, u_mean = cylinder_params(lbm, method)
        s = lbm.make_solver(params, backend="cuda-naive")
        probe = lbm.ForceProbe.build(params, links) if links is not None else None
        scale = 0.5 * u_mean**2 * 40.0
        samples = []

        def sample(solver):
            fx, fy = probe.evaluate(solver) if probe is not None else solver.immersed_force
            samples.append((solver.time_step, fx / scale, fy / scale))

        s._advance(s.GRAPH_CHUNK)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s._advance(2000)
        b.record()
        b.synchronize()
        ms_step = a.elapsed_time(b) / 2000
        s.initialize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.run(steps, every=every, callback=sample, check_every=steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        tail = np.array([v for v in samples if v[0] > 0.75 * steps])
        nodes = params.nx * params.ny
        out[method] = {"mlups_run": round(nodes * steps / wall / 1e6, 1),
                       "mlups_steps": round(nodes / ms_step / 1e3, 1), "us_per_step": round(ms_step * 1e3, 2),
                       "cd_mean": float(tail[:, 1].mean()), "cl_min": float(tail[:, 2].min()),
                       "cl_max": float(tail[:, 2].max()), "samples": len(samples)}
        del s
        torch.cuda.empty_cache()
    out["config"] = (f"D2Q9 880x164 channel, cylinder D=40 at (200, 82), Zou-He parabolic inflow U_max=0.05, Re=100, "
                     f"float32, {steps} steps, C_D/C_L every {every} steps (tail: last quarter)")
    return out


def batched_study(lbm, torch, steps: int = 640, separate_steps: int = 20):
    """Batched configuration: 256 lid-driven cavities, sides U{64..512} (seeded), lid 0.1, Re U(100, 1000),
    float32 TRT. Aggregate MLUPS of the persistent batched launch (CUDA graph, autotuned tile and grid)
    against every domain launched on its own each step, host-driven and replayed from a CUDA graph.
    """
    from lbm_b200.batched import BatchedSolver, cavity_batch

    params, sizes, _ = cavity_batch(lbm, count=256, n_min=64, n_max=512, seed=0)
    batch = BatchedSolver(params)
    nodes = batch.nodes
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, k):
        torch.cuda.synchronize()
        ev[0].record()
        fn(k)
        ev[1].record()
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1]) / k

    batch.run(64)
    ms_batched = timed(batch._advance, steps)
    batch.run_separately(2)
    ms_separate = timed(batch.run_separately, separate_steps)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batch.run_separately(2)  # two steps: the buffers end where they started
    graph.replay()
    ms_separate_graph = timed(lambda k: [graph.replay() for _ in range(k // 2)], separate_steps)
    batch.check_health()
    return {"domains": len(params), "nodes": int(nodes), "side_min": int(sizes.min()), "side_max": int(sizes.max()),
            "block": list(batch.block), "blocks": batch.blocks,
            "batched_mlups": round(nodes / ms_batched / 1e3, 1),
            "separate_host_launches_mlups": round(nodes / ms_separate / 1e3, 1),
            "separate_graph_launches_mlups": round(nodes / ms_separate_graph / 1e3, 1),
            "steps": {"batched": steps, "separate": separate_steps}}


def setup_study(lbm, torch):
    """Set-up time of two bodies in a channel, host builders against the device-side compiler
    (voxelisation, wall links, Bouzidi rules; the solver's own tables after): the sphere channel
    (128 x 64 x 64, r = 8) and a 256^3 duct with a sphere of radius 40; then the Zou-He inlet and
    outlet rules of open channels of both sizes. Wall-clock seconds."""
    from lbm_b200 import device_rules

    out = {}
    for label, shape, body in (("sphere_channel_128x64x64", (64, 64, 128), lbm.sphere(32.0, 31.5, 31.5, 8.0)),
                               ("duct_256_sphere_r40", (256, 256, 256), lbm.sphere(256 / 3, 127.5, 127.5, 40.0))):
        nz, ny, nx = shape
        solid = lbm.duct_walls(nx, ny, nz)
        lattice = lbm.D3Q19
        device_rules.ball_channel(lattice, body, solid)  # warm: module load, first launches
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ds, dl, dr = device_rules.ball_channel(lattice, body, solid)
        t_dev = time.perf_counter() - t0
        t0 = time.perf_counter()
        hs = solid | lbm.voxelize(body, solid.shape)
        hl = lbm.wall_links(lattice, body, hs)
        hr = lbm.bouzidi_rules(lattice, hl, hs)
        t_host = time.perf_counter() - t0
        same = bool(np.array_equal(ds, hs) and np.array_equal(dl.q, hl.q) and np.array_equal(dr.values.coeff, hr.values.coeff))
        t0 = time.perf_counter()
        params = lbm.SimulationParams(nx=nx, ny=ny, nz=nz, tau=0.6, collision="trt", solid=ds, link_rules=dr)
        t_params = time.perf_counter() - t0
        t0 = time.perf_counter()
        solver = lbm.make_solver(params, backend="cuda-naive")
        torch.cuda.synchronize()
        t_solver = time.perf_counter() - t0
        out[label] = {"links": len(dl), "rules": len(dr), "host_builders_s": round(t_host, 3),
                      "device_builders_s": round(t_dev, 4), "speedup": round(t_host / t_dev, 1),
                      "identical": same, "params_validation_s": round(t_params, 3),
                      "solver_tables_s": round(t_solver, 3)}
        del solver
        torch.cuda.empty_cache()
    # Zou-He inlet and outlet rules of an open channel (walls y/z), host builder against the device
    for label, n_x, n_yz in (("open_channel_128x64x64", 128, 64), ("open_channel_256x256x256", 256, 256)):
        solid = lbm.duct_walls(n_x, n_yz, n_yz)
        inflow = np.zeros((3, n_yz, n_yz))
        inflow[0, 1:-1, 1:-1] = 0.04
        device_rules.open_channel(lbm.D3Q19, solid, inflow)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ds, dr = device_rules.open_channel(lbm.D3Q19, solid, inflow)
        t_dev = time.perf_counter() - t0
        t0 = time.perf_counter()
        hs, hr = lbm.open_channel(lbm.D3Q19, solid, inflow)
        t_host = time.perf_counter() - t0
        same = bool(np.array_equal(ds, hs) and all(
            np.array_equal(a, b) for a, b in ((dr.node, hr.node), (dr.direction, hr.direction),
                                              (dr.values.coeff, hr.values.coeff),
                                              (dr.values.constant, hr.values.constant),
                                              (dr.values.node, hr.values.node))))
        out[label] = {"rules": len(hr), "host_builder_s": round(t_host, 4), "device_builder_s": round(t_dev, 4),
                      "speedup": round(t_host / t_dev, 1), "identical": same}
    return out


def kernels_study(lbm, torch):
    """Every kernel family outside the headline step, each launched a few times on a small case
    whose inputs exceed L2 (a few hundred MB on the device), timed with CUDA events: the workload of
    the per-family ncu launch list (``ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,
    dram__bytes_write.sum``). Families: the 16-bit node-pair fallbacks (nx = 200, pull and AA);
    on a 192^3 float32 duct the checked step (state check fused), the separate scan, the
    macroscopic readout and the regularised step; on a D2Q9 2048^2 periodic grid the TRT and the cumulant
    steps; the device Zou-He builder on a 256^3 open channel; the per-pass immersed boundary of a large body
    (sphere r = 20, 5 027 markers); the immersed-body adjoint (3D channel); the device-side rule
    compiler on a 256^3 duct with a sphere of radius 40."""
    import dataclasses

    from lbm_b200 import _native as N
    from lbm_b200 import device_rules
    from lbm_b200.adjoint import AdjointRun
    from tests import cases
    from tests.helpers import NS

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(n):
            fn()
        ev[1].record()
        ev[1].synchronize()
        return round(ev[0].elapsed_time(ev[1]) / n * 1e3, 1)

    out = {}
    for backend in ("cuda-naive", "cuda-aa"):
        s = lbm.make_solver(cases.duct(NS, n=128, nx=200, dtype="float16"), backend=backend, graph=False)
        out[f"float16_pair_kernel_{backend}_us_per_step"] = timed(lambda: s._advance(2)) / 2
        del s
    p = cases.duct(NS, n=192, dtype="float32")
    s = lbm.make_solver(p, backend="cuda-naive", graph=False)
    out["checked_step_us"] = timed(lambda: s._advance_checked(1))
    def scan():
        s._health_fresh = False  # the separate scan, as after a state set from outside the run loop
        s._check_health()

    out["health_scan_us"] = timed(scan)
    out["macroscopic_ms"] = timed(lambda: s.macroscopic()) / 1e3
    del s
    s = lbm.make_solver(dataclasses.replace(p, collision="regularized"), backend="cuda-naive", graph=False)
    out["regularized_step_us"] = timed(lambda: s._advance(1))
    del s
    torch.cuda.empty_cache()
    # D2Q9 2048^2 periodic, float32 (2 x 151 MB lattices, above L2): TRT against the cumulant model
    p2 = cases.tgv(NS, n=2048, dtype="float32", tau=0.56)[0]
    for model in ("trt", "cumulant"):
        s = lbm.make_solver(dataclasses.replace(p2, collision=model), backend="cuda-naive", graph=False)
        out[f"d2q9_2048_{model}_step_us"] = timed(lambda: s._advance(1))
        del s
    torch.cuda.empty_cache()
    # the device Zou-He builder on a 256^3 open channel (both columns: count, scan, write)
    solid = lbm.duct_walls(256, 256, 256)
    inflow = np.zeros((3, 256, 256))
    inflow[0, 1:-1, 1:-1] = 0.04
    out["device_zou_he_256_ms"] = timed(lambda: device_rules.open_channel(lbm.D3Q19, solid, inflow), 2) / 1e3
    solid = lbm.duct_walls(96, 64, 64)
    body = lbm.ImmersedBoundary.from_ball(lbm.sphere(40.0, 31.5, 31.5, 20.0), spacing=1.0, iterations=3)
    p = lbm.SimulationParams(nx=96, ny=64, nz=64, tau=0.7, collision="trt", solid=solid, force=(1e-6, 0, 0),
                             immersed=body)
    s = lbm.make_solver(p, backend="cuda-naive", graph=False)
    out["ibm_large_body"] = {"markers": int(s._ibm.tables.n_markers), "nodes": int(s._ibm.tables.n_nodes),
                             "force_us": timed(lambda: s._ibm.run(s._f, N.LAYOUT_PULL)),
                             "step_us": timed(lambda: s._advance(1))}
    del s
    # immersed sphere in a Zou-He duct channel, loss = the body's drag
    lat, solid = lbm.D3Q19, lbm.duct_walls(16, 11, 11)
    inflow = np.zeros((3, 11, 11))
    inflow[0, 1:-1, 1:-1] = 0.04
    ball = lbm.ImmersedBoundary.from_ball(lbm.sphere(6.4, 5.3, 5.1, 1.7), spacing=1.0, iterations=3)

    def make(scale):
        s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
        return lbm.SimulationParams(nx=16, ny=11, nz=11, tau=0.6, collision="trt", solid=s2, dtype="float32",
                                    link_rules=rules, immersed=ball), d_rules

    p, _ = make(1.0)
    run = AdjointRun(make, None, steps=12, window=4, checkpoint=4)
    field = np.zeros((p.d, *p.shape))
    run.forward(1.0, field)
    out["ibm_adjoint_3d_backward_ms"] = timed(run.backward, 2) / 1e3
    solid = lbm.duct_walls(256, 256, 256)
    out["device_compiler_256_ms"] = timed(lambda: device_rules.ball_channel(lbm.D3Q19, lbm.sphere(256 / 3, 127.5, 127.5,
                                                                                                 40.0), solid), 2) / 1e3
    return out


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest value over all ranks (the slowest replica's time); x itself on one rank."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_mlups(nodes: int, steps: int, ms: float, world: int) -> float:
    """Whole-job MLUPS: every rank advances its own replica of `nodes` nodes by `steps` steps;
    `ms` is the slowest rank's time."""
    return world * nodes * steps / (ms / 1e3) / 1e6


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import lbm_b200 as lbm

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    n = args.n
    nodes = n**3
    params = duct_params(lbm, n, storage=args.storage)
    backend = "cuda-aa" if args.variant == "aa" else "cuda-naive"
    block = tuple(int(v) for v in args.block.split("x"))
    solver = lbm.make_solver(params, backend=backend, launch=args.launch, block=block)
    steps = args.steps + (args.steps % solver.step_multiple)
    warm = args.warmup + (args.warmup % solver.step_multiple)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    stream = torch.cuda.current_stream()
    # The CUDA graph that chunks of GRAPH_CHUNK steps replay is captured first:
    # capture records the launches without running them, so the warm-up below
    # is exactly the requested number of steps.
    if solver.use_graph and steps >= solver.GRAPH_CHUNK:
        solver._graph(solver.GRAPH_CHUNK)
    solver._advance(warm)
    barrier()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
    except Exception:  # noqa: BLE001
        uuid = None
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_steps() -> float:
        """One timed region of exactly `steps` steps between barriers; the slowest rank's milliseconds."""
        barrier()
        start.record(stream)
        solver._advance(steps)
        stop.record(stream)
        stop.synchronize()
        barrier()
        return max_over_ranks(start.elapsed_time(stop), world, device)

    # The timed region (exactly `steps` steps) is repeated until the repeats
    # span at least MIN_TIMED_SECONDS, so that the clock sampler sees the GPU
    # under load; the repeat count follows from the first repeat's max over
    # ranks, the same on every rank. `ms_per_step` is the median repeat.
    with ClockSampler(uuid, interval_ms=50) as clocks:
        times = [timed_steps()]
        repeats = int(min(MAX_REPEATS, max(MIN_REPEATS, math.ceil(args.repeat_seconds * 1e3 / max(times[0], 1e-3)))))
        for _ in range(repeats - 1):
            times.append(timed_steps())
    solver.time_step += warm + steps * len(times)
    solver._check_health()
    ms = statistics.median(times)
    mlups = whole_job_mlups(nodes, steps, ms, world)
    ms_step = ms / steps

    # ---- the public run loop: the state check (NaN / rho <= 0 scan, float64 mass) fused into the
    # last step of every check_every-step chunk, read back with one small copy per chunk
    run_loop = None
    if world == 1 and args.run_loop:
        loop_steps, check_every = 2000, 500
        loop_steps += loop_steps % solver.step_multiple
        solver.run(check_every, check_every=check_every)  # warm: the checked-step kernel
        barrier()
        start.record(stream)
        solver.run(loop_steps, check_every=check_every)
        stop.record(stream)
        stop.synchronize()
        loop_ms = start.elapsed_time(stop) / loop_steps
        run_loop = {"ms_per_step": round(loop_ms, 5), "steps": loop_steps, "check_every": check_every,
                    "vs_plain_steps": round(loop_ms / ms_step, 4), "mass": solver.mass,
                    "what": "solver.run(steps, check_every) through the public API; CUDA events"}

    # ---- end to end through the public API, host buffers in pinned memory
    e2e = None
    if not args.no_e2e:
        shape = params.shape
        rho_h = torch.ones(shape, dtype=torch.float64).pin_memory()
        u_h = [torch.zeros(shape, dtype=torch.float64).pin_memory() for _ in range(3)]
        chunk = args.e2e_chunk + args.e2e_chunk % solver.step_multiple
        for _ in range(2):  # warm-up: graphs, and the two page-locked readout blocks the loop alternates
            solver.initialize(rho_h, *u_h)
            solver.run(chunk, check_every=chunk)
            fields = solver.macroscopic()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_iters):
            solver.initialize(rho_h, *u_h)
            solver.run(chunk, check_every=chunk)
            fields = solver.macroscopic()
        barrier()
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, world, device)
        h2d = 4 * nodes * 8
        d2h = 4 * nodes * fields.rho.itemsize + 16
        e2e = {"value": round(world * nodes * chunk * args.e2e_iters / dt / 1e6, 2), "unit": "MLUPS",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "step": f"initialize(pinned host rho,u f64) + run({chunk}) + macroscopic() to host",
               "iters": args.e2e_iters}

    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    bpu = 2 * 19 * BYTES[args.storage]
    achieved = mlups / world * 1e6 * bpu / 1e9
    traffic = profile_traffic(args.variant, args.storage)
    copy_now = copy_peak_gbs(torch, device)
    res = solver.kernel_resources()
    n_fluid = int(params.fluid.sum())
    line = {
        "metric": METRIC, "value": round(mlups, 2), "unit": "MLUPS", "n_gpus": world, "steps": steps,
        "warmup": warm, "ms_per_step": round(ms_step, 5), "higher_is_better": True, "scaling": "weak",
        "timing": {"repeats": len(times), "region_steps": steps, "stat": "median over repeats of the timed region",
                   "ms_per_step_min": round(min(times) / steps, 5), "ms_per_step_max": round(max(times) / steps, 5),
                   "seconds_timed": round(sum(times) / 1e3, 3), "launches_per_region": steps,
                   "launches_all_repeats": steps * len(times)},
        "vs_baseline": None, "dtype": DTYPE_TAG[args.storage], "data": "synthetic (analytic duct set-up, fluid at rest)",
        "config": workload_config(args),
        "roofline": {"bound": "hbm", "kernel": step_kernel_name(args),
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_update": bpu, "copy_peak_in_run_gbs": round(copy_now, 1),
                     "frac_of_copy_in_run": round(achieved / copy_now, 4)},
        "gpu_launches": steps,
        "fluid_nodes": {"count": n_fluid, "mlups": round(mlups * n_fluid / nodes, 2),
                        "note": "value counts every node of the box, as the reference's benchmark does; "
                                "the solid wall layers are not updated"},
        "kernel_resources": res,
        "clocks": clocks.summary(),
    }
    if e2e is not None:
        line["e2e"] = e2e
    if run_loop is not None:
        line["run_loop"] = run_loop
    if args.precision_steps > 0 and world == 1:
        del solver
        torch.cuda.empty_cache()
        study = precision_study(lbm, torch, n, args.precision_steps, args.variant)
        line["storage_precision"] = study
        fp16 = study["float16"]
        line["fp16_store"] = {"mlups": fp16["mlups"], "vs_fp32_mlups": round(fp16["mlups"] / study["float32"]["mlups"], 3),
                              "u_rel_l2_vs_f64": fp16["u_rel_l2_vs_f64"], "u_rel_max_vs_f64": fp16["u_rel_max_vs_f64"],
                              "steps": args.precision_steps}
    if args.configs and world == 1:
        torch.cuda.empty_cache()
        line["tgv"] = tgv_study(lbm, torch)
        line["cylinder"] = cylinder_study(lbm, torch)
    if args.batched and world == 1:
        torch.cuda.empty_cache()
        line["batched"] = batched_study(lbm, torch)
    if args.adjoint and world == 1:
        torch.cuda.empty_cache()
        line["adjoint"] = adjoint_study(lbm, torch)
    if not args.no_cpu_baseline and world == 1:
        mlups_cpu, done, dt, kind = cpu_reference_mlups(n, 8, 3, 1, budget=args.cpu_seconds)
        line["cpu_baseline"] = {"value": round(mlups_cpu, 4), "unit": "MLUPS", "cores": 1, "kind": kind,
                                "sample": f"{n}x{n}x8 slab of the duct, {done} steps in {dt:.1f} s ({CPU_KIND_NOTE[kind]}; "
                                          f"single-threaded element-wise; host has {os.cpu_count()} cores)"}
    print(json.dumps(line), flush=True)


def run_study(args):
    """One configuration study on cuda:0 (for profiling one kernel family at a time)."""
    import torch

    import lbm_b200 as lbm

    torch.cuda.set_device(0)
    k = args.study_steps
    if args.study == "tgv":
        result = tgv_study(lbm, torch, **({"steps": k} if k else {}))
    elif args.study == "cylinder":
        methods = ("bouzidi", "ibm") if args.cylinder_method == "both" else (args.cylinder_method,)
        result = cylinder_study(lbm, torch, methods=methods, **({"steps": k} if k else {}))
    elif args.study == "batched":
        result = batched_study(lbm, torch, **({"steps": k} if k else {}))
    elif args.study == "adjoint":
        kw = {"steps": k, "window": max(1, k // 4), "fd": False} if k else {}
        result = adjoint_study(lbm, torch, **kw)
    elif args.study == "setup":
        result = setup_study(lbm, torch)
    elif args.study == "kernels":
        result = kernels_study(lbm, torch)
    else:
        result = precision_study(lbm, torch, args.n, k or args.precision_steps, args.variant)
    print(json.dumps({"study": args.study, "result": result}), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.study is not None:
        run_study(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()

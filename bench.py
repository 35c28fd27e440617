#!/usr/bin/env python3
"""Benchmark of the batched PSC-IMB step on B200 (one JSON line on rank 0).

Workload ("batch24"): 24 seeded periodic pore windows, edges drawn from
{48, 64, 96, 128, 160}, geometry type skeleton / passive fines / preloaded
fines, 4^3 sub-samples, BGK tau = 0.8, body force 1e-6 along x; FP32
deviation storage; every step is one persistent launch over all windows,
replayed from a captured CUDA graph.  A step is one lattice update of every
window; ``value`` is MLUPS over all ranks.  The populations (about 5 GB per
GPU) exceed the 126 MB L2, so no flush is needed between steps.

Also reported on the same line:
  fp64_plain  -- the same windows solved one at a time in FP64 (deviation
                 storage, one launch per step, no graph): MLUPS, windows/hour
                 at 5000 steps
  perm_error  -- the accuracy gate (<= 1e-4): the benchmark batch's per-window
                 Darcy K in FP32 against FP64 storage at the same step count
                 (1000 steps from rest, both counts printed), and the 96^3
                 packed-bed windows run to steady state in both precisions
  fp64_exact_dropin -- the plain FP64 drop-in (reference arithmetic, per-call
                 diagnostics), one window at a time, and the windows/hour ratio
  e2e         -- MLUPS through the batched C ABI with host buffers: every step
                 uploads each window's particle array and reads back every
                 window's diagnostics (psc_batch_set_particles + psc_batch_step)
  e2e_dropin  -- MLUPS through the drop-in SparsePscD3Q19.collide_stream_psc(),
                 one window per call (particle upload, step, loads,
                 diagnostics read back per call)
  roofline    -- achieved HBM GB/s of the step kernel vs the measured peak
  cpu_baseline-- the NumPy oracle port on this host's cores (bounded sample)

``--impl reference`` times the reference algorithm's CPU implementation (the
NumPy oracle port, run on all host cores) on the same workload instead.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "PSC-IMB MLUPS & %HBM peak, FP32/batched vs plain FP64 at <=1e-4 perm. error"
UNIT = "MLUPS"
TAU = 0.8
FORCE = (1.0e-6, 0.0, 0.0)
SUBSAMPLES = 4
NWIN = 24
STEPS_PER_WINDOW = 5000
# untimed end-to-end iterations before each e2e timing: a drop-in window's reporting step is
# captured as a CUDA graph once its launch arguments repeat, which the first loads call on a
# geometry changes (it writes the loads list the later calls read)
E2E_WARMUP = 6
# algorithmic bytes per lattice update: 19 populations read + 19 written,
# plus the 1-byte solid level (static particles: no solid-velocity field)
BYTES_PER_LUP = {"fp32": 2 * 19 * 4 + 1, "fp64": 2 * 19 * 8 + 1, "fp16": 2 * 19 * 2 + 1, "bf16": 2 * 19 * 2 + 1}


# ---------------------------------------------------------------------------
# CPU side (oracle port) -- runs in spawned worker processes
# ---------------------------------------------------------------------------
def _oracle_worker(args):
    n, parts, steps, warm = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import psc_oracle as orc

    s = orc.OracleSolver(n, parts, tau=TAU, subsamples=SUBSAMPLES, force=FORCE, static_geometry=True)
    for _ in range(warm):
        s.collide_stream_psc()
    t0 = time.perf_counter()
    for _ in range(steps):
        s.collide_stream_psc()
    return n ** 3, steps, time.perf_counter() - t0


def cpu_sample(windows, steps: int, warm: int, procs: int | None = None):
    """Oracle steps on the smallest windows, one process per host core."""
    procs = procs or os.cpu_count() or 1
    small = sorted(windows, key=lambda w: w.n)
    jobs = [(small[k % len(small)].n, small[k % len(small)].particles, steps, warm) for k in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_oracle_worker, jobs)
    wall = time.perf_counter() - t0
    cells = sum(r[0] * r[1] for r in res)
    slowest = max(r[2] for r in res)
    return {
        "value": cells / slowest / 1e6,
        "unit": UNIT,
        "cores": procs,
        "sample": f"{procs} processes x {steps} oracle steps (after {warm} warm-up) on {len(set(j[0] for j in jobs))} "
                  f"window size(s) {sorted(set(j[0] for j in jobs))}^3 of the batch; NumPy single-threaded per process",
        "wall_s": round(wall, 2),
    }


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of one GPU, polled through NVML from a thread every ~1 ms
    (read-only queries), so that even a timed region of a few milliseconds holds several samples.
    ``mark(True)`` / ``mark(False)`` bracket the timed region; ``stop()`` reports the samples taken
    inside it (and says so), else every sample of the sampler's window.  Falls back to
    ``nvidia-smi -lms 100`` when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NVML_REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                    ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, index: int, period_s: float = 0.001):
        self.index = index
        self.period = period_s
        self.proc = None
        self.thread = None
        self.samples = []  # (t, sm_mhz, sm_max_mhz, reasons bitmask)
        self.region = [None, None]
        self._stop = None
        self.t0 = None

    def _poll(self, nvml, handle):
        import time as _t

        smax = nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                rs = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                self.samples.append((_t.perf_counter(), float(sm), float(smax), int(rs)))
            except Exception:  # a failed query drops one sample
                pass
            self._stop.wait(self.period)

    def start(self):
        import threading

        self.t0 = time.perf_counter()
        try:
            import pynvml as nvml

            nvml.nvmlInit()
            handle = nvml.nvmlDeviceGetHandleByIndex(self.index)
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nvml, handle), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def mark(self, begin: bool):
        self.region[0 if begin else 1] = time.perf_counter()

    def stop(self) -> dict:
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            a, b = self.region
            inside = [s for s in self.samples if a is not None and b is not None and a <= s[0] <= b]
            use = inside or self.samples
            if not use:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            reasons = sorted({name for s in use for name, bit in self.NVML_REASONS if s[3] & bit})
            out = {"sm_mhz": statistics.median(s[1] for s in use), "sm_max_mhz": max(s[2] for s in use),
                   "reasons": reasons, "samples": len(use), "source": "nvml, ~1 ms polling",
                   "window": "timed region" if inside else "whole GPU phase (no sample fell inside the timed region)"}
            if a is not None and b is not None:
                out["timed_region_ms"] = round((b - a) * 1e3, 2)
            return out
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi -lms 100",
                "window": "whole GPU phase (100 ms sampling cannot resolve the timed region)"}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


STEP_KERNELS = {
    "direct": ("psc::k_step_fast", "k_step_batch24.txt"),
    "pair": ("psc::k_step_pair", "k_step_pair_batch24.txt"),
    "tma": ("psc::k_step_tma", "k_step_batch24.txt"),
}


def ncu_traffic(kernel_tag: str, launch_kernel: str = "direct"):
    """DRAM bytes per launch of the step kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / STEP_KERNELS.get(launch_kernel, STEP_KERNELS["direct"])[1]
    if not p.exists() or launch_kernel == "tma":
        return None
    for line in p.read_text().splitlines():
        if line.startswith(f"traffic_bytes_per_launch[{kernel_tag}]"):
            try:
                return float(line.split("=", 1)[1].split()[0])
            except (IndexError, ValueError):
                return None
    return None


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def free_port() -> int:
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return int(s.getsockname()[1])


def spawn_ranks(n: int, cmd: list[str], timeout_s: float | None = None) -> int:
    """Run ``cmd`` as ``n`` local ranks (one process per GPU), the way torchrun would: RANK,
    LOCAL_RANK, WORLD_SIZE, LOCAL_WORLD_SIZE and MASTER_ADDR / MASTER_PORT (127.0.0.1, a free port)
    set per process.  Rank 0 keeps this process's stdout (it prints the JSON line); the other
    ranks' stdout is discarded, their stderr kept.  If a rank fails, the others are terminated
    after a grace period (their next collective would wait for it until the process-group
    timeout).  Returns the first non-zero exit code, else 0."""
    port = free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(cmd, env=env, stdout=None if r == 0 else subprocess.DEVNULL))
    t0 = time.monotonic()
    failed_at = None
    while True:
        codes = [p.poll() for p in procs]
        if all(c is not None for c in codes):
            break
        if failed_at is None and any(c not in (None, 0) for c in codes):
            failed_at = time.monotonic()
        late = failed_at is not None and time.monotonic() - failed_at > 30.0
        over = timeout_s is not None and time.monotonic() - t0 > timeout_s
        if late or over:
            for p in procs:
                if p.poll() is None:
                    p.terminate()
            for p in procs:
                try:
                    p.wait(timeout=30)
                except subprocess.TimeoutExpired:
                    p.kill()
                    p.wait()
            break
        time.sleep(0.05)
    codes = [p.returncode for p in procs]
    return next((c for c in codes if c != 0), 0)


def dist_setup(backend: str | None = None):
    """(world, rank, local rank) from the torchrun environment; initialises the process group when
    world > 1 (NCCL on GPUs, gloo for CPU-only processes) with a short timeout."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
    if backend == "nccl":
        torch.cuda.set_device(local if world > 1 else 0)
    if world > 1:
        import datetime

        import torch.distributed as dist

        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return world, rank, local


def _reduce_scalar(x: float, world: int, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, world: int) -> float:
    return _reduce_scalar(x, world, "max")


def sum_over_ranks(x: float, world: int) -> float:
    return _reduce_scalar(x, world, "sum")


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def timed(fn, world):
    import torch

    barrier(world)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    barrier(world)
    return a.elapsed_time(b)


def run_fp64_plain(windows, steps: int, warm: int):
    """Each window alone in FP64 (one launch per step, no graph)."""
    import torch

    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    per_window = []
    for w in windows:
        b = PscBatch([WindowSpec(w.n, w.particles, TAU, FORCE, SUBSAMPLES)], precision="fp64", graph_steps=0)
        b.run(warm)
        ms = timed(lambda: b.run(steps), 1)
        per_window.append(ms / steps)
        del b
        torch.cuda.empty_cache()
    return per_window


def run_fp64_exact_dropin(windows, steps: int, warm: int = E2E_WARMUP):
    """Per-window ms/step of the plain FP64 drop-in (reference arithmetic, per-call diagnostics).
    The untimed calls cover the first launches and one CUDA-graph capture per buffer parity."""
    import torch

    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19

    per_window = []
    for w in windows:
        s = SparsePscD3Q19(w.n, w.particles, tau=TAU, subsamples=SUBSAMPLES, static_geometry=True,
                           precision="fp64-exact", force=FORCE)
        for _ in range(warm):
            s.collide_stream_psc()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            s.collide_stream_psc()
        torch.cuda.synchronize()
        per_window.append((time.perf_counter() - t0) / steps * 1e3)
        del s
        torch.cuda.empty_cache()
    return per_window


def run_e2e_dropin(windows, steps: int):
    """MLUPS through the drop-in class, one window at a time (host particle upload + diagnostics read back per call)."""
    import torch

    from particuology_hydraulic_penalty_b200 import SparsePscD3Q19
    from particuology_hydraulic_penalty_b200 import _native as nat

    solvers = [SparsePscD3Q19(w.n, w.particles, tau=TAU, subsamples=SUBSAMPLES, static_geometry=True,
                              precision="fp32", force=FORCE) for w in windows]
    for _ in range(E2E_WARMUP):  # untimed: voxelisation, first launches, one graph capture per buffer parity
        for s in solvers:
            s.collide_stream_psc()
    torch.cuda.synchronize()
    h2d = sum(int(w.particles.nbytes) for w in windows)
    d2h = len(windows) * (2 * nat.NRED + nat.NDIAG) * 8  # reductions + diagnostics of each call
    t0 = time.perf_counter()
    for _ in range(steps):
        for s in solvers:
            s.collide_stream_psc()
    wall = time.perf_counter() - t0
    cells = sum(w.n ** 3 for w in windows)
    del solvers
    torch.cuda.empty_cache()
    return {"value": round(cells * steps / wall / 1e6, 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "api": "SparsePscD3Q19(precision='fp32').collide_stream_psc() per window (one psc_step call each), "
                   "static geometry", "steps": steps}


def run_e2e_batch(windows, steps: int, graph_steps: int, world: int = 1):
    """MLUPS through the batched C ABI with host buffers: every step uploads each window's particle
    array (psc_batch_set_particles_all) and reads back every window's diagnostics (psc_batch_step with
    PSC_RUN_DIAG: particle loads, post-stream reductions, Darcy K).  With several ranks each rank runs
    its own batch; the ranks start the timed loop together (barrier) and the job's rate is all ranks'
    cells over the slowest rank's wall time; the copied bytes are summed over the ranks."""
    import torch

    from particuology_hydraulic_penalty_b200 import _native as nat
    from particuology_hydraulic_penalty_b200.handle import BatchHandle, make_config

    dev = torch.cuda.current_device() if torch.cuda.is_available() else 0  # this rank's GPU
    cfgs = [make_config((w.n,) * 3, tau=TAU, force=FORCE, subsamples=SUBSAMPLES, store=nat.STORE_F32,
                        device_index=dev) for w in windows]
    b = BatchHandle(cfgs, graph_steps=graph_steps)
    for k, w in enumerate(windows):
        b.set_particles(k, w.particles)
    b.step(3, nat.RUN_DIAG)  # voxelisation and first launches outside the timed region
    h2d = sum(int(w.particles.nbytes) for w in windows)
    d2h = len(windows) * (2 * nat.NRED + nat.NDIAG) * 8
    arrays = [w.particles for w in windows]
    for _ in range(E2E_WARMUP):  # untimed iterations of the timed loop body
        b.set_particles_all(arrays)
        b.step(1, nat.RUN_DIAG)
    k_sum = 0.0
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        b.set_particles_all(arrays)
        st = b.step(1, nat.RUN_DIAG)
        k_sum += st[0].diag.permeability
    wall = max_over_ranks(time.perf_counter() - t0, world)
    cells = sum_over_ranks(float(sum(w.n ** 3 for w in windows)), world)
    h2d = int(sum_over_ranks(float(h2d), world))
    d2h = int(sum_over_ranks(float(d2h), world))
    finite = sum_over_ranks(0.0 if np.isfinite(k_sum) else 1.0, world) == 0.0
    b.close()
    torch.cuda.empty_cache()
    return {"value": round(cells * steps / wall / 1e6, 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "finite": bool(finite), "ranks": world,
            "api": "C ABI psc_batch_set_particles_all (every window) + psc_batch_step(1, PSC_RUN_DIAG) per step: "
                   "host particle arrays in, per-window diagnostics and Darcy K out, one persistent launch for "
                   "all windows", "steps": steps}


ACCURACY_STEPS = 1000  # equal-step FP32 / FP64 comparison of the benchmark batch


def perm_error_equal_steps(specs, batch32, graph_steps: int, steps: int = ACCURACY_STEPS) -> dict:
    """Darcy K of the FP32 batch against the same windows in FP64 storage at the SAME step count from
    rest: the FP32 batch (the timed one) is advanced to ``steps`` (or kept where it is if it went
    further), a fresh FP64 batch runs exactly as many; both counts are reported."""
    import torch

    from particuology_hydraulic_penalty_b200.batch import PscBatch

    target = max(int(steps), batch32.steps_done)
    batch32.run(target - batch32.steps_done)
    k32 = batch32.permeability()
    b64 = PscBatch(specs, precision="fp64", graph_steps=graph_steps)
    b64.run(target)
    k64 = b64.permeability()
    s32, s64 = batch32.steps_done, b64.steps_done
    del b64
    torch.cuda.empty_cache()
    if s32 != s64:
        raise RuntimeError(f"FP32 / FP64 step counts differ: {s32} vs {s64}")
    err = np.abs(k32 - k64) / np.maximum(np.abs(k64), 1e-300)
    return {"steps_fp32": int(s32), "steps_fp64": int(s64), "max": float(err.max()),
            "median": float(np.median(err)), "windows": len(err),
            "what": "per-window Darcy K, FP32 deviation storage vs FP64 deviation storage, same windows, "
                    "same step count from rest"}


def perm_error_steady(tol: float = 1.0e-8, check_every: int = 200, max_steps: int = 100000) -> dict:
    """The packed-bed permeability case (one seeded 96^3 window in its three geometries) run to
    steady state in FP32 and in FP64 storage; relative K error of FP32 against FP64."""
    import torch

    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = [wgen.make_window(96, kind, 1000) for kind in wgen.GEOMETRY_TYPES]
    specs = [WindowSpec(w.n, w.particles, TAU, FORCE, SUBSAMPLES, name=w.kind) for w in wins]
    res = {}
    for prec in ("fp64", "fp32"):
        b = PscBatch(specs, precision=prec, graph_steps=20)
        r = b.run_to_convergence(tol=tol, check_every=check_every, max_steps=max_steps)
        res[prec] = r
        del b
        torch.cuda.empty_cache()
    k64, k32 = res["fp64"]["permeability"], res["fp32"]["permeability"]
    err = np.abs(k32 - k64) / np.abs(k64)
    return {"windows": [w.kind for w in wins], "rel_err": [float(e) for e in err], "max": float(err.max()),
            "K_fp64": [float(k) for k in k64],
            "steps_fp64": [int(s) for s in res["fp64"]["steps"]], "steps_fp32": [int(s) for s in res["fp32"]["steps"]],
            "converged": bool(res["fp64"]["converged"].all() and res["fp32"]["converged"].all()),
            "criterion": f"per-step relative change of K < {tol:g}, checked every {check_every} steps",
            "what": "96^3 skeleton / passive fines / preloaded fines, S=4, tau=0.8, F=1e-6 x, each precision "
                    "run to its own steady state"}


STORE_BYTES = {"fp32": 4, "fp64": 8, "fp16": 2, "bf16": 2}  # bytes per stored population
WORKLOADS = {
    "batch24": "batch24: 24 uneven periodic pore windows, edges {{48,64,96,128,160}}, S=4, BGK tau=0.8, "
               "F=1e-6 x, {prec} deviation storage, one persistent launch per step, CUDA graph",
    "window96x3": "window96x3: one seeded 96^3 window in its three geometries (skeleton, passive fines, "
                  "preloaded fines), S=4, BGK tau=0.8, F=1e-6 x, {prec} deviation storage, one launch per step",
    "batch8": "batch8: the first 8 windows of batch24 (a profiling case: about 1.3 GB on the device, fields "
              "larger than the L2), {prec} deviation storage, one persistent launch per step, CUDA graph",
}


def make_windows(workload: str, rank: int):
    from particuology_hydraulic_penalty_b200 import windows as wgen

    if workload == "batch24":
        return wgen.batched_windows(NWIN, seed0=NWIN * rank)
    if workload == "batch8":
        return wgen.batched_windows(NWIN, seed0=NWIN * rank)[:8]
    seed = 1000 + rank
    return [wgen.make_window(96, kind, seed) for kind in wgen.GEOMETRY_TYPES]


def run_ours(args):
    import torch

    world, rank, local = dist_setup()
    from particuology_hydraulic_penalty_b200 import windows as wgen
    from particuology_hydraulic_penalty_b200.batch import PscBatch, WindowSpec

    wins = make_windows(args.workload, rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(wins, steps=args.cpu_steps, warm=1)
        cpu["cpu_model"] = cpu_model()

    specs = [WindowSpec(w.n, w.particles, TAU, FORCE, SUBSAMPLES, name=w.kind) for w in wins]
    from particuology_hydraulic_penalty_b200 import _native as nat

    kernel = {"auto": nat.KERNEL_AUTO, "direct": nat.KERNEL_DIRECT, "tma": nat.KERNEL_TMA,
              "pair": nat.KERNEL_PAIR}[args.kernel]
    batch = PscBatch(specs, precision=args.precision, graph_steps=args.graph_steps, kernel=kernel)
    tuned = None
    if not args.no_autotune and args.kernel == "auto":
        from particuology_hydraulic_penalty_b200 import autotune

        # the launch (kernel, persistent grid, TMA rows and stages) chosen by the project's autotuner,
        # measured afresh on this GPU (no cache); tuning leaves the simulation state untouched
        tuned = autotune.tune(batch, steps=20, use_cache=False)
    clocks = ClockSampler(local)
    clocks.start()
    batch.prepare()  # graph capture of both buffer parities happens here, outside the timed region
    batch.run(args.warmup)
    torch.cuda.synchronize()

    def timed_steps():
        clocks.mark(True)
        batch.run(args.steps)

    ms = timed(timed_steps, world)
    clocks.mark(False)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world)
    red = batch.observe()
    nonfinite = bool(batch.nonfinite(red).any())
    cells_rank = batch.total_cells
    cells_all = sum_over_ranks(float(cells_rank), world)
    value = cells_all * args.steps / (ms_max * 1e-3) / 1e6
    lups_rank = cells_rank * args.steps / (ms * 1e-3)
    bpl = BYTES_PER_LUP[args.precision]
    peak, peak_kind = measured_peak_hbm()
    achieved = bpl * lups_rank / 1e9
    launch_kernel = batch.launch_config()["kernel"]
    traffic = ncu_traffic(args.precision, launch_kernel)
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else args.precision,
        "data": "synthetic (seeded FCC skeleton / passive / preloaded pore windows; the reference's dumps are not shipped)",
        "config": {"workload": WORKLOADS[args.workload].format(prec=args.precision.upper()),
                   "windows_per_gpu": len(wins), "cells_per_gpu": cells_rank,
                   "l2": f"populations (~{2 * 19 * cells_rank * STORE_BYTES[args.precision] / 1e9:.1f} GB/GPU, two "
                         f"buffers) exceed the 126 MB L2; no flush", "parallelism": f"window-parallel x{world}",
                   "graph_steps": args.graph_steps, "launch": batch.launch_config(),
                   "autotuned": tuned is not None,
                   "autotune": None if tuned is None else {
                       "candidates": len(tuned.get("candidates", [])), "chosen_ms_per_step": tuned.get("ms_per_step"),
                       "default_pair_ms_per_step": next((t for c, t in tuned.get("candidates", [])
                                                         if c.get("kernel") == "pair" and not c.get("grid_ctas")),
                                                        None)}},
        "gpu_launches": args.steps * batch.launches_per_step(),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic, "bytes_per_lup": bpl,
                     "kernel": STEP_KERNELS[launch_kernel][0] + " (fused pull-stream + PSC collide, deviation "
                               "storage); avg launch = timed region / steps"},
        "clocks": clk,
        "nonfinite": nonfinite,
    }
    if rank == 0 and world == 1 and not args.no_fp64:
        # the accuracy gate: FP32 vs FP64 permeability at equal step counts, and at steady state
        acc_equal = perm_error_equal_steps(specs, batch, args.graph_steps) if args.precision == "fp32" else None
        del batch
        torch.cuda.empty_cache()
        acc_steady = perm_error_steady() if args.precision == "fp32" and not args.no_steady else None
        per_ms = run_fp64_plain(wins, steps=args.fp64_steps, warm=3)
        t_plain_h = sum(STEPS_PER_WINDOW * m * 1e-3 for m in per_ms) / 3600.0
        t_batch_h = STEPS_PER_WINDOW * (ms / args.steps) * 1e-3 / 3600.0  # all windows advance together
        exact_ms = run_fp64_exact_dropin(wins, steps=args.fp64_steps)
        t_exact_h = sum(STEPS_PER_WINDOW * m * 1e-3 for m in exact_ms) / 3600.0
        out["fp64_exact_dropin"] = {
            "what": "plain FP64 form: SparsePscD3Q19(precision='fp64-exact').collide_stream_psc() per window, "
                    "reference arithmetic and per-call diagnostics, one window at a time",
            "mlups": round(sum(w.n ** 3 for w in wins) / (sum(exact_ms) * 1e-3) / 1e6, 1),
            "windows_per_hour": round(len(wins) / t_exact_h, 1),
            "fp32_batched_over_this_windows_per_hour": round(t_exact_h / t_batch_h, 2),
        }
        out["fp64_plain"] = {
            "mlups": round(sum(w.n ** 3 for w in wins) / (sum(per_ms) * 1e-3) / 1e6, 1),
            "windows_per_hour": round(len(wins) / t_plain_h, 1),
            "fp32_batched_windows_per_hour": round(len(wins) / t_batch_h, 1),
            "windows_per_hour_ratio": round(t_plain_h / t_batch_h, 3),
            "steps_per_window_assumed": STEPS_PER_WINDOW,
        }
        if acc_equal is not None:
            out["fp64_plain"]["perm_rel_err_max_fp32_vs_fp64"] = acc_equal["max"]
            out["perm_error"] = {"bound": 1e-4, "batch_equal_steps": acc_equal, "steady_state": acc_steady,
                                 "within_bound": bool(acc_equal["max"] <= 1e-4 and
                                                      (acc_steady is None or acc_steady["max"] <= 1e-4))}
    if not args.no_e2e:  # every rank: its own batch through the C ABI, timed together
        out["e2e"] = run_e2e_batch(wins, steps=args.e2e_steps, graph_steps=args.graph_steps, world=world)
        if world == 1:
            out["e2e_dropin"] = run_e2e_dropin(wins, steps=max(3, args.e2e_steps // 4))
    else:
        out["e2e"] = None
    if cpu is not None:
        out["cpu_baseline"] = {"value": round(cpu["value"], 4), "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                               "sample": cpu["sample"], "cpu_model": cpu["cpu_model"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_reference(args):
    """The reference algorithm on the host cores (the oracle port), same workload and metric."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wins = make_windows(args.workload, 0)
    procs = os.cpu_count() or 1
    small = sorted(wins, key=lambda w: w.n)
    jobs = [(small[k % len(small)].n, small[k % len(small)].particles, args.steps, args.warmup) for k in range(procs)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_oracle_worker, jobs)
    cells = sum(r[0] * r[1] for r in res)
    slowest = max(r[2] for r in res)
    value = cells / slowest / 1e6
    sample = (f"{procs} processes x {args.steps} timed steps (after {args.warmup} warm-up) of the NumPy oracle "
              f"port on the batch's smallest window size(s) {sorted(set(j[0] for j in jobs))}^3; "
              f"one NumPy thread per process")
    out = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(slowest / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
        "data": "synthetic (seeded pore windows)",
        "config": {"workload": args.workload + " sample (smallest windows), reference algorithm on host cores",
                   "cpu_model": cpu_model()},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="batch24")
    ap.add_argument("--precision", choices=["fp32", "fp64", "fp16", "bf16"], default="fp32")
    ap.add_argument("--graph-steps", type=int, default=20)
    ap.add_argument("--kernel", choices=["auto", "direct", "tma", "pair"], default="auto",
                    help="auto: the pair kernel when every window has an even nz, else direct")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the project autotuner (default with --kernel auto: it picks the launch before the "
                         "timed run)")
    ap.add_argument("--fp64-steps", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-steady", action="store_true", help="skip the steady-state FP32/FP64 permeability leg")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.gpus < 1:
        ap.error("--gpus must be >= 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not under torchrun: start one rank per GPU here, each running this same command line
        sys.exit(spawn_ranks(args.gpus, [sys.executable, str(Path(__file__).resolve()), *sys.argv[1:]]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        print(f"bench.py: WORLD_SIZE={world} overrides --gpus {args.gpus}", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

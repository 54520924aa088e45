"""Benchmark of the B200 DIM step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c1|c2|c0|c3|c4|e2|e3]
    python bench.py --impl reference ...      # the reference's own CPU code

A step is one DIM time step (CFL reduction, one split sweep per axis, a
boundary fill after each) over the whole grid of the workload:

  c1  2D shock-bubble, 1024x512, two materials (the default: the metric's
      configuration that fits one GPU);
  c2  3D bubble cloud, 512^3, two materials;
  c0  1D two-material Riemann tube, 1000 cells;
  c3  256 uneven 2D instances in one persistent batch (solves/s);
  c4  the serving loop (p50 / p99 latency, solves/s);
  e2  single-material Euler step (the sharp-interface solver's no-level-set
      path), 2D blast 2048x2048;  e3  the same, 3D 256^3.

value  = cell updates per second with the state resident in HBM (CUDA events
         on the session's stream, one event pair per step; the L2 is flushed
         between steps when the state fits in it);
e2e    = the same metric through the C-ABI with host buffers: every step
         uploads the state from pinned host memory, steps, and downloads the
         new state and dt (dim::advance_one_step's by-value contract);
roofline = the sweep kernel's algorithmic bytes (read + write of the V-double
         state per cell) over its average event-timed duration, against the
         measured HBM copy bandwidth.
Multi-GPU: the single-grid step does not shard; N GPUs run N replicas
("scaling": "weak") and value is the sum over ranks / the slowest rank.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DIM cell-updates/s"
UNIT = "cell-updates/s"

WORKLOADS = {
    "c1": ("2D shock-bubble 1024x512, 2 materials, Mach 1.22, CFL 0.8", 0.8),
    "c2": ("3D bubble cloud 512^3, 64 air bubbles in stiffened water, CFL 0.6", 0.6),
    "c0": ("1D two-material Riemann tube 1000 cells, CFL 0.8", 0.8),
    "c4": ("Poisson stream of DIM requests: 40% 1D N in [256,8192], 60% 2D sides in [128,2048], "
           "steps in [100,2000], 150 GB budget", 0.6),
    "c3": ("256 independent 2D instances, sides log-uniform in [64,1024], Riemann or bubble, CFL 0.6", 0.6),
    "e2": ("single-material Euler step (no level set): 2D blast 2048x2048, ideal gas, CFL 0.6", 0.6),
    "e3": ("single-material Euler step (no level set): 3D blast 256^3, ideal gas, CFL 0.6", 0.6),
}
EULER_WORKLOADS = ("e2", "e3")


def make_workload(name: str, scale: int = 1):
    from diffuse_vs_gfm_mms_b200 import workloads as W
    if name == "c1":
        return W.shock_bubble_2d(N=(1024 // scale, 512 // scale))
    if name == "c2":
        n = 512 // scale
        return W.bubble_cloud_3d(N=(n, n, n), nbubbles=64)
    if name == "c0":
        return W.riemann(seed=0, N=(1000,))
    if name == "e2":
        return W.euler_blast(N=(2048 // scale, 2048 // scale), seed=0)
    if name == "e3":
        return W.euler_blast(N=(256 // scale,) * 3, seed=0)
    raise SystemExit(f"unknown workload {name}")


def device_workload(name: str, scale: int = 1):
    """(desc, init): the workload's descriptor and a function that writes its
    initial field into a session.  c1 and c2 are generated on the device
    (dimgpu_init_shock_bubble / dimgpu_init_bubble_cloud, the same bits as
    the host generators); the others are built on the host and uploaded."""
    from diffuse_vs_gfm_mms_b200 import workloads as W
    if name == "c1":
        d, ic = W.shock_bubble_2d_setup(N=(1024 // scale, 512 // scale))
        return d, lambda s: s.init_shock_bubble(ic)
    if name == "c2":
        n = 512 // scale
        d, ic, bubbles = W.bubble_cloud_3d_setup(N=(n, n, n), nbubbles=64)
        return d, lambda s: s.init_bubble_cloud(ic, bubbles)
    d, U = make_workload(name, scale)
    return d, lambda s: s.upload(U)


def reference_sample(name: str):
    """What the CPU reference runs for a workload: the whole grid wherever
    the reference can hold and step it in seconds (c0, c1, e2); a block of
    the grid at the same spacing where it cannot (c2 at 512^3 needs ~95 GB of
    host memory, e3 ~7 s per step)."""
    from diffuse_vs_gfm_mms_b200 import workloads as W
    if name in ("c0", "c1", "e2"):
        d, U = make_workload(name)
        return d, U, "the whole grid"
    if name == "c2":
        d, U = W.bubble_cloud_3d(N=(64, 64, 64), nbubbles=64)
        d.dx[0] = d.dx[1] = d.dx[2] = 1.0 / 512
        return d, U, "64^3 block of the 512^3 case (same spacing, 64 bubbles)"
    if name == "e3":
        d, U = make_workload(name)
        V = d.nvar
        U4 = U.reshape(V, 256, 256, 256)[:, 112:144, :, :]
        d2 = d.copy()
        d2.N[2] = 32
        return d2, np.ascontiguousarray(U4.reshape(V, -1)), "256x256x32 slab through the blast centre"
    raise SystemExit(f"no CPU reference for workload {name}")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_figure(key: str, workload: str):
    """A per-launch figure from the committed ncu summaries under profiles/:
    a line `<key> <workload> <value>` (workload `c1`, or `c1-mixed` for the
    mixed-precision form)."""
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                m = re.match(r"\s*" + re.escape(key) + r"\s+(\S+)\s+([0-9.eE+]+)", line)
                if m and m.group(1) == workload:
                    return float(m.group(2)), os.path.relpath(path, ROOT)
    return None, None


def ncu_traffic(workload: str, ncell: int):
    """DRAM bytes (read + write) per sweep launch (all kernels of one sweep):
    the committed per-cell figure times the cells of this run."""
    per_cell, src = _profile_figure("traffic_bytes_per_cell_sweep", workload)
    return (per_cell * ncell if per_cell else None), src


def ncu_fp64_flops_per_cell(workload: str):
    """FP64 operations per cell and sweep (DADD + DMUL + 2 DFMA thread
    instructions of one sweep's kernels, divided by the cells swept)."""
    return _profile_figure("fp64_flops_per_cell_sweep", workload)


def fp64_peak():
    """Measured FP64 throughput of this GPU: a DFMA loop with eight
    independent chains per thread on every SM (libdimprobe.so), timed with
    CUDA events; the best of five launches, in FLOP/s (2 per DFMA)."""
    import ctypes as C
    path = os.path.join(ROOT, "diffuse_vs_gfm_mms_b200", "libdimprobe.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    inst, flops = C.c_double(), C.c_double()
    if lib.dimprobe_fp64_peak(5, C.byref(inst), C.byref(flops)) != 0:
        return None
    return flops.value


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    A thread reads NVML (the library nvidia-smi reports from) every 2 ms, so
    that even a timed region of a few milliseconds holds several samples;
    without NVML, nvidia-smi is polled every 200 ms and the region may fall
    between two of its samples."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.thread = None
        self.path = os.path.join("/tmp", f"dimgpu_clocks_{os.getpid()}.csv")
        self.sm, self.smax, self.reasons = [], None, set()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        masks = [(name, getattr(nv, attr, bit)) for name, attr, bit in self.REASONS]
        while not self.stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                bits = get_reasons(h)
                for name, m in masks:
                    if bits & m:
                        self.reasons.add(name)
            except Exception:
                pass
            self.stop.wait(0.002)

    def __enter__(self):
        try:
            import threading
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.thread:
            sm = self.sm
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "samples": len(sm), "source": "nvml every 2 ms", "reasons": sorted(self.reasons)}
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = [r[0] for r in self.REASONS]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "source": "nvidia-smi every 200 ms", "reasons": sorted(reasons)}


def max_over_ranks(values, device="cuda"):
    """Element-wise maximum of per-rank timings over the process group (the
    slowest rank sets a replica run's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_value(world: int, cells: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput of N replicas: every rank advanced `cells` cells
    `steps` times; the job took as long as its slowest rank."""
    return world * cells * steps / (max_ms * 1e-3)


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_rate(workload: str, steps: int, warmup: int = 1, repeats: int = 3):
    """The reference's OpenMP code (oracle/_ref) on all host cores, run the
    way its performance suite runs it (scripts/run_report2_local.sh:13-14,
    tools/quant/runner.hpp:326-333): the runner's OpenMP settings, `warmup`
    untimed steps, then `repeats` timed repeats of `steps` steps from the
    same warmed state, and the median rate.  Falls back to the C
    restatement where the reference was not built."""
    nthreads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(nthreads))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    os.environ.setdefault("OMP_SCHEDULE", "guided,1")
    os.environ.setdefault("OMP_DYNAMIC", "FALSE")
    from oracle import oracle as O
    if workload in EULER_WORKLOADS:
        kind = "reference" if os.path.exists(O.EREF_SO) else "port"
        chk = O.EulerChecker(kind)
    else:
        kind = "reference" if O.reference_available() else "port"
        chk = O.reference() if kind == "reference" else O.port()
    chk.set_threads(nthreads)
    d, U, sample = reference_sample(workload)
    cfl = WORKLOADS[workload][1]
    if warmup:
        U, _ = chk.advance(d, U, cfl, 1e300, warmup)
    secs = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        chk.advance(d, U, cfl, 1e300, steps)
        secs.append(time.perf_counter() - t0)
    el = float(np.median(secs))
    rate = d.ncell * steps / el
    cores = chk.max_threads() if hasattr(chk, "max_threads") else (nthreads if kind == "reference" else 1)
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{sample} ({d.ncell} cells); {warmup} warm-up step(s), then the median of {repeats} "
                      f"repeats of {steps} steps", "seconds": el, "cells": d.ncell}


def run_reference(args):
    world, rank, _ = dist_init()
    if rank != 0:
        return
    steps = max(1, args.steps)
    cb = cpu_reference_rate(args.workload, steps, warmup=1, repeats=3)
    config = {"workload": WORKLOADS[args.workload][0], "parallelism": "cpu-openmp"}
    if args.workload in ("c0", "c1", "e2"):
        d, _ = make_workload(args.workload)
        config.update({"cells": d.ncell, "components": d.nvar})
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": cb["seconds"] / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config,
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_slabs(args):
    """One grid cut into `--slabs` slabs along its slowest axis
    (dimgpu_slabs_*), every slab on its own GPU where the node has enough,
    else several slabs per GPU; against one session on the whole grid.  Both
    run the same steps; a slab step ends with a host synchronisation (the dt
    minimum over the slabs), so both are timed with the wall clock around
    synchronised steps."""
    import time

    import torch

    from diffuse_vs_gfm_mms_b200.dim import Session, Slabs

    d, U = make_workload(args.workload, args.scale)
    cfl = WORKLOADS[args.workload][1]
    ngpu = max(1, torch.cuda.device_count())
    devices = [k % ngpu for k in range(args.slabs)]

    def timed(obj):
        obj.steps(args.warmup, cfl, 1e300)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            obj.step(cfl, 1e300)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / args.steps

    with Session(d, U) as s:
        one = timed(s)
    with Slabs(d, devices, U) as L:
        sl = timed(L)
    line = {
        "metric": METRIC, "value": d.ncell / sl, "unit": UNIT, "n_gpus": len(set(devices)), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sl * 1e3, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "cells": d.ncell, "slabs": args.slabs,
                   "devices": devices, "parallelism": f"slabs x{args.slabs}"},
        "one_session": {"value": d.ncell / one, "ms_per_step": one * 1e3},
        "timing": "wall clock around host-synchronised steps (both arms)",
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from diffuse_vs_gfm_mms_b200 import native
    from diffuse_vs_gfm_mms_b200.dim import Session

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    d, init = device_workload(args.workload, args.scale)
    if args.precision == "mixed":
        from diffuse_vs_gfm_mms_b200 import abi as _abi
        d.precision = _abi.PRECISION_MIXED
    cfl = WORKLOADS[args.workload][1]
    ncell, V = d.ncell, d.nvar
    state_bytes = ncell * V * 8
    l2_bytes = 126 * 1024 * 1024
    flush_l2 = 2 * state_bytes < 2 * l2_bytes  # both ping-pong buffers could stay resident
    stream = torch.cuda.Stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda") if flush_l2 else None

    s = Session(d)
    init(s)
    if args.schedule == "fused":
        from diffuse_vs_gfm_mms_b200 import abi as _abi
        for direction in range(d.dim):
            s.set_schedule(direction, _abi.SCHEDULE_FUSED)
    U = s.download() if args.precision == "mixed" else None  # the initial field, for the error analysis
    s.set_stream(stream.cuda_stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            s.enqueue_steps(1, cfl, 1e300)
        s.collect()

    # ---- device-resident timing
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    s.profile(True)
    k0 = native.lib().dimgpu_kernel_launches()
    with ClockSampler(local) as clk, torch.cuda.stream(stream):
        for k in range(args.steps):
            if flush is not None:
                flush.zero_()
            evs[k][0].record(stream)
            s.enqueue_steps(1, cfl, 1e300)
            evs[k][1].record(stream)
        stream.synchronize()
    barrier()
    kernels_timed = native.lib().dimgpu_kernel_launches() - k0
    step_ms = [a.elapsed_time(b) for a, b in evs]
    prof = s.profile_read()
    s.profile(False)
    dts = s.collect()
    total_ms = float(sum(step_ms))
    clocks = clk.summary()

    # ---- end to end through the C-ABI with pinned host buffers
    pin_in = torch.empty(V * ncell, dtype=torch.float64, pin_memory=True)
    pin_out = torch.empty(V * ncell, dtype=torch.float64, pin_memory=True)
    pin_in.numpy()[:] = s.download().reshape(-1)
    e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for k in range(max(1, args.warmup)):
            s.upload(pin_in.numpy())
            s.enqueue_steps(1, cfl, 1e300)
            s.collect()
            s.download(pin_out.numpy().reshape(V, ncell))
            pin_in, pin_out = pin_out, pin_in
        barrier()
        for k in range(args.steps):
            if flush is not None:
                flush.zero_()
            e2e_evs[k][0].record(stream)
            s.upload(pin_in.numpy())
            s.enqueue_steps(1, cfl, 1e300)
            s.download(pin_out.numpy().reshape(V, ncell))
            s.collect()
            e2e_evs[k][1].record(stream)
            pin_in, pin_out = pin_out, pin_in
        stream.synchronize()
    barrier()
    e2e_ms = float(sum(a.elapsed_time(b) for a, b in e2e_evs))

    # ---- max over ranks
    if world > 1:
        total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], device="cuda")

    error_vs_fp64 = None
    if args.precision == "mixed":
        # the FP64 path is bit-identical to the oracle: compare the mixed
        # state after the same warm-up + timed + e2e steps with it
        mixed_out = s.download()
        nsteps = args.warmup + args.steps + max(1, args.warmup) + args.steps
        d64 = d.copy()
        d64.precision = 0
        with Session(d64, U) as s64:
            s64.steps(nsteps, cfl, 1e300)
            ref = s64.download()
        den = np.abs(ref).sum(axis=1)
        l1 = np.abs(mixed_out - ref).sum(axis=1) / np.where(den > 0, den, 1.0)
        linf = np.abs(mixed_out - ref).max(axis=1) / np.maximum(np.abs(ref).max(axis=1), 1e-300)
        # a momentum component that is zero in exact arithmetic (its L1 below
        # 1e-6 of the largest momentum component's) is also scored against
        # the momentum scale, where its own L1 is round-off
        mom = slice(d.nmat, d.nmat + d.dim)
        den2 = den.copy()
        scale = den2[mom].max()
        den2[mom] = np.where(den2[mom] < 1e-6 * scale, scale, den2[mom])
        l1s = np.abs(mixed_out - ref).sum(axis=1) / np.where(den2 > 0, den2, 1.0)
        # the FP64 step's own conditioning on this input: its response to a
        # seeded 1e-15 relative perturbation of the initial state, after the
        # same steps (a stiffened gas far below gamma * p_inf amplifies it)
        rng = np.random.default_rng(7)
        Up = U.copy()
        for c in range(Up.shape[0]):
            Up[c] *= 1.0 + 1e-15 * rng.standard_normal(Up.shape[1:])
        with Session(d64, Up) as sp:
            sp.steps(nsteps, cfl, 1e300)
            pert = sp.download()
        del Up
        sens = np.abs(pert - ref).sum(axis=1) / np.where(den > 0, den, 1.0)
        error_vs_fp64 = {"steps": nsteps, "rel_l1_per_variable": [float(x) for x in l1],
                         "rel_linf_per_variable": [float(x) for x in linf], "max_rel_l1": float(l1.max()),
                         "max_rel_l1_zero_momentum_scored": float(l1s.max()),
                         "fp64_rel_l1_response_to_1e-15_input_perturbation": [float(x) for x in sens]}
    s.close()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    value = replica_value(world, ncell, args.steps, total_ms)
    e2e_value = replica_value(world, ncell, args.steps, e2e_ms)
    sweep = prof["sweep"]
    avg_sweep_s = sweep["ms"] / max(sweep["launches"], 1) * 1e-3
    alg_bytes = 2 * V * 8 * ncell  # read + write of the state, per sweep launch
    achieved = alg_bytes / avg_sweep_s / 1e9
    peak, peak_src = measured_peaks()
    pkey = args.workload + ("-mixed" if args.precision == "mixed" else "") + \
        ("-fused" if args.schedule == "fused" else "")
    traffic, traffic_src = ncu_traffic(pkey, ncell)
    flops_cell, flops_src = ncu_fp64_flops_per_cell(pkey)
    fp64_peak_flops = fp64_peak()
    sched = "mixed staged sweep (mixed_a, mixed_b, mixed_cd, staged_e)" if args.precision == "mixed" else \
        "staged sweep (staged_a..staged_e)"
    if args.schedule == "fused" and args.precision != "mixed":
        sched = "sweep_kernel (fused tile, TMA-staged input)"
    if args.workload in EULER_WORKLOADS:
        sched = "euler_sweep_kernel (fused tile)"

    hbm = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "traffic": traffic, "kernel": sched,
           "note": f"algorithmic {alg_bytes} B per sweep launch (2*V*8*cells); avg sweep "
                   f"{avg_sweep_s * 1e3:.4f} ms over {sweep['launches']} launches; peak {peak_src} (hbm_gbs)"
                   + (f"; traffic from {traffic_src}" if traffic_src else "")}
    fp64 = None
    if flops_cell and fp64_peak_flops:
        fa = flops_cell * ncell / avg_sweep_s / 1e12
        fp = fp64_peak_flops / 1e12
        fp64 = {"bound": "fp64", "achieved": fa, "peak": fp, "unit": "TFLOP/s", "frac": fa / fp,
                "kernel": sched,
                "note": f"{flops_cell:.1f} FP64 operations per cell and sweep (DADD + DMUL + 2 DFMA, ncu, "
                        f"{flops_src}) x {ncell} cells / avg sweep; peak = DFMA loop on every SM measured "
                        f"in this run (libdimprobe.so)"}
    roofline = dict(fp64 if fp64 and fp64["frac"] > hbm["frac"] else hbm)
    roofline["hbm"] = hbm
    roofline["fp64"] = fp64

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": WORKLOADS[args.workload][0], "cells": ncell, "components": V,
            "parallelism": f"replicas x{world}" if world > 1 else "single-gpu",
            "l2": "flushed between steps" if flush_l2 else "state larger than L2",
            "tiles": "default", "last_dt": float(dts[-1]) if len(dts) else None,
        },
        "roofline": roofline,
        "phase_ms": {k: v["ms"] for k, v in prof.items()},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": V * ncell * 8,
                "d2h_bytes_per_step": V * ncell * 8 + 8},
        "gpu_launches": kernels_timed,
        "clocks": clocks,
    }
    if error_vs_fp64 is not None:
        line["dtype"] = "f64 state / f32 flux"
        line["precision"] = "mixed"
        line["error_vs_fp64_oracle"] = error_vs_fp64
    if world == 1 and not args.no_cpu:
        cb = cpu_reference_rate(args.workload, steps=200 if args.workload == "c0" else 3, warmup=1, repeats=3)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_batch(args):
    """Config 3: the batched form against sequential plain solves.

    value = instances solved per second by one batched run of every instance
    for `c3_steps` steps (persistent-grid launches replayed from a CUDA
    graph); the sequential baseline runs a sample of the same instances one
    at a time through the plain session path on the same GPU."""
    import torch

    from diffuse_vs_gfm_mms_b200.batch import Batch
    from diffuse_vs_gfm_mms_b200.dim import Session
    from diffuse_vs_gfm_mms_b200 import workloads as W

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    cfl = WORKLOADS["c3"][1]
    steps = args.c3_steps
    inst = W.batch_instances(args.c3_instances, seed=rank)
    cells = sum(d.ncell for d, _ in inst)
    stream = torch.cuda.Stream()

    # warm-up: kernels loaded, graphs captured on a small batch
    with Batch(2, 2) as w:
        w.set_stream(stream.cuda_stream)
        for d, U in W.batch_instances(4, seed=99, side_range=(64, 96)):
            w.add(d, U, 3 * 8, cfl)
        w.run(3 * 8)

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    with Batch(2, 2) as b, ClockSampler(local) as clk:
        b.set_stream(stream.cuda_stream)
        torch.cuda.synchronize()
        ev[0].record(stream)
        ids = [b.add(d, U, steps, cfl) for d, U in inst]
        ev[1].record(stream)
        b.run(steps)
        ev[2].record(stream)
        outs = [b.download(i, with_dts=False)[0] for i in ids[:: max(1, len(ids) // 8)]]
        ev[3].record(stream)
        stream.synchronize()
    run_ms = ev[1].elapsed_time(ev[2])
    e2e_ms = ev[0].elapsed_time(ev[3])
    clocks = clk.summary()

    # sequential plain solves on a sample of the same instances
    sample = inst[:: max(1, len(inst) // args.c3_sequential)]
    seq_ms = 0.0
    for d, U in sample:
        with Session(d, U) as s:
            s.set_stream(stream.cuda_stream)
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.enqueue_steps(steps, cfl, 1e300)
            z.record(stream)
            s.collect()
            seq_ms += a.elapsed_time(z)
    sample_cells = sum(d.ncell for d, _ in sample)
    seq_cell_rate = sample_cells * steps / (seq_ms * 1e-3)
    # the whole instance set run one at a time, estimated from the sample's
    # per-cell cost (the sample's mean size differs from the set's)
    seq_rate = len(inst) / (cells * steps / seq_cell_rate)
    value = len(inst) / (run_ms * 1e-3)
    if rank == 0:
        line = {
            "metric": "DIM batched solves/s", "value": world * value, "unit": "solves/s", "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": run_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS["c3"][0], "instances": len(inst), "cells": cells,
                       "steps_per_instance": steps, "l2": "state larger than L2"},
            "batched_cell_updates_per_s": cells * steps / (run_ms * 1e-3),
            "sequential_plain": {"solves_per_s": seq_rate, "cell_updates_per_s": seq_cell_rate,
                                 "sample": f"{len(sample)} of the {len(inst)} instances run one at a time; "
                                           "solves/s of the whole set at the sample's cost per cell update"},
            "speedup_vs_sequential_plain": value / seq_rate,
            "e2e": {"value": world * len(inst) / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": sum(U.nbytes for _, U in inst) / steps,
                    "d2h_bytes_per_step": sum(o.nbytes for o in outs) / steps},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def _fifo_latencies(arrivals, service):
    """Latencies of a single server that takes requests first come first
    served: request k starts at max(arrival_k, end of request k-1)."""
    t, out = 0.0, []
    for a, w in sorted(zip(arrivals, service)):
        t = max(t, a) + w
        out.append(t - a)
    return np.array(out)


def run_serving(args):
    """Config 4: the continuous-batching server (dimgpu_server_*) against the
    sequential plain path on the same request stream, at each arrival rate
    of --c4-rates.

    Served: the whole stream of --c4-requests requests per rate, submitted at
    their Poisson arrival times, latency from submission to completion.
    Sequential: each request of a sample (every --c4-seq-every-th) is solved
    alone through a session and timed with CUDA events; the whole stream's
    sequential time is estimated from the sample's device time per cell
    update, per (dimension, precision) class, and its latencies from a
    first-come-first-served queue of those service times at the same
    arrivals.  The decomposition says where the sequential time goes: the
    share of requests that fill the GPU on their own (>= 2^20 cells), whose
    rate batching cannot raise."""
    import torch

    from diffuse_vs_gfm_mms_b200 import serve
    from diffuse_vs_gfm_mms_b200.dim import Session

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    warm = serve.make_requests(4, 0.0, seed=1000, steps_range=(16, 16), n1d_range=(256, 256),
                               side2d_range=(128, 128))
    with serve.Server(hbm_budget_bytes=8e9) as srv:
        srv.serve(warm)
    serve.sequential(warm[:1], stream_handle=stream.cuda_stream)

    # sequential sample: device time per cell update by class
    base = serve.make_requests(args.c4_requests, 1.0, seed=7 + rank)
    sample = base[::max(1, args.c4_seq_every)]
    cost = {}
    for r in sample:
        with Session(r.desc, r.U) as s:
            s.set_stream(stream.cuda_stream)
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s.enqueue_steps(r.steps, r.cfl, r.dt_max)
            z.record(stream)
            s.collect()
            key = (r.desc.dim, r.desc.precision, r.desc.ncell >= (1 << 20))
            t, cu = cost.get(key, (0.0, 0))
            cost[key] = (t + a.elapsed_time(z) * 1e-3, cu + r.desc.ncell * r.steps)

    def service(r):
        key = (r.desc.dim, r.desc.precision, r.desc.ncell >= (1 << 20))
        if key not in cost:  # class absent from the sample: nearest class of the same dimension
            key = min(cost, key=lambda k: (k[0] != r.desc.dim, k[1] != r.desc.precision))
        t, cu = cost[key]
        return t / cu * r.desc.ncell * r.steps

    rows = []
    with ClockSampler(local) as clk:
        for rate in args.c4_rates:
            reqs = serve.make_requests(args.c4_requests, rate, seed=7 + rank)
            with serve.Server(hbm_budget_bytes=150e9, max_slots=args.c4_slots, quantum=8,
                              solo_min_cells=args.c4_solo_min_cells, solo_slots=args.c4_solo_slots) as srv:
                st = srv.serve(reqs)
            p50, p99 = st.latency_percentiles()
            svc = [service(r) for r in reqs]
            arr = [r.arrival for r in reqs]
            seq_lat = _fifo_latencies(arr, svc)
            seq_elapsed = float(max(a + lat for a, lat in zip(sorted(arr), seq_lat)))
            rows.append({"rate_per_s": rate,
                         "served": {"solves_per_s": st.solves_per_s, "p50_s": p50, "p99_s": p99,
                                    "elapsed_s": st.elapsed, "peak_slots": st.peak_slots,
                                    "peak_gb": st.peak_bytes / 1e9, "quanta": st.quanta},
                         "sequential_plain": {"solves_per_s": len(reqs) / seq_elapsed,
                                              "p50_s": float(np.percentile(seq_lat, 50)),
                                              "p99_s": float(np.percentile(seq_lat, 99)),
                                              "elapsed_s": seq_elapsed}})
    if rank == 0:
        best = max(rows, key=lambda r: r["served"]["solves_per_s"])
        svc_all = [service(r) for r in base]
        big = sum(w for r, w in zip(base, svc_all) if r.desc.ncell >= (1 << 20))
        decomposition = {
            "sequential_device_s_total": float(sum(svc_all)),
            "share_in_gpu_filling_requests": float(big / sum(svc_all)),
            "speedup_ceiling_if_small_requests_were_free": float(sum(svc_all) / big) if big > 0 else None,
            "sample": f"{len(sample)} of {len(base)} requests run alone (every {max(1, args.c4_seq_every)}th)",
            "device_s_per_cell_update_by_class": {f"{k[0]}D,{'mixed' if k[1] else 'fp64'},"
                                                  f"{'>=1M' if k[2] else '<1M'} cells": v[0] / v[1]
                                                  for k, v in cost.items()},
        }
        line = {
            "metric": "DIM served solves/s", "value": world * best["served"]["solves_per_s"], "unit": "solves/s",
            "n_gpus": world, "steps": args.c4_requests, "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOADS["c4"][0],
                       "requests_per_rate": args.c4_requests, "rates": args.c4_rates,
                       "solo_min_cells": args.c4_solo_min_cells, "solo_slots": args.c4_solo_slots,
                       "sample": f"{args.c4_requests} requests per rate of the 10,000-request stream"},
            "rates": rows,
            "speedup_vs_sequential_plain": best["served"]["solves_per_s"] / best["sequential_plain"]["solves_per_s"],
            "decomposition": decomposition,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--scale", type=int, default=1, help="divide the grid sides (profiling runs)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--schedule", default="staged", choices=["staged", "fused"],
                    help="sweep schedule of the FP64 step (fused: one tile kernel per sweep)")
    ap.add_argument("--slabs", type=int, default=0, help="cut the grid into this many slabs (dimgpu_slabs_*)")
    ap.add_argument("--c3-steps", type=int, default=500)
    ap.add_argument("--c3-instances", type=int, default=256)
    ap.add_argument("--c3-sequential", type=int, default=16, help="instances in the sequential sample")
    ap.add_argument("--c4-requests", type=int, default=32)
    ap.add_argument("--c4-rates", type=float, nargs="+", default=[0.5, 1.0, 2.0, 4.0])
    ap.add_argument("--c4-slots", type=int, default=128)
    ap.add_argument("--c4-solo-min-cells", type=int, default=1 << 18, help="solves this large run on solo lanes")
    ap.add_argument("--c4-solo-slots", type=int, default=4)
    ap.add_argument("--c4-seq-every", type=int, default=8, help="sequential sample: every k-th request")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.slabs > 0:
        run_slabs(args)
    elif args.workload == "c3":
        run_batch(args)
    elif args.workload == "c4":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

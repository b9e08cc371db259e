"""Benchmark: 128^3 delta pressure projections per second on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size 128]

Workload: the seeded 128^3 box-basin scene (16 submerged boxes cut by their signed distance, a
sinusoidal free surface, a divergence-free background flow plus N(0, 0.5) m/s face noise; see
fluidisim_b200/scenes.py), projected from p = 0 by the multigrid-preconditioned CG of water-core's
`project_mobile3` to relative residual 1e-6 and plain divergence 1e-5.  One step = one projection.

  value  device-resident: the input faces are restored from HBM each step (fd3_set_velocity_device,
         which also checks them), p is zeroed, then fd3_project_mobile.  L2 is flushed (a 256 MiB
         write) between steps, outside the timed events.
  e2e    the same through the host-buffer C ABI: faces from pinned host memory (fd3_set_velocity),
         projection, then the projected faces and the pressure back to pinned host memory.
N > 1 runs N independent replicas (the projection of one domain does not shard: one 128^3 domain
fits one GPU), one per rank, timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import functools
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "128³ projections/s at rel. residual 1e-6: learned-FCG vs plain MGPCG, 1 B200"


def metric_for(workload: str, size: int) -> str:
    """The headline metric for the 128^3 basin; the same wording for the other single-volume scenes."""
    if workload == "basin" and size == 128:
        return METRIC
    return f"{size}³ {workload} projections/s at rel. residual 1e-6: plain MGPCG, 1 B200"

# Algorithmic bytes per cell of each fine-level kernel (f32 fields): every distinct array a pass
# must touch, counted once (stencil neighbours are not re-counted).  The hot kernels read the
# 2-byte row code of the projection; apertures are read only at cut faces and column heights
# only at ghost faces (both negligible in bulk).  Set-up kernels read the full geometry: the
# fluid fraction (4 B) and three face apertures (12 B).
GEOM = 16
BYTES_PER_CELL = {
    # 2.5-D blocked fine kernels, one cell per thread (f64 mode with kernels = 2)
    "kz_dir_apply_dot": 2 + 4 + 4 + 4 + 4,     # code, z, d in, d out, q
    "kv_update_rn": 4 * 6,                     # p, r read+write; d, q
    "kz_fine_pre": 2 + 4 + 4 + 4,              # code, prec, r, z out
    "kz_fine_restrict": 2 + 4 + 4 + 0.5,       # code, r, z, coarse r (1/8 cell)
    "kz_fine_post1": 2 + 4 + 4 + 4 + 0.5 + 4,  # code, prec, r, z in, coarse x, z out
    "kz_fine_post2_rz": 2 + 4 + 4 + 4 + 4,     # code, prec, r, z in, z out
    # the same passes with two cells per thread (f64 mode, the default when nx is even)
    "kx_dir_apply_dot": 2 + 4 + 4 + 4 + 4,
    "kx_fine_pre": 2 + 4 + 4 + 4,
    "kx_fine_restrict": 2 + 4 + 4 + 0.5,
    "kx_fine_post1": 2 + 4 + 4 + 4 + 0.5 + 4,
    "kx_fine_post2_rz": 2 + 4 + 4 + 4 + 4,
    # the same passes with four cells per thread (f64 mode, the default when nx % 4 == 0, f32 storage)
    "kq_dir_apply_dot": 2 + 4 + 4 + 4 + 4,
    "kq_fine_pre": 2 + 4 + 4 + 4,
    "kq_fine_restrict": 2 + 4 + 4 + 0.5,
    "kq_fine_post1": 2 + 4 + 4 + 4 + 0.5 + 4,
    "kq_fine_post2_rz": 2 + 4 + 4 + 4 + 4,
    "kq_residual": 2 + 4 * 3,
    # the same passes on TMA-staged layers (f64 mode, the default from 2^23 cells with nx % 8 == 0)
    "kt_dir_apply_dot": 2 + 4 + 4 + 4 + 4,
    "kt_fine_pre": 2 + 4 + 4 + 4,
    "kt_fine_restrict": 2 + 4 + 4 + 0.5,
    "kt_fine_post1": 2 + 4 + 4 + 4 + 0.5 + 4,
    "kt_fine_post2_rz": 2 + 4 + 4 + 4 + 4,
    "kt_residual": 2 + 4 * 3,                  # code, p, rhs, res out
    # one-cell-per-thread kernels (ordered mode, and f64 mode with kernels = 1)
    "k_dir_apply_dot": 2 + 4 + 4 + 4 + 4,
    "k_update_rn": 4 * 6,
    "k_fine_pre": 2 + 4 + 4 + 4,
    "k_fine_restrict_c": 2 + 4 + 4 + 0.5,
    "k_fine_post1": 2 + 4 + 4 + 4 + 0.5 + 4,
    "k_fine_post2_rz": 2 + 4 + 4 + 4 + 4,
    "k_apply_dot_c": 2 + 4 + 4,                # code, d, q
    "k_dot_prec_fin": 8,
    "k_jacobi_dir": 12,
    # set-up and checks, once per projection
    "k_residual_c": 2 + 4 * 3,                 # code, p, rhs, res
    "k_rhs_b2": 4 * 3 + GEOM + 2,              # rhs read+write, prec, geometry, row code
    "k_divergence": 4 * 3 + 4 + GEOM,          # three face families in, rhs out
}


def merge_templates(entries):
    """Per-kernel profile entries with template arguments dropped (kz_fine_pre<true> and
    kz_fine_pre<false> are one kernel: full tiles and ragged tiles of the same pass)."""
    acc = {}
    for name, count, ms in entries:
        base = name.split("<", 1)[0]
        c, m = acc.get(base, (0, 0.0))
        acc[base] = (c + count, m + ms)
    return [(n, c, m) for n, (c, m) in acc.items()]


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons sampled DURING the timed region.

    NVML is polled from a thread every `period` seconds (2 ms by default), so even a timed region
    of tens of milliseconds gets samples; the GPU is found by its PCI bus id (NVML numbers GPUs
    without CUDA_VISIBLE_DEVICES).  Without NVML the sampler falls back to `nvidia-smi -lms 100`.
    `mark(True)` / `mark(False)` bracket the timed region; only samples taken between the two marks
    are summarised.  Reading clocks changes no GPU setting."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, period: float = 0.002):
        self.index = index
        self.period = period
        self.proc = None
        self.nvml = None
        self.handle = None
        self.lines = []     # nvidia-smi: (t, csv line)
        self.samples = []   # NVML: (t, sm_mhz, max_mhz, power_w, reasons)
        self.t0 = None
        self.t1 = None
        self.stop = threading.Event()
        self.source = "none"

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            self.handle = self._nvml_handle()
            self.source = "nvml"
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _poll(self):
        n = self.nvml
        bits = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        try:
            smax = float(n.nvmlDeviceGetMaxClockInfo(self.handle, n.NVML_CLOCK_SM))
        except Exception:
            smax = float("nan")
        while not self.stop.is_set():
            try:
                sm = float(n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM))
                reasons = int(n.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                try:
                    power = n.nvmlDeviceGetPowerUsage(self.handle) / 1000.0
                except Exception:
                    power = float("nan")
                active = {name for name, b in zip(self.NAMES, bits) if reasons & b}
                self.samples.append((time.monotonic(), sm, smax, power, active))
            except Exception:
                pass
            self.stop.wait(self.period)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self, start: bool):
        if start:
            self.t0 = time.monotonic()
        else:
            self.t1 = time.monotonic()

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nvml is not None:
            try:
                self.thread.join(timeout=2)
                self.nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        sm, smax, power, reasons = [], [], [], set()
        t0 = self.t0 if self.t0 is not None else float("-inf")
        t1 = self.t1 if self.t1 is not None else float("inf")
        for t, a, b, pw, active in self.samples:
            if t0 <= t <= t1:
                sm.append(a)
                smax.append(b)
                power.append(pw)
                reasons |= active
        for t, line in self.lines:
            if not (t0 <= t <= t1):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(self.NAMES, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0, "source": self.source}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "power_w_max": max(power), "samples": len(sm), "source": self.source}


def dist_setup(gpus: int):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


@functools.lru_cache(maxsize=2)
def make_scene(workload: str, size: int):
    from fluidisim_b200 import scenes
    if workload == "wave":
        return scenes.breaking_wave(size)
    return scenes.box_basin(size)


WORKLOAD_NAMES = {
    "basin": "box_basin {n}^3 (16 boxes, sinusoidal surface, curl background + N(0,0.5) noise)",
    "wave": "breaking_wave {n}^3 (32 obstacles, tanh surface, 2 m/s crest + N(0,0.3) noise)",
}


def workload_label(workload: str, size: int) -> str:
    """The workload name both arms print (the same scene, solver recipe and stopping rule)."""
    return WORKLOAD_NAMES[workload].format(n=size) + ": multigrid-PCG projection (reference V-cycle recipe)"


def run_reference(args):
    """The reference arm: the CPU oracle (a restatement of the reference's Rust projection, whose own
    toolchain is absent here) on the host cores, same scene, metric and unit."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from fluidisim_b200 import scenes
    from oracle import oracle as O
    O.build()
    threads = O.max_threads()
    O.set_threads(threads)
    s = make_scene(args.workload, args.size)
    scale, k1 = scenes.projection_scalars(s)
    v = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    v.enable_multigrid()
    v.set_free_surface(s["eta"], s["rest"])
    # A CPU projection at 128^3 takes most of a second, so the arm is bounded: at most 2 warm-up
    # projections, then timed projections until K are done or 90 s have passed.
    times, rep = [], None
    warm = min(args.warmup, 2)
    t_begin = None
    for step in range(warm + args.steps):
        v.set_velocity(s["u"], s["v"], s["w"])
        v.set_free_surface(s["eta"], s["rest"])
        t0 = time.perf_counter()
        rep = v.project_mobile(scale, k1, 4000)
        dt = time.perf_counter() - t0
        if step >= warm:
            times.append(dt)
            t_begin = t_begin if t_begin is not None else t0
            if time.perf_counter() - t_begin > 90.0:
                break
    ms = 1e3 * sum(times) / len(times)
    value = 1e3 / ms
    out = {
        "impl": "reference", "metric": metric_for(args.workload, args.size), "value": value, "unit": "projections/s",
        "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.workload} scene)",
        "config": {"workload": workload_label(args.workload, args.size),
                   "cells": s["nx"] * s["ny"] * s["nz"], "solver": "mgpcg", "iterations": rep["iterations"],
                   "rel_residual": rep["residual"], "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "projections/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} timed projections of the {args.size}^3 scene after {warm} warm-up "
                                   f"(capped at {args.steps} or 90 s)"},
        "e2e": {"value": value, "unit": "projections/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def cpu_baseline_sample(workload: str, size: int, budget_s: float = 20.0):
    """The oracle (OpenMP on every host core) timed on a bounded sample of the same workload."""
    from fluidisim_b200 import scenes
    from oracle import oracle as O
    O.build()
    threads = O.max_threads()
    O.set_threads(threads)
    s = make_scene(workload, size)
    scale, k1 = scenes.projection_scalars(s)
    v = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"])
    v.enable_multigrid()
    times = []
    t_start = time.perf_counter()
    while not times or (time.perf_counter() - t_start < budget_s and len(times) < 5):
        v.set_velocity(s["u"], s["v"], s["w"])
        v.set_free_surface(s["eta"], s["rest"])
        t0 = time.perf_counter()
        v.project_mobile(scale, k1, 4000)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    # the reference's own semantics: one thread (its reductions are serial by design)
    O.set_threads(1)
    v.set_velocity(s["u"], s["v"], s["w"])
    v.set_free_surface(s["eta"], s["rest"])
    t0 = time.perf_counter()
    v.project_mobile(scale, k1, 4000)
    one = time.perf_counter() - t0
    O.set_threads(threads)
    return {"value": 1e3 / ms, "unit": "projections/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} full {size}^3 {workload} projections (same scene), oracle with OpenMP",
            "single_thread": {"value": 1.0 / one, "unit": "projections/s", "cores": 1,
                              "sample": f"1 full {size}^3 {workload} projection, oracle on one thread"}}


def fp64_pressure_check(workload: str, size: int, pressures: dict, max_cells: int = 128 ** 3):
    """The checker of the mixed-precision leg (CPU, beside the CPU baseline): the oracle's f64
    build solves the same projection to relative residual 1e-12, and each GPU pressure is reported
    as its L-inf difference relative to that solution's L-inf.  Skipped above max_cells."""
    import numpy as np

    from fluidisim_b200 import scenes
    from oracle import oracle as O
    s = make_scene(workload, size)
    if s["nx"] * s["ny"] * s["nz"] > max_cells:
        return None
    O.build()
    O.set_threads(O.max_threads("f64"), "f64")
    o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], bottom=s["bottom"], solid=s["solid"],
                       real="f64")
    o.enable_multigrid()
    o.set_free_surface(s["eta"], s["rest"])
    o.set_velocity(s["u"], s["v"], s["w"])
    o.set_tolerance(1e-24)
    scale, k1 = scenes.projection_scalars(s)
    t0 = time.perf_counter()
    rep = o.project_mobile(scale, k1, 4000)
    secs = time.perf_counter() - t0
    p64 = o.pressure().astype(np.float64)
    pmax = float(np.abs(p64).max())
    out = {"fp64_rel_residual": rep["residual"], "fp64_iterations": rep["iterations"], "fp64_seconds": secs,
           "fp64_pressure_max": pmax}
    for k, p in pressures.items():
        out[f"{k}_linf_rel"] = float(np.abs(p.astype(np.float64) - p64).max() / pmax)
    return out


def mixed_measure(args, s, stream, flush, p_f32, ms_f32):
    """The FP16-storage V-cycle (fd3_options.storage = FP16) on the bench scene, timed as the main
    leg (device-resident inputs, L2 flushed between steps, CUDA events on the solver's stream)."""
    import numpy as np
    import torch

    from fluidisim_b200 import scenes
    from fluidisim_b200.delta3d import STORAGE_F16, Volume3
    scale, k1 = scenes.projection_scalars(s)
    vol = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    vol.set_options(use_graphs=args.graphs, storage=STORAGE_F16)
    vol.set_stream(stream.cuda_stream)
    vol.enable_multigrid()
    vol.set_free_surface(s["eta"], s["rest"])
    du = torch.from_numpy(s["u"]).cuda()
    dv = torch.from_numpy(s["v"]).cuda()
    dw = torch.from_numpy(s["w"]).cuda()

    def step():
        vol.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
        vol.reset_pressure()
        return vol.project_mobile3(scale, k1, 4000)

    for _ in range(max(3, args.warmup)):
        rep = step()
    torch.cuda.synchronize()
    steps = max(10, min(args.steps, 100))
    evs = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    p16 = vol.pressure()
    vol.close()
    pmax = float(np.abs(p_f32).max())
    return {"storage": "fp16 V-cycle vectors (fine z, coarse x, r), f32 arithmetic; f32 CG vectors; f64 dots, "
                       "alpha/beta and true residual; outer loop restarts from b - A p (defect correction)",
            "value": 1e3 / ms, "unit": "projections/s", "ms_per_step": ms, "steps": steps,
            "speedup_vs_f32_storage": ms_f32 / ms,
            "note": "slower than f32 storage here and on the 256^3 wave (wave_256.fp16_mgpcg): the 128^3 passes are "
                    "latency-bound, so halving the bytes of the V-cycle vectors saves nothing, and the rounding "
                    "costs iterations; built, tested and off by default",
            "iterations": rep.iterations, "rel_residual": rep.residual,
            "divergence_plain": rep.divergence_plain, "degraded": bool(rep.degraded),
            "pressure_linf_rel_vs_f32_storage": float(np.abs(p16.astype(np.float64) - p_f32).max() / pmax)}, p16


def learned_fcg_measure(args, s, vol_plain_p, stream):
    """The learned preconditioner, measured in the same run: training throughput at 64^3 (batch
    32, sphere-lake scenes with seeded random velocities), the validation FCG iteration count on
    held-out lakes, and learned-FCG projections/s on the bench scene (device-resident inputs, the
    same L2 flush), with its fallback work and its pressure against plain MGPCG's."""
    import numpy as np
    import torch

    from fluidisim_b200 import learned, scenes
    from fluidisim_b200.delta3d import REDUCE_F64, Volume3

    def lake(seed):
        sc = scenes.sphere_lake(64, seed=seed)
        v = Volume3.configure_with_solid(sc["nx"], sc["ny"], sc["nz"], sc["dx"], sc["rho"], sc["g"], sc["bottom"],
                                         sc["solid"])
        v.set_options(reduction=REDUCE_F64)
        v.enable_multigrid()
        v.set_free_surface(sc["eta"], sc["rest"])
        return v, sc

    train = [lake(1000 + q)[0] for q in range(8)]
    sc0 = scenes.sphere_lake(64, seed=1000)
    tscale, _ = scenes.projection_scalars(sc0)
    net = learned.UNet(32, 64, 64, 64)
    net.set_params(learned.init_params(0))
    tr = learned.Trainer(net, train, tscale, batch=32, seed=1)
    rng = np.random.default_rng(0)
    steps = max(1, args.train_samples // 32)
    tr.step(1e-3, rng)  # warm-up (kernel load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = [tr.step(1e-3 if q < 0.7 * steps else 3e-4, rng) for q in range(steps)]
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    params = net.params()
    net.close()
    # validation on held-out lakes: FCG + fallback iterations against plain MGPCG's
    vnet = learned.UNet(1, 64, 64, 64)
    vnet.set_params(params)
    val = []
    for seed in (2000, 2001):
        v, sc = lake(seed)
        v.set_velocity(sc["u"], sc["v"], sc["w"])
        sc_s, sc_k = scenes.projection_scalars(sc)
        r = learned.project_learned(v, vnet, sc_s, sc_k, 4000, 200)
        ref, _ = lake(seed)
        ref.set_velocity(sc["u"], sc["v"], sc["w"])
        rr = ref.project_mobile3(sc_s, sc_k, 4000)
        val.append({"fcg": r.fcg_iterations, "fallback_mg": r.report.iterations, "fell_back": r.fell_back,
                    "plain_mgpcg": rr.iterations, "residual": r.report.residual})
    vnet.close()
    # the bench scene
    n = s["nx"]
    inet = learned.UNet(1, s["nz"], s["ny"], s["nx"])
    inet.set_params(params)
    scale, k1 = scenes.projection_scalars(s)
    lv = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    lv.set_options(reduction=REDUCE_F64)
    lv.set_stream(stream.cuda_stream)
    lv.enable_multigrid()
    lv.set_free_surface(s["eta"], s["rest"])
    du = torch.from_numpy(s["u"]).cuda()
    dv = torch.from_numpy(s["v"]).cuda()
    dw = torch.from_numpy(s["w"]).cuda()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def step():
        lv.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
        lv.reset_pressure()
        return learned.project_learned(lv, inet, scale, k1, 4000, 100)

    for _ in range(2):
        step()
    K = max(3, min(args.steps, 20))
    ms, rep = [], None
    for _ in range(K):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rep = step()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    p = lv.pressure()
    dp = float(np.max(np.abs(p - vol_plain_p)) / max(np.max(np.abs(vol_plain_p)), 1e-30))
    inet.close()
    lv.close()
    args._learned_params = params
    return {
        "metric_value": K / (sum(ms) * 1e-3), "unit": "projections/s", "ms_per_projection": sum(ms) / K,
        "fcg_iterations": rep.fcg_iterations, "fallback_mg_iterations": rep.report.iterations,
        "fell_back": rep.fell_back, "rel_residual": rep.report.residual,
        "divergence_plain": rep.report.divergence_plain, "pressure_linf_vs_plain_mgpcg": dp,
        "network": "3-level U-Net 16/32/64, 3x3x3 convs, BF16 storage / FP32 accumulation; convolutions on tcgen05.mma (TMEM accumulators), weight gradients on mma.sync m16n8k16",
        "training": {"samples": steps * 32, "batch": 32, "grid": "64^3 sphere lakes (8 geometries)",
                     "samples_per_s": steps * 32 / train_s, "seconds": train_s,
                     "loss_first": float(np.mean(losses[:3])), "loss_last": float(np.mean(losses[-3:]))},
        "validation_64": val,
    }


def wave_measure(args, stream, flush):
    """The 256^3 breaking wave (16.8M cells, inputs far above L2), three solvers on the same scene:
    FP32-storage MGPCG (the default path), FP16-storage MGPCG and learned FCG with the network the
    learned leg trained at 64^3, inferred at 256^3.  Each: ms per projection (CUDA events on the
    solver's stream, device-resident inputs), iterations, the fraction of projections that fell
    back to MGPCG, and the HBM roofline of the solver's dominant kernel (algorithmic bytes of a
    launch / its event-timed duration in an instrumented replay / measured peak)."""
    import numpy as np
    import torch

    from fluidisim_b200 import learned, scenes
    from fluidisim_b200.delta3d import REDUCE_F64, STORAGE_F16, STORAGE_F32, Volume3
    s = make_scene("wave", 256)
    scale, k1 = scenes.projection_scalars(s)
    cells = s["nx"] * s["ny"] * s["nz"]
    du, dv, dw = (torch.from_numpy(s[k]).cuda() for k in ("u", "v", "w"))
    peak, peak_kind = peaks()
    steps = max(3, min(args.steps, 10))
    out = {"workload": WORKLOAD_NAMES["wave"].format(n=256), "cells": cells, "steps": steps,
           "l2": "inputs far above L2 (about 0.8 GB of fields); 256 MiB written between steps"}

    def volume(storage):
        v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
        v.set_options(reduction=REDUCE_F64, use_graphs=args.graphs, storage=storage)
        v.set_stream(stream.cuda_stream)
        v.enable_multigrid()
        v.set_free_surface(s["eta"], s["rest"])
        return v

    def timed(step):
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        ms, reps = [], []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            reps.append(step())
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return sum(ms) / steps, reps

    def roofline(v, step):
        v.set_options(use_graphs=0)
        v.profile(True)
        for _ in range(2):
            step()
        torch.cuda.synchronize()
        prof = merge_templates(v.profile_entries())
        v.profile(False)
        v.set_options(use_graphs=args.graphs)
        known = [(n, c, m) for n, c, m in prof if n in BYTES_PER_CELL and BYTES_PER_CELL[n] >= 8]
        name, count, msum = max(known, key=lambda e: e[2])
        avg = msum / count
        ach = BYTES_PER_CELL[name] * cells / (avg * 1e-3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic_wave_256.txt")
        if os.path.exists(tf):
            for line in open(tf):
                parts = line.split()
                if len(parts) == 2 and not line.startswith("#") and parts[0] == name:
                    traffic = float(parts[1])
        return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": peak_kind, "avg_launch_ms": avg, "alg_bytes_per_launch": BYTES_PER_CELL[name] * cells,
                "traffic": traffic, "timing": "instrumented replay of 2 projections without the loop graph"}

    pressures = {}
    for key, storage in (("fp32_mgpcg", STORAGE_F32), ("fp16_mgpcg", STORAGE_F16)):
        v = volume(storage)

        def step(v=v):
            v.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
            v.reset_pressure()
            return v.project_mobile3(scale, k1, 4000)
        ms, reps = timed(step)
        r = reps[-1]
        out[key] = {"ms_per_projection": ms, "projections_per_s": 1e3 / ms, "iterations": r.iterations,
                    "rel_residual": r.residual, "divergence_plain": r.divergence_plain, "fallback_rate": None,
                    "roofline": roofline(v, step)}
        pressures[key] = v.pressure().astype(np.float64)
        v.close()
    pm = np.abs(pressures["fp32_mgpcg"]).max()
    out["fp16_mgpcg"]["pressure_linf_rel_vs_fp32"] = float(np.abs(pressures["fp16_mgpcg"] - pressures["fp32_mgpcg"]).max() / pm)
    params = getattr(args, "_learned_params", None)
    if params is not None:
        v = volume(STORAGE_F32)
        net = learned.UNet(1, s["nz"], s["ny"], s["nx"])
        net.set_params(params)

        def lstep():
            v.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
            v.reset_pressure()
            return learned.project_learned(v, net, scale, k1, 4000, 100)
        ms, reps = timed(lstep)
        r = reps[-1]
        out["learned_fcg"] = {"ms_per_projection": ms, "projections_per_s": 1e3 / ms,
                              "fcg_iterations": r.fcg_iterations, "fallback_mg_iterations": r.report.iterations,
                              "fallback_rate": float(np.mean([x.fell_back for x in reps])),
                              "rel_residual": r.report.residual, "divergence_plain": r.report.divergence_plain,
                              "pressure_linf_rel_vs_fp32": float(np.abs(v.pressure() - pressures["fp32_mgpcg"]).max() / pm),
                              "speedup_vs_fp32_mgpcg": out["fp32_mgpcg"]["ms_per_projection"] / ms}
        net.close()
        v.close()
    return out


def parts_measure(args, s, stream):
    """The other parts of the path on the same 128^3 scene, each timed with CUDA events on the
    volume's stream after warm-up: a whole mobile step (advection, projection, extrapolation,
    transport), the same with the second-order advection term, a re-cut of the moving solid, and a
    level change of the flat-bottomed state to half the resolution."""
    import numpy as np
    import torch

    from fluidisim_b200.delta3d import REDUCE_F64, Volume3

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        total = 0.0
        out = None
        for _ in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = fn()
            b.record(stream)
            torch.cuda.synchronize()
            total += a.elapsed_time(b)
        return total / n, out

    def volume(correction=False):
        v = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
        v.set_options(reduction=REDUCE_F64, use_graphs=args.graphs)
        v.set_stream(stream.cuda_stream)
        v.enable_multigrid()
        v.set_free_surface(s["eta"], s["rest"])
        v.set_velocity(s["u"], s["v"], s["w"])
        if correction:
            v.enable_advection_correction()
        return v

    out = {}
    dt_us = int(round(s["dt"] * 1e6))
    for key, corr in (("mobile_step", False), ("mobile_step_second_order", True)):
        v = volume(corr)
        its = []
        ms, _ = timed(lambda: its.append(v.step_surface_mobile(dt_us, 4000).iterations), 10)
        out[key] = {"ms": ms, "iterations_mean": float(np.mean(its)), "dt_us": dt_us}
        v.close()
    v = volume()
    ms, _ = timed(lambda: v.set_solid_rigid(s["solid"], (0.1, 0.0, 0.0), (0.0, 0.0, 0.2),
                                             (0.5 * s["nx"] * s["dx"], 0.5 * s["ny"] * s["dx"], 0.3 * s["nz"] * s["dx"])), 10)
    out["set_solid_rigid"] = {"ms": ms, "note": "re-cut of the 16 boxes from the kept base, wall velocities, displaced water"}
    v.close()
    n = s["nx"]
    fine = Volume3.configure(n, n, n, s["dx"], s["rho"], s["g"])
    coarse = Volume3.configure(n // 2, n // 2, n // 2, float(np.float32(2 * s["dx"])), s["rho"], s["g"])
    for x in (fine, coarse):
        x.set_stream(stream.cuda_stream)
    fine.set_free_surface(s["eta"], s["rest"])
    coarse.set_free_surface(np.full((n // 2) ** 2, s["rest"], np.float32), s["rest"])
    fine.set_velocity(s["u"], s["v"], s["w"])
    ms, ch = timed(lambda: coarse.resample_from(fine), 10)
    out["resample_from"] = {"ms": ms, "case": f"{n}^3 -> {n // 2}^3, flat bottom",
                            "volume_error_m3": ch["volume_after"] - ch["volume_before"]}
    fine.close()
    coarse.close()
    return out


def run_b200(args):
    import numpy as np
    import torch

    from fluidisim_b200 import build as B
    from fluidisim_b200 import scenes
    from fluidisim_b200.delta3d import REDUCE_F64, Volume3

    rank, world, local = dist_setup(args.gpus)
    B.build()
    s = make_scene(args.workload, args.size)
    scale, k1 = scenes.projection_scalars(s)
    stream = torch.cuda.Stream()
    vol = Volume3.configure_with_solid(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"], s["bottom"], s["solid"])
    vol.set_options(reduction=REDUCE_F64, use_graphs=args.graphs, kernels=args.kernels)
    vol.set_stream(stream.cuda_stream)
    vol.enable_multigrid()
    vol.set_free_surface(s["eta"], s["rest"])
    # inputs resident in HBM
    du = torch.from_numpy(s["u"]).cuda()
    dv = torch.from_numpy(s["v"]).cuda()
    dw = torch.from_numpy(s["w"]).cuda()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def step():
        vol.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
        vol.reset_pressure()
        return vol.project_mobile3(scale, k1, 4000)

    rep = None
    evs = []
    with ClockSampler(local) as clocks:
        t_warm = time.monotonic()
        for _ in range(args.warmup):
            rep = step()
        torch.cuda.synchronize()
        while clocks.source == "nvidia-smi" and time.monotonic() - t_warm < 1.0:  # its first lines
            rep = step()
            torch.cuda.synchronize()
        barrier(world)
        launches0 = vol.kernel_launches()
        torch.cuda.synchronize()
        barrier(world)
        clocks.mark(True)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            rep = step()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        clocks.mark(False)
        barrier(world)
        launches = vol.kernel_launches() - launches0
    ms_total = sum(a.elapsed_time(b) for a, b in evs)
    ms_total = max_over_ranks(ms_total, world)
    ms_per_step = ms_total / args.steps
    value = world * args.steps / (ms_total * 1e-3)

    # e2e through the host-buffer ABI
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    hu, hv, hw = pin(s["u"]), pin(s["v"]), pin(s["w"])
    ou = torch.empty(vol.nu, dtype=torch.float32).pin_memory()
    ov = torch.empty(vol.nv, dtype=torch.float32).pin_memory()
    ow = torch.empty(vol.nw, dtype=torch.float32).pin_memory()
    op = torch.empty(vol.cells, dtype=torch.float32).pin_memory()
    import ctypes as C
    L = vol._L
    fp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float))  # noqa: E731

    def e2e_step():
        e = L.fd3_set_velocity(vol._h, fp(hu), vol.nu, fp(hv), vol.nv, fp(hw), vol.nw)
        assert e == 0, e
        vol.reset_pressure()
        r = vol.project_mobile3(scale, k1, 4000)
        e = L.fd3_get_velocity(vol._h, fp(ou), vol.nu, fp(ov), vol.nv, fp(ow), vol.nw)
        assert e == 0, e
        e = L.fd3_get_pressure(vol._h, fp(op), vol.cells)
        assert e == 0, e
        return r

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e2e_step()
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = world * args.steps / (e2e_total * 1e-3)
    h2d = 4 * (vol.nu + vol.nv + vol.nw)
    d2h = 4 * (vol.nu + vol.nv + vol.nw + vol.cells)

    # per-kernel timing: an instrumented replay of the same steps right after the timed region
    vol.set_options(use_graphs=0)
    vol.profile(True)
    prof_steps = min(args.steps, 20)
    for _ in range(prof_steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        step()
    torch.cuda.synchronize()
    prof = merge_templates(vol.profile_entries())
    vol.profile(False)
    vol.set_options(use_graphs=args.graphs)
    total_prof = sum(ms for _, _, ms in prof)
    known = [(n, c, ms) for n, c, ms in prof if n in BYTES_PER_CELL and BYTES_PER_CELL[n] >= 8]
    top = max(known, key=lambda e: e[2])
    name, count, ms = top
    cells = s["nx"] * s["ny"] * s["nz"]
    alg_bytes = BYTES_PER_CELL[name] * cells
    avg_ms = ms / count
    peak, peak_kind = peaks()
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    ncu_traffic = None
    traffic_file = os.path.join(ROOT, "profiles", f"traffic_{args.workload}_{args.size}.txt")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2 and not line.startswith("#") and parts[0] == name:
                    ncu_traffic = float(parts[1])

    learned_line = None
    mixed_line, p16 = None, None
    plain_p = vol.pressure()
    if world == 1 and args.mixed:
        mixed_line, p16 = mixed_measure(args, s, stream, flush, plain_p.astype(np.float64), ms_per_step)
    if world == 1 and args.learned:
        learned_line = learned_fcg_measure(args, s, plain_p, stream)
    parts_line = parts_measure(args, s, stream) if (world == 1 and args.parts) else None
    wave_line = wave_measure(args, stream, flush) if (world == 1 and args.wave and args.workload == "basin") else None

    if rank == 0:
        cpu = cpu_baseline_sample(args.workload, args.size) if (world == 1 and not args.no_cpu) else None
        if mixed_line is not None and not args.no_cpu:
            mixed_line["fp64_check"] = fp64_pressure_check(args.workload, args.size,
                                                           {"f32_storage": plain_p, "fp16_storage": p16})
        out = {
            "impl": "b200", "metric": metric_for(args.workload, args.size), "value": value, "unit": "projections/s",
            "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": f"synthetic (seeded {args.workload} scene)",
            "config": {"workload": workload_label(args.workload, args.size),
                       "cells": cells, "solver": "mgpcg", "reduction": "f64", "iterations": rep.iterations,
                       "rel_residual": rep.residual, "divergence_plain": rep.divergence_plain,
                       "l2": "flushed between steps (256 MiB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": ncu_traffic, "alg_bytes_per_launch": alg_bytes,
                         "avg_launch_ms": avg_ms, "launches": count,
                         "share_of_step": ms / total_prof if total_prof else None},
            "kernels": {n: {"launches": c, "ms_per_step": round(m / prof_steps, 5)}
                        for n, c, m in sorted(prof, key=lambda e: -e[2])[:14]},
            "kernels_source": f"an instrumented replay of {prof_steps} steps right after the timed region: the "
                              "loop driven from the host without its CUDA graph, CUDA events around every launch "
                              "(the kernel table and roofline.avg_launch_ms come from it)",
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "projections/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "learned_fcg": learned_line,
            "mixed_precision": mixed_line,
            "parts": parts_line,
            "wave_256": wave_line,
        }
        print(json.dumps(out), flush=True)
    vol.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_patches(args):
    """Batched patches: every rank projects its share of the seeded patch set (dealt by decreasing
    size) in ONE persistent launch per step (fd3_batch_project: thread-block clusters as independent
    solvers, each taking its share of the patches, largest first), the cluster size chosen by timing
    the whole set.  Inputs stay resident in HBM and are copied in by the launch.  The earlier path
    (fd3_project_batch: per-patch loop graphs from host workers) is timed beside it.  No data-path
    collective: only the timing max and a count reduction."""
    import numpy as np
    import torch

    from fluidisim_b200 import batch, scenes
    from fluidisim_b200 import build as B

    rank, world, local = dist_setup(args.gpus)
    B.build()
    ps = batch.patch_scenes(args.patches, seed=3)
    cells = [p["nx"] * p["ny"] * p["nz"] for p in ps]
    mine = [ps[i] for i in batch.deal(cells, world, rank)]
    vols = [batch.configure(p) for p in mine]
    inputs = [tuple(torch.from_numpy(p[k]).cuda() for k in ("u", "v", "w")) for p in mine]
    ptrs = [tuple(t.data_ptr() for t in x) for x in inputs]
    sk = [scenes.projection_scalars(p) for p in mine]
    scales, k1s = [a for a, _ in sk], [b for _, b in sk]
    torch.cuda.synchronize()

    def timed_set(fn, reps):
        out, best = None, float("inf")
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        return best, out

    # the cluster size: the whole set timed with each (best of 3 after one warm-up)
    tuning = {}
    for cs in (1, 2, 4, 8):
        pb = batch.PersistentBatch(vols, cluster_size=cs)
        ms_cs, _ = timed_set(lambda: pb.project(scales, k1s, reset_pressure=True, inputs=ptrs), 4)
        tuning[cs] = {"ms": round(ms_cs, 3), "clusters": pb.clusters}
        pb.close()
    best_cs = min(tuning, key=lambda c: tuning[c]["ms"])
    pb = batch.PersistentBatch(vols, cluster_size=best_cs)

    def step():
        return pb.project(scales, k1s, reset_pressure=True, inputs=ptrs)

    for _ in range(args.warmup):
        reps, st = step()
    torch.cuda.synchronize()
    barrier(world)
    ms = []
    launches0 = pb.kernel_launches()
    with ClockSampler(local) as clocks:
        clocks.mark(True)
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            reps, st = step()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        clocks.mark(False)
    launches = pb.kernel_launches() - launches0
    assert all(x == 0 for x in st), st
    assert all(not r.degraded and r.residual <= 1e-6 for r in reps)
    my_ci = sum(p["nx"] * p["ny"] * p["nz"] * r.iterations for p, r in zip(mine, reps))
    ms_total, ci = batch.reduce_totals(sum(ms), my_ci, world, device="cuda")
    its = [r.iterations for r in reps]
    pb.close()
    # the per-patch path on the same volumes: host workers issuing each patch's loop graph
    streams_line = None
    if world == 1 and args.streams:
        tuned = batch.autotune(batch.by_class(mine))

        def sstep():
            for v, (du, dv, dw) in zip(vols, inputs):
                v.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
                v.reset_pressure()
            return batch.project_batch(vols, scales, k1s, threads=args.threads)
        sstep()
        ms_s = []
        for _ in range(max(3, min(args.steps, 10))):
            m_, _ = timed_set(sstep, 1)
            ms_s.append(m_)
        streams_line = {"value": len(ps) / (np.mean(ms_s) * 1e-3), "unit": "patches/s", "ms_per_step": float(np.mean(ms_s)),
                        "note": "fd3_project_batch: every patch its own stream and device-side loop graph, issued by "
                                "host workers; inputs set through set_velocity_device per patch",
                        "autotuned": {k: {"kernels": v.kernels, "mg_max_levels": v.levels, "ms": round(v.ms, 3)}
                                      for k, v in tuned.items()}}
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_patches_sample(ps)
        out = {
            "impl": "b200", "metric": f"patches/s ({args.patches} seeded delta patches, 16-96 cells per side)",
            "value": args.steps * len(ps) / (ms_total * 1e-3), "unit": "patches/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded patch set)",
            "config": {"workload": f"{args.patches} patches: sides log-uniform in [16,96] rounded to 8, spheres "
                                   f"5-15% of cells, fill U[0.3,0.8], faces U[-1,1]; one persistent launch per step",
                       "cells_total": sum(cells), "parallelism": f"patches sharded x{world}",
                       "autotuned": {"cluster_size": best_cs, "candidates": tuning,
                                     "threads_per_cta": 1024, "mg_depth": "every level (the reference's hierarchy)"},
                       "iterations_rank0": {"min": min(its), "max": max(its), "mean": float(np.mean(its))},
                       "l2": "inputs restored each step by the launch; the patch set exceeds L2"},
            "cells_iterations_per_s": args.steps * ci / (ms_total * 1e-3),
            "gpu_launches": launches,
            "streams_path": streams_line,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        print(json.dumps(out), flush=True)
    for v in vols:
        v.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference_patches(args):
    """The reference arm of the patches workload: the oracle projects the patch set one patch at a
    time on the host cores (the reference has no batched path); bounded to 90 s."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from fluidisim_b200 import batch
    ps = batch.patch_scenes(args.patches, seed=3)
    cpu = cpu_patches_sample(ps, budget_s=90.0)
    out = {"impl": "reference", "metric": f"patches/s ({args.patches} seeded delta patches, 16-96 cells per side)",
           "value": cpu["value"], "unit": "patches/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * args.patches / cpu["value"], "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded patch set)",
           "config": {"workload": f"{args.patches} patches (see the b200 arm)", "parallelism": "host threads"},
           "cpu_baseline": cpu,
           "e2e": {"value": cpu["value"], "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def cpu_patches_sample(ps, budget_s: float = 20.0):
    """The oracle (OpenMP) on the patches in order until the budget is spent: patches/s and
    cells x iterations / s of that sample."""
    from fluidisim_b200 import scenes
    from oracle import oracle as O
    O.build()
    threads = O.max_threads()
    O.set_threads(threads)
    t0 = time.perf_counter()
    done, ci = 0, 0
    for p in ps:
        v = O.OracleVolume(p["nx"], p["ny"], p["nz"], p["dx"], p["rho"], p["g"], bottom=p["bottom"], solid=p["solid"])
        v.enable_multigrid()
        v.set_free_surface(p["eta"], p["rest"])
        v.set_velocity(p["u"], p["v"], p["w"])
        scale, k1 = scenes.projection_scalars(p)
        r = v.project_mobile(scale, k1, 4000)
        done += 1
        ci += p["nx"] * p["ny"] * p["nz"] * r["iterations"]
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "patches/s", "cores": threads, "kind": "port",
            "cells_iterations_per_s": ci / dt,
            "sample": f"the first {done} patches of the set, oracle with OpenMP (setup excluded)"}


def run_sparse(args):
    """A sparse set in a 256 x 256 x 32 window (37% of the columns, blocks along a curved path):
    projections per second of the set, against the same set with every tile of the window
    processed (what looping over the whole window costs) and against the dense window.  N > 1
    runs replicas."""
    import numpy as np
    import torch

    from fluidisim_b200 import build as B
    from fluidisim_b200 import scenes
    from fluidisim_b200.delta3d import REDUCE_F64, Volume3

    rank, world, local = dist_setup(args.gpus)
    B.build()
    s = scenes.sparse_window(args.size)
    scale, k1 = float(np.float32(-s["rho"] / s["dt"])), float(np.float32(s["dt"] / s["rho"]))
    du, dv, dw = (torch.from_numpy(s[k]).cuda() for k in ("u", "v", "w"))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    rest = np.float32(s["rest"])

    def volume(mask, skip):
        v = Volume3.configure(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"])
        v.set_options(reduction=REDUCE_F64, use_graphs=args.graphs, no_tile_skip=0 if skip else 1)
        v.set_stream(stream.cuda_stream)
        v.enable_multigrid()
        v.enable_sparse()
        v.set_active_columns(mask)
        v.set_free_surface(np.where(mask != 0, s["eta"], rest).astype(np.float32), s["rest"])
        return v

    def timed(v, steps, clocks=None):
        def step():
            v.set_velocity_device(du.data_ptr(), dv.data_ptr(), dw.data_ptr())
            v.reset_pressure()
            return v.project_mobile3(scale, k1, 4000)
        for _ in range(args.warmup):
            rep = step()
        torch.cuda.synchronize()
        barrier(world)
        launches0 = v.kernel_launches()
        if clocks:
            clocks.mark(True)
        total = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            rep = step()
            b.record(stream)
            torch.cuda.synchronize()
            total += a.elapsed_time(b)
        if clocks:
            clocks.mark(False)
        return max_over_ranks(total, world), rep, v.kernel_launches() - launches0

    full = np.ones(s["nx"] * s["ny"], np.uint8)
    side_steps = max(10, args.steps // 3)
    with ClockSampler(local) as clocks:
        ms_set, rep, launches = timed(volume(s["mask"], True), args.steps, clocks)
    ms_all_tiles, rep_all, _ = timed(volume(s["mask"], False), side_steps)
    ms_dense, rep_dense, _ = timed(volume(full, True), side_steps)
    if rank == 0:
        frac = float(s["mask"].mean())
        cpu = None
        if world == 1 and not args.no_cpu:
            from oracle import oracle as O
            O.build()
            O.set_threads(O.max_threads())
            o = O.OracleVolume(s["nx"], s["ny"], s["nz"], s["dx"], s["rho"], s["g"])
            o.enable_multigrid()
            o.enable_sparse()
            o.set_active_columns(s["mask"])
            times = []
            t_start = time.perf_counter()
            while not times or (time.perf_counter() - t_start < 20.0 and len(times) < 3):
                o.set_free_surface(np.where(s["mask"] != 0, s["eta"], rest).astype(np.float32), s["rest"])
                o.set_velocity(s["u"], s["v"], s["w"])
                t0 = time.perf_counter()
                o.project_mobile(scale, k1, 4000)
                times.append(time.perf_counter() - t0)
            cpu = {"value": len(times) / sum(times), "unit": "projections/s", "cores": O.max_threads(), "kind": "port",
                   "sample": f"{len(times)} projections of the same set, oracle with OpenMP (it loops over the window)"}
        out = {
            "impl": "b200",
            "metric": f"sparse-set projections/s ({args.size}x{args.size}x{s['nz']} window, {100 * frac:.0f}% of the "
                      f"columns in the set)",
            "value": world * args.steps / (ms_set * 1e-3), "unit": "projections/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_set / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded sparse window)",
            "config": {"workload": f"sparse_window {args.size}^2 x {s['nz']}: 8x8-column blocks within 3 blocks of a "
                                   f"curved path, 5 cm bumps, N(0,0.3) faces; projection from p = 0",
                       "active_fraction": frac, "iterations": rep.iterations, "parallelism": f"replicas x{world}",
                       "l2": "256 MiB written between steps"},
            "every_tile": {"value": world * side_steps / (ms_all_tiles * 1e-3), "iterations": rep_all.iterations,
                           "note": "the same set, every tile of the window processed"},
            "dense_window": {"value": world * side_steps / (ms_dense * 1e-3), "iterations": rep_dense.iterations,
                             "note": "every column of the window in the set"},
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="basin", choices=["basin", "wave", "patches", "sparse"],
                    help="basin: the 128^3 box basin the metric is quoted on; wave: the 256^3 breaking wave; "
                         "patches: the batched delta patches; sparse: a sparse set in a 256^2 x 32 window")
    ap.add_argument("--patches", type=int, default=256, help="patch count of the patches workload")
    ap.add_argument("--threads", type=int, default=0, help="host workers of fd3_project_batch (0 = up to 16)")
    ap.add_argument("--streams", type=int, default=1,
                    help="patches workload: 1 also times the per-patch stream path (fd3_project_batch) beside it")
    ap.add_argument("--size", type=int, default=None, help="grid side (default 128 for basin, 256 for wave)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--learned", type=int, default=1,
                    help="1: also train the learned preconditioner and time learned-FCG projections (N=1 only)")
    ap.add_argument("--mixed", type=int, default=1, help="1: also time the FP16-storage V-cycle on the same scene")
    ap.add_argument("--parts", type=int, default=1,
                    help="1: also time a mobile step, the second-order advection, a solid re-cut and a level change")
    ap.add_argument("--wave", type=int, default=1,
                    help="1: also compare FP32 MGPCG, FP16-storage MGPCG and learned FCG on the 256^3 breaking wave "
                         "(N=1, basin workload only)")
    ap.add_argument("--train-samples", type=int, default=20000,
                    help="training samples of the learned preconditioner (20,000 at 64^3, as config 4 asks)")
    ap.add_argument("--kernels", type=int, default=0,
                    help="fine-level kernel family (fd3_options.kernels): 0 the default (TMA-staged layers from "
                         "2^23 cells, else two cells per thread), 3 two cells per thread, 4 four cells per thread, "
                         "5 TMA-staged layers, 2 one cell per thread in the same blocking")
    ap.add_argument("--graphs", type=int, default=1,
                    help="1: the inner loop as a CUDA graph with a WHILE node; 0: host-driven (for ncu launch lists)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.size is None:
        args.size = 256 if args.workload in ("wave", "sparse") else 128
    if args.workload == "sparse":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the sparse-window workload has no reference arm; "
                              "its line carries the oracle's cpu_baseline"}), flush=True)
        else:
            run_sparse(args)
    elif args.workload == "patches":
        if args.impl == "reference":
            run_reference_patches(args)
        else:
            run_patches(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()

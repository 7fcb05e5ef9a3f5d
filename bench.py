#!/usr/bin/env python
"""Fluid MLUPS of the fused D3Q27 stream + collide step on one B200 (and N replicas).

Workload (one time step = one "step"): the synthetic TCPC junction 256x192x160, FP32
storage, cumulant collision, Carreau-Yasuda viscosity from the non-equilibrium moments,
plug IVC/SVC inflow, rho = 1 outlets, FP64 mean/rms accumulators on.  The junction is
sparse (about 5 % fluid), so the data one step touches fits in the 126 MB L2: every timed
step is preceded by a 512 MB buffer write that flushes L2, and steps are timed one by one
with CUDA events on the library's stream.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--workload junction|dense_box] [--shape nx,ny,nz]
                    [--dtype f32|f16|bf16|f64] [--collision CUM] [--no-stats] [--no-extras]

On one GPU the FP32 line also carries, unless --no-extras, the same workload in FP16
storage with the errors of FP32 and FP16 against FP64 on a short noisy-inflow run
("storage_f16"), and, for the junction, the 15-case study batched in one launch group
against the cases stepped one after another ("batch") and the throughput configuration,
the dense 768x576x480 box, for the cumulant in FP32/FP16/BF16 storage with and without
the FP64 mean/rms sums, BGK and MRT_LES in FP32 and FP16, and KBC_N4 in FP32 ("dense_box").

Multi-GPU (launched by torchrun, one rank per GPU): every rank runs its own replica of the
case (the path has no exchange step on one GPU); value = all fluid-cell updates / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fluid MLUPS & %HBM roofline; FP16 vs FP32 storage at stated error; batch gain"
STORAGE_BYTES = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dtype", default="f32")
    ap.add_argument("--collision", default="CUM")
    ap.add_argument("--cy-mode", default="local-neq")
    ap.add_argument("--workload", default="junction", choices=["junction", "dense_box"])
    ap.add_argument("--shape", default=None, help="dense box nx,ny,nz (default 768,576,480)")
    ap.add_argument("--no-stats", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=400)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-extras", action="store_true", help="skip the FP16-storage, dense-box and 15-case batch measurements")
    ap.add_argument("--dense-warmup", type=int, default=200)
    ap.add_argument("--dense-steps", type=int, default=100)
    ap.add_argument("--launch", default=None,
                    help="block,cells_per_thread (e.g. 128,2) instead of the autotuned launch shape")
    return ap.parse_args()


class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str = "nccl"):
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(self.local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                        device_id=torch.device("cuda", self.local))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
            self.backend = backend
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        dev = f"cuda:{self.local}" if getattr(self, "backend", "nccl") == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(key: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get(key)
    return None


def bytes_per_update(dtype: str, stats: bool, stats_f64: bool = True) -> float:
    """Algorithmic bytes per fluid-cell update: 27 reads + 27 writes of the populations,
    the 1-byte label, and the mean/rms sums (6 read + 6 written)."""
    b = 2 * 27 * STORAGE_BYTES[dtype] + 1
    if stats:
        b += 2 * 6 * (8 if stats_f64 else 4)
    return float(b)


def workload(a, dtype=None):
    """The measured case: the junction configuration (sparse TCPC junction with
    Carreau-Yasuda blood) or the dense-box throughput configuration."""
    from nonnewlbm_b200 import workloads as W

    dt = dtype or a.dtype
    if a.workload == "dense_box":
        shape = tuple(int(v) for v in a.shape.split(",")) if a.shape else (768, 576, 480)
        return W.dense_box(dtype=dt, collision=a.collision, shape=shape)
    return W.junction_cy(dtype=dt, collision=a.collision, cy_mode=a.cy_mode)


def reference_lattice(w, collision: str):
    """The reference's own headers (oracle/_ref, single precision like the production
    build) on the workload's lattice; the dense box is sampled as an 8-cell slab in z.
    Returns (RefLattice, fluid cells, sample text)."""
    import oracle as O
    from nonnewlbm_b200 import geometry as G

    nx, ny, nz = w.shape
    if w.kind == "tcpc":
        orc = O.Oracle(nx, ny, nz)
        rc, counts = orc.setup_tcpc(w.wall)
        m = orc.get_map()
        del orc
        ref = O.RefLattice(nx, ny, nz, collision=O.COLLISIONS.index(collision), equilibrium=O.EQ_INV_CUM_REF,
                           nu=w.nu, prec=4, fast=True)
        ref.set_map(m)
        ref.set_inflow(ivc_flux=w.u_ivc * counts[0], svc_flux=w.u_svc * counts[1])
        what = (f"the full {nx}x{ny}x{nz} junction; the single-rank reference leaves Carreau-Yasuda inert "
                f"(zero strain), so the Newtonian step is timed")
    else:
        nz = min(nz, 8)
        m, prof = G.dense_box_map(nx, ny, nz)
        ref = O.RefLattice(nx, ny, nz, collision=O.COLLISIONS.index(collision), equilibrium=O.EQ_INV_CUM_REF,
                           nu=w.nu, prec=4, fast=True)
        ref.set_map(m)
        ref.set_inflow_profile(G.expand_profile(m, prof) * w.u_ivc)
        what = f"a {nx}x{ny}x{nz} slab of the dense box (same rows, periodic in y and z)"
    ref.init_equilibrium()
    fluid = int(np.count_nonzero((m == G.MAP_FLUID) | (m == G.MAP_PERIODIC)))
    return ref, fluid, what


def run_reference(a, dist: Dist):
    """Times the reference's own per-cell collision / streaming headers on the host cores."""
    if dist.rank != 0:
        return 0
    import oracle as O

    if not O.ref_available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libnnlbm_ref_fast.so not built "
                          "(the reference checkout was absent at build time)"}))
        return 0
    w = workload(a, "f32")
    threads = os.cpu_count() or 1
    O.ref_lib(fast=True).ref_set_threads(threads)
    ref, fluid, what = reference_lattice(w, a.collision)
    # at least 3 warm-up steps like the GPU arm, at most 5 (a reference step takes ~0.2 s)
    warm = min(max(a.warmup, 3), 5)
    for _ in range(warm):
        ref.step(1, accumulate_stats=not a.no_stats)
    times = []
    t_end = time.perf_counter() + a.cpu_seconds
    steps = 0
    while steps < max(1, a.steps) and (time.perf_counter() < t_end or steps < 2):
        t0 = time.perf_counter()
        ref.step(1, accumulate_stats=not a.no_stats)
        times.append(time.perf_counter() - t0)
        steps += 1
    sec = float(np.mean(times))
    mlups = fluid / sec / 1e6
    sample = (f"{steps} steps of {what} ({fluid} fluid cells) on {threads} host threads, reference collision and "
              f"streaming headers in single precision (TraitsSP)")
    line = {"impl": "reference", "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": a.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": round(sec * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "collision": a.collision, "storage": "f32 (reference TraitsSP)",
                       "cells": int(np.prod(w.shape)), "fluid_cells_timed": fluid},
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline_sample(w, seconds: float, collision: str) -> dict:
    import oracle as O

    if not O.ref_available(fast=True):
        return {"value": None, "unit": "MLUPS", "cores": 0, "kind": "reference", "sample": "oracle/_ref not built"}
    threads = os.cpu_count() or 1
    O.ref_lib(fast=True).ref_set_threads(threads)
    ref, fluid, what = reference_lattice(w, collision)
    ref.step(1)
    t0 = time.perf_counter()
    n = 0
    while n < 2 or time.perf_counter() - t0 < seconds:
        ref.step(1)
        n += 1
    sec = (time.perf_counter() - t0) / n
    return {"value": round(fluid / sec / 1e6, 3), "unit": "MLUPS", "cores": threads, "kind": "reference",
            "sample": f"{n} steps of {what} ({fluid} fluid cells), reference headers in single precision, "
                      f"{threads} OpenMP threads"}


def main() -> int:
    a = parse()
    dist = Dist()
    dist.init()
    try:
        if a.impl == "reference":
            return run_reference(a, dist)
        return run_ours(a, dist)
    finally:
        dist.close()


class L2Flush:
    """Every timed step starts from a cold L2: a 512 MB write, then a 256 MB read that leaves
    L2 holding clean lines (so the flush's own write-back does not land in the step)."""

    def __init__(self, dev: int):
        import torch

        self.flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.int32, device=f"cuda:{dev}")
        self.clean = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.int32, device=f"cuda:{dev}")
        self.sink = torch.zeros(1, dtype=torch.int64, device=f"cuda:{dev}")

    def __call__(self):
        self.flush.zero_()
        self.sink += self.clean.sum()


def timed_steps(lat, steps: int, stats: bool, flush: L2Flush, dev: int) -> float:
    """Device milliseconds of `steps` single steps, each bracketed by CUDA events on the
    library's stream after an L2 flush outside the events; the steps are enqueued without
    host waits (NNLBM_STEP_ASYNC) and the watchdog is checked once at the end."""
    import torch

    stream = torch.cuda.ExternalStream(lat.stream, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush()
            ev[k][0].record(stream)
            lat.step(1, stats=stats, wait=False)
            ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    lat.sync()
    return sum(e0.elapsed_time(e1) for e0, e1 in ev)


def cold_kernel_times(lat, steps: int, stats: bool, flush: L2Flush, dev: int) -> dict:
    """Mean device milliseconds per launch of each kernel kind of `steps` single steps, each
    launched as separate kernels with CUDA events around them (Lattice.profile_step) after an
    L2 flush on the library's stream."""
    import torch

    stream = torch.cuda.ExternalStream(lat.stream, device=dev)
    tot = {}
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush()
        for k, (ms, n) in lat.profile_step(1, stats=stats).items():
            t = tot.setdefault(k, [0.0, 0])
            t[0] += ms * n
            t[1] += n
    return {k: ((t[0] / t[1]) if t[1] else 0.0, t[1]) for k, t in tot.items()}


def storage_comparison(a, flush: L2Flush, dev: int, f32_mlups: float) -> dict:
    """FP16 storage on the same workload and timing, beside the FP32 line, with the error of
    a short FP16 and FP32 run of the junction against FP64 (studies.precision_study)."""
    from nonnewlbm_b200 import studies
    from nonnewlbm_b200 import workloads as W

    w = workload(a, "f16")
    lat = W.build_lattice(w, device=dev)
    fluid = lat.step_info()["fluid_cells"]
    lat.autotune(stats=not a.no_stats)
    lat.step(max(3, a.warmup), stats=not a.no_stats)
    n = max(20, min(a.steps, 200))
    ms = timed_steps(lat, n, not a.no_stats, flush, dev)
    lat.close()
    f16 = fluid * n / (ms / 1e3) / 1e6
    err = studies.precision_study(scale=1.0, steps=2000, collision=a.collision, dtypes=("f64", "f32", "f16"), device=dev)
    r = err["runs"]
    return {"f16_mlups": round(f16, 2), "f32_mlups": round(f32_mlups, 2), "ratio_f16_f32": round(f16 / f32_mlups, 3),
            "error_vs_f64": {k: {e: r[k][e] for e in ("velocity_l2_rel", "velocity_linf_rel", "outlet_split_abs_err",
                                                       "wss_l2_rel")} for k in ("f32", "f16")},
            "error_run": f"{err['workload']} {err['collision']} local-neq CY, 2000 steps, inflow noise +-5 %/100 steps, "
                         f"seed {err['seed']}"}


# the throughput configuration's variants: (collision, storage, FP64 mean/rms on)
DENSE_VARIANTS = [("CUM", "f32", True), ("CUM", "f32", False), ("CUM", "f16", False), ("CUM", "bf16", False),
                  ("CUM", "f16", True), ("BGK", "f32", False), ("BGK", "f16", False), ("MRT_LES", "f32", False),
                  ("MRT_LES", "f16", False), ("KBC_N4", "f32", False)]


def dense_box_lines(dev: int, warmup: int, steps: int, shape=(768, 576, 480), variants=DENSE_VARIANTS) -> dict:
    """The dense periodic box (212 M cells, 22.9 GB of FP32 populations, far above L2) for
    each variant: `warmup` untimed steps, then `steps` steps timed as one block with CUDA
    events on the library's stream (steady state), the step kernel's mean launch time from
    events around 5 single launches, its roofline against the measured copy bandwidth, and
    the clocks sampled during the timed block."""
    import torch

    from nonnewlbm_b200 import workloads as W

    peak, peak_kind = measured_peaks()
    out = {"shape": list(shape), "warmup": warmup, "steps": steps,
           "timing": "one block of steps between two CUDA events (inputs 12-23 GB, far above L2)"}
    for col, dt, stats in variants:
        w = W.dense_box(dtype=dt, collision=col, shape=shape)
        lat = W.build_lattice(w, device=dev)
        fluid = lat.step_info()["fluid_cells"]
        lat.autotune(stats=stats)
        lat.step(warmup, stats=stats)
        stream = torch.cuda.ExternalStream(lat.stream, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(dev)
        sampler.start()
        time.sleep(0.3)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        lat.step(steps, stats=stats, wait=False)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        lat.sync()
        clocks = sampler.stop()
        ms = e0.elapsed_time(e1)
        prof_ms = lat.profile_step(5, stats=stats)
        k_ms = prof_ms["step"][0]
        bpu = bytes_per_update(dt, stats)
        mlups = fluid * steps / (ms / 1e3) / 1e6
        achieved = fluid * bpu / (k_ms / 1e3) / 1e9
        key = f"{col}_{dt}_{'stats' if stats else 'nostats'}"
        out[key] = {"mlups": round(mlups, 1), "ms_per_step": round(ms / steps, 4), "fluid_cells": fluid,
                    "kernel_ms": round(k_ms, 4),
                    "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                 "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "bytes_per_update": bpu,
                                 "traffic": ncu_traffic(f"{w.name}:{dt}:{col}:none:{'stats' if stats else 'nostats'}")},
                    "clocks": clocks}
        lat.close()
        del lat
    # FP16 over FP32 storage, per collision and accumulator setting
    for col in sorted({v[0] for v in variants}):
        for stats in (False, True):
            s = "stats" if stats else "nostats"
            a16, a32 = out.get(f"{col}_f16_{s}"), out.get(f"{col}_f32_{s}")
            if a16 and a32:
                out[f"ratio_f16_f32_{col}_{s}"] = round(a16["mlups"] / a32["mlups"], 3)
    return out


def batch_gain(dev: int, dtype: str = "f32") -> dict:
    """The 15-case study (5 inflow pairs x 3 rheologies, seeded scales in [0.5, 1]): one
    batched launch group against the cases stepped one after another."""
    from nonnewlbm_b200 import studies

    r = studies.run_batch(studies.batch_cases(seed=2024, dtype=dtype), steps=100, warmup=10, device=dev)
    return {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items() if k != "scales"}


def run_ours(a, dist: Dist) -> int:
    import torch

    from nonnewlbm_b200 import workloads as W

    dev = dist.local
    torch.cuda.set_device(dev)
    stats = not a.no_stats
    w = workload(a)
    lat = W.build_lattice(w, device=dev)
    info = lat.step_info()
    if a.launch:
        block, cpt = (int(v) for v in a.launch.split(","))
        lat.set_launch(block, cpt)
    else:
        lat.autotune(stats=stats)
    lat.step(max(3, a.warmup), stats=stats)
    # the populations touched per step can be smaller than the 126 MB L2 (a sparse
    # junction), so every timed step starts from a cold L2
    flush = L2Flush(dev)
    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.3)
    dist.barrier()
    ms = timed_steps(lat, a.steps, stats, flush, dev)
    dist.barrier()
    clocks = sampler.stop()
    ms = dist.max(ms)
    fluid = info["fluid_cells"]
    value = fluid * a.steps * dist.world / (ms / 1e3) / 1e6

    # dominant kernel: per-launch device time with events around every kernel, each step
    # from a cold L2 like the timed steps
    prof = cold_kernel_times(lat, 20, stats, flush, dev)
    t_step_ms = prof["step"][0]
    bpu = bytes_per_update(a.dtype, stats)
    peak, peak_kind = measured_peaks()
    achieved = fluid * bpu / (t_step_ms / 1e3) / 1e9
    key = f"{w.name}:{a.dtype}:{a.collision}:{w.cy_mode}:{'stats' if stats else 'nostats'}"
    traffic = ncu_traffic(key)

    # end to end through the public API: per step the host sends that step's inflow row
    # (a +-1 % pulsation, so every row differs from the last and is uploaded) and reads
    # back the step's status block with its FP64 mass / flux sums (NNLBM_STEP_READBACK),
    # one step deep: step k + 1 is enqueued before the host waits for the sums of step k
    if w.kind == "tcpc":
        q0 = np.array([w.u_ivc * w.notes["counts"]["left_area"], w.u_svc * w.notes["counts"]["right_area"]])
    else:
        q0 = np.zeros(2)
    rows = [np.array([[*(q0 * (1.0 + 0.01 * np.sin(0.1 * k))), 1.0]]) for k in range(a.e2e_steps)]
    dist.barrier()
    t0 = time.perf_counter()
    red = None
    for k in range(a.e2e_steps):
        lat.set_schedule(rows[k])
        lat.step(1, stats=stats, reduce=True, wait=False, readback=True)
        if k > 0:
            red = lat.readback()[0]
    red = lat.readback()[0]
    t_e2e = time.perf_counter() - t0
    t_e2e = dist.max(t_e2e)
    e2e = fluid * a.e2e_steps * dist.world / t_e2e / 1e6
    h2d = 32 if w.dtype != "f64" else 56  # the step's control row
    d2h = 16 + 32 * 64 + 8  # the context's status block: step cursors, 32 stripes of mass/flux sums, watchdog flag
    lat.close()

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": dist.world, "steps": a.steps,
            "warmup": max(3, a.warmup), "ms_per_step": round(ms / a.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": a.dtype, "data": "synthetic",
            "config": {"workload": w.name, "timing": "per-step CUDA events; before every step L2 is flushed by a 512 MB "
                                                      "write followed by a 256 MB read (clean lines)", "shape": list(w.shape), "fluid_cells": fluid, "collision": a.collision,
                       "cy_mode": w.cy_mode, "storage": a.dtype, "stats": "fp64 mean/rms" if stats else "off",
                       "bc_cells": info["bc_cells"], "parallelism": f"replicas x{dist.world}",
                       "dt_s": w.notes.get("dt_s"), "dx_m": w.notes.get("dx_m")},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": f"k_step<{a.dtype},{a.collision}>", "bytes_per_update": bpu,
                         "kernel_ms": round(t_step_ms, 5),
                         "kernel_timing": "CUDA events around each launch of 20 single steps, L2 flushed before each",
                         "step_kernels_ms": {k: round(v[0], 5) for k, v in prof.items() if v[1]}},
            "e2e": {"value": round(e2e, 2), "unit": "MLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": a.steps * info["launches_per_step"],
            "clocks": clocks,
        }
        if dist.world == 1:
            line["cpu_baseline"] = cpu_baseline_sample(w, a.cpu_seconds, a.collision)
            if not a.no_extras and a.dtype == "f32":
                line["storage_f16"] = storage_comparison(a, flush, dev, value)
                if a.workload == "junction":
                    line["batch"] = batch_gain(dev)
                    line["batch_f16"] = batch_gain(dev, "f16")
                    line["dense_box"] = dense_box_lines(dev, a.dense_warmup, a.dense_steps)
        line["reduce_last"] = [float(v) for v in red] if red is not None else None
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

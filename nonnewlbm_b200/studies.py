"""The batched-case study and the storage-precision study of the TCPC step (one GPU).

Both stand on the synthetic junction of ``geometry.junction`` (the real TCPC mask needs
the reference's STL pipeline, which is not available).

* ``batch_cases`` / ``run_batch``: the 15-case study -- 5 (IVC, SVC) lattice inflow pairs,
  the last one pulsating at 1 Hz with 20 % amplitude, times 3 rheologies (Newtonian blood
  nu = 3.3e-6 m^2/s and two Carreau-Yasuda parameter sets), each on a junction scaled by a
  seeded factor in [0.5, 1.0] of the 256x192x160 base.  The reference runs one case per
  solver process (scripts/run_all_cases.py:132-150); here all 15 share one launch group
  (one work list, one CUDA graph per A-A parity).  ``run_batch`` times the batched steps
  and the same cases stepped one context after another.
* ``precision_study``: one junction stepped in FP64, FP32, FP16 and BF16 storage with the
  same inflow, perturbed by +-5 % white noise redrawn every 100 steps from a seeded
  generator; errors of the reduced-precision runs against the FP64 run (velocity L2 and
  L-infinity, outlet flow split, wall-shear proxy).

    python -m nonnewlbm_b200.studies batch [--steps N] [--dtype f32]
    python -m nonnewlbm_b200.studies precision [--steps N] [--scale 1.5] [--collision KBC_N4]
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass

import numpy as np

from . import capi
from . import geometry as G
from . import units
from .lattice import CaseSpec, Lattice

BLOOD_DENSITY = 1060.0
RHEOLOGIES = {
    "newtonian": units.Material("newtonian_blood", BLOOD_DENSITY, 3.3e-6, 3.3e-6 * BLOOD_DENSITY, 1.0, 2.0, 1.0, False),
    "cy_0.056_0.3568": units.Material("cy_a", BLOOD_DENSITY, 0.00345 / BLOOD_DENSITY, 0.056, 3.313, 2.0, 0.3568, True),
    "cy_0.022_0.5": units.Material("cy_b", BLOOD_DENSITY, 0.00345 / BLOOD_DENSITY, 0.022, 3.313, 2.0, 0.5, True),
}
INFLOW_PAIRS = [(0.02, 0.015, 0.0), (0.03, 0.02, 0.0), (0.04, 0.025, 0.0), (0.05, 0.03, 0.0), (0.05, 0.05, 0.2)]
BASE_DX = 0.25e-3
NU_LBM = 0.01


@dataclass
class StudyCase:
    name: str
    scale: float
    wall: np.ndarray            # geometry wall array [z][y][x]
    spec: CaseSpec
    u_ivc: float
    u_svc: float
    pulse: float                # relative amplitude of the 1 Hz pulsation
    dt_s: float


def junction_wall(scale: float) -> np.ndarray:
    return G.study_to_geometry(G.junction(scale=scale) if scale != 1.0 else G.junction())


def batch_cases(seed: int = 2024, dtype: str = "f32", collision: str = "CUM") -> list[StudyCase]:
    """The 15 cases: inflow pair x rheology, geometry scale U[0.5, 1.0] from ``seed``."""
    rng = np.random.default_rng(seed)
    out = []
    for ip, (u_ivc, u_svc, pulse) in enumerate(INFLOW_PAIRS):
        for rname, mat in RHEOLOGIES.items():
            scale = float(rng.uniform(0.5, 1.0))
            wall = junction_wall(scale)
            nz, ny, nx = wall.shape
            dx = BASE_DX / scale
            conv = units.lattice_units(mat, dx, NU_LBM)
            spec = CaseSpec((nx, ny, nz), collision=collision, dtype=dtype,
                            cy_mode="local-neq" if mat.carreau_yasuda else "none", nu=conv["nu"],
                            cy=(conv["nu0"], conv["lambda"], conv["a"], conv["n"]))
            out.append(StudyCase(f"pair{ip}_{rname}", scale, wall, spec, u_ivc, u_svc, pulse, conv["dt"]))
    return out


def _schedule(case: StudyCase, areas: dict, step0: int, n: int) -> np.ndarray:
    t = (step0 + np.arange(n)) * case.dt_s
    f = 1.0 + case.pulse * np.sin(2.0 * math.pi * 1.0 * t)
    rows = np.empty((n, 3))
    rows[:, 0] = case.u_ivc * areas["left_area"] * f
    rows[:, 1] = case.u_svc * areas["right_area"] * f
    rows[:, 2] = 1.0
    return rows


def _setup(lat: Lattice, cases: list[StudyCase], first: int = 0) -> list[dict]:
    areas = []
    for k, case in enumerate(cases):
        a = lat.setup_tcpc(case.wall, ic=first + k)
        lat.set_inflow(ivc_flux=case.u_ivc * a["left_area"], svc_flux=case.u_svc * a["right_area"], ic=first + k)
        areas.append(a)
    lat.init_equilibrium()
    return areas


def run_batch(cases: list[StudyCase], steps: int = 200, warmup: int = 20, device: int = 0, autotune: bool = True) -> dict:
    """Batched (one context, one launch group) against sequential (one context per case,
    stepped one after another) wall time of ``steps`` steps of every case, each measured
    after ``warmup`` steps; the per-step inflow rows (with the pulsation) are uploaded in
    one call before each timed run, outside the clock.  With ``autotune`` both the batched
    context and every single one pick their launch shape first (nnlbm_autotune)."""
    fluid = 0
    # batched
    lat = Lattice([c.spec for c in cases], device=device)
    areas = _setup(lat, cases)
    if autotune:
        lat.autotune()
    lat.step(warmup)
    for k, c in enumerate(cases):
        lat.set_schedule(_schedule(c, areas[k], warmup, steps), ic=k)
    t0 = time.perf_counter()
    lat.step(steps)
    t_batched = time.perf_counter() - t0
    fluid = sum(lat.step_info(k)["fluid_cells"] for k in range(len(cases)))
    lat.close()
    # one after another
    t_seq = 0.0
    for c in cases:
        one = Lattice(c.spec, device=device)
        a = _setup(one, [c])[0]
        if autotune:
            one.autotune()
        one.step(warmup)
        one.set_schedule(_schedule(c, a, warmup, steps))
        t0 = time.perf_counter()
        one.step(steps)
        t_seq += time.perf_counter() - t0
        one.close()
    return {"cases": len(cases), "steps": steps, "fluid_cells": int(fluid), "dtype": cases[0].spec.dtype,
            "autotuned": bool(autotune),
            "batched_s": t_batched, "sequential_s": t_seq, "gain": t_seq / t_batched,
            "batched_mlups": fluid * steps / t_batched / 1e6, "sequential_mlups": fluid * steps / t_seq / 1e6,
            "scales": [round(c.scale, 4) for c in cases]}


def shard_cases(cases: list, rank: int, world: int, size=lambda c: int(c.wall.size)) -> list:
    """This rank's share of a batch split over `world` GPUs (one process each): the cases
    are independent, so they are dealt out whole, largest first, each to the rank with the
    least work so far; every rank computes the same split and no data crosses GPUs."""
    load = [0] * world
    owner = {}
    for i in sorted(range(len(cases)), key=lambda i: (-size(cases[i]), i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += size(cases[i])
    return [cases[i] for i in range(len(cases)) if owner[i] == rank]


def _near_wall(wall_flags: np.ndarray) -> np.ndarray:
    wf = wall_flags
    near = np.zeros(wf.shape, dtype=bool)
    near[:, :, 1:] |= wf[:, :, :-1]
    near[:, :, :-1] |= wf[:, :, 1:]
    near[:, 1:, :] |= wf[:, :-1, :]
    near[:, :-1, :] |= wf[:, 1:, :]
    near[1:, :, :] |= wf[:-1, :, :]
    near[:-1, :, :] |= wf[1:, :, :]
    return near


def precision_study(scale: float = 1.5, steps: int = 50000, seed: int = 7, collision: str = "KBC_N4",
                    dtypes=("f64", "f32", "f16", "bf16"), device: int = 0) -> dict:
    """The scaled junction with Carreau-Yasuda blood stepped in each storage type with the
    same noisy inflow (IVC 0.03, SVC 0.02 lattice units, +-5 % white noise per 100 steps);
    errors of each run against the FP64 one, on the last step:
      velocity: ||u - u64||_2 / ||u64||_2 and max|u - u64| / max|u64| over fluid cells;
      split:    outlet flow split Q5 / (Q5 + Q6) (FP64 plane sums of nnlbm_reduce) and its
                absolute difference;
      wss:      the wall-shear proxy nu(gamma) gamma on fluid cells next to a wall (lattice
                units), L2-relative difference."""
    wall = junction_wall(scale)
    nz, ny, nx = wall.shape
    mat = RHEOLOGIES["cy_0.056_0.3568"]
    conv = units.lattice_units(mat, BASE_DX / scale, NU_LBM)
    m, counts, rc, wflags = capi.tcpc_labels(wall, with_wall_flags=True)
    fluid = m == G.MAP_FLUID
    near = _near_wall(wflags) & fluid
    rng = np.random.default_rng(seed)
    noise = rng.uniform(-0.05, 0.05, size=(steps + 99) // 100)
    results = {}
    ref = None
    for dt in dtypes:
        lat = Lattice(CaseSpec((nx, ny, nz), collision=collision, dtype=dt, cy_mode="local-neq", nu=conv["nu"],
                               cy=(conv["nu0"], conv["lambda"], conv["a"], conv["n"])), device=device)
        a = lat.setup_tcpc(wall)
        lat.init_equilibrium()
        t0 = time.perf_counter()
        done = 0
        for blk, e in enumerate(noise):
            n = min(100, steps - done)
            f = 1.0 + e
            lat.set_schedule(np.array([[0.03 * a["left_area"] * f, 0.02 * a["right_area"] * f, 1.0]]))
            last = done + n == steps
            lat.step(n, macro=last, reduce=last)
            done += n
        wall_s = time.perf_counter() - t0
        u = np.stack([lat.macro(capi.M_VX), lat.macro(capi.M_VY), lat.macro(capi.M_VZ)])
        S = np.stack([lat.macro(f) for f in (capi.M_S11, capi.M_S12, capi.M_S13, capi.M_S22, capi.M_S32, capi.M_S33)])
        red = lat.reduce()
        lat.close()
        gam = math.sqrt(2.0) * np.sqrt(S[0] ** 2 + S[3] ** 2 + S[5] ** 2 + 2.0 * (S[1] ** 2 + S[2] ** 2 + S[4] ** 2))
        nu = conv["nu"] + (conv["nu0"] - conv["nu"]) * np.power(1.0 + np.power(gam * conv["lambda"], conv["a"]),
                                                                  (conv["n"] - 1.0) / conv["a"])
        wss = (nu * gam)[near]
        split = red[3] / (red[3] + red[4]) if red[3] + red[4] != 0 else float("nan")
        row = {"steps": steps, "wall_s": round(wall_s, 3), "mlups": round(int(fluid.sum()) * steps / wall_s / 1e6, 1),
               "outlet_split": float(split), "q_ivc": float(red[1]), "q_svc": float(red[2]), "q5": float(red[3]),
               "q6": float(red[4])}
        uf = u[:, fluid]
        if ref is None:
            ref = (uf, split, wss)
        else:
            du = uf - ref[0]
            row["velocity_l2_rel"] = float(np.sqrt((du ** 2).sum()) / np.sqrt((ref[0] ** 2).sum()))
            row["velocity_linf_rel"] = float(np.abs(du).max() / np.abs(ref[0]).max())
            row["outlet_split_abs_err"] = float(abs(split - ref[1]))
            row["wss_l2_rel"] = float(np.sqrt(((wss - ref[2]) ** 2).sum()) / np.sqrt((ref[2] ** 2).sum()))
        results[dt] = row
    return {"workload": f"junction_{nx}x{ny}x{nz}", "collision": collision, "cy": "local-neq CY mu0=0.056 n=0.3568",
            "seed": seed, "noise": "+-5 % uniform, redrawn every 100 steps", "fluid_cells": int(fluid.sum()),
            "near_wall_cells": int(near.sum()), "runs": results}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("study", choices=["batch", "precision"])
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--dtype", default="f32")
    ap.add_argument("--scale", type=float, default=1.5)
    ap.add_argument("--collision", default=None)
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.study == "batch":
        cases = batch_cases(seed=a.seed if a.seed is not None else 2024, dtype=a.dtype, collision=a.collision or "CUM")
        print(json.dumps(run_batch(cases, steps=a.steps or 200, device=a.device)))
    else:
        print(json.dumps(precision_study(scale=a.scale, steps=a.steps or 50000, seed=a.seed if a.seed is not None else 7,
                                         collision=a.collision or "KBC_N4", device=a.device)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

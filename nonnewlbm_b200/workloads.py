"""Synthetic study workloads (the five study configurations of the TCPC step) in lattice
units, shared by the bench, the tests and the driver.

The real TCPC25_03 voxel mask is produced by the reference's STL pipeline
(geometry/tcpc_geometry.py), which needs trimesh and vtk; seeded synthetic geometries with
the same label conventions stand in for it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import geometry as G
from . import units


@dataclass
class Workload:
    name: str
    shape: tuple                 # (nx, ny, nz)
    collision: str
    dtype: str
    nu: float                    # lattice nu (nu_inf with Carreau-Yasuda)
    cy_mode: str = "none"
    cy: tuple = (0.0, 0.0, 2.0, 1.0)
    kind: str = "tcpc"           # tcpc | map
    wall: np.ndarray | None = None
    map: np.ndarray | None = None
    profile: np.ndarray | None = None
    u_ivc: float = 0.0           # plug velocities (TCPC) or profile peak (map)
    u_svc: float = 0.0
    stats: bool = False
    notes: dict = field(default_factory=dict)


def junction_cy(dtype: str = "f32", collision: str = "CUM", scale: float = 1.0, cy_mode: str = "local-neq",
                nu_lbm: float = 0.01) -> Workload:
    """Synthetic TCPC junction 256x192x160 (times ``scale``), dx = 0.25 mm / scale,
    Carreau-Yasuda blood (mu0 0.056 Pa s, mu_inf 0.00345 Pa s, lambda 3.313 s, n 0.3568,
    a 2, 1060 kg/m^3), plug inflow IVC 0.03 / SVC 0.02 lattice units, rho = 1 outlets,
    mean/rms accumulators on."""
    study = G.junction(scale=scale) if scale != 1.0 else G.junction()
    wall = G.study_to_geometry(study)
    nz, ny, nx = wall.shape
    dx = 0.25e-3 / scale
    mat = units.Material("cy_blood", 1060.0, 0.00345 / 1060.0, 0.056, 3.313, 2.0, 0.3568, True)
    conv = units.lattice_units(mat, dx, nu_lbm)
    return Workload(name=f"junction_{nx}x{ny}x{nz}_cy", shape=(nx, ny, nz), collision=collision, dtype=dtype,
                    nu=conv["nu"], cy_mode=cy_mode, cy=(conv["nu0"], conv["lambda"], conv["a"], conv["n"]),
                    kind="tcpc", wall=wall, u_ivc=0.03, u_svc=0.02, stats=True,
                    notes={"dx_m": dx, "dt_s": conv["dt"], "material": "CY mu0=0.056 mu_inf=0.00345 lambda=3.313 n=0.3568 a=2"})


def pipe(dtype: str = "f64", collision: str = "CUM") -> Workload:
    """96x32x32 pipe of radius 12, parabolic inlet peak 0.04, rho = 1 outlet, tau = 0.6."""
    m, prof = G.pipe_map(96, 32, 32, 12.0)
    return Workload(name="pipe_96x32x32", shape=(96, 32, 32), collision=collision, dtype=dtype, nu=(0.6 - 0.5) / 3.0,
                    kind="map", map=m, profile=prof, u_ivc=0.04, stats=True)


def dense_box(dtype: str = "f32", collision: str = "CUM", shape=(768, 576, 480)) -> Workload:
    """Dense periodic-y/z box, x inlet u = 0.05, rho = 1 outlet, tau = 0.55."""
    m, prof = G.dense_box_map(*shape)
    return Workload(name=f"dense_box_{shape[0]}x{shape[1]}x{shape[2]}", shape=tuple(shape), collision=collision,
                    dtype=dtype, nu=(0.55 - 0.5) / 3.0, kind="map", map=m, profile=prof, u_ivc=0.05, stats=True)


def build_lattice(w: Workload, device: int = 0, stats_f64: bool = True):
    """Create a Lattice for the workload, set its map and inflow, initialise at rest."""
    from .lattice import CaseSpec, Lattice

    lat = Lattice(CaseSpec(w.shape, collision=w.collision, dtype=w.dtype, cy_mode=w.cy_mode, nu=w.nu, cy=w.cy,
                           stats_f64=stats_f64), device=device)
    if w.kind == "tcpc":
        counts = lat.setup_tcpc(w.wall)
        lat.set_inflow(ivc_flux=w.u_ivc * counts["left_area"], svc_flux=w.u_svc * counts["right_area"])
        w.notes["counts"] = counts
    else:
        lat.set_map(w.map)
        lat.set_inflow_profile(w.profile * w.u_ivc)
    lat.init_equilibrium()
    return lat

"""Materials and unit conversion of the TCPC solver.

Materials are the solver's hard-coded table (solver/sim_tcpc/sim_tcpc.cu:52-68), not
configs/materials.yaml, which nothing in the reference reads (its gx nu_inf also differs).
Conversions follow sim_tcpc.cu:795-814:
  dt      = nu_lbm / nu_phys * dx^2
  nu0_lbm = mu0 / rho / dx^2 * dt          (Carreau-Yasuda materials; else nu_lbm)
  lambda  = lambda_phys / dt, a and n unchanged (else 1, 2, 1)
  Q_lbm   = Q[ml/s] * 1e-6 / dx^3 * dt
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Material:
    name: str
    density: float
    nu_inf: float
    mu0: float
    lam: float
    a: float
    n: float
    carreau_yasuda: bool


MATERIALS = {
    "newtonian": Material("newtonian", 1000.0, 1.0e-6, 1.0e-3, 1.0, 2.0, 1.0, False),
    "sx": Material("sx", 1151.0, 3.72863999716223e-3 / 1151.0, 3.32933884442747e-2, 1.20785676226298,
                   0.925354152818718, 0.463126647, True),
    "gx": Material("gx", 1088.0, 4.85563692580026e-3 / 1088.0, 1.58517801201338e-2, 0.0280506051570583,
                   2.34147778848562, 0.463126647, True),
}


def material_by_name(name: str) -> Material:
    """materialByName (sim_tcpc.cu:52-68); unknown names raise like the reference."""
    if name not in MATERIALS:
        raise ValueError(f"Unknown material '{name}'. Use newtonian, sx, or gx.")
    return MATERIALS[name]


def lattice_units(mat: Material, dx: float, nu_lbm: float) -> dict:
    """Lattice parameters of a material at spacing dx and lattice viscosity nu_lbm."""
    if not dx > 0:
        raise ValueError("Geometry spacing must be positive.")
    dt = nu_lbm / mat.nu_inf * dx * dx
    if mat.carreau_yasuda:
        nu0 = mat.mu0 / mat.density / dx / dx * dt
        lam, a, n = mat.lam / dt, mat.a, mat.n
    else:
        nu0, lam, a, n = nu_lbm, 1.0, 2.0, 1.0
    return {"dt": dt, "nu": nu_lbm, "nu0": nu0, "lambda": lam, "a": a, "n": n}


def flux_lbm(q_mls: float, dx: float, dt: float) -> float:
    """ml/s -> lattice flux (cells^3 per step), sim_tcpc.cu:813-814."""
    return q_mls * 1e-6 / (dx * dx * dx) * dt

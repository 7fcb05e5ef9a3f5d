"""The VTK output fields of StateTcpc::outputData (solver/sim_tcpc/sim_tcpc.cu:684-784),
restated in numpy from the macro fields, the mean/rms sums and the wall flags
(test infrastructure: the checker of nnlbm_output_fields and of the files the TCPC driver
writes).

Per cell, in double, as the reference's host code computes them (sim_tcpc.cu:716-745):
velocity = u * dx/dt; mean = sums / steps; rms = |<(rho u)^2> - <rho u>^2| per axis and their
norm (not square roots); turbulence = rms / |mean| (0 where |mean| <= 1e-10); pressure =
(rho - 1) rho_phys (dx/dt)^2 / 3; gamma_dot = sqrt(2) sqrt(S:S) / dt (gammaLbm, :684-695);
nu from the Carreau-Yasuda law or the lattice reference viscosity (localNuLbm, :697-707);
wss_proxy = mu gamma_dot next to a wall (nearWall, :709-714, neighbours outside the box are
not walls); strain rates S / dt.
"""
from __future__ import annotations

import numpy as np

FIELDS = ["velocity", "mean_velocity", "lbm_rho", "pressure_pa", "gamma_dot", "nu_phys_m2_s", "mu_phys_pa_s",
          "wss_proxy_pa", "turbulence_intensity", "rms_velocity", "strain_diag_1_s", "strain_shear_1_s"]


def output_data(rho, u, S, sums, steps, wall, dx, dt, density, nu_lbm, cy=None):
    """rho [z][y][x]; u [3][z][y][x] lattice velocity; S [6] as S11 S12 S13 S22 S32 S33; sums
    [6] as sum rho u_x, rho u_y, rho u_z, (rho u_x)^2, ...; steps summed; wall flags; cy =
    lattice (nu0, lambda, a, n) or None.  Returns {name: array} in double."""
    v2p = dx / dt
    diff = max(1.0, float(steps))
    mean = np.asarray(sums[:3]) * v2p / diff
    meansq = np.asarray(sums[3:]) * v2p * v2p / diff
    r = np.abs(meansq - mean * mean)
    rms = np.sqrt(r[0] ** 2 + r[1] ** 2 + r[2] ** 2)
    meanv = np.sqrt(mean[0] ** 2 + mean[1] ** 2 + mean[2] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        turb = np.where(np.abs(meanv) <= 1e-10, 0.0, rms / np.abs(meanv))
    S11, S12, S13, S22, S32, S33 = S
    gl = np.sqrt(2.0) * np.sqrt(S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S32 * S32))
    gdot = gl / dt
    if cy is None:
        nul = np.full(rho.shape, nu_lbm)
    else:
        nu0, lam, a, n = cy
        nul = nu_lbm + (nu0 - nu_lbm) * np.power(1.0 + np.power(gl * lam, a), (n - 1.0) / a)
    nup = nul * dx * dx / dt
    mup = nup * density
    wf = np.asarray(wall, dtype=bool)
    near = np.zeros(wf.shape, dtype=bool)
    near[:, :, 1:] |= wf[:, :, :-1]
    near[:, :, :-1] |= wf[:, :, 1:]
    near[:, 1:, :] |= wf[:, :-1, :]
    near[:, :-1, :] |= wf[:, 1:, :]
    near[1:, :, :] |= wf[:-1, :, :]
    near[:-1, :, :] |= wf[1:, :, :]
    return {"velocity": np.asarray(u) * v2p, "mean_velocity": mean, "lbm_rho": np.asarray(rho),
            "pressure_pa": (np.asarray(rho) - 1.0) * density * v2p * v2p / 3.0, "gamma_dot": gdot,
            "nu_phys_m2_s": nup, "mu_phys_pa_s": mup, "wss_proxy_pa": np.where(near, mup * gdot, 0.0),
            "turbulence_intensity": turb, "rms_velocity": rms,
            "strain_diag_1_s": np.stack([S11, S22, S33]) / dt, "strain_shear_1_s": np.stack([S12, S13, S32]) / dt}

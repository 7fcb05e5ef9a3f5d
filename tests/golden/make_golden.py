"""Generate the golden known-answer fixtures of tests/golden/ from the reference itself.

Every expected value here is computed by the reference's own code in FP64, on seeded
inputs: the per-cell headers (solver/lbm3d/*.h of buresjan/nonnewlbm) and, for the lattice
cases, the step kernels of solver/lbm3d/core.h (LBMKernel, and for the finite-difference
Carreau-Yasuda cases LBMKernelVelocity and LBMKernelStress before it), all compiled
unmodified into oracle/_ref/libnnlbm_ref.so by oracle/Makefile.  The reference ships no tests or fixtures of
its own, so these vectors are what pins the C oracle.  Run in a container that has the
reference checkout:

    make -C oracle all ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from nonnewlbm_b200 import geometry as G  # noqa: E402

SEED = 20261203


def tiny_junction():
    study = G.junction(14, 12, 10, r_ivc=2.5, r_svc=2.0, r_chamber=3.2, r_out=2.0, z_offset=1.0)
    return G.study_to_geometry(study)


def per_cell(rng):
    n = 16
    rho = 1 + 0.03 * rng.standard_normal(n)
    u = 0.05 * rng.standard_normal((n, 3))
    F = 2e-4 * rng.standard_normal((n, 3))
    noise = 1 + 0.03 * rng.standard_normal((n, 27))
    nu = 10 ** rng.uniform(-4, -1, n)
    f_in = np.array([O.ref_feq(O.EQ_DEFAULT, rho[k], *u[k]) for k in range(n)]) * noise
    dv = np.array([O.ref_density_velocity(f_in[k], *F[k]) for k in range(n)])
    col_out = np.zeros((11, n, 27))
    for col in range(11):
        for k in range(n):
            col_out[col, k] = O.ref_collide(col, nu[k], f_in[k], dv[k, 0], dv[k, 1], dv[k, 2], dv[k, 3], *F[k])
    eq_in = np.column_stack([rho, u])
    eq_out = np.zeros((4, n, 27))
    for eq in (O.EQ_INV_CUM_REF, O.EQ_DEFAULT, O.EQ_ENTROPIC):
        for k in range(n):
            eq_out[eq, k] = O.ref_feq(eq, *eq_in[k])
    np.savez_compressed(HERE / "per_cell.npz", f_in=f_in, force=F, nu=nu, dv=dv, col_out=col_out, eq_in=eq_in,
                        eq_out=eq_out)


def lattice_case(name, labels, col, eq, nu, steps, inflow=None, profile=None, force=(0.0, 0.0, 0.0),
                 cy_mode=O.CY_NONE, cy=(0.0, 0.0, 2.0, 1.0)):
    nz, ny, nx = labels.shape
    ref = O.RefLattice(nx, ny, nz, collision=col, equilibrium=eq, nu=nu, force=force, cy_mode=cy_mode, cy=cy)
    ref.set_map(labels)
    if inflow is not None:
        ref.set_inflow(*inflow)
    if profile is not None:
        ref.set_inflow_profile(profile)
    ref.init_equilibrium()
    ref.step(steps)
    # every macro field, numbered as in the C oracle (M_RHO ... M_S33)
    macro = np.stack([ref.get_macro(k) for k in range(20)])
    np.savez_compressed(HERE / f"{name}.npz", labels=labels, df=ref.get_df(), macro=macro,
                        meta=np.array([col, eq, nu, steps, *force]), cy=np.array([cy_mode, *cy], dtype=float),
                        inflow=np.array(inflow if inflow is not None else [0, 0, 1, 1, 1], dtype=float),
                        profile=profile if profile is not None else np.zeros(0))


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libnnlbm_ref.so is not built (needs the reference checkout)")
    rng = np.random.default_rng(SEED)
    per_cell(rng)
    # TCPC junction labels from the oracle's boundary setup (itself checked against the
    # product's host setup in the tests)
    wall = tiny_junction()
    nz, ny, nx = wall.shape
    orc = O.Oracle(nx, ny, nz)
    rc, counts = orc.setup_tcpc(wall)
    assert rc == 0, counts
    labels = orc.get_map()
    np.savez_compressed(HERE / "tcpc_setup.npz", wall=wall, labels=labels, counts=counts)
    inflow = (0.03 * counts[0], 0.02 * counts[1], 1.0, 1.0, 1.0)
    lattice_case("step_tcpc_cum", labels, O.COLLISIONS.index("CUM"), O.EQ_INV_CUM_REF, 0.02, 30, inflow=inflow)
    lattice_case("step_tcpc_kbc_n4", labels, O.COLLISIONS.index("KBC_N4"), O.EQ_INV_CUM_REF, 0.02, 30, inflow=inflow)
    lattice_case("step_tcpc_kbc_c4", labels, O.COLLISIONS.index("KBC_C4"), O.EQ_ENTROPIC, 0.02, 30, inflow=inflow)
    lattice_case("step_tcpc_bgk_force", labels, O.COLLISIONS.index("BGK"), O.EQ_DEFAULT, 0.02, 30, inflow=inflow,
                 force=(1e-5, -2e-5, 5e-6))
    # the finite-difference Carreau-Yasuda coupling of the multi-rank step (core.h:273-800)
    cy = (0.05, 40.0, 2.0, 0.3568)  # nu0, lambda, a, n in lattice units (nu_inf = 0.02)
    lattice_case("step_tcpc_cum_reffd", labels, O.COLLISIONS.index("CUM"), O.EQ_INV_CUM_REF, 0.02, 30, inflow=inflow,
                 cy_mode=O.CY_REF_FD, cy=cy)
    lattice_case("step_tcpc_bgk_reffd", labels, O.COLLISIONS.index("BGK"), O.EQ_DEFAULT, 0.02, 30, inflow=inflow,
                 force=(1e-5, -2e-5, 5e-6), cy_mode=O.CY_REF_FD, cy=cy)
    m, prof = G.pipe_map(16, 9, 9, 3.2)
    lattice_case("step_pipe_mrt", m, O.COLLISIONS.index("MRT_LES"), O.EQ_INV_CUM_REF, 1.0 / 30.0, 30,
                 profile=G.expand_profile(m, prof) * 0.04)
    m, prof = G.dense_box_map(10, 6, 5)
    lattice_case("step_box_cum", m, O.COLLISIONS.index("CUM"), O.EQ_INV_CUM_REF, 0.05 / 3, 30,
                 profile=G.expand_profile(m, prof) * 0.05)
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()

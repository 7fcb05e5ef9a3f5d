"""The FP64 C oracle against the reference's own known answers (tests/golden/, produced by
tests/golden/make_golden.py from the unmodified reference headers) and against physical
invariants.  CPU only."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import geometry as G

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return np.load(GOLD / name, allow_pickle=False)


def test_golden_equilibria():
    g = _load("per_cell.npz")
    for eq in (O.EQ_INV_CUM_REF, O.EQ_DEFAULT, O.EQ_ENTROPIC):
        for k, (rho, ux, uy, uz) in enumerate(g["eq_in"]):
            f = O.feq(eq, rho, ux, uy, uz)
            np.testing.assert_allclose(f, g["eq_out"][eq, k], rtol=2e-15, atol=0)


def test_golden_density_velocity_bit_exact():
    g = _load("per_cell.npz")
    for k in range(len(g["f_in"])):
        np.testing.assert_array_equal(O.density_velocity(g["f_in"][k], *g["force"][k]), g["dv"][k])


@pytest.mark.parametrize("col", range(11), ids=O.COLLISIONS)
def test_golden_collisions(col):
    g = _load("per_cell.npz")
    for k in range(len(g["f_in"])):
        rho, ux, uy, uz = g["dv"][k]
        out = O.collide(col, g["nu"][k], g["f_in"][k], rho, ux, uy, uz, *g["force"][k])
        # CUM, MRT and BGK restate the reference operation order exactly; the KBC moment
        # sums are accumulated in a different order
        tol = 0.0 if O.COLLISIONS[col] in ("CUM", "MRT_LES", "BGK") else 5e-14
        np.testing.assert_allclose(out, g["col_out"][col, k], rtol=tol, atol=0)


def test_golden_tcpc_setup():
    g = _load("tcpc_setup.npz")
    nz, ny, nx = g["wall"].shape
    orc = O.Oracle(nx, ny, nz)
    rc, counts = orc.setup_tcpc(g["wall"])
    assert rc == 0
    np.testing.assert_array_equal(orc.get_map(), g["labels"])
    np.testing.assert_array_equal(counts, g["counts"])


@pytest.mark.parametrize("name", ["step_tcpc_cum", "step_tcpc_kbc_n4", "step_tcpc_kbc_c4", "step_tcpc_bgk_force",
                                  "step_tcpc_cum_reffd", "step_tcpc_bgk_reffd", "step_pipe_mrt", "step_box_cum"])
def test_golden_lattice_steps(name):
    g = _load(name + ".npz")
    col, eq, nu, steps, fx, fy, fz = g["meta"]
    cy_mode, *cy = g["cy"]
    labels = g["labels"]
    nz, ny, nx = labels.shape
    orc = O.Oracle(nx, ny, nz, collision=int(col), equilibrium=int(eq), nu=float(nu), force=(fx, fy, fz),
                   cy_mode=int(cy_mode), cy=tuple(cy))
    orc.set_map(labels)
    orc.set_inflow(*g["inflow"])
    if g["profile"].size:
        orc.set_inflow_profile(g["profile"])
    orc.init_equilibrium()
    orc.step(int(steps))
    df = orc.get_df()
    rel = np.abs(df - g["df"]) / np.abs(g["df"])
    assert rel.max() <= 1e-13, rel.max()
    # macro fields in the oracle's numbering: rho, u, the mean/rms sums and the force (the
    # finite-difference Carreau-Yasuda force of the reffd cases); the strain of the cells
    # whose strain the step reads (FLUID)
    for fo in (O.M_RHO, O.M_VX, O.M_VY, O.M_VZ, O.M_VM_PLUS_X, O.M_VM_MINUS_X, O.M_VM_XX, O.M_VM_ZZ, O.M_FX, O.M_FY,
               O.M_FZ):
        np.testing.assert_allclose(orc.get_macro(fo), g["macro"][fo], rtol=0, atol=1e-14)
    fluid = labels == O.FLUID
    for fo in (O.M_S11, O.M_S12, O.M_S13, O.M_S22, O.M_S32, O.M_S33):
        np.testing.assert_allclose(orc.get_macro(fo)[fluid], g["macro"][fo][fluid], rtol=0, atol=1e-14)
    if int(cy_mode) == O.CY_REF_FD:
        # the coupling was live: the strain force is far from zero
        assert np.max(np.abs(g["macro"][O.M_FX] - fx)) > 1e-4


@pytest.mark.parametrize("col", range(11), ids=O.COLLISIONS)
def test_collision_conserves_mass_and_momentum(col):
    rng = np.random.default_rng(7)
    for _ in range(5):
        f = O.feq(O.EQ_DEFAULT, 1.0, 0.03, -0.02, 0.01) * (1 + 0.02 * rng.standard_normal(27))
        r = O.density_velocity(f)
        g = O.collide(col, 0.02, f, *r)
        r2 = O.density_velocity(g)
        assert abs(r2[0] - r[0]) < 1e-14
        # without forcing the momentum is conserved by every operator
        np.testing.assert_allclose(r2[1:] * r2[0], r[1:] * r[0], atol=1e-14)


@pytest.mark.parametrize("col", ["CUM", "BGK"])
def test_equilibrium_is_fixed_point(col):
    """CUM and BGK leave the (corrected) factorised equilibrium unchanged."""
    f = O.feq(O.EQ_INV_CUM, 1.02, 0.04, 0.01, -0.02)
    r = O.density_velocity(f)
    g = O.collide(O.COLLISIONS.index(col), 1.0 / 30.0, f, *r)
    assert np.max(np.abs(g - f)) < 1e-15


def test_inv_cum_typo_only_touches_pmm():
    a = O.feq(O.EQ_INV_CUM_REF, 1.02, 0.04, 0.01, -0.02)
    b = O.feq(O.EQ_INV_CUM, 1.02, 0.04, 0.01, -0.02)
    d = np.nonzero(a != b)[0]
    assert list(d) == [18]  # pmm
    assert abs(a[18] / b[18] - 1.02) < 1e-15


def test_local_nu_limits():
    f = O.feq(O.EQ_INV_CUM, 1.0, 0.0, 0.0, 0.0)
    nu, S = O.local_nu(f, 1.0, 0.0, 0.0, 0.0, 0.01, 0.16, 1e4, 2.0, 0.3568)
    assert abs(nu - 0.16) < 1e-15 and np.max(np.abs(S)) < 1e-15
    # strong shear: nu tends towards nu_inf and solves the fixed point
    g = f.copy()
    g[O.COLLISIONS.index("CUM") + 21] += 1e-3  # perturb one population
    r = O.density_velocity(g)
    nu, S = O.local_nu(g, *r, 0.01, 0.16, 1e4, 2.0, 0.3568)
    gam = np.sqrt(2.0 * (S[0] ** 2 + S[3] ** 2 + S[5] ** 2 + 2 * (S[1] ** 2 + S[2] ** 2 + S[4] ** 2)))
    nu_cy = 0.01 + (0.16 - 0.01) * (1 + (1e4 * gam) ** 2.0) ** ((0.3568 - 1) / 2.0)
    assert 0.01 < nu < 0.16
    assert abs(nu - nu_cy) / nu < 1e-6


def test_oracle_rest_state_stays_at_rest():
    m, prof = G.pipe_map(12, 8, 8, 2.5)
    orc = O.Oracle(12, 8, 8, collision=0)
    orc.set_map(m)
    orc.set_inflow_profile(np.zeros((3, 8, 8, 12)))
    orc.init_equilibrium()
    orc.step(10)
    assert np.max(np.abs(orc.get_macro(O.M_VX))) < 1e-15

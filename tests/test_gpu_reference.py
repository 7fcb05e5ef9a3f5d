"""The sm_100a step (through the C ABI) against the reference's own step kernels, directly.

The reference side is oracle/_ref/libnnlbm_ref.so: solver/lbm3d/core.h of buresjan/nonnewlbm
compiled unmodified (LBMKernel, and LBMKernelVelocity / LBMKernelStress for the
finite-difference Carreau-Yasuda coupling), driven on one rank by oracle/ref_shim.cpp.  These
tests skip, with that reason, only where the library was not built (no reference checkout
at build time).

Bar: FP64 storage matches the reference to 1e-12 relative per population (populations that
no cell ever reads are excluded, helpers.dead_mask); the mean/rms sums to 1e-12 relative to
their largest magnitude.  Wall treatment: full-way bounce-back wall nodes, the reference's
only wall (solver/lbm3d/lbm_streaming.h:78-107).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import geometry as G

from helpers import dead_mask, max_rel, small_junction

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libnnlbm_ref.so not built: no reference "
                                                                "checkout when oracle/ was built")]

FP64_TOL = 1e-12
CY = (0.05, 40.0, 2.0, 0.3568)  # nu0, lambda, a, n in lattice units (nu_inf = 0.02)


def _pipe_config(steps_plain: int, steps_stats: int):
    """The FP64 pipe configuration as written: 96x32x32, radius 12, cumulant, tau = 0.6,
    parabolic inlet with peak 0.04, rho = 1 outlet, rest initial state."""
    m, prof = G.pipe_map(96, 32, 32, 12.0)
    nz, ny, nx = m.shape
    nu = 1.0 / 30.0  # tau = 3 nu + 1/2 = 0.6
    ref = O.RefLattice(nx, ny, nz, collision=0, equilibrium=O.EQ_INV_CUM_REF, nu=nu)
    ref.set_map(m)
    ref.set_inflow_profile(G.expand_profile(m, prof) * 0.04)
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype="f64", nu=nu))
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.04)
    for L in (ref, lat):
        L.init_equilibrium()
    if steps_plain:
        ref.step(steps_plain, accumulate_stats=False)
        lat.step(steps_plain)
    if steps_stats:
        ref.step(steps_stats, accumulate_stats=True)
        lat.step(steps_stats, stats=True, macro=True)
    return m, ref, lat


def test_pipe_config_100_steps_vs_reference():
    m, ref, lat = _pipe_config(100, 0)
    assert max_rel(lat.export_df(), ref.get_df(), dead_mask(m)) <= FP64_TOL


def test_pipe_config_2000_steps_with_stats_vs_reference():
    """The whole configuration: 2000 steps, mean/rms sums over steps 1001..2000."""
    m, ref, lat = _pipe_config(1000, 1000)
    assert max_rel(lat.export_df(), ref.get_df(), dead_mask(m)) <= FP64_TOL
    st, n = lat.stats()
    assert n == 1000
    fluid = m == G.MAP_FLUID
    ref_sums = [ref.get_macro(O.M_VM_PLUS_X) + ref.get_macro(O.M_VM_MINUS_X), ref.get_macro(O.M_VM_Y),
                ref.get_macro(O.M_VM_Z), ref.get_macro(O.M_VM_XX), ref.get_macro(O.M_VM_YY), ref.get_macro(O.M_VM_ZZ)]
    for k, r in enumerate(ref_sums):
        scale = np.max(np.abs(r[fluid]))
        assert scale > 0 or k in (1, 2, 4, 5)
        err = np.max(np.abs(st[k][fluid] - r[fluid])) / max(scale, 1e-300)
        assert err <= FP64_TOL, (k, err)
    # the developed flow: the centre-line velocity near the outlet is close to the inlet peak
    for fo, fl in ((O.M_RHO, capi.M_RHO), (O.M_VX, capi.M_VX)):
        assert np.max(np.abs(lat.macro(fl)[fluid] - ref.get_macro(fo)[fluid])) <= 1e-13


def _junction_pair(collision, eq=O.EQ_INV_CUM_REF, force=(0.0, 0.0, 0.0), cy_mode=O.CY_NONE, cy=(0.0, 0.0, 2.0, 1.0)):
    wall = small_junction()
    nz, ny, nx = wall.shape
    orc = O.Oracle(nx, ny, nz)
    rc, counts = orc.setup_tcpc(wall)
    assert rc == 0
    labels = orc.get_map()
    del orc
    ref = O.RefLattice(nx, ny, nz, collision=collision, equilibrium=eq, nu=0.02, force=force, cy_mode=cy_mode, cy=cy)
    ref.set_map(labels)
    eqname = {v: k for k, v in capi.EQUILIBRIA.items()}[eq]
    cyname = {0: "none", 1: "ref-fd"}[cy_mode]
    lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype="f64", equilibrium=eqname,
                           cy_mode=cyname, nu=0.02, cy=cy, force=force))
    lat.setup_tcpc(wall)
    for L in (ref, lat):
        L.set_inflow(ivc_flux=0.03 * counts[0], svc_flux=0.02 * counts[1])
        L.init_equilibrium()
    return labels, ref, lat


@pytest.mark.parametrize("collision,eq", [(0, O.EQ_INV_CUM_REF), (10, O.EQ_DEFAULT), (4, O.EQ_INV_CUM_REF)],
                         ids=["CUM", "BGK", "KBC_N4"])
def test_ref_fd_carreau_yasuda_vs_reference(collision, eq):
    """The finite-difference Carreau-Yasuda coupling (velocity, strain and force phases of
    core.h:273-800) against the reference's own three kernels, BGK with a homogeneous force
    on top."""
    force = (1e-5, -2e-5, 5e-6) if collision == 10 else (0.0, 0.0, 0.0)
    labels, ref, lat = _junction_pair(collision, eq=eq, force=force, cy_mode=O.CY_REF_FD, cy=CY)
    ref.step(100)
    lat.step(100, macro=True)
    assert max_rel(lat.export_df(), ref.get_df(), dead_mask(labels)) <= FP64_TOL
    fluid = labels == G.MAP_FLUID
    fx = ref.get_macro(O.M_FX)[fluid]
    assert np.max(np.abs(fx - force[0])) > 1e-4  # the strain force was live
    assert np.max(np.abs(lat.macro(capi.M_FX)[fluid] - fx)) <= 1e-12 * np.max(np.abs(fx))


@pytest.mark.parametrize("collision,eq", [(10, O.EQ_DEFAULT), (4, O.EQ_INV_CUM_REF), (8, O.EQ_ENTROPIC),
                                          (0, O.EQ_INV_CUM_REF)], ids=["BGK", "KBC_N4", "KBC_C4", "CUM"])
def test_homogeneous_force_vs_reference(collision, eq):
    """A non-zero homogeneous body force (the forcing source of lbm_col_bgk.h:57-83 and the KBC
    forms, the F/2 velocity shift of lbm_common.h:36-38)."""
    force = (2e-5, -1e-5, 3e-6)
    labels, ref, lat = _junction_pair(collision, eq=eq, force=force)
    ref.step(100)
    lat.step(100, macro=True)
    assert max_rel(lat.export_df(), ref.get_df(), dead_mask(labels)) <= FP64_TOL
    fluid = labels == G.MAP_FLUID
    assert np.max(np.abs(lat.macro(capi.M_VZ)[fluid] - ref.get_macro(O.M_VZ)[fluid])) <= 1e-13


@pytest.mark.parametrize("collision", [0, 4, 9, 10], ids=["CUM", "KBC_N4", "MRT_LES", "BGK"])
def test_tcpc_junction_vs_reference(collision):
    labels, ref, lat = _junction_pair(collision)
    ref.step(100)
    lat.step(100)
    assert max_rel(lat.export_df(), ref.get_df(), dead_mask(labels)) <= FP64_TOL

"""Parity of the sm_100a step (through the C ABI) against the FP64 C oracle.

Bars: FP64 storage matches the oracle to 1e-12 relative per population after 100 steps
(dead populations excluded, see helpers.dead_mask); FP32/FP16/BF16 storage are checked
against the FP64 oracle with the tolerances written in each test.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import geometry as G

from helpers import dead_mask, max_rel, small_junction

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _tcpc_pair(collision: int, dtype="f64", eq=O.EQ_INV_CUM_REF, nu=0.02, cy_mode=O.CY_NONE, cy=(0.0, 0.0, 2.0, 1.0),
               ivc=0.03, svc=0.02):
    wall = small_junction()
    nz, ny, nx = wall.shape
    orc = O.Oracle(nx, ny, nz, collision=collision, equilibrium=eq, nu=nu, cy_mode=cy_mode, cy=cy)
    rc, counts = orc.setup_tcpc(wall)
    assert rc == 0
    eqname = {v: k for k, v in capi.EQUILIBRIA.items()}[eq]
    cyname = {0: "none", 1: "ref-fd", 2: "local-neq"}[cy_mode]
    lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype=dtype, equilibrium=eqname,
                           cy_mode=cyname, nu=nu, cy=cy))
    c2 = lat.setup_tcpc(wall)
    assert c2["left_area"] == counts[0] and c2["outlet6"] == counts[3]
    for L in (orc, lat):
        L.set_inflow(ivc_flux=ivc * counts[0], svc_flux=svc * counts[1])
        L.init_equilibrium()
    return orc, lat


@pytest.mark.parametrize("collision", range(11), ids=O.COLLISIONS)
def test_fp64_tcpc_100_steps(collision):
    orc, lat = _tcpc_pair(collision)
    orc.step(100)
    lat.step(100, macro=True)
    labels = orc.get_map()
    a, b = lat.export_df(), orc.get_df()
    assert max_rel(a, b, dead_mask(labels)) <= FP64_TOL
    for fo, fl in ((O.M_RHO, capi.M_RHO), (O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        assert np.max(np.abs(lat.macro(fl) - orc.get_macro(fo))) <= 1e-13


def test_fp64_odd_step_count_and_layout():
    """Odd and even step counts leave the two A-A layouts; both must export the same state."""
    orc, lat = _tcpc_pair(O.COLLISIONS.index("CUM"))
    labels = orc.get_map()
    dead = dead_mask(labels)
    for n in (1, 2, 3, 7):
        orc.step(n)
        lat.step(n)
        assert max_rel(lat.export_df(), orc.get_df(), dead) <= FP64_TOL, n


def test_fp64_import_export_roundtrip():
    orc, lat = _tcpc_pair(0)
    orc.step(5)
    df = orc.get_df()
    lat.import_df(df)
    dead = dead_mask(orc.get_map())
    assert max_rel(lat.export_df(), df, dead) == 0.0
    orc.step(10)
    lat.step(10)
    assert max_rel(lat.export_df(), orc.get_df(), dead) <= FP64_TOL


@pytest.mark.parametrize("eq", [O.EQ_INV_CUM, O.EQ_DEFAULT, O.EQ_ENTROPIC])
def test_fp64_equilibria(eq):
    orc, lat = _tcpc_pair(0, eq=eq)
    orc.step(40)
    lat.step(40)
    assert max_rel(lat.export_df(), orc.get_df(), dead_mask(orc.get_map())) <= FP64_TOL


def test_fp64_pipe_generic_bcs():
    m, prof = G.pipe_map(24, 12, 12, 4.5)
    nz, ny, nx = m.shape
    orc = O.Oracle(nx, ny, nz, collision=0, nu=1.0 / 30.0)
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype="f64", nu=1.0 / 30.0))
    orc.set_map(m)
    orc.set_inflow_profile(G.expand_profile(m, prof) * 0.04)
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.04)
    for L in (orc, lat):
        L.init_equilibrium()
    orc.step(100)
    lat.step(100)
    assert max_rel(lat.export_df(), orc.get_df(), dead_mask(m)) <= FP64_TOL


@pytest.mark.parametrize("collision", [0, 9, 10])
def test_fp64_periodic_box(collision):
    m, prof = G.dense_box_map(16, 10, 8)
    nz, ny, nx = m.shape
    orc = O.Oracle(nx, ny, nz, collision=collision, nu=0.05 / 3)
    lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype="f64", nu=0.05 / 3))
    orc.set_map(m)
    orc.set_inflow_profile(G.expand_profile(m, prof) * 0.05)
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.05)
    for L in (orc, lat):
        L.init_equilibrium()
    orc.step(100)
    lat.step(100)
    assert max_rel(lat.export_df(), orc.get_df()) <= FP64_TOL


CY = (0.05, 40.0, 2.0, 0.3568)  # nu0, lambda, a, n in lattice units (nu_inf = 0.02)


def test_fp64_cy_local_neq():
    orc, lat = _tcpc_pair(0, cy_mode=O.CY_LOCAL_NEQ, cy=CY)
    orc.step(100)
    lat.step(100, macro=True)
    assert max_rel(lat.export_df(), orc.get_df(), dead_mask(orc.get_map())) <= FP64_TOL
    fluid = orc.get_map() == G.MAP_FLUID
    s_o = orc.get_macro(O.M_S12)[fluid]
    s_l = lat.macro(capi.M_S12)[fluid]
    assert np.max(np.abs(s_o - s_l)) <= 1e-12 * max(1.0, np.max(np.abs(s_o)))


def test_fp64_cy_ref_fd():
    orc, lat = _tcpc_pair(0, cy_mode=O.CY_REF_FD, cy=CY)
    orc.step(100)
    lat.step(100, macro=True)
    assert max_rel(lat.export_df(), orc.get_df(), dead_mask(orc.get_map())) <= FP64_TOL
    # the force field is non-zero, so the three-phase path was exercised
    assert np.max(np.abs(orc.get_macro(O.M_FX))) > 0


def test_fp64_stats_and_reduce():
    orc, lat = _tcpc_pair(0)
    orc.step(30, accumulate_stats=False)
    lat.step(30)
    orc.step(20, accumulate_stats=True)
    lat.step(20, stats=True, macro=True, reduce=True)
    st, n = lat.stats()
    assert n == 20
    jx = orc.get_macro(O.M_VM_PLUS_X) + orc.get_macro(O.M_VM_MINUS_X)
    assert np.max(np.abs(st[0] - jx)) <= 1e-12
    assert np.max(np.abs(st[4] - orc.get_macro(O.M_VM_YY))) <= 1e-14
    r_l, r_o = lat.reduce(), orc.reduce()
    assert abs(r_l[0] - r_o[0]) <= 1e-9
    assert np.max(np.abs(r_l[1:] - r_o[1:])) <= 1e-12


@pytest.mark.parametrize("dtype,tol_u", [("f32", 2e-5), ("f16", 2e-3), ("bf16", 2e-2)])
def test_reduced_precision_vs_fp64_oracle(dtype, tol_u):
    """Velocity of FP32 / FP16 / BF16 storage against the FP64 oracle after 200 steps,
    relative to the peak velocity."""
    orc, lat = _tcpc_pair(0, dtype=dtype)
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= tol_u, (dtype, err)


@pytest.mark.parametrize("collision", [9, 10, 4, 5], ids=["MRT_LES", "BGK", "KBC_N4", "KBC_C1"])
def test_fp32_collisions_vs_fp64_oracle(collision):
    """FP32 storage and arithmetic of the other collisions against the FP64 oracle after 200
    steps (MRT and BGK run two cells per thread on the packed FP32 pipe, KBC one), relative to
    the peak velocity."""
    orc, lat = _tcpc_pair(collision, dtype="f32")
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= 2e-5, (O.COLLISIONS[collision], err)


@pytest.mark.parametrize("cells", [1, 2])
@pytest.mark.parametrize("collision,dtype,tol_u", [(0, "f32", 2e-5), (9, "f32", 2e-5), (10, "f32", 2e-5), (0, "f16", 2e-3)],
                         ids=["CUM-f32", "MRT_LES-f32", "BGK-f32", "CUM-f16"])
def test_both_launch_forms_vs_fp64_oracle(collision, dtype, tol_u, cells):
    """The one-cell (64 registers) and the paired (two cells a thread) form of a collision that
    pairs, each against the FP64 oracle after 200 steps, relative to the peak velocity."""
    orc, lat = _tcpc_pair(collision, dtype=dtype)
    lat.set_launch(128, cells)
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= tol_u, (O.COLLISIONS[collision], dtype, cells, err)


def test_set_launch_rejects_bad_shapes():
    orc, lat = _tcpc_pair(0, dtype="f32")
    for block, cells in ((96, 1), (256, 3)):
        with pytest.raises(capi.NnlbmError):
            lat.set_launch(block, cells)


@pytest.mark.parametrize("dtype,tol_u", [("f32", 5e-5), ("f16", 2e-3)])
def test_reduced_precision_cy_local_neq(dtype, tol_u):
    """The cumulant with the local Carreau-Yasuda viscosity (solved two cells at a time in
    packed single precision) against the FP64 oracle after 200 steps, relative to the peak
    velocity; the viscosity field itself within 1e-3 of its largest value."""
    orc, lat = _tcpc_pair(0, dtype=dtype, cy_mode=O.CY_LOCAL_NEQ, cy=CY)
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= tol_u, (dtype, err)
    s_o, s_l = orc.get_macro(O.M_S12)[fluid], lat.macro(capi.M_S12)[fluid]
    assert np.max(np.abs(s_l - s_o)) <= 1e-3 * np.max(np.abs(s_o)), dtype


def test_autotune_keeps_state():
    orc, lat = _tcpc_pair(0)
    orc.step(4)
    lat.step(4)
    lat.autotune()
    orc.step(6)
    lat.step(6)
    assert max_rel(lat.export_df(), orc.get_df(), dead_mask(orc.get_map())) <= FP64_TOL


def test_autotune_with_stats_restores_state():
    """Tuning with the accumulators on (which may switch an FP32 cumulant between one and two
    cells a thread) leaves populations, mean/rms sums and their step count as they were."""
    orc, lat = _tcpc_pair(0, dtype="f32", cy_mode=O.CY_LOCAL_NEQ, cy=CY)
    lat.step(10, stats=True)
    df0, (st0, n0) = lat.export_df(), lat.stats()
    lat.autotune(stats=True)
    st1, n1 = lat.stats()
    assert np.array_equal(lat.export_df(), df0) and np.array_equal(st1, st0) and n1 == n0 == 10
    # the tuned form steps on correctly
    lat.step(10, stats=True, macro=True)
    assert lat.stats()[1] == 20
    orc.step(20)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    err = np.max(np.abs(lat.macro(capi.M_VX)[fluid] - orc.get_macro(O.M_VX)[fluid])) / umax
    assert err <= 5e-5, err


def test_batched_cases_match_single():
    wall = small_junction()
    nz, ny, nx = wall.shape
    specs = [CaseSpec((nx, ny, nz), dtype="f64", nu=nu) for nu in (0.02, 0.05)]
    lat = Lattice(specs)
    singles = [Lattice(s) for s in specs]
    for k in range(2):
        lat.setup_tcpc(wall, ic=k)
        singles[k].setup_tcpc(wall)
        for L, ic in ((lat, k), (singles[k], 0)):
            L.set_inflow(ivc_flux=5.0, svc_flux=3.0, ic=ic)
    lat.init_equilibrium()
    for s in singles:
        s.init_equilibrium()
        s.step(25)
    lat.step(25)
    for k in range(2):
        assert np.array_equal(lat.export_df(k), singles[k].export_df())


@pytest.mark.parametrize("collision", [0, 4])
def test_fp64_open_box_plane_corners(collision):
    """A geometry without walls: every open plane reaches the domain edges, so plane
    corners are gathered, and one fluid cell finishes two open-plane neighbours."""
    wall = np.zeros((10, 12, 14), dtype=np.int32)
    nz, ny, nx = wall.shape
    orc = O.Oracle(nx, ny, nz, collision=collision, nu=0.05)
    rc, counts = orc.setup_tcpc(wall)
    lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype="f64", nu=0.05))
    lat.setup_tcpc(wall)
    for L in (orc, lat):
        L.set_inflow(ivc_flux=0.02 * counts[0], svc_flux=0.01 * counts[1])
        L.init_equilibrium()
    for n in (1, 10, 49):
        orc.step(n)
        lat.step(n, macro=True, reduce=True, stats=True)
        assert max_rel(lat.export_df(), orc.get_df(), dead_mask(orc.get_map())) <= FP64_TOL
    r_l, r_o = lat.reduce(), orc.reduce()
    assert np.max(np.abs(r_l[1:] - r_o[1:])) <= 1e-12


def test_batched_mixed_groups_and_sizes():
    """Cases of different sizes and collisions in one context: same results as alone."""
    w1 = small_junction()
    w2 = G.study_to_geometry(G.junction(32, 24, 20, r_ivc=5, r_svc=4, r_chamber=6, r_out=3.5, z_offset=2))
    specs = [CaseSpec(w1.shape[::-1], dtype="f32", collision="CUM", nu=0.02),
             CaseSpec(w2.shape[::-1], dtype="f32", collision="CUM", nu=0.03),
             CaseSpec(w2.shape[::-1], dtype="f32", collision="BGK", nu=0.03)]
    walls = [w1, w2, w2]
    lat = Lattice(specs)
    singles = [Lattice(s) for s in specs]
    for k in range(3):
        for L, ic in ((lat, k), (singles[k], 0)):
            c = L.setup_tcpc(walls[k], ic=ic)
            L.set_inflow(ivc_flux=0.03 * c["left_area"], svc_flux=0.02 * c["right_area"], ic=ic)
    lat.init_equilibrium()
    for s in singles:
        s.init_equilibrium()
        s.step(31, stats=True)
    lat.step(31, stats=True)
    for k in range(3):
        assert np.array_equal(lat.export_df(k), singles[k].export_df())
        assert np.array_equal(lat.stats(k)[0], singles[k].stats()[0])


def test_reduce_sums_after_sync_async_and_plain_steps():
    """The FP64 sums (striped over 32 addresses, added on the host) come back the same after a
    synchronous step, after an asynchronous step and nnlbm_sync, and stay those of the last
    reducing step across steps that do not reduce."""
    lats = [_tcpc_pair(0)[1] for _ in range(2)]
    lats[0].step(6, reduce=True)
    r_sync = lats[0].reduce()
    lats[1].step(6, reduce=True, wait=False)
    lats[1].sync()
    r_async = lats[1].reduce()
    # FP64 atomic sums: the order of the additions may differ between runs
    assert np.all(np.abs(r_sync - r_async) <= 1e-12 * np.maximum(1.0, np.abs(r_sync)))
    lats[0].step(3)
    assert np.array_equal(lats[0].reduce(), r_sync)
    assert r_sync[0] > 0 and np.all(np.isfinite(r_sync))


def test_async_steps_and_control_rows_match_sync():
    """Steps enqueued without waiting (NNLBM_STEP_ASYNC, then nnlbm_sync) and one-step calls
    whose unchanged control rows are not sent again give the same lattice as synchronous
    multi-step calls; a changed inflow between calls takes effect."""
    wall = small_junction()
    nz, ny, nx = wall.shape
    lats = [Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype="f64", nu=0.02)) for _ in range(2)]
    for L in lats:
        c = L.setup_tcpc(wall)
        L.set_inflow(ivc_flux=0.03 * c["left_area"], svc_flux=0.02 * c["right_area"])
        L.init_equilibrium()
    a, b = lats
    a.step(6, stats=True)
    for _ in range(6):
        b.step(1, stats=True, wait=False)
    b.sync()
    for L in lats:
        L.set_inflow(ivc_flux=40.0, svc_flux=10.0)
    a.step(5)
    for _ in range(5):
        b.step(1, wait=False)
    b.sync()
    assert np.array_equal(a.export_df(), b.export_df())
    assert np.array_equal(a.stats()[0], b.stats()[0])


@pytest.mark.parametrize("dtype,tol_u", [("f32", 5e-5), ("f16", 2e-3), ("bf16", 2e-2)])
def test_reduced_precision_kbc_n4_cy_local_neq(dtype, tol_u):
    """KBC_N4 with the local Carreau-Yasuda viscosity, the collision of the storage-precision
    study, in FP32 / FP16 / BF16 storage against the FP64 oracle after 200 steps, relative to
    the peak velocity."""
    orc, lat = _tcpc_pair(O.COLLISIONS.index("KBC_N4"), dtype=dtype, cy_mode=O.CY_LOCAL_NEQ, cy=CY)
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= tol_u, (dtype, err)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_watchdog_reports_density_out_of_range_and_recovers(dtype):
    """The device watchdog (density outside (0.25, 4) or not finite) turns into
    NNLBM_ERR_NAN with its message; importing a sound state clears it and the case steps on.
    The bad state is made on the host: nothing on the device faults."""
    orc, lat = _tcpc_pair(0, dtype=dtype)
    orc.step(3)
    good = orc.get_df()
    labels = orc.get_map()
    bad = good.copy()
    # a fluid cell whose 26 neighbours are fluid too: the next step pulls its populations from
    # them, so all 27 cells are scaled to give it density 5
    fl = labels == G.MAP_FLUID
    inner = fl.copy()
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                inner &= np.roll(fl, (dz, dy, dx), axis=(0, 1, 2))
    z, y, x = [int(v[len(v) // 2]) for v in np.nonzero(inner)]
    bad[:, z - 1:z + 2, y - 1:y + 2, x - 1:x + 2] *= 5.0
    lat.import_df(bad)
    with pytest.raises(capi.NnlbmError) as e:
        lat.step(1)
    assert e.value.code == capi.ERR_NAN
    assert "density" in str(e.value)
    # asynchronous steps report it at the next sync
    lat.import_df(bad)
    lat.step(1, wait=False)
    with pytest.raises(capi.NnlbmError) as e:
        lat.sync()
    assert e.value.code == capi.ERR_NAN
    # a sound state clears the flag; the case then matches the oracle again
    lat.import_df(good)
    lat.step(5)
    orc.step(5)
    tol = FP64_TOL if dtype == "f64" else 1e-5
    fluid = labels == G.MAP_FLUID
    assert max_rel(lat.export_df()[:, fluid], orc.get_df()[:, fluid]) <= tol


# -- halfway bounce-back (no reference counterpart; against the oracle's halfway mode) ----------
def _halfway_pair(collision=0, dtype="f64", geometry="pipe", cy_mode=O.CY_NONE, cy=(0.0, 0.0, 2.0, 1.0), eq=O.EQ_INV_CUM_REF):
    cyname = {0: "none", 1: "ref-fd", 2: "local-neq"}[cy_mode]
    eqname = {v: k for k, v in capi.EQUILIBRIA.items()}[eq]
    if geometry == "pipe":
        m, prof = G.pipe_map(96, 32, 32, 12.0)
        nz, ny, nx = m.shape
        nu = 1.0 / 30.0
        orc = O.Oracle(nx, ny, nz, collision=collision, equilibrium=eq, nu=nu, cy_mode=cy_mode, cy=cy, halfway=True)
        orc.set_map(m)
        orc.set_inflow_profile(G.expand_profile(m, prof) * 0.04)
        lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype=dtype, equilibrium=eqname,
                               cy_mode=cyname, nu=nu, cy=cy, bounce_back="halfway"))
        lat.set_map(m)
        lat.set_inflow_profile(prof * 0.04)
    else:
        wall = small_junction()
        nz, ny, nx = wall.shape
        orc = O.Oracle(nx, ny, nz, collision=collision, equilibrium=eq, nu=0.02, cy_mode=cy_mode, cy=cy, halfway=True)
        rc, counts = orc.setup_tcpc(wall)
        lat = Lattice(CaseSpec((nx, ny, nz), collision=O.COLLISIONS[collision], dtype=dtype, equilibrium=eqname,
                               cy_mode=cyname, nu=0.02, cy=cy, bounce_back="halfway"))
        lat.setup_tcpc(wall)
        for L in (orc, lat):
            L.set_inflow(ivc_flux=0.03 * counts[0], svc_flux=0.02 * counts[1])
    return orc, lat


def _live(labels):
    """[27][z][y][x] True at the populations of every cell but the walls (with halfway
    bounce-back nothing reads a wall cell's populations)."""
    return np.broadcast_to(labels != G.MAP_WALL, (27,) + labels.shape)


def test_fp64_halfway_pipe_configuration():
    """The pipe configuration with the halfway bounce-back it names: both A-A layouts, then
    100 steps."""
    orc, lat = _halfway_pair()
    for L in (orc, lat):
        L.init_equilibrium()
    live = _live(orc.get_map())
    for n in (1, 2, 3, 94):
        orc.step(n)
        lat.step(n)
        assert max_rel(lat.export_df()[live], orc.get_df()[live]) <= FP64_TOL, n


@pytest.mark.parametrize("collision,eq", [(0, O.EQ_INV_CUM_REF), (10, O.EQ_DEFAULT), (4, O.EQ_INV_CUM_REF)],
                         ids=["CUM", "BGK", "KBC_N4"])
def test_fp64_halfway_junction(collision, eq):
    """The TCPC junction: open-plane nodes finished by their inward neighbour and walls next to
    the planes."""
    orc, lat = _halfway_pair(collision, geometry="junction", eq=eq)
    for L in (orc, lat):
        L.init_equilibrium()
    orc.step(100)
    lat.step(100, macro=True)
    live = _live(orc.get_map())
    assert max_rel(lat.export_df()[live], orc.get_df()[live]) <= FP64_TOL


def test_fp64_halfway_ref_fd_and_gathered_nodes():
    """The finite-difference Carreau-Yasuda coupling: every open-plane node gathered by its own
    kernel, and the velocity phase pulls next to walls."""
    orc, lat = _halfway_pair(0, geometry="junction", cy_mode=O.CY_REF_FD, cy=CY)
    for L in (orc, lat):
        L.init_equilibrium()
    orc.step(60)
    lat.step(60, macro=True)
    live = _live(orc.get_map())
    assert max_rel(lat.export_df()[live], orc.get_df()[live]) <= FP64_TOL


def test_fp64_halfway_moving_initial_state_and_import():
    orc, lat = _halfway_pair()
    for L in (orc, lat):
        L.init_equilibrium(1.0, 0.01, 0.004, -0.003)
    live = _live(orc.get_map())
    orc.step(7)
    lat.step(7)
    assert max_rel(lat.export_df()[live], orc.get_df()[live]) <= FP64_TOL
    lat.import_df(orc.get_df())
    assert max_rel(lat.export_df()[live], orc.get_df()[live]) == 0.0
    orc.step(9)
    lat.step(9)
    assert max_rel(lat.export_df()[live], orc.get_df()[live]) <= FP64_TOL


def test_fp32_halfway_pipe_vs_fp64_oracle():
    """FP32 storage with halfway walls against the FP64 oracle after 200 steps: velocity within
    5e-5 of the peak (the pipe's inlet peak is 0.04)."""
    orc, lat = _halfway_pair(dtype="f32")
    for L in (orc, lat):
        L.init_equilibrium()
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= 5e-5, err


def _adjacent_box(nx, dtype, cells_per_thread):
    m, prof = G.dense_box_map(nx, 6, 5)
    nz, ny, _ = m.shape
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype=dtype, nu=0.05 / 3))
    lat.set_launch(128, cells_per_thread)
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.05)
    lat.init_equilibrium()
    return m, lat


@pytest.mark.parametrize("nx", [130, 131])
def test_adjacent_spans_match_one_cell_form(nx):
    """The paired form, whose full 64-cell spans collide as x-adjacent pairs (one 8-byte access
    moves a population of two cells; with nx = 131 some odd-step accesses begin at odd elements
    and are put together across lanes), against the one-cell form after 1, 2 and 5 FP32 steps:
    the two differ only in rounding (packed against scalar arithmetic), 1e-5 relative per
    population; a misplaced element would differ by the populations' spread."""
    m, paired = _adjacent_box(nx, "f32", 2)
    _, single = _adjacent_box(nx, "f32", 1)
    live = np.broadcast_to(m != G.MAP_INFLOW_EQ, (27,) + m.shape)
    for n in (1, 1, 3):
        paired.step(n)
        single.step(n)
        assert max_rel(paired.export_df()[live], single.export_df()[live]) <= 1e-5, n


@pytest.mark.parametrize("nx", [130, 131])
@pytest.mark.parametrize("dtype,tol_u", [("f32", 5e-5), ("f16", 5e-3), ("bf16", 2e-2)])
def test_adjacent_spans_vs_fp64_oracle(nx, dtype, tol_u):
    """Full 64-cell spans of a periodic box collide as x-adjacent pairs (one 4- or 8-byte access
    moves a population of two cells).  With nx = 131 the rows start at alternating element
    parity, so the odd step's shifted accesses of some directions begin at odd elements and
    are put together across lanes.  Velocity against the FP64 oracle after 200 steps,
    relative to the peak velocity 0.05 (tau = 0.55, the least viscous flow of these tests)."""
    m, prof = G.dense_box_map(nx, 6, 5)
    nz, ny, _ = m.shape
    orc = O.Oracle(nx, ny, nz, collision=0, nu=0.05 / 3)
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype=dtype, nu=0.05 / 3))
    lat.set_launch(128, 2)
    orc.set_map(m)
    orc.set_inflow_profile(G.expand_profile(m, prof) * 0.05)
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.05)
    for L in (orc, lat):
        L.init_equilibrium()
    for n in (1, 199):
        orc.step(n)
        lat.step(n, macro=True)
    inner = m != G.MAP_INFLOW_EQ
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[inner]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[inner] - orc.get_macro(fo)[inner])) / umax
        assert err <= tol_u, (fo, err)

"""Checkpoint and resume through the C ABI: a run saved after n1 steps and resumed in a new
context for n2 steps ends where an uninterrupted run of n1 + n2 steps ends."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import checkpoint as C

from helpers import dead_mask, max_rel, small_junction

pytestmark = pytest.mark.gpu

CY = (0.05, 40.0, 2.0, 0.3568)


def _lattice(wall, dtype, cy_mode):
    nz, ny, nx = wall.shape
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype=dtype, cy_mode=cy_mode, nu=0.02, cy=CY))
    counts = lat.setup_tcpc(wall)
    lat.set_inflow(ivc_flux=0.03 * counts["left_area"], svc_flux=0.02 * counts["right_area"])
    return lat


def _labels(wall):
    orc = O.Oracle(*wall.shape[::-1])
    orc.setup_tcpc(wall)
    return orc.get_map()


@pytest.mark.parametrize("dtype,cy_mode", [("f64", "none"), ("f64", "ref-fd"), ("f32", "local-neq")])
def test_resume_matches_uninterrupted(tmp_path, dtype, cy_mode):
    wall = small_junction()
    labels = _labels(wall)
    n1, n2 = 12, 17
    ref = _lattice(wall, dtype, cy_mode)
    ref.init_equilibrium()
    ref.step(n1 + n2, stats=True, macro=True)

    first = _lattice(wall, dtype, cy_mode)
    first.init_equilibrium()
    first.step(n1, stats=True, macro=True)
    C.save_state(tmp_path, first, n1, 1.0, {C.VTK3D: (2, 0.1)}, labels)
    first.close()

    resumed = _lattice(wall, dtype, cy_mode)
    cfg = C.load_state(tmp_path, resumed, labels=labels)
    assert cfg["iterations"] == n1 and cfg["stats_count"] == n1
    resumed.step(n2, stats=True, macro=True)

    dead = dead_mask(labels)
    a, b = resumed.export_df(), ref.export_df()
    (sa, na), (sb, nb) = resumed.stats(), ref.stats()
    assert na == nb == n1 + n2
    if dtype == "f64":
        # the same values in either A-A layout step to the same bits
        assert max_rel(a, b, dead) == 0.0
        assert np.array_equal(sa, sb)
        assert np.array_equal(resumed.macro(capi.M_VX), ref.macro(capi.M_VX))
    else:
        # FP32 storage: the canonical FP64 file rounds each population once on reload
        assert max_rel(a, b, dead) <= 1e-5
        assert np.max(np.abs(sa - sb)) <= 1e-5 * max(1.0, np.max(np.abs(sb)))


def test_driver_wall_time_then_resume(tmp_path):
    """sim_tcpc's loop (core.h:1578-1602) through the driver: the wall time is reached after the
    first call, the state is saved and `loadstate` left behind; the next start resumes from
    that iteration and runs to the final time."""
    from nonnewlbm_b200 import tcpc, units, vtk

    dx = 2.5e-4
    wall = small_junction()
    geo = tmp_path / "geometry.vtk"
    vtk.write_geometry(geo, wall, dx)
    dt = units.lattice_units(units.material_by_name("newtonian"), dx, 1e-4)["dt"]
    final = 250.5 * dt
    base = ["--geometry", str(geo), "--material", "newtonian", "--ivc-mls", "0.02", "--svc-mls", "0.012",
            "--case-id", "ck", "--final-time", repr(final), "--vtk-period", "1e9", "--print-period", "1e9",
            "--results-root", str(tmp_path)]
    results = tmp_path / "results_ck"
    assert tcpc.main(base + ["--wall-time", "1e-9"]) == 0
    assert C.flag_exists(results, "loadstate")
    saved = C.read_config(results)["iterations"]
    assert 0 < saved <= 100
    assert tcpc.main(base) == 0
    log = (results / "log_rank000").read_text()
    assert "maximum wall time reached" in log and "[loadState invoked]" in log
    assert log.rstrip().endswith("physFinalTime reached")

"""Host-side checks that need no GPU: the C ABI library loads and exports what
include/nnlbm.h declares, the host boundary setup matches the oracle, configuration and
unit conversions, and error paths."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import CaseSpec, Lattice, capi, units
from nonnewlbm_b200 import geometry as G

from helpers import small_junction

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "nnlbm.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void\s*\*|void)\s+(nnlbm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(capi.EXPORTED) <= set(names)


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.NnlbmError) as e:
        Lattice(CaseSpec((8, 8, 8)))
    assert e.value.code == capi.ERR_CUDA


@pytest.mark.parametrize("scale", [None, 0.125])
def test_host_tcpc_setup_matches_oracle(scale):
    wall = small_junction() if scale is None else G.study_to_geometry(G.junction(scale=scale))
    nz, ny, nx = wall.shape
    m, counts, rc = capi.tcpc_labels(wall)
    orc = O.Oracle(nx, ny, nz)
    orc_rc, orc_counts = orc.setup_tcpc(wall)
    np.testing.assert_array_equal(m, orc.get_map())
    assert list(counts.values()) == list(orc_counts)
    assert (rc == capi.OK) == (orc_rc == 0)


def test_host_tcpc_setup_zero_area():
    wall = np.ones((10, 12, 14), dtype=np.int32)  # all wall: no inlet can open
    m, counts, rc = capi.tcpc_labels(wall)
    assert rc == capi.ERR_AREA
    assert counts["left_area"] == 0
    assert np.all(m == G.MAP_WALL)


def test_tcpc_plane_opening_carves_through_walls():
    # a tube that starts two cells inside x = 0: the setup opens the inflow plane and the
    # wall layer in front of it where the first open plane is open
    wall = np.ones((12, 12, 16), dtype=np.int32)
    wall[3:9, 3:9, 3:13] = 0
    wall[5:7, 0:3, 6:9] = 0
    wall[5:7, 9:12, 6:9] = 0
    m, counts, rc = capi.tcpc_labels(wall)
    assert rc == capi.OK
    assert counts["left_area"] == 36 and counts["right_area"] == 36
    assert np.all(m[3:9, 3:9, 0] == G.MAP_INFLOW_LEFT)
    assert np.all(m[3:9, 3:9, 1:3] == G.MAP_FLUID)


def test_study_label_translation():
    s = np.array([[[1, 2, 3, 4, 5, 6]]], dtype=np.uint8)
    np.testing.assert_array_equal(G.study_to_geometry(s), [[[0, 1, 3, 4, 5, 6]]])
    with pytest.raises(ValueError):
        G.study_to_geometry(np.array([[[0]]]))


def test_materials_and_units():
    gx = units.material_by_name("gx")
    assert gx.density == 1088.0 and gx.carreau_yasuda
    with pytest.raises(ValueError):
        units.material_by_name("water")
    dx = 0.25e-3
    conv = units.lattice_units(gx, dx, 1e-4)
    # sim_tcpc.cu:800-806
    dt = 1e-4 / gx.nu_inf * dx * dx
    assert conv["dt"] == pytest.approx(dt, rel=1e-15)
    assert conv["nu0"] == pytest.approx(gx.mu0 / gx.density / dx / dx * dt, rel=1e-15)
    assert conv["lambda"] == pytest.approx(gx.lam / dt, rel=1e-15)
    nw = units.lattice_units(units.material_by_name("newtonian"), dx, 1e-4)
    assert nw["nu0"] == 1e-4 and nw["a"] == 2.0 and nw["n"] == 1.0
    assert units.flux_lbm(8.0, dx, dt) == pytest.approx(8.0e-6 / dx ** 3 * dt, rel=1e-15)


def test_pipe_and_box_maps():
    m, prof = G.pipe_map(96, 32, 32, 12.0)
    n_in = int((m == G.MAP_INFLOW_EQ).sum())
    assert prof.shape == (n_in, 3) and n_in == int((m == G.MAP_OUTFLOW_RIGHT_EQ).sum())
    assert prof[:, 0].max() <= 1.0 and prof[:, 0].min() >= 0.0
    b, bp = G.dense_box_map(8, 6, 5)
    assert (b == G.MAP_PERIODIC).sum() == 6 * 6 * 5
    assert bp.shape == (30, 3)

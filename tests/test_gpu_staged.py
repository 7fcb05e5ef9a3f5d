"""The staged two-cell step form (persistent warps that bring each pair of chunks into shared
memory with bulk copies while the pair before collides) against the plain two-cell form,
which computes the same packed arithmetic from the same values.  Pairs must come out bitwise
equal.  Chunks that do not pair (faces, walls next to halfway bounce-back, the
finite-difference force) are stepped one cell a thread by both kernels; the compiler may
contract their scalar products and sums differently in the two kernels, so FP32 populations
are compared to 1e-5 relative (a few rounding steps after 21 steps; a misplaced population
differs by the populations' spread), macro fields and sums also to 1e-7 absolute.  The plain form itself is checked against the FP64
oracle in test_gpu_parity.py; one test here checks the staged form against the oracle
directly.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import geometry as G

from helpers import small_junction

pytestmark = pytest.mark.gpu

CY = (0.05, 40.0, 2.0, 0.3568)  # nu0, lambda, a, n in lattice units (nu_inf = 0.02)


def _junction(dtype="f32", collision="CUM", cy_mode="none", nu=0.02, bounce_back="fullway", n_cases=1):
    wall = small_junction()
    nz, ny, nx = wall.shape
    cy = CY if cy_mode != "none" else (0.0, 0.0, 2.0, 1.0)
    specs = [CaseSpec((nx, ny, nz), collision=collision, dtype=dtype, cy_mode=cy_mode, nu=nu * (1 + 0.25 * k), cy=cy,
                      bounce_back=bounce_back) for k in range(n_cases)]
    lat = Lattice(specs)
    for k in range(n_cases):
        counts = lat.setup_tcpc(wall, ic=k)
        lat.set_inflow(ivc_flux=0.03 * counts["left_area"], svc_flux=0.02 * counts["right_area"], ic=k)
    lat.init_equilibrium()
    return lat


def _box(nx, dtype="f32", collision="CUM"):
    m, prof = G.dense_box_map(nx, 6, 5)
    nz, ny, _ = m.shape
    lat = Lattice(CaseSpec((nx, ny, nz), collision=collision, dtype=dtype, nu=0.05 / 3))
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.05)
    lat.init_equilibrium()
    return lat


def _close(x, y, exact, atol=1e-9):
    if exact:
        return np.array_equal(x, y)
    return np.allclose(x, y, rtol=1e-5, atol=atol)


def _same(a: Lattice, b: Lattice, n_cases=1, stats=False, exact=True):
    for k in range(n_cases):
        assert _close(a.export_df(k), b.export_df(k), exact), k
        # velocities of order 0.05 that cross zero: 1e-7 absolute beside the relative bound
        assert _close(a.macro_all(k), b.macro_all(k), exact, atol=1e-7), k
        if stats:
            sa, na = a.stats(k)
            sb, nb = b.stats(k)
            assert na == nb and _close(sa, sb, exact, atol=1e-7), k


def _compare(make, n_cases=1, stats=False, steps=(1, 1, 5, 13), exact=True):
    plain, staged = make(), make()
    plain.set_launch(128, 2)
    staged.set_launch(128, 2, staged=True)
    assert staged.launch() == {"block": 128, "cells_per_thread": 2, "staged": True}
    assert plain.launch()["staged"] is False
    for n in steps:
        plain.step(n, macro=True, stats=stats, reduce=True)
        staged.step(n, macro=True, stats=stats, reduce=True)
        _same(plain, staged, n_cases, stats, exact)
    for k in range(n_cases):
        assert _close(plain.reduce(k), staged.reduce(k), exact, atol=1e-7)


@pytest.mark.parametrize("nx", [130, 131])
@pytest.mark.parametrize("dtype", ["f32", "f16", "bf16"])
def test_staged_box_bitwise(nx, dtype):
    """Full 64-cell spans (x-adjacent pairs); with nx = 131 the odd step's windows start at
    every offset within their 16-byte boundary.  The box's face chunks step one cell a
    thread (FP32 to rounding, FP16/BF16 storage bitwise)."""
    _compare(lambda: _box(nx, dtype), exact=dtype != "f32")


@pytest.mark.parametrize("collision", ["CUM", "BGK", "MRT_LES"])
def test_staged_junction_bitwise(collision):
    """Partial chunks (non-adjacent pairs), fused open-plane nodes, gathered nodes, the
    local Carreau-Yasuda viscosity and the FP64 mean/rms sums."""
    _compare(lambda: _junction(collision=collision, cy_mode="local-neq"), stats=True)


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
def test_staged_junction_16bit_bitwise(dtype):
    _compare(lambda: _junction(dtype=dtype, cy_mode="local-neq"), stats=True)


@pytest.mark.parametrize("n_cases", [2, 17])
def test_staged_batched_bitwise(n_cases):
    """Cases read from the kernel parameters (2) and from the device array (17)."""
    _compare(lambda: _junction(n_cases=n_cases), n_cases=n_cases, steps=(1, 4))


def test_staged_unstaged_chunks_bitwise():
    """Halfway bounce-back (chunks next to a wall take the general path) and the
    finite-difference Carreau-Yasuda force (no chunk pairs): the staged kernel steps them
    unstaged."""
    _compare(lambda: _junction(bounce_back="halfway"), exact=False)
    _compare(lambda: _junction(cy_mode="ref-fd"), steps=(1, 2), exact=False)


def test_staged_vs_fp64_oracle():
    """The staged form against the FP64 oracle after 200 steps, relative to the peak velocity."""
    wall = small_junction()
    nz, ny, nx = wall.shape
    orc = O.Oracle(nx, ny, nz, collision=0, nu=0.02)
    rc, counts = orc.setup_tcpc(wall)
    assert rc == 0
    lat = _junction()
    lat.set_launch(128, 2, staged=True)
    orc.set_inflow(ivc_flux=0.03 * counts[0], svc_flux=0.02 * counts[1])
    orc.init_equilibrium()
    orc.step(200)
    lat.step(200, macro=True)
    fluid = orc.get_map() == G.MAP_FLUID
    umax = np.max(np.abs(orc.get_macro(O.M_VX)[fluid]))
    for fo, fl in ((O.M_VX, capi.M_VX), (O.M_VY, capi.M_VY), (O.M_VZ, capi.M_VZ)):
        err = np.max(np.abs(lat.macro(fl)[fluid] - orc.get_macro(fo)[fluid])) / umax
        assert err <= 2e-5, err


def test_staged_form_only_where_collisions_pair():
    """KBC and FP64 have no two-cell form: asking for the staged one leaves them one cell a
    thread."""
    for dtype, col in (("f32", "KBC_N4"), ("f64", "CUM")):
        lat = _box(130, dtype, col)
        lat.set_launch(128, 2, staged=True)
        assert lat.launch() == {"block": 128, "cells_per_thread": 1, "staged": False}


_STALL = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import geometry as G
m, prof = G.dense_box_map(130, 6, 5)
nz, ny, nx = m.shape
def box():
    lat = Lattice(CaseSpec((nx, ny, nz), collision="CUM", dtype="f32", nu=0.05 / 3))
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.05)
    lat.init_equilibrium()
    lat.set_launch(128, 2, staged=True)
    return lat
lat = box()
try:
    lat.step(2)
    print("NO_ERROR")
except capi.NnlbmError as e:
    print("CODE", e.code)
lat.close()
# a context created without the stall steps normally on the same device
os.environ.pop("NNLBM_TEST_STAGE_STALL")
ok = box()
ok.step(4)
print("RECOVERED", ok.launch()["staged"])
"""


def test_staged_wait_gives_up_with_timeout():
    """Every wait of the staged step expects 16 bytes more than its copies bring (all of them
    land), so each gives up after its 1 ms limit: the step returns NNLBM_ERR_TIMEOUT, and a
    new context steps normally afterwards."""
    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ, NNLBM_TEST_STAGE_STALL="1")
    p = subprocess.run([sys.executable, "-c", _STALL, str(root)], capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "CODE -4" in p.stdout, p.stdout
    assert "RECOVERED True" in p.stdout, p.stdout

"""Pipelined stepping with NNLBM_STEP_READBACK: every step's control row goes to the device and its
status block (step cursors, watchdog flags, FP64 sums) comes back, with the next step enqueued
before the host waits for the copy.  The sums and the populations must be bitwise those of the
same steps taken synchronously one by one."""
from __future__ import annotations

import numpy as np
import pytest

from nonnewlbm_b200 import CaseSpec, Lattice, capi

from helpers import small_junction

pytestmark = pytest.mark.gpu


def _lattice(n_cases=1):
    wall = small_junction()
    nz, ny, nx = wall.shape
    lat = Lattice([CaseSpec((nx, ny, nz), dtype="f32", nu=0.02 * (1 + 0.5 * k)) for k in range(n_cases)])
    areas = []
    for k in range(n_cases):
        c = lat.setup_tcpc(wall, ic=k)
        areas.append((c["left_area"], c["right_area"]))
    lat.init_equilibrium()
    return lat, areas


def _row(areas, k, step):
    a, b = areas[k]
    s = 1.0 + 0.05 * np.sin(0.3 * step + k)
    return np.array([[0.03 * a * s, 0.02 * b * s, 1.0]])


@pytest.mark.parametrize("n_cases", [1, 3])
def test_pipelined_readback_matches_synchronous_steps(n_cases):
    n = 12
    sync, areas = _lattice(n_cases)
    pipe, _ = _lattice(n_cases)
    expect = []
    for step in range(n):
        for k in range(n_cases):
            sync.set_schedule(_row(areas, k, step), ic=k)
        sync.step(1, stats=True, reduce=True)
        expect.append(np.array([sync.reduce(k) for k in range(n_cases)]))
    got = []
    for step in range(n):
        for k in range(n_cases):
            pipe.set_schedule(_row(areas, k, step), ic=k)
        pipe.step(1, stats=True, reduce=True, wait=False, readback=True)
        if step > 0:
            got.append(pipe.readback())  # the step before this one
    got.append(pipe.readback())
    assert len(got) == n
    for e, g in zip(expect, got):
        assert np.array_equal(e, g)
    for k in range(n_cases):
        assert np.array_equal(sync.export_df(k), pipe.export_df(k))
        assert np.array_equal(sync.stats(k)[0], pipe.stats(k)[0])


def test_pipelined_readback_two_launch_groups():
    """A context of two launch groups (cumulant and BGK): each group's cursors are checked at
    its own parity, and the sums match synchronous steps."""
    wall = small_junction()
    nz, ny, nx = wall.shape
    def make():
        lat = Lattice([CaseSpec((nx, ny, nz), dtype="f32", collision=col, nu=0.02) for col in ("CUM", "BGK")])
        areas = []
        for k in range(2):
            c = lat.setup_tcpc(wall, ic=k)
            areas.append((c["left_area"], c["right_area"]))
        lat.init_equilibrium()
        return lat, areas
    sync, areas = make()
    pipe, _ = make()
    expect, got = [], []
    for step in range(7):
        for k in range(2):
            sync.set_schedule(_row(areas, k, step), ic=k)
            pipe.set_schedule(_row(areas, k, step), ic=k)
        sync.step(1, reduce=True)
        expect.append(np.array([sync.reduce(k) for k in range(2)]))
        pipe.step(1, reduce=True, wait=False, readback=True)
        if step > 0:
            got.append(pipe.readback())
    got.append(pipe.readback())
    for e, g in zip(expect, got):
        assert np.array_equal(e, g)


def test_readback_refusals():
    lat, _ = _lattice()
    with pytest.raises(capi.NnlbmError):
        lat.readback()  # nothing pending
    with pytest.raises(capi.NnlbmError):
        lat.step(1, reduce=True, readback=True)  # needs NNLBM_STEP_ASYNC
    for _ in range(capi.READBACK_SLOTS):
        lat.step(1, reduce=True, wait=False, readback=True)
    with pytest.raises(capi.NnlbmError):
        lat.step(1, reduce=True, wait=False, readback=True)  # every slot pending
    for _ in range(capi.READBACK_SLOTS):
        assert lat.readback().shape == (1, 5)
    with pytest.raises(capi.NnlbmError):
        lat.readback()
    lat.step(2, reduce=True)  # synchronous steps go on as before
    assert np.isfinite(lat.reduce()).all()


def test_copy_paths_match_kernel_paths(monkeypatch):
    """NNLBM_PROLOGUE_COPY=1 and NNLBM_READBACK_COPY=1 (read at context creation) move the control
    rows and the status block with copies instead of the prologue and publish kernels: the sums
    and the populations are bitwise the same."""
    n = 9
    fast, areas = _lattice(2)
    monkeypatch.setenv("NNLBM_PROLOGUE_COPY", "1")
    monkeypatch.setenv("NNLBM_READBACK_COPY", "1")
    copy, _ = _lattice(2)
    got = {id(fast): [], id(copy): []}
    for lat in (fast, copy):
        for step in range(n):
            for k in range(2):
                lat.set_schedule(_row(areas, k, step), ic=k)
            lat.step(1, stats=True, reduce=True, wait=False, readback=True)
            if step > 0:
                got[id(lat)].append(lat.readback())
        got[id(lat)].append(lat.readback())
    for a, b in zip(got[id(fast)], got[id(copy)]):
        assert np.array_equal(a, b)
    for k in range(2):
        assert np.array_equal(fast.export_df(k), copy.export_df(k))

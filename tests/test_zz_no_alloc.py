"""nnlbm_step_noalloc (steps without any device allocation) against nnlbm_step.

Both entry points run the same kernels on the same state; the no-allocation one keeps its
per-call scratch (step counters, gathered open-plane node values) in the library's static
device array.  The comparison runs two calls in a row, so the second call starts from a
scratch array that the first one left behind.

Tolerances (FP32 storage and arithmetic): populations, macro fields and mean/rms sums
within 1e-6 relative to their peak magnitude (the kernels are identical, so equal bits are
expected); FP64 reduction sums within 1e-9 relative (atomic summation order).

This file is named to be collected last; it also passes on its own.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from nonnewlbm_b200 import CaseSpec, Lattice, capi
from nonnewlbm_b200 import geometry as G

from helpers import small_junction

pytestmark = pytest.mark.gpu

FLAGS = capi.STEP_STATS | capi.STEP_MACRO | capi.STEP_REDUCE
TOL = 1e-6
TOL_RED = 1e-9


def _context():
    """FP32 cumulant junction (local Carreau-Yasuda) and an open box whose plane corners
    are gathered, batched in one launch group."""
    wall_j = small_junction()
    wall_b = np.zeros((10, 12, 14), dtype=np.int32)
    specs = [CaseSpec(wall_j.shape[::-1], dtype="f32", collision="CUM", cy_mode="local-neq", nu=0.01,
                      cy=(0.05, 2.0, 2.0, 0.4)),
             CaseSpec(wall_b.shape[::-1], dtype="f32", collision="CUM", nu=0.05)]
    lat = Lattice(specs)
    for ic, wall in enumerate((wall_j, wall_b)):
        c = lat.setup_tcpc(wall, ic=ic)
        lat.set_inflow(ivc_flux=0.03 * c["left_area"], svc_flux=0.02 * c["right_area"], ic=ic)
    lat.init_equilibrium()
    return lat


def _noalloc(lat: Lattice, n: int, flags: int) -> int:
    return capi.lib().nnlbm_step_noalloc(lat.h, n, flags)


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def test_noalloc_matches_step_two_calls():
    ref, na = _context(), _context()
    assert ref.step_info(1)["launches_per_step"] >= 2, "the open box must exercise the gathered-node scratch"
    # the first nnlbm_step of each context allocates the group, macro and mean/rms buffers
    for L in (ref, na):
        L.step(3, stats=True, macro=True, reduce=True)
    for call in range(2):
        n = 7 + call
        ref.step(n, stats=True, macro=True, reduce=True)
        rc = _noalloc(na, n, FLAGS)
        assert rc == capi.OK, capi.last_error(na.h)
        for ic in range(2):
            assert _rel(na.export_df(ic), ref.export_df(ic)) <= TOL, (call, ic)
            for f in (capi.M_RHO, capi.M_VX, capi.M_VY, capi.M_VZ, capi.M_S11, capi.M_S12):
                assert _rel(na.macro(f, ic), ref.macro(f, ic)) <= TOL, (call, ic, f)
            s_na, n_na = na.stats(ic)
            s_ref, n_ref = ref.stats(ic)
            assert n_na == n_ref == 3 + 7 + (8 if call else 0)
            assert _rel(s_na, s_ref) <= TOL, (call, ic)
            r_na, r_ref = na.reduce(ic), ref.reduce(ic)
            assert np.all(np.abs(r_na - r_ref) <= TOL_RED * np.maximum(np.abs(r_ref), 1.0)), (call, ic)


def test_noalloc_refuses_what_it_would_have_to_allocate():
    lat = _context()
    # no device work list yet
    rc = _noalloc(lat, 1, 0)
    assert rc == capi.ERR_ARG and "nnlbm_step or nnlbm_step_info" in capi.last_error(lat.h)
    lat.step_info(0)
    # mean/rms and macro buffers do not exist before a step with those flags
    rc = _noalloc(lat, 1, capi.STEP_STATS)
    assert rc == capi.ERR_ARG and "NNLBM_STEP_STATS" in capi.last_error(lat.h)
    # more steps than control rows
    rc = _noalloc(lat, 1 << 20, 0)
    assert rc == capi.ERR_ARG and "control rows" in capi.last_error(lat.h)
    # nothing ran: the state is still the initial one and a plain call works
    assert _noalloc(lat, 2, capi.STEP_REDUCE) == capi.OK, capi.last_error(lat.h)


def test_noalloc_refuses_more_nodes_than_the_scratch_holds():
    # 520 x 520 prescribed-velocity inlet nodes: 270,400 x 4 FP32 values > 4 MiB - 1 KiB
    m, prof = G.dense_box_map(4, 520, 520)
    lat = Lattice(CaseSpec((4, 520, 520), dtype="f32", collision="BGK", nu=0.05))
    lat.set_map(m)
    lat.set_inflow_profile(prof * 0.01)
    lat.init_equilibrium()
    lat.step_info(0)
    rc = _noalloc(lat, 1, 0)
    msg = capi.last_error(lat.h)
    assert rc == capi.ERR_ARG and "NNLBM_NOALLOC_SCRATCH_BYTES" in msg, msg
    lat.close()


# Run in a fresh interpreter (torch switches CUDA's lazy module loading on, as a host
# application usually has it): free device memory around two no-allocation calls.  First
# after nnlbm_step has run the kernels once (the documented order), then, printed for the
# record, in a context whose kernels have never been launched.
_FRESH = r"""
import sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/tests"]
import torch
from nonnewlbm_b200 import CaseSpec, Lattice, capi
from helpers import small_junction

def context(collision):
    wall = small_junction()
    lat = Lattice(CaseSpec(wall.shape[::-1], dtype="f32", collision=collision, nu=0.02))
    c = lat.setup_tcpc(wall)
    lat.set_inflow(ivc_flux=0.03 * c["left_area"], svc_flux=0.02 * c["right_area"])
    lat.init_equilibrium()
    return lat

def free():
    torch.cuda.synchronize(0)
    return torch.cuda.mem_get_info(0)[0]

def two_calls(lat):
    for _ in range(2):
        rc = capi.lib().nnlbm_step_noalloc(lat.h, 5, capi.STEP_REDUCE)
        assert rc == capi.OK, capi.last_error(lat.h)

free()
a = context("CUM")
a.step(1, reduce=True)
f0 = free()
two_calls(a)
f1 = free()
b = context("BGK")  # a launch group whose kernels this process has not run
b.step_info(0)
g0 = free()
two_calls(b)
g1 = free()
print("after-step", f0, f1, "never-launched", g0, g1)
sys.exit(0 if f1 == f0 else 1)
"""


def test_noalloc_first_calls_take_no_device_memory():
    """The first two calls in a fresh process leave the device's free memory unchanged."""
    root = Path(__file__).resolve().parents[1]
    p = subprocess.run([sys.executable, "-c", _FRESH, str(root)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr

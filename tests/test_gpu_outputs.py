"""The driver's output path on the device: a geometry file in the geometry pipeline's layout
read by the drop-in driver, FP64 steps with the local Carreau-Yasuda viscosity, and the
result file rank000_data_<n>.vtk written from nnlbm_output_fields, checked field by field
against the FP64 oracle run of the same case put through the oracle's restatement of
outputData (oracle/outputs.py, solver/sim_tcpc/sim_tcpc.cu:684-784).

Tolerance: the file holds floats; each value within 2e-6 of its field's largest magnitude
(float rounding of values that agree to 1e-12 in double)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import oracle.outputs as OO
from nonnewlbm_b200 import vtk
from nonnewlbm_b200.tcpc import TcpcOptions, TcpcRun

from helpers import raw_pipeline_labels, small_junction, write_pipeline_geometry

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("material", ["gx", "newtonian"])
def test_result_file_against_oracle(tmp_path, material):
    wall = small_junction()
    nz, ny, nx = wall.shape
    geo = tmp_path / "geometry.vtk"
    write_pipeline_geometry(geo, raw_pipeline_labels(wall), 2.5e-4, legacy_51=True)
    o = TcpcOptions(geometry=str(geo), material=material, case_id="out", ivc_mls=0.02, svc_mls=0.012,
                    lbm_viscosity=0.02, dtype="f64", cy_mode="local-neq", results_root=str(tmp_path))
    run = TcpcRun(o)
    steps, stats_from = 40, 15
    run.lat.step(stats_from)
    run.lat.stat_reset()
    run.prev_iter = stats_from
    run.lat.step(steps - stats_from, stats=True, macro=True)
    run.iterations = steps
    path = run.write_vtk(3)
    assert path.name == "rank000_data_3.vtk"
    got = vtk.read_rectilinear(path)

    c = run.conv
    cy = (c["nu0"], c["lambda"], c["a"], c["n"]) if run.mat.carreau_yasuda else None
    orc = O.Oracle(nx, ny, nz, collision=0, nu=c["nu"], cy_mode=O.CY_LOCAL_NEQ if cy else O.CY_NONE,
                   cy=cy if cy else (0.0, 0.0, 2.0, 1.0))
    rc, counts = orc.setup_tcpc(wall)
    assert rc == 0
    orc.set_inflow(ivc_flux=run.ivc, svc_flux=run.svc)
    orc.init_equilibrium()
    orc.step(stats_from, accumulate_stats=False)
    orc.step(steps - stats_from, accumulate_stats=True)
    S = [orc.get_macro(f) for f in (O.M_S11, O.M_S12, O.M_S13, O.M_S22, O.M_S32, O.M_S33)]
    if cy is None:
        S = [np.zeros_like(s) for s in S]  # the collision viscosity is Newtonian: no strain is stored
    sums = [orc.get_macro(O.M_VM_PLUS_X) + orc.get_macro(O.M_VM_MINUS_X), orc.get_macro(O.M_VM_Y),
            orc.get_macro(O.M_VM_Z), orc.get_macro(O.M_VM_XX), orc.get_macro(O.M_VM_YY), orc.get_macro(O.M_VM_ZZ)]
    u = np.stack([orc.get_macro(O.M_VX), orc.get_macro(O.M_VY), orc.get_macro(O.M_VZ)])
    ref = OO.output_data(orc.get_macro(O.M_RHO), u, S, sums, steps - stats_from, run.wall_flags, run.dx, run.dt,
                         run.mat.density, run.dt / run.dx / run.dx * run.mat.nu_inf, cy=cy)

    pd = got["point_data"]
    assert list(pd) == ["wall"] + OO.FIELDS
    np.testing.assert_array_equal(pd["wall"].reshape(nz, ny, nx), orc.get_map())
    n = nx * ny * nz
    for name in OO.FIELDS:
        r = ref[name]
        g = pd[name]
        r = r.reshape(3, n).T if r.ndim == 4 else r.reshape(-1)
        scale = max(float(np.max(np.abs(r))), 1e-30)
        err = float(np.max(np.abs(g - r))) / scale
        assert err <= 2e-6, (name, err)
    # the fields are not trivially zero
    assert np.max(np.abs(pd["velocity"])) > 0 and np.max(np.abs(pd["mean_velocity"])) > 0
    if cy is not None:
        assert np.max(pd["wss_proxy_pa"]) > 0 and np.max(pd["gamma_dot"]) > 0
    run.lat.close()

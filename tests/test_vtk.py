"""The file contract of the driver on the host (no GPU): the 3D result file of
State::writeVTK_3D_singlefile (solver/lbm3d/state.hpp:782-851, big-endian writer of
solver/lbm3d/vtk_writer.hpp:1-60) byte by byte, and the geometry input written in the layout
of the geometry pipeline (geometry/tcpc_geometry.py:619-679) read back and set up like the
reference's readGeometry + setupBoundaries (solver/sim_tcpc/sim_tcpc.cu:134-185, 494-645)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from nonnewlbm_b200 import capi, vtk

from helpers import raw_pipeline_labels, small_junction, write_pipeline_geometry


def _take_line(buf: bytes, i: int):
    j = buf.index(b"\n", i)
    return buf[i:j].decode(), j + 1


def test_result_file_layout(tmp_path):
    rng = np.random.default_rng(5)
    nz, ny, nx = 3, 4, 5
    n = nx * ny * nz
    labels = rng.integers(0, 7, (nz, ny, nx)).astype(np.uint8)
    fields = []
    for name, dofs in capi.OUTPUT_FIELDS:
        shape = (dofs, nz, ny, nx) if dofs > 1 else (nz, ny, nx)
        fields.append((name, rng.standard_normal(shape).astype(np.float32)))
    dx, t, cycle = 2.5e-4, 0.125, 7
    p = tmp_path / "rank000_data_7.vtk"
    vtk.write_output(p, labels, dx, t, cycle, fields)
    b = p.read_bytes()
    i = 0
    for want in ("# vtk DataFile Version 3.0", "Written using RF writer", "BINARY", "DATASET RECTILINEAR_GRID",
                 f"DIMENSIONS {nx} {ny} {nz}"):
        line, i = _take_line(b, i)
        assert line == want
    for axis, m in (("X", nx), ("Y", ny), ("Z", nz)):
        line, i = _take_line(b, i)
        assert line == f"{axis}_COORDINATES {m} float"
        got = np.frombuffer(b, dtype=">f4", count=m, offset=i)
        np.testing.assert_array_equal(got, (np.arange(m) * dx).astype(np.float32))
        i += 4 * m
    line, i = _take_line(b, i)
    assert line == "FIELD FieldData 2"
    for name, val in (("TIME", t), ("CYCLE", cycle)):
        line, i = _take_line(b, i)
        assert line == f"{name} 1 1 float"
        assert np.frombuffer(b, dtype=">f4", count=1, offset=i)[0] == np.float32(val)
        i += 4
    for want in (f"POINT_DATA {n}", "SCALARS wall int 1", "LOOKUP_TABLE default"):
        line, i = _take_line(b, i)
        assert line == want
    np.testing.assert_array_equal(np.frombuffer(b, dtype=">i4", count=n, offset=i), labels.reshape(-1))
    i += 4 * n
    # every field in the order of outputData (sim_tcpc.cu:747-782), x fastest, vector
    # components interleaved per point
    for name, arr in fields:
        if arr.ndim == 4:
            line, i = _take_line(b, i)
            assert line == f"VECTORS {name} float"
            got = np.frombuffer(b, dtype=">f4", count=3 * n, offset=i).reshape(n, 3)
            np.testing.assert_array_equal(got, arr.reshape(3, n).T)
            i += 12 * n
        else:
            for want in (f"SCALARS {name} float 1", "LOOKUP_TABLE default"):
                line, i = _take_line(b, i)
                assert line == want
            np.testing.assert_array_equal(np.frombuffer(b, dtype=">f4", count=n, offset=i), arr.reshape(-1))
            i += 4 * n
    assert i == len(b)
    # and the general reader gives the same arrays back
    r = vtk.read_rectilinear(p)
    assert list(r["point_data"]) == ["wall"] + [nm for nm, _ in fields]


@pytest.mark.parametrize("legacy_51", [False, True], ids=["vtk3.0", "vtk5.1-metadata"])
def test_pipeline_geometry_file(tmp_path, legacy_51):
    wall = small_junction()
    nz, ny, nx = wall.shape
    dx = 3.125e-4
    p = tmp_path / "geometry.vtk"
    write_pipeline_geometry(p, raw_pipeline_labels(wall), dx, legacy_51=legacy_51)
    got, dims, gdx = vtk.read_geometry(p)
    assert dims == (nx, ny, nz) and gdx == pytest.approx(dx, rel=1e-15)
    np.testing.assert_array_equal(got, wall)
    # the boundary setup of the product (host C ABI) and of the oracle agree on it
    m, counts, rc, wf = capi.tcpc_labels(got, with_wall_flags=True)
    orc = O.Oracle(nx, ny, nz)
    rc_o, counts_o = orc.setup_tcpc(got)
    assert rc == rc_o == 0
    np.testing.assert_array_equal(m, orc.get_map())
    assert counts["left_area"] == counts_o[0] and counts["outlet6"] == counts_o[3]

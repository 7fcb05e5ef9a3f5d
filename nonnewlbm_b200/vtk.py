"""Legacy-VTK rectilinear-grid I/O in numpy (the reference uses the VTK C++ library).

* ``read_geometry``: the solver's geometry input -- a RECTILINEAR_GRID whose cell array
  ``wall`` holds the voxel labels; dimensions are the point counts minus one and the
  spacing is the first positive step of the x coordinates
  (solver/sim_tcpc/sim_tcpc.cu:134-185).
* ``write_geometry``: the same file as geometry/tcpc_geometry.py:619-661 writes (binary,
  big endian, double coordinates and a double cell array).
* ``write_output``: the 3D result file of State::writeVTK_3D_singlefile
  (solver/lbm3d/state.hpp:782-851): BINARY big-endian, float coordinates, TIME/CYCLE
  field data, POINT_DATA with the int ``wall`` map labels and then every output field as
  float SCALARS or VECTORS (solver/lbm3d/vtk_writer.hpp:25-60).
* ``read_rectilinear``: a general reader for both (ASCII or BINARY, SCALARS, VECTORS and
  FIELD arrays, METADATA blocks skipped).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

_TYPES = {"bit": None, "unsigned_char": ">u1", "char": ">i1", "unsigned_short": ">u2", "short": ">i2",
          "unsigned_int": ">u4", "int": ">i4", "unsigned_long": ">u8", "long": ">i8", "vtktypeint64": ">i8",
          "vtktypeuint64": ">u8", "float": ">f4", "double": ">f8"}


class _Cursor:
    def __init__(self, data: bytes, binary: bool):
        self.d = data
        self.i = 0
        self.binary = binary

    def line(self) -> str:
        j = self.d.index(b"\n", self.i)
        s = self.d[self.i:j].decode("latin-1").strip()
        self.i = j + 1
        return s

    def next_line(self) -> str | None:
        while self.i < len(self.d):
            s = self.line()
            if s:
                return s
        return None

    def array(self, n: int, vtype: str) -> np.ndarray:
        dt = _TYPES.get(vtype.lower())
        if dt is None:
            raise ValueError(f"unsupported VTK type {vtype}")
        if self.binary:
            size = np.dtype(dt).itemsize * n
            a = np.frombuffer(self.d, dtype=dt, count=n, offset=self.i)
            self.i += size
            # a newline usually follows binary blocks
            if self.i < len(self.d) and self.d[self.i:self.i + 1] == b"\n":
                self.i += 1
            return a.astype(np.dtype(dt).newbyteorder("="))
        vals = []
        while len(vals) < n:
            vals.extend(self.line().split())
        return np.array(vals[:n], dtype=np.dtype(dt).newbyteorder("="))

    def skip_metadata(self):
        # METADATA blocks end at an empty line
        while self.i < len(self.d):
            s = self.line()
            if s == "":
                break


def read_rectilinear(path) -> dict:
    data = Path(path).read_bytes()
    head = data[:2048].split(b"\n")
    fmt = head[2].strip().upper()
    cur = _Cursor(data, binary=(fmt == b"BINARY"))
    for _ in range(3):
        cur.line()
    out = {"dims": None, "coords": {}, "point_data": {}, "cell_data": {}, "field": {}}
    section = None
    while True:
        s = cur.next_line()
        if s is None:
            break
        tok = s.split()
        key = tok[0].upper()
        if key == "DATASET":
            if tok[1].upper() != "RECTILINEAR_GRID":
                raise ValueError(f"{path}: not a RECTILINEAR_GRID")
        elif key == "DIMENSIONS":
            out["dims"] = tuple(int(v) for v in tok[1:4])
        elif key in ("X_COORDINATES", "Y_COORDINATES", "Z_COORDINATES"):
            out["coords"][key[0].lower()] = cur.array(int(tok[1]), tok[2])
        elif key == "POINT_DATA":
            section = out["point_data"]
            out["n_points"] = int(tok[1])
        elif key == "CELL_DATA":
            section = out["cell_data"]
            out["n_cells"] = int(tok[1])
        elif key == "METADATA":
            cur.skip_metadata()
        elif key == "FIELD":
            nfields = int(tok[2])
            dest = section if section is not None else out["field"]
            for _ in range(nfields):
                t = cur.next_line().split()
                if t[0].upper() == "METADATA":
                    cur.skip_metadata()
                    t = cur.next_line().split()
                name, ncomp, ntup, vt = t[0], int(t[1]), int(t[2]), t[3]
                a = cur.array(ncomp * ntup, vt)
                dest[name] = a.reshape(ntup, ncomp) if ncomp > 1 else a
        elif key == "SCALARS":
            name, vt = tok[1], tok[2]
            ncomp = int(tok[3]) if len(tok) > 3 else 1
            t = cur.next_line()
            if not t.upper().startswith("LOOKUP_TABLE"):
                raise ValueError(f"{path}: expected LOOKUP_TABLE after SCALARS {name}")
            n = out["n_points"] if section is out["point_data"] else out["n_cells"]
            a = cur.array(n * ncomp, vt)
            section[name] = a.reshape(n, ncomp) if ncomp > 1 else a
        elif key in ("VECTORS", "NORMALS"):
            name, vt = tok[1], tok[2]
            n = out["n_points"] if section is out["point_data"] else out["n_cells"]
            section[name] = cur.array(3 * n, vt).reshape(n, 3)
        elif key == "LOOKUP_TABLE":
            n = int(tok[2])
            cur.array(4 * n, "float")
        else:
            raise ValueError(f"{path}: unsupported legacy VTK keyword {key}")
    return out


def read_geometry(path):
    """readGeometry (sim_tcpc.cu:134-185): returns (wall [z][y][x] int32, (nx, ny, nz), dx)."""
    g = read_rectilinear(path)
    if g["dims"] is None:
        raise ValueError(f"{path} is not a legacy VTK RectilinearGrid file.")
    nx, ny, nz = (d - 1 for d in g["dims"])
    xs = g["coords"].get("x")
    if xs is None or len(xs) < 2:
        raise ValueError("Missing rectilinear x coordinates.")
    steps = np.abs(np.diff(np.asarray(xs, dtype=np.float64)))
    pos = steps[steps > 0]
    if pos.size == 0:
        raise ValueError("Cannot infer positive rectilinear x spacing.")
    dx = float(pos[0])
    if "wall" not in g["cell_data"]:
        raise ValueError(f"{path} does not contain a cell-data array named 'wall'.")
    wall = np.asarray(g["cell_data"]["wall"]).reshape(-1)
    if wall.size != nx * ny * nz:
        raise ValueError(f"{path}: wall array has {wall.size} values for {nx}x{ny}x{nz} cells")
    return wall.astype(np.int32).reshape(nz, ny, nx), (nx, ny, nz), dx


def write_geometry(path, wall: np.ndarray, dx: float) -> None:
    """Geometry file with a double cell array ``wall`` ([z][y][x]) and point coordinates
    0, dx, ..., n*dx (geometry/tcpc_geometry.py:619-661)."""
    w = np.asarray(wall)
    nz, ny, nx = w.shape
    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 3.0\nvtk output\nBINARY\nDATASET RECTILINEAR_GRID\n")
        f.write(f"DIMENSIONS {nx + 1} {ny + 1} {nz + 1}\n".encode())
        for axis, n in (("X", nx), ("Y", ny), ("Z", nz)):
            f.write(f"{axis}_COORDINATES {n + 1} double\n".encode())
            f.write((np.arange(n + 1) * dx).astype(">f8").tobytes())
            f.write(b"\n")
        f.write(f"CELL_DATA {nx * ny * nz}\nSCALARS wall double 1\nLOOKUP_TABLE default\n".encode())
        f.write(w.reshape(-1).astype(">f8").tobytes())
        f.write(b"\n")


def write_output(path, labels: np.ndarray, dx: float, time: float, cycle: int, fields) -> None:
    """Result file of writeVTK_3D_singlefile (state.hpp:782-851).  ``fields`` is an ordered
    list of (name, array) with arrays shaped [z][y][x] (scalars) or [3][z][y][x] (vectors)."""
    lab = np.asarray(labels)
    nz, ny, nx = lab.shape
    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 3.0\nWritten using RF writer\nBINARY\n")
        f.write(b"DATASET RECTILINEAR_GRID\n")
        f.write(f"DIMENSIONS {nx} {ny} {nz}\n".encode())
        for axis, n in (("X", nx), ("Y", ny), ("Z", nz)):
            f.write(f"{axis}_COORDINATES {n} float\n".encode())
            f.write((np.arange(n) * dx).astype(">f4").tobytes())
        f.write(b"FIELD FieldData 2\n")
        f.write(b"TIME 1 1 float\n")
        f.write(np.array([time], dtype=">f4").tobytes())
        f.write(b"CYCLE 1 1 float\n")
        f.write(np.array([cycle], dtype=">f4").tobytes())
        f.write(f"POINT_DATA {nx * ny * nz}\n".encode())
        f.write(b"SCALARS wall int 1\nLOOKUP_TABLE default\n")
        f.write(lab.reshape(-1).astype(">i4").tobytes())
        for name, arr in fields:
            a = np.asarray(arr)
            if a.ndim == 4:
                f.write(f"VECTORS {name} float\n".encode())
                f.write(np.moveaxis(a, 0, -1).reshape(-1).astype(">f4").tobytes())
            else:
                f.write(f"SCALARS {name} float 1\nLOOKUP_TABLE default\n".encode())
                f.write(a.reshape(-1).astype(">f4").tobytes())

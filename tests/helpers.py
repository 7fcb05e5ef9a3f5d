"""Shared test helpers: synthetic cases and the comparison rules."""
from __future__ import annotations

import numpy as np

from nonnewlbm_b200 import geometry as G


def small_junction():
    """40x32x28 synthetic TCPC-like junction, geometry 'wall' array (0 fluid, 1 wall, 3..6)."""
    study = G.junction(40, 32, 28, r_ivc=6, r_svc=5, r_chamber=7, r_out=4.5, z_offset=2)
    return G.study_to_geometry(study)


def dead_mask(labels: np.ndarray) -> np.ndarray:
    """[27][z][y][x] True where a population is never read by any cell: the outward
    populations of wall nodes on the domain faces.  The reference fills them from clamped
    neighbour indices (solver/lbm3d/core.h:651-661); the A-A layout leaves them undefined."""
    nz, ny, nx = labels.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    out = np.zeros((27,) + labels.shape, dtype=bool)
    wall = labels == G.MAP_WALL
    for q in range(27):
        cx, cy, cz = q // 9 - 1, (q // 3) % 3 - 1, q % 3 - 1
        leaves = (x + cx < 0) | (x + cx >= nx) | (y + cy < 0) | (y + cy >= ny) | (z + cz < 0) | (z + cz >= nz)
        out[q] = wall & leaves
    return out


def max_rel(a: np.ndarray, b: np.ndarray, mask: np.ndarray | None = None) -> float:
    d = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    if mask is not None:
        d = np.where(mask, 0.0, d)
    return float(np.max(d))


# raw labels of the geometry pipeline's voxel array and their newIndex2 translation
# (geometry/tcpc_geometry.py:663-679): 2 wall -> 1, 1 fluid -> 0, 13..16 caps -> 3..6
NEW_INDEX2 = {2: 1, 1: 0, 16: 6, 14: 4, 15: 5, 13: 3}


def raw_pipeline_labels(wall_zyx: np.ndarray) -> np.ndarray:
    """A geometry 'wall' array [z][y][x] (0 fluid, 1 wall, 3..6 caps) back in the pipeline's raw
    labels, indexed [x][y][z] like its `labeled` array."""
    inv = {v: k for k, v in NEW_INDEX2.items()}
    raw = np.vectorize(lambda v: inv.get(int(v), int(v)))(wall_zyx)
    return np.ascontiguousarray(np.transpose(raw, (2, 1, 0)))


def write_pipeline_geometry(path, labeled_xyz: np.ndarray, dx: float, legacy_51: bool = False) -> None:
    """The geometry file as saveToVTK2 (geometry/tcpc_geometry.py:619-661) has VTK's
    vtkRectilinearGridWriter write it in binary: point coordinates 0, dx, ..., n*dx as double,
    and a double cell array 'wall' set as the cell scalars, cell i = x + nx*(y + ny*z) holding
    newIndex2(labeled[x, y, z]).  legacy_51: the header and METADATA blocks of the legacy
    format version 5.1 that newer VTK releases write."""
    nx, ny, nz = labeled_xyz.shape
    cells = np.zeros(nx * ny * nz)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                v = int(labeled_xyz[x, y, z])
                cells[x + nx * (y + ny * z)] = NEW_INDEX2.get(v, v)
    meta = b"METADATA\nINFORMATION 0\n\n" if legacy_51 else b""
    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 5.1\n" if legacy_51 else b"# vtk DataFile Version 3.0\n")
        f.write(b"vtk output\nBINARY\nDATASET RECTILINEAR_GRID\n")
        f.write(f"DIMENSIONS {nx + 1} {ny + 1} {nz + 1}\n".encode())
        for axis, n in (("X", nx), ("Y", ny), ("Z", nz)):
            f.write(f"{axis}_COORDINATES {n + 1} double\n".encode())
            f.write((np.arange(n + 1) * dx).astype(">f8").tobytes() + b"\n" + meta)
        f.write(f"CELL_DATA {nx * ny * nz}\nSCALARS wall double 1\nLOOKUP_TABLE default\n".encode())
        f.write(cells.astype(">f8").tobytes() + b"\n" + meta)

"""Synthetic voxel geometries and label conventions.

Three label conventions meet here:

* geometry input ("wall" cell array of ``runtime/geometry.vtk``): 0 fluid, 1 wall, 3/4/5/6
  cap or near-wall layers (geometry/tcpc_geometry.py:619-679).  Only ``wall == 1`` matters
  to the solver (solver/sim_tcpc/sim_tcpc.cu:505-519).
* solver map labels (``MAP_*`` below): 0 FLUID, 1 WALL, 2 PERIODIC, 3 INFLOW_LEFT (IVC),
  4 INFLOW_RIGHT (SVC), 5 OUTFLOW_FRONT (y-min), 6 OUTFLOW_BACK (y-max)
  (sim_tcpc.cu:194-203), plus 7 INFLOW_EQ and 8 OUTFLOW_RIGHT_EQ for the generic inflow
  and outflow blocks (solver/lbm3d/lbm_bc.h:126-129,147-152).
* synthetic study masks: 1 fluid, 2 wall, 3 IVC, 4 SVC, 5 y-min outlet, 6 y-max outlet.

All arrays are indexed ``[z][y][x]`` (x fastest in memory), the order of the geometry
reader (sim_tcpc.cu:508-512).  The real TCPC mask is produced by the reference's STL
pipeline, which needs trimesh/vtk; the seeded synthetic junction below stands in for it.
"""
from __future__ import annotations

import numpy as np

MAP_FLUID, MAP_WALL, MAP_PERIODIC = 0, 1, 2
MAP_INFLOW_LEFT, MAP_INFLOW_RIGHT, MAP_OUTFLOW_FRONT, MAP_OUTFLOW_BACK = 3, 4, 5, 6
MAP_INFLOW_EQ, MAP_OUTFLOW_RIGHT_EQ = 7, 8

STUDY_FLUID, STUDY_WALL, STUDY_IVC, STUDY_SVC, STUDY_OUT_YMIN, STUDY_OUT_YMAX = 1, 2, 3, 4, 5, 6


def study_to_geometry(study: np.ndarray) -> np.ndarray:
    """Translate a study mask (1 fluid, 2 wall, 3..6 caps) to the geometry 'wall' array
    convention (0 fluid, 1 wall, 3..6 caps) read by the TCPC boundary setup."""
    s = np.asarray(study)
    out = np.zeros(s.shape, dtype=np.int32)
    out[s == STUDY_WALL] = 1
    for lab in (3, 4, 5, 6):
        out[s == lab] = lab
    bad = ~np.isin(s, [1, 2, 3, 4, 5, 6])
    if bad.any():
        raise ValueError(f"study mask holds labels outside 1..6: {np.unique(s[bad])}")
    return out


def _grid(nx: int, ny: int, nz: int):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return x, y, z


def junction(nx: int = 256, ny: int = 192, nz: int = 160, scale: float | None = None,
             r_ivc: float = 20.0, r_svc: float = 16.0, r_chamber: float = 24.0,
             r_out: float = 14.0, z_offset: float = 8.0) -> np.ndarray:
    """Synthetic TCPC-like junction as a study mask (1 fluid, 2 wall, 3..6 caps).

    An IVC tube along +x from x-min (axis at z = zc - z_offset) and an SVC tube along -x
    from x-max (axis at z = zc + z_offset) meet a spherical chamber at the centre, which
    drains into two outlet tubes along -y and +y.  ``scale`` multiplies the dimensions,
    radii and offset of the 256x192x160 base.
    """
    if scale is not None:
        nx, ny, nz = (max(8, int(round(v * scale))) for v in (256, 192, 160))
        r_ivc, r_svc, r_chamber, r_out, z_offset = (v * scale for v in (r_ivc, r_svc, r_chamber, r_out, z_offset))
    x, y, z = _grid(nx, ny, nz)
    xc, yc, zc = (nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0
    ivc = ((y - yc) ** 2 + (z - (zc - z_offset)) ** 2 <= r_ivc ** 2) & (x <= xc)
    svc = ((y - yc) ** 2 + (z - (zc + z_offset)) ** 2 <= r_svc ** 2) & (x >= xc)
    chamber = (x - xc) ** 2 + (y - yc) ** 2 + (z - zc) ** 2 <= r_chamber ** 2
    outlets = (x - xc) ** 2 + (z - zc) ** 2 <= r_out ** 2
    fluid = ivc | svc | chamber | outlets
    m = np.where(fluid, STUDY_FLUID, STUDY_WALL).astype(np.uint8)
    m[:, :, 0][fluid[:, :, 0]] = STUDY_IVC
    m[:, :, -1][fluid[:, :, -1]] = STUDY_SVC
    m[:, 0, :][fluid[:, 0, :]] = STUDY_OUT_YMIN
    m[:, -1, :][fluid[:, -1, :]] = STUDY_OUT_YMAX
    return m


def pipe_map(nx: int = 96, ny: int = 32, nz: int = 32, radius: float = 12.0):
    """Straight circular pipe along x as solver map labels plus its inlet profile.

    Wall iff (y-c)^2+(z-c)^2 > r^2 with c=(n-1)/2; x = 0 is a prescribed-velocity inlet
    (INFLOW_EQ) with the parabolic profile u_x = 1 - r^2/R^2 (scaled by the peak velocity
    at run time); x = nx-1 is a rho = 1 outlet (OUTFLOW_RIGHT_EQ).  Returns (map [z][y][x]
    uint8, profile [n_inflow_eq][3] float64 in cell order for unit peak velocity).
    """
    x, y, z = _grid(nx, ny, nz)
    yc, zc = (ny - 1) / 2.0, (nz - 1) / 2.0
    r2 = (y - yc) ** 2 + (z - zc) ** 2
    inside = r2 <= radius ** 2
    m = np.where(inside, MAP_FLUID, MAP_WALL).astype(np.uint8)
    m[:, :, 0][inside[:, :, 0]] = MAP_INFLOW_EQ
    m[:, :, -1][inside[:, :, -1]] = MAP_OUTFLOW_RIGHT_EQ
    sel = (m == MAP_INFLOW_EQ).reshape(-1)
    prof = np.zeros((int(sel.sum()), 3))
    prof[:, 0] = (1.0 - r2 / radius ** 2).reshape(-1)[sel]
    return m, prof


def dense_box_map(nx: int = 768, ny: int = 576, nz: int = 480):
    """Dense fluid box, periodic in y and z, velocity inlet at x = 0 and rho = 1 outlet at
    x = nx-1.  Returns (map [z][y][x] uint8, unit profile [n_inflow_eq][3] along +x)."""
    m = np.full((nz, ny, nx), MAP_PERIODIC, dtype=np.uint8)
    m[:, :, 0] = MAP_INFLOW_EQ
    m[:, :, -1] = MAP_OUTFLOW_RIGHT_EQ
    prof = np.zeros((ny * nz, 3))
    prof[:, 0] = 1.0
    return m, prof


def expand_profile(map_: np.ndarray, prof: np.ndarray) -> np.ndarray:
    """Compact per-INFLOW_EQ-cell profile [n][3] -> dense [3][z][y][x] (small lattices)."""
    m = np.asarray(map_)
    sel = (m == MAP_INFLOW_EQ).reshape(-1)
    out = np.zeros((3, m.size))
    out[:, sel] = np.asarray(prof, dtype=np.float64).T
    return out.reshape((3,) + m.shape)


def label_counts(map_: np.ndarray) -> dict:
    m = np.asarray(map_)
    return {int(k): int(v) for k, v in zip(*np.unique(m, return_counts=True))}

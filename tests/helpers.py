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

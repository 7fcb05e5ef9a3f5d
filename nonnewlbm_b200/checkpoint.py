"""Checkpoint and resume of a run, with the semantics of State::saveState / loadState
(solver/lbm3d/state.hpp:1552-1758, called from the time loop at solver/lbm3d/core.h:1511-1602)
and the reference's flag files (state.hpp:88-135).

Files under ``results_<id>/current_state/`` (one rank, suffix ``_rank000`` as in
state.hpp:1482):

- ``config``: text, one value per line: iterations, global X, Y, Z, local X, Y, Z, physFinalTime
  (state.hpp:1572);
- ``cnt_<c>``: text, count and period of each counter of state.h:72 (``MAX_COUNTER`` = 11);
- ``df_0``: the canonical populations after the last step, float64 [27][nz][ny][nx] (the
  layout of nnlbm_export_df; the reference dumps its own df arrays, state.hpp:1605-1613);
- ``map``: the solver labels, uint8 [nz][ny][nx];
- ``macro``: every macro field, float64 [13][nz][ny][nx];
- ``stats`` and ``stats_count``: the mean/rms sums, float64 [6][nz][ny][nx], and how many steps
  they hold (the reference keeps them inside its macro array).

Flags in ``results_<id>/``: ``loadstate`` present at start resumes from the saved state (it
stays, so a restarted job resumes again); ``savestate`` present when the save counter fires
saves, then is deleted and ``savestate_done`` gets a time stamp; reaching the wall time saves
unconditionally and creates ``loadstate``.
"""
from __future__ import annotations

import os
import shutil
import time
from pathlib import Path

import numpy as np

# counters of state.h:72, in order
STAT_RESET, STAT2_RESET, PRINT, VTK1D, VTK2D, VTK3D, PROBE1, PROBE2, PROBE3, SAVESTATE, VTK3DCUT = range(11)
MAX_COUNTER = 11
STATE_DIR = "current_state"


def _name(d: Path, stem: str) -> Path:
    return Path(d) / f"{stem}_rank000"


# -- flag files (state.hpp:88-135) ------------------------------------------------------------
def flag_create(results: Path, flag: str) -> None:
    """Append a time stamp to the flag file, creating it."""
    results = Path(results)
    results.mkdir(parents=True, exist_ok=True)
    with open(results / flag, "a") as f:
        f.write(time.strftime("%Y-%m-%d %H:%M:%S") + "\n")


def flag_delete(results: Path, flag: str) -> None:
    p = Path(results) / flag
    if p.exists():
        p.unlink()


def flag_exists(results: Path, flag: str) -> bool:
    return (Path(results) / flag).exists()


# -- the state files (state.hpp:1552-1721) ----------------------------------------------------
def _write(path: Path, data) -> None:
    """One state file, flushed to the disk before it is closed."""
    with open(path, "wb") as f:
        if isinstance(data, np.ndarray):
            data.tofile(f)
        else:
            f.write(data.encode())
        f.flush()
        os.fsync(f.fileno())


def save_state(results: Path, lat, iterations: int, final_time: float, counters: dict, labels: np.ndarray,
               ic: int = 0) -> Path:
    """Write the state of case ic of `lat` (a Lattice) into results/current_state/.
    `counters` maps counter index -> (count, period); missing counters are saved as (0, -1).

    The files go to a sibling directory first and replace current_state/ only once all of
    them are on the disk (the reference stages a save through a .tmp copy for the same
    reason, state.hpp:1558-1572), so a job killed in the middle of a save leaves the previous
    complete state behind; a caller creates the loadstate flag after this returns."""
    results = Path(results)
    d = results / STATE_DIR
    tmp = results / (STATE_DIR + ".tmp")
    old = results / (STATE_DIR + ".old")
    for p in (tmp, old):
        if p.exists():
            shutil.rmtree(p)
    tmp.mkdir(parents=True)
    nz, ny, nx = lat.shape(ic)
    _write(_name(tmp, "config"),
           "".join(f"{v:d}\n" for v in (int(iterations), nx, ny, nz, nx, ny, nz)) + f"{float(final_time):e}\n")
    for c in range(MAX_COUNTER):
        count, period = counters.get(c, (0, -1.0))
        _write(_name(tmp, f"cnt_{c}"), f"{int(count):d}\n{float(period):e}\n")
    _write(_name(tmp, "df_0"), lat.export_df(ic).astype(np.float64))
    _write(_name(tmp, "map"), np.ascontiguousarray(labels, dtype=np.uint8))
    _write(_name(tmp, "macro"), lat.macro_all(ic).astype(np.float64))
    sums, n = lat.stats(ic)
    _write(_name(tmp, "stats"), sums.astype(np.float64))
    _write(_name(tmp, "stats_count"), f"{int(n):d}\n")
    # swap: the previous state steps aside, the new one takes its name, the old one goes
    if d.exists():
        os.rename(d, old)
    os.rename(tmp, d)
    if old.exists():
        shutil.rmtree(old)
    return d


def _state_dir(results: Path) -> Path:
    """current_state/, or the previous complete state that a save interrupted between its two
    renames left under current_state.old/."""
    d = Path(results) / STATE_DIR
    old = Path(results) / (STATE_DIR + ".old")
    return old if not d.exists() and old.exists() else d


def read_config(results: Path) -> dict:
    d = _state_dir(results)
    v = _name(d, "config").read_text().split()
    cfg = {"iterations": int(v[0]), "global": tuple(int(x) for x in v[1:4]), "local": tuple(int(x) for x in v[4:7]),
           "final_time": float(v[7])}
    cnt = {}
    for c in range(MAX_COUNTER):
        p = _name(d, f"cnt_{c}")
        if p.exists():
            w = p.read_text().split()
            cnt[c] = (int(w[0]), float(w[1]))
    cfg["counters"] = cnt
    return cfg


def load_state(results: Path, lat, labels: np.ndarray | None = None, ic: int = 0) -> dict:
    """Read results/current_state/ into case ic of `lat`: populations, macro fields and mean/rms
    sums.  Returns the config (iterations, sizes, final time, counters, stats_count).  The
    saved box must match the lattice, and the saved labels the given ones."""
    d = _state_dir(results)
    cfg = read_config(results)
    nz, ny, nx = lat.shape(ic)
    if cfg["global"] != (nx, ny, nz):
        raise ValueError(f"saved state is {cfg['global']}, the lattice is {(nx, ny, nz)}")
    n = nx * ny * nz
    if labels is not None:
        saved = np.fromfile(_name(d, "map"), dtype=np.uint8)
        if saved.size != n or not np.array_equal(saved, np.asarray(labels, dtype=np.uint8).reshape(-1)):
            raise ValueError("saved labels differ from the lattice's")
    lat.import_df(np.fromfile(_name(d, "df_0"), dtype=np.float64), ic)
    lat.import_macro(np.fromfile(_name(d, "macro"), dtype=np.float64), ic)
    cfg["stats_count"] = int(_name(d, "stats_count").read_text().split()[0])
    lat.import_stats(np.fromfile(_name(d, "stats"), dtype=np.float64), cfg["stats_count"], ic)
    return cfg

"""Checkpoint files and flag semantics of State::saveState / loadState (state.hpp:88-135,
1552-1758) on the host, with a stand-in lattice (no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from nonnewlbm_b200 import checkpoint as C
from nonnewlbm_b200.tcpc import Counter, TcpcOptions, TcpcRun


class FakeLattice:
    """The Lattice methods the checkpoint uses, over numpy arrays."""

    def __init__(self, shape, seed=0):
        self._shape = shape  # (nz, ny, nx)
        rng = np.random.default_rng(seed)
        self.df = rng.random((27,) + shape)
        self.mac = rng.random((13,) + shape)
        self.sums = rng.random((6,) + shape)
        self.n = int(rng.integers(1, 100))

    def shape(self, ic=0):
        return self._shape

    def export_df(self, ic=0):
        return self.df.copy()

    def macro_all(self, ic=0):
        return self.mac.copy()

    def stats(self, ic=0):
        return self.sums.copy(), self.n

    def import_df(self, a, ic=0):
        self.df = np.asarray(a, dtype=np.float64).reshape(self.df.shape).copy()

    def import_macro(self, a, ic=0):
        self.mac = np.asarray(a, dtype=np.float64).reshape(self.mac.shape).copy()

    def import_stats(self, a, n, ic=0):
        self.sums = np.asarray(a, dtype=np.float64).reshape(self.sums.shape).copy()
        self.n = int(n)


def test_files_and_roundtrip(tmp_path):
    src, dst = FakeLattice((3, 4, 5), seed=1), FakeLattice((3, 4, 5), seed=2)
    labels = np.arange(60, dtype=np.uint8).reshape(3, 4, 5) % 9
    d = C.save_state(tmp_path, src, 1234, 2.5, {C.VTK3D: (7, 0.1), C.PRINT: (3, 0.05)}, labels)
    assert d == tmp_path / "current_state"
    names = {p.name for p in d.iterdir()}
    assert {"config_rank000", "df_0_rank000", "map_rank000", "macro_rank000", "stats_rank000",
            "stats_count_rank000"} <= names
    assert {f"cnt_{c}_rank000" for c in range(C.MAX_COUNTER)} <= names
    # config: iterations, global X Y Z, local X Y Z, physFinalTime, one per line (state.hpp:1572)
    assert (d / "config_rank000").read_text().splitlines() == ["1234", "5", "4", "3", "5", "4", "3", "2.500000e+00"]
    assert (d / "cnt_5_rank000").read_text().split() == ["7", "1.000000e-01"]
    assert (d / "cnt_9_rank000").read_text().split() == ["0", "-1.000000e+00"]
    cfg = C.load_state(tmp_path, dst, labels=labels)
    assert cfg["iterations"] == 1234 and cfg["final_time"] == 2.5 and cfg["global"] == (5, 4, 3)
    assert cfg["counters"][C.VTK3D] == (7, 0.1) and cfg["stats_count"] == src.n
    assert np.array_equal(dst.df, src.df) and np.array_equal(dst.mac, src.mac)
    assert np.array_equal(dst.sums, src.sums) and dst.n == src.n


def test_load_rejects_another_box_or_map(tmp_path):
    src = FakeLattice((3, 4, 5))
    labels = np.zeros((3, 4, 5), dtype=np.uint8)
    C.save_state(tmp_path, src, 10, 1.0, {}, labels)
    with pytest.raises(ValueError):
        C.load_state(tmp_path, FakeLattice((3, 4, 6)))
    with pytest.raises(ValueError):
        C.load_state(tmp_path, FakeLattice((3, 4, 5)), labels=labels + 1)


def _run(tmp_path):
    r = TcpcRun.__new__(TcpcRun)
    r.o = TcpcOptions(final_time=3.0)
    r.dir = tmp_path
    r.lat = FakeLattice((3, 4, 5))
    r.map = np.zeros((3, 4, 5), dtype=np.uint8)
    r.iterations, r.prev_iter = 40, 0
    r.log = lambda msg: None
    cnt = {"print": Counter(0.1), "stat": Counter(-1.0), "vtk": Counter(0.5), "save": Counter(60.0)}
    return r, cnt


def test_driver_flags(tmp_path):
    r, cnt = _run(tmp_path)
    # the save counter fires, but without the `savestate` flag nothing is written (state.hpp:1727)
    assert not r.save_state(cnt) and not (tmp_path / "current_state").exists()
    C.flag_create(tmp_path, "savestate")
    cnt["vtk"].count = 4
    assert r.save_state(cnt)
    assert not C.flag_exists(tmp_path, "savestate") and C.flag_exists(tmp_path, "savestate_done")
    assert not C.flag_exists(tmp_path, "loadstate")
    # the wall-time save is forced and leaves `loadstate` for the next start
    r.iterations = 55
    assert r.save_state(cnt, forced=True) and C.flag_exists(tmp_path, "loadstate")
    # a new run resumes the iteration, the counters and the statistics window
    r2, cnt2 = _run(tmp_path)
    r2.iterations = 0
    r2.load_state(cnt2)
    assert r2.iterations == 55 and cnt2["vtk"].count == 4 and r2.prev_iter == 55 - r.lat.n
    assert np.array_equal(r2.lat.df, r.lat.df)


def test_interrupted_save_keeps_the_previous_state(tmp_path):
    """A save that dies before its files are complete leaves the last complete state in
    place (files go to a sibling directory and are swapped in at the end)."""
    labels = np.arange(60, dtype=np.uint8).reshape(3, 4, 5) % 9
    first = FakeLattice((3, 4, 5), seed=1)
    C.save_state(tmp_path, first, 10, 1.0, {}, labels)

    class Killed(FakeLattice):
        def macro_all(self, ic=0):
            raise RuntimeError("job killed")

    with pytest.raises(RuntimeError):
        C.save_state(tmp_path, Killed((3, 4, 5), seed=2), 20, 1.0, {}, labels)
    dst = FakeLattice((3, 4, 5), seed=3)
    cfg = C.load_state(tmp_path, dst, labels)
    assert cfg["iterations"] == 10 and np.array_equal(dst.df, first.df)
    # killed between the two renames of the swap: the previous state is under .old
    (tmp_path / "current_state").rename(tmp_path / "current_state.old")
    cfg = C.load_state(tmp_path, dst, labels)
    assert cfg["iterations"] == 10
    # the next complete save takes over and clears the leftovers
    second = FakeLattice((3, 4, 5), seed=4)
    C.save_state(tmp_path, second, 30, 1.0, {}, labels)
    assert not (tmp_path / "current_state.old").exists() and not (tmp_path / "current_state.tmp").exists()
    cfg = C.load_state(tmp_path, dst, labels)
    assert cfg["iterations"] == 30 and np.array_equal(dst.df, second.df)

"""Host-side lattice object over the C ABI (numpy in, numpy out).

``Lattice`` is the Python face of the reference's policy composition (LBM_TYPE x
STREAMING x MACRO x LBM_DATA x LBM_BC, solver/sim_tcpc/sim_tcpc.cu:431-438): a collision
selector string, an equilibrium, a Carreau-Yasuda mode, a storage type and a label map.
One ``Lattice`` owns one or more cases of a single library context.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import capi


@dataclass
class CaseSpec:
    shape: tuple            # (nx, ny, nz)
    collision: str = "CUM"
    dtype: str = "f32"
    equilibrium: str = "inv_cum_ref"
    cy_mode: str = "none"
    nu: float = 1.0 / 30.0
    cy: tuple = (0.0, 0.0, 2.0, 1.0)   # nu0, lambda, a, n in lattice units
    force: tuple = (0.0, 0.0, 0.0)
    stats_f64: bool = True
    storage_scale: float = 0.0
    bounce_back: str = "fullway"       # fullway (wall nodes, the reference) | halfway

    def desc(self) -> capi.CaseDesc:
        nx, ny, nz = self.shape
        col = self.collision.upper()
        if col not in capi.COLLISIONS:
            raise ValueError(f"unknown collision {self.collision!r}; choose one of {capi.COLLISIONS}")
        return capi.CaseDesc(int(nx), int(ny), int(nz), capi.DTYPES[self.dtype.lower()], capi.COLLISIONS.index(col),
                             capi.EQUILIBRIA[self.equilibrium.lower()], capi.CY_MODES[self.cy_mode.lower()],
                             int(bool(self.stats_f64)), float(self.nu), float(self.cy[0]), float(self.cy[1]),
                             float(self.cy[2]), float(self.cy[3]), float(self.force[0]), float(self.force[1]),
                             float(self.force[2]), float(self.storage_scale),
                             {"fullway": 0, "halfway": 1}[self.bounce_back.lower()], 0)


class Lattice:
    """One library context holding ``len(specs)`` cases on CUDA device ``device``."""

    def __init__(self, specs, device: int = 0):
        if isinstance(specs, CaseSpec):
            specs = [specs]
        self.specs = list(specs)
        arr = (capi.CaseDesc * len(self.specs))(*[s.desc() for s in self.specs])
        h = ctypes.c_void_p()
        rc = capi.lib().nnlbm_create(arr, len(self.specs), int(device), ctypes.byref(h))
        self.h = h.value
        if rc != capi.OK:
            msg = capi.last_error(self.h) if self.h else "nnlbm_create failed"
            self.close()
            raise capi.NnlbmError(rc, msg)

    # -- lifetime ---------------------------------------------------------------------
    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            capi.lib().nnlbm_destroy(h)
        self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chk(self, rc):
        capi.check(self.h, rc)

    def shape(self, ic: int = 0):
        nx, ny, nz = self.specs[ic].shape
        return (nz, ny, nx)

    def ncells(self, ic: int = 0) -> int:
        nx, ny, nz = self.specs[ic].shape
        return nx * ny * nz

    # -- set-up -------------------------------------------------------------------------
    def set_map(self, labels: np.ndarray, ic: int = 0) -> None:
        a = np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1)
        if a.size != self.ncells(ic):
            raise ValueError(f"map has {a.size} cells, case {ic} has {self.ncells(ic)}")
        self._chk(capi.lib().nnlbm_set_map(self.h, ic, a.ctypes.data))

    def setup_tcpc(self, wall: np.ndarray, ic: int = 0) -> dict:
        a = np.ascontiguousarray(wall, dtype=np.int32).reshape(-1)
        if a.size != self.ncells(ic):
            raise ValueError("wall array size does not match the lattice")
        counts = np.zeros(10, dtype=np.int64)
        self._chk(capi.lib().nnlbm_setup_tcpc(self.h, ic, a.ctypes.data, counts.ctypes.data))
        keys = ["left_area", "right_area", "outlet5", "outlet6", "wall", "fluid", "vtk3", "vtk4", "vtk5", "vtk6"]
        return dict(zip(keys, (int(v) for v in counts)))

    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0, ic: int | None = None) -> None:
        for k in self._cases(ic):
            self._chk(capi.lib().nnlbm_init_equilibrium(self.h, k, rho, ux, uy, uz))

    def set_inflow(self, ivc_flux=0.0, svc_flux=0.0, rho_left=1.0, rho_right=1.0, rho_eq=1.0, ic: int = 0) -> None:
        self._chk(capi.lib().nnlbm_set_inflow(self.h, ic, ivc_flux, svc_flux, rho_left, rho_right, rho_eq))

    def set_inflow_profile(self, u: np.ndarray, ic: int = 0) -> None:
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        self._chk(capi.lib().nnlbm_set_inflow_profile(self.h, ic, capi.dptr(a), a.shape[0]))

    def set_schedule(self, rows: np.ndarray, ic: int = 0) -> None:
        a = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 3)
        self._chk(capi.lib().nnlbm_set_schedule(self.h, ic, capi.dptr(a), a.shape[0]))

    # -- time stepping --------------------------------------------------------------------
    def step(self, n: int = 1, stats: bool = False, macro: bool = False, reduce: bool = False, wait: bool = True,
             readback: bool = False) -> None:
        """Advance n steps.  wait=False enqueues them and returns at once (NNLBM_STEP_ASYNC);
        sync() then waits and checks the watchdog.  readback=True (with wait=False) also
        enqueues a copy of the step cursors, watchdog flags and FP64 sums for readback()."""
        flags = (capi.STEP_STATS if stats else 0) | (capi.STEP_MACRO if macro else 0) | (capi.STEP_REDUCE if reduce else 0)
        if not wait:
            flags |= capi.STEP_ASYNC
        if readback:
            flags |= capi.STEP_READBACK
        self._chk(capi.lib().nnlbm_step(self.h, int(n), flags))

    def sync(self) -> None:
        self._chk(capi.lib().nnlbm_sync(self.h))

    def step_noalloc(self, n: int = 1, stats: bool = False, macro: bool = False, reduce: bool = False) -> None:
        """nnlbm_step_noalloc: the same steps without any device allocation (the buffers the
        flags need must exist already; see include/nnlbm.h)."""
        flags = (capi.STEP_STATS if stats else 0) | (capi.STEP_MACRO if macro else 0) | (capi.STEP_REDUCE if reduce else 0)
        self._chk(capi.lib().nnlbm_step_noalloc(self.h, int(n), flags))

    def autotune(self, stats: bool = False, macro: bool = False) -> None:
        """Pick the fastest step-kernel launch shape, timing steps with these flags."""
        flags = (capi.STEP_STATS if stats else 0) | (capi.STEP_MACRO if macro else 0)
        self._chk(capi.lib().nnlbm_autotune_flags(self.h, flags))

    def set_launch(self, block: int = 256, cells_per_thread: int = 2, staged: bool = False) -> None:
        """Fix the step kernel's launch shape instead of autotuning it; `staged` picks the
        two-cell form whose warps stage their populations in shared memory (block 128)."""
        cpt = int(cells_per_thread) | (capi.LAUNCH_STAGED if staged else 0)
        self._chk(capi.lib().nnlbm_set_launch(self.h, int(block), cpt))

    def launch(self, ic: int = 0) -> dict:
        """The launch shape case ic steps with now: block size, cells a thread, staged."""
        b, c = ctypes.c_int(), ctypes.c_int()
        self._chk(capi.lib().nnlbm_get_launch(self.h, ic, ctypes.byref(b), ctypes.byref(c)))
        return {"block": b.value, "cells_per_thread": c.value & ~capi.LAUNCH_STAGED,
                "staged": bool(c.value & capi.LAUNCH_STAGED)}

    def stat_reset(self, ic: int | None = None) -> None:
        for k in self._cases(ic):
            self._chk(capi.lib().nnlbm_stat_reset(self.h, k))

    # -- results --------------------------------------------------------------------------
    def macro(self, field: int, ic: int = 0) -> np.ndarray:
        out = np.empty(self.ncells(ic))
        self._chk(capi.lib().nnlbm_get_macro(self.h, ic, int(field), capi.dptr(out)))
        return out.reshape(self.shape(ic))

    def stats(self, ic: int = 0):
        out = np.empty(6 * self.ncells(ic))
        n = ctypes.c_int64()
        self._chk(capi.lib().nnlbm_get_stats(self.h, ic, capi.dptr(out), ctypes.byref(n)))
        return out.reshape((6,) + self.shape(ic)), int(n.value)

    def export_df(self, ic: int = 0) -> np.ndarray:
        out = np.empty(27 * self.ncells(ic))
        self._chk(capi.lib().nnlbm_export_df(self.h, ic, capi.dptr(out)))
        return out.reshape((27,) + self.shape(ic))

    def import_df(self, df: np.ndarray, ic: int = 0) -> None:
        a = np.ascontiguousarray(df, dtype=np.float64).reshape(-1)
        if a.size != 27 * self.ncells(ic):
            raise ValueError("population array size does not match the lattice")
        self._chk(capi.lib().nnlbm_import_df(self.h, ic, capi.dptr(a)))

    def import_stats(self, sums: np.ndarray, n_accumulated: int, ic: int = 0) -> None:
        a = np.ascontiguousarray(sums, dtype=np.float64).reshape(-1)
        if a.size != 6 * self.ncells(ic):
            raise ValueError("mean/rms array size does not match the lattice")
        self._chk(capi.lib().nnlbm_import_stats(self.h, ic, capi.dptr(a), int(n_accumulated)))

    def macro_all(self, ic: int = 0) -> np.ndarray:
        """Every macro field, [M_N][nz][ny][nx]."""
        return np.stack([self.macro(k, ic) for k in range(capi.M_N)])

    def import_macro(self, fields: np.ndarray, ic: int = 0) -> None:
        a = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1)
        if a.size != capi.M_N * self.ncells(ic):
            raise ValueError("macro array size does not match the lattice")
        self._chk(capi.lib().nnlbm_import_macro(self.h, ic, capi.dptr(a)))

    def output_fields(self, dx: float, dt: float, density: float, nu_lbm: float, cy=None, steps_summed: int = 1,
                      wall_flags: np.ndarray | None = None, ic: int = 0) -> list:
        """The VTK output fields of case ic computed on the device (nnlbm_output_fields), as
        [(name, float32 array [z][y][x] or [3][z][y][x])] in file order.  cy: the lattice
        Carreau-Yasuda parameters (nu0, lambda, a, n) of a Carreau-Yasuda material, else None."""
        n = self.ncells(ic)
        p = np.array([dx, dt, density, nu_lbm, 0.0 if cy is None else 1.0, *(cy if cy is not None else (0, 0, 1, 1)),
                      float(steps_summed)], dtype=np.float64)
        out = np.empty(20 * n, dtype=np.float32)
        wf = None if wall_flags is None else np.ascontiguousarray(wall_flags, dtype=np.uint8).reshape(-1)
        if wf is not None and wf.size != n:
            raise ValueError("wall flags must have one byte per cell")
        self._chk(capi.lib().nnlbm_output_fields(self.h, ic, capi.dptr(p), None if wf is None else wf.ctypes.data,
                                                 out.ctypes.data))
        shape = self.shape(ic)
        fields, k = [], 0
        for name, dofs in capi.OUTPUT_FIELDS:
            a = out[k * n:(k + dofs) * n].reshape((dofs,) + shape) if dofs > 1 else out[k * n:(k + 1) * n].reshape(shape)
            fields.append((name, a))
            k += dofs
        return fields

    def readback(self) -> np.ndarray:
        """The oldest copy enqueued by step(readback=True), checked like sync(): [case][5] FP64
        sums in the layout of reduce()."""
        out = np.zeros((len(self.specs), 5))
        self._chk(capi.lib().nnlbm_readback(self.h, capi.dptr(out), len(self.specs)))
        return out

    def reduce(self, ic: int = 0) -> np.ndarray:
        out = np.zeros(5)
        self._chk(capi.lib().nnlbm_reduce(self.h, ic, capi.dptr(out)))
        return out

    def step_info(self, ic: int = 0) -> dict:
        fl, bc, la = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        by = ctypes.c_double()
        self._chk(capi.lib().nnlbm_step_info(self.h, ic, ctypes.byref(fl), ctypes.byref(bc), ctypes.byref(la),
                                             ctypes.byref(by)))
        return {"fluid_cells": fl.value, "bc_cells": bc.value, "launches_per_step": la.value,
                "bytes_per_step": by.value}

    def profile_step(self, n: int, stats: bool = False, ic: int = 0) -> dict:
        """Run n real steps as separate launches with CUDA events around each kernel; returns
        the mean device milliseconds per launch of each kernel kind."""
        ms = np.zeros(5)
        cnt = np.zeros(5, dtype=np.int64)
        self._chk(capi.lib().nnlbm_profile_step(self.h, ic, int(n), capi.STEP_STATS if stats else 0, capi.dptr(ms),
                                                cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        names = ["bc_gather", "step", "unused", "refd_velocity", "refd_stress"]
        return {k: (float(ms[i] / cnt[i]) if cnt[i] else 0.0, int(cnt[i])) for i, k in enumerate(names)}

    @property
    def stream(self) -> int:
        return capi.lib().nnlbm_stream(self.h) or 0

    def _cases(self, ic):
        return range(len(self.specs)) if ic is None else [ic]

"""FP64 CPU oracle for the fused D3Q27 stream + collide step (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` import this package, and only as the checker or the timed CPU
baseline.  The product (``nonnewlbm_b200``) never imports it.

Two libraries are wrapped:

* ``liboracle.so`` -- the plain-C restatement in ``nnlbm_oracle.c`` (always built).
* ``_ref/libnnlbm_ref.so`` -- the reference's own collision / equilibrium / streaming
  headers (``solver/lbm3d`` of buresjan/nonnewlbm) compiled unmodified behind
  ``ref_shim.cpp``.  It is built only where the reference checkout is present and is used
  to pin the restatement (``tests/golden/make_golden.py``) and as the CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libnnlbm_ref.so"
REF_FAST_PATH = HERE / "_ref" / "libnnlbm_ref_fast.so"

FLUID, WALL, PERIODIC, INFLOW_LEFT, INFLOW_RIGHT, OUTFLOW_FRONT, OUTFLOW_BACK, INFLOW_EQ, OUTFLOW_RIGHT_EQ = range(9)
COLLISIONS = ["CUM", "KBC_N1", "KBC_N2", "KBC_N3", "KBC_N4", "KBC_C1", "KBC_C2", "KBC_C3", "KBC_C4", "MRT_LES", "BGK"]
EQ_INV_CUM_REF, EQ_INV_CUM, EQ_DEFAULT, EQ_ENTROPIC = range(4)
CY_NONE, CY_REF_FD, CY_LOCAL_NEQ = range(3)
M_RHO, M_VX, M_VY, M_VZ = 0, 1, 2, 3
M_VM_PLUS_X, M_VM_MINUS_X, M_VM_Y, M_VM_Z, M_VM_XX, M_VM_YY, M_VM_ZZ = range(4, 11)
M_FX, M_FY, M_FZ = 11, 12, 13
M_S11, M_S12, M_S13, M_S22, M_S32, M_S33 = range(14, 20)

_dp = ctypes.POINTER(ctypes.c_double)


class _Desc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("collision", ctypes.c_int), ("equilibrium", ctypes.c_int), ("cy_mode", ctypes.c_int),
        ("halfway_bounce_back", ctypes.c_int),
        ("nu", ctypes.c_double), ("cy_nu0", ctypes.c_double), ("cy_lambda", ctypes.c_double),
        ("cy_a", ctypes.c_double), ("cy_n", ctypes.c_double),
        ("fx", ctypes.c_double), ("fy", ctypes.c_double), ("fz", ctypes.c_double),
    ]


def ref_dir() -> Path:
    """The reference checkout: $NNLBM_REF_DIR, else a checkout named ``reference`` beside
    this repository."""
    env = os.environ.get("NNLBM_REF_DIR")
    return Path(env) if env else HERE.parents[1] / "reference"


def build(ref: bool | None = None) -> None:
    """Build liboracle.so, and the reference libraries when the checkout exists."""
    subprocess.check_call(["make", "-s", "-C", str(HERE), "all"])
    rdir = ref_dir()
    if ref is None:
        ref = (rdir / "solver" / "lbm3d" / "core.h").exists()
    if ref:
        subprocess.check_call(["make", "-s", "-C", str(HERE), "ref", f"NNLBM_REF_DIR={rdir}"])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build(ref=False)
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(_Desc)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_map.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_get_map.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_setup_tcpc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_init_equilibrium.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4
        L.orc_set_inflow.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 5
        L.orc_set_inflow_profile.argtypes = [ctypes.c_void_p, _dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_get_df.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_df.argtypes = [ctypes.c_void_p, _dp]
        L.orc_get_macro.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_set_macro.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_stat_reset.argtypes = [ctypes.c_void_p]
        L.orc_reduce.argtypes = [ctypes.c_void_p, _dp]
        L.orc_iterations.restype = ctypes.c_int64
        L.orc_iterations.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_feq.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [_dp]
        L.orc_density_velocity.argtypes = [_dp] + [ctypes.c_double] * 3 + [_dp]
        L.orc_collide.argtypes = [ctypes.c_int, ctypes.c_double, _dp] + [ctypes.c_double] * 7
        L.orc_local_nu.restype = ctypes.c_double
        L.orc_local_nu.argtypes = [_dp] + [ctypes.c_double] * 9 + [_dp]
        _lib = L
    return _lib


def feq(eq: int, rho: float, ux: float, uy: float, uz: float) -> np.ndarray:
    f = np.zeros(27)
    lib().orc_feq(eq, rho, ux, uy, uz, _ptr(f))
    return f


def density_velocity(f: np.ndarray, fx=0.0, fy=0.0, fz=0.0) -> np.ndarray:
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(4)
    lib().orc_density_velocity(_ptr(f), fx, fy, fz, _ptr(out))
    return out


def collide(col: int, nu: float, f: np.ndarray, rho, ux, uy, uz, fx=0.0, fy=0.0, fz=0.0) -> np.ndarray:
    g = np.array(f, dtype=np.float64)
    lib().orc_collide(col, nu, _ptr(g), rho, ux, uy, uz, fx, fy, fz)
    return g


def local_nu(f, rho, ux, uy, uz, nu_inf, nu0, lam, a, n):
    f = np.ascontiguousarray(f, dtype=np.float64)
    S = np.zeros(6)
    nu = lib().orc_local_nu(_ptr(f), rho, ux, uy, uz, nu_inf, nu0, lam, a, n, _ptr(S))
    return nu, S


class Oracle:
    """One lattice of the C oracle; the interface mirrors ``nonnewlbm_b200.Lattice``."""

    def __init__(self, nx, ny, nz, collision=0, equilibrium=EQ_INV_CUM_REF, cy_mode=CY_NONE,
                 nu=1.0 / 30.0, cy=(0.0, 0.0, 2.0, 1.0), force=(0.0, 0.0, 0.0), halfway=False):
        d = _Desc(nx, ny, nz, collision, equilibrium, cy_mode, int(halfway), nu, cy[0], cy[1], cy[2], cy[3],
                  force[0], force[1], force[2])
        self.h = lib().orc_create(ctypes.byref(d))
        if not self.h:
            raise ValueError("oracle lattice needs every dimension >= 3")
        self.shape = (nz, ny, nx)
        self.N = nx * ny * nz

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def set_map(self, labels: np.ndarray) -> None:
        a = np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1)
        assert a.size == self.N
        if lib().orc_set_map(self.h, a.ctypes.data) != 0:
            raise ValueError("invalid label")

    def get_map(self) -> np.ndarray:
        a = np.zeros(self.N, dtype=np.uint8)
        lib().orc_get_map(self.h, a.ctypes.data)
        return a.reshape(self.shape)

    def setup_tcpc(self, wall: np.ndarray):
        a = np.ascontiguousarray(wall, dtype=np.int32).reshape(-1)
        counts = np.zeros(10, dtype=np.int64)
        rc = lib().orc_setup_tcpc(self.h, a.ctypes.data, counts.ctypes.data)
        return rc, counts

    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        lib().orc_init_equilibrium(self.h, rho, ux, uy, uz)

    def set_inflow(self, ivc_flux=0.0, svc_flux=0.0, rho_left=1.0, rho_right=1.0, rho_eq=1.0):
        lib().orc_set_inflow(self.h, ivc_flux, svc_flux, rho_left, rho_right, rho_eq)

    def set_inflow_profile(self, u3: np.ndarray):
        a = np.ascontiguousarray(u3, dtype=np.float64).reshape(-1)
        assert a.size == 3 * self.N
        lib().orc_set_inflow_profile(self.h, _ptr(a))

    def step(self, n=1, accumulate_stats=True):
        for _ in range(n):
            lib().orc_step(self.h, int(bool(accumulate_stats)))

    def get_df(self) -> np.ndarray:
        a = np.zeros(27 * self.N)
        lib().orc_get_df(self.h, _ptr(a))
        return a.reshape((27,) + self.shape)

    def set_df(self, df: np.ndarray):
        a = np.ascontiguousarray(df, dtype=np.float64).reshape(-1)
        lib().orc_set_df(self.h, _ptr(a))

    def get_macro(self, field: int) -> np.ndarray:
        a = np.zeros(self.N)
        lib().orc_get_macro(self.h, field, _ptr(a))
        return a.reshape(self.shape)

    def set_macro(self, field: int, v: np.ndarray):
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        lib().orc_set_macro(self.h, field, _ptr(a))

    def stat_reset(self):
        lib().orc_stat_reset(self.h)

    def reduce(self) -> np.ndarray:
        out = np.zeros(5)
        lib().orc_reduce(self.h, _ptr(out))
        return out

    @property
    def iterations(self) -> int:
        return int(lib().orc_iterations(self.h))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ------------------------------------------------------------------------------------
# the reference headers behind ref_shim.cpp
# ------------------------------------------------------------------------------------
_ref = {}


def ref_available(fast: bool = False) -> bool:
    return (REF_FAST_PATH if fast else REF_PATH).exists()


def ref_lib(fast: bool = False):
    key = "fast" if fast else "parity"
    if key not in _ref:
        path = REF_FAST_PATH if fast else REF_PATH
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference checkout)")
        L = ctypes.CDLL(str(path))
        L.ref_feq.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + [_dp]
        L.ref_density_velocity.argtypes = [ctypes.c_int, _dp] + [ctypes.c_double] * 3 + [_dp]
        L.ref_collide.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp] + [ctypes.c_double] * 7
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_int] * 6 + [ctypes.c_double] * 4
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_set_map.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.ref_set_inflow.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 5
        L.ref_set_inflow_profile.argtypes = [ctypes.c_void_p, _dp]
        L.ref_init.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 4
        L.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_get_df.argtypes = [ctypes.c_void_p, _dp]
        L.ref_get_macro.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.ref_set_cy.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 4
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        _ref[key] = L
    return _ref[key]


def ref_feq(eq, rho, ux, uy, uz, prec=8):
    f = np.zeros(27)
    ref_lib().ref_feq(prec, eq, rho, ux, uy, uz, _ptr(f))
    return f


def ref_density_velocity(f, fx=0.0, fy=0.0, fz=0.0, prec=8):
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(4)
    ref_lib().ref_density_velocity(prec, _ptr(f), fx, fy, fz, _ptr(out))
    return out


def ref_collide(col, nu, f, rho, ux, uy, uz, fx=0.0, fy=0.0, fz=0.0, prec=8):
    g = np.array(f, dtype=np.float64)
    ref_lib().ref_collide(prec, col, nu, _ptr(g), rho, ux, uy, uz, fx, fy, fz)
    return g


class RefLattice:
    """The reference's own step kernels (solver/lbm3d/core.h, built by ref_shim.cpp) on one
    rank: LBMKernel alone (cy_mode CY_NONE, the deployed single-rank step) or, with
    CY_REF_FD, the velocity / strain / step phases of the multi-rank step.  Macro fields
    are numbered as in the C oracle (M_RHO ... M_S33)."""

    def __init__(self, nx, ny, nz, collision=0, equilibrium=EQ_INV_CUM_REF, nu=1.0 / 30.0,
                 force=(0.0, 0.0, 0.0), prec=8, fast=False, cy_mode=CY_NONE, cy=(0.0, 0.0, 2.0, 1.0)):
        self.L = ref_lib(fast)
        self.h = self.L.ref_create(prec, nx, ny, nz, collision, equilibrium, nu, *force)
        if not self.h:
            raise ValueError("bad reference lattice parameters")
        if cy_mode != CY_NONE and self.L.ref_set_cy(self.h, cy_mode, *cy) != 0:
            raise ValueError("the reference has no Carreau-Yasuda mode %d" % cy_mode)
        self.shape = (nz, ny, nx)
        self.N = nx * ny * nz

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.ref_destroy(h)
            self.h = None

    def set_map(self, labels):
        a = np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1)
        self.L.ref_set_map(self.h, a.ctypes.data)

    def set_inflow(self, ivc_flux=0.0, svc_flux=0.0, rho_left=1.0, rho_right=1.0, rho_eq=1.0):
        self.L.ref_set_inflow(self.h, ivc_flux, svc_flux, rho_left, rho_right, rho_eq)

    def set_inflow_profile(self, u3):
        a = np.ascontiguousarray(u3, dtype=np.float64).reshape(-1)
        self._prof = a
        self.L.ref_set_inflow_profile(self.h, _ptr(a))

    def init_equilibrium(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self.L.ref_init(self.h, rho, ux, uy, uz)

    def step(self, n=1, accumulate_stats=True):
        for _ in range(n):
            self.L.ref_step(self.h, int(bool(accumulate_stats)))

    def get_df(self):
        a = np.zeros(27 * self.N)
        self.L.ref_get_df(self.h, _ptr(a))
        return a.reshape((27,) + self.shape)

    def get_macro(self, field):
        a = np.zeros(self.N)
        if self.L.ref_get_macro(self.h, field, _ptr(a)) != 0:
            raise ValueError(f"bad macro field {field}")
        return a.reshape(self.shape)

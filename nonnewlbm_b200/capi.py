"""ctypes binding of libnnlbm.so (the C ABI declared in include/nnlbm.h).

The library is built in-tree by ``nonnewlbm_b200.build``.  Loading fails loudly when it is
missing: there is no CPU fallback for the step.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libnnlbm.so"

OK, ERR_ARG, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_OOM, ERR_AREA = 0, -1, -2, -3, -4, -5, -6
F64, F32, F16, BF16 = 0, 1, 2, 3
DTYPES = {"f64": F64, "fp64": F64, "float64": F64, "f32": F32, "fp32": F32, "float32": F32,
          "f16": F16, "fp16": F16, "float16": F16, "bf16": BF16, "bfloat16": BF16}
COLLISIONS = ["CUM", "KBC_N1", "KBC_N2", "KBC_N3", "KBC_N4", "KBC_C1", "KBC_C2", "KBC_C3", "KBC_C4", "MRT_LES", "BGK"]
EQ_INV_CUM_REF, EQ_INV_CUM, EQ_DEFAULT, EQ_ENTROPIC = 0, 1, 2, 3
EQUILIBRIA = {"inv_cum_ref": 0, "inv_cum": 1, "default": 2, "entropic": 3}
CY_NONE, CY_REF_FD, CY_LOCAL_NEQ = 0, 1, 2
CY_MODES = {"none": 0, "ref-fd": 1, "ref_fd": 1, "local-neq": 2, "local_neq": 2}
STEP_STATS, STEP_MACRO, STEP_REDUCE, STEP_ASYNC, STEP_READBACK = 1, 2, 4, 8, 16
READBACK_SLOTS = 4
LAUNCH_STAGED = 16  # OR into cells_per_thread: the staged two-cell form
M_RHO, M_VX, M_VY, M_VZ, M_FX, M_FY, M_FZ, M_S11, M_S12, M_S13, M_S22, M_S32, M_S33 = range(13)
M_N = 13

EXPORTED = [
    "nnlbm_create", "nnlbm_set_map", "nnlbm_setup_tcpc", "nnlbm_init_equilibrium", "nnlbm_set_inflow",
    "nnlbm_set_inflow_profile", "nnlbm_set_schedule", "nnlbm_step", "nnlbm_step_noalloc", "nnlbm_stat_reset", "nnlbm_get_macro",
    "nnlbm_get_stats", "nnlbm_export_df", "nnlbm_import_df", "nnlbm_import_stats", "nnlbm_import_macro", "nnlbm_reduce", "nnlbm_autotune", "nnlbm_autotune_flags", "nnlbm_set_launch", "nnlbm_get_launch", "nnlbm_readback", "nnlbm_step_info", "nnlbm_profile_step",
    "nnlbm_stream", "nnlbm_last_error", "nnlbm_destroy", "nnlbm_tcpc_labels", "nnlbm_sync", "nnlbm_output_fields",
]
# the VTK output fields of nnlbm_output_fields, in file order, with their components
OUTPUT_FIELDS = [("velocity", 3), ("mean_velocity", 3), ("lbm_rho", 1), ("pressure_pa", 1), ("gamma_dot", 1),
                 ("nu_phys_m2_s", 1), ("mu_phys_pa_s", 1), ("wss_proxy_pa", 1), ("turbulence_intensity", 1),
                 ("rms_velocity", 1), ("strain_diag_1_s", 3), ("strain_shear_1_s", 3)]


class CaseDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("dtype", ctypes.c_int32), ("collision", ctypes.c_int32), ("equilibrium", ctypes.c_int32),
        ("cy_mode", ctypes.c_int32), ("stats_f64", ctypes.c_int32),
        ("nu", ctypes.c_double), ("cy_nu0", ctypes.c_double), ("cy_lambda", ctypes.c_double),
        ("cy_a", ctypes.c_double), ("cy_n", ctypes.c_double),
        ("fx", ctypes.c_double), ("fy", ctypes.c_double), ("fz", ctypes.c_double),
        ("storage_scale", ctypes.c_double),
        ("bounce_back", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class NnlbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nnlbm error {code}: {msg}")
        self.code = code


_lib = None
_vp, _dp, _i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)


def lib():
    """Load libnnlbm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m nonnewlbm_b200.build` "
                                    "(the step has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        i, d = ctypes.c_int, ctypes.c_double
        L.nnlbm_create.argtypes = [ctypes.POINTER(CaseDesc), i, i, ctypes.POINTER(_vp)]
        L.nnlbm_set_map.argtypes = [_vp, i, _vp]
        L.nnlbm_setup_tcpc.argtypes = [_vp, i, _vp, _vp]
        L.nnlbm_init_equilibrium.argtypes = [_vp, i, d, d, d, d]
        L.nnlbm_set_inflow.argtypes = [_vp, i, d, d, d, d, d]
        L.nnlbm_set_inflow_profile.argtypes = [_vp, i, _dp, ctypes.c_int64]
        L.nnlbm_set_schedule.argtypes = [_vp, i, _dp, ctypes.c_int64]
        L.nnlbm_step.argtypes = [_vp, ctypes.c_int64, i]
        L.nnlbm_step_noalloc.argtypes = [_vp, ctypes.c_int64, i]
        L.nnlbm_stat_reset.argtypes = [_vp, i]
        L.nnlbm_get_macro.argtypes = [_vp, i, i, _dp]
        L.nnlbm_get_stats.argtypes = [_vp, i, _dp, _i64p]
        L.nnlbm_export_df.argtypes = [_vp, i, _dp]
        L.nnlbm_import_df.argtypes = [_vp, i, _dp]
        L.nnlbm_import_stats.argtypes = [_vp, i, _dp, ctypes.c_int64]
        L.nnlbm_import_macro.argtypes = [_vp, i, _dp]
        L.nnlbm_reduce.argtypes = [_vp, i, _dp]
        L.nnlbm_autotune.argtypes = [_vp]
        L.nnlbm_autotune_flags.argtypes = [_vp, i]
        L.nnlbm_set_launch.argtypes = [_vp, i, i]
        L.nnlbm_get_launch.argtypes = [_vp, i, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.nnlbm_readback.argtypes = [_vp, _dp, i]
        L.nnlbm_step_info.argtypes = [_vp, i, _i64p, _i64p, _i64p, _dp]
        L.nnlbm_profile_step.argtypes = [_vp, i, ctypes.c_int64, i, _dp, _i64p]
        L.nnlbm_sync.argtypes = [_vp]
        L.nnlbm_stream.argtypes = [_vp]
        L.nnlbm_stream.restype = _vp
        L.nnlbm_last_error.argtypes = [_vp, ctypes.c_char_p, ctypes.c_size_t]
        L.nnlbm_destroy.argtypes = [_vp]
        L.nnlbm_tcpc_labels.argtypes = [ctypes.c_int32] * 3 + [_vp, _vp, _vp, _vp]
        L.nnlbm_output_fields.argtypes = [_vp, i, _dp, _vp, _vp]
        _lib = L
    return _lib


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def last_error(h) -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().nnlbm_last_error(h, buf, 1024)
    return buf.value.decode(errors="replace")


def check(h, rc: int) -> None:
    if rc != OK:
        raise NnlbmError(rc, last_error(h))


def tcpc_labels(wall: np.ndarray, with_wall_flags: bool = False):
    """Host-only TCPC boundary setup (nnlbm_tcpc_labels): geometry wall array [z][y][x] ->
    (solver map, counts dict, status[, wall flags])."""
    w = np.ascontiguousarray(wall, dtype=np.int32)
    nz, ny, nx = w.shape
    m = np.zeros(w.shape, dtype=np.uint8)
    wf = np.zeros(w.shape, dtype=np.uint8)
    counts = np.zeros(10, dtype=np.int64)
    rc = lib().nnlbm_tcpc_labels(nx, ny, nz, w.ctypes.data, m.ctypes.data, wf.ctypes.data, counts.ctypes.data)
    if rc not in (OK, ERR_AREA):
        raise NnlbmError(rc, "invalid TCPC geometry")
    keys = ["left_area", "right_area", "outlet5", "outlet6", "wall", "fluid", "vtk3", "vtk4", "vtk5", "vtk6"]
    out = (m, dict(zip(keys, (int(v) for v in counts))), rc)
    return out + (wf.astype(bool),) if with_wall_flags else out

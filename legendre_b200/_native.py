"""ctypes binding of ``liblegendre_b200.so`` (declared in include/legendre_b200.h).

Importing this module loads the in-tree shared library and fails loudly if it
is missing: there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "liblegendre_b200.so"

LG_OK = 0
LG_ERR_INVALID = -1
LG_ERR_CUDA = -2
LG_ERR_NOMEM = -3
LG_ERR_TIMEOUT = -4
LG_ERR_STATE = -5
LG_ERR_DEVICE = -6

LG_F64 = 0
LG_F32 = 1
LG_RUN_GRAPH = 1

_STATUS = {
    LG_ERR_INVALID: "invalid argument",
    LG_ERR_CUDA: "CUDA error",
    LG_ERR_NOMEM: "out of device memory",
    LG_ERR_TIMEOUT: "timed out",
    LG_ERR_STATE: "invalid state",
    LG_ERR_DEVICE: "device-side error",
}


class LegendreError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, 'error')} ({status}): {message}")
        self.status = status


class ModelCParams(C.Structure):
    _fields_ = [
        ("eps4", C.c_double),
        ("lambda_", C.c_double),
        ("d_thermal", C.c_double),
        ("noise_amplitude", C.c_double),
        ("anisotropy_tol", C.c_double),
        ("flux_tol", C.c_double),
    ]


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -m legendre_b200.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    return C.CDLL(str(_LIB_PATH))


lib = _load()

_p = C.c_void_p
_i64 = C.c_int64
_u64 = C.c_uint64
_d = C.c_double
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)

_SIGS = {
    "lg_abi_version": (C.c_int, []),
    "lg_ctx_create": (C.c_int, [C.c_int, _p, C.POINTER(_p)]),
    "lg_ctx_destroy": (C.c_int, [_p]),
    "lg_last_error": (C.c_char_p, [_p]),
    "lg_sync": (C.c_int, [_p, _i64]),
    "lg_ctx_kernel_launches": (_i64, [_p]),
    "lg_grid_create_cartesian": (C.c_int, [_p, C.c_int, _pi64, _pi64, _pd, _pd, C.POINTER(C.c_int), C.POINTER(_p)]),
    "lg_grid_destroy": (C.c_int, [_p]),
    "lg_grid_num_blocks": (_i64, [_p]),
    "lg_grid_face_neighbor": (C.c_int, [_p, _i64, C.c_int, C.c_int, _pi64]),
    "lg_state_create": (C.c_int, [_p, _p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(_p)]),
    "lg_state_destroy": (C.c_int, [_p]),
    "lg_state_upload_field": (C.c_int, [_p, C.c_int, _p, _i64]),
    "lg_state_download_field": (C.c_int, [_p, C.c_int, _p, _i64]),
    "lg_state_slab": (C.c_int, [_p, _i64, C.c_int, C.POINTER(_p), _pi64]),
    "lg_state_get_time": (C.c_int, [_p, _pd, _pi64]),
    "lg_state_set_time": (C.c_int, [_p, _d, _i64]),
    "lg_fill_ghosts": (C.c_int, [_p, C.c_int]),
    "lg_heat_fe_run": (C.c_int, [_p, C.c_int, _d, _d, _i64, C.c_uint32]),
    "lg_modelc_em_run": (C.c_int, [_p, C.POINTER(ModelCParams), _d, _u64, _i64, C.c_int, C.c_uint32]),
    "lg_modelc_initialize_grains": (C.c_int, [_p, _pd, _i64, _d]),
    "lg_heat_initialize_sine_noise": (C.c_int, [_p, C.c_int, _u64, _d]),
    "lg_standard_normal": (C.c_int, [_p, C.POINTER(C.c_uint64), _i64, _pd]),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def check(status: int, ctx=None) -> None:
    """Raise LegendreError for a negative status, with the context's message."""
    if status != LG_OK:
        msg = lib.lg_last_error(ctx).decode() if ctx else ""
        raise LegendreError(status, msg)


def exported_symbols():
    """Names of the C-ABI functions this binding declares."""
    return sorted(_SIGS)

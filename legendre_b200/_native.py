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
LG_RUN_PERSISTENT = 2

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


class AmrPolicy(C.Structure):
    _fields_ = [
        ("every", C.c_int64),
        ("buffer", C.c_int64),
        ("min_width", C.c_int64),
        ("efficiency", C.c_double),
        ("threshold", C.c_double),
        ("field", C.c_int),
    ]


class ComputePeaks(C.Structure):
    _fields_ = [
        ("dfma_per_s", C.c_double),
        ("ffma_per_s", C.c_double),
        ("imad_per_s", C.c_double),
        ("alu_per_s", C.c_double),
        ("sms", C.c_int32),
        ("clock_mhz", C.c_double),
    ]


LG_MODEL_HEAT = 0
LG_MODEL_C = 1
LG_AMR_SUBCYCLING = 0
LG_AMR_GLOBAL_DT = 1


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python legendre_b200/build.py` "
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
    "lg_state_field_sum": (C.c_int, [_p, C.c_int, _pd]),
    "lg_amr_cluster": (C.c_int, [_pi64, _i64, _d, _i64, _pi64, _i64, _pi64]),
    "lg_amr_check_hierarchy": (C.c_int, [_pi64, _pi64, C.POINTER(C.c_uint32), C.c_int, _pi64, _i64, C.c_char_p,
                                         _i64]),
    "lg_state_set_time": (C.c_int, [_p, _d, _i64]),
    "lg_fill_ghosts": (C.c_int, [_p, C.c_int]),
    "lg_heat_fe_run": (C.c_int, [_p, C.c_int, _d, _d, _i64, C.c_uint32]),
    "lg_modelc_em_run": (C.c_int, [_p, C.POINTER(ModelCParams), _d, _u64, _i64, C.c_int, C.c_uint32]),
    "lg_modelc_autotune": (C.c_int, [_p, C.POINTER(ModelCParams), _d, _u64, C.c_int, C.POINTER(C.c_int), _pd]),
    "lg_modelc_initialize_grains": (C.c_int, [_p, _pd, _i64, _d]),
    "lg_modelc_set_orientations": (C.c_int, [_p, C.c_int]),
    "lg_heat_rk4_run": (C.c_int, [_p, C.c_int, _d, _d, _i64, C.c_uint32]),
    "lg_modelc_rk4_run": (C.c_int, [_p, C.POINTER(ModelCParams), _d, _i64, C.c_uint32]),
    "lg_modelc_initialize_orientations": (C.c_int, [_p, C.c_int, _pd, _i64]),
    "lg_heat_initialize_sine_noise": (C.c_int, [_p, C.c_int, _u64, _d]),
    "lg_standard_normal": (C.c_int, [_p, C.POINTER(C.c_uint64), _i64, _pd]),
    "lg_amr_sim_create": (C.c_int, [_p, _pi64, _pi64, _pd, _pd, C.POINTER(C.c_uint32), C.c_int, _pi64, _i64, C.c_int,
                                    C.POINTER(ModelCParams), _d, C.c_int, _u64, C.POINTER(AmrPolicy), C.POINTER(_p)]),
    "lg_amr_sim_destroy": (C.c_int, [_p]),
    "lg_amr_sim_info": (C.c_int, [_p, _pi64, C.POINTER(C.c_int), _pi64]),
    "lg_amr_sim_patch": (C.c_int, [_p, _i64, _pi64]),
    "lg_amr_sim_field_len": (C.c_int, [_p, _pi64]),
    "lg_amr_sim_get_field": (C.c_int, [_p, C.c_int, _pd, _i64]),
    "lg_amr_sim_set_field": (C.c_int, [_p, C.c_int, _pd, _i64]),
    "lg_amr_sim_time": (C.c_int, [_p, _pd, _pi64]),
    "lg_amr_sim_suggested_dt": (C.c_int, [_p, _pd]),
    "lg_amr_sim_step": (C.c_int, [_p, _d, _i64, C.c_uint32]),
    "lg_amr_sim_set_barrier_spin_limit": (C.c_int, [_p, _i64]),
    "lg_amr_restrict": (C.c_int, [_p, C.c_int]),
    "lg_amr_fill_ghosts": (C.c_int, [_p]),
    "lg_amr_tag_level": (C.c_int, [_p, C.c_int, C.c_int, _d, _pi64, _i64, _pi64]),
    "lg_ensemble_create": (C.c_int, [_p, _pi64, _pi64, _pd, _i64, C.POINTER(ModelCParams), _pd, C.POINTER(C.c_uint64),
                                     C.c_int, C.POINTER(_p)]),
    "lg_ensemble_destroy": (C.c_int, [_p]),
    "lg_ensemble_upload": (C.c_int, [_p, C.c_int, _pd, _i64]),
    "lg_ensemble_download": (C.c_int, [_p, C.c_int, _pd, _i64]),
    "lg_ensemble_set_time": (C.c_int, [_p, _d, _i64]),
    "lg_ensemble_get_time": (C.c_int, [_p, _pd, _pi64]),
    "lg_ensemble_run": (C.c_int, [_p, _d, _i64, C.c_uint32]),
    "lg_ensemble_value_and_grad": (C.c_int, [_p, _d, _i64, _i64, _pd, _pd, _pd, _pd, _pd]),
    "lg_ensemble_set_adjoint_kernel": (C.c_int, [_p, C.c_int]),
    "lg_modelc_value_and_grad": (C.c_int, [_p, C.POINTER(ModelCParams), _d, _u64, _i64, _i64, _pd, _pd, _pd, _pd,
                                           _pd]),
    "lg_ensemble_set_resident_budget": (C.c_int, [_p, C.c_uint64]),
    "lg_snapshot_ring_create": (C.c_int, [_p, C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(_p)]),
    "lg_snapshot_ring_destroy": (C.c_int, [_p]),
    "lg_snapshot_ring_capture": (C.c_int, [_p, _i64, _d, _i64, C.POINTER(C.c_int)]),
    "lg_snapshot_ring_poll": (C.c_int, [_p, C.c_int, C.POINTER(C.c_int), _pi64, _pd, _pi64, C.POINTER(_pd)]),
    "lg_snapshot_ring_release": (C.c_int, [_p, C.c_int]),
    "lg_snapshot_ring_stats": (C.c_int, [_p, _pi64, _pi64, _pi64]),
    "lg_cell_centers": (C.c_int, [C.c_int, _pi64, _pi64, _pd, _pd, _pd]),
    "lg_amr_tag_level_static": (C.c_int, [_p, C.c_int, C.c_int, _d, _pi64, _i64, _pi64]),
    "lg_measure_compute_peaks": (C.c_int, [_p, C.POINTER(ComputePeaks)]),
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

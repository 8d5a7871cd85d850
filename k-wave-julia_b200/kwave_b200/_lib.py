"""ctypes binding of libkwb (the C ABI declared in include/kwb.h).

The shared library is built in-tree (``make -C k-wave-julia_b200/csrc``) and loaded from this
directory.  There is no CPU fallback: if the library or a CUDA device is missing, every entry
point raises ``KWaveB200Error``.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkwb.so")

KWB_OK = 0
KWB_E_INVALID = -1
KWB_E_UNSUPPORTED = -2
KWB_E_NOMEM = -3
KWB_E_DEVICE = -4
KWB_E_TIMEOUT = -5
KWB_E_CANCELLED = -6
KWB_E_BUSY = -7
KWB_E_NOTFOUND = -8

NO_ABSORPTION, NO_DISPERSION, STOKES = 0, 1, 2

RECORD_FIELDS = ("p", "p_max", "p_min", "p_rms", "p_final", "ux", "uy", "uz",
                 "u_max", "u_rms", "u_final", "I_avg", "I_max")
REC = {name: i for i, name in enumerate(RECORD_FIELDS)}
REC_COUNT = len(RECORD_FIELDS)
SERIES_FIELDS = ("p", "ux", "uy", "uz")


class KWaveB200Error(RuntimeError):
    """An error reported by libkwb (status code + message)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[kwb {code}] {message}")
        self.code = code


class Field(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_double)), ("count", C.c_int64)]


class Signal(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_double)), ("n_rows", C.c_int64), ("n_cols", C.c_int64)]


class SensorGroup(C.Structure):
    _fields_ = [("index", C.POINTER(C.c_int64)), ("n_index", C.c_int64), ("dense", C.c_int32),
                ("cartesian", C.c_int32), ("record_mask", C.c_uint32),
                ("record_count", C.c_uint8 * REC_COUNT),
                ("directivity_angle", C.POINTER(C.c_double)), ("n_directivity_angle", C.c_int64),
                ("directivity_size", C.c_double), ("has_frequency_response", C.c_int32),
                ("frequency_center", C.c_double), ("frequency_bandwidth", C.c_double)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_int64, C.c_int64, C.POINTER(C.c_float), C.c_void_p)


class Problem(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32), ("N", C.c_int64 * 3), ("d", C.c_double * 3), ("dt", C.c_double),
        ("Nt", C.c_int64), ("pml_size", C.c_int64 * 3), ("pml_alpha", C.c_double * 3),
        ("c0", Field), ("rho0", Field), ("BonA", Field),
        ("alpha_mode", C.c_int32), ("alpha_coeff", C.c_double), ("alpha_power", C.c_double),
        ("p0", Field),
        ("p_index", C.POINTER(C.c_int64)), ("n_p_index", C.c_int64), ("p_mode", C.c_int32),
        ("p_signal", Signal),
        ("u_index", C.POINTER(C.c_int64)), ("n_u_index", C.c_int64), ("u_mode", C.c_int32),
        ("u_signal", Signal * 3),
        ("tr", Signal),
        ("n_groups", C.c_int32), ("groups", C.POINTER(SensorGroup)),
        ("progress", PROGRESS_FN), ("progress_user", C.c_void_p),
        ("row_major", C.c_int32), ("axisymmetric", C.c_int32),
        ("elastic", C.c_int32), ("cs", Field), ("has_alpha_shear", C.c_int32),
        ("alpha_coeff_shear", C.c_double),
        ("s_index", C.POINTER(C.c_int64)), ("n_s_index", C.c_int64), ("s_mode", C.c_int32),
        ("s_signal", Signal * 6),
    ]


class GroupSizes(C.Structure):
    _fields_ = [("rows", C.c_int64 * REC_COUNT), ("cols", C.c_int64 * REC_COUNT)]


class GroupOutputs(C.Structure):
    _fields_ = [("field", C.POINTER(C.c_double) * REC_COUNT)]


class Outputs(C.Structure):
    _fields_ = [("groups", C.POINTER(GroupOutputs)), ("p_final_full", C.POINTER(C.c_double))]


class KernelTimes(C.Structure):
    _fields_ = [("n", C.c_int32), ("name", (C.c_char * 32) * 16), ("total_ms", C.c_double * 16),
                ("launches", C.c_int64 * 16), ("bytes_per_launch", C.c_double * 16)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("submit_ns", C.c_int64), ("start_ns", C.c_int64),
                ("end_ns", C.c_int64), ("error", C.c_char * 256)]


class ServingStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "admitted", "completed", "failed", "cancelled",
                                          "chunks", "peak_running", "queued", "running", "running_bytes")]


EXPORTS = (
    "kwb_version", "kwb_context_create", "kwb_context_destroy", "kwb_last_error",
    "kwb_query_outputs", "kwb_solve", "kwb_sim_create", "kwb_sim_advance",
    "kwb_sim_advance_timed", "kwb_sim_steps_done", "kwb_sim_sync", "kwb_sim_read_outputs",
    "kwb_sim_read_pressure", "kwb_sim_destroy", "kwb_sim_profile", "kwb_sim_info", "kwb_sim_schedule",
)

_lib = None
_lock = threading.Lock()


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libkwb.so and declare every exported signature (raises if it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise KWaveB200Error(KWB_E_DEVICE,
                                 f"libkwb.so not found at {path}; build it with "
                                 "`make -C k-wave-julia_b200/csrc` (there is no CPU fallback)")
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.kwb_version.restype = C.c_int
        lib.kwb_version.argtypes = []
        lib.kwb_context_create.restype = C.c_int
        lib.kwb_context_create.argtypes = [C.c_int, C.POINTER(vp)]
        lib.kwb_context_destroy.restype = None
        lib.kwb_context_destroy.argtypes = [vp]
        lib.kwb_last_error.restype = C.c_char_p
        lib.kwb_last_error.argtypes = [vp]
        lib.kwb_query_outputs.restype = C.c_int
        lib.kwb_query_outputs.argtypes = [vp, C.POINTER(Problem), C.POINTER(GroupSizes), C.POINTER(C.c_int64)]
        lib.kwb_solve.restype = C.c_int
        lib.kwb_solve.argtypes = [vp, C.POINTER(Problem), C.POINTER(Outputs)]
        lib.kwb_sim_create.restype = C.c_int
        lib.kwb_sim_create.argtypes = [vp, C.POINTER(Problem), C.POINTER(vp)]
        lib.kwb_sim_advance.restype = C.c_int
        lib.kwb_sim_advance.argtypes = [vp, C.c_int64]
        lib.kwb_sim_advance_timed.restype = C.c_int
        lib.kwb_sim_advance_timed.argtypes = [vp, C.c_int64, C.POINTER(C.c_double)]
        lib.kwb_sim_steps_done.restype = C.c_int64
        lib.kwb_sim_steps_done.argtypes = [vp]
        lib.kwb_sim_sync.restype = C.c_int
        lib.kwb_sim_sync.argtypes = [vp]
        lib.kwb_sim_read_outputs.restype = C.c_int
        lib.kwb_sim_read_outputs.argtypes = [vp, C.POINTER(Outputs)]
        lib.kwb_sim_finish.restype = C.c_int
        lib.kwb_sim_finish.argtypes = [vp, C.POINTER(Outputs)]
        lib.kwb_sim_read_pressure.restype = C.c_int
        lib.kwb_sim_read_pressure.argtypes = [vp, C.POINTER(C.c_float)]
        lib.kwb_sim_destroy.restype = None
        lib.kwb_sim_destroy.argtypes = [vp]
        lib.kwb_sim_profile.restype = C.c_int
        lib.kwb_sim_profile.argtypes = [vp, C.c_int64, C.POINTER(KernelTimes)]
        lib.kwb_sim_info.restype = C.c_int
        lib.kwb_sim_info.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        lib.kwb_sim_schedule.restype = C.c_int
        lib.kwb_sim_schedule.argtypes = [vp, C.c_char_p, C.c_int64]
        lib.kwb_estimate_device_bytes.restype = C.c_int
        lib.kwb_estimate_device_bytes.argtypes = [vp, C.POINTER(Problem), C.POINTER(C.c_int64)]
        lib.kwb_serving_config.restype = C.c_int
        lib.kwb_serving_config.argtypes = [vp, C.c_int32, C.c_int32, C.c_int64]
        lib.kwb_serving_voxel_budget.restype = C.c_int
        lib.kwb_serving_voxel_budget.argtypes = [vp, C.c_int64]
        lib.kwb_submit.restype = C.c_int
        lib.kwb_submit.argtypes = [vp, C.POINTER(Problem), C.POINTER(Outputs), C.POINTER(C.c_uint64)]
        lib.kwb_poll.restype = C.c_int
        lib.kwb_poll.argtypes = [vp, C.c_uint64, C.POINTER(C.c_int32)]
        lib.kwb_wait.restype = C.c_int
        lib.kwb_wait.argtypes = [vp, C.c_uint64, C.c_int64, C.POINTER(RequestInfo)]
        lib.kwb_cancel.restype = C.c_int
        lib.kwb_cancel.argtypes = [vp, C.c_uint64]
        lib.kwb_serving_stats_get.restype = C.c_int
        lib.kwb_serving_stats_get.argtypes = [vp, C.POINTER(ServingStats)]
        _lib = lib
        return lib


def check(lib, ctx, rc: int):
    if rc != KWB_OK:
        msg = lib.kwb_last_error(ctx)
        raise KWaveB200Error(rc, msg.decode() if msg else "unknown error")
    return rc

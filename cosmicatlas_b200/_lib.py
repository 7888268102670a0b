"""ctypes binding of libcam.so (the C ABI in include/cam.h).

The library is loaded from this package directory.  There is no CPU
fallback: every entry point runs the CUDA kernels, and loading fails loudly
when the library is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcam.so")

CAM_OK, CAM_E_INVAL, CAM_E_NOMEM, CAM_E_CUDA = 0, -1, -2, -3
CAM_E_TIMEOUT, CAM_E_BUSY, CAM_E_NOTFOUND, CAM_E_UNSUPPORTED, CAM_E_NONFINITE = -4, -5, -6, -7, -8
NGP, CIC, TSC = 0, 1, 2
F32, F64 = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
INPUT_DENSITY, INPUT_DELTA, INPUT_POTENTIAL = 0, 1, 2
TWEB_FFT, TWEB_FD = 0, 1
KERNEL_SET, KERNEL_SCALE = 0, 1

_STATUS = {CAM_E_INVAL: "CAM_E_INVAL", CAM_E_NOMEM: "CAM_E_NOMEM", CAM_E_CUDA: "CAM_E_CUDA",
           CAM_E_TIMEOUT: "CAM_E_TIMEOUT", CAM_E_BUSY: "CAM_E_BUSY", CAM_E_NOTFOUND: "CAM_E_NOTFOUND",
           CAM_E_UNSUPPORTED: "CAM_E_UNSUPPORTED", CAM_E_NONFINITE: "CAM_E_NONFINITE"}


class CamError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


class Particles(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("x", ctypes.c_void_p), ("y", ctypes.c_void_p),
                ("z", ctypes.c_void_p), ("w", ctypes.c_void_p), ("mem", ctypes.c_int)]


class Grid(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64 * 3), ("L", ctypes.c_float * 3), ("d", ctypes.c_float * 3),
                ("min", ctypes.c_float * 3)]


class AssignStats(ctypes.Structure):
    _fields_ = [("n_in", ctypes.c_int64), ("n_lost", ctypes.c_int64), ("sum_mesh", ctypes.c_double)]


class PkOpts(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("mas_correction", ctypes.c_int), ("sn_correction", ctypes.c_int),
                ("input_type", ctypes.c_int), ("nbins", ctypes.c_int), ("DeltaKmin", ctypes.c_double),
                ("ndel", ctypes.c_double)]


class PkInfo(ctypes.Structure):
    _fields_ = [("n_obj", ctypes.c_double), ("shot_noise", ctypes.c_double), ("normal", ctypes.c_double),
                ("kf", ctypes.c_double)]


class TwebOpts(ctypes.Structure):
    _fields_ = [("smoothing_R", ctypes.c_float), ("lambda_th", ctypes.c_double), ("tie_band", ctypes.c_double),
                ("input_type", ctypes.c_int), ("method", ctypes.c_int)]


class TwebStats(ctypes.Structure):
    _fields_ = [("counts", ctypes.c_int64 * 4), ("ties", ctypes.c_int64), ("mean", ctypes.c_double)]


class JobDesc(ctypes.Structure):
    _fields_ = [("parts", Particles), ("grid", Grid), ("scheme", ctypes.c_int), ("precision", ctypes.c_int),
                ("pk", PkOpts), ("want_tweb", ctypes.c_int), ("tweb", TwebOpts)]


class JobResult(ctypes.Structure):
    _fields_ = [("pk", ctypes.c_void_p), ("modes", ctypes.c_void_p), ("kvector", ctypes.c_void_p),
                ("labels", ctypes.c_void_p), ("pk_info", PkInfo), ("assign", AssignStats),
                ("tweb", TwebStats)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("queued", ctypes.c_int64), ("running", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("batched_jobs", ctypes.c_int64), ("graph_replays", ctypes.c_int64),
                ("bytes_reserved", ctypes.c_size_t), ("peak_bytes_reserved", ctypes.c_size_t),
                ("budget", ctypes.c_size_t), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double)]


class AllocStats(ctypes.Structure):
    _fields_ = [("allocs", ctypes.c_int64), ("failures", ctypes.c_int64), ("bytes", ctypes.c_int64),
                ("total_ms", ctypes.c_double), ("max_ms", ctypes.c_double)]


class JobTrace(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("submit_ms", ctypes.c_double), ("start_ms", ctypes.c_double),
                ("end_ms", ctypes.c_double), ("worker", ctypes.c_int), ("batch", ctypes.c_int),
                ("status", ctypes.c_int), ("big", ctypes.c_int)]


# Exported symbols with their signatures; the non-GPU tests check every one
# of these resolves.
_P = ctypes.c_void_p
SIGNATURES = {
    "cam_version": ([], ctypes.c_char_p),
    "cam_ctx_create": ([ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_P)], ctypes.c_int),
    "cam_ctx_destroy": ([_P], ctypes.c_int),
    "cam_ctx_set_stream": ([_P, _P], ctypes.c_int),
    "cam_ctx_sync": ([_P], ctypes.c_int),
    "cam_last_error": ([_P], ctypes.c_char_p),
    "cam_kernel_launches": ([_P], ctypes.c_int64),
    "cam_pool_trim": ([ctypes.c_int], ctypes.c_int),
    "cam_alloc_stats_get": ([ctypes.POINTER(AllocStats), ctypes.c_int], ctypes.c_int),
    "cam_profile_enable": ([_P, ctypes.c_int], ctypes.c_int),
    "cam_profile_read": ([_P, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int], ctypes.c_int),
    "cam_assign": ([_P, ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int, _P,
                    ctypes.c_int, ctypes.POINTER(AssignStats)], ctypes.c_int),
    "cam_count_ngp": ([_P, ctypes.POINTER(Particles), ctypes.POINTER(Grid), _P, ctypes.c_int,
                       ctypes.POINTER(AssignStats)], ctypes.c_int),
    "cam_cell_keys": ([_P, ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.c_int, _P, ctypes.c_int],
                      ctypes.c_int),
    "cam_fft_r2c": ([_P, ctypes.c_int64, ctypes.c_int, _P, _P, ctypes.c_int], ctypes.c_int),
    "cam_fft_c2r": ([_P, ctypes.c_int64, ctypes.c_int, _P, _P, ctypes.c_int], ctypes.c_int),
    "cam_power": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PkOpts), _P, _P, _P,
                   ctypes.POINTER(PkInfo)], ctypes.c_int),
    "cam_tweb": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TwebOpts), _P, _P,
                  ctypes.c_int, ctypes.POINTER(TwebStats)], ctypes.c_int),
    "cam_power_multipoles": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PkOpts),
                              ctypes.c_int, _P, _P, _P, _P, _P, ctypes.POINTER(PkInfo)], ctypes.c_int),
    "cam_cross_power": ([_P, ctypes.POINTER(Grid), _P, _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(PkOpts),
                         ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P], ctypes.c_int),
    "cam_poisson": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.c_float, _P, ctypes.c_int],
                    ctypes.c_int),
    "cam_gradfindif": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int],
                       ctypes.c_int),
    "cam_fkp_weights": ([_P, ctypes.c_int64, _P, ctypes.c_double, _P, ctypes.c_int, ctypes.c_double, ctypes.c_int, _P,
                         ctypes.c_int, _P], ctypes.c_int),
    "cam_bam_kernel_update": ([_P, ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                               _P, ctypes.c_int, _P, ctypes.c_int, _P, _P], ctypes.c_int),
    "cam_konvolve": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_int],
                     ctypes.c_int),
    "cam_tweb_invariants": ([_P, ctypes.POINTER(Grid), _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(TwebOpts), _P,
                             _P, _P, ctypes.c_int, ctypes.POINTER(TwebStats)], ctypes.c_int),
    "cam_job_run": ([_P, ctypes.POINTER(JobDesc), ctypes.POINTER(JobResult)], ctypes.c_int),
    "cam_particles_stage": ([_P, ctypes.POINTER(Particles), ctypes.POINTER(Particles)], ctypes.c_int),
    "cam_power_noalloc": ([_P, ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_double,
                           ctypes.POINTER(PkOpts), _P, _P, _P], ctypes.c_int),
    "cam_batch_run": ([_P, ctypes.POINTER(JobDesc), ctypes.c_int, ctypes.POINTER(JobResult)], ctypes.c_int),
    "cam_server_create": ([ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)],
                          ctypes.c_int),
    "cam_server_submit": ([_P, ctypes.POINTER(JobDesc), ctypes.POINTER(JobResult), ctypes.POINTER(ctypes.c_uint64)],
                          ctypes.c_int),
    "cam_server_poll": ([_P, ctypes.c_uint64], ctypes.c_int),
    "cam_server_wait": ([_P, ctypes.c_uint64, ctypes.c_int64], ctypes.c_int),
    "cam_server_stats_get": ([_P, ctypes.POINTER(ServerStats), ctypes.c_int], ctypes.c_int),
    "cam_server_last_error": ([_P], ctypes.c_char_p),
    "cam_server_trace": ([_P, ctypes.POINTER(JobTrace), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cam_server_destroy": ([_P], ctypes.c_int),
    "cam_devloop_create": ([ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                            ctypes.POINTER(_P)],
                           ctypes.c_int),
    "cam_devloop_submit": ([_P, ctypes.POINTER(JobDesc), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "cam_devloop_wait": ([_P, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(JobDesc), ctypes.POINTER(JobResult)],
                         ctypes.c_int),
    "cam_devloop_state": ([_P, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cam_devloop_destroy": ([_P], ctypes.c_int),
    "cam_devloop_last_error": ([_P], ctypes.c_char_p),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libcam.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m cosmicatlas_b200.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.argtypes = args
            fn.restype = res
        _lib = l
    return _lib


def ptr(a) -> int | None:
    """Data pointer of a numpy array or torch tensor (None passes NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


def is_device(a) -> bool:
    return a is not None and not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)

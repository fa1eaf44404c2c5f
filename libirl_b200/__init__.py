"""libirl_b200: B200-native (sm_100a) implementation of libirl's OSEM
projector/backprojector path behind libirl's own C API.

The product is the shared library libirl_b200/libirl_b200.so (host C driver
plus CUDA kernels).  This package only locates, builds and loads it for
Python callers (tests, benchmarks); C applications link the .so directly
against include/irl.h.  There is no CPU fallback: loading fails loudly when
the library is missing and every compute call fails without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

from . import api

PKG = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(PKG, "libirl_b200.so")

_lib = None


def build(force: bool = False) -> str:
    from .build import build as _b
    return _b(force=force)


def load() -> C.CDLL:
    """Load libirl_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO):
        raise ImportError(f"{SO} is missing: run `python -m libirl_b200.build`")
    lib = api.declare_irl(C.CDLL(SO))
    _declare_irlcu(lib)
    _lib = lib
    return lib


def _declare_irlcu(lib):
    F, I, S = api.FLOAT_P, C.c_int, C.c_size_t
    lib.irlcu_error_string.restype = C.c_char_p
    lib.irlcu_error_string.argtypes = []
    lib.irlcu_init.restype = I
    lib.irlcu_init.argtypes = [C.POINTER(IrlcuGeom)]
    lib.irlcu_shutdown.restype = None
    lib.irlcu_shutdown.argtypes = []
    lib.irlcu_set_angles.restype = I
    lib.irlcu_set_angles.argtypes = [F]
    lib.irlcu_upload.restype = I
    lib.irlcu_upload.argtypes = [I, I, F, S]
    lib.irlcu_upload_now.restype = I
    lib.irlcu_upload_now.argtypes = [I, I, F, S]
    lib.irlcu_esse_expand.restype = I
    lib.irlcu_esse_expand.argtypes = [C.c_void_p, I, F]
    lib.irlcu_download.restype = I
    lib.irlcu_download.argtypes = [I, I, F, S]
    lib.irlcu_download_external.restype = I
    lib.irlcu_download_external.argtypes = [I, F]
    lib.irlcu_upload_external.restype = I
    lib.irlcu_upload_external.argtypes = [I, F, C.c_float, I]
    lib.irlcu_rotate_volume.restype = I
    lib.irlcu_rotate_volume.argtypes = [C.c_float, F, F, I, I]
    lib.irlcu_rotate_volume_noalloc.restype = I
    lib.irlcu_rotate_volume_noalloc.argtypes = [C.c_float, C.c_void_p, C.c_void_p, I, I]
    lib.irlcu_prepare_attenuation.restype = I
    lib.irlcu_prepare_attenuation.argtypes = [I]
    lib.irlcu_project.restype = I
    lib.irlcu_project.argtypes = [I, C.POINTER(C.c_int), I, C.c_float, F, I]
    lib.irlcu_stage_times.restype = I
    lib.irlcu_stage_times.argtypes = [F, I]
    lib.irl_gendrf.restype = None
    lib.irl_gendrf.argtypes = [C.c_float] * 8 + [I, I, C.POINTER(api.Drf)]
    lib.irl_compute_subsets.restype = I
    lib.irl_compute_subsets.argtypes = [I, I, C.POINTER(C.POINTER(C.c_int))]
    lib.irlcu_drf_tuning.restype = I
    lib.irlcu_drf_tuning.argtypes = [C.POINTER(C.c_float)]
    lib.irlcu_shear_tuning.restype = I
    lib.irlcu_shear_tuning.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_int)]
    lib.irlcu_shape_trials.restype = I
    lib.irlcu_shape_trials.argtypes = [I]
    lib.irlcu_iteration_graphs.restype = I
    lib.irlcu_iteration_graphs.argtypes = [I]
    lib.irlcu_mem_info.restype = I
    lib.irlcu_mem_info.argtypes = [C.POINTER(S), C.POINTER(S)]
    lib.irlcu_grids.restype = I
    lib.irlcu_grids.argtypes = [C.POINTER(C.c_int)]
    lib.irlcu_stream.restype = C.c_void_p
    lib.irlcu_stream.argtypes = []
    lib.irlcu_launch_count.restype = C.c_longlong
    lib.irlcu_launch_count.argtypes = []
    lib.irlcu_profile_enable.restype = I
    lib.irlcu_profile_enable.argtypes = [I]
    lib.irlcu_profile_read.restype = I
    lib.irlcu_profile_read.argtypes = [C.POINTER(IrlcuProfile)]
    lib.IrlOsemBegin.restype = I
    lib.IrlOsemBegin.argtypes = list(lib.IrlOsem.argtypes)
    lib.IrlOsemIterate.restype = I
    lib.IrlOsemIterate.argtypes = [I]
    lib.IrlOsemEnd.restype = I
    lib.IrlOsemEnd.argtypes = [F]
    V = C.c_void_p
    lib.irlcu_sur_create.restype = I
    lib.irlcu_sur_create.argtypes = [I, C.c_ulonglong, C.POINTER(V)]
    lib.irlcu_sur_destroy.restype = None
    lib.irlcu_sur_destroy.argtypes = [V]
    lib.irlcu_sur_nparams.restype = S
    lib.irlcu_sur_nparams.argtypes = [V]
    lib.irlcu_sur_get_weights.restype = I
    lib.irlcu_sur_get_weights.argtypes = [V, F, S]
    lib.irlcu_sur_set_weights.restype = I
    lib.irlcu_sur_set_weights.argtypes = [V, F, S]
    lib.irlcu_sur_forward.restype = I
    lib.irlcu_sur_forward.argtypes = [V, I, V, V]
    lib.irlcu_sur_test_refill_wait.restype = C.c_uint
    lib.irlcu_sur_test_refill_wait.argtypes = [C.c_uint]
    lib.irlcu_sur_gradient.restype = I
    lib.irlcu_sur_gradient.argtypes = [V, I, V, V, C.POINTER(C.c_float), F]
    lib.irlcu_sur_train_step.restype = I
    lib.irlcu_sur_train_step.argtypes = [V, I, V, V, C.c_float, C.POINTER(C.c_float)]
    lib.irlcu_sur_pairs.restype = I
    lib.irlcu_sur_pairs.argtypes = [I, C.POINTER(C.c_int), I, V, V, V]
    lib.irlcu_set_surrogate.restype = I
    lib.irlcu_set_surrogate.argtypes = [V, V]
    lib.irlcu_sur_check.restype = I
    lib.irlcu_sur_check.argtypes = [V, I, C.POINTER(C.c_int), I, F]
    lib.IrlSetScatterSurrogate.restype = I
    lib.IrlSetScatterSurrogate.argtypes = [C.c_char_p, C.c_float]
    lib.IrlGetScatterSurrogateNrmse.restype = I
    lib.IrlGetScatterSurrogateNrmse.argtypes = [F, I]
    lib.IrlOsemBatch.restype = I
    lib.IrlOsemBatch.argtypes = [I, C.POINTER(api.OsemProblem)]
    lib.irlcu_set_subsets.restype = I
    lib.irlcu_set_subsets.argtypes = [I, I, C.POINTER(C.c_int), C.c_void_p]
    lib.irlcu_osem_iteration.restype = I
    lib.irlcu_osem_iteration.argtypes = [I, I, I, I]
    lib.irlcu_ctx_detach.restype = C.c_void_p
    lib.irlcu_ctx_detach.argtypes = []
    lib.irlcu_ctx_attach.restype = I
    lib.irlcu_ctx_attach.argtypes = [C.c_void_p]


NSTAGE = 8
STAGES = ["rotate", "esse", "project", "reduce_ratio", "backproject", "unrotate_accumulate", "-", "-"]


class IrlcuProfile(C.Structure):
    """irlcu_profile (include/irlcu.h)."""

    _fields_ = [
        ("ms", C.c_double * NSTAGE),
        ("flops", C.c_double * NSTAGE),
        ("bytes", C.c_double * NSTAGE),
        ("launches", C.c_longlong * NSTAGE),
    ]


class IrlcuGeom(C.Structure):
    """irlcu_geom (include/irlcu.h)."""

    _fields_ = [
        ("n", C.c_int),
        ("nz", C.c_int),
        ("nviews", C.c_int),
        ("fast_rotate", C.c_int),
        ("max_batch", C.c_int),
    ]


def check(lib, rc):
    if rc != 0:
        raise RuntimeError(f"irlcu error {rc}: {lib.irlcu_error_string().decode(errors='replace')}")

"""ctypes binding of the C ABI declared in include/mercury_b200.h.

The shared library is built in-tree (mercury_b200/libmercury_b200.so) by
__graft_entry__.build().  There is no fallback: importing this module raises
if the library is missing, and every call that fails raises MercuryError.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmercury_b200.so")

MB_OK = 0
STATUS_NAMES = {
    0: "MB_OK",
    1: "MB_ERR_ARGUMENT",
    2: "MB_ERR_CUDA",
    3: "MB_ERR_CAPACITY",
    4: "MB_ERR_STATE",
    5: "MB_ERR_NONFINITE",
}
COMPOSITE_COUNT = 254
MODE_REF_XPBD, MODE_FORCE_LAND, MODE_FORCE_WATER = 0, 1, 2
DEVO_MAX_REPLACED = 1024
DEVO_REFERENCE_RANKS = 1


class MercuryError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class BatchDesc(ctypes.Structure):
    _fields_ = [
        ("n_robots", ctypes.c_uint32),
        ("mass_offsets", ctypes.c_void_p),
        ("pos", ctypes.c_void_p),
        ("vel", ctypes.c_void_p),
        ("mass_material", ctypes.c_void_p),
        ("spring_offsets", ctypes.c_void_p),
        ("pairs", ctypes.c_void_p),
        ("spring_material", ctypes.c_void_p),
        ("lbar", ctypes.c_void_p),
        ("face_offsets", ctypes.c_void_p),
        ("faces", ctypes.c_void_p),
    ]


class Environment(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("g", "floor_stiffness", "friction_static",
                                              "friction_kinetic", "drag", "damping", "face_drag")]


class PlanStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("threads", "springs_per_thread", "masses_per_thread",
                                               "bins", "streamed", "max_smem_bytes")] + \
               [(n, ctypes.c_uint64) for n in ("masses", "active_springs", "incidence_entries",
                                               "incidence_padding")] + \
               [(n, ctypes.c_uint32) for n in ("aligned_slices", "rank_slices", "material_slots",
                                               "max_bin_springs", "min_bin_springs",
                                               "ctas", "max_cta_springs", "min_cta_springs", "cluster",
                                               "cluster2", "split_bins0")]


class LaunchConfig(ctypes.Structure):
    _fields_ = [
        ("threads", ctypes.c_uint32),
        ("springs_per_thread", ctypes.c_uint32),
        ("masses_per_thread", ctypes.c_uint32),
        ("bins", ctypes.c_uint32),
        ("chunk", ctypes.c_uint32),
        ("use_graph", ctypes.c_uint32),
        ("streamed", ctypes.c_uint32),
        ("cluster", ctypes.c_uint32),
    ]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    lib = ctypes.CDLL(LIB_PATH)
    P, U32, I32, F32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    sigs = {
        "mb_context_create": (I32, [I32, ctypes.POINTER(P)]),
        "mb_context_destroy": (None, [P]),
        "mb_last_error": (ctypes.c_char_p, [P]),
        "mb_set_materials": (I32, [P, P]),
        "mb_set_time_step": (I32, [P, F32]),
        "mb_get_time_step": (F32, [P]),
        "mb_set_total_time": (I32, [P, F32]),
        "mb_get_total_time": (F32, [P]),
        "mb_set_mode": (I32, [P, I32]),
        "mb_get_mode": (I32, [P, ctypes.POINTER(ctypes.c_int)]),
        "mb_set_environment": (I32, [P, ctypes.POINTER(Environment)]),
        "mb_get_environment": (I32, [P, ctypes.POINTER(Environment)]),
        "mb_set_elements": (I32, [P, ctypes.POINTER(BatchDesc)]),
        "mb_set_state": (I32, [P, P, P]),
        "mb_simulate": (I32, [P, F32, I32, ctypes.POINTER(U32)]),
        "mb_run_steps": (I32, [P, U32, I32]),
        "mb_collect": (I32, [P, P, P, P]),
        "mb_centre_of_mass": (I32, [P, P]),
        "mb_robot_flags": (I32, [P, P]),
        "mb_synchronize": (I32, [P]),
        "mb_get_stream": (P, [P]),
        "mb_device_state": (I32, [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P)]),
        "mb_get_launch_config": (I32, [P, ctypes.POINTER(LaunchConfig)]),
        "mb_get_step_variant": (I32, [P, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
        "mb_get_packed_springs": (I32, [P, P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
        "mb_set_launch_config": (I32, [P, ctypes.POINTER(LaunchConfig)]),
        "mb_kernel_shapes": (U32, [ctypes.POINTER(LaunchConfig), U32]),
        "mb_plan_population": (I32, [ctypes.POINTER(BatchDesc), ctypes.POINTER(LaunchConfig), U32, U32,
                                     ctypes.POINTER(PlanStats)]),
        "mb_voxel_build": (I32, [I32, I32, I32, F32, P, ctypes.POINTER(I32), ctypes.POINTER(I32), P, P, P, P, P]),
        "mb_devo": (I32, [P, U32, ctypes.c_uint64, U32, ctypes.POINTER(U32)]),
        "mb_collect_springs": (I32, [P, P, P, P]),
        "mb_devo_profile": (I32, [P, P]),
        "mb_set_voxel_population": (I32, [P, U32, I32, I32, I32, P, F32, F32]),
        "mb_collect_mass_materials": (I32, [P, P]),
        "mb_knn_springs": (I32, [I32, U32, P, P, P, U32, P, P, P, P, ctypes.c_uint64]),
        "mb_surrogate_create": (I32, [I32, U32, ctypes.c_uint64, ctypes.POINTER(P)]),
        "mb_surrogate_destroy": (None, [P]),
        "mb_surrogate_last_error": (ctypes.c_char_p, [P]),
        "mb_surrogate_param_count": (U32, []),
        "mb_surrogate_layout": (None, [P]),
        "mb_surrogate_get_params": (I32, [P, P]),
        "mb_surrogate_set_params": (I32, [P, P]),
        "mb_surrogate_predict": (I32, [P, P, U32, P]),
        "mb_surrogate_gradients": (I32, [P, P, P, U32, P, P]),
        "mb_surrogate_train_step": (I32, [P, P, P, U32, F32, P]),
        "mb_surrogate_set_weight_decay": (I32, [P, F32]),
        "mb_surrogate_use_tcgen05": (I32, [P, I32]),
        "mb_measure_smem_bandwidth": (I32, [I32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
        "mb_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def ptr(a: np.ndarray | None) -> int | None:
    """Address of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def check(status: int, ctx=None) -> None:
    if status != MB_OK:
        msg = LIB.mb_last_error(ctx).decode() if ctx else ""
        raise MercuryError(status, msg)

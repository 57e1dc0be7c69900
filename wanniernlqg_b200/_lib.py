"""Loader for the in-tree CUDA library ``libwnlqg_b200.so`` (the C ABI of include/wnlqg_b200.h).

There is no CPU fallback: if the library is missing or cannot be loaded, every engine call
raises.  ``build()`` in :mod:`wanniernlqg_b200.build` compiles it with nvcc for sm_100a.
"""
from __future__ import annotations

import ctypes
import os

from . import _abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libwnlqg_b200.so")

# Every symbol include/wnlqg_b200.h declares.
EXPORTED_SYMBOLS = (
    "wnlqg_b200_version", "wnlqg_b200_last_error", "wnlqg_b200_device_count",
    "wnlqg_b200_model_create", "wnlqg_b200_model_destroy",
    "wnlqg_b200_plan_create", "wnlqg_b200_plan_destroy", "wnlqg_b200_plan_value_count",
    "wnlqg_b200_eval_mesh", "wnlqg_b200_eval_mesh_device", "wnlqg_b200_eval_mesh_many", "wnlqg_b200_eval_points",
    "wnlqg_b200_eval_points_weighted", "wnlqg_b200_eval_points_weighted_device", "wnlqg_b200_eval_mesh_weighted",
    "wnlqg_b200_eval_spectrum", "wnlqg_b200_plan_last_timing", "wnlqg_b200_plan_last_launch_count",
    "wnlqg_b200_spectrum_noalloc",
    "wnlqg_b200_mlp_param_count", "wnlqg_b200_mlp_create", "wnlqg_b200_mlp_destroy", "wnlqg_b200_mlp_get_params",
    "wnlqg_b200_mlp_set_params", "wnlqg_b200_mlp_forward", "wnlqg_b200_mlp_loss_grad", "wnlqg_b200_mlp_train",
    "wnlqg_b200_graph_capture_mesh_many", "wnlqg_b200_graph_capture_points_weighted", "wnlqg_b200_graph_launch",
    "wnlqg_b200_graph_status", "wnlqg_b200_graph_kernel_count", "wnlqg_b200_graph_destroy",
    "wnlqg_b200_plan_autotune", "wnlqg_b200_plan_status", "wnlqg_b200_measure_peaks",
)

_lib = None


class EngineError(RuntimeError):
    """A non-OK status from the C ABI; ``status`` holds the wnlqg_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load():
    """Load the CUDA library (raises OSError when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python -m wanniernlqg_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int64)
    L.wnlqg_b200_version.restype = ctypes.c_char_p
    L.wnlqg_b200_version.argtypes = []
    L.wnlqg_b200_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.wnlqg_b200_device_count.restype = ctypes.c_int32
    L.wnlqg_b200_device_count.argtypes = []
    L.wnlqg_b200_model_create.argtypes = [ctypes.POINTER(_abi.ModelDesc), ctypes.c_int32, ctypes.POINTER(vp)]
    L.wnlqg_b200_model_destroy.argtypes = [vp]
    L.wnlqg_b200_plan_create.argtypes = [vp, ctypes.POINTER(_abi.TaskDesc), ctypes.c_int64, ctypes.POINTER(vp)]
    L.wnlqg_b200_plan_destroy.argtypes = [vp]
    L.wnlqg_b200_plan_value_count.restype = ctypes.c_int64
    L.wnlqg_b200_plan_value_count.argtypes = [vp]
    L.wnlqg_b200_eval_mesh.argtypes = [vp, ip, ctypes.c_int64, ctypes.c_int64, dp]
    L.wnlqg_b200_eval_mesh_device.argtypes = [vp, ip, ctypes.c_int64, ctypes.c_int64, vp, vp]
    L.wnlqg_b200_eval_mesh_many.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ip, ip, ip, ctypes.POINTER(vp), vp]
    L.wnlqg_b200_eval_points.argtypes = [vp, dp, ctypes.c_int64, dp]
    L.wnlqg_b200_eval_points_weighted.argtypes = [vp, dp, dp, ctypes.c_int64, dp]
    L.wnlqg_b200_eval_points_weighted_device.argtypes = [vp, vp, vp, ctypes.c_int64, vp, vp]
    L.wnlqg_b200_eval_mesh_weighted.argtypes = [vp, ip, ip, dp, ctypes.c_int64, dp]
    L.wnlqg_b200_eval_spectrum.argtypes = [vp, dp, ctypes.c_int64, dp, dp]
    L.wnlqg_b200_plan_last_timing.argtypes = [vp, dp, dp, dp, dp]
    L.wnlqg_b200_spectrum_noalloc.argtypes = [ctypes.c_int64, ctypes.c_int64, vp, vp, vp, vp, ctypes.c_int64, vp, vp,
                                              vp]
    L.wnlqg_b200_spectrum_noalloc.restype = ctypes.c_int
    fp = ctypes.POINTER(ctypes.c_float)
    L.wnlqg_b200_mlp_param_count.restype = ctypes.c_int64
    L.wnlqg_b200_mlp_param_count.argtypes = []
    L.wnlqg_b200_mlp_create.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.wnlqg_b200_mlp_destroy.argtypes = [vp]
    L.wnlqg_b200_mlp_get_params.argtypes = [vp, fp]
    L.wnlqg_b200_mlp_set_params.argtypes = [vp, fp]
    L.wnlqg_b200_mlp_forward.argtypes = [vp, fp, ctypes.c_int64, fp]
    L.wnlqg_b200_mlp_loss_grad.argtypes = [vp, fp, fp, ctypes.c_int64, fp, fp]
    L.wnlqg_b200_mlp_train.argtypes = [vp, fp, fp, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, fp]
    for name in ("wnlqg_b200_mlp_create", "wnlqg_b200_mlp_destroy", "wnlqg_b200_mlp_get_params",
                 "wnlqg_b200_mlp_set_params", "wnlqg_b200_mlp_forward", "wnlqg_b200_mlp_loss_grad",
                 "wnlqg_b200_mlp_train"):
        getattr(L, name).restype = ctypes.c_int
    L.wnlqg_b200_plan_last_launch_count.restype = ctypes.c_int64
    L.wnlqg_b200_plan_last_launch_count.argtypes = [vp]
    L.wnlqg_b200_plan_status.argtypes = [vp]
    L.wnlqg_b200_plan_status.restype = ctypes.c_int
    L.wnlqg_b200_measure_peaks.argtypes = [ctypes.c_int32, dp, dp, dp]
    L.wnlqg_b200_measure_peaks.restype = ctypes.c_int
    L.wnlqg_b200_graph_capture_mesh_many.argtypes = [ctypes.POINTER(vp), ctypes.c_int32, ip, ip, ip,
                                                     ctypes.POINTER(vp), ctypes.POINTER(vp)]
    L.wnlqg_b200_graph_capture_points_weighted.argtypes = [vp, vp, vp, ctypes.c_int64, vp, ctypes.POINTER(vp)]
    L.wnlqg_b200_graph_launch.argtypes = [vp, vp]
    L.wnlqg_b200_graph_status.argtypes = [vp]
    L.wnlqg_b200_graph_kernel_count.restype = ctypes.c_int64
    L.wnlqg_b200_graph_kernel_count.argtypes = [vp]
    L.wnlqg_b200_graph_destroy.argtypes = [vp]
    L.wnlqg_b200_plan_autotune.argtypes = [vp, ip, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.POINTER(_abi.AutotuneReport)]
    for name in ("wnlqg_b200_graph_capture_mesh_many", "wnlqg_b200_graph_capture_points_weighted",
                 "wnlqg_b200_graph_launch", "wnlqg_b200_graph_status", "wnlqg_b200_graph_destroy",
                 "wnlqg_b200_plan_autotune"):
        getattr(L, name).restype = ctypes.c_int
    for name in ("wnlqg_b200_last_error", "wnlqg_b200_model_create", "wnlqg_b200_model_destroy",
                 "wnlqg_b200_plan_create", "wnlqg_b200_plan_destroy", "wnlqg_b200_eval_mesh",
                 "wnlqg_b200_eval_mesh_device", "wnlqg_b200_eval_mesh_many", "wnlqg_b200_eval_points",
                 "wnlqg_b200_eval_points_weighted",
                 "wnlqg_b200_eval_points_weighted_device", "wnlqg_b200_eval_mesh_weighted", "wnlqg_b200_eval_spectrum",
                 "wnlqg_b200_plan_last_timing"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    load().wnlqg_b200_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != _abi.WNLQG_OK:
        raise EngineError(status, last_error())


def measure_peaks(device: int = 0) -> dict:
    """Measured dense throughput of `device` in TFLOP/s: FP64 DMMA, FP64 FMA and FP32 FMA
    (wnlqg_b200_measure_peaks, about 20 ms of compute)."""
    L = load()
    vals = [ctypes.c_double(0.0) for _ in range(3)]
    st = L.wnlqg_b200_measure_peaks(int(device), *[ctypes.byref(v) for v in vals])
    check(st)
    return {"fp64_dmma_tflops": vals[0].value, "fp64_fma_tflops": vals[1].value, "fp32_fma_tflops": vals[2].value}

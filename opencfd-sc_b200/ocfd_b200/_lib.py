"""ctypes binding of the C ABI (include/ocfd_gpu.h).

The library is built in-tree (``make -C opencfd-sc_b200``) into this package's
directory.  There is no CPU fallback: when the library is missing, loading
raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .params import OcfdParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_FAST = os.path.join(_HERE, "libocfdgpu.so")
LIB_STRICT = os.path.join(_HERE, "libocfdgpu_strict.so")

OCFD_OK = 0
OCFD_E_PARAM = -1
OCFD_E_CUDA = -2
OCFD_E_NEGT = -3
OCFD_E_STATE = -4
OCFD_E_NOMEM = -5
OCFD_E_TIMEOUT = -6

_libs: dict[str, C.CDLL] = {}


class OcfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


class NegativeTemperatureStop(OcfdError):
    """The reference stops when more than 10 points have T <= 0 in one stage."""


class OcfdBcLayer(C.Structure):
    """ocfd_bc_layer of include/ocfd_gpu.h."""
    _fields_ = [("inlet", C.POINTER(C.c_double)), ("upper", C.POINTER(C.c_double)),
                ("pertb", C.POINTER(C.c_double)), ("mt", C.c_int32), ("beta", C.c_double),
                ("tm", C.POINTER(C.c_double)), ("fait", C.POINTER(C.c_double))]


def _declare(L: C.CDLL) -> C.CDLL:
    P = C.POINTER(OcfdParams)
    H = C.c_void_p
    dp = C.POINTER(C.c_double)
    L.ocfd_default_params.argtypes = [P]
    L.ocfd_set_parameters.argtypes = [P]
    L.ocfd_set_parameters.restype = C.c_int
    L.ocfd_gpu_footprint.argtypes = [P]
    L.ocfd_gpu_footprint.restype = C.c_size_t
    L.ocfd_gpu_create.argtypes = [P, C.c_int, C.POINTER(H)]
    L.ocfd_gpu_create.restype = C.c_int
    L.ocfd_gpu_destroy.argtypes = [H]
    L.ocfd_gpu_destroy.restype = None
    L.ocfd_gpu_last_error.argtypes = [H]
    L.ocfd_gpu_last_error.restype = C.c_char_p
    L.ocfd_gpu_stream.argtypes = [H]
    L.ocfd_gpu_stream.restype = C.c_void_p
    for name in ["ocfd_gpu_sync", "ocfd_gpu_save_fn", "ocfd_gpu_halo_prims", "ocfd_gpu_rhybrid",
                 "ocfd_gpu_du_inviscous", "ocfd_gpu_du_inviscous_character", "ocfd_gpu_du_viscous", "ocfd_gpu_bc",
                 "ocfd_gpu_filter", "ocfd_gpu_advance_clock"]:
        f = getattr(L, name)
        f.argtypes = [H]
        f.restype = C.c_int
    L.ocfd_gpu_upload_metrics.argtypes = [H, dp * 22]
    L.ocfd_gpu_upload_metrics.restype = C.c_int
    L.ocfd_gpu_download_metrics.argtypes = [H, dp * 22]
    L.ocfd_gpu_download_metrics.restype = C.c_int
    L.ocfd_gpu_init_mesh.argtypes = [H, dp, dp, dp]
    L.ocfd_gpu_init_mesh.restype = C.c_int
    L.ocfd_gpu_init_mesh_jacobian.argtypes = [H, dp, dp, dp, dp * 10]
    L.ocfd_gpu_init_mesh_jacobian.restype = C.c_int
    L.ocfd_gpu_upload_state.argtypes = [H, dp, C.c_void_p, C.c_int, C.c_double]
    L.ocfd_gpu_upload_state.restype = C.c_int
    L.ocfd_gpu_init3d.argtypes = [H, dp * 5, C.c_int, C.c_double]
    L.ocfd_gpu_init3d.restype = C.c_int
    L.ocfd_gpu_download_state.argtypes = [H, dp, C.c_void_p]
    L.ocfd_gpu_download_state.restype = C.c_int
    L.ocfd_gpu_download_du.argtypes = [H, dp]
    L.ocfd_gpu_download_du.restype = C.c_int
    L.ocfd_gpu_download_rhybrid.argtypes = [H, dp]
    L.ocfd_gpu_download_rhybrid.restype = C.c_int
    L.ocfd_gpu_get_time.argtypes = [H, C.POINTER(C.c_int), dp]
    L.ocfd_gpu_get_time.restype = C.c_int
    L.ocfd_gpu_rk3.argtypes = [H, C.c_int]
    L.ocfd_gpu_rk3.restype = C.c_int
    L.ocfd_gpu_duvwt.argtypes = [H, C.POINTER(C.c_int)]
    L.ocfd_gpu_duvwt.restype = C.c_int
    L.ocfd_gpu_step.argtypes = [H, C.c_int, C.c_int]
    L.ocfd_gpu_step.restype = C.c_int
    L.ocfd_gpu_step_kernels.argtypes = [H]
    L.ocfd_gpu_step_kernels.restype = C.c_int
    L.ocfd_gpu_show_flow_msg.argtypes = [H, dp]
    L.ocfd_gpu_show_flow_msg.restype = C.c_int
    L.ocfd_gpu_ana_box.argtypes = [H, dp]
    L.ocfd_gpu_ana_box.restype = C.c_int
    L.ocfd_gpu_profile_steps.argtypes = [H, C.c_int, dp]
    L.ocfd_gpu_profile_steps.restype = C.c_int
    L.ocfd_batch_create.argtypes = [C.POINTER(H), C.c_int, C.POINTER(H)]
    L.ocfd_batch_create.restype = C.c_int
    L.ocfd_batch_step.argtypes = [H, C.c_int, C.c_int]
    L.ocfd_batch_step.restype = C.c_int
    L.ocfd_batch_destroy.argtypes = [H]
    L.ocfd_batch_destroy.restype = None
    L.ocfd_gpu_ana_q.argtypes = [H, dp]
    L.ocfd_gpu_ana_q.restype = C.c_int
    L.ocfd_gpu_ana_time_average.argtypes = [H]
    L.ocfd_gpu_ana_time_average.restype = C.c_int
    L.ocfd_gpu_download_average.argtypes = [H, C.c_void_p, C.POINTER(C.c_int), dp]
    L.ocfd_gpu_download_average.restype = C.c_int
    L.ocfd_gpu_upload_average.argtypes = [H, C.c_void_p, C.c_int, C.c_double]
    L.ocfd_gpu_upload_average.restype = C.c_int
    L.ocfd_gpu_ana_corner.argtypes = [H, dp]
    L.ocfd_gpu_ana_corner.restype = C.c_int
    L.ocfd_gpu_download_block.argtypes = [H, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
    L.ocfd_gpu_download_block.restype = C.c_int
    L.ocfd_gpu_set_bc_layer.argtypes = [H, C.POINTER(OcfdBcLayer)]
    L.ocfd_gpu_set_bc_layer.restype = C.c_int
    L.ocfd_gpu_metric_zero_mask.argtypes = [H]
    L.ocfd_gpu_metric_zero_mask.restype = C.c_uint
    L.ocfd_batch_set_tiles.argtypes = [H, C.POINTER(C.c_int)]
    L.ocfd_batch_set_tiles.restype = C.c_int
    L.ocfd_batch_info.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ocfd_batch_info.restype = C.c_int
    L.ocfd_batch_set_persistent.argtypes = [H, C.c_int]
    L.ocfd_batch_set_persistent.restype = C.c_int
    L.ocfd_batch_mode.argtypes = [H]
    L.ocfd_batch_mode.restype = C.c_int
    L.ocfd_batch_mode_times.argtypes = [H, C.POINTER(C.c_float)]
    L.ocfd_batch_mode_times.restype = C.c_int
    L.ocfd_batch_last_error.argtypes = [H]
    L.ocfd_batch_last_error.restype = C.c_char_p
    L.ocfd_show_flow_msg_noalloc.argtypes = [P, C.c_void_p, C.c_void_p * 5, C.c_void_p, C.c_void_p, dp]
    L.ocfd_show_flow_msg_noalloc.restype = C.c_int
    return L


def lib(strict: bool = False) -> C.CDLL:
    """Load libocfdgpu.so (or the no-FMA strict build).  Raises if it is not built."""
    path = LIB_STRICT if strict else LIB_FAST
    if not strict and os.environ.get("OCFD_GPU_LIB"):
        path = os.environ["OCFD_GPU_LIB"]  # an alternative build of the same ABI
    if path not in _libs:
        if not os.path.exists(path):
            raise OSError(f"{path} is not built; run `make -C opencfd-sc_b200` (no CPU fallback exists)")
        _libs[path] = _declare(C.CDLL(path))
    return _libs[path]


EXPORTED = [
    "ocfd_default_params", "ocfd_set_parameters", "ocfd_gpu_footprint", "ocfd_gpu_create", "ocfd_gpu_destroy",
    "ocfd_gpu_last_error", "ocfd_gpu_sync", "ocfd_gpu_stream", "ocfd_gpu_upload_metrics", "ocfd_gpu_init_mesh",
    "ocfd_gpu_download_metrics", "ocfd_gpu_upload_state", "ocfd_gpu_init3d", "ocfd_gpu_download_state",
    "ocfd_gpu_download_du", "ocfd_gpu_download_rhybrid", "ocfd_gpu_get_time", "ocfd_gpu_save_fn",
    "ocfd_gpu_halo_prims", "ocfd_gpu_rhybrid", "ocfd_gpu_du_inviscous", "ocfd_gpu_du_inviscous_character",
    "ocfd_gpu_du_viscous", "ocfd_gpu_rk3", "ocfd_gpu_duvwt", "ocfd_gpu_bc", "ocfd_gpu_filter",
    "ocfd_gpu_advance_clock", "ocfd_gpu_step", "ocfd_gpu_show_flow_msg", "ocfd_gpu_ana_box", "ocfd_batch_create",
    "ocfd_batch_step", "ocfd_batch_destroy", "ocfd_gpu_profile_steps", "ocfd_show_flow_msg_noalloc",
    "ocfd_batch_set_tiles", "ocfd_batch_info", "ocfd_batch_last_error", "ocfd_gpu_metric_zero_mask",
    "ocfd_gpu_set_bc_layer", "ocfd_gpu_ana_q", "ocfd_gpu_ana_time_average", "ocfd_gpu_download_average",
    "ocfd_gpu_upload_average", "ocfd_gpu_ana_corner", "ocfd_gpu_download_block", "ocfd_gpu_step_kernels",
    "ocfd_gpu_init_mesh_jacobian", "ocfd_batch_set_persistent", "ocfd_batch_mode",
    "ocfd_batch_mode_times",
]

"""ctypes binding of the vipe_b200 C ABI (include/vipe_b200.h).

The shared library is built in-tree by ``python -m vipe_b200.build``.  There is
no fallback: every op in vipe_b200.ext raises if the library is missing or if
its tensors are not CUDA tensors.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libvipe_b200.so"

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None

P = ctypes.c_void_p
I = ctypes.c_int
I64 = ctypes.c_int64
F = ctypes.c_float
SZ = ctypes.c_size_t

# name -> (restype, argtypes); mirrors include/vipe_b200.h
_SIGS: dict[str, tuple] = {
    "vipe_status_string": (ctypes.c_char_p, [I]),
    "vipe_last_error": (ctypes.c_char_p, []),
    "vipe_profile_enable": (None, [I]),
    "vipe_profile_collect": (I, [ctypes.c_char_p, I, P, P, I]),
    "vipe_slam_ba_workspace_size": (SZ, [I, I, I, I, I, I, I]),
    "vipe_slam_ba_extended": (
        I,
        [P, P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, I, F, F, F, I, P, P, P, P, SZ, P, P],
    ),
    "vipe_slam_ba": (I, [P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, P, P, P, P, SZ, P, P]),
    "vipe_slam_ba_extended_robust": (
        I,
        [P, P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, I, F, F, F, I, P, P, P, I, F, P, P, SZ,
         P, P],
    ),
    "vipe_slam_ba_rig_workspace_size": (SZ, [I, I, I, I, I, I, I, I, I]),
    "vipe_slam_ba_rig": (
        I,
        [P, P, I, P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, I, P, P, P, I, F, P, I, F, P, I, F,
         F, P, SZ, P, P],
    ),
    "vipe_slam_ba_extended_generic": (
        I,
        [P, P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, I, F, F, F, I, P, P, P, I, F, P, I, F, P,
         SZ, P, P],
    ),
    "vipe_slam_ba_extended_noalloc": (
        I,
        [P, P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, F, I, F, I, F, F, F, I, P, P, P, P, P],
    ),
    "vipe_slam_ba_batch_plan_create": (I, [I, P, P, P, P, P, I, I, I, I, I, I, P]),
    "vipe_slam_ba_batch_workspace_size": (SZ, [P]),
    "vipe_slam_ba_batch_totals": (I, [P, P]),
    "vipe_slam_ba_batch_bind": (I, [P, P, SZ, P]),
    "vipe_slam_ba_batch_solve": (
        I,
        [P, P, P, P, P, P, P, P, P, P, P, I, F, F, I, F, I, F, F, F, I, P, P, P, P, P, P, P, P, P],
    ),
    "vipe_slam_ba_batch_plan_destroy": (None, [P]),
    "vipe_slam_ba_batch_backward": (
        I,
        [P, P, P, P, P, P, P, P, P, P, P, P, P, I, F, F, F, P, P, P, P, P, P, P, P],
    ),
    "vipe_slam_ba_index_debug": (I, [P, P, I, I, I, I, I, P, P, P, I, P, P, P, P, SZ, P]),
    "vipe_slam_frame_distance": (I, [P, P, P, P, P, P, P, P, I, I, I, I, I, I, F, P, P]),
    "vipe_slam_projmap": (I, [P, P, P, P, P, I, I, I, I, P, P, P]),
    "vipe_slam_depth_filter": (I, [P, P, P, P, P, I, I, I, I, P, P]),
    "vipe_slam_iproj": (I, [P, P, P, I, I, I, P, P]),
    "vipe_corr_index_forward": (I, [I, P, P, I, I, I, I, I, I, P, P]),
    "vipe_corr_index_backward": (I, [I, P, P, I, I, I, I, I, I, P, P]),
    "vipe_corr_index_coords_backward": (I, [I, P, P, P, I, I, I, I, I, I, P, P]),
    "vipe_altcorr_forward": (I, [I, P, P, P, I, I, I, I, I, I, I, I, P, P]),
    "vipe_altcorr_backward": (I, [P, P, P, P, I, I, I, I, I, I, I, I, I, P, P, P, P]),
    "vipe_altcorr_index_forward": (I, [I, P, P, P, P, I, P, P, P, I, I, I, I, I, I, I, P, P]),
    "vipe_altcorr_index_backward": (I, [I, P, P, P, P, I, P, P, P, P, I, I, I, I, I, I, I, I, P, P, P, P]),
    "vipe_corr_pyramid_nhwc": (I, [I, P, I, I, I, I, I, P, P]),
    "vipe_corr_pyramid_nhwc_backward": (I, [I, P, I, I, I, I, I, P, P]),
    "vipe_corr_sample_forward": (I, [I, P, P] + [I] * 16 + [P, P]),
    "vipe_corr_sample_backward": (I, [I, P, P, P] + [I] * 16 + [P, P, P]),
    "vipe_slam_proximity_edges_workspace_size": (SZ, [I, I, I]),
    "vipe_slam_proximity_edges_capacity": (ctypes.c_long, [I, I, I, I, I, I]),
    "vipe_slam_proximity_edges": (I, [P, P, P, I, I, I, I, I, I, F, I, I, P, P, I, P, P, SZ, P]),
    "vipe_corr_volume_workspace_size": (SZ, [I, I, I, I]),
    "vipe_corr_volume_backward": (I, [I, I, P, P, P, I, I, I, I, I, P, P, P, P]),
    "vipe_corr_volume_backward_force_generic": (None, [I]),
    "vipe_corr_encoder_lookup": (I, [I, P, I, P, I, I, I, P, P, P, P, P]),
    "vipe_hbm_write_probe": (I, [P, SZ, P]),
    "vipe_corr_volume_build": (I, [I, I, P, P, I, I, I, I, I, P, P, SZ, P]),
}
for _op in ("expm", "logm", "inv", "as_matrix", "projector"):
    _SIGS[f"vipe_lie_{_op}"] = (I, [I, I, I64, P, P, P])
for _op in ("mul", "adj", "adjT", "act", "act4", "Jinv"):
    _SIGS[f"vipe_lie_{_op}"] = (I, [I, I, I64, P, P, P, P])
for _op in ("expm", "logm", "inv"):
    _SIGS[f"vipe_lie_{_op}_backward"] = (I, [I, I, I64, P, P, P, P])
for _op in ("mul", "adj", "adjT", "act", "act4"):
    _SIGS[f"vipe_lie_{_op}_backward"] = (I, [I, I, I64, P, P, P, P, P, P])

EXPORTED = tuple(_SIGS)

# status codes (enum vipe_status)
VIPE_OK = 0
VIPE_ERR_ARG = 1
VIPE_ERR_INDEX = 2
VIPE_ERR_RANGE = 3
VIPE_ERR_KX_MISMATCH = 4
VIPE_ERR_CAPACITY = 6
VIPE_ERR_DTYPE = 8
VIPE_ERR_GROUP = 9
VIPE_ERR_DEVICE_WAIT = 10
VIPE_WARN_SOLVER = 16

# dtypes (enum vipe_dtype)
VIPE_F32, VIPE_F64, VIPE_F16, VIPE_BF16 = 0, 1, 2, 3
DTYPE_CODE = {torch.float32: VIPE_F32, torch.float64: VIPE_F64, torch.float16: VIPE_F16, torch.bfloat16: VIPE_BF16}


def load() -> ctypes.CDLL:
    """Loads the library (once) and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"vipe_b200 CUDA library not found at {LIB_PATH}; build it with `python -m vipe_b200.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue  # reported by missing_symbols(); calling it raises AttributeError
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def missing_symbols() -> list[str]:
    """Entry points declared in include/vipe_b200.h that the library lacks."""
    lib = load()
    return [n for n in _SIGS if getattr(lib, n, None) is None]


def status_string(code: int) -> str:
    return load().vipe_status_string(code).decode()


def check(rc: int, what: str) -> None:
    if rc != VIPE_OK:
        extra = load().vipe_last_error().decode()
        raise RuntimeError(f"{what} failed: {status_string(rc)}" + (f" ({extra})" if extra else ""))


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_of(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def require_cuda(name: str, t: torch.Tensor) -> None:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor (vipe_b200 has no CPU path)")


def require_contiguous(name: str, t: torch.Tensor) -> None:
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def require_dtype(name: str, t: torch.Tensor, *dtypes: torch.dtype) -> None:
    if t.dtype not in dtypes:
        raise RuntimeError(f"expected {name} of dtype {' or '.join(map(str, dtypes))} but found {t.dtype}")

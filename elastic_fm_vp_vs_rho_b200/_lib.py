"""ctypes binding of libefm.so (the C ABI in include/efm.h).

The library is built in-tree for sm_100a by :mod:`elastic_fm_vp_vs_rho_b200.build`.
There is no CPU fallback: if the library is missing and cannot be built, every call
raises :class:`EfmError`.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

EFM_OK = 0
EFM_ERR_ARG = 1
EFM_ERR_CUDA = 2
EFM_ERR_STATE = 3
EFM_ERR_NOMEM = 4
EFM_ERR_TIMEOUT = 5
EFM_OPT_STREAM_KERNELS = 1
EFM_OPT_YCHUNK = 2
EFM_MAX_SRC = 4
EFM_GRAD_MODEL = 1
EFM_GRAD_MT = 2
EFM_GRAD_NT1 = 4
EFM_GRAD_EXACT = 8
EFM_SAVE_STRIPS = 1
EFM_SAVE_CHECKPOINTS = 2
EFM_OPT_CHECKPOINT_EVERY = 3
EFM_OPT_TILE_ROWS = 4
EFM_OPT_RING_DEPTH = 5
EFM_OPT_PAIR_LAUNCH = 6
EFM_OPT_PDL = 7
EFM_OPT_GRAPH = 8
EFM_OPT_WAIT_LIMIT = 9
EFM_OPT_EXACT_FORM = 10
EFM_OPT_EXACT_FUSED = EFM_OPT_EXACT_FORM
EFM_EXACT_TWO_PASS, EFM_EXACT_GATHER, EFM_EXACT_STREAM = 0, 1, 2
EFM_NKERN = 11
KERNEL_NAMES = ("fwd_stress", "fwd_velocity", "adj_stress", "adj_velocity", "rev_velocity",
                "rev_stress", "residual_misfit", "model_reciprocals", "imaging",
                "adj_stress+rev_velocity", "rev_stress+adj_velocity")

_ERRNAMES = {EFM_ERR_ARG: "EFM_ERR_ARG", EFM_ERR_CUDA: "EFM_ERR_CUDA",
             EFM_ERR_STATE: "EFM_ERR_STATE", EFM_ERR_NOMEM: "EFM_ERR_NOMEM",
             EFM_ERR_TIMEOUT: "EFM_ERR_TIMEOUT"}


class EfmError(RuntimeError):
    """A libefm call returned an error status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class InstanceDesc(ctypes.Structure):
    """Mirror of efm_instance_desc."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lenpml", ctypes.c_int), ("dx", ctypes.c_float), ("dt", ctypes.c_float),
        ("nt", ctypes.c_int), ("cpml_host", ctypes.c_void_p), ("lam_dev", ctypes.c_void_p),
        ("mu_dev", ctypes.c_void_p), ("rho_dev", ctypes.c_void_p),
        ("wavelet_dev", ctypes.c_void_p), ("nsrc", ctypes.c_int),
        ("src_host", ctypes.c_void_p), ("mt_host", ctypes.c_void_p), ("nrec", ctypes.c_int),
        ("rec_host", ctypes.c_void_p),
    ]


class ConvDesc(ctypes.Structure):
    """Mirror of efm_conv_desc."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("cin", ctypes.c_int), ("cout", ctypes.c_int)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_F = ctypes.c_float

# name -> (restype, argtypes); every symbol declared in include/efm.h
SIGNATURES = {
    "efm_create": (_I, [ctypes.POINTER(_P)]),
    "efm_destroy": (_I, [_P]),
    "efm_last_error": (ctypes.c_char_p, []),
    "efm_version": (_I, []),
    "efm_add_instance": (_I, [_P, ctypes.POINTER(InstanceDesc), ctypes.POINTER(_I)]),
    "efm_clear": (_I, [_P]),
    "efm_num_instances": (_I, [_P]),
    "efm_set_model": (_I, [_P, _I, _P, _P, _P]),
    "efm_set_moment_tensor": (_I, [_P, _I, _P]),
    "efm_gather_size": (_L, [_P]),
    "efm_gather_offset": (_L, [_P, _I]),
    "efm_workspace_bytes": (_L, [_P, _I]),
    "efm_forward": (_I, [_P, _P, _I, _P]),
    "efm_forward_illumination": (_I, [_P, _P, _I, _P, _P]),
    "efm_gradient": (_I, [_P, _P, _P, _P, _I, _P]),
    "efm_residual_misfit": (_I, [_P, _P, _P, _P, _P, _P]),
    "efm_residual_misfit_noalloc": (_I, [_P, _P, _P, _P, _I, _P, _P]),
    "efm_set_option": (_I, [_P, _I, _I]),
    "efm_status": (_I, [_P, _P]),
    "efm_set_timing": (_I, [_P, _I]),
    "efm_kernel_stats": (_I, [_P, _P, _P, _I]),
    "efm_kernel_time": (_I, [_P, _I, _I, _I, _P, _P]),
    "efm_dot": (_I, [_P, _P, _L, _P, _P]),
    "efm_lbfgs_history": (_I, [_P, _P, _P, _P, _I, _L, _I, _P]),
    "efm_lbfgs_direction": (_I, [_P, _P, _P, _P, _P, _I, _L, _I, _P]),
    "efm_smooth_mask": (_I, [_P, _P, _I, _I, _I, _F, _I, _I, _P]),
    "efm_chain_rule": (_I, [_P, _P, _P, _P, _P, _P, _L, _P]),
    "efm_xcorr_residual_misfit": (_I, [_P, _P, _P, _P, _I, _I, _P, _P]),
    "efm_conv3d_supported": (_I, [_I, _I]),
    "efm_conv3d_prep_weights": (_I, [_I, _I, _P, _P, _P, _P]),
    "efm_conv3d_forward": (_I, [ctypes.POINTER(ConvDesc), _P, _P, _P, _I, _P, _P, _P]),
    "efm_conv3d_backward_data": (_I, [ctypes.POINTER(ConvDesc), _P, _P, _P, _P, _P]),
    "efm_conv3d_wgrad_workspace": (ctypes.c_size_t, [ctypes.POINTER(ConvDesc)]),
    "efm_conv3d_backward_weights": (_I, [ctypes.POINTER(ConvDesc), _P, _P, _P, _P, _P,
                                         ctypes.c_size_t, _P]),
    "efm_conv3d_status": (_I, [_P]),
    "efm_conv3d_set_grouped_loads": (None, [_I]),
    "efm_conv3d_set_swizzled_loads": (None, [_I]),
}

_lock = threading.Lock()
_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libefm.so (building it with nvcc first when it is absent or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if build_if_missing and not _build.up_to_date():
            try:
                _build.build()
            except Exception as e:  # pragma: no cover - toolchain problems
                if not os.path.exists(path):
                    raise EfmError(EFM_ERR_STATE, f"libefm.so missing and build failed: {e}") from e
        if not os.path.exists(path):
            raise EfmError(EFM_ERR_STATE, f"libefm.so not found at {path}")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L


def check(rc: int):
    if rc != EFM_OK:
        raise EfmError(rc, load().efm_last_error().decode(errors="replace"))


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream (default: the current stream) as a ctypes pointer."""
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t) -> ctypes.c_void_p:
    """Device pointer of a contiguous CUDA tensor."""
    if not t.is_cuda:
        raise EfmError(EFM_ERR_ARG, "tensor is not on a CUDA device")
    if not t.is_contiguous():
        raise EfmError(EFM_ERR_ARG, "tensor is not contiguous")
    return ctypes.c_void_p(t.data_ptr())

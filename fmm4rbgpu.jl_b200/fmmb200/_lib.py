"""ctypes binding of libfmmb200.so (the C-ABI declared in include/fmmb200.h).

The library is loaded from the package tree (``fmm4rbgpu.jl_b200/lib``).  There
is no fallback: if the library is missing or no CUDA device is present every
call raises :class:`FMMB200Error`.
"""
from __future__ import annotations

import ctypes
import os
import threading

from ._build import LIB_PATH, build

_lock = threading.Lock()
_lib = None

c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_f64 = ctypes.c_double
c_vp = ctypes.c_void_p
p_f64 = ctypes.POINTER(ctypes.c_double)
p_i64 = ctypes.POINTER(ctypes.c_int64)

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_MEMORY = 2
ERR_CUDA = 3
ERR_TREE_SHAPE = 4
ERR_NO_STATE = 5
ERR_DEVICE = 6
ERR_CAPACITY = 7

PRECISION_FP64 = 0
PRECISION_MIXED = 1

M2L_AUTO = 0
M2L_CUDA_CORES = 1
M2L_TENSOR_CORES = 2


class FMMB200Error(RuntimeError):
    """A non-zero status from libfmmb200 (the reference raises ErrorException)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


class Stats(ctypes.Structure):
    _fields_ = [
        ("npar", c_i64), ("n", c_i64), ("N0", c_i64), ("max_level", c_i64), ("ncluster", c_i64),
        ("nleaf", c_i64), ("nm2l", c_i64), ("np2p", c_i64), ("m2l_groups", c_i64), ("p2p_groups", c_i64),
        ("traversal_steps", c_i64), ("device_bytes", c_i64),
        ("pavg", c_f64 * 3), ("stretch", c_f64 * 3),
        ("ms_h2d", c_f64), ("ms_tree", c_f64), ("ms_lists", c_f64), ("ms_upward", c_f64), ("ms_m2l", c_f64),
        ("ms_p2p", c_f64), ("ms_downward", c_f64), ("ms_d2h", c_f64), ("ms_total", c_f64), ("ms_backward", c_f64),
        ("m2l_kernel_evals", c_f64), ("p2p_kernel_evals", c_f64), ("kernel_launches", c_i64),
        ("tree_reused", c_i64),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, ctypes.Array) else v
        return out


# name -> (restype, argtypes); the exact exports of include/fmmb200.h
SIGNATURES = {
    "fmmb200_version": (ctypes.c_int, []),
    "fmmb200_create": (ctypes.c_int, [ctypes.POINTER(c_vp), ctypes.c_int]),
    "fmmb200_destroy": (ctypes.c_int, [c_vp]),
    "fmmb200_last_error": (ctypes.c_char_p, [c_vp]),
    "fmmb200_set_stream": (ctypes.c_int, [c_vp, c_vp]),
    "fmmb200_set_timing": (ctypes.c_int, [c_vp, ctypes.c_int]),
    "fmmb200_debug_fail_alloc": (ctypes.c_int, [c_vp, c_i64]),
    "fmmb200_update_particles_field": (ctypes.c_int, [c_vp, c_i64, c_f64, p_f64, p_f64, p_f64, p_f64,
                                                      c_i32, c_i64, c_f64, c_f64, c_i32]),
    "fmmb200_forward": (ctypes.c_int, [c_vp, c_i64, p_f64, p_f64, c_f64, c_f64, c_i32, c_i64, c_f64, c_i32,
                                       p_f64, c_i32, p_f64, p_f64]),
    "fmmb200_forward_device": (ctypes.c_int, [c_vp, c_i64, c_vp, c_vp, c_f64, c_f64, c_i32, c_i64, c_f64, c_i32,
                                              p_f64, c_i32, c_vp, c_vp]),
    "fmmb200_backward": (ctypes.c_int, [c_vp, p_f64, p_f64, p_f64, p_f64]),
    "fmmb200_backward_device": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "fmmb200_get_stats": (ctypes.c_int, [c_vp, ctypes.POINTER(Stats)]),
    "fmmb200_get_tree_info": (ctypes.c_int, [c_vp, p_i64]),
    "fmmb200_get_tree": (ctypes.c_int, [c_vp, p_i64, p_i64, p_i64, p_i64, p_i64, p_f64]),
    "fmmb200_get_lists": (ctypes.c_int, [c_vp, p_i64, p_i64]),
    "fmmb200_get_expansions": (ctypes.c_int, [c_vp, p_f64, p_f64, p_f64, p_f64]),
    "fmmb200_cluster_tree": (ctypes.c_int, [c_vp, c_i64, p_f64, c_i64, p_f64, p_i64, p_i64, p_i64, p_i64,
                                            p_i64, p_f64]),
    "fmmb200_interaction_lists": (ctypes.c_int, [c_vp, p_f64, c_f64, p_i64]),
    "fmmb200_p2m": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, p_f64, p_f64, p_i64, c_i64, p_i64, p_f64, c_i64,
                                   p_i64, p_f64, p_f64]),
    "fmmb200_m2m": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, p_i64, p_f64, c_i64, p_f64, p_f64]),
    "fmmb200_m2l": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, p_f64, p_f64, p_f64, c_i64, p_i64, p_f64, p_f64,
                                   p_f64]),
    "fmmb200_p2p": (ctypes.c_int, [c_vp, c_i32, c_i64, p_f64, p_f64, p_i64, c_i64, p_i64, p_f64, c_i64, p_i64,
                                   p_f64, p_f64]),
    "fmmb200_l2l": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, p_i64, p_f64, c_i64, p_f64, p_f64]),
    "fmmb200_l2p": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, p_f64, p_i64, c_i64, p_i64, p_f64, c_i64, p_i64,
                                   p_f64, p_f64, p_f64, p_f64]),
    "fmmb200_direct": (ctypes.c_int, [c_vp, c_i64, p_f64, p_f64, c_f64, c_f64, c_i64, p_i64, p_f64, p_f64]),
    "fmmb200_direct_device": (ctypes.c_int, [c_vp, c_i64, c_vp, c_vp, c_f64, c_f64, c_i64, c_vp, c_vp, c_vp]),
    "fmmb200_measure_fma_peak": (ctypes.c_int, [c_vp, p_f64, p_f64, p_f64]),
    "fmmb200_measure_p2p_body": (ctypes.c_int, [c_vp, p_f64, p_f64]),
    "fmmb200_set_m2l_engine": (ctypes.c_int, [c_vp, ctypes.c_int]),
    "fmmb200_set_tree_reuse": (ctypes.c_int, [c_vp, ctypes.c_int]),
    "fmmb200_set_shard": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.c_int]),
    "fmmb200_direct_noalloc": (ctypes.c_int, [c_i64, c_vp, c_vp, c_f64, c_f64, c_i64, c_vp, c_vp, c_vp, c_vp]),
    "fmmb200_shard_record_bytes": (ctypes.c_int, [c_i32, c_i32, p_i64, p_i64]),
    "fmmb200_shard_subtree": (ctypes.c_int, [c_vp, c_i64, c_vp, c_vp, c_i64, c_i32, p_f64, c_i32, c_i32]),
    "fmmb200_shard_boxes": (ctypes.c_int, [c_vp, c_vp]),
    "fmmb200_shard_pack": (ctypes.c_int, [c_vp, c_i64, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp]),
    "fmmb200_shard_lists": (ctypes.c_int, [c_vp, c_i64, c_i32, c_vp, p_f64, c_f64, c_i32, c_i32, p_i64]),
    "fmmb200_shard_get_lists": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "fmmb200_shard_evaluate": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i64, c_f64, c_i64, c_vp, c_vp, c_vp, c_i64,
                                              c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_i64, c_f64, c_f64, c_vp,
                                              c_vp]),
}


def load(auto_build: bool = True):
    """Load (building first if the sources are newer) and return the CDLL."""
    global _lib
    with _lock:
        if _lib is None:
            if auto_build and not os.path.exists(LIB_PATH):
                build()
            if not os.path.exists(LIB_PATH):
                raise FMMB200Error(ERR_CUDA, f"{LIB_PATH} is missing: build it with fmmb200._build.build()")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib

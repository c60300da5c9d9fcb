"""ctypes bindings of libckd.so (declared in include/ckd.h).

The library is built in-tree by ``cosmokdtree_b200/csrc/Makefile`` and loaded from the
package directory.  There is no CPU fallback: if the library or a B200 is missing,
every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libckd.so")

CKD_OK = 0
CKD_ERR_BAD_DIM = 1
CKD_ERR_OUT_OF_BOX = 2
CKD_ERR_BAD_ARG = 3
CKD_ERR_OOM = 4
CKD_ERR_TIMEOUT = 5
CKD_ERR_CUDA = 6
CKD_ERR_NO_DEVICE = 7
CKD_ERR_DEPTH = 8

CKD_F64 = 0
CKD_F32 = 1


class CKDError(RuntimeError):
    """Base class of libckd failures; ``status`` is the ckd_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


class CKDArgumentError(CKDError, ValueError, AssertionError):
    """Bad argument.  Also an AssertionError: the reference Python API rejects these
    inputs with ``assert`` (src/cosmokdtree/kdtree.py:21,26,42,57)."""


class CKDOutOfMemory(CKDError, MemoryError):
    pass


class CKDTimeout(CKDError, TimeoutError):
    pass


def build_library(force: bool = False) -> str:
    """Compile libckd.so for sm_100a with nvcc (works without a GPU)."""
    csrc = os.path.join(_HERE, "csrc")
    if force:
        subprocess.run(["make", "-s", "-C", csrc, "clean"], check=True)
    subprocess.run(["make", "-s", "-j8", "-C", csrc], check=True)
    return LIB_PATH


_lib = None

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double
_pi32 = ctypes.POINTER(ctypes.c_int32)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pdbl = ctypes.POINTER(ctypes.c_double)
_pint = ctypes.POINTER(ctypes.c_int)

# name -> argtypes (restype is ckd_status = int unless listed in _RESTYPES)
SIGNATURES = {
    "ckd_version": [],
    "ckd_last_error": [],
    "ckd_build": [_vp, _i64, _int, _int, _int, _pdbl, _int, _vp, ctypes.POINTER(_vp)],
    "ckd_free": [_vp],
    "ckd_release_cached_memory": [],
    "ckd_pool_usage": [_pi64, _pi64],
    "ckd_forest_plan_create": [_vp, _pi64, _i64, _int, _int, _pdbl, _vp, _pi64, _i64, _int, _int,
                               _vp, _vp, _dbl, _int, ctypes.POINTER(_vp)],
    "ckd_forest_plan_run": [_vp, _vp],
    "ckd_forest_plan_status": [_vp, _vp],
    "ckd_forest_plan_forest": [_vp, ctypes.POINTER(_vp)],
    "ckd_forest_plan_free": [_vp],
    "ckd_tree_info": [_vp, _pi64, _pint, _pint, _pint, _pi32, _pi32, _pi32, _pint],
    "ckd_tree_export": [_vp, _pi32, _pdbl, _pi64, _pi64, _pi64, _pi64, _pdbl, _pdbl, _pi64],
    "ckd_knn": [_vp, _vp, _i64, _int, _int, _vp, _vp, _vp],
    "ckd_knn_host": [_vp, _vp, _i64, _int, _int, _vp, _vp, _vp],
    "ckd_knn_multi_k": [_vp, _vp, _i64, _vp, _int, _int, _vp, _vp, _vp],
    "ckd_knn_noalloc": [_vp, _vp, _i64, _int, _int, _vp, _vp, _vp],
    "ckd_query_order": [_vp, _vp, _i64, _vp, _vp],
    "ckd_knn_ordered": [_vp, _vp, _i64, _vp, _int, _int, _vp, _vp, _vp],
    "ckd_launch_count": [],
    "ckd_set_knn_variant": [_int],
    "ckd_set_tuning": [_int, _int],
    "ckd_set_kernel_timing": [_int],
    "ckd_kernel_ms": [ctypes.POINTER(ctypes.c_float)],
    "ckd_knn_stats": [_int, _pi64],
    "ckd_ball_count": [_vp, _vp, _i64, _dbl, _vp, _vp],
    "ckd_ball_fill": [_vp, _vp, _i64, _dbl, _int, _vp, _vp, _vp, _vp],
    "ckd_box_count": [_vp, _vp, _i64, _vp, _vp],
    "ckd_box_fill": [_vp, _vp, _i64, _vp, _vp, _vp],
    "ckd_ball_count_host": [_vp, _vp, _i64, _dbl, _vp, _vp],
    "ckd_ball_fill_host": [_vp, _vp, _i64, _dbl, _int, _vp, _vp, _vp, _vp],
    "ckd_box_count_host": [_vp, _vp, _i64, _vp, _vp],
    "ckd_box_fill_host": [_vp, _vp, _i64, _vp, _vp, _vp],
    "ckd_exclusive_scan": [_vp, _vp, _i64, _vp],
    "ckd_tree_save": [_vp, ctypes.c_char_p],
    "ckd_tree_load": [ctypes.c_char_p, ctypes.POINTER(_vp)],
    "ckd_forest_build": [_vp, _pi64, _i64, _int, _int, _int, _pdbl, _int, _vp,
                         ctypes.POINTER(_vp)],
    "ckd_forest_info": [_vp, _pi64, _pi64],
    "ckd_forest_knn": [_vp, _vp, _vp, _i64, _int, _int, _vp, _vp, _vp],
    "ckd_forest_box_count": [_vp, _vp, _vp, _i64, _vp, _vp],
    "ckd_forest_box_fill": [_vp, _vp, _vp, _i64, _vp, _vp, _vp],
    "ckd_forest_ball_count": [_vp, _vp, _vp, _i64, _dbl, _vp, _vp],
    "ckd_forest_ball_fill": [_vp, _vp, _vp, _i64, _dbl, _int, _vp, _vp, _vp, _vp],
    "ckd_mlp_create": [ctypes.c_uint64, ctypes.POINTER(_vp)],
    "ckd_mlp_free": [_vp],
    "ckd_mlp_get": [_vp, _vp, _vp, _vp, _vp],
    "ckd_mlp_set": [_vp, _vp, _vp, ctypes.c_float],
    "ckd_mlp_features": [_vp, _vp, _i64, _int, _vp, _vp],
    "ckd_mlp_grad": [_vp, _vp, _vp, _i64, _vp, _vp, _vp],
    "ckd_mlp_train": [_vp, _vp, _vp, _i64, _int, _int, ctypes.c_float, _vp, _vp],
    "ckd_mlp_predict": [_vp, _vp, _i64, _vp, _vp],
    "ckd_knn_learned": [_vp, _vp, _vp, _i64, _int, _int, _vp, _vp, _vp, _vp],
    "ckd_knn_learned_multi_k": [_vp, _vp, _vp, _i64, _vp, _int, _int, _vp, _vp, _vp, _vp],
}

MLP_FEATURES = 12
MLP_HIDDEN = 64
MLP_PARAMS = 5057
MLP_NORM = 26
_RESTYPES = {"ckd_last_error": ctypes.c_char_p, "ckd_launch_count": ctypes.c_int64}


def load(path: str = LIB_PATH):
    """Load libckd.so (once).  Raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"libckd.so not found at {path}; build it with `make -C cosmokdtree_b200/csrc` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = L
    return L


def last_error() -> str:
    msg = load().ckd_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = "") -> None:
    if status == CKD_OK:
        return
    msg = last_error() or what
    if status in (CKD_ERR_BAD_DIM, CKD_ERR_OUT_OF_BOX, CKD_ERR_BAD_ARG):
        raise CKDArgumentError(status, msg)
    if status == CKD_ERR_OOM:
        raise CKDOutOfMemory(status, msg)
    if status == CKD_ERR_TIMEOUT:
        raise CKDTimeout(status, msg)
    raise CKDError(status, msg)

"""ctypes binding of libqann_gpu.so (the C ABI declared in include/qann_gpu.h).

The library is built in-tree by ``qann_b200/build.py``. There is no fallback:
if the library is missing, importing this module raises ImportError, and
every call that needs the GPU raises when no CUDA device is usable.
"""
from __future__ import annotations

import ctypes as C
import pathlib

_PATH = pathlib.Path(__file__).resolve().parent / "libqann_gpu.so"

if not _PATH.exists():
    raise ImportError(f"{_PATH} is missing: build it with `python -m qann_b200.build` (needs nvcc)")

lib = C.CDLL(str(_PATH))

_vp, _sz, _i64 = C.c_void_p, C.c_size_t, C.c_int64
_H = C.POINTER(C.c_void_p)

# name -> (restype, argtypes)
_SIGS = {
    "qg_last_error": (C.c_char_p, []),
    "qg_version": (C.c_char_p, []),
    "qg_create_ivf": (C.c_int, [_sz, _sz, _sz, C.c_int, C.c_int, _H]),
    "qg_enable_pq": (C.c_int, [_vp, _sz, _sz, C.c_int, C.c_int]),
    "qg_create_flat": (C.c_int, [_sz, C.c_int, C.c_int, _H]),
    "qg_create_refine": (C.c_int, [_vp, _sz, C.c_int, _H]),
    "qg_refine_base": (C.c_int, [_vp, _H]),
    "qg_free": (None, [_vp]),
    "qg_train": (C.c_int, [_vp, _vp, _sz, _sz, _i64, C.c_int, _sz]),
    "qg_add": (C.c_int, [_vp, _vp, _sz, _vp, _vp]),
    "qg_remove": (C.c_int, [_vp, _vp, _sz, C.POINTER(_sz)]),
    "qg_compact": (C.c_int, [_vp, C.POINTER(_sz)]),
    "qg_search": (C.c_int, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, _vp]),
    "qg_search_bitmap": (C.c_int, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, _vp]),
    "qg_search_device": (C.c_int, [_vp, _vp, _sz, _sz, _vp, _vp, _vp]),
    "qg_candidate_count": (C.c_int, [_vp, _sz, C.POINTER(_sz)]),
    "qg_search_candidates_device": (C.c_int, [_vp, _vp, _sz, _sz, _vp, _vp, _vp]),
    "qg_merge_candidates_device": (C.c_int, [_vp, _vp, _sz, _sz, _sz, _vp, _vp, _vp]),
    "qg_finish_candidates_device": (C.c_int, [_vp, _vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp]),
    "qg_get": (C.c_int, [_vp, C.c_char_p, C.POINTER(_i64)]),
    "qg_set": (C.c_int, [_vp, C.c_char_p, _i64]),
    "qg_ivf_list_sizes": (C.c_int, [_vp, _vp]),
    "qg_ivf_centroids": (C.c_int, [_vp, _vp]),
    "qg_save": (C.c_int, [_vp, C.c_char_p]),
    "qg_load": (C.c_int, [C.c_char_p, _H, C.POINTER(C.c_int)]),
    "qg_load_mapped": (C.c_int, [C.c_char_p, _H, C.POINTER(C.c_int)]),
    "qg_profile_enable": (C.c_int, [C.c_int]),
    "qg_profile_reset": (C.c_int, []),
    "qg_profile_get": (C.c_int, [C.c_char_p, C.POINTER(C.c_double), C.POINTER(_i64)]),
    "qg_launch_count": (_i64, []),
    "qg_quantize_lut_dev": (C.c_int, [_vp, _sz, _sz, _vp, _vp, _vp, _vp]),
    "qg_build_quantize_lut_dev": (C.c_int, [_vp, _vp, _vp, _sz, _sz, _vp, _vp, _vp, _vp]),
    "qg_fast_scan_dev": (C.c_int, [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]),
    "qg_exact_scores_dev": (C.c_int, [_vp, _sz, _vp, _sz, _sz, C.c_int, _vp, _vp]),
    "qg_fast_scan_noalloc_dev": (C.c_int, [_vp, _sz, _sz, _vp, _vp, _sz, _vp, _vp]),
    "qg_set_option": (C.c_int, [C.c_char_p, _i64]),
    "qg_get_option": (C.c_int, [C.c_char_p, C.POINTER(_i64)]),
    "qg_server_create": (C.c_int, [_vp, C.c_int, C.c_int, _sz, C.POINTER(_vp)]),
    "qg_server_add_filter": (C.c_int, [_vp, _vp, _sz, C.POINTER(C.c_int)]),
    "qg_server_submit": (C.c_int, [_vp, _vp, _sz, C.c_int, _vp, _sz, C.c_int, C.POINTER(C.c_uint64)]),
    "qg_server_wait": (C.c_int, [_vp, C.c_uint64, _vp, _vp, C.POINTER(C.c_double)]),
    "qg_server_replay": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "qg_server_stats": (C.c_int, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "qg_server_free": (None, [_vp]),
    "qg_symmetric_eigen": (C.c_int, [_vp, _sz, _vp, _vp]),
    "qg_balanced_rotation": (C.c_int, [_vp, _sz, _sz, _vp]),
}

EXPORTS = tuple(_SIGS)

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

OK, INVALID_ARGUMENT, LOGIC_ERROR, RUNTIME_ERROR, CUDA_ERROR, OUT_OF_MEMORY, UNSUPPORTED = range(7)


class CudaError(RuntimeError):
    """A CUDA call inside the library failed (no device, a launch error, ...)."""


def check(rc: int) -> None:
    """Raises the exception class the reference's Python layer uses for the
    same failure (reference bindings: invalid_argument -> ValueError,
    logic_error / runtime_error -> RuntimeError)."""
    if rc == OK:
        return
    msg = lib.qg_last_error().decode()
    if rc == INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc in (LOGIC_ERROR, RUNTIME_ERROR):
        raise RuntimeError(msg)
    if rc == CUDA_ERROR:
        raise CudaError(msg)
    if rc == OUT_OF_MEMORY:
        raise MemoryError(msg)
    if rc == UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)

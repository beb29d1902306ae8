"""Kernel timing and launch counts of the qann_b200 library (CUDA events
recorded on the stream each kernel runs on)."""
from __future__ import annotations

import ctypes as C

from . import _lib

KERNELS = ("pair_scores", "select_rows", "coarse_mm", "coarse_recheck", "probe_terms", "query_tables", "scan", "merge",
           "refine", "rank_lists", "probe_walk", "mm_filter", "tscan_prep", "tscan", "tscan_final")


def enable(on: bool = True) -> None:
    _lib.check(_lib.lib.qg_profile_enable(int(on)))


def reset() -> None:
    _lib.check(_lib.lib.qg_profile_reset())


def get(kernel: str):
    """(total milliseconds, launches) of one kernel since the last reset."""
    ms, n = C.c_double(), C.c_int64()
    _lib.check(_lib.lib.qg_profile_get(kernel.encode(), C.byref(ms), C.byref(n)))
    return ms.value, n.value


def launch_count() -> int:
    """Kernel launches by this library since it was loaded."""
    return int(_lib.lib.qg_launch_count())

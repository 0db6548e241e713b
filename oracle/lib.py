"""ctypes bindings of oracle/_build/liboracle.so — test infrastructure only."""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def load():
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = ctypes.CDLL(path)
        _lib.oracle_collatz_steps.restype = ctypes.c_uint32
        _lib.oracle_collatz_steps.argtypes = [ctypes.c_uint64]
        _lib.oracle_collatz_range.restype = None
        _lib.oracle_collatz_range.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    return _lib


def collatz_range(start, count):
    """Stopping times of start .. start+count-1 (uint32 array)."""
    out = np.zeros(count, dtype=np.uint32)
    load().oracle_collatz_range(start, count, out.ctypes.data)
    return out

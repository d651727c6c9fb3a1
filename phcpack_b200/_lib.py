"""Loader of the CUDA library (libphcb200.so, C ABI in include/phc_b200.h).

The library is built in-tree by ``phcpack_b200.build``.  There is no CPU
fallback: if the library cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

_lock = threading.Lock()
_lib = None

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p


class PhcError(RuntimeError):
    """An entry point returned a negative status."""

    def __init__(self, name: str, rc: int, msg: str):
        super().__init__(f"{name} failed with status {rc}: {msg}")
        self.rc = rc


def lib() -> ctypes.CDLL:
    """Load the library, building it first when the sources are newer."""
    global _lib
    with _lock:
        if _lib is None:
            if _build.stale():
                _build.build()
            _lib = ctypes.CDLL(_build.LIB)
            _lib.phc_last_error.restype = ctypes.c_char_p
        return _lib


def call(name: str, *args) -> int:
    """Call an int-returning entry point; raise PhcError on a negative status."""
    f = getattr(lib(), name)
    f.restype = c_int
    rc = f(*args)
    if rc < 0:
        raise PhcError(name, rc, lib().phc_last_error().decode(errors="replace"))
    return rc


def ptr(x) -> c_void_p:
    """Device or host address of a torch tensor, numpy array or int."""
    if x is None:
        return c_void_p(0)
    if isinstance(x, int):
        return c_void_p(x)
    if hasattr(x, "data_ptr"):
        return c_void_p(x.data_ptr())
    if hasattr(x, "ctypes"):
        return c_void_p(x.ctypes.data)
    raise TypeError(f"cannot take the address of {type(x)}")

"""Locating the in-tree native builds.

The product has no CPU fallback: if the extension or the C-ABI library is
missing, importing the API raises ImportError with the build command.
"""
from __future__ import annotations

import ctypes
import importlib
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcumpm_b200.so")

_ext = None
_lib = None


def extension():
    """The pybind11 module ``cumpm_b200._cuMPM``."""
    global _ext
    if _ext is None:
        try:
            _ext = importlib.import_module("cumpm_b200._cuMPM")
        except ImportError as e:  # pragma: no cover - exercised only on broken installs
            raise ImportError("cumpm_b200 native extension is not built; run `python cumpm_b200/build.py` "
                              f"({e})") from e
    return _ext


def library():
    """ctypes handle of ``libcumpm_b200.so`` (the C ABI of include/cumpm_b200.h)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcumpm_b200.so is not built; run `python cumpm_b200/build.py`")
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib

"""Loads libapocharmm_c.so (the C ABI of this package).

Mirrors the reference's python/apocharmm/_lib.py: the library path may be
given with APOCHARMM_LIBRARY_PATH; by default the in-tree build next to this
file is used.  There is no fallback: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIBRARY = os.path.join(_HERE, "libapocharmm_c.so")

_library = None


class ApoCharmmError(RuntimeError):
    """A C entry point returned a status other than APO_STATUS_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "RUNTIME_ERROR", 3: "CUDA_ERROR",
                4: "NOT_INITIALIZED", 5: "NOT_IMPLEMENTED"}


def library_path() -> str:
    return os.environ.get("APOCHARMM_LIBRARY_PATH") or DEFAULT_LIBRARY


def lib() -> ctypes.CDLL:
    global _library
    if _library is None:
        path = library_path()
        if not os.path.exists(path):
            raise RuntimeError(
                f"libapocharmm_c.so not found at {path}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`make -C apocharmm_b200/csrc`")
        _library = ctypes.CDLL(path)
        _library.apo_last_error.argtypes = []
        _library.apo_last_error.restype = ctypes.c_char_p
    return _library


def check(status: int, what: str) -> None:
    if status != 0:
        msg = lib().apo_last_error()
        text = msg.decode() if msg else ""
        raise ApoCharmmError(status, f"{what} failed with {STATUS_NAMES.get(status, status)}: {text}")


def call(name: str, *args):
    """Calls a status-returning entry point and raises on failure."""
    fn = getattr(lib(), name)
    fn.restype = ctypes.c_int
    check(fn(*args), name)

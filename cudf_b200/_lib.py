"""Loads libgbx.so (the sm_100a kernels behind the C ABI).

There is no fallback: if the shared library is missing or lacks a symbol the
import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgbx.so")

_lib = None


class GbxError(RuntimeError):
    """Raised for a non-zero gbx_status; mirrors cudf::logic_error / cuda_error."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{_abi.Status(status).name}] {message}")
        self.status = status


class LogicError(GbxError, ValueError):
    """cudf::logic_error (CUDF_EXPECTS / CUDF_FAIL)."""


class UnsupportedError(GbxError, NotImplementedError):
    """A request libcudf would route to its sort-based groupby."""


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libgbx.so not found at {LIB_PATH}; build it with `python -m cudf_b200.build`"
            )
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _abi.SIGNATURES.items():
            fn = getattr(h, name)  # AttributeError if the symbol is missing
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def check(status: int) -> None:
    if status == _abi.Status.OK:
        return
    msg = lib().gbx_last_error().decode(errors="replace")
    if status == _abi.Status.ERR_LOGIC:
        raise LogicError(status, msg)
    if status == _abi.Status.ERR_UNSUPPORTED:
        raise UnsupportedError(status, msg)
    raise GbxError(status, msg)

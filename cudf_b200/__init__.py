"""cudf_b200 -- a B200 (sm_100a) hash groupby-aggregation with libcudf's API.

The compute path is libgbx.so (hand-written CUDA kernels behind a C ABI,
include/gbx.h); this package is the Python host-side mirror of pylibcudf's
groupby interface.  There is no CPU fallback: if libgbx.so is missing the
first use raises ImportError.
"""
from ._abi import BatchMode, Interpolation, Kind, NullPolicy, Sorted, Status, Strategy, Tune, TypeId  # noqa: F401
from ._lib import GbxError, LogicError, UnsupportedError  # noqa: F401
from . import aggregation  # noqa: F401
from .column import Column, Table  # noqa: F401
from .groupby import GroupBy, GroupByRequest, TorchAllocator  # noqa: F401
from .batch import BatchGroupBy, BatchInstance, BatchResult  # noqa: F401
from .server import Server  # noqa: F401

__all__ = [
    "Column", "Table", "GroupBy", "GroupByRequest", "TorchAllocator", "aggregation",
    "BatchGroupBy", "BatchInstance", "BatchResult", "BatchMode", "Tune", "Server",
    "Interpolation", "Kind", "NullPolicy", "Sorted", "Status", "Strategy", "TypeId",
    "GbxError", "LogicError", "UnsupportedError",
]

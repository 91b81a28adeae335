"""ctypes mirror of include/gbx.h (the C ABI of libgbx).

Only type and constant definitions live here; loading the shared library is
done by :mod:`cudf_b200._lib`.
"""
from __future__ import annotations

import ctypes as C
import enum


class TypeId(enum.IntEnum):
    """cudf::type_id (cpp/include/cudf/types.hpp:203-235)."""

    EMPTY = 0
    INT8 = 1
    INT16 = 2
    INT32 = 3
    INT64 = 4
    UINT8 = 5
    UINT16 = 6
    UINT32 = 7
    UINT64 = 8
    FLOAT32 = 9
    FLOAT64 = 10
    BOOL8 = 11
    TIMESTAMP_DAYS = 12
    TIMESTAMP_SECONDS = 13
    TIMESTAMP_MILLISECONDS = 14
    TIMESTAMP_MICROSECONDS = 15
    TIMESTAMP_NANOSECONDS = 16
    DURATION_DAYS = 17
    DURATION_SECONDS = 18
    DURATION_MILLISECONDS = 19
    DURATION_MICROSECONDS = 20
    DURATION_NANOSECONDS = 21
    DICTIONARY32 = 22
    STRING = 23
    LIST = 24
    DECIMAL32 = 25
    DECIMAL64 = 26
    DECIMAL128 = 27
    STRUCT = 28


class Kind(enum.IntEnum):
    """cudf::aggregation::Kind (cpp/include/cudf/aggregation.hpp:86-124)."""

    SUM = 0
    PRODUCT = 1
    MIN = 2
    MAX = 3
    COUNT_VALID = 4
    COUNT_ALL = 5
    ANY = 6
    ALL = 7
    SUM_OF_SQUARES = 8
    MEAN = 9
    M2 = 10
    VARIANCE = 11
    STD = 12
    MEDIAN = 13
    QUANTILE = 14
    ARGMAX = 15
    ARGMIN = 16
    NUNIQUE = 17
    NTH_ELEMENT = 18


class NullPolicy(enum.IntEnum):
    """cudf::null_policy (types.hpp:126)."""

    EXCLUDE = 0
    INCLUDE = 1


class Sorted(enum.IntEnum):
    """cudf::sorted (types.hpp:167)."""

    NO = 0
    YES = 1


class Status(enum.IntEnum):
    OK = 0
    ERR_LOGIC = 1
    ERR_CUDA = 2
    ERR_ALLOC = 3
    ERR_UNSUPPORTED = 4
    ERR_DEVICE = 5


class Strategy(enum.IntEnum):
    AUTO = 0
    PRIVATIZED = 1
    GLOBAL = 2
    PARTITIONED = 3
    WARP = 4
    BUCKETED = 5


# element width in bytes of each fixed-width type (0: not fixed width)
TYPE_WIDTH = {
    TypeId.INT8: 1, TypeId.INT16: 2, TypeId.INT32: 4, TypeId.INT64: 8,
    TypeId.UINT8: 1, TypeId.UINT16: 2, TypeId.UINT32: 4, TypeId.UINT64: 8,
    TypeId.FLOAT32: 4, TypeId.FLOAT64: 8, TypeId.BOOL8: 1,
    TypeId.TIMESTAMP_DAYS: 4, TypeId.TIMESTAMP_SECONDS: 8, TypeId.TIMESTAMP_MILLISECONDS: 8,
    TypeId.TIMESTAMP_MICROSECONDS: 8, TypeId.TIMESTAMP_NANOSECONDS: 8,
    TypeId.DURATION_DAYS: 4, TypeId.DURATION_SECONDS: 8, TypeId.DURATION_MILLISECONDS: 8,
    TypeId.DURATION_MICROSECONDS: 8, TypeId.DURATION_NANOSECONDS: 8,
    TypeId.DECIMAL32: 4, TypeId.DECIMAL64: 8,
}


class gbx_column_view(C.Structure):
    pass


gbx_column_view._fields_ = [
    ("type_id", C.c_int32),
    ("scale", C.c_int32),
    ("size", C.c_int64),
    ("offset", C.c_int64),
    ("data", C.c_void_p),
    ("null_mask", C.c_void_p),
    ("null_count", C.c_int64),
    ("index_type_id", C.c_int32),
    ("num_children", C.c_int32),
    ("dict_keys", C.POINTER(gbx_column_view)),
]


class gbx_table_view(C.Structure):
    _fields_ = [
        ("num_columns", C.c_int32),
        ("reserved0", C.c_int32),
        ("columns", C.POINTER(gbx_column_view)),
    ]


class NullEquality(enum.IntEnum):
    """cudf::null_equality (types.hpp:151-154)."""

    EQUAL = 0
    UNEQUAL = 1


class NanEquality(enum.IntEnum):
    """cudf::nan_equality (types.hpp:143-146)."""

    ALL_EQUAL = 0
    UNEQUAL = 1


class JoinKind(enum.IntEnum):
    """gbx_join_kind: the joins of cudf::inner_join / left_join / full_join /
    left_semi_join / left_anti_join (join.hpp:107-260)."""

    INNER = 0
    LEFT = 1
    FULL = 2
    LEFT_SEMI = 3
    LEFT_ANTI = 4


class DuplicateKeep(enum.IntEnum):
    """cudf::duplicate_keep_option (stream_compaction.hpp:225-230)."""

    KEEP_ANY = 0
    KEEP_FIRST = 1
    KEEP_LAST = 2
    KEEP_NONE = 3


class Interpolation(enum.IntEnum):
    """cudf::interpolation (types.hpp:192-198), for QUANTILE."""

    LINEAR = 0
    LOWER = 1
    HIGHER = 2
    MIDPOINT = 3
    NEAREST = 4


class gbx_aggregation(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("ddof", C.c_int32),
        ("null_policy", C.c_int32),
        ("interpolation", C.c_int32),
        ("num_quantiles", C.c_int32),
        ("reserved0", C.c_int32),
        ("quantiles", C.POINTER(C.c_double)),
    ]


def fill_aggregation(dst: "gbx_aggregation", agg, keep: list) -> None:
    """Writes one aggregation -- an object with .kind/.ddof (and optionally
    .null_policy, .interpolation, .quantiles) or a (kind, ddof[, extra]) tuple,
    extra a dict of those fields -- into a gbx_aggregation; arrays it
    allocates are appended to `keep`."""
    if isinstance(agg, tuple):
        kind, ddof = agg[0], agg[1]
        extra = agg[2] if len(agg) > 2 else {}
        null_policy = extra.get("null_policy", 0)
        interp = extra.get("interpolation", 0)
        quantiles = tuple(extra.get("quantiles", ()))
    else:
        kind, ddof = agg.kind, agg.ddof
        null_policy = getattr(agg, "null_policy", 0)
        interp = getattr(agg, "interpolation", 0)
        quantiles = tuple(getattr(agg, "quantiles", ()))
    dst.kind = int(kind)
    dst.ddof = int(ddof)
    dst.null_policy = int(null_policy)
    dst.interpolation = int(interp)
    dst.num_quantiles = len(quantiles)
    if quantiles:
        arr = (C.c_double * len(quantiles))(*[float(q) for q in quantiles])
        keep.append(arr)
        dst.quantiles = C.cast(arr, C.POINTER(C.c_double))
    else:
        dst.quantiles = None


def aggregation_array(aggs):
    """A gbx_aggregation array for `aggs` and the objects it borrows."""
    keep = []
    arr = (gbx_aggregation * max(1, len(aggs)))()
    for j, a in enumerate(aggs):
        fill_aggregation(arr[j], a, keep)
    keep.append(arr)
    return arr, keep


class gbx_request(C.Structure):
    _fields_ = [
        ("values", gbx_column_view),
        ("num_aggregations", C.c_int32),
        ("reserved0", C.c_int32),
        ("aggregations", C.POINTER(gbx_aggregation)),
    ]


ALLOC_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)
DEALLOC_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


class gbx_allocator(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("allocate", ALLOC_FN), ("deallocate", DEALLOC_FN)]


class gbx_column(C.Structure):
    _fields_ = [
        ("view", gbx_column_view),
        ("data", C.c_void_p),
        ("null_mask", C.c_void_p),
        ("data_bytes", C.c_size_t),
        ("mask_bytes", C.c_size_t),
    ]


class gbx_aggregation_result(C.Structure):
    _fields_ = [
        ("num_results", C.c_int32),
        ("reserved0", C.c_int32),
        ("results", C.POINTER(gbx_column)),
    ]


class gbx_result(C.Structure):
    _fields_ = [
        ("num_groups", C.c_int64),
        ("num_key_columns", C.c_int32),
        ("num_requests", C.c_int32),
        ("keys", C.POINTER(gbx_column)),
        ("requests", C.POINTER(gbx_aggregation_result)),
        ("internal", C.c_void_p),
    ]


class gbx_stats(C.Structure):
    _fields_ = [
        ("num_rows", C.c_int64),
        ("num_groups", C.c_int64),
        ("estimated_groups", C.c_int64),
        ("table_capacity", C.c_int64),
        ("strategy", C.c_int32),
        ("retries", C.c_int32),
        ("scratch_bytes", C.c_int64),
        ("kernel_launches", C.c_int32),
        ("timed", C.c_int32),
        ("sample_ms", C.c_float),
        ("init_ms", C.c_float),
        ("aggregate_ms", C.c_float),
        ("compact_ms", C.c_float),
        ("finalize_ms", C.c_float),
        ("total_ms", C.c_float),
        ("partition_bits", C.c_int32),
        ("bucket_slots", C.c_int32),
        ("partition_ms", C.c_float),
        ("reserved1", C.c_int32),
    ]


class BatchMode(enum.IntEnum):
    """gbx_batch_mode."""

    AUTO = 0
    SHARED = 1
    WARP = 2
    GLOBAL = 3


class Tune(enum.IntEnum):
    """gbx_batch_tune."""

    OFF = 0
    CACHED = 1
    MISSING = 2
    ALL = 3


class gbx_batch_instance(C.Structure):
    _fields_ = [("keys", gbx_table_view), ("requests", C.POINTER(gbx_request))]


class gbx_batch_options(C.Structure):
    _fields_ = [
        ("null_policy", C.c_int32),
        ("tune", C.c_int32),
        ("tune_file", C.c_char_p),
        ("force_mode", C.c_int32),
        ("block_threads", C.c_int32),
        ("one_shot", C.c_int32),
        ("tile_rows", C.c_int64),
    ]


class gbx_batch_output(C.Structure):
    _fields_ = [
        ("num_instances", C.c_int32),
        ("reserved", C.c_int32),
        ("group_offsets", C.POINTER(C.c_int64)),
        ("device_group_offsets", C.c_void_p),
        ("columns", gbx_result),
    ]


class gbx_batch_stats(C.Structure):
    _fields_ = [
        ("num_instances", C.c_int32),
        ("block_threads", C.c_int32),
        ("grid", C.c_int32),
        ("work_items", C.c_int32),
        ("num_rows", C.c_int64),
        ("num_groups", C.c_int64),
        ("dynamic_smem", C.c_int64),
        ("arena_bytes", C.c_int64),
        ("output_rows", C.c_int64),
        ("mode_count", C.c_int32 * 4),
        ("classes", C.c_int32),
        ("classes_measured", C.c_int32),
        ("classes_cached", C.c_int32),
        ("retries", C.c_int32),
        ("graph_nodes", C.c_int32),
        ("kernels_per_execute", C.c_int32),
        ("create_ms", C.c_float),
        ("tune_ms", C.c_float),
        ("execute_ms", C.c_float),
        ("init_ms", C.c_float),
        ("aggregate_ms", C.c_float),
        ("output_ms", C.c_float),
    ]


class gbx_server_options(C.Structure):
    _fields_ = [
        ("workers", C.c_int32),
        ("null_policy", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("batch_max_rows", C.c_int64),
        ("batch_max_requests", C.c_int32),
        ("large_in_flight", C.c_int32),
        ("large_rows", C.c_int64),
    ]


class gbx_server_timing(C.Structure):
    _fields_ = [
        ("submitted_s", C.c_double),
        ("admitted_s", C.c_double),
        ("done_s", C.c_double),
        ("reserved_bytes", C.c_int64),
        ("batched", C.c_int32),
        ("worker", C.c_int32),
    ]


class gbx_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("batches", C.c_int64),
        ("batched_requests", C.c_int64),
        ("peak_reserved_bytes", C.c_int64),
        ("rows", C.c_int64),
        ("max_in_flight", C.c_int32),
        ("workers", C.c_int32),
        ("busy_s", C.c_double),
    ]


# Every entry point include/gbx.h declares, with (restype, argtypes).
SIGNATURES = {
    "gbx_batch_create": (
        C.c_int,
        [C.POINTER(gbx_batch_instance), C.c_int32, C.c_int32, C.POINTER(gbx_batch_options), C.c_void_p,
         C.POINTER(gbx_allocator), C.POINTER(C.c_void_p)],
    ),
    "gbx_batch_execute": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.POINTER(gbx_batch_output))]),
    "gbx_batch_rebind": (C.c_int, [C.c_void_p, C.POINTER(gbx_batch_instance), C.c_int32]),
    "gbx_batch_instance_plan": (
        C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "gbx_batch_last_stats": (C.c_int, [C.c_void_p, C.POINTER(gbx_batch_stats)]),
    "gbx_batch_destroy": (None, [C.c_void_p]),
    "gbx_server_create": (C.c_int, [C.POINTER(gbx_server_options), C.POINTER(C.c_void_p)]),
    "gbx_server_submit": (
        C.c_int, [C.c_void_p, C.POINTER(gbx_table_view), C.POINTER(gbx_request), C.c_int32, C.POINTER(C.c_uint64)]),
    "gbx_server_wait": (
        C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.POINTER(gbx_result)), C.POINTER(gbx_server_timing)]),
    "gbx_server_now": (C.c_double, [C.c_void_p]),
    "gbx_server_last_stats": (C.c_int, [C.c_void_p, C.POINTER(gbx_server_stats)]),
    "gbx_server_destroy": (None, [C.c_void_p]),
    "gbx_groupby_create": (C.c_int, [C.POINTER(gbx_table_view), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "gbx_groupby_aggregate": (
        C.c_int,
        [C.c_void_p, C.POINTER(gbx_request), C.c_int32, C.c_void_p, C.POINTER(gbx_allocator),
         C.POINTER(C.POINTER(gbx_result))],
    ),
    "gbx_can_use_hash_groupby": (C.c_int, [C.POINTER(gbx_request), C.c_int32]),
    "gbx_target_type": (C.c_int32, [C.c_int32, C.c_int32]),
    "gbx_result_release": (None, [C.POINTER(gbx_result)]),
    "gbx_groupby_destroy": (None, [C.c_void_p]),
    "gbx_last_error": (C.c_char_p, []),
    "gbx_abi_version": (C.c_int32, []),
    "gbx_groupby_set_strategy": (C.c_int, [C.c_void_p, C.c_int32]),
    "gbx_groupby_last_stats": (C.c_int, [C.c_void_p, C.POINTER(gbx_stats)]),
    "gbx_groupby_set_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "gbx_distinct_count": (
        C.c_int, [C.POINTER(gbx_table_view), C.c_int32, C.c_void_p, C.POINTER(gbx_allocator), C.POINTER(C.c_int64)]),
    "gbx_distinct_indices": (
        C.c_int, [C.POINTER(gbx_table_view), C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(gbx_allocator),
                  C.POINTER(gbx_column)]),
    "gbx_distinct_join": (
        C.c_int, [C.POINTER(gbx_table_view), C.POINTER(gbx_table_view), C.c_int32, C.c_int32, C.c_void_p,
                  C.POINTER(gbx_allocator), C.POINTER(gbx_column), C.POINTER(gbx_column)]),
    "gbx_hash_join": (
        C.c_int, [C.POINTER(gbx_table_view), C.POINTER(gbx_table_view), C.c_int32, C.c_int32, C.c_void_p,
                  C.POINTER(gbx_allocator), C.POINTER(gbx_column), C.POINTER(gbx_column)]),
    "gbx_column_release": (None, [C.POINTER(gbx_column), C.POINTER(gbx_allocator), C.c_void_p]),
    "gbx_groupby_aggregate_noalloc": (
        C.c_int,
        [C.c_void_p, C.POINTER(gbx_request), C.c_int32, C.c_void_p, C.POINTER(gbx_column), C.POINTER(gbx_column),
         C.c_int64, C.POINTER(C.c_int64)],
    ),
}

NOALLOC_SCRATCH_BYTES = 16 << 20
NOALLOC_MAX_GROUPS = 32768

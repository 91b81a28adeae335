"""Aggregation factories mirroring pylibcudf.aggregation / cudf::make_*_aggregation
(cpp/include/cudf/aggregation.hpp:261-337, python/cudf/cudf/_lib/pylibcudf/aggregation.pyx:157-403)."""
from __future__ import annotations

from dataclasses import dataclass

from ._abi import Kind, NullPolicy


@dataclass(frozen=True)
class Aggregation:
    kind: Kind
    ddof: int = 0

    def __repr__(self):
        return f"Aggregation({self.kind.name}{', ddof=%d' % self.ddof if self.kind in (Kind.VARIANCE, Kind.STD) else ''})"


def sum() -> Aggregation:  # noqa: A001 - mirrors the reference name
    return Aggregation(Kind.SUM)


def product() -> Aggregation:
    return Aggregation(Kind.PRODUCT)


def min() -> Aggregation:  # noqa: A001
    return Aggregation(Kind.MIN)


def max() -> Aggregation:  # noqa: A001
    return Aggregation(Kind.MAX)


def count(null_handling: NullPolicy = NullPolicy.EXCLUDE) -> Aggregation:
    """COUNT_VALID for EXCLUDE, COUNT_ALL for INCLUDE (cpp/src/aggregation/aggregation.cpp:494-499)."""
    return Aggregation(Kind.COUNT_VALID if null_handling == NullPolicy.EXCLUDE else Kind.COUNT_ALL)


def sum_of_squares() -> Aggregation:
    return Aggregation(Kind.SUM_OF_SQUARES)


def mean() -> Aggregation:
    return Aggregation(Kind.MEAN)


def variance(ddof: int = 1) -> Aggregation:
    return Aggregation(Kind.VARIANCE, ddof)


def std(ddof: int = 1) -> Aggregation:
    return Aggregation(Kind.STD, ddof)


def argmax() -> Aggregation:
    return Aggregation(Kind.ARGMAX)


def argmin() -> Aggregation:
    return Aggregation(Kind.ARGMIN)


def nth_element(n: int) -> Aggregation:
    return Aggregation(Kind.NTH_ELEMENT, n)


def median() -> Aggregation:
    return Aggregation(Kind.MEDIAN)

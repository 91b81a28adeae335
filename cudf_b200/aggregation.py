"""Aggregation factories mirroring pylibcudf.aggregation / cudf::make_*_aggregation
(cpp/include/cudf/aggregation.hpp:261-337, python/cudf/cudf/_lib/pylibcudf/aggregation.pyx:157-403)."""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence, Tuple

from ._abi import Interpolation, Kind, NullPolicy


@dataclass(frozen=True)
class Aggregation:
    """One aggregation of a request.  `ddof` is VARIANCE/STD's delta degrees of
    freedom and NTH_ELEMENT's n; `null_policy` is NUNIQUE's and NTH_ELEMENT's
    null handling; `interpolation` and `quantiles` are QUANTILE's."""

    kind: Kind
    ddof: int = 0
    null_policy: NullPolicy = NullPolicy.EXCLUDE
    interpolation: Interpolation = Interpolation.LINEAR
    quantiles: Tuple[float, ...] = ()

    def __repr__(self):
        extra = ""
        if self.kind in (Kind.VARIANCE, Kind.STD):
            extra = f", ddof={self.ddof}"
        elif self.kind == Kind.NTH_ELEMENT:
            extra = f", n={self.ddof}, null_handling={NullPolicy(self.null_policy).name}"
        elif self.kind == Kind.NUNIQUE:
            extra = f", null_handling={NullPolicy(self.null_policy).name}"
        elif self.kind == Kind.QUANTILE:
            extra = f", quantiles={list(self.quantiles)}, interp={Interpolation(self.interpolation).name}"
        return f"Aggregation({self.kind.name}{extra})"


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


def m2() -> Aggregation:
    """Sum of squared deviations from the group mean (make_m2_aggregation)."""
    return Aggregation(Kind.M2)


def median() -> Aggregation:
    """QUANTILE 0.5 with LINEAR interpolation (groupby/sort/aggregate.cpp:344-362)."""
    return Aggregation(Kind.MEDIAN)


def quantile(quantiles: Sequence[float], interp: Interpolation = Interpolation.LINEAR) -> Aggregation:
    """make_quantile_aggregation (aggregation.hpp:364): the result column has
    len(quantiles) rows per group, group by group."""
    return Aggregation(Kind.QUANTILE, interpolation=Interpolation(interp), quantiles=tuple(float(q) for q in quantiles))


def nunique(null_handling: NullPolicy = NullPolicy.EXCLUDE) -> Aggregation:
    """Distinct values per group; under INCLUDE the nulls count as one value
    (make_nunique_aggregation, aggregation.hpp:397)."""
    return Aggregation(Kind.NUNIQUE, null_policy=NullPolicy(null_handling))


def nth_element(n: int, null_handling: NullPolicy = NullPolicy.INCLUDE) -> Aggregation:
    """The n-th row of each group in row order (negative n counts from the
    end); EXCLUDE drops null values first (make_nth_element_aggregation,
    aggregation.hpp:410-411)."""
    return Aggregation(Kind.NTH_ELEMENT, n, null_policy=NullPolicy(null_handling))

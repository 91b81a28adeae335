"""Seeded synthetic inputs with the shapes and distributions of the groupby
benchmark workloads (plain: 10M / 100M / 200M rows; batched: 4,096
instances; served: a Poisson request stream).  No public dataset is used.

Every generator takes the row count so the same distribution serves the
full-size benchmark and the small parity cases.  Seeds are 20241003 + the
workload number.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

SEED0 = 20241003


@dataclass
class PlainInput:
    """Key columns and value columns as host numpy arrays (validity optional)."""

    keys: List[np.ndarray]
    key_valid: List[Optional[np.ndarray]]
    values: List[np.ndarray]
    value_valid: List[Optional[np.ndarray]]
    name: str

    @property
    def rows(self) -> int:
        return len(self.keys[0])

    def input_bytes(self) -> int:
        b = 0
        for a, m in zip(self.keys + self.values, self.key_valid + self.value_valid):
            b += a.nbytes + (0 if m is None else (len(m) + 7) // 8)
        return b


def plain_10m(n: int = 10_000_000, seed: int = SEED0 + 1) -> PlainInput:
    """int32 key uniform over 1,000 values; float64 ~N(0,1); no nulls."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 1000, size=n, dtype=np.int32)
    v = rng.standard_normal(n)
    return PlainInput([k], [None], [v], [None], f"plain int32 key, 1e3 groups, {n} rows")


def plain_100m(cardinality: int, n: int = 100_000_000, seed: int = SEED0 + 2) -> PlainInput:
    """int64 key uniform over `cardinality`; int64 uniform in [-1e6, 1e6];
    float32 ~N(0,1) with 10% nulls (Bernoulli)."""
    rng = np.random.default_rng(seed + cardinality)
    k = rng.integers(0, cardinality, size=n, dtype=np.int64)
    a = rng.integers(-1_000_000, 1_000_000, size=n, dtype=np.int64, endpoint=True)
    b = rng.standard_normal(n, dtype=np.float32)
    bv = rng.random(n) >= 0.10
    return PlainInput([k], [None], [a, b], [None, bv], f"plain int64 key, C={cardinality:g}, {n} rows")


def zipf_ranks(rng, n: int, s: float = 1.2, ranks: int = 100_000) -> np.ndarray:
    """Inverse-CDF sampling of a Zipf(s) law truncated to `ranks` ranks (0-based)."""
    w = np.arange(1, ranks + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = rng.random(n)
    return np.minimum(np.searchsorted(cdf, u, side="right"), ranks - 1)


@dataclass
class BatchSpec:
    """Per-instance row counts and key cardinalities of a batched workload."""

    rows: np.ndarray
    cards: np.ndarray
    seed: int

    @property
    def num_instances(self) -> int:
        return len(self.rows)

    @property
    def total_rows(self) -> int:
        return int(self.rows.sum())


def batched_spec(num_instances: int = 4096, rows_range=(1e3, 1e6), card_range=(10, 1e4),
                 seed: int = SEED0 + 4) -> BatchSpec:
    """Row counts log-uniform in rows_range, cardinalities log-uniform in
    card_range (floored), one draw per instance."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log10(rows_range[0]), np.log10(rows_range[1])
    rows = np.floor(10.0 ** rng.uniform(lo, hi, num_instances)).astype(np.int64)
    clo, chi = np.log10(card_range[0]), np.log10(card_range[1])
    cards = np.maximum(1, np.floor(10.0 ** rng.uniform(clo, chi, num_instances))).astype(np.int64)
    return BatchSpec(rows, cards, seed)


def batched_instance(spec: BatchSpec, i: int):
    """Instance i on the host: int32 key uniform in [0, C_i), int64 value
    uniform in [0, 1e9]."""
    rng = np.random.default_rng([spec.seed, i])
    n = int(spec.rows[i])
    k = rng.integers(0, int(spec.cards[i]), size=n, dtype=np.int32)
    v = rng.integers(0, 1_000_000_000, size=n, dtype=np.int64, endpoint=True)
    return k, v


def plain_200m(n: int = 200_000_000, seed: int = SEED0 + 3, ranks: int = 100_000) -> PlainInput:
    """Composite (int32, int16) key, joint index Zipf(1.2) over `ranks` distinct
    pairs; 2% nulls per key column; float64 ~LogNormal(0, 1)."""
    rng = np.random.default_rng(seed)
    # fixed random distinct pairs
    pairs = set()
    k1 = np.empty(ranks, np.int32)
    k2 = np.empty(ranks, np.int16)
    i = 0
    while i < ranks:
        a = int(rng.integers(-2**31, 2**31 - 1))
        b = int(rng.integers(-2**15, 2**15 - 1))
        if (a, b) in pairs:
            continue
        pairs.add((a, b))
        k1[i], k2[i] = a, b
        i += 1
    j = zipf_ranks(rng, n, 1.2, ranks)
    c1 = k1[j]
    c2 = k2[j]
    v1 = rng.random(n) >= 0.02
    v2 = rng.random(n) >= 0.02
    v = rng.lognormal(0.0, 1.0, n)
    return PlainInput([c1, c2], [v1, v2], [v], [None], f"plain (int32,int16) Zipf(1.2) key, {n} rows")


# ------------------------------------------------------- device-side inputs
# The benchmark generates its full-size inputs on the device (seconds instead
# of minutes on the host); the full-size parity tests copy the same columns
# back to the host for the oracle.

def _bitmask_device(valid):
    """Bool tensor -> cudf bitmask words (int32, LSB-first) padded to 64 bytes."""
    import torch

    n = valid.numel()
    nbits = ((n + 511) // 512) * 512
    v = torch.zeros(nbits, dtype=torch.int64, device=valid.device)
    v[:n] = valid.to(torch.int64)
    w = (v.view(-1, 32) << torch.arange(32, device=valid.device, dtype=torch.int64)).sum(dim=1)
    return torch.where(w >= (1 << 31), w - (1 << 32), w).to(torch.int32)


def plain_100m_device(card: int, n: int, seed: int, device):
    """The 100M-row workload (int64 key uniform over `card` values, int64 a in
    [-1e6, 1e6], float32 b ~N(0,1) with 10% nulls) generated on `device`.
    Returns (key, a, b) Columns."""
    import torch

    from .column import Column
    from ._abi import TypeId

    g = torch.Generator(device=device)
    g.manual_seed(seed * 1_000_003 + card)
    k = torch.randint(0, card, (n,), generator=g, device=device, dtype=torch.int64)
    a = torch.randint(-1_000_000, 1_000_001, (n,), generator=g, device=device, dtype=torch.int64)
    b = torch.randn(n, generator=g, device=device, dtype=torch.float32)
    bvalid = torch.rand(n, generator=g, device=device) >= 0.10
    words = _bitmask_device(bvalid)
    nulls = int(n - int(bvalid.sum().item()))
    return (Column(TypeId.INT64, n, k), Column(TypeId.INT64, n, a),
            Column(TypeId.FLOAT32, n, b, words, 0, nulls))


def plain_200m_device(n: int, seed: int, device, ranks: int = 100_000, s: float = 1.2):
    """The 200M-row composite-key workload generated on `device`: `ranks`
    fixed random distinct (int32, int16) pairs (drawn on the host, seeded),
    the joint key index Zipf(s) by inverse-CDF sampling, 2% nulls per key
    column (independent Bernoulli), float64 value ~LogNormal(0, 1).
    Returns (k32, k16, v) Columns."""
    import torch

    from .column import Column
    from ._abi import TypeId

    rng = np.random.default_rng(seed)
    # distinct pairs: draw with replacement, keep first occurrences, top up
    a = np.empty(0, np.int64)
    b = np.empty(0, np.int64)
    while len(a) < ranks:
        ca = rng.integers(-2**31, 2**31 - 1, size=2 * ranks)
        cb = rng.integers(-2**15, 2**15 - 1, size=2 * ranks)
        a = np.concatenate([a, ca])
        b = np.concatenate([b, cb])
        joint = (a << 16) ^ (b & 0xffff)
        _, first = np.unique(joint, return_index=True)
        first.sort()
        a, b = a[first], b[first]
    pa = torch.from_numpy(a[:ranks].astype(np.int32)).to(device)
    pb = torch.from_numpy(b[:ranks].astype(np.int16)).to(device)
    w = torch.arange(1, ranks + 1, dtype=torch.float64, device=device) ** (-s)
    cdf = torch.cumsum(w, 0)
    cdf /= cdf[-1].clone()
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    j = torch.empty(n, dtype=torch.int64, device=device)
    chunk = 1 << 26
    for lo in range(0, n, chunk):
        hi = min(n, lo + chunk)
        u = torch.rand(hi - lo, generator=g, device=device, dtype=torch.float64)
        j[lo:hi] = torch.clamp(torch.searchsorted(cdf, u, right=True), max=ranks - 1)
    k32 = pa[j]
    k16 = pb[j]
    del j
    v1 = torch.rand(n, generator=g, device=device) >= 0.02
    v2 = torch.rand(n, generator=g, device=device) >= 0.02
    v = torch.randn(n, generator=g, device=device, dtype=torch.float64).exp_()
    m1, m2 = _bitmask_device(v1), _bitmask_device(v2)
    n1, n2 = int(n - int(v1.sum().item())), int(n - int(v2.sum().item()))
    del v1, v2
    return (Column(TypeId.INT32, n, k32, m1, 0, n1), Column(TypeId.INT16, n, k16, m2, 0, n2),
            Column(TypeId.FLOAT64, n, v))

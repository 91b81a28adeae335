"""cudf_b200.stream_compaction.gather (the helper that turns the library's
row indices into rows) on host tensors: fixed-width, STRING (offsets and
characters rebuilt, sliced input) and STRUCT (members gathered under the
struct's own mask) columns."""
from __future__ import annotations

import numpy as np

from cudf_b200 import stream_compaction as sc
from cudf_b200.column import Column


def _idx(v):
    return Column.from_numpy(np.array(v, np.int32), device="cpu")


def test_fixed_width_and_mask():
    c = Column.from_numpy(np.arange(10, dtype=np.int64), np.arange(10) % 3 != 0, device="cpu")
    vals, valid = sc.gather(c, _idx([9, 0, 4, 4])).to_numpy()
    assert list(vals) == [9, 0, 4, 4] and list(valid) == [False, False, True, True]


def test_strings_sliced_and_empty():
    s = Column.from_strings(["", "a", "bb", None, "año", "xyz"], device="cpu")
    vals, valid = sc.gather(s.slice(1, 6), _idx([3, 0, 2, 1, 3])).to_numpy()
    assert list(vals) == ["año", "a", "", "bb", "año"]
    assert list(valid) == [True, True, False, True, True]
    vals, _ = sc.gather(s, _idx([])).to_numpy()
    assert len(vals) == 0


def test_struct_members_and_mask():
    a = Column.from_numpy(np.array([1, 2, 3, 4], np.int32), np.array([1, 1, 0, 1], bool), device="cpu")
    s = Column.from_strings(["w", "x", "y", "z"], device="cpu")
    st = Column.struct([a, s], np.array([1, 0, 1, 1], bool), device="cpu")
    members, valid = sc.gather(st, _idx([2, 1, 3])).to_numpy()
    assert list(valid) == [True, False, True]
    assert list(members[0][0]) == [3, 2, 4] and list(members[0][1]) == [False, True, True]
    assert list(members[1][0]) == ["y", "x", "z"]

"""Distinct rows of STRING and STRUCT keys on the CPU: the distinct oracle
(oracle/distinct.py, over the keys' leaves from oracle/structs.py) against
the reference gtests' known answers (tests/golden/distinct_kats.py)."""
from __future__ import annotations

import numpy as np

from cudf_b200._abi import TypeId
from oracle import distinct as od
from oracle.oracle import HostCol
from oracle.structs import leaves
from tests.golden import distinct_kats as K
from tests.test_struct_keys import host_of


def spec_host(spec):
    """struct_kats column forms, type names allowed for fixed columns."""
    kind = spec[0]
    if kind == "fixed" and isinstance(spec[1], str):
        return host_of(("fixed", TypeId[spec[1].upper()], spec[2], spec[3]))
    if kind == "struct":
        _, members, valid = spec
        return HostCol(None, None if valid is None else np.array(valid, bool), type_id=TypeId.STRUCT,
                       children=[spec_host(m) for m in members])
    return host_of(spec)


def leaf_cols(keys):
    """Each key leaf as (values, valid) for oracle/distinct.py (a struct's
    validity leaf with zeros as values)."""
    n = keys[0].size
    out = []
    for k in keys:
        for leaf in leaves(k, n):
            vals = np.zeros(n, dtype=np.int8) if leaf.values is None else np.asarray(leaf.values)
            out.append((vals, leaf.valid))
    return out


def classes_kept_once(kept, classes):
    kept = set(int(x) for x in kept)
    return len(kept) == len(classes) and all(len(kept & set(c)) == 1 for c in classes)


def test_string_key_column_kat():
    specs, want = K.STRING_KEY_COLUMN
    cols = leaf_cols([spec_host(s) for s in specs])
    for keep, rows in want.items():
        assert list(od.distinct_indices(cols, keep)) == rows
    assert od.distinct_count(cols) == 5


def test_structs_of_structs_kat():
    specs, want = K.STRUCTS_OF_STRUCTS
    cols = leaf_cols([spec_host(s) for s in specs])
    assert classes_kept_once(od.distinct_indices(cols, 0, True), want["equal"])
    assert classes_kept_once(od.distinct_indices(cols, 0, False), want["unequal"])

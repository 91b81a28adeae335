"""Runs the C++ drop-in facade test (tests/cpp/groupby_facade_test.cpp): the
reference's groupby gtest vectors written against cudf::groupby::groupby /
cudf::make_*_aggregation, compiled against include/cudf and libgbx.so."""
from __future__ import annotations

import os
import subprocess

import pytest

from cudf_b200 import build


@pytest.mark.gpu
def test_cpp_facade_reference_style_cases():
    exe = build.FACADE_TEST_BIN
    if not os.path.exists(exe) or os.path.getmtime(exe) < os.path.getmtime(build.FACADE_TEST_SRC):
        build.build_facade_test()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout


def test_cpp_facade_compiles():
    """The drop-in headers compile with caller code written like the reference's."""
    assert os.path.exists(build.build_facade_test())

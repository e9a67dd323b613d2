"""
The C ABI without a GPU: libqpopdiff.so loads, exports every symbol include/qpopdiff.h
declares, plans axes on the host, and reports a missing device as an error code
instead of aborting.
"""

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from qpop_diffraction_b200 import _native, build

HEADER = Path(__file__).resolve().parents[1] / "include" / "qpopdiff.h"


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _native.load()


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"QPD_API\s+[\w\s\*]+?\b(qpd_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared() == sorted(_native.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (qpd_\w+)", out))
    assert set(declared()) <= exported
    # nothing else leaks out of the library's C namespace
    assert exported == set(declared())


@pytest.mark.parametrize("n,expect", [(1, []), (2, [2]), (4, [4]), (16, [4, 4]), (104, [8, 13]), (68, [4, 17]),
                                      (512, [8, 8, 8]), (4000, [8, 4, 5, 5, 5]), (400, [4, 4, 5, 5]),
                                      (37, [37]), (30, [2, 3, 5])])
def test_axis_radices(lib, n, expect):
    r = _native.axis_radices(n)
    assert int(np.prod(r)) == n if n > 1 else r == []
    if n > 1:
        assert sorted(r) == sorted(expect)


def test_no_device_is_an_error_not_an_abort(lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = ctypes.c_void_p()
    rc = lib.qpd_create(0, 0, ctypes.byref(ctx))
    assert rc == _native.QPD_ERR_CUDA or rc == _native.QPD_ERR_ARG
    assert not ctx
    assert lib.qpd_last_error(None)


def test_null_arguments_are_rejected(lib):
    assert lib.qpd_create(0, 0, None) == _native.QPD_ERR_ARG
    assert lib.qpd_plan(None, None, 1, 3, 0, 0) == _native.QPD_ERR_ARG
    assert lib.qpd_run_device(None, None, None, None, None, None, None, None) == _native.QPD_ERR_ARG
    assert lib.qpd_set_cta_tiles(None, 4) == _native.QPD_ERR_ARG
    assert lib.qpd_destroy(None) == _native.QPD_OK

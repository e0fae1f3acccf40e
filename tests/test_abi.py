"""The C-ABI library loads without a GPU and exports every symbol the header declares."""
import ctypes
import re
from pathlib import Path

import pytest

from qmtools import _native as N

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "qmtools_b200.h").read_text()
    return sorted(set(re.findall(r"\b(qmt_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    lib = N.load()
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    declared = set(header_symbols())
    bound = set(N.SIGNATURES) | set(N.OTHER)
    assert declared == bound, (declared - bound, bound - declared)


def test_abi_version_and_error_string():
    lib = N.load()
    assert lib.qmt_abi_version() >= 1
    assert isinstance(lib.qmt_last_error(), bytes)


def test_bad_arguments_rejected_without_device():
    """Argument checks run before any CUDA call: they must report BAD_ARG, not crash."""
    lib = N.load()
    out = ctypes.c_double()
    assert lib.qmt_grid_total(None, 10, ctypes.byref(out), None) == N.BAD_ARG
    assert lib.qmt_density(None, 8, 8, 8, 0.1, 0, 0, 0, 1, 1, 1, None, None, None) == N.BAD_ARG
    assert lib.qmt_jacobi(8, 8, 8, 0.1, None, None, None, 10, 1, 0.0, None, None, None) == N.BAD_ARG
    assert b"Jacobi" in lib.qmt_last_error()


def test_wait_limit_and_launch_count_without_device():
    """The wait limit is checked and set without a device; the launch counter starts at zero
    in a process that has launched nothing (this suite launches nothing)."""
    lib = N.load()
    assert lib.qmt_set_wait_limit_ns(61 * 10 ** 9) == N.BAD_ARG
    assert lib.qmt_set_wait_limit_ns(1000) == N.OK
    assert lib.qmt_set_wait_limit_ns(0) == N.OK
    assert lib.qmt_launch_count() == 0

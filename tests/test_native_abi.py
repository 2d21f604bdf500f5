"""The C-ABI library builds for sm_100a, loads, and exports every entry point of
include/pcb200.h (no GPU calls). CPU only."""

import ctypes
import os
import re

import pytest

from pyjuice_b200 import _native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "pcb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pcb_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_exports_header_symbols():
    nat.build()
    lib = ctypes.CDLL(nat.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    # the Python binding declares exactly the header's functions
    assert sorted(nat.EXPORTED_SYMBOLS) == names


def test_version_and_error_string():
    lib = nat.load()
    assert lib.pcb_version() == 1
    assert isinstance(lib.pcb_last_error(), bytes)


def test_argument_validation_without_gpu():
    """Bad arguments are rejected on the host before any launch."""
    lib = nat.load()
    rc = lib.pcb_fill_rows(None, 0, 0, 1, ctypes.c_float(0.0), None)
    assert rc == -1
    assert b"pcb_fill_rows" in lib.pcb_last_error()
    rc = lib.pcb_sum_em(None, None, None, None, None, None, 1, ctypes.c_double(0.5), ctypes.c_double(0.0), 0, None)
    assert rc == -1

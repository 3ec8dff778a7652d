"""The C ABI library loads without a GPU and exports every entry point include/ld.h declares."""
import ctypes
import pathlib
import re

import pytest

from lucky_droplets_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parent.parent


def header_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        names += re.findall(r"^LD_API\s+[\w\s\*]+?\b(ld_\w+)\s*\(", h.read_text(), flags=re.M)
    return names


def test_header_declares_entry_points():
    names = header_functions()
    assert "ld_plan_create" in names and "ld_rk2if_stage" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    L = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_header():
    assert sorted(_lib.SIGNATURES) == sorted(header_functions())


def test_version_and_argument_errors_without_gpu():
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    L = _lib.lib()
    assert L.ld_version() >= 1
    # argument validation happens before any CUDA call
    h = ctypes.c_void_p()
    assert L.ld_plan_create(ctypes.byref(h), 100, 0) == -3   # LD_ERR_UNSUPPORTED
    assert b"powers of two" in L.ld_last_error() and b"360" in L.ld_last_error()
    assert L.ld_plan_create(ctypes.byref(h), 64, 7) == -1     # LD_ERR_ARG
    assert L.ld_rfft_mpi(None, None, None, 1, None) == -1

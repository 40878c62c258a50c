"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"GNUFFT_API[^;{]*?\b(gnufft_\w+)\s*\(", text,
                                re.S))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "gnufft_plan_create" in names and "gnufft_adjoint_device" in names


def test_library_exports_every_declared_symbol():
    from gpunufft_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        pytest.fail("libgpunufft_b200.so not built (python -m "
                    "gpunufft_b200.build)")
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.EXPORTED) <= set(declared_symbols())


def test_version_and_errors_without_gpu():
    import gpunufft_b200 as G
    assert "sm_100a" in G.version()
    L = G.lib()
    assert L.gnufft_status_string(1) == b"invalid argument"
    # NULL plan pointer is rejected on the host before touching the device
    assert L.gnufft_plan_create(None, None, None, None, None) == 1
    assert b"NULL" in L.gnufft_last_error()

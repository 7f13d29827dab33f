"""The C-ABI library loads and exports every symbol include/litho_b200.h declares (CPU)."""
import ctypes
import importlib
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "litho_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(litho_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def pkg():
    p = importlib.import_module("c-version-lithography_b200")
    if not os.path.exists(p.library_path()):
        importlib.import_module("c-version-lithography_b200.build").build()
    return p


def test_header_declares_entry_points():
    names = declared_functions()
    assert "litho_imaging_compute" in names and "litho_pe_gradient" in names
    assert "litho_lsm_rk2_update" in names and "litho_ctm_evaluate" in names


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.library_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header(pkg):
    """The ctypes host layer binds exactly the header's functions."""
    assert sorted(pkg.SIGNATURES) == declared_functions()
    pkg.load_library()


def test_status_strings(pkg):
    lib = pkg.load_library()
    assert lib.litho_status_string(0) == b"ok"
    assert lib.litho_status_string(3) == b"non-finite input"
    assert lib.litho_version() >= 1


def test_no_device_calls_fail_cleanly(pkg):
    """Without a GPU the context constructor reports a CUDA error instead of crashing."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    assert lib.litho_ctx_create(0, None, ctypes.byref(h)) != 0
    assert not h.value

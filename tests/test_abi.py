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


def declared_prototypes():
    """{name: (return type, [parameter types])} of every function the header declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"#[^\n]*", "", text)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(litho_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        ret = " ".join(m.group(1).split())
        params = [p.strip() for p in m.group(3).split(",")] if m.group(3).strip() != "void" else []
        types = []
        for p in params:
            p = " ".join(p.split())
            # split off the parameter name (the last identifier) unless the type is all there is
            named = re.search(r"[\w\*]\s+\**([A-Za-z_]\w*)$", p)
            t = re.sub(r"\s*\b[A-Za-z_]\w*$", "", p) if named else p
            types.append((t.replace(" *", "*").strip(), named.group(1) if named else ""))
        protos[m.group(2)] = (ret.replace(" *", "*"), types)
    return protos


def ctypes_class(c_type):
    """The ctypes argument class a C parameter type must be bound with."""
    import ctypes as C
    t = c_type.replace("const ", "").strip()
    if t.endswith("*"):
        base = t[:-1].strip()
        return {"double": C.POINTER(C.c_double), "int": C.POINTER(C.c_int),
                "long long": C.POINTER(C.c_longlong), "char": C.c_char_p}.get(base, "pointer")
    return {"int": C.c_int, "double": C.c_double, "long long": C.c_longlong,
            "size_t": C.c_size_t, "float": C.c_float}[t]


def test_binding_signatures_match_the_header(pkg):
    """Every ctypes binding has the header's parameter count, and each parameter the
    class its C type needs: int / long long / double by value, host double* and int* as
    typed pointers, device addresses (d_ names) and any other pointer (handles, float
    buffers, streams, structs) as a pointer."""
    import ctypes as C
    protos = declared_prototypes()
    assert sorted(protos) == declared_functions()
    pointer_like = (C.c_void_p, C.c_char_p)
    for name, (res, args) in pkg.SIGNATURES.items():
        ret, params = protos[name]
        assert len(args) == len(params), (name, params, args)
        want_ret = ctypes_class(ret)
        assert (res is want_ret) or (want_ret == "pointer" and res in pointer_like), (name, ret, res)
        for i, ((p, pname), a) in enumerate(zip(params, args)):
            want = ctypes_class(p)
            if pname.startswith("d_") and p.replace("const ", "").endswith("*"):
                want = "pointer"    # a device address: passed as a plain pointer
            if want == "pointer":
                ok = a in pointer_like or (isinstance(a, type) and issubclass(a, C._Pointer))
            else:
                ok = a is want
            assert ok, (name, i, p, a)

"""The C-ABI library loads and exports every function include/xtn_b200.h declares
(no compute call: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

import xtn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "xtn_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(xtn_\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("xtn_callback")))


def test_header_declares_the_reference_entry_point():
    names = declared_functions()
    assert "xtn_perform" in names
    assert len(names) >= 10


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(xtn.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    assert set(xtn.SYMBOLS) <= set(declared_functions())


def test_version_and_error_strings():
    lib = xtn.load()
    assert lib.xtn_version().decode().startswith("2.0.0")
    assert isinstance(lib.xtn_last_error(), bytes)


def test_argument_errors_need_no_device():
    lib = xtn.load()
    out = ctypes.c_void_p()
    assert lib.xtn_context_create(0, None) == xtn.ERR_ARG
    args = xtn.Args(0, 0, 0, 0)
    cb = xtn.CALLBACK(lambda *a: None)
    # a null context / null inputs are rejected before any CUDA call
    assert lib.xtn_context_perform(None, ctypes.byref(args), None, None, 0, None, cb, None) == xtn.ERR_ARG
    assert lib.xtn_context_nn_device(None, ctypes.byref(args), None, None, 0, None) == xtn.ERR_ARG


def test_index_argument_errors_need_no_device():
    """Invalid index arguments are rejected before any device work."""
    import ctypes

    lib = xtn.load()
    h = ctypes.c_void_p()
    assert lib.xtn_index_create(0, None, None, 0, 2, ctypes.byref(h)) == xtn.ERR_ARG
    chars, offs = xtn.pack_sequences(["CASSF", "CASSG"])
    assert lib.xtn_index_create(0, chars.ctypes.data, offs.ctypes.data, 2, 3, ctypes.byref(h)) == xtn.ERR_ARG
    assert b"maximum distance" in lib.xtn_last_error()
    assert lib.xtn_index_serve(None, None, 0, None, None, xtn.REQUEST_CALLBACK(0), None) == xtn.ERR_ARG


def test_autotune_argument_errors_need_no_device():
    lib = xtn.load()
    args = xtn.Args(1, 0, 0, 0)
    import ctypes

    assert lib.xtn_context_autotune(None, ctypes.byref(args), None, None, 0, 1, None, 0) == xtn.ERR_ARG


def test_every_option_is_documented():
    """The names xtn_context_set_option accepts are exactly the ones the header documents."""
    src = open(os.path.join(ROOT, "xt-neighbor_b200", "csrc", "xtn_engine.cu")).read()
    fn = src[src.index("int xtn_context_set_option(") :]
    fn = fn[: fn.index("\n}\n")]
    accepted = set(re.findall(r'strcmp\(name, "(\w+)"\)', fn))
    hdr = open(HEADER).read()
    block = hdr[hdr.index("Tuning and engine options") : hdr.index("int xtn_context_set_option")]
    documented = set(re.findall(r'^ \*   "(\w+)"', block, flags=re.M))
    assert accepted and accepted == documented

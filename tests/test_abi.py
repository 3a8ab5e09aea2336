"""CPU-only checks of the C ABI: the library loads and exports every entry
point include/mgv.h declares; status strings and error paths work without a
GPU (no compute call is made)."""
import ctypes
import os
import subprocess

import pytest

import mgv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ensure_built():
    if not os.path.exists(mgv.LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.dirname(mgv.LIB_PATH)], check=True)


def test_every_declared_symbol_is_exported():
    ensure_built()
    lib = ctypes.CDLL(mgv.LIB_PATH)
    names = mgv.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    ensure_built()
    lib = mgv.load()
    for n in mgv.header_functions():
        assert getattr(lib, n).argtypes is not None, f"{n} has no ctypes signature"


def test_status_strings():
    ensure_built()
    lib = mgv.load()
    for s in range(9):
        assert lib.mgv_status_string(s)
    assert lib.mgv_status_string(99) == b"unknown status"


def test_null_arguments_are_rejected():
    ensure_built()
    lib = mgv.load()
    assert lib.mgv_ctx_create(0, None) == mgv.EINVAL
    assert lib.mgv_ctx_info_get(None, None) == mgv.EINVAL
    assert lib.mgv_op_open(None, None) == mgv.EINVAL
    assert lib.mgv_pool_create(None, 1, 128, 1, None) == mgv.EINVAL
    assert b"NULL" in lib.mgv_last_error_string()


def test_no_device_is_an_error_not_a_crash():
    ensure_built()
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    st = mgv.load().mgv_ctx_create(0, ctypes.byref(h))
    assert st in (mgv.ECUDA, mgv.EINVAL)
    assert not h.value

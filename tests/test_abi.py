"""The C-ABI library: loads, exports every entry point include/qas.h declares,
and behaves on a machine without a GPU.  No compute calls here."""
import ctypes
import os
import re

import pytest

from qasmhd_b200 import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "qas.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qas_[a-z_0-9]+)\s*\(", txt)))


def test_header_matches_binding():
    assert sorted(L.EXPORTS) == declared_functions()


def test_library_exports_every_declared_symbol():
    lib = L.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    abi = int(re.search(r"#define QAS_ABI_VERSION (\d+)", open(os.path.join(ROOT, "include", "qas.h")).read())[1])
    assert lib.qas_abi_version() == abi == L.ABI_VERSION


def test_status_strings():
    lib = L.load()
    for s in range(8):
        assert lib.qas_status_str(s)
    assert lib.qas_status_str(99) == b"unknown status"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_create_without_gpu_reports_no_device():
    lib = L.load()
    h = ctypes.c_void_p()
    g = L.Grid(2, 16, 16, 1, 0.1, 0.1, 0.0, 5.0 / 3.0)
    s = L.Scheme(1, 4, 3, 1)
    b = L.BC()
    assert lib.qas_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(s), ctypes.byref(b), -1) == L.QAS_ERR_NO_DEVICE


def test_invalid_arguments_rejected_before_device():
    lib = L.load()
    h = ctypes.c_void_p()
    b = L.BC()
    for g, s in [(L.Grid(4, 16, 16, 1, .1, .1, 0, 1.4), L.Scheme(1, 4, 3, 1)),    # bad dim
                 (L.Grid(2, 2, 16, 1, .1, .1, 0, 1.4), L.Scheme(1, 4, 3, 1)),     # too small
                 (L.Grid(2, 16, 16, 1, .1, .1, 0, 1.4), L.Scheme(4, 4, 3, 1)),    # bad rmn
                 (L.Grid(2, 16, 16, 1, .1, .1, 0, 1.4), L.Scheme(1, 5, 3, 1)),    # bad odr
                 (L.Grid(2, 16, 16, 1, .1, .1, 0, 1.4), L.Scheme(1, 4, 4, 1))]:   # bad rk
        assert lib.qas_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(s), ctypes.byref(b), -1) == L.QAS_ERR_INVALID
    assert lib.qas_destroy(None) == L.QAS_ERR_INVALID


def test_missing_library_fails_loudly(tmp_path):
    saved = L._lib
    try:
        L._lib = None
        with pytest.raises(FileNotFoundError):
            L.load(str(tmp_path / "nope.so"))
    finally:
        L._lib = saved

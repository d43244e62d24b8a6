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
    for s in range(10):
        assert lib.qas_status_str(s) != b"unknown status"
    assert lib.qas_status_str(99) == b"unknown status"


_NO_THROW = r"""
import ctypes, resource, sys
import numpy as np
from qasmhd_b200 import lib as L
lib = L.load()
n = 50_000_000
src = np.zeros(n, dtype=np.int32)
fac = np.zeros(n, dtype=np.float64)
g = L.Grid(1, n - 8, 1, 1, 1e-3, 0.0, 0.0, 5.0 / 3.0)
bc = L.BC()
vm = [int(l.split()[1]) * 1024 for l in open("/proc/self/status") if l.startswith("VmSize")][0]
resource.setrlimit(resource.RLIMIT_AS, (vm + (200 << 20), resource.RLIM_INFINITY))
st = lib.qas_bc_map(ctypes.byref(g), ctypes.byref(bc), 0, 0, 0,
                    src.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                    fac.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n)
print(st, lib.qas_last_cuda_error().decode())
"""


def test_no_exception_crosses_the_abi():
    """A host allocation that fails inside an entry point (qas_bc_map's 600 MB of maps under a
    200 MB address-space headroom) comes back as QAS_ERR_NOMEM with a message instead of an
    exception crossing the C-ABI (which would end the process)."""
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-c", _NO_THROW], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    status, msg = r.stdout.strip().split(" ", 1)
    assert int(status) == L.QAS_ERR_NOMEM and "host memory allocation failed" in msg, r.stdout


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

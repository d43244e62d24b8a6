"""The device point functions of the step against the reference's own, bit for bit, on the CPU.

qas_device.cuh is host+device code, so a host build of it (tests/native/device_points.cpp,
g++ without FP contraction: the library is built with --fmad=false and IEEE division and
square root) is compared with the known-answer vectors of the reference's point functions
(tests/golden/kat_*.npz, from common/mhd_flux.c, common/common_interp.c, common/mhd_func.c
built from source): the four Riemann solvers, the linear and nonlinear face interpolations the
schemes use, the characteristic face states of mhd_lrstate at every order -- the per-field
form and the grouped-stencil form the kernels run --, the primitive-variable face states of
its mhd_reconst form (qas_scheme.char_mode = 1), its mhd_c_reconst form (char_mode = 2) and the
CUCT weight."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.cases import assert_bitwise
from tests.golden import make_golden as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
D = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def dev(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("pts") / "device_points.so")
    subprocess.run([cxx, "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(ROOT, "qasmhd_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "device_points.cpp"), "-o", out], check=True)
    lib = ctypes.CDLL(out)
    lib.t_cuct.restype = ctypes.c_double
    lib.t_cuct.argtypes = [D]
    for f in (lib.t_flux, lib.t_lin, lib.t_nl):
        f.argtypes = [ctypes.c_int, D, D]
    lib.t_face_states.argtypes = [ctypes.c_int, ctypes.c_int, D, D]
    lib.t_face_states_prim.argtypes = [ctypes.c_int, D, D]
    lib.t_face_states_char.argtypes = [ctypes.c_int, D, D]
    return lib


def _run(fn, inp, nout, *lead):
    out = np.zeros((inp.shape[0], nout))
    for c in range(inp.shape[0]):
        a = np.ascontiguousarray(inp[c])
        fn(*lead, a.ctypes.data_as(D), out[c].ctypes.data_as(D))
    return out


@pytest.mark.parametrize("rmn", [0, 1, 2, 3])
def test_riemann_solvers(dev, rmn):
    inp = G.kat_inputs("flux")
    gold = np.load(os.path.join(GOLD, "kat_flux.npz"))[f"f{rmn}"]
    assert_bitwise(_run(dev.t_flux, inp, 7, rmn), gold, f"riemann {rmn}")


@pytest.mark.parametrize("kat,form,odr", [(10, "lin", 1), (11, "lin", 2), (12, "lin", 3), (13, "lin", 4),
                                          (10, "nl", 1), (14, "nl", 2), (15, "nl", 3), (16, "nl", 4)])
def test_face_interpolations(dev, kat, form, odr):
    inp = G.kat_inputs("interp")
    gold = np.load(os.path.join(GOLD, "kat_interp.npz"))[f"f{kat}"]
    fn = dev.t_lin if form == "lin" else dev.t_nl
    assert_bitwise(_run(fn, inp, 2, odr), gold, f"{form} order {odr}")


@pytest.mark.parametrize("kind", ["lrstate", "lrstate_vac"])
@pytest.mark.parametrize("grouped", [0, 1])
@pytest.mark.parametrize("odr", [1, 2, 3, 4])
def test_characteristic_face_states(dev, odr, grouped, kind):
    """lrstate: generic stencils; lrstate_vac: near-vacuum stencils, where the reconstructed
    density or pressure reaches the positivity fallback to first order (26 of the 200 rows at
    4th order in the reference's own answers)."""
    inp = G.kat_inputs(kind)
    gold = np.load(os.path.join(GOLD, f"kat_{kind}.npz"))[f"f{19 + odr}"]
    assert_bitwise(_run(dev.t_face_states, inp, 14, odr, grouped), gold,
                   f"mhd_lrstate {kind} order {odr} grouped {grouped}")


@pytest.mark.parametrize("odr", [1, 2, 3, 4])
def test_primitive_face_states(dev, odr):
    """mhd_lrstate with mhd_reconst (the reference's known answers from the harness built against
    it), the device face_states_prim of qas_scheme.char_mode = 1."""
    inp = G.kat_inputs("lrstate_prim")
    gold = np.load(os.path.join(GOLD, "kat_lrstate_prim.npz"))[f"f{23 + odr}"]
    assert_bitwise(_run(dev.t_face_states_prim, inp, 14, odr), gold, f"primitive face states order {odr}")


@pytest.mark.parametrize("odr", [1, 2, 3, 4])
def test_athena_face_states(dev, odr):
    """mhd_lrstate with mhd_c_reconst (the reference's known answers from the harness built against
    it), the device face_states_athena of qas_scheme.char_mode = 2."""
    inp = G.kat_inputs("lrstate_char")
    gold = np.load(os.path.join(GOLD, "kat_lrstate_char.npz"))[f"f{39 + odr}"]
    assert_bitwise(_run(dev.t_face_states_char, inp, 14, odr), gold, f"Athena-type face states order {odr}")


def test_cuct_weight(dev):
    inp = G.kat_inputs("cuct")
    gold = np.load(os.path.join(GOLD, "kat_cuct.npz"))["f30"]
    got = np.array([[dev.t_cuct(np.ascontiguousarray(r).ctypes.data_as(D))] for r in inp])
    assert_bitwise(got, gold, "cuct weight")

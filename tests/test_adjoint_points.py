"""Reverse-mode point functions of the adjoint (qas_adjoint.cuh) against central
finite differences, on the CPU: the header is host+device, so a host build of the
same code (tests/native/vjp_points.cpp) is checked here.  Random states cover the
subsonic and supersonic eigen-systems of the characteristic reconstruction and
generic (non-degenerate) Roe states."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GAM = 5.0 / 3.0
D = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def vjp(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("vjp") / "vjp_points.so")
    subprocess.run([cxx, "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                    "-I", os.path.join(ROOT, "qasmhd_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "vjp_points.cpp"), "-o", out], check=True)
    lib = ctypes.CDLL(out)
    lib.t_cuct.restype = ctypes.c_double
    return lib


def p(a):
    return a.ctypes.data_as(D)


def directional_errors(f, vjp_fn, x, g, rng, ndir=8, eps=1e-6):
    errs = []
    for _ in range(ndir):
        d = rng.standard_normal(x.shape)
        fd = np.dot(g, (f(x + eps * d) - f(x - eps * d)) / (2 * eps))
        an = np.dot(vjp_fn(x, g), d)
        errs.append(abs(fd - an) / max(abs(fd), abs(an)))
    return max(errs)


def test_wcns4_vjp(vjp):
    rng = np.random.default_rng(1)

    def f(x):
        o = np.zeros(2)
        vjp.t_wcns4(p(np.ascontiguousarray(x)), p(o))
        return o

    def b(x, g):
        o = np.zeros(5)
        vjp.t_wcns4_vjp(p(np.ascontiguousarray(x)), ctypes.c_double(g[0]), ctypes.c_double(g[1]), p(o))
        return o

    for _ in range(10):
        assert directional_errors(f, b, rng.standard_normal(5), rng.standard_normal(2), rng) < 1e-6


def _cell_stencil(rng, fast):
    q = np.zeros((7, 5))
    q[0] = 1.0 + 0.1 * rng.standard_normal(5)
    q[1] = (2.0 if fast else 0.1) + 0.1 * rng.standard_normal(5)
    q[2] = 0.3 * rng.standard_normal(5)
    q[3] = 0.3 * rng.standard_normal(5)
    q[4] = 0.5 + 0.1 * rng.standard_normal(5)
    q[5] = -0.4 + 0.1 * rng.standard_normal(5)
    q[6] = 0.8 + 0.1 * rng.standard_normal(5)
    return np.concatenate([q.ravel(), [0.6 * rng.standard_normal()]])


@pytest.mark.parametrize("fast", [False, True])
def test_face_states_vjp(vjp, fast):
    rng = np.random.default_rng(2 + fast)

    def f(x):
        vl = np.zeros(7)
        vr = np.zeros(7)
        vjp.t_face_states(p(np.ascontiguousarray(x[:35])), ctypes.c_double(x[35]), ctypes.c_double(GAM), p(vl), p(vr))
        return np.concatenate([vl, vr])

    def b(x, g):
        gq = np.zeros(35)
        gb = np.zeros(1)
        vjp.t_face_states_vjp(p(np.ascontiguousarray(x[:35])), ctypes.c_double(x[35]), ctypes.c_double(GAM),
                              p(np.ascontiguousarray(g[:7])), p(np.ascontiguousarray(g[7:])), p(gq), p(gb))
        return np.concatenate([gq, gb])

    for _ in range(6):
        x = _cell_stencil(rng, fast)
        # the state really is in the intended eigen-system
        q = x[:35].reshape(7, 5)[:, 2]
        assert (q[0] * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) > GAM * q[6]) == fast
        assert directional_errors(f, b, x, rng.standard_normal(14), rng) < 1e-6


def test_roe_vjp(vjp):
    rng = np.random.default_rng(4)

    def prim():
        return np.array([1.0 + 0.2 * rng.random(), 0.3 * rng.standard_normal(), 0.3 * rng.standard_normal(),
                         0.3 * rng.standard_normal(), 0.5 * rng.standard_normal(), 0.5 * rng.standard_normal(),
                         0.6 + 0.3 * rng.random()])

    def f(x):
        F = np.zeros(7)
        vjp.t_roe(p(np.ascontiguousarray(x[:7])), p(np.ascontiguousarray(x[7:14])), ctypes.c_double(x[14]),
                  ctypes.c_double(GAM), p(F))
        return F

    def b(x, g):
        gL = np.zeros(7)
        gR = np.zeros(7)
        gb = np.zeros(1)
        vjp.t_roe_vjp(p(np.ascontiguousarray(x[:7])), p(np.ascontiguousarray(x[7:14])), ctypes.c_double(x[14]),
                      ctypes.c_double(GAM), p(np.ascontiguousarray(g)), p(gL), p(gR), p(gb))
        return np.concatenate([gL, gR, gb])

    for _ in range(12):
        x = np.concatenate([prim(), prim(), [0.4 * rng.standard_normal()]])
        assert directional_errors(f, b, x, rng.standard_normal(7), rng) < 1e-6


def test_cuct_weight_vjp(vjp):
    rng = np.random.default_rng(5)

    def f(x):
        return np.array([vjp.t_cuct(p(np.ascontiguousarray(x)))])

    def b(x, g):
        o = np.zeros(16)
        vjp.t_cuct_vjp(p(np.ascontiguousarray(x)), ctypes.c_double(g[0]), p(o))
        return o

    for _ in range(8):
        x = np.concatenate([1 + 0.2 * rng.random(4), rng.standard_normal(8), rng.standard_normal(4)])
        assert directional_errors(f, b, x, rng.standard_normal(1), rng) < 1e-6

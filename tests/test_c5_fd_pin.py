"""Pin the extended-precision finite differences of the C5 loss to the reference's own
forward-mode derivative, on the CPU.

tests/golden/c5_fd_longdouble*.json hold central differences of the KH inversion loss taken on
the reference's 2D stepping code built in long double (tests/golden/make_c5_fd.py).  The same
directional derivatives come exactly (to round-off) from the reference's dual-number build
(oracle/_ref/ref2d_dual_ctw1) with the golden's frozen dt sequence: if the two agree, the
differences measure the derivative of the program the GPU adjoint differentiates, and the GPU
test that holds the adjoint to them tests the adjoint, not the difference quotient."""
import json
import os

import numpy as np
import pytest

from oracle import refcase as R
from tests.golden import make_c5_fd as F

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

pytestmark = pytest.mark.skipif(not os.access(R.dual_binary(1), os.X_OK),
                                reason="reference dual build (oracle/_ref) not present")


def _dual_derivatives(gold, ndir):
    """Directional derivatives of the loss along the golden's first ndir directions and eta,
    from the dual-number build: dL = 2 sum (obs - target) d(obs)."""
    n = gold["n"]
    base, amp = F.setup(n)
    dts = np.array(gold["dts"])
    ut = F.state(base, amp, np.random.default_rng(gold["target_seed"]).standard_normal((n, n)))
    fin_t, _ = R.run_reference_dual(base, ut.reshape(8, -1), np.zeros((8, base.nd)), dts,
                                    eta0=gold["eta_target"])
    target = F.observe(fin_t.reshape(8, base.ny, base.nx), n)
    dvy = np.random.default_rng(gold["dvy_seed"]).standard_normal((n, n))
    u0 = F.state(base, amp, dvy)
    ro = u0[0]
    vy = u0[2] / ro
    ampf = np.zeros_like(ro)
    ampf[F.XOFF:F.XOFF + n, F.XOFF:F.XOFF + n] = amp
    rng = np.random.default_rng(gold["dir_seed"])
    tangents = []
    for _ in range(ndir):
        dd = np.zeros_like(ro)
        dd[F.XOFF:F.XOFF + n, F.XOFF:F.XOFF + n] = rng.standard_normal((n, n))
        t = np.zeros_like(u0)
        t[2] = ro * ampf * dd  # d(my) for vy = amp * dvy
        t[7] = ro * vy * ampf * dd  # d(en) = ro vy d(vy)
        tangents.append((t, 0.0))
    tangents.append((np.zeros_like(u0), 1.0))  # eta
    out = []
    s = (slice(F.XOFF, F.XOFF + n), slice(F.XOFF, F.XOFF + n))
    for t, deta in tangents:
        v, dv = R.run_reference_dual(base, u0.reshape(8, -1), t.reshape(8, -1), dts, eta0=gold["eta"],
                                     deta=deta)
        v = v.reshape(8, base.ny, base.nx)
        dv = dv.reshape(8, base.ny, base.nx)
        d = F.observe(v, n) - target
        r, dr = v[0][s], dv[0][s]
        dobs = np.stack([dv[1][s] / r - v[1][s] * dr / (r * r), dv[2][s] / r - v[2][s] * dr / (r * r),
                         dv[4][s], dv[5][s]])
        out.append(2.0 * float(np.sum(d * dobs)))
    return np.array(out[:-1]), out[-1]


def test_small_fd_matches_reference_dual():
    """KH 32^2, 20 steps, 2 directions + eta: the long double differences against the dual build
    to 1e-8 of the largest directional derivative (measured: 7e-10, and 7e-11 on eta)."""
    gold = json.load(open(os.path.join(GOLD, "c5_fd_longdouble_32_20_2.json")))
    fd = np.array(gold["fd_dirs"])
    dual, dual_eta = _dual_derivatives(gold, len(fd))
    assert np.max(np.abs(dual - fd)) <= 1e-8 * np.max(np.abs(fd)), (dual, fd)
    assert abs(dual_eta - gold["fd_eta"]) <= 1e-8 * abs(gold["fd_eta"]), (dual_eta, gold["fd_eta"])

"""Pin the extended-precision finite differences of the C5 loss to the reference's own
forward-mode derivative, on the CPU.

tests/golden/c5_fd_longdouble*.json hold central differences of the KH inversion loss taken on
the reference's 2D stepping code built in long double (tests/golden/make_c5_fd.py).  The same
directional derivatives come exactly (to round-off) from the reference's dual-number build
(oracle/_ref/ref2d_dual_ctw1) with the golden's frozen dt sequence: where the two agree, the
differences measure the derivative of the program the GPU adjoint differentiates; where they do
not, the loss is not smooth at the scale of the difference step (the GPU test states that
floor).  The goldens also hold the dual values the script computed; they are checked here
against a live run."""
import json
import os

import numpy as np
import pytest

from oracle import refcase as R
from tests.golden import make_c5_fd as F

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

pytestmark = pytest.mark.skipif(not os.access(R.dual_binary(1), os.X_OK),
                                reason="reference dual build (oracle/_ref) not present")


def test_small_fd_matches_reference_dual():
    """KH 32^2, 20 steps, 2 directions + eta: the long double differences against the dual build
    to 1e-8 of the largest directional derivative (measured: 7e-10, and 7e-11 on eta)."""
    gold = json.load(open(os.path.join(GOLD, "c5_fd_longdouble_32_20_2.json")))
    fd = np.array(gold["fd_dirs"])
    dual, dual_eta = F.dual_derivatives(gold)
    dual = np.array(dual)
    assert np.max(np.abs(dual - fd)) <= 1e-8 * np.max(np.abs(fd)), (dual, fd)
    assert abs(dual_eta - gold["fd_eta"]) <= 1e-8 * abs(gold["fd_eta"]), (dual_eta, gold["fd_eta"])
    if "dual_dirs" in gold:  # the stored values are the dual build's, bit for bit
        assert gold["dual_dirs"] == list(dual) and gold["dual_eta"] == dual_eta

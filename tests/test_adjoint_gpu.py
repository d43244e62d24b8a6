"""Discrete adjoint of the 2D step (qas_adjoint_forward / qas_adjoint_backward).

Checks: the checkpointed forward run is bit-identical to eager stepping; the
gradient of a random linear functional of the final state matches central finite
differences on generic smooth states (periodic, mirror/open boundaries, CUCT on
and off, one and two resistive sub-cycles); the torch.autograd.Function wrapper
on the Kelvin-Helmholtz inversion (perturbation field and eta) and at the full
256^2 / 400-step size; determinism; refused configurations.

Step sizes: WCNS4 weights are rational in the smoothness indicators, which for a
smooth field are set by differences of ~1e-3; a rough random direction of size
1e-6 moves them by ~1% and the central difference is then truncation-limited, so
rough directions use eps = 1e-8.  In the Kelvin-Helmholtz problem the vy
perturbation changes en by vy*dvy ~ 1e-14 against en ~ 1.5 (tens of ulps), which
bounds the finite-difference accuracy there.
"""
import numpy as np
import pytest
import torch

from qasmhd_b200 import lib as L
from qasmhd_b200.adjoint import KHInverse, cfl_dts, directional_check
from qasmhd_b200.problems import RMN_HLLD, RMN_ROE, kelvin_helmholtz, smooth_wave

pytestmark = pytest.mark.gpu


def _fwd(ctx, u0, dts, eta, every):
    ctx.upload(u0)
    ctx.adjoint_forward(dts, eta, every)
    return ctx.download()


def _fd_check(prob, nsteps, every, eta, eps=1e-8, ndir=3, tol=1e-5, seed=3):
    with L.Context.from_problem(prob) as ctx:
        u0 = prob.state.reshape(8, -1).copy()
        dts = cfl_dts(ctx, u0, nsteps, prob.cfl, eta)
        _fwd(ctx, u0, dts, eta, every)
        rng = np.random.default_rng(seed)
        w = rng.standard_normal(u0.shape)
        g0, geta = ctx.adjoint_backward(w)
        for _ in range(ndir):
            d = rng.standard_normal(u0.shape)
            fp = _fwd(ctx, u0 + eps * d, dts, eta, every)
            fm = _fwd(ctx, u0 - eps * d, dts, eta, every)
            fd = np.sum(w * (fp - fm)) / (2 * eps)
            an = np.sum(g0 * d)
            assert abs(fd - an) <= tol * max(abs(fd), abs(an)), (fd, an)
        if eta > 0:
            he = 1e-6
            fp = _fwd(ctx, u0, dts, eta + he, every)
            fm = _fwd(ctx, u0, dts, eta - he, every)
            fd = np.sum(w * (fp - fm)) / (2 * he)
            assert abs(fd - geta) <= tol * max(abs(fd), abs(geta)), (fd, geta)


def test_forward_bit_identical_to_eager_steps():
    prob = kelvin_helmholtz(dim=2, n=32, mach=0.1, rmn=RMN_ROE, odr=4, rk=3, ctw=1)
    eta = 1e-3
    with L.Context.from_problem(prob) as ctx:
        u0 = prob.state.reshape(8, -1).copy()
        dts = cfl_dts(ctx, u0, 12, prob.cfl, eta)
        ctx.upload(u0)
        for dt in dts:
            ctx.bound()
            ctx.step(dt)
            ctx.dissipate(dt, 0.0, eta)
        ref = ctx.download()
        fin = _fwd(ctx, u0, dts, eta, 5)
        assert np.array_equal(ref, fin)
        # backward leaves the final state in the context
        ctx.adjoint_backward(np.ones_like(u0))
        assert np.array_equal(ctx.download(), fin)


def test_gradient_periodic_one_step():
    _fd_check(smooth_wave(2, 24, rmn=RMN_ROE), 1, 1, 0.0)


def test_gradient_resistive_checkpointed():
    _fd_check(smooth_wave(2, 24, rmn=RMN_ROE), 5, 2, 1e-3)


def test_gradient_mirror_open_boundaries():
    dn = ((1, -1, 1, 1, -1, 1, 1, 1), (2, 2, -2, 2, 2, -2, 2, 2), (0,) * 8)
    _fd_check(smooth_wave(2, 24, rmn=RMN_ROE, dn=dn), 5, 2, 1e-3)


def test_gradient_without_cuct_weight():
    _fd_check(smooth_wave(2, 24, rmn=RMN_ROE, ctw=0), 5, 3, 0.0)


def test_gradient_two_subcycles():
    prob = smooth_wave(2, 24, rmn=RMN_ROE)
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        dt = ctx.cfl_dt(prob.cfl)
    eta = 0.1
    assert 1 + int(2 * (eta * dt) / (prob.dx * prob.dx)) == 2  # dsptv sub-cycles twice
    _fd_check(prob, 6, 4, eta, ndir=2)


def test_deterministic():
    prob = smooth_wave(2, 24, rmn=RMN_ROE)
    with L.Context.from_problem(prob) as ctx:
        u0 = prob.state.reshape(8, -1).copy()
        dts = cfl_dts(ctx, u0, 4, prob.cfl, 1e-3)
        _fwd(ctx, u0, dts, 1e-3, 3)
        w = np.random.default_rng(0).standard_normal(u0.shape)
        a = ctx.adjoint_backward(w)
        b = ctx.adjoint_backward(w)
        assert np.array_equal(a[0], b[0]) and a[1] == b[1]


def test_refused_configurations():
    prob = smooth_wave(2, 16, rmn=RMN_HLLD)
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        with pytest.raises(L.QasError) as e:
            ctx.adjoint_forward([1e-3], 0.0, 1)
        assert e.value.status == L.QAS_ERR_UNSUPPORTED
    prob = smooth_wave(2, 16, rmn=RMN_ROE)
    with L.Context.from_problem(prob) as ctx:
        with pytest.raises(L.QasError) as e:
            ctx.adjoint_backward(np.zeros((8, ctx.nd)))
        assert e.value.status == L.QAS_ERR_INVALID
        with pytest.raises(L.QasError):
            ctx.adjoint_forward([1e-3, -1.0], 0.0, 1)


def test_adjoint_run_one_call_equals_the_pair():
    """qas_adjoint_run (forward and backward in one call) gives the bits of qas_adjoint_forward
    followed by qas_adjoint_backward, and leaves the same final state."""
    prob = smooth_wave(2, 24, rmn=RMN_ROE)
    eta = 1e-3
    u0 = prob.state.reshape(8, -1).copy()
    w = np.random.default_rng(4).standard_normal(u0.shape)
    with L.Context.from_problem(prob) as ctx:
        dts = cfl_dts(ctx, u0, 4, prob.cfl, eta)
        ctx.upload(u0)
        ctx.adjoint_forward(dts, eta, 2)
        fin_a = ctx.download()
        g_a, e_a = ctx.adjoint_backward(w)
        ctx.upload(u0)
        g_b, e_b = ctx.adjoint_run(dts, w, eta, 2)
        fin_b = ctx.download()
    assert np.array_equal(fin_a, fin_b)
    assert np.array_equal(g_a, g_b) and e_a == e_b


def test_autograd_function_kh_inversion_small():
    P = KHInverse(n=32, nsteps=20, ckpt_every=6)
    try:
        dvy = np.random.default_rng(7).standard_normal((32, 32))
        r = directional_check(P, dvy, 0.5e-4, ndir=4, eps=1e-6, eps_eta=1e-6)
        ads = np.array([a for _, a in r["pairs"]])
        fds = np.array([f for f, _ in r["pairs"]])
        assert np.max(np.abs(fds - ads)) <= 1e-4 * np.max(np.abs(ads))
        fd, an = r["eta"]
        assert abs(fd - an) <= 1e-4 * max(abs(fd), abs(an))
        # the torch graph around the C-ABI: gradient of a torch loss of the final state
        x = torch.from_numpy(dvy).requires_grad_(True)
        e = torch.tensor(0.5e-4, dtype=torch.float64, requires_grad=True)
        P.loss(x, e).backward()
        assert np.allclose(x.grad.numpy(), r["grad"], rtol=0, atol=0)
    finally:
        P.close()


def test_kh_inversion_full_size():
    """2D KH 256^2, M=0.1, Roe + WCNS4 + CT, 400 RK3 steps, checkpoints every 20 steps,
    eta target 1e-4; 32 seeded directions of the vy perturbation with eps = 1e-6."""
    P = KHInverse(n=256, nsteps=400, ckpt_every=20)
    try:
        dvy = np.random.default_rng(7).standard_normal((256, 256))
        r = directional_check(P, dvy, 0.5e-4, ndir=32, eps=1e-6, eps_eta=1e-6)
        ads = np.array([a for _, a in r["pairs"]])
        fds = np.array([f for f, _ in r["pairs"]])
        assert np.max(np.abs(fds - ads)) <= 5e-4 * np.max(np.abs(ads))
        assert np.corrcoef(fds, ads)[0, 1] > 0.9999
        fd, an = r["eta"]
        assert abs(fd - an) <= 1e-2 * abs(an)
    finally:
        P.close()


# (golden, tolerance of adjoint vs the long double differences, of max |fd|)
FD_GOLDENS = [
    # KH 32^2, 20 steps: differences and the reference's dual derivative agree to 7e-10
    ("c5_fd_longdouble_32_20_2.json", 1e-6),
    # the C5 problem at full resolution over its first 40 steps: they agree to 5.3e-10
    ("c5_fd_longdouble_256_40_32.json", 1e-6),
    # C5 as specified (256^2, 400 steps): the differences' own floor, 1.85e-5 (see below)
    ("c5_fd_longdouble.json", 3e-5),
]


@pytest.mark.parametrize("name,tol_fd", FD_GOLDENS, ids=[g[0] for g in FD_GOLDENS])
def test_kh_inversion_vs_extended_precision_fd(name, tol_fd):
    """The KH inversion gradient against central differences taken in extended precision: the
    reference's 2D stepping code built in long double (oracle/_ref/ref2d_ld_ctw1), 32 seeded
    directions of the vy perturbation (eps = 1e-6) and eta (step 1e-9), with the same frozen dt
    sequence and target (tests/golden/c5_fd_longdouble*.json, made by tests/golden/make_c5_fd.py,
    which also stores the reference's dual-number derivative along the same directions).

    The adjoint must equal the reference's dual derivative (the exact derivative of the same
    double-precision program) to 1e-9, direction by direction, and lie no farther from the
    differences than that derivative does.  On the full C5 run the differences themselves stop
    at 1.85e-5 of the largest directional derivative (dual and adjoint alike; eta 3.5e-8): the
    loss is not smooth at the scale of the step -- Roe's |vn| eigenvalues cross zero inside
    the step in some directions (the worst one falls 40x with eps = 1e-8) and some branches are
    tied at the base point, where central differences average the two one-sided derivatives
    (2-3.5e-6 whatever the step).  On the 20-step 32^2 run they agree to 7e-10, and on the C5
    problem at full resolution over 40 steps to 5.3e-10 (eta 4.5e-10): there the adjoint is held
    to 1e-6 of central FD."""
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name)
    if not os.path.exists(path):
        pytest.skip(f"tests/golden/{name} not generated")
    gold = json.load(open(path))
    P = KHInverse(n=gold["n"], nsteps=gold["nsteps"], ckpt_every=20)
    try:
        assert np.array_equal(P.dts, np.array(gold["dts"]))  # the reference's exec_ dt sequence
        dvy = np.random.default_rng(gold["dvy_seed"]).standard_normal((P.n, P.n))
        x = torch.from_numpy(dvy).requires_grad_(True)
        e = torch.tensor(gold["eta"], dtype=torch.float64, requires_grad=True)
        loss = P.loss(x, e)
        loss.backward()
        assert abs(float(loss.detach()) - gold["loss"]) <= 1e-9 * gold["loss"]
        rng = np.random.default_rng(gold["dir_seed"])
        ads = np.array([float(np.sum(x.grad.numpy() * rng.standard_normal((P.n, P.n)))) for _ in gold["fd_dirs"]])
        geta = float(e.grad)
        fds, dus = np.array(gold["fd_dirs"]), np.array(gold["dual_dirs"])
        scale = np.max(np.abs(fds))
        assert np.max(np.abs(ads - dus)) <= 1e-9 * np.max(np.abs(dus)), np.max(np.abs(ads - dus)) / np.max(np.abs(dus))
        assert abs(geta - gold["dual_eta"]) <= 1e-9 * abs(gold["dual_eta"]), (geta, gold["dual_eta"])
        assert np.max(np.abs(ads - fds)) <= np.max(np.abs(dus - fds)) + 1e-9 * scale
        assert np.max(np.abs(ads - fds)) <= tol_fd * scale, np.max(np.abs(ads - fds)) / scale
        assert abs(geta - gold["fd_eta"]) <= 1e-6 * abs(gold["fd_eta"]), (geta, gold["fd_eta"])
    finally:
        P.close()

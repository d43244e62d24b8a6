"""The GPU adjoint against the reference's own forward-mode derivative.

oracle/_ref/ref2d_dual_ctw* is the reference's 2D stepping code (bound, ideal, the
sub-cycled dsptv) compiled with a dual number in place of double; with the same
frozen dt sequence it returns the directional derivative of the final state.  For
a linear functional w of the final state, <adjoint gradient, d> must equal
<w, J d> up to round-off in the two derivative computations (both are exact
derivatives of the branch the forward run took)."""
import numpy as np
import pytest
import torch

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200.adjoint import KHInverse, cfl_dts
from qasmhd_b200.problems import RMN_ROE, XOFF, smooth_wave

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (R.reference_available(2, 1) and
                                      __import__("os").access(R.dual_binary(1), __import__("os").X_OK)),
                                 reason="reference dual build (oracle/_ref) not present")]

TOL = 1e-9


@pytest.mark.parametrize("ctw,dn", [(1, None), (0, None),
                                    (1, ((1, -1, 1, 1, -1, 1, 1, 1), (2, 2, -2, 2, 2, -2, 2, 2), (0,) * 8))])
def test_adjoint_equals_reference_dual_generic(ctw, dn):
    prob = smooth_wave(2, 24, rmn=RMN_ROE, ctw=ctw, dn=dn)
    eta = 1e-3
    u0 = prob.state.reshape(8, -1).copy()
    rng = np.random.default_rng(11)
    w = rng.standard_normal(u0.shape)
    with L.Context.from_problem(prob) as ctx:
        dts = cfl_dts(ctx, u0, 5, prob.cfl, eta)
        ctx.upload(u0)
        ctx.adjoint_forward(dts, eta, 2)
        fin = ctx.download()
        g0, geta = ctx.adjoint_backward(w)
    for k in range(2):
        d = rng.standard_normal(u0.shape)
        deta = 0.3 if k == 1 else 0.0
        v, t = R.run_reference_dual(prob, u0, d, dts, eta0=eta, deta=deta)
        assert np.array_equal(v, fin)  # same forward run, bit for bit
        jvp = float(np.sum(w * t))
        vjp = float(np.sum(g0 * d)) + geta * deta
        assert abs(jvp - vjp) <= TOL * abs(jvp), (jvp, vjp)


def test_adjoint_equals_reference_dual_kh_inversion():
    """The C5 problem at 64^2 x 40 steps: directions of the vy perturbation and of eta."""
    P = KHInverse(n=64, nsteps=40, ckpt_every=20)
    try:
        rng = np.random.default_rng(3)
        dvy = rng.standard_normal((64, 64))
        eta = 0.5e-4
        x = torch.from_numpy(dvy).requires_grad_(True)
        e = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
        P.loss(x, e).backward()
        # dL/d(final state) for the tangent contraction
        with torch.no_grad():
            u0 = P.state(torch.from_numpy(dvy))
            fin = P.final(torch.from_numpy(dvy), torch.tensor(eta, dtype=torch.float64))
        fin = fin.clone().requires_grad_(True)
        d_obs = P.observe(fin) - P.target_obs
        (d_obs * d_obs).sum().backward()
        gfin = fin.grad.numpy().reshape(8, -1)
        ro = u0[0].numpy()
        vy = (u0[2] / u0[0]).numpy()
        amp = np.zeros_like(ro)
        amp[P.interior] = P.amp[P.interior]
        for k in range(2):
            dd = np.zeros_like(ro)
            dd[P.interior] = rng.standard_normal((64, 64))
            tang = np.zeros((8,) + ro.shape)
            tang[2] = ro * amp * dd               # my = ro vy
            tang[7] = ro * vy * amp * dd          # en += ro vy^2 / 2
            deta = 1e-4 if k == 1 else 0.0
            v, t = R.run_reference_dual(P.base, u0.numpy().reshape(8, -1), tang.reshape(8, -1), P.dts,
                                        eta0=eta, deta=deta)
            assert np.array_equal(v, fin.detach().numpy().reshape(8, -1))
            jvp = float(np.sum(gfin * t))
            vjp = float(np.sum(x.grad.numpy() * dd[P.interior])) + float(e.grad) * deta
            assert abs(jvp - vjp) <= TOL * abs(jvp), (jvp, vjp)
    finally:
        P.close()


def test_adjoint_equals_reference_dual_c5_full_size():
    """C5 as specified: KH 2D 256^2, M=0.1, Roe + WCNS4 + CT, 400 RK3 steps, checkpoints
    every 20 steps; one seeded vy-perturbation direction and the eta direction (each
    dual run is ~20 s of the reference on the host cores)."""
    P = KHInverse(n=256, nsteps=400, ckpt_every=20)
    try:
        dvy = np.random.default_rng(7).standard_normal((256, 256))
        eta = 0.5e-4
        x = torch.from_numpy(dvy).requires_grad_(True)
        e = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
        P.loss(x, e).backward()
        with torch.no_grad():
            u0 = P.state(torch.from_numpy(dvy))
            fin = P.final(torch.from_numpy(dvy), torch.tensor(eta, dtype=torch.float64))
        fin = fin.clone().requires_grad_(True)
        d_obs = P.observe(fin) - P.target_obs
        (d_obs * d_obs).sum().backward()
        gfin = fin.grad.numpy().reshape(8, -1)
        ro = u0[0].numpy()
        vy = (u0[2] / u0[0]).numpy()
        amp = np.zeros_like(ro)
        amp[P.interior] = P.amp[P.interior]
        rng = np.random.default_rng(3)
        for k in range(2):
            dd = np.zeros_like(ro)
            if k == 0:
                dd[P.interior] = rng.standard_normal((256, 256))
            tang = np.zeros((8,) + ro.shape)
            tang[2] = ro * amp * dd
            tang[7] = ro * vy * amp * dd
            deta = 1e-4 if k == 1 else 0.0
            v, t = R.run_reference_dual(P.base, u0.numpy().reshape(8, -1), tang.reshape(8, -1), P.dts,
                                        eta0=eta, deta=deta)
            assert np.array_equal(v, fin.detach().numpy().reshape(8, -1))  # 400 steps, bit for bit
            jvp = float(np.sum(gfin * t))
            vjp = float(np.sum(x.grad.numpy() * dd[P.interior])) + float(e.grad) * deta
            assert abs(jvp - vjp) <= TOL * abs(jvp), (jvp, vjp)
    finally:
        P.close()

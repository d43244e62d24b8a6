"""Gradients of the 2D step through the discrete adjoint of libqas.

``QasRun`` is a ``torch.autograd.Function`` over ``qas_adjoint_forward`` /
``qas_adjoint_backward``: its forward runs ``len(dts)`` exec_ steps (bound,
ideal(dt), sub-cycled dsptv with uniform eta) from the given state on the GPU
and returns the final state; its backward returns dL/d(initial state) and
dL/deta.  The time steps are an input (frozen), as the reference's setdt rule
makes dt a non-differentiable function of the state.

The inversion problem the gradients are checked on: a 2D Kelvin-Helmholtz layer
(Roe flux, characteristic WCNS4, CT, RK3), whose loss is the L2 misfit of the
final (vx, vy, bx, by) to a target produced with eta* and another seeded vy
perturbation; the unknowns are the interior vy-perturbation field and eta.
"""
from __future__ import annotations

import dataclasses
from typing import Optional, Sequence

import numpy as np
import torch

from .lib import Context
from .problems import RMN_ROE, XOFF, Problem, kelvin_helmholtz


class QasRun(torch.autograd.Function):
    """final_state = QasRun.apply(u0, eta, ctx, dts, ckpt_every)

    u0: float64 tensor of 8*nd values (the context's field-major layout), eta: 0-d
    float64 tensor.  One context holds one forward run's checkpoints, so call
    backward before the next forward on the same context.
    """

    @staticmethod
    def forward(actx, u0: torch.Tensor, eta: torch.Tensor, qctx: Context, dts: np.ndarray, ckpt_every: int):
        shape = u0.shape
        qctx.upload(u0.detach().cpu().numpy().reshape(8, -1))
        qctx.adjoint_forward(dts, float(eta), ckpt_every)
        actx.qctx = qctx
        actx.shape = shape
        return torch.from_numpy(qctx.download()).reshape(shape)

    @staticmethod
    def backward(actx, grad: torch.Tensor):
        du0, deta = actx.qctx.adjoint_backward(grad.detach().cpu().numpy().reshape(8, -1))
        return (torch.from_numpy(du0).reshape(actx.shape), torch.tensor(deta, dtype=torch.float64), None, None,
                None)


def cfl_dts(ctx: Context, state: np.ndarray, nsteps: int, cfl: float, eta: float) -> np.ndarray:
    """dt sequence of an exec_ run from `state`: setdt at the start and after every
    second step (mhd2d_class.cpp:35-61), each step = bound, ideal, dissipate."""
    ctx.upload(state)
    dts = np.empty(nsteps)
    dt = ctx.cfl_dt(cfl)
    for n in range(nsteps):
        if n > 0 and n % 2 == 0:
            dt = ctx.cfl_dt(cfl)
        dts[n] = dt
        ctx.adjoint_forward(dts[n:n + 1], eta, 1)
    return dts


@dataclasses.dataclass
class KHInverse:
    """2D Kelvin-Helmholtz inversion for the vy perturbation and eta."""

    n: int = 256
    mach: float = 0.1
    nsteps: int = 400
    ckpt_every: int = 20
    eta_target: float = 1e-4
    target_seed: int = 2025
    beta: float = 100.0

    def __post_init__(self):
        self.base: Problem = kelvin_helmholtz(dim=2, n=self.n, mach=self.mach, beta=self.beta, rmn=RMN_ROE, odr=4,
                                              rk=3, ctw=1, dvy_field=np.zeros((self.n, self.n)))
        p = self.base
        x, y, _ = p.coords()
        Y, _X = np.meshgrid(y, x, indexing="ij")
        # perturbation amplitude of kelvin_helmholtz: noise * M * exp(-(y/0.1)^2), noise = 1e-3
        self.amp = 1e-3 * self.mach * np.exp(-(Y / 0.1) ** 2)
        self.ctx = Context.from_problem(p)
        self.nd = self.ctx.nd
        self.shape = (8, p.ny, p.nx)
        self.interior = (slice(XOFF, XOFF + p.nym), slice(XOFF, XOFF + p.nxm))
        self.dts = cfl_dts(self.ctx, p.state, self.nsteps, p.cfl, self.eta_target)
        rng = np.random.default_rng(self.target_seed)
        with torch.no_grad():
            self.target = self.final(torch.from_numpy(rng.standard_normal((self.n, self.n))),
                                     torch.tensor(self.eta_target, dtype=torch.float64))
            self.target_obs = self.observe(self.target)

    def state(self, dvy: torch.Tensor) -> torch.Tensor:
        """Initial state with vy = amp * dvy on the interior: my = ro vy, en += ro vy^2 / 2."""
        base = torch.from_numpy(self.base.state.reshape(self.shape).copy())
        amp = torch.from_numpy(self.amp[self.interior])
        vy = torch.nn.functional.pad(amp * dvy, (XOFF, XOFF, XOFF, XOFF))
        ro = base[0]
        u = base.clone()
        u[2] = ro * vy
        u[7] = base[7] + 0.5 * ro * vy * vy
        return u

    def final(self, dvy: torch.Tensor, eta: torch.Tensor) -> torch.Tensor:
        return QasRun.apply(self.state(dvy), eta, self.ctx, self.dts, self.ckpt_every)

    def observe(self, u: torch.Tensor) -> torch.Tensor:
        """(vx, vy, bx, by) on the interior."""
        s = self.interior
        ro = u[0][s]
        return torch.stack([u[1][s] / ro, u[2][s] / ro, u[4][s], u[5][s]])

    def loss(self, dvy: torch.Tensor, eta: torch.Tensor) -> torch.Tensor:
        d = self.observe(self.final(dvy, eta)) - self.target_obs
        return (d * d).sum()

    def close(self) -> None:
        self.ctx.close()


def directional_check(problem: KHInverse, dvy: np.ndarray, eta: float, ndir: int = 32, eps: float = 1e-6,
                      seed: int = 11, eps_eta: Optional[float] = None):
    """Adjoint gradient vs central finite differences on `ndir` seeded random
    directions of the perturbation field, and on eta.  Returns a dict with the
    per-direction (fd, adjoint) pairs, the eta pair and the loss."""
    x = torch.from_numpy(np.array(dvy, dtype=np.float64)).requires_grad_(True)
    e = torch.tensor(float(eta), dtype=torch.float64, requires_grad=True)
    L = problem.loss(x, e)
    L.backward()
    gx = x.grad.numpy().copy()
    ge = float(e.grad)
    rng = np.random.default_rng(seed)
    pairs = []
    with torch.no_grad():
        for _ in range(ndir):
            d = rng.standard_normal(dvy.shape)
            lp = float(problem.loss(torch.from_numpy(dvy + eps * d), torch.tensor(eta, dtype=torch.float64)))
            lm = float(problem.loss(torch.from_numpy(dvy - eps * d), torch.tensor(eta, dtype=torch.float64)))
            pairs.append(((lp - lm) / (2 * eps), float(np.sum(gx * d))))
        he = eps_eta if eps_eta is not None else eps * max(abs(eta), 1e-6)
        lp = float(problem.loss(torch.from_numpy(dvy), torch.tensor(eta + he, dtype=torch.float64)))
        lm = float(problem.loss(torch.from_numpy(dvy), torch.tensor(eta - he, dtype=torch.float64)))
    return {"loss": float(L.detach()), "pairs": pairs, "eta": ((lp - lm) / (2 * he), ge), "grad": gx}

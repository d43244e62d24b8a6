"""Helpers shared by the tests: run a problem through the CUDA path with the
same loop semantics as the oracle modes (oracle/refcase.py)."""
from __future__ import annotations

import numpy as np

from oracle import refcase as R
from qasmhd_b200 import lib as L


def run_gpu(prob, mode: int, nsteps: int = 0, dt: float = 0.0, use_graph: bool = True, state=None):
    """Mirror of refcase.run_reference for the CUDA path (through the C-ABI)."""
    st = prob.state if state is None else state
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(st)
        if mode == R.MODE_STEP:
            ctx.bound()
            ctx.step(dt)
            out = ctx.download(st.shape)
            ctx.sync()
            return {"state": out, "steps": 1}
        if mode == R.MODE_DSTEP:
            ctx.bound()
            if getattr(prob, "hall", False):  # the Hall build's DSTEP: one hall_(dt)
                ctx.hall(dt)
            else:
                ctx.dsptv(dt, prob.nu0, prob.eta0)
            out = ctx.download(st.shape)
            ctx.sync()
            return {"state": out, "steps": 1}
        if mode in (R.MODE_RUN, R.MODE_DRUN):
            resist = mode == R.MODE_DRUN
            info = ctx.run(max_steps=nsteps, flg=prob.flg, stop_rule=0, cfl=prob.cfl, dtrec=prob.dtrec,
                           nout=prob.nout, use_graph=use_graph, nu0=prob.nu0 if resist else 0.0,
                           eta0=prob.eta0 if resist else 0.0)
        elif mode == R.MODE_EXEC:
            rule = 2 if prob.dim == 1 and not prob.flg else 1
            info = ctx.run(max_steps=0, flg=prob.flg, stop_rule=rule, cfl=prob.cfl, dtrec=prob.dtrec,
                           nout=prob.nout, use_graph=use_graph)
        else:
            raise ValueError(mode)
        out = ctx.download(st.shape)
        return {"state": out, "steps": info.steps, "tim": info.tim, "dt": info.dt}


def assert_bitwise(a: np.ndarray, b: np.ndarray, label: str = "") -> None:
    """Exact equality (== semantics: +0 == -0), NaN-aware; reports the worst cell."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (label, a.shape, b.shape)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        idx = np.argwhere(~same)
        first = tuple(idx[0])
        d = np.abs(a - b)
        raise AssertionError(f"{label}: {len(idx)} cells differ; first {first}: {a[first]!r} vs {b[first]!r}; "
                             f"max |diff| {np.nanmax(d):.3e}")

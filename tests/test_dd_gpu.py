"""A domain split into slabs (qas_dd_*) gives the same bits as the oracle and as the
single-domain context.

The slabs share one B200 here (every slab its own stream; ghost planes copied between them
after each fill, after the primitives and after the shock detector); across GPUs the same
copies are peer copies.  Compared after several exec_ steps: the state (interior and the
global ghost planes) against the plain-C oracle (the restatement pinned to the reference
build) and the single-domain context, and the loop control (n, tim, dt)."""
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise

pytestmark = pytest.mark.gpu


def _single(p, nsteps, stop_rule=0):
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        info = ctx.run(max_steps=nsteps, flg=1, stop_rule=stop_rule, cfl=p.cfl, dtrec=p.dtrec, nout=p.nout)
        return ctx.download(p.state.shape), info


def _split(p, nparts, nsteps, stop_rule=0):
    with L.Decomposition(p, nparts) as dd:
        dd.upload(p.state)
        info = dd.run(max_steps=nsteps, flg=1, stop_rule=stop_rule, cfl=p.cfl, dtrec=p.dtrec, nout=p.nout)
        return dd.download(), info, dd.kernel_launches()


def _prim(p):
    p.char_mode = 1
    return p


CASES = {
    "ot2d_64_hlld": lambda: P.orszag_tang(64),
    "ot2d_72_roe_ctw0": lambda: P.orszag_tang(72, rmn=P.RMN_ROE, ctw=0),
    "kh2d_64x48_mlau_open": lambda: P.kelvin_helmholtz(2, 64, nym=48, mach=0.3),
    "kh3d_16x16x32_mlau": lambda: P.kelvin_helmholtz(3, 16, nzm=32, mach=0.3),
    "kh3d_24_lhlld": lambda: P.kelvin_helmholtz(3, 24, mach=0.3, rmn=P.RMN_LHLLD),
    "kh3d_16x16x24_prim": lambda: _prim(P.kelvin_helmholtz(3, 16, nzm=24, mach=0.3)),
    "wave3d_physical_z_roe": lambda: P.smooth_wave(3, 24, rmn=P.RMN_ROE,
                                                   dn=((0,) * 8, (0,) * 8, (2, 1, 1, -1, 1, 1, -1, 2))),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nparts", [2, 3])
def test_split_matches_oracle_and_single_domain(restatement, case, nparts):
    p = CASES[case]()
    want = restatement.run(p, 5, mode=R.MODE_RUN)
    a, ia = _single(p, 5)
    b, ib, (kernels, copies) = _split(p, nparts, 5)
    assert_bitwise(b, want["state"], f"{case} x{nparts} vs oracle")
    assert ib.dt == want["dt"]
    assert_bitwise(b, a, f"{case} x{nparts}")
    assert (ib.steps, ib.n, ib.nmax) == (ia.steps, ia.n, ia.nmax)
    assert ib.tim == ia.tim and ib.dt == ia.dt
    assert kernels > 0 and copies > 0


def test_split_exec_rule_and_resume(restatement):
    """exec_'s stop rule (n < nmax && tim < tmax) and a run continued in a second call."""
    p = P.orszag_tang(64, tmax=0.1)
    want = restatement.run(p, 0, mode=R.MODE_EXEC)
    a, ia = _single(p, 0, stop_rule=1)
    assert_bitwise(a, want["state"], "ot exec rule, single domain vs oracle")
    assert 3 < ia.steps < 100
    with L.Decomposition(p, 4) as dd:
        dd.upload(p.state)
        # both calls carry the exec_ stop rule; the first is also capped at 3 steps
        i1 = dd.run(max_steps=3, flg=1, stop_rule=1, cfl=p.cfl, dtrec=p.dtrec, nout=p.nout)
        i2 = dd.run(max_steps=200, flg=1, stop_rule=1, cfl=p.cfl, dtrec=p.dtrec, nout=p.nout)
        b = dd.download()
    assert i1.steps == 3 and i1.steps + i2.steps == ia.steps and i2.tim == ia.tim
    assert_bitwise(b, a, "ot exec rule x4")


def test_split_one_part_is_the_single_context(restatement):
    p = P.kelvin_helmholtz(3, 16, mach=0.3)
    a, _ = _single(p, 3)
    b, _, _ = _split(p, 1, 3)
    assert_bitwise(b, restatement.run(p, 3, mode=R.MODE_RUN)["state"], "kh3d x1 vs oracle")
    assert_bitwise(b, a, "kh3d x1")

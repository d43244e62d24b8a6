"""Pin the plain-C oracle (oracle/qas_oracle.c) to the reference.

* against the committed golden fixtures, which were produced by the reference's
  own code compiled from its sources (tests/golden/make_golden.py);
* against the live reference binaries (oracle/_ref) when they are present.
Everything is compared bit-for-bit (== semantics).
"""
import os

import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise
from tests.golden import make_golden as G

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("kind", sorted(G.KAT_FUNCS))
def test_kat_golden(restatement, kind):
    funcs, nout = G.KAT_FUNCS[kind]
    inp = G.kat_inputs(kind)
    gold = np.load(os.path.join(GOLD, f"kat_{kind}.npz"))
    assert str(gold["input_sha"]) == G.sha(inp), "golden inputs drifted"
    for f in funcs:
        assert_bitwise(restatement.kat(f, inp, nout), gold[f"f{f}"], f"kat {kind} f{f}")


@pytest.mark.parametrize("case", G.STEP_CASES, ids=[c[0] for c in G.STEP_CASES])
def test_steps_golden(restatement, golden_steps, case):
    name, build, mode, nsteps = case
    p = build()
    assert str(golden_steps[f"{name}__insha"]) == G.sha(p.state), "golden input state drifted"
    r = restatement.run(p, nsteps, mode=mode)
    assert_bitwise(r["state"], golden_steps[f"{name}__state"], name)
    assert_bitwise(r["dts"], golden_steps[f"{name}__dts"], name + " dts")
    meta = golden_steps[f"{name}__meta"]
    assert r["steps"] == int(meta[0])


needs_ref = pytest.mark.skipif(not R.reference_available(2, 1), reason="reference oracle binaries not built")


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_live_reference_random(restatement, seed):
    rng = np.random.default_rng(100 + seed)
    dim = int(rng.integers(1, 4))
    rmn = int(rng.integers(0, 4))
    odr = int(rng.integers(1, 5))
    ctw = int(rng.integers(0, 2))
    n = {1: 40, 2: 14, 3: 6}[dim]
    p = P.smooth_wave(dim, n, rmn=rmn, odr=odr, rk=int(rng.integers(1, 4)), ctw=ctw, seed=seed)
    a = R.run_reference(p, R.MODE_RUN, nsteps=2, nthreads=2)
    b = restatement.run(p, 2, mode=R.MODE_RUN)
    assert_bitwise(b["state"], a["state"], f"dim{dim} rmn{rmn} odr{odr}")


@needs_ref
def test_live_reference_dissipative(restatement):
    p = P.kelvin_helmholtz(2, 12, mach=0.2, rmn=P.RMN_HLLD)
    p.nu0, p.eta0 = 1e-3, 2e-3
    a = R.run_reference(p, R.MODE_DSTEP, dt=2e-3, nthreads=2)
    b = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=2e-3)
    assert_bitwise(b["state"], a["state"], "dstep")


@needs_ref
@pytest.mark.parametrize("ctw", [0, 1])
def test_live_reference_dissipative_3d(restatement, ctw):
    """DMHD3D::dsptv (3D/MPI/MRX/dmhd3d_solve.cpp) and the sub-cycled exec_ loop around it."""
    p = P.smooth_wave(3, 7, ctw=ctw, rmn=P.RMN_MLAU, seed=3)
    p.nu0, p.eta0 = 0.04, 0.25
    a = R.run_reference(p, R.MODE_DSTEP, dt=2e-3, nthreads=2)
    b = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=2e-3)
    assert_bitwise(b["state"], a["state"], "dstep3d")
    a = R.run_reference(p, R.MODE_DRUN, nsteps=2, nthreads=2)
    b = restatement.run(p, 2, mode=R.MODE_DRUN)
    assert_bitwise(b["state"], a["state"], "drun3d")


@pytest.mark.skipif(not all(R.reference_available(d, c, gravity=True) for d in (2, 3) for c in (0, 1)),
                    reason="reference gravity builds not built")
@pytest.mark.parametrize("dim,ctw,rmn", [(2, 1, P.RMN_LHLLD), (2, 0, P.RMN_ROE), (3, 1, P.RMN_MLAU),
                                         (3, 0, P.RMN_HLLD)])
def test_live_reference_gravity(restatement, dim, ctw, rmn):
    """The gravity drivers (2D/SERIAL/RTI, 3D/MPI/RTI): prmtv/setdt energy shift, gravity work
    in the energy flux and the momentum update, the ghost-layer energy rule of bound()."""
    p = P.rayleigh_taylor(dim, 16 if dim == 2 else 8, 32 if dim == 2 else 16, rmn=rmn, ctw=ctw)
    a = R.run_reference(p, R.MODE_RUN, nsteps=3, nthreads=2)
    b = restatement.run(p, 3, mode=R.MODE_RUN)
    assert_bitwise(b["state"], a["state"], f"rt{dim}d")
    assert np.array_equal(a["dts"], b["dts"])
    a = R.run_reference(p, R.MODE_STEP, dt=1e-3, nthreads=2)
    b = restatement.run(p, 1, mode=R.MODE_STEP, dt=1e-3)
    assert_bitwise(b["state"], a["state"], f"rt{dim}d step")


@pytest.mark.skipif(not R.reference_available(1, 0, gravity="hall"), reason="reference Hall build not built")
@pytest.mark.parametrize("di,odr,d_ele", [(1e-3, 4, 0.0), (0.05, 4, 0.0), (0.02, 2, 0.0), (0.01, 4, 2.0),
                                          (0.0, 4, 3.0)])
def test_live_reference_hall(restatement, di, odr, d_ele):
    """The 1D Hall driver (1D/SERIAL/h-shock, HMHD1D): one hall_ call, and runs with the Hall
    sub-cycles of exec_ (di = 0.05 gives tens of sub-cycles per step); d_ele > 0 adds the
    electron-inertia CG correction (crcte) to ideal() and hall_()."""
    p = P.hall_shock(64, di=di, odr=odr, rk=3 if odr == 4 else 2, d_ele=d_ele)
    a = R.run_reference(p, R.MODE_DSTEP, dt=1e-3, nthreads=1)
    b = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=1e-3)
    assert_bitwise(b["state"], a["state"], "hall_")
    a = R.run_reference(p, R.MODE_RUN, nsteps=4, nthreads=1)
    b = restatement.run(p, 4, mode=R.MODE_RUN)
    assert_bitwise(b["state"], a["state"], "hall run")


@needs_ref
@pytest.mark.parametrize("dim", [2, 3])
def test_live_reference_dissipation_profiles(restatement, dim):
    """Per-cell nu/eta of the reconnection drivers' setdc (localized exp(-r/lambda) profiles)."""
    base = P.orszag_tang(24) if dim == 2 else P.kelvin_helmholtz(3, 10, mach=0.3, rmn=P.RMN_HLLD)
    p = P.localized_dissipation(base, 0.01, 0.06, 0.4)
    a = R.run_reference(p, R.MODE_DSTEP, dt=2e-3, nthreads=2)
    b = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=2e-3)
    assert_bitwise(b["state"], a["state"], "dsptv profiles")
    a = R.run_reference(p, R.MODE_DRUN, nsteps=3, nthreads=2)
    b = restatement.run(p, 3, mode=R.MODE_DRUN)
    assert_bitwise(b["state"], a["state"], "drun profiles")


@pytest.mark.skipif(not R.reference_available(2, 1, gravity="prim"), reason="reference prim builds not built")
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("mode", [1, 2])
def test_live_reference_other_reconstructions(restatement, dim, mode):
    """mhd_lrstate with mhd_reconst (mode 1, primitive variables) or mhd_c_reconst (mode 2,
    Athena-type eigenvectors) in place of mhd_m/a_reconst, against the reference built so."""
    p = {1: lambda: P.brio_wu(64), 2: lambda: P.orszag_tang(20, rmn=P.RMN_ROE),
         3: lambda: P.kelvin_helmholtz(3, 8, mach=0.3, rmn=P.RMN_LHLLD)}[dim]()
    p.char_mode = mode
    a = R.run_reference(p, R.MODE_RUN, nsteps=3, nthreads=2)
    b = restatement.run(p, 3, mode=R.MODE_RUN)
    assert_bitwise(b["state"], a["state"], f"char_mode {mode} {dim}d")


@pytest.mark.skipif(R.o3_binary(2) is None or R.o3_binary(3) is None, reason="no -O3 timing build for this host")
@pytest.mark.parametrize("dim", [2, 3])
def test_o3_timing_build_runs_the_same_case(dim):
    """The -O3 -march timing build is the same driver: equal to round-off (FMA contraction),
    not bitwise, so it never pins anything."""
    p = P.orszag_tang(32) if dim == 2 else P.kelvin_helmholtz(3, 8, mach=0.3, rmn=P.RMN_MLAU)
    a = R.run_reference(p, R.MODE_RUN, nsteps=3, nthreads=2)
    b = R.run_reference(p, R.MODE_RUN, nsteps=3, nthreads=2, exe=R.o3_binary(dim))
    scale = np.abs(a["state"]).max()
    assert np.abs(a["state"] - b["state"]).max() <= 1e-9 * scale

"""Parity of the CUDA path (through the C-ABI) with the reference.

Bit-exact (== semantics) comparisons:
* every golden case (made by the reference's own code) on the same inputs;
* the plain-C oracle at moderate sizes (2D 128^2, 3D 24^3) for every solver;
* single ideal(dt) / dsptv(dt) calls and exec_ loop termination rules.
At the benchmark sizes, size-independent properties: div B at round-off, mass
conservation on periodic grids, determinism of repeated runs.
"""
import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise, run_gpu
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", G.STEP_CASES, ids=[c[0] for c in G.STEP_CASES])
def test_golden_cases(golden_steps, case):
    name, build, mode, nsteps = case
    p = build()
    r = run_gpu(p, mode, nsteps)
    assert_bitwise(r["state"], golden_steps[f"{name}__state"], name)
    assert r["steps"] == int(golden_steps[f"{name}__meta"][0])


@pytest.mark.parametrize("rmn", range(4))
@pytest.mark.parametrize("odr", [2, 4])
def test_ot2d_vs_oracle(restatement, rmn, odr):
    p = P.orszag_tang(96, rmn=rmn, odr=odr)
    a = restatement.run(p, 6, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 6)
    assert_bitwise(b["state"], a["state"], f"ot rmn{rmn} odr{odr}")


@pytest.mark.parametrize("rmn", range(4))
def test_kh3d_vs_oracle(restatement, rmn):
    p = P.kelvin_helmholtz(3, 20, mach=0.3, rmn=rmn, nym=16, nzm=12)
    a = restatement.run(p, 3, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 3)
    assert_bitwise(b["state"], a["state"], f"kh3d rmn{rmn}")


@pytest.mark.parametrize("ctw", [0, 1])
@pytest.mark.parametrize("odr", [1, 3])
def test_kh3d_ctw_odr(restatement, ctw, odr):
    p = P.kelvin_helmholtz(3, 10, mach=0.5, rmn=P.RMN_MLAU, ctw=ctw, odr=odr, rk=2)
    a = restatement.run(p, 2, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 2)
    assert_bitwise(b["state"], a["state"], f"kh3d ctw{ctw} odr{odr}")


def test_single_ideal_step(restatement):
    p = P.orszag_tang(40, rmn=P.RMN_LHLLD)
    a = restatement.run(p, 1, mode=R.MODE_STEP, dt=0.01)
    b = run_gpu(p, R.MODE_STEP, dt=0.01)
    assert_bitwise(b["state"], a["state"], "step")


def test_single_dsptv(restatement):
    p = P.kelvin_helmholtz(2, 32, mach=0.2)
    p.nu0, p.eta0 = 2e-3, 1e-3
    a = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=3e-3)
    b = run_gpu(p, R.MODE_DSTEP, dt=3e-3)
    assert_bitwise(b["state"], a["state"], "dsptv")


@pytest.mark.parametrize("odr", [2, 4])
def test_single_dsptv_3d(restatement, odr):
    p = P.smooth_wave(3, 20, odr=odr, seed=5)
    p.nu0, p.eta0 = 3e-3, 4e-3
    a = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=2e-3)
    b = run_gpu(p, R.MODE_DSTEP, dt=2e-3)
    assert_bitwise(b["state"], a["state"], f"dsptv3d odr{odr}")


@pytest.mark.parametrize("use_graph", [False, True])
def test_dissipative_run_3d(restatement, use_graph):
    """exec_ of DMHD3D: ideal step, then the sub-cycled dsptv (two sub-cycles here)."""
    p = P.kelvin_helmholtz(3, 16, mach=0.3, rmn=P.RMN_HLLD)
    p.nu0, p.eta0 = 0.01, 0.1
    a = restatement.run(p, 4, mode=R.MODE_DRUN)
    assert np.isfinite(a["state"]).all()
    b = run_gpu(p, R.MODE_DRUN, 4, use_graph=use_graph)
    assert_bitwise(b["state"], a["state"], "drun3d")


@pytest.mark.parametrize("use_graph", [False, True])
def test_graph_and_eager_agree(restatement, use_graph):
    p = P.orszag_tang(48)
    a = restatement.run(p, 7, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 7, use_graph=use_graph)
    assert_bitwise(b["state"], a["state"], f"graph={use_graph}")


def test_exec_rule_2d(restatement):
    p = P.orszag_tang(32, tmax=0.12)
    a = restatement.run(p, 0, mode=R.MODE_EXEC)
    b = run_gpu(p, R.MODE_EXEC)
    assert b["steps"] == a["steps"]
    assert b["tim"] == a["tim"]
    assert_bitwise(b["state"], a["state"], "exec 2d")


def test_exec_rule_1d(restatement):
    p = P.brio_wu(128, tmax=0.03)
    a = restatement.run(p, 0, mode=R.MODE_EXEC)
    b = run_gpu(p, R.MODE_EXEC)
    assert b["steps"] == a["steps"]
    assert_bitwise(b["state"], a["state"], "exec 1d")


def test_run_in_pieces_matches_one_call(restatement):
    p = P.orszag_tang(32)
    a = restatement.run(p, 9, mode=R.MODE_RUN)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        for k in (3, 1, 5):   # odd split exercises the graph parity handling
            ctx.run(max_steps=k, flg=1, stop_rule=0, cfl=p.cfl)
        out = ctx.download(p.state.shape)
    assert_bitwise(out, a["state"], "pieces")


def test_async_block_copies(restatement):
    """qas_upload_block_async / qas_download_block_async from pinned host blocks: queued in stream
    order behind the run, the state read back after qas_sync equals the oracle's 4-step result,
    and an upload queued behind a download does not disturb what the download reads."""
    import torch
    p = P.orszag_tang(32)
    a = restatement.run(p, 4, mode=R.MODE_RUN)
    with L.Context.from_problem(p) as ctx:
        up = torch.empty(8 * ctx.nd, dtype=torch.float64, pin_memory=True).numpy()
        up[:] = p.state.reshape(-1)
        down = torch.empty(8 * ctx.nd, dtype=torch.float64, pin_memory=True).numpy()
        ctx.upload_async(up)
        ctx.run(max_steps=4, flg=1, stop_rule=0, cfl=p.cfl)
        ctx.download_async(down)
        ctx.upload_async(up)  # restores the initial state after the download in stream order
        ctx.sync()
        assert_bitwise(down.reshape(p.state.shape), a["state"], "async round trip")
        assert_bitwise(ctx.download(p.state.shape), p.state, "upload after download")


def test_contexts_on_host_threads(restatement):
    """Distinct contexts are independent: four contexts (2D and 3D, different solvers) stepped at
    the same time from four host threads (ctypes releases the GIL during each call) give the
    oracle's results bit for bit."""
    import threading
    probs = [P.orszag_tang(32), P.kelvin_helmholtz(3, 12, mach=0.3, rmn=P.RMN_MLAU),
             P.smooth_wave(2, 24, rmn=P.RMN_ROE), P.kelvin_helmholtz(2, 32, mach=0.3, rmn=P.RMN_LHLLD)]
    want = [restatement.run(p, 3, mode=R.MODE_RUN)["state"] for p in probs]
    got = [None] * len(probs)
    errs = []

    def work(q):
        try:
            p = probs[q]
            with L.Context.from_problem(p) as ctx:
                ctx.upload(p.state)
                ctx.run(max_steps=3, flg=1, stop_rule=0, cfl=p.cfl)
                got[q] = ctx.download(p.state.shape)
        except Exception as e:  # reported below, on the test's thread
            errs.append(e)

    threads = [threading.Thread(target=work, args=(q,)) for q in range(len(probs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errs, errs
    for q in range(len(probs)):
        assert_bitwise(got[q], want[q], probs[q].name)


def test_cfl_reduction_matches(restatement):
    p = P.kelvin_helmholtz(3, 12, mach=0.4)
    import ctypes
    g = restatement.grid(p)
    st = np.ascontiguousarray(p.state)
    vm = restatement.lib.qo_cfl_dt(ctypes.byref(g), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1.0)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(st)
        assert ctx.cfl_vmax() == vm


def test_invalid_bc_rejected_on_device():
    p = P.smooth_wave(2, 8, dn=((3,) * 8, (0,) * 8, (0,) * 8))
    with pytest.raises(L.QasError) as e:
        L.Context.from_problem(p)
    assert e.value.status == L.QAS_ERR_INVALID


def test_nonfinite_state_is_reported():
    p = P.orszag_tang(16)
    st = p.state.copy()
    st[0, 0, 10, 10] = -1.0   # negative density in the interior
    with L.Context.from_problem(p) as ctx:
        ctx.upload(st)
        ctx.bound()
        ctx.step(1e-3)
        with pytest.raises(L.QasError) as e:
            ctx.sync()
        assert e.value.status == L.QAS_ERR_NONFINITE


# ---------------------------------------------------------------------------
# benchmark sizes: size-independent properties
# ---------------------------------------------------------------------------

def interior(p, a):
    s = slice(4, -4)
    if p.dim == 2:
        return a[..., 0, s, s]
    return a[..., s, s, s]


def test_ot_1024_invariants():
    p = P.orszag_tang(1024)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        d0 = ctx.max_divb()
        m0 = interior(p, p.state)[0].sum()
        info = ctx.run(max_steps=20, flg=1, stop_rule=0, cfl=p.cfl)
        out = ctx.download(p.state.shape)
        d1 = ctx.max_divb()
    assert info.steps == 20
    assert np.isfinite(out).all()
    assert d0 < 1e-11 and d1 < 1e-11, (d0, d1)
    m1 = interior(p, out)[0].sum()
    assert abs(m1 - m0) / m0 < 1e-12


def test_kh_256_determinism_and_divb():
    p = P.kelvin_helmholtz(3, 256)
    outs = []
    for _ in range(2):
        with L.Context.from_problem(p) as ctx:
            ctx.upload(p.state)
            ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
            outs.append(ctx.download(p.state.shape))
            d = ctx.max_divb()
    assert np.isfinite(outs[0]).all()
    assert_bitwise(outs[0], outs[1], "repeat")
    assert d < 1e-10, d


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("dim,rmn", [(1, 1), (2, 1), (2, 3), (3, 0), (3, 1), (3, 2), (3, 3)])
def test_sweep_forms(restatement, dim, rmn, fused):
    """Both face-sweep forms (two kernels, or one fused kernel: the 3D default) against the
    oracle; odd extents and a non-cubic 3D box exercise the flattened x warps and the y / z
    segment ends."""
    p = {1: lambda: P.brio_wu(96, rmn=rmn), 2: lambda: P.orszag_tang(48, nym=37, rmn=rmn),
         3: lambda: P.kelvin_helmholtz(3, 12, nym=9, nzm=15, mach=0.3, rmn=rmn)}[dim]()
    a = restatement.run(p, 3, mode=R.MODE_RUN)
    with L.Context.from_problem(p) as ctx:
        ctx.set_option(L.QAS_OPT_FUSED_SWEEP, fused)
        ctx.upload(p.state)
        ctx.run(max_steps=3, flg=p.flg, stop_rule=0, cfl=p.cfl)
        out = ctx.download(p.state.shape)
    assert_bitwise(out, a["state"], f"fused={fused} dim{dim} rmn{rmn}")


def test_profile_run_reports_kernels():
    p = P.orszag_tang(64)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        prof = ctx.profile(2)
    assert prof["k_lr"][0] == 2 * 3 * 2 and prof["k_flux"][0] == 2 * 3 * 2
    assert all(ms > 0 for _, ms in prof.values())


@pytest.mark.parametrize("dim", [2, 3])
def test_tiles_bit_identical(restatement, dim):
    p = P.orszag_tang(40) if dim == 2 else P.kelvin_helmholtz(3, 12, mach=0.3)
    a = restatement.run(p, 2, mode=R.MODE_RUN)
    tiles = [(128, 1, 1), (64, 2, 1), (32, 4, 1)] + ([(32, 2, 2), (32, 1, 4)] if dim == 3 else [(32, 2, 1)])
    for t in tiles:
        with L.Context.from_problem(p) as ctx:
            ctx.set_tile("all", *t)
            ctx.upload(p.state)
            ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
            assert_bitwise(ctx.download(p.state.shape), a["state"], f"tile {t}")


def test_autotune_restores_state(restatement):
    p = P.orszag_tang(64)
    a = restatement.run(p, 3, mode=R.MODE_RUN)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        tiles = ctx.autotune(1)
        assert set(tiles) == {"k_prim", "k_dv", "k_lr", "k_flux", "k_emf", "k_update"}
        ctx.run(max_steps=3, flg=1, stop_rule=0, cfl=p.cfl)
        assert_bitwise(ctx.download(p.state.shape), a["state"], "after autotune")


def _run_staging(p, staging, nsteps, use_graph=True):
    with L.Context.from_problem(p) as ctx:
        ctx.set_option(L.QAS_OPT_LR_STAGING, staging)
        ctx.upload(p.state)
        ctx.run(max_steps=nsteps, flg=1, stop_rule=0, cfl=p.cfl, use_graph=use_graph)
        return ctx.download(p.state.shape)


@pytest.mark.parametrize("case", ["ot2d_96", "ot2d_130x70", "kh3d_24", "kh3d_20x12x8_hlld", "wave3d_16_roe"])
def test_tma_staged_reconstruction(restatement, case):
    """The reconstruction with TMA-staged stencils (shared-memory ring, mbarriers) gives the
    same bits as the global-memory form and as the oracle, on grids whose tiles do not divide
    the extents (partial tiles, zero-filled out-of-range box parts)."""
    p = {"ot2d_96": lambda: P.orszag_tang(96),
         "ot2d_130x70": lambda: P.kelvin_helmholtz(2, 130, nym=70, mach=0.3, rmn=P.RMN_HLLD),
         "kh3d_24": lambda: P.kelvin_helmholtz(3, 24, mach=0.3),
         "kh3d_20x12x8_hlld": lambda: P.kelvin_helmholtz(3, 20, nym=12, nzm=8, mach=0.3, rmn=P.RMN_HLLD),
         "wave3d_16_roe": lambda: P.smooth_wave(3, 16, rmn=P.RMN_ROE, ctw=0)}[case]()
    a = _run_staging(p, 1, 4)
    b = _run_staging(p, 0, 4, use_graph=False)
    assert_bitwise(a, b, f"{case} staged vs global")
    o = restatement.run(p, 4, mode=R.MODE_RUN)
    assert_bitwise(a, o["state"], f"{case} staged vs oracle")


def test_tma_staging_unsupported_on_odd_extent():
    p = P.smooth_wave(2, 13)  # padded x extent 21: TMA rows would not be 16-byte multiples
    with L.Context.from_problem(p) as ctx:
        with pytest.raises(L.QasError) as e:
            ctx.set_option(L.QAS_OPT_LR_STAGING, 1)
        assert e.value.status == L.QAS_ERR_UNSUPPORTED
        ctx.set_option(L.QAS_OPT_LR_STAGING, 0)


@pytest.mark.parametrize("dim,rmn,ctw", [(2, P.RMN_LHLLD, 1), (2, P.RMN_HLLD, 0), (3, P.RMN_MLAU, 1),
                                         (3, P.RMN_ROE, 0)])
def test_gravity_vs_oracle(restatement, dim, rmn, ctw):
    """Gravity drivers (2D/SERIAL/RTI, 3D/MPI/RTI) through qas_set_gravity."""
    p = P.rayleigh_taylor(dim, 64 if dim == 2 else 16, 128 if dim == 2 else 32, rmn=rmn, ctw=ctw)
    a = restatement.run(p, 6, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 6)
    assert_bitwise(b["state"], a["state"], f"rt{dim}d rmn{rmn}")
    assert b["steps"] == 6


def test_gravity_forms_and_switch(restatement):
    """Graph, eager, fused sweep and TMA-staged reconstruction agree with gravity on; switching
    gravity off gives the plain driver; the dissipative form refuses a gravity context."""
    p = P.rayleigh_taylor(2, 64, 128)
    ref = restatement.run(p, 4, mode=R.MODE_RUN)["state"]
    outs = []
    for opt, val, graph in ((None, 0, True), (None, 0, False), (L.QAS_OPT_FUSED_SWEEP, 1, False),
                            (L.QAS_OPT_LR_STAGING, 1, True)):
        with L.Context.from_problem(p) as ctx:
            if opt is not None:
                ctx.set_option(opt, val)
            ctx.upload(p.state)
            ctx.run(max_steps=4, flg=1, stop_rule=0, cfl=p.cfl, use_graph=graph)
            outs.append(ctx.download(p.state.shape))
    for o in outs:
        assert_bitwise(o, ref, "gravity form")
    plain = p.copy()
    plain.phi = None
    a = restatement.run(plain, 3, mode=R.MODE_RUN)["state"]
    with L.Context.from_problem(p) as ctx:
        ctx.set_gravity(None)
        ctx.upload(p.state)
        ctx.run(max_steps=3, flg=1, stop_rule=0, cfl=p.cfl)
        assert_bitwise(ctx.download(p.state.shape), a, "gravity off")
        ctx.set_gravity(p.phi)
        with pytest.raises(L.QasError) as e:
            ctx.dissipate(1e-3, 0.0, 1e-3)
        assert e.value.status == L.QAS_ERR_UNSUPPORTED



@pytest.mark.parametrize("di,odr,d_ele", [(1e-3, 4, 0.0), (0.05, 4, 0.0), (0.02, 3, 0.0), (0.01, 4, 2.0),
                                          (0.0, 4, 1.0), (0.02, 2, 1.0)])
def test_hall_vs_oracle(restatement, di, odr, d_ele):
    """Hall form of the 1D driver (qas_set_hall): one hall_ call, runs with Hall sub-cycles, and
    the exec_(0) loop of the driver; with d_ele > 0 the electron-inertia CG correction too."""
    p = P.hall_shock(128, di=di, odr=odr, rk=3, d_ele=d_ele)
    a = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=1e-3)
    b = run_gpu(p, R.MODE_DSTEP, dt=1e-3)
    assert_bitwise(b["state"], a["state"], "hall_")
    a = restatement.run(p, 5, mode=R.MODE_RUN)
    b = run_gpu(p, R.MODE_RUN, 5)
    assert_bitwise(b["state"], a["state"], "hall run")
    q = P.hall_shock(128, di=di, odr=odr, tmax=0.01, d_ele=d_ele)
    a = restatement.run(q, 0, mode=R.MODE_EXEC)
    b = run_gpu(q, R.MODE_EXEC)
    assert b["steps"] == a["steps"]
    assert_bitwise(b["state"], a["state"], "hall exec")


def test_hall_rejects_unsupported():
    with L.Context.from_problem(P.orszag_tang(16)) as ctx:
        with pytest.raises(L.QasError):
            ctx.set_hall(1e-3)
        with pytest.raises(L.QasError):
            ctx.hall(1e-3)
    with L.Context.from_problem(P.orszag_tang(16)) as ctx:
        with pytest.raises(L.QasError) as e:
            ctx.set_hall(1e-3, 1e-2)  # the Hall driver is 1D
        assert e.value.status == L.QAS_ERR_UNSUPPORTED



@pytest.mark.parametrize("dim,use_graph", [(2, True), (2, False), (3, True)])
def test_dissipation_profiles(restatement, dim, use_graph):
    """Per-cell nu/eta (qas_set_dissipation): one dsptv call and the dissipative exec_ loop."""
    base = P.orszag_tang(48) if dim == 2 else P.kelvin_helmholtz(3, 16, mach=0.3, rmn=P.RMN_HLLD)
    p = P.localized_dissipation(base, 0.01, 0.06, 0.4)
    a = restatement.run(p, 1, mode=R.MODE_DSTEP, dt=2e-3)
    b = run_gpu(p, R.MODE_DSTEP, dt=2e-3)
    assert_bitwise(b["state"], a["state"], "dsptv profiles")
    a = restatement.run(p, 4, mode=R.MODE_DRUN)
    b = run_gpu(p, R.MODE_DRUN, 4, use_graph=use_graph)
    assert_bitwise(b["state"], a["state"], "drun profiles")
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        with pytest.raises(L.QasError) as e:  # one source of coefficients at a time
            ctx.run(max_steps=1, flg=1, stop_rule=0, cfl=p.cfl, nu0=1e-3)
        assert e.value.status == L.QAS_ERR_INVALID


@pytest.mark.parametrize("grav", [False, True])
def test_primitives_readback(grav):
    """qas_primitives: prmtv of the current state (interior cells checked against the same
    formulas in numpy, op for op), without modifying the state in the gravity form."""
    p = P.rayleigh_taylor(2, 32, 64) if grav else P.orszag_tang(32)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
        st = ctx.download(p.state.shape)
        pv = ctx.primitives(p.state.shape[1:])
        assert np.array_equal(ctx.download(p.state.shape), st)
    s = st[:, 0]
    j, i = slice(4, -4), slice(4, -4)
    bx, by = s[4], s[5]
    cx = 0.0625 * (9.0 * (bx[j, 4:-4] + bx[j, 5:-3]) - (bx[j, 3:-5] + bx[j, 6:-2]))
    cy = 0.0625 * (9.0 * (by[4:-4, i] + by[5:-3, i]) - (by[3:-5, i] + by[6:-2, i]))
    cz = s[6][j, i]
    ro = s[0][j, i]
    iro = 1.0 / ro
    vx, vy, vz = s[1][j, i] * iro, s[2][j, i] * iro, s[3][j, i] * iro
    en = s[7][j, i] - ro * p.phi[0][j, i] if grav else s[7][j, i]
    pr = (p.gam - 1) * (en - 0.5 * (ro * (vx * vx + vy * vy + vz * vz) + (cx * cx + cy * cy + cz * cz)))
    for name, ref in (("vx", vx), ("vy", vy), ("vz", vz), ("pr", pr), ("cx", cx), ("cy", cy), ("cz", cz)):
        assert_bitwise(pv[name][0][j, i], ref, name)



@pytest.mark.parametrize("case", ["bw1d", "ot2d", "kh3d_mlau", "ot2d_fused", "ot2d_staged"])
@pytest.mark.parametrize("mode", [1, 2])
def test_other_reconstructions(restatement, case, mode):
    """char_mode = 1: face values by mhd_reconst (each primitive on its own); char_mode = 2: by
    mhd_c_reconst (Athena-type eigenvectors for every state); every form."""
    p = {"bw1d": lambda: P.brio_wu(128), "ot2d": lambda: P.orszag_tang(64, rmn=P.RMN_HLLD),
         "kh3d_mlau": lambda: P.kelvin_helmholtz(3, 16, mach=0.3), "ot2d_fused": lambda: P.orszag_tang(64),
         "ot2d_staged": lambda: P.orszag_tang(64)}[case]()
    p.char_mode = mode
    a = restatement.run(p, 4, mode=R.MODE_RUN)
    with L.Context.from_problem(p) as ctx:
        if case.endswith("fused"):
            ctx.set_option(L.QAS_OPT_FUSED_SWEEP, 1)
        if case.endswith("staged"):
            ctx.set_option(L.QAS_OPT_LR_STAGING, 1)
        ctx.upload(p.state)
        ctx.run(max_steps=4, flg=p.flg, stop_rule=0, cfl=p.cfl, use_graph=not case.endswith("fused"))
        b = ctx.download(p.state.shape)
    assert_bitwise(b, a["state"], f"char_mode {mode} {case}")

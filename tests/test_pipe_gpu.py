"""qas_step_host: one exec_ step on host arrays with the copies overlapped by items of planes.

Its contract is the serial composition qas_upload_block + qas_run(one step) +
qas_download_block: every step's state (interior and ghosts) and loop state (n, tim, dt) must
be bit-identical to it, over several consecutive steps (setdt every second step), for every
solver, both boundary kinds of the last axis (periodic: the seam item wraps; open), 2D and 3D,
any item count, with the output block aliasing the input or not.  Forms the wave does not
cover (1D, gravity) must give the same bits through the serial path."""
import ctypes

import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise

pytestmark = pytest.mark.gpu


def _prim(p):
    p.char_mode = 1
    return p


CASES = {
    "ot2d_128_hlld": lambda: P.orszag_tang(128),
    "ot2d_96x160_roe_ctw0": lambda: P.orszag_tang(96, rmn=P.RMN_ROE, ctw=0, nym=160),
    "kh2d_64x128_mlau_open_y": lambda: P.kelvin_helmholtz(2, 64, nym=128, mach=0.3),
    "kh2d_80x144_lhlld_odr2": lambda: P.kelvin_helmholtz(2, 80, nym=144, mach=0.5, rmn=P.RMN_LHLLD, odr=2),
    "ot2d_128_prim": lambda: _prim(P.orszag_tang(128)),
    "kh3d_16x16x96_mlau": lambda: P.kelvin_helmholtz(3, 16, nzm=96, mach=0.3),
    "kh3d_24x16x80_lhlld": lambda: P.kelvin_helmholtz(3, 24, nym=16, nzm=80, mach=0.3, rmn=P.RMN_LHLLD),
    "wave3d_20_open_z_roe": lambda: P.smooth_wave(3, 20, rmn=P.RMN_ROE,
                                                  dn=((0,) * 8, (0,) * 8, (2, 1, 1, -1, 1, 1, -1, 2))),
}


def _serial(p, nsteps):
    """The reference composition: upload, one exec_ step, download, per step."""
    h = np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1).copy()
    states, infos = [], []
    with L.Context.from_problem(p) as ctx:
        for _ in range(nsteps):
            ctx.upload(h)
            info = ctx.run(max_steps=1, flg=p.flg, stop_rule=0, cfl=p.cfl, use_graph=False)
            ctx.download_into(h)
            states.append(h.copy())
            infos.append((info.n, info.tim, info.dt, info.steps))
    return states, infos


def _block(p, pinned):
    """The initial state as a host block of 8*nd float64 (pinned: page-locked by torch)."""
    a = np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1)
    if not pinned:
        return a.copy(), None
    import torch
    t = torch.empty((8, p.nd), dtype=torch.float64, pin_memory=True)
    t.copy_(torch.from_numpy(a))
    return t.numpy(), t  # keep the tensor alive beside its view


def _piped(p, nsteps, items=None, alias=True, pinned=False, replan_at=None, lanes=None, fused=None):
    h, keep_h = _block(p, pinned)
    out, keep_o = (h, None) if alias else _block(p, pinned)
    states, infos = [], []
    with L.Context.from_problem(p) as ctx:
        if fused is not None:
            ctx.set_option(L.QAS_OPT_FUSED_SWEEP, fused)
        if lanes is not None:
            ctx.set_option(L.QAS_OPT_PIPE_LANES, lanes)
        if items is not None:
            ctx.set_option(L.QAS_OPT_PIPE_ITEMS, items)
        for step in range(nsteps):
            if replan_at is not None and step == replan_at:
                ctx.set_option(L.QAS_OPT_PIPE_ITEMS, 3)
            info = ctx.step_host(h, out, flg=p.flg, stop_rule=0, cfl=p.cfl)
            if not alias:
                h, out = out, h
            states.append(h.copy())
            infos.append((info.n, info.tim, info.dt, info.steps))
        # the context's device state is the last step's result
        assert np.array_equal(ctx.download(), h)
    return states, infos


def _compare(a, b, label):
    (sa, ia), (sb, ib) = a, b
    for k, (x, y) in enumerate(zip(sa, sb)):
        assert_bitwise(y, x, f"{label} step {k + 1}")
    assert ib == ia, (label, ia, ib)


@pytest.mark.parametrize("case", list(CASES))
def test_step_host_matches_serial_composition(case):
    p = CASES[case]()
    _compare(_serial(p, 5), _piped(p, 5), case)


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("case,fused", [("ot2d_96x160_roe_ctw0", 1), ("kh2d_64x128_mlau_open_y", 1),
                                        ("kh3d_16x16x96_mlau", 0), ("wave3d_20_open_z_roe", 0)])
def test_step_host_sweep_forms(case, fused, pinned):
    """The wave's face sweeps in the form that is not the dimension's default (fused windows in
    2D: x rows of the window's planes and the last-axis march over its faces; two kernels in 3D)
    give the serial composition's bits as well."""
    if pinned:
        pytest.importorskip("torch")
    p = CASES[case]()
    _compare(_serial(p, 5), _piped(p, 5, items=12, pinned=pinned, fused=fused), f"{case} fused={fused}")


@pytest.mark.parametrize("items", [1, 2, 3, 5, 16, 64])
def test_step_host_any_item_count(items):
    p = P.orszag_tang(256, nym=192)
    _compare(_serial(p, 4), _piped(p, 4, items=items), f"items={items}")


def test_step_host_separate_output_block():
    p = P.kelvin_helmholtz(3, 16, nzm=64, mach=0.3)
    _compare(_serial(p, 4), _piped(p, 4, alias=False), "out != in")


def test_step_host_matches_oracle(restatement):
    p = P.orszag_tang(64, nym=96)
    states, infos = _piped(p, 4)
    want = restatement.run(p, 4, mode=R.MODE_RUN)
    assert_bitwise(states[-1].reshape(p.state.shape), want["state"], "step_host vs oracle")
    assert infos[-1][2] == want["dt"]


@pytest.mark.parametrize("case", ["bw1d", "rt2d_gravity"])
def test_step_host_serial_forms(case):
    p = {"bw1d": lambda: P.brio_wu(128), "rt2d_gravity": lambda: P.rayleigh_taylor(2, 32, 96)}[case]()
    _compare(_serial(p, 3), _piped(p, 3), case)


@pytest.mark.parametrize("case", ["ot2d_128_hlld", "kh2d_64x128_mlau_open_y", "ot2d_128_prim",
                                  "kh3d_16x16x96_mlau", "wave3d_20_open_z_roe"])
def test_step_host_pinned_graph(case):
    """Pinned blocks take the captured graph (one per setdt parity, replayed every other step)."""
    pytest.importorskip("torch")
    p = CASES[case]()
    _compare(_serial(p, 6), _piped(p, 6, pinned=True), f"{case} pinned")


def test_step_host_pinned_graph_rebuilds():
    """A new block pair (in/out swapped every step) or a new item plan captures a new graph."""
    pytest.importorskip("torch")
    p = P.orszag_tang(160, nym=200)
    _compare(_serial(p, 5), _piped(p, 5, pinned=True, alias=False), "swapped blocks")
    _compare(_serial(p, 6), _piped(p, 6, pinned=True, replan_at=3), "re-planned")


def test_step_host_stop_rule_reached():
    """exec_'s time limit (tmax = dtrec * nout) reached after three steps: later calls take no
    step and hand back the input, as qas_run does."""
    p = P.orszag_tang(128)
    with L.Context.from_problem(p) as c0:
        c0.upload(p.state)
        tmax = 2.5 * c0.run(max_steps=1, flg=1, stop_rule=0, cfl=p.cfl).dt
    h1 = np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1).copy()
    h2 = h1.copy()
    with L.Context.from_problem(p) as a, L.Context.from_problem(p) as b:
        for k in range(6):
            a.upload(h1)
            ia = a.run(max_steps=1, flg=1, stop_rule=1, cfl=p.cfl, dtrec=tmax, nout=1, use_graph=False)
            a.download_into(h1)
            ib = b.step_host(h2, h2, flg=1, stop_rule=1, cfl=p.cfl, dtrec=tmax, nout=1)
            assert_bitwise(h2, h1, f"call {k + 1}")
            assert (ib.steps, ib.n, ib.tim, ib.dt) == (ia.steps, ia.n, ia.tim, ia.dt), k
        assert ia.steps == 0 and ia.n < 6


def test_pipe_items_option_range():
    p = P.orszag_tang(64)
    with L.Context.from_problem(p) as ctx:
        for bad in (0, -1, 65):
            with pytest.raises(L.QasError):
                ctx.set_option(L.QAS_OPT_PIPE_ITEMS, bad)
        ctx.set_option(L.QAS_OPT_PIPE_ITEMS, 64)


def test_step_host_rejects_null_arguments():
    p = P.orszag_tang(64)
    h = np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1).copy()
    hp = h.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    null = ctypes.POINTER(ctypes.c_double)()
    with L.Context.from_problem(p) as ctx:
        o = L.RunOpts(1, 1, 0, float(p.cfl), 1.0, 1, 0, 0.0, 0.0)
        info = L.RunInfo()
        lib = ctx.lib
        assert lib.qas_step_host(ctx.h, null, hp, ctypes.byref(o), ctypes.byref(info)) == L.QAS_ERR_INVALID
        assert lib.qas_step_host(ctx.h, hp, null, ctypes.byref(o), ctypes.byref(info)) == L.QAS_ERR_INVALID
        assert lib.qas_step_host(ctx.h, hp, hp, None, ctypes.byref(info)) == L.QAS_ERR_INVALID
        bad = L.RunOpts(1, 1, 3, float(p.cfl), 1.0, 1, 0, 0.0, 0.0)  # no stop rule 3
        assert lib.qas_step_host(ctx.h, hp, hp, ctypes.byref(bad), ctypes.byref(info)) == L.QAS_ERR_INVALID
        ctx.step_host(h, h, flg=1, stop_rule=0, cfl=p.cfl)  # the context is still usable


@pytest.mark.parametrize("lanes", [1, 2])
@pytest.mark.parametrize("case", ["ot2d_128_hlld", "kh3d_16x16x96_mlau"])
def test_step_host_fewer_lanes(case, lanes):
    """The stages on fewer streams (what a context gets when the extra work arrays do not fit):
    one lane keeps every intermediate's halo; bit-identical all the same."""
    p = CASES[case]()
    _compare(_serial(p, 5), _piped(p, 5, lanes=lanes, items=12), f"{case} lanes={lanes}")
    _compare(_serial(p, 4), _piped(p, 4, lanes=lanes, pinned=True), f"{case} lanes={lanes} pinned")


def test_pipe_lanes_option_fixed_after_first_use():
    p = P.orszag_tang(64)
    h = np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1).copy()
    with L.Context.from_problem(p) as ctx:
        for bad in (0, 4):
            with pytest.raises(L.QasError):
                ctx.set_option(L.QAS_OPT_PIPE_LANES, bad)
        ctx.set_option(L.QAS_OPT_PIPE_LANES, 2)
        for _ in range(2):
            ctx.step_host(h, h, flg=1, stop_rule=0, cfl=p.cfl)
        with pytest.raises(L.QasError):
            ctx.set_option(L.QAS_OPT_PIPE_LANES, 3)


def test_step_host_device_blocks():
    """In and out may be device memory (e.g. torch CUDA tensors): same bits as the serial
    composition on host arrays."""
    torch = pytest.importorskip("torch")
    p = P.kelvin_helmholtz(2, 64, nym=128, mach=0.3)
    want_states, want_infos = _serial(p, 4)
    d = torch.from_numpy(np.ascontiguousarray(p.state, dtype=np.float64).reshape(8, -1).copy()).cuda()
    dp = ctypes.cast(d.data_ptr(), ctypes.POINTER(ctypes.c_double))
    infos = []
    with L.Context.from_problem(p) as ctx:
        o = L.RunOpts(1, int(p.flg), 0, float(p.cfl), 1.0, 1, 0, 0.0, 0.0)
        for k in range(4):
            info = L.RunInfo()
            assert ctx.lib.qas_step_host(ctx.h, dp, dp, ctypes.byref(o), ctypes.byref(info)) == 0
            torch.cuda.synchronize()
            assert_bitwise(d.cpu().numpy(), want_states[k], f"device blocks step {k + 1}")
            infos.append((info.n, info.tim, info.dt, info.steps))
    assert infos == want_infos

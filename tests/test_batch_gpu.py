"""The batched ensemble (qas_batch_*): every instance bit-identical to its own
single-instance run of the oracle, with uneven sizes, mixed solvers and
boundaries, per-instance dt, any tile, and after autotuning."""
import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise

pytestmark = pytest.mark.gpu


def small_ensemble():
    return P.ensemble(7, lo=12, hi=40, seed=11)


def test_batch_matches_oracle(restatement):
    probs = small_ensemble()
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        info = b.run(max_steps=5, flg=1, stop_rule=0, cfl=0.4)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        want = restatement.run(p, 5, mode=R.MODE_RUN)
        assert info[q][0] == 5
        assert info[q][2] == want["dt"]
        assert_bitwise(outs[q], want["state"], p.name)


def test_batch_exec_rule_per_instance(restatement):
    probs = small_ensemble()[:4]
    for p in probs:
        p.dtrec, p.nout = 0.05, 1
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        info = b.run(max_steps=0, flg=1, stop_rule=1, cfl=0.4, dtrec=0.05, nout=1)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        want = restatement.run(p, 0, mode=R.MODE_EXEC)
        assert info[q][0] == want["steps"], p.name
        assert_bitwise(outs[q], want["state"], p.name)


@pytest.mark.parametrize("tile", [(128, 1, 1), (64, 2, 1), (32, 2, 1)])
def test_batch_tiles(restatement, tile):
    probs = small_ensemble()[:3]
    with L.Batch(probs) as b:
        b.set_tile("all", *tile)
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        b.run(max_steps=3, flg=1, stop_rule=0, cfl=0.4, use_graph=False)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        assert_bitwise(outs[q], restatement.run(p, 3, mode=R.MODE_RUN)["state"], f"{p.name} {tile}")


def test_batch_autotune_then_run(restatement):
    probs = small_ensemble()[:3]
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        b.autotune(1)
        b.run(max_steps=4, flg=1, stop_rule=0, cfl=0.4)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        assert_bitwise(outs[q], restatement.run(p, 4, mode=R.MODE_RUN)["state"], p.name)


def test_batch_3d(restatement):
    probs = [P.kelvin_helmholtz(3, 8, mach=0.3, rmn=P.RMN_MLAU),
             P.kelvin_helmholtz(3, 10, mach=0.5, rmn=P.RMN_HLLD, nym=8, nzm=12, seed=3)]
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        b.run(max_steps=2, flg=1, stop_rule=0, cfl=0.4)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        assert_bitwise(outs[q], restatement.run(p, 2, mode=R.MODE_RUN)["state"], p.name)


def test_batch_rejects_mixed_order():
    probs = [P.orszag_tang(16), P.orszag_tang(16, odr=2)]
    with pytest.raises(L.QasError):
        L.Batch(probs)
    with pytest.raises(L.QasError):  # 1D instances run only with 1D ones
        L.Batch([P.orszag_tang(16), P.brio_wu(64)])


@pytest.mark.parametrize("tuned", [False, True])
def test_batch_mixed_2d_3d(restatement, tuned):
    """2D and 3D instances of uneven sizes in one ensemble (the face sweeps of z cover the 3D
    instances only), each bit-identical to its own oracle run, with the default linear block maps
    and after autotuning (tiles with a z extent leave the 2D instances' extra threads idle)."""
    probs = [P.orszag_tang(24, nym=18),
             P.kelvin_helmholtz(3, 8, mach=0.3, rmn=P.RMN_MLAU),
             P.kelvin_helmholtz(2, 20, nym=16, mach=0.2, rmn=P.RMN_MLAU),
             P.kelvin_helmholtz(3, 10, nym=8, nzm=12, mach=0.5, rmn=P.RMN_HLLD, seed=3),
             P.smooth_wave(3, 6, rmn=P.RMN_ROE),
             P.smooth_wave(2, 14, rmn=P.RMN_LHLLD)]
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        if tuned:
            b.autotune(1)
            for q, p in enumerate(probs):
                b.upload(q, p.state)
        info = b.run(max_steps=3, flg=1, stop_rule=0, cfl=0.4)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        want = restatement.run(p, 3, mode=R.MODE_RUN)
        assert info[q][2] == want["dt"], p.name
        assert_bitwise(outs[q], want["state"], f"{p.name} ({p.dim}D)")


def test_batch_mixed_reconstruction(restatement):
    """Instances with characteristic and primitive-variable face values in one ensemble."""
    probs = small_ensemble()[:4]
    for q, p in enumerate(probs):
        p.char_mode = q & 1
    with L.Batch(probs) as b:
        for q, p in enumerate(probs):
            b.upload(q, p.state)
        b.run(max_steps=3, flg=1, stop_rule=0, cfl=0.4)
        outs = [b.download(q, p.state.shape) for q, p in enumerate(probs)]
    for q, p in enumerate(probs):
        assert_bitwise(outs[q], restatement.run(p, 3, mode=R.MODE_RUN)["state"], f"{p.name} char_mode {q & 1}")

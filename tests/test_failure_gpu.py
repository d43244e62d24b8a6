"""Failure detection on the device without faulting it: the bounded mbarrier waits of the
TMA-staged reconstruction (qas_tma.cuh) are made to run out by the test hook
QAS_OPT_TEST_TMA_STALL (one plane per CTA never loaded, waits bounded at 100 us), and the
host must get QAS_ERR_TIMEOUT from the next synchronising call; the kernel returns by itself,
and a fresh context on the same device then runs bit-identical to the oracle.  (A planted
non-physical state is covered in test_parity_gpu.py: QAS_ERR_NONFINITE.)"""
import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("plane", [0, 3])
def test_tma_wait_runs_out_and_is_reported(restatement, plane):
    p = P.orszag_tang(64)
    with L.Context.from_problem(p) as ctx:
        ctx.set_option(L.QAS_OPT_LR_STAGING, 1)
        ctx.set_option(L.QAS_OPT_TEST_TMA_STALL, plane)
        ctx.upload(p.state)
        with pytest.raises(L.QasError) as e:
            ctx.run(max_steps=1, flg=1, stop_rule=0, cfl=p.cfl, use_graph=False)
        assert e.value.status == L.QAS_ERR_TIMEOUT
    want = restatement.run(p, 2, mode=R.MODE_RUN)["state"]
    with L.Context.from_problem(p) as ctx:  # the device is still usable
        ctx.set_option(L.QAS_OPT_LR_STAGING, 1)
        ctx.upload(p.state)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl, use_graph=False)
        got = ctx.download(p.state.shape)
    assert_bitwise(got, want, "after a timed-out context")


def test_tma_stall_hook_off_restores_the_normal_path(restatement):
    p = P.kelvin_helmholtz(3, 16, mach=0.3)
    want = restatement.run(p, 2, mode=R.MODE_RUN)["state"]
    with L.Context.from_problem(p) as ctx:
        ctx.set_option(L.QAS_OPT_LR_STAGING, 1)
        ctx.set_option(L.QAS_OPT_TEST_TMA_STALL, 1)
        ctx.set_option(L.QAS_OPT_TEST_TMA_STALL, -1)
        ctx.upload(p.state)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
        got = ctx.download(p.state.shape)
    assert_bitwise(got, want, "stall hook switched off")


"""The largest grid the GPU tests run: the 3D Kelvin-Helmholtz step (MLAU, WCNS4, CUCT, RK3) at
512^3 (520^3 padded: 140.6 M cells, 77 FP64 arrays = 86.6 GB of device memory), twice the
benchmark's extent per axis and beyond what the CPU oracle finishes in a test, checked through
size-independent properties:

* shift equivariance, bit for bit: the problem is periodic in x and z, every cell runs the same
  arithmetic on its own neighbourhood and the step's only reduction (setdt's maximum) is exact,
  so advancing the state shifted by (sx, sz) cells must give the shifted result exactly --
  which also exercises every 64-bit index and launch extent at this size;
* the discrete div B stays at round-off; every value stays finite."""
import numpy as np
import pytest
import torch

from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P
from tests.cases import assert_bitwise

pytestmark = pytest.mark.gpu

N = 512
GH = 4


def _room(n):
    dev = 77 * 8 * (n + 2 * GH) ** 3
    free, _ = torch.cuda.mem_get_info()
    try:
        import psutil
        host = psutil.virtual_memory().available
    except ImportError:
        host = float("inf")
    return free >= 1.05 * dev and host >= 48e9


def _shifted(u, sx, sz, out):
    """out = u shifted by sx cells along x and sz along z, ghosts included (periodic axes)."""
    nx, nz = u.shape[3], u.shape[1]
    ix = (np.arange(nx) - GH - sx) % (nx - 2 * GH) + GH
    iz = (np.arange(nz) - GH - sz) % (nz - 2 * GH) + GH
    for m in range(8):
        out[m] = u[m][iz][:, :, ix]


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")
def test_kh3d_512_shift_equivariance_and_divb():
    if not _room(N):
        pytest.skip("needs ~91 GB of free device memory and 48 GB of host memory")
    p = P.kelvin_helmholtz(3, N)
    shape = p.state.shape
    sx, sz = 37, 11
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
        a = ctx.download(shape)
        d_a = ctx.max_divb()
        u = p.state.reshape(shape)
        s = np.empty_like(u)
        _shifted(u, sx, sz, s)
        del u
        p.state = None
        ctx.run_reset()
        ctx.upload(s)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=p.cfl)
        ctx.download_into(s.reshape(-1))
        d_b = ctx.max_divb()
    assert np.isfinite(a).all()
    want = np.empty_like(a)
    _shifted(a, sx, sz, want)
    del a
    assert_bitwise(s, want, "KH 512^3 after 2 steps, shifted start vs shifted result")
    assert d_a < 1e-10 and d_b == d_a, (d_a, d_b)

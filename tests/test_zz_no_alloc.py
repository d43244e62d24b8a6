"""qas_max_divb_noalloc: max |div B| of a caller-owned device state with no device
allocation inside the call, for callers whose device memory belongs to an arena or
caching allocator under a fixed budget.  Checked against the context entry point
qas_max_divb on the same state (same per-cell expression, so the maxima agree to the
test tolerance -- in fact exactly), on two calls in a row, and the device's free memory
is the same before and after a call.  Kept in its own file, named to be collected last,
so it also runs after every other GPU test in the same process."""
import numpy as np
import pytest
import torch

from qasmhd_b200 import lib as L
from qasmhd_b200.problems import orszag_tang, smooth_wave

pytestmark = pytest.mark.gpu

RTOL = 1e-14


def _grid(p):
    return L.Grid(p.dim, p.nxm, p.nym, p.nzm, p.dx, p.dy if p.dim >= 2 else 0.0, p.dz if p.dim >= 3 else 0.0, p.gam)


def _cases():
    ot = orszag_tang(64)
    wave = smooth_wave(3, 16)
    rough = smooth_wave(2, 40)
    st = rough.state.copy()
    st[4:6] += 1e-3 * np.random.default_rng(5).standard_normal(st[4:6].shape)  # div B far from round-off
    rough.state = st
    return [("ot2d_steps", ot, 6), ("wave3d", wave, 2), ("rough2d", rough, 0)]


@pytest.mark.parametrize("name,prob,nsteps", _cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_matches_context_entry_point_twice(name, prob, nsteps):
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        if nsteps:
            ctx.run(max_steps=nsteps, flg=1, stop_rule=0, cfl=prob.cfl)
        ref = ctx.max_divb()
        state = ctx.download()
        nd = ctx.nd
    d = torch.from_numpy(np.ascontiguousarray(state.reshape(8, nd))).cuda()  # the caller's own buffer
    stream = torch.cuda.current_stream().cuda_stream
    g = _grid(prob)
    first = L.max_divb_noalloc(g, prob.odr, d.data_ptr(), nd, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    second = L.max_divb_noalloc(g, prob.odr, d.data_ptr(), nd, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)  # the second call allocated no device memory
    assert ref > 0.0
    assert abs(first - ref) <= RTOL * ref, (first, ref)
    assert abs(second - ref) <= RTOL * ref, (second, ref)


def test_padded_field_stride():
    prob = orszag_tang(32)
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        ref = ctx.max_divb()
        nd = ctx.nd
    stride = nd + 37
    buf = torch.zeros(8 * stride, dtype=torch.float64, device="cuda")
    for m in range(8):
        buf[m * stride:m * stride + nd] = torch.from_numpy(prob.state.reshape(8, nd)[m]).cuda()
    got = L.max_divb_noalloc(_grid(prob), prob.odr, buf.data_ptr(), stride, torch.cuda.current_stream().cuda_stream)
    assert abs(got - ref) <= RTOL * max(ref, 1e-300)


def test_oversize_grid_rejected():
    g = L.Grid(3, 8, 300, 300, 0.1, 0.1, 0.1, 5.0 / 3.0)  # 90000 interior rows > QAS_NOALLOC_MAX_ROWS
    nd = (8 + 8) * (300 + 8) * (300 + 8)
    tiny = torch.zeros(1, dtype=torch.float64, device="cuda")  # never read: the size check comes first
    with pytest.raises(L.QasError) as e:
        L.max_divb_noalloc(g, 4, tiny.data_ptr(), nd, torch.cuda.current_stream().cuda_stream)
    assert e.value.status == L.QAS_ERR_UNSUPPORTED
    assert "static scratch" in L.load().qas_last_cuda_error().decode()

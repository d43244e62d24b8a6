"""The reference's on-disk formats, written and read by the CUDA library.

Byte-for-byte comparison with the files the reference's own writers produce on the
same state:
* dout_ -- MHD1D::dout_ (1D/SERIAL/shock/mhd1d_class.cpp:57-95), MHD2D::dout_
  (2D/SERIAL/OTvortex/mhd2d_class.cpp:63-114), MHD3D::dout_ on one rank
  (3D/MPI/KHI/mhd3d_class.cpp:78-145): header files at n == 0, t.dat appended at
  later outputs, outdat_<cnt> in double (1D/2D) or float (3D);
* bkup_save / bkup_load (common/common_func.c:280-344), both directions: the library
  loads the reference's restart files and the reference loads the library's.
The reference side runs the reference binaries built by oracle/Makefile.
"""
import os

import numpy as np
import pytest

from oracle import refcase as R
from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not all(R.reference_available(d, 1) for d in (1, 2, 3)),
                                 reason="reference oracle binaries not built")]

OUTPUTS = [  # (n, cnt, tim, dt, trec): a header output, then a later one
    (0, 0, 0.25, 0.01, 0.1),
    (3, 1, 0.5, 0.0125, 0.2),
]


def _states(p):
    rng = np.random.default_rng(7 + p.dim)
    a = p.state.copy()
    b = a * (1.0 + 1e-3 * rng.standard_normal(a.shape))
    return a, b


def _files(d):
    return sorted(f for f in os.listdir(d) if f != "loaded.txt")


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_dout_and_bkup_match_reference(tmp_path, dim):
    p = P.smooth_wave(dim, 12 if dim < 3 else 8)
    states = _states(p)
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    with L.Context.from_problem(p) as ctx:
        for st, (n, cnt, tim, dt, trec) in zip(states, OUTPUTS):
            ctx.upload(st)
            ctx.dout(str(ours), n, cnt, tim, coords=p.coords()[:dim] if n == 0 else None)
            ctx.dout_wait()
            ctx.bkup_save(str(ours), n, cnt, tim, dt, trec)
            R.reference_io(p, str(ref), st, n=n, cnt=cnt, tim=tim, dt=dt, trec=trec)
    assert _files(ours) == _files(ref)
    for f in _files(ref):
        assert (ours / f).read_bytes() == (ref / f).read_bytes(), f


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_bkup_load_both_ways(tmp_path, dim):
    p = P.smooth_wave(dim, 12 if dim < 3 else 8)
    _, st = _states(p)
    n, cnt, tim, dt, trec = OUTPUTS[1]
    a, b = tmp_path / "ref_wrote", tmp_path / "lib_wrote"
    a.mkdir()
    b.mkdir()
    R.reference_io(p, str(a), st, n=n, cnt=cnt, tim=tim, dt=dt, trec=trec)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(np.zeros_like(st))
        got = ctx.bkup_load(str(a))
        assert got == (n, cnt, tim, dt, trec)
        back = ctx.download(st.shape)
        assert np.array_equal(back, st)
        ctx.bkup_save(str(b), n, cnt, tim, dt, trec)
    loaded, counters = R.reference_io(p, str(b), np.zeros_like(st), load=True)
    assert counters == (n, cnt, tim, dt, trec)
    assert np.array_equal(loaded.reshape(st.shape), st)


def test_bkup_load_without_stamp_is_a_no_op(tmp_path):
    p = P.smooth_wave(2, 12)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        assert ctx.bkup_load(str(tmp_path)) is None
        assert np.array_equal(ctx.download(p.state.shape), p.state)


def test_dout_snapshots_in_stream_order(tmp_path):
    """The writer runs while the caller keeps stepping; the file holds the state at the call."""
    p = P.orszag_tang(64)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        ctx.dout(str(tmp_path), 0, 0, 0.0, coords=p.coords()[:2])
        ctx.bound()
        for _ in range(3):
            ctx.step(1e-3)
        ctx.dout_wait()
        after = ctx.download(p.state.shape)
    raw = np.fromfile(tmp_path / "outdat_00000.dat", dtype=np.float64).reshape(p.state.shape)
    assert np.array_equal(raw, p.state)
    assert not np.array_equal(after, p.state)


def test_dout_errors_are_reported(tmp_path):
    p = P.smooth_wave(2, 12)
    with L.Context.from_problem(p) as ctx:
        ctx.upload(p.state)
        with pytest.raises(L.QasError):
            ctx.dout(str(tmp_path), 0, 0, 0.0, coords=None)  # header output needs the coordinates
        ctx.dout(str(tmp_path / "missing"), 1, 0, 0.0)
        with pytest.raises(L.QasError):
            ctx.dout_wait()
        ctx.dout(str(tmp_path), 1, 1, 0.0)  # the context stays usable
        ctx.dout_wait()
    assert (tmp_path / "outdat_00001.dat").stat().st_size == 8 * p.nd * 8

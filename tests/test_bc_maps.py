"""The device ghost fill is a gather over per-axis (source, factor) maps built
on the host (qas_bc_map).  Check on CPU that composing the maps reproduces the
reference's ordered fill passes exactly (the oracle restates bc1d/bc2d and the
single-rank 3D MPI order), for random boundary-flag mixes."""
import numpy as np
import pytest

from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P


def gather_fill(prob, state, group=0):
    nz, ny, nx = prob.nz, prob.ny, prob.nx
    out = state.copy()
    for m in range(8):
        sx, fx = L.bc_map(prob, group, m, 0)
        sy, fy = L.bc_map(prob, group, m, 1) if prob.dim >= 2 else (np.zeros(1, np.int32), np.ones(1))
        sz, fz = L.bc_map(prob, group, m, 2) if prob.dim >= 3 else (np.zeros(1, np.int32), np.ones(1))
        f = state[m]
        K, J, I = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        src = f[sz[K], sy[J], sx[I]]
        fac = (fx[I] * fy[J]) * fz[K]
        written = (sx[I] != I) | (sy[J] != J) | (sz[K] != K)
        out[m] = np.where(written, fac * src, f)
    return out


def random_flags(rng, dim):
    def flags():
        f = [int(rng.choice([-2, -1, 1, 2])) for _ in range(8)]
        f[0] = int(rng.choice([1, 2]))
        f[7] = int(rng.choice([1, 2]))
        return tuple(f)
    return tuple(flags() if a < dim and rng.random() < 0.6 else (0,) * 8 for a in range(3))


@pytest.mark.parametrize("seed", range(12))
def test_gather_equals_ordered_passes(restatement, seed):
    rng = np.random.default_rng(seed)
    dim = 1 + seed % 3
    p = P.smooth_wave(dim, 9 if dim < 3 else 5, dn=random_flags(rng, dim))
    st = rng.normal(size=p.state.shape)
    st[:, ...] += 2.0
    ref = st.copy()
    import ctypes
    g = restatement.grid(p)
    restatement.lib.qo_bound(ctypes.byref(g), ref.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    got = gather_fill(p, st)
    assert np.array_equal(got, ref)


def test_unset_ghosts_rejected():
    p = P.smooth_wave(3, 5, dn=((0,) * 8, (1, 1, 1, 1, 1, 1, 1, 0), (0,) * 8))
    with pytest.raises(L.QasError):
        L.bc_map(p, 0, 7, 1)   # ro's y flag is physical, en's is periodic: ghosts left unset in 3D
    p2 = P.smooth_wave(2, 8, dn=((3,) * 8, (0,) * 8, (0,) * 8))
    with pytest.raises(L.QasError):
        L.bc_map(p2, 0, 0, 0)


def test_staggered_periodic_face():
    p = P.smooth_wave(2, 8)
    sx, fx = L.bc_map(p, 0, 4, 0)   # bx, x axis, periodic: face nx-4 mirrors face 4
    assert sx[p.nx - 4] == 4 and fx[p.nx - 4] == 1.0
    p = P.smooth_wave(2, 8, dn=((2,) * 8, (0,) * 8, (0,) * 8))
    sx, fx = L.bc_map(p, 0, 4, 0)   # open: the boundary face nx-4 is computed, not filled
    assert sx[p.nx - 4] == p.nx - 4
    assert list(sx[p.nx - 3:]) == [p.nx - 4] * 3

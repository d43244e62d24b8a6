"""Host-side problem setup (initial states of the benchmark configurations)."""
import math

import numpy as np

from qasmhd_b200 import problems as P


def divb_cells(p):
    st = p.state
    bx, by = st[4, 0], st[5, 0]
    d = lambda f, ax: np.take(f, range(1, f.shape[ax] - 2), axis=ax)  # noqa: E731
    s = slice(4, -4)
    dbx = (27.0 * (np.roll(bx, -1, 1) - bx) - (np.roll(bx, -2, 1) - np.roll(bx, 1, 1))) / 24.0 / p.dx
    dby = (27.0 * (np.roll(by, -1, 0) - by) - (np.roll(by, -2, 0) - np.roll(by, 1, 0))) / 24.0 / p.dy
    return (dbx + dby)[s, s]


def test_orszag_tang_divergence_free():
    p = P.orszag_tang(64)
    assert p.state.shape == (8, 1, 72, 72)
    assert np.abs(divb_cells(p)).max() < 1e-12


def test_orszag_tang_values():
    p = P.orszag_tang(32)
    ro = p.state[0, 0]
    assert np.allclose(ro, 25.0 / (36.0 * math.pi))


def test_kelvin_helmholtz_seeded():
    a = P.kelvin_helmholtz(3, 8, seed=5)
    b = P.kelvin_helmholtz(3, 8, seed=5)
    c = P.kelvin_helmholtz(3, 8, seed=6)
    assert np.array_equal(a.state, b.state)
    assert not np.array_equal(a.state, c.state)
    assert a.state.shape == (8, 16, 16, 16)
    # beta = 2 p / B^2 = 100 for the guide field
    bz = a.state[6, 8, 8, 8]
    assert abs(2 * (1 / a.gam) / bz ** 2 - 100.0) < 1e-9


def test_brio_wu_states():
    p = P.brio_wu(64)
    ro = p.state[0, 0, 0]
    assert ro[4] == 1.0 and ro[-5] == 0.125
    assert p.flg == 0 and p.dnx == (2,) * 8


def test_energy_and_pack_match_reference_mhd_energy():
    """The initial-state builders' prim -> cons (cnsvt: mmntm + mhd_energy with the cell-centre
    field, common/mhd_class.hpp:67-79, common/mhd_func.c:18-28) against the reference's own
    mhd_energy on the known-answer inputs of tests/golden/kat_energy.npz, bit for bit."""
    import os

    from tests.golden import make_golden as G
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "kat_energy.npz"))
    inp = G.kat_inputs("energy")
    assert str(gold["input_sha"]) == G.sha(inp)
    ro, vx, vy, vz, bx, by, bz, pr, gam = inp.T
    want = gold["f32"][:, 0]
    got = np.array([P._energy(*row) for row in inp])  # scalar path, as the builders call it per cell
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    vec = P._energy(ro, vx, vy, vz, bx, by, bz, pr, gam)  # vectorised path
    assert np.array_equal(vec.view(np.uint64), want.view(np.uint64))
    # _pack: momenta ro*v, staggered B passed through, energy from the cell-centre field
    st = P._pack(ro, vx, vy, vz, bx * 2, by * 2, bz * 2, pr, bx, by, bz, gam[0])
    same_gam = gam == gam[0]
    assert np.array_equal(st[7][same_gam].view(np.uint64), want[same_gam].view(np.uint64))
    assert np.array_equal(st[1], ro * vx) and np.array_equal(st[3], ro * vz)
    assert np.array_equal(st[4], bx * 2)

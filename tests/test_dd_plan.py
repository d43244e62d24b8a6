"""Host-side logic of the slab decomposition (qas_dd_plan; no GPU needed).

For every slab and every ghost plane of the split axis, the plan must copy exactly the
planes whose single-domain value comes from another slab: the neighbour's interior plane
across an internal boundary, and the far end of the axis through the periodic fill
(the global ghost map of bound(), qas_bc_map, for every field).  Ghost planes on a physical
boundary are left to the slab's own fill, which then must only read its own planes.
"""
import pytest

from qasmhd_b200 import lib as L
from qasmhd_b200 import problems as P

GH = 4


def _problems():
    yield "ot2d_64_periodic", P.orszag_tang(64)
    yield "kh2d_64x40_open", P.kelvin_helmholtz(2, 64, nym=40, mach=0.3)
    yield "kh3d_16x16x40_periodic", P.kelvin_helmholtz(3, 16, nzm=40, mach=0.3)
    phys = ((0,) * 8, (0,) * 8, (2, 1, 1, -1, 1, 1, -1, 2))
    yield "wave3d_physical_z", P.smooth_wave(3, 32, dn=phys)


@pytest.mark.parametrize("name,prob", list(_problems()), ids=[n for n, _ in _problems()])
@pytest.mark.parametrize("nparts", [1, 2, 3, 4])
def test_plan_matches_global_ghost_maps(name, prob, nparts):
    axis = prob.dim - 1
    nz = (prob.nxm, prob.nym, prob.nzm)[axis]
    if nz // nparts < 2 * GH:
        with pytest.raises(L.QasError):
            L.dd_plan(prob, nparts)
        return
    lo, copies = L.dd_plan(prob, nparts)
    assert lo[0] == 0 and lo[-1] == nz and all(lo[p + 1] - lo[p] >= 2 * GH for p in range(nparts))
    got = {}
    for part, src_part, src_plane, dst_plane, nplanes in copies:
        assert nplanes == GH and src_part != part
        for t in range(nplanes):
            got[(part, dst_plane + t)] = (src_part, src_plane + t)
    dn = (prob.dnx, prob.dny, prob.dnz)[axis]
    periodic = all(d == 0 for d in dn)
    maps = [L.bc_map(prob, 0, f, axis) for f in range(8)]

    def owner(gi):  # slab holding global interior plane gi
        return max(p for p in range(nparts) if lo[p] <= gi)

    want = {}
    for p in range(nparts):
        nl = lo[p + 1] - lo[p]
        for k in list(range(GH)) + list(range(nl + GH, nl + 2 * GH)):
            G = lo[p] + k  # global padded plane of this ghost plane
            if GH <= G < nz + GH:
                q = owner(G - GH)
                want[(p, k)] = (q, G - lo[q])
                continue
            srcs = {int(m[0][G]) for m in maps}
            if periodic:
                assert len(srcs) == 1 and all(m[1][G] == 1.0 for m in maps)
                s = srcs.pop()
                q = owner(s - GH)
                if q != p:
                    want[(p, k)] = (q, s - lo[q])
            else:
                for s in srcs:  # a physical fill reads this slab's own planes
                    assert s == G or owner(s - GH) == p, (p, k, s)
    assert got == want


def test_plan_rejects_mixed_flags_and_thin_slabs():
    mixed = ((0,) * 8, (0,) * 8, (0, 0, 0, 0, 0, 0, 0, 2))
    with pytest.raises(L.QasError) as e:
        L.dd_plan(P.smooth_wave(3, 32, dn=mixed), 2)
    assert e.value.status == L.QAS_ERR_UNSUPPORTED
    with pytest.raises(L.QasError) as e:
        L.dd_plan(P.orszag_tang(24), 4)  # 6 planes per slab
    assert e.value.status == L.QAS_ERR_UNSUPPORTED
    with pytest.raises(L.QasError):
        L.dd_plan(P.brio_wu(64), 2)  # 1D has no decomposition

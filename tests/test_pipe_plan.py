"""The plan of qas_step_host's wave (qas_pipe_plan, host only): the library's own windows, seam,
issue lag and kernel ranges, checked on the CPU for many axis lengths and window counts.

Invariants:
* the copied planes of all items partition the axis, the updated planes partition
  [GH, n-GH] (the last face plane of the staggered field included), the ghost-filled interior
  planes partition [GH, n-GH); only the first item (the seam) holds the ghost planes;
* an item other than the seam reads the previous stage's state only on interior planes
  ([a-6, b+7) inside [GH, n-GH)), and every item whose planes it reads comes at most `lag`
  items later in the issue order;
* the kernel ranges cover what each kernel's stencil reads along the last axis, from launches
  of the same stage issued before it: within the item itself for the shared-stream ranges,
  within the lane (all earlier items of the stage) for the compute-once ranges.  The seam's
  ghost planes gather from the far end of a periodic axis, so its shock detector there reads
  primitives at the other end."""
import pytest

from qasmhd_b200 import lib as L

GH = 4
SIZES = [21, 24, 40, 72, 104, 136, 168, 200, 264, 520, 1032, 2056]
WINDOWS = [0, 1, 2, 3, 5, 8, 16, 24, 32, 64]


def _ranges(it, name):
    return [r for s, r in enumerate(it[name]) if s < it["nseg"] and r[1] > r[0]]


def _planes(rs):
    out = []
    for lo, hi in rs:
        out.extend(range(lo, hi))
    return out


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("windows", WINDOWS)
def test_partitions_and_lag(n, windows):
    items, lag = L.pipe_plan(n, windows)
    assert lag >= 1
    for name, lo, hi in (("seg", 0, n), ("upd", GH, n - GH + 1), ("bnd", GH, n - GH)):
        got = sorted(_planes([r for it in items for r in _ranges(it, name)]))
        assert got == list(range(lo, hi)), (n, windows, name)
    assert items[0]["ends"] and not any(it["ends"] for it in items[1:])
    owner = {}
    for q, it in enumerate(items):
        for p in _planes(_ranges(it, "seg")):
            owner[p] = q
    for q, it in enumerate(items):
        for lo, hi in _ranges(it, "upd"):
            reads = range(max(0, lo - 6), min(n, hi + 7))
            if q > 0:
                assert reads.start >= GH and reads.stop <= n - GH, (n, windows, q)
            assert all(owner[p] <= q + lag for p in reads), (n, windows, q)


@pytest.mark.parametrize("own_lanes", [True, False])
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("windows", [0, 2, 5, 16, 32, 64])
def test_kernel_ranges_cover_their_reads(n, windows, own_lanes):
    items, _ = L.pipe_plan(n, windows, own_lanes)
    valid = {k: set() for k in ("prim", "dv", "fin", "lax", "fax", "emf")}

    def need(kind, lo, hi, who):
        miss = [p for p in range(max(0, lo), min(n, hi)) if p not in valid[kind]]
        assert not miss, (n, windows, own_lanes, who, kind, miss[:4])

    def launch(kind, rs, needs, who):
        # every read of a launch is covered by earlier launches; then its planes are written
        for lo, hi in rs:
            for k, before, after in needs:
                need(k, lo - before, hi + after, who)
        for lo, hi in rs:
            valid[kind].update(range(lo, hi))

    for q, it in enumerate(items):
        if not own_lanes:  # each item on its own: nothing carried over from earlier items
            for v in valid.values():
                v.clear()
        launch("prim", _ranges(it, "prim"), [], (q, "prim"))
        dv = _ranges(it, "dv")
        if it["ends"]:  # ghost planes of a periodic axis gather from the far end
            for lo, hi in dv:
                if lo < GH:
                    need("prim", n - 2 * GH - 1, n - GH + 1, (q, "dv ghost low"))
                if hi > n - GH:
                    need("prim", GH - 1, 2 * GH + 1, (q, "dv ghost high"))
        launch("dv", dv, [("prim", 1, 1)], (q, "dv"))
        launch("fin", _ranges(it, "fin"), [("prim", 0, 0), ("dv", 0, 0)], (q, "fin"))
        valid["lax"].clear()  # the face-state arrays are shared by the axes
        launch("lax", _ranges(it, "lax"), [("prim", 2, 2)], (q, "lax"))
        launch("fax", _ranges(it, "fax"), [("lax", 1, 0), ("dv", 1, 0), ("prim", 1, 0)], (q, "fax"))
        launch("emf", _ranges(it, "emf"), [("fin", 3, 2), ("fax", 0, 0), ("prim", 1, 0)], (q, "emf"))
        for lo, hi in _ranges(it, "upd"):
            need("fax", lo - 1, hi + 2, (q, "update"))
            need("fin", lo, hi, (q, "update"))
            need("emf", lo - 1, hi + 2, (q, "update"))


def test_compute_once_ranges_do_each_plane_once():
    """With a lane per stage the primitives and in-plane fluxes of every plane are computed by one
    item only (the two fronts of the last pair may meet inside one launch)."""
    for n in (264, 1032):
        items, _ = L.pipe_plan(n, 32, True)
        for name in ("prim", "fin"):
            planes = _planes([r for it in items for r in _ranges(it, name)])
            assert len(planes) - len(set(planes)) <= 2 * 5 + 1, (n, name)
            assert set(planes) == set(range(n)), (n, name)


def test_invalid_arguments():
    with pytest.raises(L.QasError):
        L.pipe_plan(2 * GH, 8)
    with pytest.raises(L.QasError):
        L.pipe_plan(264, 65)


def test_record_size_matches_the_header():
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    txt = open(os.path.join(root, "include", "qas.h")).read()
    assert int(re.search(r"#define QAS_PIPE_ITEM_INTS (\d+)", txt)[1]) == L.PIPE_ITEM_INTS == 2 + 2 * 2 * len(
        L.PIPE_RANGE_NAMES)

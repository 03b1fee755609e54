"""Systems whose panels outgrow one CTA: the grid-wide panel factorisation.

The plain path hands a 32-column panel taller than 400 rows to the
cooperative many-CTA kernel; the mixed path does so above 800 rows.  The
exact path must stay bit-identical to the oracle's GEPP (linear.rs:1321-1383)
there too, including with several tall units of different heights in one
launch; the mixed path must keep its accuracy gate.
"""
import numpy as np
import pytest

import bench
from oracle import oracle as O
from test_gpu_parity import _check_unit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    return nec_accel


def _mesh(cells):
    wl, src, f = bench.mesh_workload(cells)
    return O.wires_array(wl), O.sources_array(src), f


def test_grid_panel_bit_exact_given_z(acc):
    """Mesh of 10x10 cells: S = 660, the first nine panels go grid-wide."""
    w, s, f = _mesh(10)
    segs = O.build_geometry(w)
    rhs, cosv = O.hallen_rhs(segs, f, s)
    z = O.assemble_z(segs, f, 1)
    m = O.merge_collinear(segs)
    ja, jb, js = O.cli_junctions(segs, m)
    assert len(segs) + len(m) > 400
    x0, p0 = O.solve_hallen(z, rhs, cosv, m, ja, jb, js, nthreads=8)
    x1, p1 = acc.solve_hallen(z, rhs, cosv, m, list(zip(ja, jb, js)), return_pivots=True)
    assert np.array_equal(p0, p1)
    assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64))


def test_grid_panel_several_units(acc):
    """Three tall units of different heights and one short one in one batch:
    the grid launch spans units whose panels end at different steps."""
    cases = [_mesh(10), _mesh(9), _mesh(8), _mesh(3)]
    ants = [acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], 1, (5, 4, 0.0, 0.0, 20.0, 90.0))
            for w, s, f in cases]
    batch = acc.HallenBatch(ants)
    res = batch.solve()
    assert np.all(res.status == 0)
    for u, (w, s, f) in enumerate(cases):
        _check_unit(acc, batch, res, u, w, s, 1, f, O.rp_card_points(5, 4, 0, 0, 20, 90))


def test_grid_panel_and_gmres_mixed(acc):
    """Mesh of 18x18 cells (S = 2052) in the mixed form, two copies in one
    batch: the first panels run grid-wide in FP32 and both solves are
    refined by the grid-wide GMRES (one cooperative launch each).  The
    result meets the 1e-6 gate against the plain GPU path (itself pinned to
    the oracle above)."""
    w, s, f = _mesh(18)
    ant = acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], 1, None)
    plain = acc.HallenBatch([ant])
    rp = plain.solve()
    mixed = acc.HallenBatch([ant, ant], precision=acc.PRECISION_MIXED)
    rm = mixed.solve()
    it, rs = mixed.refinement_stats()
    assert np.all(it > 0) and np.all(rs <= 1e-9)
    assert np.all(rm.status == 0) and np.all(rp.status == 0)
    zp = complex(*rp.feeds[0][0, 5:7])
    for u in range(2):
        zm = complex(*rm.feeds[u][0, 5:7])
        assert abs(zm - zp) / abs(zp) <= 1e-6
        xm, _ = mixed.read_unit(u)
        xp, _ = plain.read_unit(0)
        assert np.linalg.norm(xm - xp) / np.linalg.norm(xp) <= 1e-7


def test_mesh_20x20_plain_end_to_end_bit_exact(acc):
    """Mesh of 20x20 cells over PEC ground (N = 1680 segments, W = 840
    wires, S = 2520, 2,398 pairwise junction rows): the plain form end to
    end -- fill with image terms, Gram with the constraint rows, grid-wide
    panels, back substitution, feedpoint -- against the oracle (its
    row-parallel GEPP is the reference's elimination bit for bit): pivots,
    currents and Zin identical."""
    w, s, f = _mesh(20)
    ant = acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], 1, None)
    batch = acc.HallenBatch([ant])
    res = batch.solve()
    assert res.status[0] == 0
    assert batch.units[0]["s"] == 2520
    p = O.Problem(w, s, f, ground=1)
    O.solve_problems([p], 8)
    assert p.status == 0
    _check_unit(acc, batch, res, 0, w, s, 1, f, None, bit_exact=True, solved=p)
    batch.close()

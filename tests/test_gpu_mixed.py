"""The chosen (mixed-precision) form against the FP64 oracle.

Its gate is the metric's: feedpoint |dZin|/|Zin| <= 1e-6 against the FP64
oracle.  The errors of the currents (normwise) and of the gain grid are
stated here as the bars the refinement actually meets: 1e-7 normwise on
currents and 1e-5 dB on gains (the far field itself runs in FP64 on the
refined currents).
"""
import numpy as np
import pytest

from _corpus import deck_arrays, load_cases
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = load_cases()
ZIN_GATE = 1e-6
CUR_BAR = 1e-7
GAIN_BAR_DB = 1e-5


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _check(res, batch, u, wires, sources, ground, freq, pts, errs):
    p = O.Problem(wires, sources, freq, ground=ground, points=pts)
    O.solve_problem(p)
    assert res.status[u] == 0
    for row, zr in zip(res.feeds[u], p.zin):
        dz = abs(complex(row[5], row[6]) - zr) / abs(zr)
        errs["zin"] = max(errs.get("zin", 0.0), dz)
        assert dz <= ZIN_GATE, (dz, zr)
    peak = np.abs(p.currents).max()
    if peak > 0:
        dc = np.abs(res.currents[u] - p.currents).max() / peak
        errs["cur"] = max(errs.get("cur", 0.0), dc)
        assert dc <= CUR_BAR
    if pts is not None:
        g = res.pattern[u][:, 0]
        live = p.pattern[:, 0] > -999
        dg = np.abs(g[live] - p.pattern[live, 0]).max(initial=0.0)
        errs["gain"] = max(errs.get("gain", 0.0), dg)
        assert dg <= GAIN_BAR_DB


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_corpus_cases(acc, name):
    deck = CASES[name]["deck"]
    wires, sources, pts = deck_arrays(deck)
    rp = tuple(deck["rp"]) if deck.get("rp") else None
    ant = acc.Antenna(wires.view(acc.WIRE_DTYPE), sources.view(acc.SOURCE_DTYPE), deck["freqs"], deck["ground"], rp)
    batch = acc.HallenBatch([ant], precision=acc.PRECISION_MIXED)
    res = batch.solve()
    errs = {}
    for u, f in enumerate(deck["freqs"]):
        _check(res, batch, u, wires, sources, deck["ground"], f, pts, errs)
    it, rs = batch.refinement_stats()
    assert np.all(it > 0) and np.all(it <= 96)


def test_mixed_sweep_matches_plain_gpu_and_oracle(acc):
    """All 201 units of the 5-wire sweep: mixed vs plain GPU everywhere,
    and vs the oracle on a few units with the full 91 x 361 grid."""
    rng = np.random.default_rng(11)
    lam = 299792458.0 / 14.2e6
    x, wl = 0.0, []
    for t in range(5):
        L = rng.uniform(0.9, 1.1) * lam / 2
        wl.append((t + 1, 51, (x, 0.0, -L / 2), (x, 0.0, L / 2), 1e-3))
        x += rng.uniform(0.15, 0.25) * lam
    wires = O.wires_array(wl)
    sources = O.sources_array([(2, 26, 1.0)])
    freqs = [13.0e6 + i * 2.5e6 / 200 for i in range(201)]
    rp = (91, 361, 0.0, 0.0, 1.0, 1.0)
    ant = acc.Antenna(wires.view(acc.WIRE_DTYPE), sources.view(acc.SOURCE_DTYPE), freqs, 0, rp)
    mixed = acc.HallenBatch([ant], precision=acc.PRECISION_MIXED).solve()
    plain = acc.HallenBatch([ant]).solve()
    dz = [abs(complex(*m[0, 5:7]) - complex(*p[0, 5:7])) / abs(complex(*p[0, 5:7]))
          for m, p in zip(mixed.feeds, plain.feeds)]
    assert max(dz) <= ZIN_GATE, max(dz)
    pts = O.rp_card_points(*rp)
    errs = {}
    for u in (0, 100, 200):
        _check(mixed, None, u, wires, sources, 0, freqs[u], pts, errs)


def test_mixed_uneven_batch_with_ground_and_junctions(acc):
    rng = np.random.default_rng(21)
    ants, refs = [], []
    for a in range(8):
        nw = int(rng.integers(1, 5))
        wl = []
        for t in range(nw):
            p0 = rng.uniform(-5, 5, 3)
            p0[2] = rng.uniform(1, 6)
            p1 = p0 + rng.uniform(-4, 4, 3)
            p1[2] = max(p1[2], 0.5)
            wl.append((t + 1, int(rng.integers(5, 51)) * 2 + 1, tuple(p0), tuple(p1), 10 ** rng.uniform(-3.3, -2.3)))
        if a == 3:  # a T-junction antenna
            wl = [(1, 9, (0, 0, 1.0), (0, 0, 3.0), 1e-3), (2, 7, (0, 0, 3.0), (1.5, 0, 3.0), 1e-3),
                  (3, 7, (0, 0, 3.0), (-1.5, 0, 3.0), 1e-3)]
        w = O.wires_array(wl)
        s = O.sources_array([(1, (wl[0][1] + 1) // 2, 1.0)])
        ground = int(a % 2)
        f = float(10 ** rng.uniform(np.log10(3e6), np.log10(30e6)))
        ants.append(acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], ground,
                                (7, 5, 0.0, 0.0, 15.0, 72.0)))
        refs.append((w, s, ground, f))
    batch = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    res = batch.solve()
    errs = {}
    for u, (w, s, ground, f) in enumerate(refs):
        _check(res, batch, u, w, s, ground, f, O.rp_card_points(7, 5, 0, 0, 15, 72), errs)


def test_mixed_resident_entry_point(acc):
    deck = CASES["yagi-5elm-51seg"]["deck"]
    wires, sources, _ = deck_arrays(deck)
    segs = O.build_geometry(wires)
    f = deck["freqs"][0]
    rhs, cosv = O.hallen_rhs(segs, f, sources)
    m = O.merge_collinear(segs)
    x = acc.solve_hallen_gpu_resident(acc.zsegments_from(segs), rhs, cosv, m, [], f,
                                      precision=acc.PRECISION_MIXED)
    x0, _ = O.solve_hallen(O.assemble_z(segs, f), rhs, cosv, m, [], [], [])
    assert np.abs(x - x0)[: len(segs)].max() / np.abs(x0[: len(segs)]).max() <= CUR_BAR


def test_mixed_uneven_random_antenna_batch_sample(acc):
    import bench

    wl = bench.uneven_workload(64, seed=7)
    ants = [acc.Antenna(acc.wires_array(w), acc.sources_array(s), [f], g, None) for w, s, g, f in wl]
    batch = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    res = batch.solve()
    errs = {}
    for u in range(0, 64, 7):
        w, s, g, f = wl[u]
        _check(res, batch, u, O.wires_array(w), O.sources_array(s), g, f, None, errs)
    it, rs = batch.refinement_stats()
    assert it.max() <= 96


def test_mixed_extra_right_hand_sides(acc):
    wl = [(1, 21, (0, 0, 1.0), (0, 0, 6.0), 1e-3), (2, 15, (1.2, 0, 1.0), (1.2, 0, 5.0), 1e-3)]
    srcs = [(1, 11, 1.0), (2, 8, 0.5 - 0.25j), (1, 3, 1.0), (2, 14, 1j)]
    w = O.wires_array(wl)
    b = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), O.sources_array(srcs).view(acc.SOURCE_DTYPE), [24e6],
                                     1, None, separate_sources=True)], precision=acc.PRECISION_MIXED)
    res = b.solve()
    errs = {}
    for r, src in enumerate(srcs):
        _check(res, b, r, w, O.sources_array([src]), 1, 24e6, None, errs)


def test_mixed_junctioned_mesh(acc):
    import bench

    wl, src, f = bench.mesh_workload(6)
    w, s = O.wires_array(wl), O.sources_array(src)
    b = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], 1, None)],
                        precision=acc.PRECISION_MIXED)
    res = b.solve()
    _check(res, b, 0, w, s, 1, f, None, {})

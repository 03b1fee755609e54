"""The degree-2 conductor-path form (solve_session.rs:1338-1378) on the
device: decks whose wires join into bent or reversed chains (a
start-to-start split dipole, an inverted V, a three-arm zig-zag, a chain
beside a straight parasite, over free space and GN 1) are solved with one
homogeneous column per path, I = 0 only at the chain's free ends and
cos / source terms along the signed arc length.

Plain FP64 form vs the CPU oracle: pivots bit-exact, Zin and currents
within 1e-9, gains within 1e-6 dB.  Mixed form: Zin within 1e-6.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

F = 14.2e6
RP = (19, 13, 0.0, 0.0, 10.0, 30.0)

DECKS = {
    "split_dipole": ([(1, 26, (0, 0, 0), (0, 0, 5.282), 0.001), (2, 26, (0, 0, 0), (0, 0, -5.282), 0.001)],
                     [(1, 1, 1.0)], 0),
    "split_dipole_fed_reversed_arm": ([(1, 26, (0, 0, 0), (0, 0, 5.282), 0.001),
                                       (2, 26, (0, 0, 0), (0, 0, -5.282), 0.001)], [(2, 1, 1.0)], 0),
    "inverted_v": ([(1, 26, (0, 0, 5.0), (4.46, 0, 2.42), 0.001), (2, 26, (0, 0, 5.0), (-4.46, 0, 2.42), 0.001)],
                   [(1, 1, 1.0)], 0),
    "inverted_v_gn1": ([(1, 25, (0, 0, 6.0), (4.46, 0, 3.42), 0.001), (2, 25, (0, 0, 6.0), (-4.46, 0, 3.42), 0.001)],
                       [(1, 1, 1.0 + 0.5j)], 1),
    "zigzag_three_arms": ([(1, 11, (0, 0, 0), (3, 0, 1), 0.001), (2, 13, (3, 0, 1), (1, 2, 4), 0.0015),
                           (3, 9, (-1, 1, 5), (1, 2, 4), 0.001)], [(2, 7, 1.0)], 0),
    "chain_beside_parasite": ([(1, 21, (0, 0, 0), (0, 0, 5.2), 0.001), (2, 21, (0, 0, 0), (0.5, 0, -5.1), 0.001),
                               (3, 41, (2.5, 0, -5.0), (2.5, 0, 5.0), 0.002)], [(1, 1, 1.0)], 0),
    # two cards on one tag: the path form adds both (the plain form keeps one per tag)
    "two_sources_one_path": ([(1, 15, (0, 0, 0), (0, 0, 5.0), 0.001), (2, 15, (0, 0, 0), (0, 3, -4.0), 0.001)],
                             [(1, 3, 1.0), (1, 9, 0.5j), (2, 4, -0.3)], 0),
}


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _oracle(wires, sources, ground, pts):
    p = O.Problem(O.wires_array(wires), O.sources_array(sources), F, ground=ground, points=pts)
    O.solve_problem(p)
    assert p.status == 0
    return p


def _antenna(acc, wires, sources, ground, separate=False):
    return acc.Antenna(acc.wires_array(wires), acc.sources_array(sources), [F], ground, RP,
                       separate_sources=separate)


def test_decks_take_the_path_form():
    for name, (wires, _, _) in DECKS.items():
        segs = O.build_geometry(O.wires_array(wires))
        paths = O.conductor_paths(segs)
        assert paths is not None and paths.nontrivial, name


@pytest.mark.parametrize("name", sorted(DECKS))
def test_plain_matches_oracle(acc, name):
    wires, sources, ground = DECKS[name]
    pts = O.rp_card_points(*RP)
    p = _oracle(wires, sources, ground, pts)
    b = acc.HallenBatch([_antenna(acc, wires, sources, ground)], precision=acc.PRECISION_FP64)
    res = b.solve()
    assert res.status[0] == 0
    segs = O.build_geometry(O.wires_array(wires))
    n_paths = len(O.conductor_paths(segs))
    assert b.units[0]["s"] == len(segs) + n_paths
    _, piv = b.read_unit(0)
    assert np.array_equal(piv, p.pivots[: len(piv)])
    for row, zr in zip(res.feeds[0], p.zin):
        assert abs(complex(row[5], row[6]) - zr) <= 1e-9 * abs(zr)
    peak = np.abs(p.currents).max()
    assert np.abs(res.currents[0] - p.currents).max() <= 1e-9 * peak
    g, ref = res.pattern[0][:, :3], p.pattern[:, :3]
    live = ref > -999.0
    assert np.abs(g[live] - ref[live]).max() <= 1e-6
    assert np.array_equal(g[~live], ref[~live])
    b.close()


def test_separate_sources_are_their_single_source_decks(acc):
    wires, sources, ground = DECKS["two_sources_one_path"]
    b = acc.HallenBatch([_antenna(acc, wires, sources, ground, separate=True)], precision=acc.PRECISION_FP64)
    res = b.solve()
    assert len(res.currents) == len(sources)
    for k, src in enumerate(sources):
        p = _oracle(wires, [src], ground, None)
        assert abs(complex(*res.feeds[k][0, 5:7]) - p.zin[0]) <= 1e-9 * abs(p.zin[0])
    b.close()


def test_mixed_within_gate(acc):
    ants = [_antenna(acc, w, s, g) for w, s, g in DECKS.values()]
    plain = acc.HallenBatch(ants, precision=acc.PRECISION_FP64).solve()
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    mixed = b.solve()
    assert np.all(mixed.status == 0)
    for fm, fp in zip(mixed.feeds, plain.feeds):
        zm, zp = complex(*fm[0, 5:7]), complex(*fp[0, 5:7])
        assert abs(zm - zp) <= 1e-6 * abs(zp)
    b.close()

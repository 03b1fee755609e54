"""Plane-wave receive solves on the device (planewave.rs:162-348,
linear.rs:910-1090, solve_session.rs:262-375) against the CPU oracle.

Plain FP64 form: pivots bit-exact, currents and the homogeneous constants
within 1e-9 of the largest entry, the receive pattern's dB within 1e-9.
Each incidence direction of the card is one right-hand side of the
frequency's factorisation, as the reference re-solves the same normal
equations for each.  Junctioned non-path decks and the mixed form are
refused with an error, never answered another way.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

F14 = 14.2e6
HALF = 5.282
DIPOLE = [(1, 51, (0, 0, -HALF), (0, 0, HALF), 0.001)]
TWO = [(1, 21, (0, 0, -2.5), (0, 0, 2.5), 0.001), (2, 21, (1.0, 0, -2.5), (1.0, 0, 2.5), 0.001)]
TILT = [(1, 41, (-3.0, -3.0, 0.0), (3.0, 3.0, 0.0), 0.001)]
SPLIT = [(1, 26, (0, 0, 0), (0, 0, HALF), 0.001), (2, 26, (0, 0, 0), (0, 0, -HALF), 0.001)]
VEE = [(1, 26, (0, 0, 5.0), (4.46, 0, 2.42), 0.001), (2, 26, (0, 0, 5.0), (-4.46, 0, 2.42), 0.001)]
# three wires of different lengths, a one-segment wire among them
MIXED = [(1, 13, (0, 0, -3.0), (0, 0, 3.0), 0.001), (2, 9, (1.5, 0, -2.0), (1.5, 0.5, 2.0), 0.002),
         (3, 1, (3.0, 0, 0), (3.0, 0, 0.4), 0.001)]


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _ant(acc, wires, freqs, card, ground=0, loads=None, rp=None):
    return acc.Antenna(acc.wires_array(wires), acc.sources_array([]), freqs, ground, rp,
                       loads=None if loads is None else acc.loads_array(loads), plane_wave=card)


def _oracle(wires, f, w, ground=0, loads=None):
    p = O.Problem(O.wires_array(wires), O.sources_array([]), f, ground=ground, wave=w,
                  loads=None if loads is None else O.loads_array(loads))
    O.solve_problem(p)
    assert p.status == 0
    return p


CASES = [
    ("dipole-linear", DIPOLE, (1, 30.0, 0.0, 0.0, 0.0), 0, None),
    ("dipole-broadside-pec", DIPOLE, (1, 90.0, 0.0, 0.0, 0.0), 1, None),
    ("two-wire", TWO, (1, 30.0, 0.0, 0.0, 0.0), 0, None),
    ("tilted-right-elliptic", TILT, (2, 45.0, 0.0, 0.0, 0.5), 0, None),
    ("tilted-left-elliptic", TILT, (3, 60.0, 25.0, 15.0, 0.3), 0, None),
    ("three-wires-eta", MIXED, (1, 50.0, 20.0, 30.0, 0.0), 0, None),
    ("split-path", SPLIT, (1, 55.0, 0.0, 0.0, 0.0), 0, None),
    ("inverted-v-path", VEE, (2, 70.0, 10.0, 20.0, 0.4), 0, None),
    ("dipole-loaded", DIPOLE, (1, 40.0, 0.0, 0.0, 0.0), 0, [(0, 1, 26, 26, 50.0, 1e-6, 1e-10)]),
]


@pytest.mark.parametrize("name,wires,wv,ground,loads", CASES, ids=[c[0] for c in CASES])
def test_receive_solve_matches_the_oracle(acc, name, wires, wv, ground, loads):
    t, th, ph, eta, ar = wv
    freqs = [F14, 21.1e6] if name != "two-wire" else [28.0e6]
    card = acc.plane_wave(t, th, ph, eta, axial_ratio=ar)
    b = acc.HallenBatch([_ant(acc, wires, freqs, card, ground, loads)])
    res = b.solve()
    assert np.all(res.status == 0)
    for u, f in enumerate(freqs):
        p = _oracle(wires, f, O.wave(t, th, ph, eta, ar), ground, loads)
        peak = np.abs(p.currents).max()
        assert np.abs(res.currents[u] - p.currents).max() <= 1e-9 * peak, name
        x, piv = b.read_unit(u)
        assert np.array_equal(piv, p.pivots[: len(piv)])
        assert len(x) == len(p.currents) + 2 * (1 if "path" in name else len(wires))
    b.close()


def test_currents_bit_level_on_the_dipole(acc):
    """With the same Z, forcing and normal equations the device solve is
    the oracle's to the last bit in most entries."""
    b = acc.HallenBatch([_ant(acc, DIPOLE, [F14], acc.plane_wave(1, 30.0))])
    res = b.solve()
    p = _oracle(DIPOLE, F14, O.wave(1, 30.0))
    same = np.mean(res.currents[0].view(np.uint64) == p.currents.view(np.uint64))
    assert same > 0.5, same
    b.close()


def test_receive_sweep_matches_the_oracle(acc):
    """An EX card with I2 x I3 directions: every direction one right-hand
    side of one factorisation per frequency (45 directions: the grouped
    kernels, two groups per frequency, the second partial); the response
    relative to the largest peak of its frequency."""
    card = acc.plane_wave(1, 10.0, 0.0, 0.0, n_theta=5, n_phi=9, d_theta=20.0, d_phi=40.0)
    freqs = [F14, 16.0e6]
    b = acc.HallenBatch([_ant(acc, DIPOLE, freqs, card)])
    res = b.solve()
    assert np.all(res.status == 0)
    rec = b.read_receive()
    waves = O.wave_directions(1, 5, 9, 10.0, 0.0, 20.0, 40.0)
    assert len(rec) == len(freqs) * len(waves)
    for fi, f in enumerate(freqs):
        peaks, db, cur = O.receive_sweep(O.wires_array(DIPOLE), f, waves)
        for d, w in enumerate(waves):
            u = fi * len(waves) + d
            assert b.units[u]["rhs"] == d
            assert rec[u, 0] == w.theta_deg and rec[u, 1] == w.phi_deg
            assert abs(rec[u, 2] - db[d]) <= 1e-9, (f, d, rec[u, 2], db[d])
            assert np.abs(res.currents[u] - cur[d]).max() <= 1e-9 * np.abs(cur[d]).max()
            _, piv = b.read_unit(u)
            _, piv0 = b.read_unit(fi * len(waves))
            assert np.array_equal(piv, piv0)  # one factorisation
        assert rec[fi * len(waves):(fi + 1) * len(waves), 2].max() == 0.0
    b.close()


def test_voltage_antennas_report_nan_receive_rows(acc):
    ants = [acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]), [F14], 0, None),
            _ant(acc, DIPOLE, [F14], acc.plane_wave(1, 30.0, n_theta=2, d_theta=30.0))]
    b = acc.HallenBatch(ants)
    res = b.solve()
    assert np.all(res.status == 0)
    rec = b.read_receive()
    assert np.all(np.isnan(rec[0]))
    assert rec[1, 0] == 30.0 and rec[2, 0] == 60.0 and max(rec[1, 2], rec[2, 2]) == 0.0
    p = O.Problem(O.wires_array(DIPOLE), O.sources_array([(1, 26, 1.0)]), F14)
    O.solve_problem(p)
    assert abs(complex(*res.feeds[0][0, 5:7]) - p.zin[0]) <= 1e-9 * abs(p.zin[0])
    b.close()


def test_pattern_of_a_receive_solve(acc):
    """An RP card on a receiving antenna: the pattern of the induced
    currents, as compute_radiation_pattern of those currents."""
    rp = (7, 3, 0.0, 0.0, 30.0, 60.0)
    b = acc.HallenBatch([_ant(acc, TILT, [F14], acc.plane_wave(2, 45.0, axial_ratio=0.5), rp=rp)])
    res = b.solve()
    p = _oracle(TILT, F14, O.wave(2, 45.0, 0.0, 0.0, 0.5))
    segs = O.build_geometry(O.wires_array(TILT))
    pts = O.rp_card_points(*rp)
    ref, _ = O.radiation_pattern(segs, p.currents, F14, pts)
    got = res.pattern[0][:, :4]
    live = ref[:, 0] > -999
    assert np.abs(got[live, :3] - ref[live, :3]).max() < 1e-6
    b.close()


def test_junctioned_plane_wave_deck_is_refused(acc):
    tee = [(1, 11, (0, 0, -2.5), (0, 0, 2.5), 0.001), (2, 11, (0, 0, 2.5), (2.5, 0, 2.5), 0.001),
           (3, 11, (0, 0, 2.5), (-2.5, 0, 2.5), 0.001)]
    coll = [(1, 11, (0, 0, -2.5), (0, 0, 0.0), 0.001), (2, 11, (0, 0, 0.0), (0, 0, 2.5), 0.001)]
    for wires in (tee, coll):
        with pytest.raises(Exception, match="junctioned"):
            acc.HallenBatch([_ant(acc, wires, [F14], acc.plane_wave(1, 30.0))])


def test_mixed_form_and_sources_are_refused(acc):
    with pytest.raises(Exception, match="FP64"):
        acc.HallenBatch([_ant(acc, DIPOLE, [F14], acc.plane_wave(1, 30.0))], precision=acc.PRECISION_MIXED)
    ant = acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]), [F14], 0, None,
                      plane_wave=acc.plane_wave(1, 30.0))
    with pytest.raises(Exception, match="voltage sources"):
        acc.HallenBatch([ant])


def test_grouped_right_hand_sides_equal_single_direction_solves(acc):
    """The grouped many-right-hand-side kernels against the first-solve path
    (the right-hand side carried through the Gram and the elimination):
    the same directions, one antenna each, give the same currents to the
    last bit."""
    card = acc.plane_wave(2, 15.0, 10.0, 25.0, n_theta=4, n_phi=9, d_theta=25.0, d_phi=35.0, axial_ratio=0.3)
    b = acc.HallenBatch([_ant(acc, MIXED, [F14], card)])
    res = b.solve()
    singles = [_ant(acc, MIXED, [F14], acc.plane_wave(2, 15.0 + it * 25.0, 10.0 + ip * 35.0, 25.0, axial_ratio=0.3))
               for it in range(4) for ip in range(9)]
    one = acc.HallenBatch(singles).solve()
    for u in range(36):
        assert np.array_equal(res.currents[u].view(np.uint64), one.currents[u].view(np.uint64)), u
    b.close()


def test_grouped_right_hand_sides_on_a_tall_factor(acc):
    """S = 393: beyond the four-warp kernel's shared tile, the grouped
    directions take the 16-lane kernel; still the single-direction solves
    to the last bit."""
    wire = [(1, 391, (0, 0, -15.0), (0, 0, 15.0), 0.001)]
    card = acc.plane_wave(1, 20.0, 0.0, 0.0, n_theta=9, d_theta=15.0)
    b = acc.HallenBatch([_ant(acc, wire, [F14], card)])
    res = b.solve()
    assert b.units[0]["s"] == 393
    one = acc.HallenBatch([_ant(acc, wire, [F14], acc.plane_wave(1, 20.0 + it * 15.0, 0.0, 0.0))
                           for it in range(9)]).solve()
    for u in range(9):
        assert np.array_equal(res.currents[u].view(np.uint64), one.currents[u].view(np.uint64)), u
    b.close()

"""The oracle's TL and NT stamps (tl.rs:47-241, network.rs:55-142) against
the reference's own unit tests of them, restated; the corpus TL/NT decks
are pinned in test_oracle_golden.py.

Geometry of the reference's TL tests: two parallel z wires of 3 (or 4)
segments, 1 m apart.
"""
import cmath
import math

import numpy as np

from oracle import oracle as O

F = 14.2e6
K = 2.0 * math.pi * F / 299792458.0


def _two_wires(nseg=3):
    return O.build_geometry(O.wires_array([(1, nseg, (0, 0, -1.0), (0, 0, 1.0), 0.001),
                                           (2, nseg, (1.0, 0, -1.0), (1.0, 0, 1.0), 0.001)]))


def _tl(*cards):
    return O.tls_array(cards)


def test_lossless_tl_stamps_a_symmetric_two_port():
    segs = _two_wires()
    st = O.tl_stamps(segs, F, _tl((1, 2, 2, 2, 1, 0, 50.0, 1.0, 1.0)))
    assert [(r, c) for r, c, _ in st] == [(1, 1), (4, 4), (1, 4), (4, 1)]
    theta = K * 1.0
    assert st[0][2] == st[1][2] and st[2][2] == st[3][2]
    assert abs(st[0][2] - (-50j * math.cos(theta) / math.sin(theta))) < 1e-12
    assert abs(st[2][2] - (-50j / math.sin(theta))) < 1e-12


def test_section_count_does_not_change_the_stamps():
    segs = _two_wires()
    base = O.tl_stamps(segs, F, _tl((1, 2, 2, 2, 1, 0, 50.0, 1.0, 1.0)))
    for nseg in (0, 3):
        assert O.tl_stamps(segs, F, _tl((1, 2, 2, 2, nseg, 0, 50.0, 1.0, 1.0))) == base


def test_segment_zero_is_the_centre():
    st = O.tl_stamps(_two_wires(3), F, _tl((1, 0, 2, 0, 1, 0, 50.0, 1.0, 1.0)))
    assert (st[0][0], st[1][0]) == (1, 4)  # the middle of 3
    st = O.tl_stamps(_two_wires(4), F, _tl((1, 0, 2, 0, 1, 0, 50.0, 1.0, 1.0)))
    assert (st[0][0], st[1][0]) == (1, 5)  # the lower centre (segment 2) of 4


def test_lossy_tl_is_z0_coth_and_csch():
    segs = _two_wires()
    st = O.tl_stamps(segs, F, _tl((1, 2, 2, 2, 1, 1, 50.0, 1.0, 3.0)))
    assert len(st) == 4
    gl = complex(3.0 * math.log(10.0) / 20.0, K * 1.0)
    assert abs(st[0][2] - 50.0 * cmath.cosh(gl) / cmath.sinh(gl)) < 1e-9
    assert abs(st[2][2] - 50.0 / cmath.sinh(gl)) < 1e-9


def test_invalid_tl_cards_are_ignored():
    segs = _two_wires()
    for card in ((1, 2, 1, 2, 1, 0, 50.0, 1.0, 1.0),    # both ends on one segment
                 (1, 2, 2, 2, 1, 0, 0.0, 1.0, 1.0),     # z0 <= 0
                 (1, 2, 2, 2, 1, 0, 50.0, 0.0, 1.0),    # length <= 0
                 (1, 9, 2, 2, 1, 0, 50.0, 1.0, 1.0),    # no such segment
                 (1, 2, 2, 2, 1, 0, 50.0, math.pi / K, 1.0)):  # sin(theta) ~ 0
        assert O.tl_stamps(segs, F, _tl(card)) == []


def test_nt_inverse_of_a_tl_stamps_like_that_tl():
    """network.rs: an NT whose Y-parameters invert a lossless TL's Z-parameters
    stamps what that TL stamps (to rounding)."""
    segs = _two_wires()
    tl = O.tl_stamps(segs, F, _tl((1, 2, 2, 2, 1, 0, 50.0, 1.0, 1.0)))
    z = np.array([[tl[0][2], tl[2][2]], [tl[3][2], tl[1][2]]])
    y = np.linalg.inv(z)
    nt = O.nt_stamps(segs, O.nts_array([(1, 2, 2, 2, y[0, 0].real, y[0, 0].imag, y[0, 1].real, y[0, 1].imag,
                                         y[1, 1].real, y[1, 1].imag)]))
    assert [(r, c) for r, c, _ in nt] == [(r, c) for r, c, _ in tl]
    for (_, _, a), (_, _, b) in zip(nt, tl):
        assert abs(a - b) < 1e-9 * abs(b)


def test_singular_or_degenerate_nt_is_ignored():
    segs = _two_wires()
    assert O.nt_stamps(segs, O.nts_array([(1, 2, 2, 2, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0)])) == []  # det = 0
    assert O.nt_stamps(segs, O.nts_array([(1, 2, 1, 2, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0)])) == []  # one segment

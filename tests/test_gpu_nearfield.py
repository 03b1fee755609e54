"""Near E and H fields on the device (farfield.rs:154-261 near_e_field /
near_h_field) against the CPU oracle's restatement.

Every operation of the per-segment sum is a separately rounded FP64 op in
the reference's order and sin/cos(kr) are correctly rounded on the device,
so most components agree bit for bit; the bar is 1e-13 of each point's
field magnitude, allowing a last-bit difference of the CPU's libm cos/sin
to propagate.  End to end (device solve, then device near field) the fields
match the oracle's within the 1e-9 current bar.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

FREQ = 14.2e6
DIPOLE = [(1, 51, (0, 0, -5.282), (0, 0, 5.282), 0.001)]
# a bent three-wire structure: segments along x, y and a slanted wire
BENT = [(1, 21, (0, 0, 1.0), (0, 0, 8.0), 0.002), (2, 15, (0, 0, 8.0), (4.0, 0, 8.0), 0.002),
        (3, 11, (4.0, 0, 8.0), (4.0, 3.0, 6.0), 0.001)]


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _solved(wires, feed):
    w = O.wires_array(wires)
    p = O.solve_problem(O.Problem(w, O.sources_array([feed]), FREQ))
    assert p.status == 0
    return O.build_geometry(w), p.currents


def _points(segs):
    """An NE rectangular grid through the structure, an NE spherical shell,
    points on the wire axis, a point exactly at a segment midpoint (that
    segment is skipped) and far points."""
    rect = O.near_field_points(0, 7, 5, 9, -3.0, -2.0, -6.0, 1.0, 1.0, 1.5)
    sph = O.near_field_points(1, 3, 8, 7, 2.0, 0.0, 0.0, 15.0, 45.0, 30.0)
    mids = np.array([s["mid"] for s in segs[:: max(1, len(segs) // 5)]], np.float64)
    axis = np.array([[0.0, 0.0, 20.0], [0.0, 0.0, -7.5], [1e-3, 0.0, 0.05]])
    far = np.array([[4000.0, 300.0, 2500.0], [-1.0e5, 2.0e4, 3.0e4]])
    return np.vstack([rect, sph, mids, axis, far])


def _check(got, want):
    mag = np.linalg.norm(want, axis=1)
    assert np.all(np.isfinite(got))
    err = np.abs(got - want).max(axis=1)
    assert np.all(err <= 1e-13 * mag + 1e-300), (err / np.maximum(mag, 1e-300)).max()
    same = np.mean(got.view(np.uint64) == want.view(np.uint64))
    return same


@pytest.mark.parametrize("wires,feed", [(DIPOLE, (1, 26, 1.0)), (BENT, (1, 1, 1.0))])
def test_near_field_matches_the_oracle(acc, wires, feed):
    segs, cur = _solved(wires, feed)
    pts = _points(segs)
    e, h = acc.near_field(acc.gpu_segments_from(segs), cur, FREQ, pts)
    e0, h0 = O.near_field(segs, cur, FREQ, pts)
    assert _check(e, e0) > 0.9
    assert _check(h, h0) > 0.9


def test_e_or_h_alone_and_empty_points(acc):
    segs, cur = _solved(DIPOLE, (1, 26, 1.0))
    pts = _points(segs)
    g = acc.gpu_segments_from(segs)
    e, h = acc.near_field(g, cur, FREQ, pts)
    e1, none_h = acc.near_field(g, cur, FREQ, pts, magnetic=False)
    none_e, h1 = acc.near_field(g, cur, FREQ, pts, electric=False)
    assert none_h is None and none_e is None
    assert np.array_equal(e1.view(np.uint64), e.view(np.uint64))
    assert np.array_equal(h1.view(np.uint64), h.view(np.uint64))
    e2, h2 = acc.near_field(g, cur, FREQ, np.zeros((0, 3)))
    assert e2.shape == (0, 3) and h2.shape == (0, 3)


def test_point_on_every_midpoint_skips_that_segment(acc):
    """A point within 1e-9 m of a midpoint leaves that segment out of the
    sum (farfield.rs:171-173): one segment alone at its own midpoint gives 0."""
    segs, cur = _solved(DIPOLE, (1, 26, 1.0))
    g = acc.gpu_segments_from(segs)
    e, h = acc.near_field(g[25:26], cur[25:26], FREQ, segs["mid"][25:26])
    assert np.all(e == 0) and np.all(h == 0)
    e, h = acc.near_field(g, cur, FREQ, segs["mid"])
    e0, h0 = O.near_field(segs, cur, FREQ, segs["mid"])
    _check(e, e0)
    _check(h, h0)


def test_far_limit_and_impedance_on_device(acc):
    """The reference's near-field properties (nec_solver/tests/near_field.rs)
    hold for the device fields: transverse E, |E| = eta |H| and azimuthal H
    at 200 wavelengths, and an axis-polarised broadside field."""
    segs, cur = _solved(DIPOLE, (1, 26, 1.0))
    g = acc.gpu_segments_from(segs)
    r = 200.0 * 299792458.0 / FREQ
    th = math.radians(60.0)
    e, h = acc.near_field(g, cur, FREQ, np.array([[r * math.sin(th), 0.0, r * math.cos(th)]]))
    e, h = e[0], h[0]
    e_r = e[0] * math.sin(th) + e[2] * math.cos(th)
    e_t = e[0] * math.cos(th) - e[2] * math.sin(th)
    assert abs(e_r) / abs(e_t) < 0.01
    eta = 4.0 * math.pi * 1e-7 * 299792458.0
    assert abs(np.linalg.norm(e) / np.linalg.norm(h) - eta) / eta < 0.02
    assert abs(h[0]) < 1e-6 * np.linalg.norm(h) and abs(h[2]) < 1e-6 * np.linalg.norm(h)
    e, _ = acc.near_field(g, cur, FREQ, np.array([[3.0, 0.0, 0.0]]), magnetic=False)
    assert abs(e[0][1]) < 1e-12 and abs(e[0][0]) < 1e-6 * abs(e[0][2])


def test_device_solve_then_device_near_field(acc):
    """End to end: the device's currents from a batch solve drive the device
    near field; against the oracle's solve and near field within 1e-9."""
    segs = O.build_geometry(O.wires_array(BENT))
    ant = acc.Antenna(acc.wires_array(BENT), acc.sources_array([(1, 1, 1.0)]), [FREQ], 0, None)
    b = acc.HallenBatch([ant])
    res = b.solve()
    assert res.status[0] == 0
    cur = np.asarray(res.currents[0])
    _, cur0 = _solved(BENT, (1, 1, 1.0))
    pts = _points(segs)
    e, h = acc.near_field(acc.gpu_segments_from(segs), cur, FREQ, pts)
    e0, h0 = O.near_field(segs, cur0, FREQ, pts)
    for got, want in ((e, e0), (h, h0)):
        mag = np.linalg.norm(want, axis=1)
        assert np.all(np.abs(got - want).max(axis=1) <= 1e-9 * mag)
    b.close()


def test_bad_arguments_are_errors(acc):
    segs, cur = _solved(DIPOLE, (1, 26, 1.0))
    g = acc.gpu_segments_from(segs)
    with pytest.raises(Exception):
        acc.near_field(g, cur, -1.0, np.zeros((2, 3)))
    with pytest.raises(ValueError):
        acc.near_field(g, cur, FREQ, np.zeros((2, 3)), electric=False, magnetic=False)

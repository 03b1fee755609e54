"""The oracle's near-field sums (farfield.rs:154-261) and NE/NH grid points
(solve_session.rs:645-688) against the reference's own tests of them
(nec_solver/tests/near_field.rs), restated on the same 51-segment
half-wave dipole at 14.2 MHz solved by the oracle."""
import math

import numpy as np
import pytest

from oracle import oracle as O

FREQ = 14.2e6
ETA = 4.0 * math.pi * 1e-7 * 299792458.0


@pytest.fixture(scope="module")
def dipole():
    w = O.wires_array([(1, 51, (0, 0, -5.282), (0, 0, 5.282), 0.001)])
    s = O.sources_array([(1, 26, 1.0)])
    p = O.solve_problem(O.Problem(w, s, FREQ))
    return O.build_geometry(w), p.currents, p.currents[25]


def _far_point(theta_deg=60.0):
    r = 200.0 * 299792458.0 / FREQ
    th = math.radians(theta_deg)
    return np.array([[r * math.sin(th), 0.0, r * math.cos(th)]]), r, th


def test_far_limit_is_transverse_and_matches_the_gain(dipole):
    segs, cur, i_feed = dipole
    pt, r, th = _far_point()
    e, _ = O.near_field(segs, cur, FREQ, pt)
    e = e[0]
    e_r = e[0] * math.sin(th) + e[2] * math.cos(th)
    e_t = e[0] * math.cos(th) - e[2] * math.sin(th)
    assert abs(e_r) / abs(e_t) < 0.01
    g_dbi = O.radiation_pattern(segs, cur, FREQ, np.array([[60.0, 0.0]]))[0][0, 1]  # gain_theta
    p_in = 0.5 * (1.0 * np.conj(i_feed)).real
    want = math.sqrt(10 ** (g_dbi / 10.0) * 2.0 * ETA * p_in / (4.0 * math.pi)) / r
    assert abs(abs(e_t) - want) / want < 0.02


def test_broadside_field_is_axis_polarised(dipole):
    segs, cur, _ = dipole
    e, _ = O.near_field(segs, cur, FREQ, np.array([[3.0, 0.0, 0.0]]))
    e = e[0]
    assert abs(e[1]) < 1e-12
    assert abs(e[0]) < 1e-6 * abs(e[2]) and abs(e[2]) > 0


def test_far_limit_impedance_and_azimuthal_h(dipole):
    segs, cur, _ = dipole
    pt, _, th = _far_point()
    e, h = O.near_field(segs, cur, FREQ, pt)
    emag, hmag = np.linalg.norm(e[0]), np.linalg.norm(h[0])
    assert abs(emag / hmag - ETA) / ETA < 0.02
    assert abs(h[0][0]) < 1e-6 * hmag and abs(h[0][2]) < 1e-6 * hmag  # H is along phi-hat = y here


def test_point_on_a_segment_midpoint_skips_that_segment(dipole):
    segs, cur, _ = dipole
    mid = np.array([segs["mid"][10]])
    e, h = O.near_field(segs, cur, FREQ, mid)
    e2, h2 = O.near_field(np.delete(segs, 10), np.delete(cur, 10), FREQ, mid)
    assert np.array_equal(e, e2) and np.array_equal(h, h2)


def test_grid_points_order():
    p = O.near_field_points(0, 2, 3, 2, 1.0, 2.0, 3.0, 0.5, 0.25, 1.0)
    assert len(p) == 12 and tuple(p[0]) == (1.0, 2.0, 3.0) and tuple(p[1]) == (1.0, 2.0, 4.0)
    assert tuple(p[2]) == (1.0, 2.25, 3.0) and tuple(p[6]) == (1.5, 2.0, 3.0)
    s = O.near_field_points(1, 2, 1, 2, 10.0, 0.0, 0.0, 5.0, 0.0, 90.0)  # theta outer, R inner
    assert np.allclose(s[0], (0, 0, 10.0)) and np.allclose(s[1], (0, 0, 15.0))
    assert np.allclose(s[2], (10.0, 0, 0), atol=1e-12) and np.allclose(s[3], (15.0, 0, 0), atol=1e-12)

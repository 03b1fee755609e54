"""The oracle's plane-wave receive solve (planewave.rs:37-348, linear.rs:
910-1090, solve_session.rs:262-375) against the reference's own tests of it,
restated: nec2c current-shape parity on the three tables that
nec_solver/tests/planewave_nec2c.rs holds (fixture
tests/golden/planewave_nec2c.json, with that file's bars), broadside
symmetry, elliptic-to-linear reductions, Rayleigh-Carson reciprocity, the
junction rejection, and the path receive solve of
nec_solver/tests/planewave_junction.rs.  Also: the structure-skipping Gram
equals the literal dense triple loop bit for bit.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
HALF = 5.282
F14 = 14.2e6
DIPOLE = [(1, 51, (0, 0, -HALF), (0, 0, HALF), 0.001)]


def _receive(wires, freq, w, ground=0):
    p = O.solve_problem(O.Problem(O.wires_array(wires), O.sources_array([]), freq, ground=ground, wave=w))
    assert p.status == 0
    return p.currents


def _golden():
    with open(os.path.join(HERE, "golden", "planewave_nec2c.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["NEC2C_CURRENTS", "NEC2C_TILT_ELLIPTIC", "NEC2C_TWO_WIRE"])
def test_shape_matches_the_nec2c_tables(name):
    g = _golden()[name]
    wires = [(t, s, tuple(a), tuple(b), r) for t, s, a, b, r in g["wires"]]
    cur = _receive(wires, g["freq_hz"], O.wave(*g["wave"]))
    ref = np.array([complex(a, b) for a, b in g["currents"]])
    assert len(cur) == len(ref)
    for lo, hi, pk, bar in g["groups"]:
        align = ref[pk] / cur[pk]
        dev = max(abs(cur[i] * align - ref[i]) / abs(ref[pk]) for i in range(lo, hi))
        assert dev < bar, (name, dev)


def test_broadside_current_is_symmetric():
    cur = _receive(DIPOLE, F14, O.wave(1, 90.0, 0.0, 0.0))
    n = len(cur)
    peak = max(abs(cur[n // 2]), 1e-30)
    assert max(abs(cur[i] - cur[n - 1 - i]) for i in range(n)) / peak < 1e-6


def test_elliptic_reduces_to_linear():
    lin = _receive(DIPOLE, F14, O.wave(1, 30.0, 0.0, 0.0, 0.0))
    ell = _receive(DIPOLE, F14, O.wave(2, 30.0, 0.0, 0.0, 0.5))
    assert np.abs(lin - ell).max() / abs(lin[25]) < 1e-9
    tilt = [(1, 41, (-3.0, -3.0, 0.0), (3.0, 3.0, 0.0), 0.001)]
    lin = _receive(tilt, F14, O.wave(1, 45.0, 0.0, 0.0, 0.0))
    ell0 = _receive(tilt, F14, O.wave(2, 45.0, 0.0, 0.0, 0.0))
    assert np.abs(lin - ell0).max() / abs(lin[20]) < 1e-9
    ell = _receive(tilt, F14, O.wave(3, 45.0, 0.0, 0.0, 0.5))  # left-hand differs on a tilted wire
    assert np.abs(lin - ell).max() / abs(lin[20]) > 1e-3


def test_reciprocity_tracks_the_transmit_pattern():
    tx = O.solve_problem(O.Problem(O.wires_array(DIPOLE), O.sources_array([(1, 26, 1.0)]), F14))
    segs = O.build_geometry(O.wires_array(DIPOLE))
    ratios = []
    for theta in (40.0, 55.0, 70.0, 90.0):
        g = O.radiation_pattern(segs, tx.currents, F14, np.array([[theta, 0.0]]))[0][0, 1]
        rx = _receive(DIPOLE, F14, O.wave(1, theta, 0.0, 0.0))
        ratios.append(abs(rx[25]) ** 2 / 10 ** (g / 10.0))
    mean = sum(ratios) / len(ratios)
    assert max(abs(r - mean) / mean for r in ratios) < 0.05


def test_two_parallel_wires_broadside_are_equal():
    wires = [(1, 21, (0, 0, -2.5), (0, 0, 2.5), 0.001), (2, 21, (1.0, 0, -2.5), (1.0, 0, 2.5), 0.001)]
    cur = _receive(wires, 28.0e6, O.wave(1, 90.0, 90.0, 0.0))
    assert np.abs(cur[:21] - cur[21:]).max() / abs(cur[10]) < 1e-9


def test_junctioned_geometry_is_rejected():
    wires = [(1, 11, (0, 0, -2.5), (0, 0, 2.5), 0.001), (2, 11, (0, 0, 2.5), (2.5, 0, 2.5), 0.001)]
    segs = O.build_geometry(O.wires_array(wires))
    with pytest.raises(O.OracleError):
        O.planewave_rhs(segs, F14, O.wave(1, 30.0, 0.0, 0.0))
    # the collinear continuation is a trivial path: per-wire form, rejected too
    coll = [(1, 11, (0, 0, -2.5), (0, 0, 0.0), 0.001), (2, 11, (0, 0, 0.0), (0, 0, 2.5), 0.001)]
    p = O.solve_problem(O.Problem(O.wires_array(coll), O.sources_array([]), F14, wave=O.wave(1, 30.0, 0.0, 0.0)))
    assert p.status == -8


def test_start_to_start_split_matches_the_single_wire():
    single = [(1, 52, (0, 0, -HALF), (0, 0, HALF), 0.001)]
    split = [(1, 26, (0, 0, 0), (0, 0, HALF), 0.001), (2, 26, (0, 0, 0), (0, 0, -HALF), 0.001)]
    paths = O.conductor_paths(O.build_geometry(O.wires_array(split)))
    assert len(paths) == 1 and paths.nontrivial
    for theta in (35.0, 55.0, 75.0, 90.0):
        a = np.abs(_receive(single, F14, O.wave(1, theta, 0.0, 0.0))).max()
        b = np.abs(_receive(split, F14, O.wave(1, theta, 0.0, 0.0))).max()
        assert abs(a - b) / a < 1e-8


def test_bent_inverted_v_reciprocity():
    vee = [(1, 26, (0, 0, 5.0), (4.46, 0, 2.42), 0.001), (2, 26, (0, 0, 5.0), (-4.46, 0, 2.42), 0.001)]
    tx = O.solve_problem(O.Problem(O.wires_array(vee), O.sources_array([(1, 1, 1.0)]), F14))
    assert tx.status == 0
    segs = O.build_geometry(O.wires_array(vee))
    ratios = []
    for theta in (40.0, 55.0, 70.0, 85.0):
        g = O.radiation_pattern(segs, tx.currents, F14, np.array([[theta, 0.0]]))[0][0, 1]
        rx = _receive(vee, F14, O.wave(1, theta, 0.0, 0.0))
        ratios.append(abs(rx[0]) ** 2 / 10 ** (g / 10.0))
    mean = sum(ratios) / len(ratios)
    assert max(abs(r - mean) / mean for r in ratios) < 0.05


@pytest.mark.parametrize("path_form", [False, True])
def test_skipping_gram_equals_the_dense_loop(path_form):
    wires = ([(1, 13, (0, 0, 0), (0, 0, 3.0), 0.001), (2, 9, (0, 0, 0), (2.0, 0, -1.0), 0.001)] if path_form else
             [(1, 13, (0, 0, -3.0), (0, 0, 3.0), 0.001), (2, 9, (1.5, 0, -2.0), (1.5, 0, 2.0), 0.002),
              (3, 1, (3.0, 0, 0), (3.0, 0, 0.4), 0.001)])
    segs = O.build_geometry(O.wires_array(wires))
    n = len(segs)
    z = O.assemble_z(segs, F14)
    w = O.wave(2, 50.0, 20.0, 30.0, 0.4)
    if path_form:
        paths = O.conductor_paths(segs)
        assert paths.nontrivial
        rhs, cosv, sinv = O.planewave_rhs(segs, F14, w, paths)
        args = (paths.path_of, len(paths), paths.free_ends)
    else:
        rhs, cosv, sinv = O.planewave_rhs(segs, F14, w)
        ep = O.wire_endpoints(segs)
        rw = np.zeros(n, np.int64)
        for q, (a, b) in enumerate(ep):
            rw[a:b + 1] = q
        args = (rw, len(ep), None)
    x1, p1, g1 = O.solve_hallen_planewave(z, rhs, cosv, sinv, *args, naive=False)
    x2, p2, g2 = O.solve_hallen_planewave(z, rhs, cosv, sinv, *args, naive=True)
    assert np.array_equal(g1.view(np.uint64), g2.view(np.uint64))
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64)) and np.array_equal(p1, p2)


def test_receive_sweep_response():
    waves = O.wave_directions(1, 3, 2, 20.0, 0.0, 35.0, 90.0)
    assert [(w.theta_deg, w.phi_deg) for w in waves] == [(20.0, 0.0), (20.0, 90.0), (55.0, 0.0), (55.0, 90.0),
                                                        (90.0, 0.0), (90.0, 90.0)]
    peaks, db, _ = O.receive_sweep(O.wires_array(DIPOLE), F14, waves)
    assert max(db) == 0.0 and np.argmax(peaks) in (4, 5)
    assert np.allclose(db, [20 * math.log10(p / peaks.max()) for p in peaks], rtol=0, atol=1e-12)

"""The oracle's LD load builder (loads.rs:103-222) against the reference's
own unit tests of it (loads.rs test module), restated; the corpus decks
with LD cards are pinned in test_oracle_golden.py.

Segments are built from one GW card of 2 segments of 0.1 m, radius 1 mm.
"""
import math

import numpy as np

from oracle import oracle as O

TWO_PI = 2.0 * math.pi
MU0 = 4.0 * math.pi * 1e-7


def _segs(nseg=2, tag=1):
    return O.build_geometry(O.wires_array([(tag, nseg, (0, 0, 0), (0, 0, 0.1 * nseg), 0.001)]))


def _load(segs, f, *cards):
    return O.build_loads(segs, f, O.loads_array(cards))


def test_type4_series_impedance_on_the_matching_segment_only():
    z, ign = _load(_segs(), 14.2e6, (4, 1, 2, 2, 100.0, 50.0, 0.0))
    assert ign == 0
    assert z[0] == 0
    assert abs(z[1].real - 100.0) < 1e-9 and abs(z[1].imag - 50.0) < 1e-9


def test_type0_series_rlc():
    f, l, c = 14.2e6, 1e-6, 1e-12
    z, _ = _load(_segs(1), f, (0, 1, 1, 1, 10.0, l, c))
    w = TWO_PI * f
    assert abs(z[0].real - 10.0) < 1e-6
    assert abs(z[0].imag - (w * l - 1.0 / (w * c))) < 1e-3


def test_type5_conductivity_dc_and_high_frequency_limits():
    sigma, a, dl = 5.8e7, 0.001, 0.1
    segs = _segs(1)
    lo, ign = _load(segs, 1e3, (5, 1, 1, 1, sigma, 0.0, 0.0))
    assert ign == 0
    r_dc = dl / (sigma * math.pi * a * a)
    assert abs(lo[0].real - r_dc) < 0.05 * r_dc
    assert abs(lo[0].imag) < 0.15 * lo[0].real
    f = 1e9
    delta = math.sqrt(2.0 / (TWO_PI * f * MU0 * sigma))
    r_hf = dl / (TWO_PI * a * sigma * delta)
    hi, _ = _load(segs, f, (5, 1, 1, 1, sigma, 0.0, 0.0))
    assert abs(hi[0].real - r_hf) < 0.02 * r_hf
    assert abs(hi[0].imag - hi[0].real) < 0.05 * hi[0].real
    assert hi[0].real > 100.0 * r_dc


def test_type5_non_positive_conductivity_is_ignored():
    z, ign = _load(_segs(1), 14.2e6, (5, 1, 1, 1, 0.0, 0.0, 0.0))
    assert ign == 1 and z[0] == 0


def test_type2_series_rl_and_type3_series_rc():
    f = 14.2e6
    z, _ = _load(_segs(1), f, (2, 1, 1, 1, 10.0, 1e-6, 0.0))
    assert abs(z[0].real - 10.0) < 1e-6 and abs(z[0].imag - TWO_PI * f * 1e-6) < 1e-6
    z, _ = _load(_segs(1), f, (3, 1, 1, 1, 10.0, 0.0, 1e-12))
    assert abs(z[0].real - 10.0) < 1e-6 and abs(z[0].imag + 1.0 / (TWO_PI * f * 1e-12)) < 1e-3


def test_unsupported_type_gives_zero_load():
    z, ign = _load(_segs(1), 14.2e6, (9, 1, 1, 1, 0.0, 0.0, 0.0))
    assert ign == 1 and z[0] == 0


def test_type1_parallel_forms():
    f = 14.2e6
    w = TWO_PI * f
    z, _ = _load(_segs(1), f, (1, 1, 1, 1, 200.0, 0.0, 0.0))
    assert abs(z[0].real - 200.0) < 1e-9 and abs(z[0].imag) < 1e-9
    r, l, c = 50.0, 1e-6, 100e-12
    z, _ = _load(_segs(1), f, (1, 1, 1, 1, r, l, c))
    want = 1.0 / complex(1.0 / r, -1.0 / (w * l) + w * c)
    assert abs(z[0] - want) < 1e-9 * abs(want)
    z, _ = _load(_segs(1), f, (1, 1, 1, 1, 0.0, 0.0, 0.0))
    assert z[0] == 0


def test_tag_zero_applies_to_every_segment_and_cards_add():
    segs = np.concatenate([_segs(2, 1), _segs(3, 2)])
    z, _ = _load(segs, 14.2e6, (4, 0, 0, 0, 50.0, 0.0, 0.0), (4, 2, 2, 3, 1.0, 2.0, 0.0))
    assert np.all(z.real[:2] == 50.0) and np.all(z.imag[:2] == 0.0)
    assert z[2] == 50.0 and np.all(z[3:] == 51.0 + 2.0j)

"""The library's deck reader (fnec_deck_parse, restating nec_parser::parse)
against a test-side restatement of the same semantics (tests/_deck.py), on
every corpus deck and on the reference parser's own edge cases.  Host code
only: no GPU."""
import ctypes
import json
import os

import numpy as np
import pytest

import _deck as R

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    return nec_accel


def _decks():
    with open(os.path.join(HERE, "golden", "corpus_decks.json")) as f:
        return json.load(f)["decks"]


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    raw = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(raw, dtype=dtype).copy()


@pytest.mark.parametrize("name", sorted(_decks()))
def test_reader_matches_the_restated_parser(acc, name):
    text = _decks()[name]
    try:
        ref = R.parse(text)
    except R.ParseFail as e:
        with pytest.raises(acc.AccelError, match=str(e).replace("$", r"\$")):
            acc.Deck(text)
        return
    d = acc.Deck(text)
    info = d.info()
    assert info["warnings"] == ref["warnings"]
    a, freqs = d.antenna()
    w = _arr(a.wires, a.n_wires, acc.WIRE_DTYPE)
    assert len(w) == len(ref["wires"])
    for got, (tag, nseg, s, e, r) in zip(w, ref["wires"]):
        assert (int(got["tag"]), int(got["segments"])) == (tag, nseg)
        assert tuple(got["start"]) == s and tuple(got["end"]) == e and float(got["radius"]) == r
    srcs = _arr(a.sources, a.n_sources, acc.SOURCE_DTYPE)
    want = [(e[1], e[2], e[4], e[5]) for e in ref["ex"] if e[0] in (0, 5)]
    assert [tuple(x.tolist()) for x in srcs] == want
    assert info["n_ex"] == len(ref["ex"])
    assert list(freqs) == R.frequencies(ref)  # bit for bit
    assert info["n_points"] == len(R.rp_points(ref))
    if len(ref["rp"]) > 1:
        pts = _arr(a.rp_points, a.n_rp_points * 2, np.float64).reshape(-1, 2)
        assert [tuple(p) for p in pts] == R.rp_points(ref)
    lds = _arr(a.loads, a.n_loads, acc.LOAD_DTYPE)
    assert [tuple(x.tolist()) for x in lds] == ref["ld"]
    tls = _arr(a.tls, a.n_tls, acc.TL_DTYPE)
    assert [tuple(x.tolist()) for x in tls] == ref["tl"]
    nts = _arr(a.nts, a.n_nts, acc.NT_DTYPE)
    assert [tuple(x.tolist()) for x in nts] == R.nts(ref)
    g = R.ground(ref)
    if g in (0, 1):
        assert info["ground"] == g
    pw = [e for e in ref["ex"] if e[0] in (1, 2, 3)]
    assert info["plane_wave"] == (1 if pw else 0)
    runnable = not ref["transforms"] and g in (0, 1) and not any(e[0] == 4 for e in ref["ex"]) and \
        bool(R.frequencies(ref)) and not (pw and want)
    assert info["runnable"] == (1 if runnable else 0), info["why"]
    d.close()


def test_fatal_errors_name_the_line_and_field(acc):
    with pytest.raises(acc.AccelError, match="line 2: GW needs 9 fields, got 3"):
        acc.Deck("CM x\nGW 1 2 3\nEN\n")
    with pytest.raises(acc.AccelError, match="line 1: GW field 3: cannot parse 'abc'"):
        acc.Deck("GW 1 5 abc 0 0 0 0 1 0.001\n")
    with pytest.raises(acc.AccelError, match="line 1: EX needs 4 fields, got 2"):
        acc.Deck("EX 0 1\n")
    with pytest.raises(acc.AccelError, match="field 5: cannot parse '0x10'"):
        acc.Deck("EX 0 1 1 0 0x10\n")


def test_unknown_cards_and_en(acc):
    d = acc.Deck("CM a\nZZ 1 2\nGW 1 11 0 0 -1 0 0 1 0.001\nXQ\nEX 0 1 6 0 1\nFR 0 1 0 0 28 0\nEN\nGW bad\n")
    i = d.info()
    assert i["warnings"] == 2 and "line 2: unknown card 'ZZ'" in i["why"]
    assert i["n_wires"] == 1 and i["runnable"] == 1  # nothing after EN is read


def test_field_forms(acc):
    """4nec2's float-written integers, the FR shorthand and canonical forms,
    RP with and without XNDA, EX/LD/TL defaults, saturating integer casts."""
    d = acc.Deck("GW 1.0 11.7 0 0 -1 0 0 1 1e-3\nEX 0 1 6 0\nFR 0 3 0 0 14.0 0.5\n"
                 "RP 0 2 3 1001 10 20 30 40\nLD 4 1 1 1 5\nTL 1 1 1 11 0 0 50 2\nGE -1\n")
    a, f = d.antenna()
    w = _arr(a.wires, a.n_wires, acc.WIRE_DTYPE)[0]
    assert int(w["tag"]) == 1 and int(w["segments"]) == 11
    s = _arr(a.sources, a.n_sources, acc.SOURCE_DTYPE)[0]
    assert (float(s["v_re"]), float(s["v_im"])) == (0.0, 0.0)
    assert list(f) == [14.0e6, 14.5e6, 15.0e6]
    rp = ctypes.cast(a.rp, ctypes.POINTER(acc._RpCard)).contents
    assert (rp.n_theta, rp.n_phi, rp.theta0, rp.phi0, rp.d_theta, rp.d_phi) == (2, 3, 10.0, 20.0, 30.0, 40.0)
    ld = _arr(a.loads, a.n_loads, acc.LOAD_DTYPE)[0]
    assert tuple(ld.tolist()) == (4, 1, 1, 1, 5.0, 0.0, 0.0)
    tl = _arr(a.tls, a.n_tls, acc.TL_DTYPE)[0]
    assert float(tl["f3"]) == 1.0
    assert d.info()["ground"] == 0
    d = acc.Deck("GW 1 5 0 0 0 0 0 1 0.001\nEX 0 1 1 0 1\nFR 1 4 10.0 1.1\nRP 0 2 1 0 0 45 0\nGN 1\n")
    _, f = d.antenna()
    assert list(f) == R.frequencies(R.parse("FR 1 4 10.0 1.1\n"))
    assert d.info()["ground"] == 1 and d.info()["n_points"] == 2
    d = acc.Deck("GW -3 -5 0 0 0 0 0 1 0.001\n")
    w = _arr(d.antenna()[0].wires, 1, acc.WIRE_DTYPE)[0]
    assert int(w["tag"]) == 0 and int(w["segments"]) == 0  # `as u32` saturates at 0


def test_unsupported_decks_say_why(acc):
    base = "GW 1 11 0 0 -1 0 0 1 0.001\nFR 0 1 0 0 28 0\n"
    for extra, why in (("GN 0\nEX 0 1 6 0 1\n", "GN 0"), ("GM 0 0 0 0 0 0 0 1 0\nEX 0 1 6 0 1\n", "GM / GR"),
                       ("EX 4 1 6 0 1\n", "EX 4"), ("EX 0 1 6 0 1\nEX 1 1 1 0 30 0\n", "both voltage")):
        i = acc.Deck(base + extra).info()
        assert i["runnable"] == 0 and why in i["why"], (extra, i["why"])
    assert acc.Deck("GW 1 11 0 0 -1 0 0 1 0.001\nEX 0 1 6 0 1\n").info()["why"] == "deck has no FR card"


def test_build_geometry_is_the_oracle_geometry(acc):
    from oracle import oracle as O

    wires = [(1, 7, (0.1, -2.0, 0.3), (1.7, 2.5, -0.9), 0.002), (5, 1, (3.0, 0, 0), (3.0, 0.4, 0.1), 0.001)]
    got = acc.build_geometry(acc.wires_array(wires))
    want = O.build_geometry(O.wires_array(wires))
    assert np.array_equal(got["midpoint"], want["mid"]) and np.array_equal(got["direction"], want["dir"])
    assert np.array_equal(got["length"], want["length"]) and np.array_equal(got["radius"], want["radius"])


def test_restated_formats_match_the_reference_strings():
    """The test-side report formats against the reference's own fixed
    strings (nec_report/src/lib.rs tests: format_feedpoint_row_is_stable,
    pattern_row_format_is_stable), plus Rust's exponent form and specials."""
    row = [0.1234567, -0.7654321, 1.0, -2.0, 74.242874, 13.899516]
    assert "1 26 " + " ".join(R.rfix(v, 6) for v in row) == \
        "1 26 0.123457 -0.765432 1.000000 -2.000000 74.242874 13.899516"
    assert [R.rfix(v, 4) for v in (90.0, 0.0, 2.1428, -999.99)] == ["90.0000", "0.0000", "2.1428", "-999.9900"]
    assert R.rfix(0.0078125, 6) == "0.007812"  # an exact tie rounds to even, as Rust and C do
    assert R.rfix(-0.0, 6) == "-0.000000" and R.rfix(-1e-9, 6) == "-0.000000"
    assert R.rexp(1234.5, 6) == "1.234500e3" and R.rexp(-0.00123, 6) == "-1.230000e-3"
    assert R.rexp(0.0, 6) == "0.000000e0" and R.rfix(float("nan"), 4) == "NaN" and R.rexp(float("-inf"), 6) == "-inf"


def test_restated_ne_points_are_the_oracle_points():
    """The test-side NE/NH grid (which the library's deck path must equal,
    tests/test_gpu_deck.py) against the oracle's near_field_grid_points."""
    from oracle import oracle as O

    for card in ((0, 3, 2, 4, -1.0, 0.5, 2.0, 0.7, 1.1, 0.25), (1, 2, 5, 3, 4.0, 10.0, 20.0, 1.5, 30.0, 25.0),
                 (1, 0, 0, 0, 2.0, 0.0, 90.0, 0.0, 0.0, 0.0)):
        want = O.near_field_points(*card)
        got = np.array(R.ne_points(card))
        assert got.shape == want.shape and np.array_equal(got, want), card


@pytest.mark.parametrize("card,what", [("RP 0 100000 100000 0 0 1 1", "RP cards ask for 10000000000 pattern points"),
                                       ("RP 0 2049 2048 0 0 1 1", "RP cards ask for 4196352 pattern points"),
                                       ("NE 0 2000 2000 2 0 0 0 1 1 1", "NE/NH cards ask for 8000000 field points"),
                                       ("FR 0 2000000 0 0 14.2 0.001", "FR card asks for 2000000 frequencies")])
def test_oversize_grids_are_refused_with_too_large(acc, card, what):
    """Grids the deck expands on the host are bounded: a card that asks for
    more than FNEC_DECK_MAX_POINTS points or FNEC_DECK_MAX_FREQS
    frequencies is refused with TOO_LARGE and a message, instead of an
    allocation failure escaping the C boundary."""
    base = ["CM big", "CE", "GW 1 11 0 0 -1 0 0 1 0.001", "GE 0", "EX 0 1 6 0 1 0", "FR 0 1 0 0 14.2 0"]
    lines = base[:-1] + [card] if card.startswith("FR") else base + [card]
    with pytest.raises(acc.AccelError) as ei:
        acc.Deck("\n".join(lines + ["EN"]) + "\n")
    assert ei.value.code == acc.ERR_TOO_LARGE
    assert what in str(ei.value)


def test_grid_at_the_limit_is_accepted(acc):
    d = acc.Deck("CM ok\nCE\nGW 1 11 0 0 -1 0 0 1 0.001\nGE 0\nEX 0 1 6 0 1 0\nFR 0 1 0 0 14.2 0\n"
                 "RP 0 2048 2048 0 0 0.05 0.1\nEN\n")
    assert d.info()["n_points"] == 2048 * 2048
    d.close()

"""Decks end to end on the device (fnec_deck_solve): the corpus decks'
text through the library's reader, one batch, and the report contract v1
text, gated as corpus_validation gates them -- the printed feedpoint
impedances against the reference's published values -- and checked byte
for byte against a test-side restatement of render_text_report
(tests/_deck.py) fed by the batch interface's results for the same deck.
"""
import json
import os

import numpy as np
import pytest

import _deck as R

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TL_COND = 2e-6  # the cond 1e13 linked-dipole TL decks (see test_gpu_parity.py)


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _golden():
    with open(os.path.join(HERE, "golden", "corpus_golden.json")) as f:
        return json.load(f)["cases"]


def _expected_report(acc, text):
    """The report of `text` rendered by tests/_deck.py from a batch built
    from the test-side parse."""
    ref = R.parse(text)
    ex_v = [e for e in ref["ex"] if e[0] in (0, 5)]
    pw = [e for e in ref["ex"] if e[0] in (1, 2, 3)]
    card = None
    if pw:
        t, tag, seg, _, vr, vi, f3, f4, f5, f6 = pw[0]
        card = acc.plane_wave(t, vr, vi, f3, n_theta=max(tag, 1), n_phi=max(seg, 1), d_theta=f4, d_phi=f5,
                              axial_ratio=f6)
    rp, rp_points = None, None
    if len(ref["rp"]) == 1:
        rp = tuple(ref["rp"][0][:6])
    elif ref["rp"]:
        rp_points = np.array(R.rp_points(ref))
    freqs = R.frequencies(ref)
    ant = acc.Antenna(acc.wires_array(ref["wires"]), acc.sources_array([(e[1], e[2], complex(e[4], e[5])) for e in ex_v]),
                      freqs, R.ground(ref), rp, loads=acc.loads_array(ref["ld"]) if ref["ld"] else None,
                      tls=acc.tls_array(ref["tl"]) if ref["tl"] else None,
                      nts=acc.nts_array(R.nts(ref)) if R.nts(ref) else None, plane_wave=card, rp_points=rp_points)
    b = acc.HallenBatch([ant])
    res = b.solve()
    assert np.all(res.status == 0)
    recv = b.read_receive() if card else None
    tags = [(w[0], i + 1) for w in ref["wires"] for i in range(w[1])]
    segs = acc.build_geometry(acc.wires_array(ref["wires"]))
    gsegs = acc.gpu_segments_from(segs)
    pts = R.rp_points(ref)
    per = (card[1] * card[2]) if card else 1
    out = []
    for fi, f in enumerate(freqs):
        u = fi * per
        feeds = [(*tags[int(r[0])], complex(r[1], r[2]), complex(r[3], r[4]), complex(r[5], r[6]))
                 for r in res.feeds[u]]
        pattern = [(pts[k][0], pts[k][1], *res.pattern[u][k, :4]) for k in range(len(res.pattern[u]))]
        receive = [tuple(recv[u + k]) for k in range(per)] if card and per > 1 else []
        near = {"NE": [], "NH": []}
        for kind, c in ref["ne"]:
            near[kind] += R.ne_points(c)
        rows = {}
        for kind in ("NE", "NH"):
            if near[kind]:
                e, h = acc.near_field(gsegs, res.currents[u], f, np.array(near[kind]))
                fld = e if kind == "NE" else h
                rows[kind] = [(*p, tuple(fld[k])) for k, p in enumerate(near[kind])]
        out.append(R.render(ref, f, "hallen-planewave" if card else "hallen", feeds, tags, res.currents[u], pattern,
                            receive, rows.get("NE", []), rows.get("NH", [])))
    b.close()
    return "\n".join(out)


def _feed_z(report):
    """(freq MHz, Z) of every FEEDPOINTS row of a report text."""
    out, freq, on = [], None, False
    for line in report.splitlines():
        if line.startswith("FREQ_MHZ "):
            freq = float(line.split()[1])
        elif line == "FEEDPOINTS":
            on = True
        elif on and line.startswith("TAG "):
            continue
        elif on and line and line[0].isdigit():
            c = line.split()
            out.append((freq, complex(float(c[6]), float(c[7]))))
        else:
            on = False
    return out


@pytest.mark.parametrize("name", sorted(_golden()))
def test_corpus_deck_report_gates(acc, name):
    case = _golden()[name]
    deck = acc.Deck(case["text"])
    text = deck.solve()
    assert text == _expected_report(acc, case["text"])
    zs = _feed_z(text)
    gold = case["feedpoint_impedance"]
    if "real_ohm" in gold:
        want = [complex(gold["real_ohm"], gold["imag_ohm"])]
        got = [z for _, z in zs]
    elif all(k.startswith("source_") for k in gold):
        want = [complex(gold[k]["real_ohm"], gold[k]["imag_ohm"]) for k in sorted(gold)]
        got = [z for _, z in zs]
    else:
        want = [complex(v["real_ohm"], v["imag_ohm"]) for _, v in sorted(gold.items(), key=lambda kv: float(kv[0]))]
        got = [z for _, z in sorted(zs, key=lambda fz: fz[0])]
    assert len(got) == len(want)
    for g, w in zip(got, want):
        digits = len(repr(w.real).split(".")[-1])
        tol = 2e-6 if digits >= 6 else 0.05
        if name.startswith("tl-"):
            tol = max(tol, TL_COND * abs(w))
        assert abs(g.real - w.real) <= tol and abs(g.imag - w.imag) <= tol, (name, g, w)
    deck.close()


def test_synthetic_deck_with_every_section(acc):
    """Sections the corpus decks do not use: an FR multiplicative sweep, PT
    filtering, several LD cards, NE and NH grids, RP with the normalise and
    average-gain digits over PEC ground."""
    text = ("CM every section\nCE\nGW 1 21 0 0 1.0 0 0 10.5 0.001\nGW 2 15 1.5 0 1.5 1.5 0 8.0 0.001\nGN 1\n"
            "EX 0 1 11 0 1.0 0.0\nLD 0 2 8 8 5.0 1e-6 0\nLD 4 1 3 3 10 -5\nPT 1 1 5 9\n"
            "FR 1 2 0 0 13.0 1.05\nRP 0 4 3 1001 0 0 25 60\nNE 0 2 1 3 2.0 0.5 1.0 1.0 0 2.0\n"
            "NH 1 2 3 2 5.0 0 30 2.0 45 40\nEN\n")
    deck = acc.Deck(text)
    got = deck.solve()
    assert got == _expected_report(acc, text)
    for sec in ("CURRENTS", "RADIATION_PATTERN", "NEAR_FIELD", "NEAR_H_FIELD", "NORMALIZED_PATTERN",
                "AVERAGE_POWER_GAIN", "LOADS", "SOURCES"):
        assert sec in got
    assert got.count("FNEC FEEDPOINT REPORT") == 2
    cur = got.split("CURRENTS\n")[1].split("\n\n")[0].splitlines()[1:]
    assert [tuple(map(int, c.split()[:2])) for c in cur] == [(1, s) for s in range(5, 10)]


def test_several_rp_cards_concatenate_their_grids(acc):
    """main.rs:292-304: two RP cards' points in card order, one pattern (the
    explicit point list of fnec_antenna), normalised over both."""
    text = ("GW 1 21 0 0 -2.5 0 0 2.5 0.001\nEX 0 1 11 0 1 0\nFR 0 1 0 0 28 0\n"
            "RP 0 5 1 1000 0 0 45 0\nRP 0 3 4 10 90 30 45 0\nEN\n")
    deck = acc.Deck(text)
    got = deck.solve()
    assert got == _expected_report(acc, text)
    assert "RADIATION_PATTERN\nN_POINTS 17" in got and "NORMALIZED_PATTERN\nN_POINTS 17" in got


def test_plane_wave_deck_reports_the_receive_pattern(acc):
    text = ("GW 1 31 0 0 -5.282 0 0 5.282 0.001\nEX 2 3 4 0 20.0 0.0 10.0 30.0 45.0 0.5\n"
            "FR 0 1 0 0 14.2 0\nRP 0 3 2 0 10 0 40 90\nEN\n")
    deck = acc.Deck(text)
    got = deck.solve()
    assert got == _expected_report(acc, text)
    assert "SOLVER_MODE hallen-planewave" in got and "RECEIVE_PATTERN\nN_POINTS 12" in got
    assert "FEEDPOINTS\nTAG SEG V_RE V_IM I_RE I_IM Z_RE Z_IM\n\n" in got  # a receiving antenna has no feed rows


def test_unsupported_and_singular_decks_are_errors(acc):
    deck = acc.Deck("GW 1 11 0 0 -1 0 0 1 0.001\nGN 2\nEX 0 1 6 0 1\nFR 0 1 0 0 28 0\n")
    with pytest.raises(acc.AccelError):
        deck.solve()


@pytest.mark.parametrize("name", ["dipole-ex1-freesp-51seg", "dipole-ex2-freesp-51seg", "dipole-ex3-freesp-51seg"])
def test_corpus_plane_wave_decks_print_the_oracle_currents(acc, name):
    """The corpus's receive decks end to end: the CURRENTS the report prints
    (6 significant digits) are the oracle's receive solve of the deck's
    first direction."""
    from oracle import oracle as O

    with open(os.path.join(HERE, "golden", "corpus_decks.json")) as f:
        text = json.load(f)["decks"][name]
    ref = R.parse(text)
    rep = acc.Deck(text).solve()
    e = [x for x in ref["ex"] if x[0] in (1, 2, 3)][0]
    p = O.Problem(O.wires_array(ref["wires"]), O.sources_array([]), R.frequencies(ref)[0],
                  wave=O.wave(e[0], e[4], e[5], e[6], e[9]))
    O.solve_problem(p)
    assert p.status == 0
    rows = rep.split("CURRENTS\n")[1].split("\n\n")[0].splitlines()[1:]
    got = np.array([complex(float(r.split()[2]), float(r.split()[3])) for r in rows])
    peak = np.abs(p.currents).max()
    assert len(got) == len(p.currents) and np.abs(got - p.currents).max() <= 1e-6 * peak

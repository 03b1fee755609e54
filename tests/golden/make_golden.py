"""Extract the Hallen-path golden vectors of the reference corpus into a small
committed fixture (tests/golden/corpus_golden.json).

Source: corpus/reference-results.json and the corpus/*.nec decks of
dc0sk/fnec-rust, read as text.  Only decks built from GW/GE/GN/EX/FR/RP
LD/TL/NT cards (no GM/GR transforms or plane waves) are kept:
those are the cases that exercise exactly the hot path (geometry, Hallen
RHS, Z fill, load stamps, normal-equation solve, feedpoint, RP pattern).

It also writes tests/golden/corpus_decks.json: the text of every corpus deck,
for the deck reader's tests.

Run in a checkout that has the reference mounted:
    python tests/golden/make_golden.py /path/to/fnec-rust
The GPU test host never runs this script; it only reads the JSON output.
"""
from __future__ import annotations

import json
import os
import sys

CASES = [
    "dipole-freesp-51seg",
    "dipole-freesp-rp-51seg",
    "dipole-ground-rp-51seg",
    "dipole-xaxis-rp-grid-51seg",
    "dipole-ground-51seg",
    "dipole-gn-1-null",
    "yagi-5elm-51seg",
    "frequency-sweep-dipole",
    "multi-source",
    "dipole-loaded",
    "dipole-ld-loaded-51seg",
    "dipole-ld-series-rl-51seg",
    "dipole-ld-series-rc-51seg",
    "tl-two-dipoles-linked",
    "tl-two-dipoles-linked-seg0",
    "tl-two-dipoles-linked-nseg0",
    "tl-two-dipoles-linked-seg0-even52",
    "dipole-nt-freesp-51seg",
    "dipole-nt-tl-equiv-freesp-51seg",
]


def parse_deck(text: str) -> dict:
    """Minimal NEC card reader for GW/GN/GE/EX/FR/RP/LD (columns as in NEC-2)."""
    deck = {"wires": [], "sources": [], "ground": 0, "freqs": [], "rp": None, "loads": [], "tls": [], "nts": []}
    ge_flag = 0
    gn = None
    for line in text.splitlines():
        f = line.split()
        if not f:
            continue
        card = f[0].upper()
        if card == "GW":
            tag, nseg = int(f[1]), int(f[2])
            x1, y1, z1, x2, y2, z2, rad = map(float, f[3:10])
            deck["wires"].append([tag, nseg, [x1, y1, z1], [x2, y2, z2], rad])
        elif card == "GE":
            ge_flag = int(f[1]) if len(f) > 1 else 0
        elif card == "GN":
            gn = int(f[1])
        elif card == "EX":
            ex_type, tag, seg = int(f[1]), int(f[2]), int(f[3])
            vr = float(f[5]) if len(f) > 5 else 0.0
            vi = float(f[6]) if len(f) > 6 else 0.0
            assert ex_type in (0, 5), "only voltage sources are on the hot path"
            deck["sources"].append([tag, seg, vr, vi])
        elif card == "FR":
            # nec_parser/src/lib.rs:273-291: >= 6 fields -> F1/F2 at 4/5,
            # else the shorthand at 2/3.  solve_session.rs:998 expands a
            # linear sweep as (f0 + i*df) * 1e6.
            g = f[1:]
            fi, si = (4, 5) if len(g) >= 6 else (2, 3)
            nfr, f0, df = int(g[1]), float(g[fi]), float(g[si])
            deck["freqs"] = [(f0 + i * df) * 1e6 for i in range(max(nfr, 1))]
        elif card == "LD":
            # nec_parser/src/lib.rs:325-355: I1 type, I2 tag, I3/I4 segments,
            # F1-F3 defaulting to 0
            g = f[1:]
            fl = [float(x) for x in g[4:7]] + [0.0] * (3 - len(g[4:7]))
            deck["loads"].append([int(g[0]), int(g[1]), int(g[2]), int(g[3])] + fl)
        elif card == "TL":
            # nec_parser/src/lib.rs:356-377: 6 integers, Z0, length, F3 (default 1)
            g = f[1:]
            deck["tls"].append([int(x) for x in g[:6]] + [float(g[6]), float(g[7]),
                                                           float(g[8]) if len(g) > 8 else 1.0])
        elif card == "NT":
            # network.rs:60-93: only a card with all 10 fields is stamped;
            # the reference warns and ignores any other
            g = f[1:]
            if len(g) >= 10:
                deck["nts"].append([int(x) for x in g[:4]] + [float(x) for x in g[4:10]])
        elif card == "RP":
            # nec_parser/src/lib.rs:293-325: angles start at field 4 with
            # XNDA present (>= 8 fields), else at field 3.
            g = f[1:]
            a = 4 if len(g) >= 8 else 3
            nt, nph = int(g[1]), int(g[2])
            th0, ph0, dth, dph = map(float, g[a:a + 4])
            deck["rp"] = [nt, nph, th0, ph0, dth, dph]
    # geometry.rs:71-111 ground_model_from_deck: GN 1 -> PEC, GN -1 -> free.
    if gn is not None:
        deck["ground"] = 1 if gn == 1 else 0
        assert gn in (1, -1), "only free space / PEC are on the hot path"
    elif ge_flag == 1:
        deck["ground"] = 1
    return deck


def main(ref_root: str) -> None:
    corpus = os.path.join(ref_root, "corpus")
    with open(os.path.join(corpus, "reference-results.json")) as fh:
        results = json.load(fh)["cases"]
    out = {
        "source": "dc0sk/fnec-rust corpus/reference-results.json (corpus_version 1.0)",
        "note": "feedpoint impedances printed to 6 decimals, pattern gains to 4",
        "cases": {},
    }
    for name in CASES:
        case = results[name]
        with open(os.path.join(corpus, case["deck_file"])) as fh:
            text = fh.read()
        deck = parse_deck(text)
        entry = {"deck_file": case["deck_file"], "deck": deck, "text": text,
                 "feedpoint_impedance": case.get("feedpoint_impedance", {}),
                 "tolerance_gates": case.get("tolerance_gates", {})}
        if "current_samples" in case:
            entry["current_samples"] = case["current_samples"]
        if "pattern_samples" in case:
            entry["pattern_samples"] = case["pattern_samples"]
        out["cases"][name] = entry
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "corpus_golden.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {dst} ({len(out['cases'])} cases)")
    # every corpus deck's text, for the deck reader's tests
    decks = {}
    for fn in sorted(os.listdir(corpus)):
        if fn.endswith(".nec"):
            with open(os.path.join(corpus, fn)) as fh:
                decks[fn[:-4]] = fh.read()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "corpus_decks.json")
    with open(dst, "w") as fh:
        json.dump({"source": "dc0sk/fnec-rust corpus/*.nec", "decks": decks}, fh, indent=1)
    print(f"wrote {dst} ({len(decks)} decks)")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FNEC_REFERENCE")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set FNEC_REFERENCE)" % os.path.basename(sys.argv[0]))
    main(ref)

"""Shared helpers: load the committed golden corpus fixture."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "corpus_golden.json")


def load_cases():
    with open(GOLDEN) as fh:
        return json.load(fh)["cases"]


def deck_arrays(deck):
    from oracle import oracle as O

    wires = O.wires_array([(w[0], w[1], tuple(w[2]), tuple(w[3]), w[4]) for w in deck["wires"]])
    sources = O.sources_array([(s[0], s[1], complex(s[2], s[3])) for s in deck["sources"]])
    pts = None
    if deck.get("rp"):
        pts = O.rp_card_points(*deck["rp"])
    return wires, sources, pts


def deck_loads(deck):
    """The deck's LD cards as the oracle's load array (None without any)."""
    from oracle import oracle as O

    ld = deck.get("loads") or []
    return O.loads_array([tuple(x) for x in ld]) if ld else None


def deck_networks(deck):
    """The deck's TL and NT cards as the oracle's arrays (None without any)."""
    from oracle import oracle as O

    tl, nt = deck.get("tls") or [], deck.get("nts") or []
    return (O.tls_array([tuple(x) for x in tl]) if tl else None, O.nts_array([tuple(x) for x in nt]) if nt else None)


def golden_zins(case):
    """Golden feedpoint impedances as {freq_hz: [z per source]}."""
    fp = case["feedpoint_impedance"]
    freqs = case["deck"]["freqs"]
    if "real_ohm" in fp:
        return {freqs[0]: [complex(fp["real_ohm"], fp["imag_ohm"])]}
    out = {}
    if all(k.startswith("source_") for k in fp):
        out[freqs[0]] = [complex(fp[k]["real_ohm"], fp[k]["imag_ohm"]) for k in sorted(fp)]
        return out
    for k, v in fp.items():
        out[float(k) * 1e6] = [complex(v["real_ohm"], v["imag_ohm"])]
    return out

"""Extract the nec2c current tables that the reference's plane-wave tests
compare against into a small committed fixture
(tests/golden/planewave_nec2c.json).

Source: crates/nec_solver/tests/planewave_nec2c.rs of dc0sk/fnec-rust, read
as text: the `const NAME: [(f64, f64); N]` arrays of (re, im) amps.  Each is
stored with the geometry and wave that the reference test builds it for
(planewave_nec2c.rs:89-127, :306-324, :420-437), and with the reference's
own shape bar (the relative deviation after aligning on the named peak
segment).

Run in a checkout that has the reference mounted:
    python tests/golden/make_planewave_golden.py /path/to/fnec-rust
The GPU test host never runs this script; it only reads the JSON output.
"""
from __future__ import annotations

import json
import os
import re
import sys

SRC = "crates/nec_solver/tests/planewave_nec2c.rs"
HALF = 5.282

TABLES = {
    # planewave_currents_match_nec2c_shape: 51-segment half-wave dipole, EX 1
    # theta 30, 14.2 MHz; aligned on segment 26 (index 25), bar 5 %
    "NEC2C_CURRENTS": {
        "wires": [[1, 51, [0.0, 0.0, -HALF], [0.0, 0.0, HALF], 0.001]],
        "freq_hz": 14.2e6,
        "wave": [1, 30.0, 0.0, 0.0, 0.0],
        "groups": [[0, 51, 25, 0.05]],
    },
    # elliptic_matches_nec2c_shape_on_tilted_wire: 41 segments from (-3,-3,0)
    # to (3,3,0), EX 2 theta 45 axial ratio 0.5; aligned on index 20, bar 7 %
    "NEC2C_TILT_ELLIPTIC": {
        "wires": [[1, 41, [-3.0, -3.0, 0.0], [3.0, 3.0, 0.0], 0.001]],
        "freq_hz": 14.2e6,
        "wave": [2, 45.0, 0.0, 0.0, 0.5],
        "groups": [[0, 41, 20, 0.07]],
    },
    # planewave_two_wire_per_wire_shape_matches_nec2c: two parallel 21-segment
    # z-dipoles 1 m apart at 28 MHz, EX 1 theta 30; each wire aligned on its
    # own peak (indices 10 and 31), bar 12 %
    "NEC2C_TWO_WIRE": {
        "wires": [[1, 21, [0.0, 0.0, -2.5], [0.0, 0.0, 2.5], 0.001],
                  [2, 21, [1.0, 0.0, -2.5], [1.0, 0.0, 2.5], 0.001]],
        "freq_hz": 28.0e6,
        "wave": [1, 30.0, 0.0, 0.0, 0.0],
        "groups": [[0, 21, 10, 0.12], [21, 42, 31, 0.12]],
    },
}


def parse_table(text: str, name: str):
    m = re.search(r"const\s+" + name + r"\s*:\s*\[\(f64,\s*f64\);\s*(\d+)\]\s*=\s*\[(.*?)\];", text, re.S)
    if not m:
        raise SystemExit(f"{name} not found in {SRC}")
    count = int(m.group(1))
    pairs = re.findall(r"\(\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\)", m.group(2))
    if len(pairs) != count:
        raise SystemExit(f"{name}: {len(pairs)} pairs, declared {count}")
    return [[float(a), float(b)] for a, b in pairs]


def main(root: str) -> None:
    with open(os.path.join(root, SRC)) as f:
        text = f.read()
    out = {}
    for name, meta in TABLES.items():
        out[name] = dict(meta, currents=parse_table(text, name), source=SRC)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "planewave_nec2c.json")
    with open(dst, "w") as f:
        json.dump(out, f)
        f.write("\n")
    print(f"wrote {dst}: " + ", ".join(f"{k} ({len(v['currents'])})" for k, v in out.items()))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FNEC_REFERENCE")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set FNEC_REFERENCE)" % os.path.basename(sys.argv[0]))
    main(ref)

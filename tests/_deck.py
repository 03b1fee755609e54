"""Test-side restatement of the reference's deck semantics, to check the
library's deck reader against: nec_parser::parse (crates/nec_parser/src/
lib.rs:78-485) for the cards the device path maps, ground_model_from_deck
(geometry.rs:71-110), frequencies_from_fr (solve_session.rs:984-1011), the
RP points of main.rs:292-304 (farfield.rs:677-699).  Python floats follow
the same IEEE operations in the same order.
"""
from __future__ import annotations

import math


class ParseFail(Exception):
    pass


def _f64(line, card, field, raw):
    try:
        low = raw.lower().lstrip("+-")
        if low.startswith("0x") or raw != raw.strip() or raw == "":
            raise ValueError
        return float(raw)
    except ValueError:
        raise ParseFail(f"line {line}: {card} field {field}: cannot parse '{raw}'")


def _as_u32(v):
    if v != v or v <= 0:
        return 0
    return min(int(v), 4294967295)


def _as_i32(v):
    if v != v:
        return 0
    return max(min(int(v), 2147483647), -2147483648)


def _need(line, card, f, n):
    if len(f) < n:
        raise ParseFail(f"line {line}: {card} needs {n} fields, got {len(f)}")


def _powi(a, b):  # compiler-rt __powidf2
    recip = b < 0
    r = 1.0
    while True:
        if b & 1:
            r *= a
        b = int(b / 2)
        if b == 0:
            break
        a *= a
    return 1.0 / r if recip else r


def parse(text: str) -> dict:
    d = {"wires": [], "gn": [], "ge": [], "transforms": False, "ex": [], "fr": [], "rp": [], "ld": [], "tl": [],
         "nt": [], "pt": [], "ne": [], "warnings": 0}
    for idx, raw in enumerate(text.split("\n")):
        no = idx + 1
        tok = raw.rstrip("\r").split()
        if not tok:
            continue
        m, f = tok[0].upper(), tok[1:]
        F = lambda k, r, _m=m, _no=no: _f64(_no, _m, k, r)  # noqa: E731
        if m in ("CM", "CE"):
            continue
        if m == "GW":
            _need(no, m, f, 9)
            d["wires"].append((_as_u32(F(1, f[0])), _as_u32(F(2, f[1])), tuple(F(3 + k, f[2 + k]) for k in range(3)),
                               tuple(F(6 + k, f[5 + k]) for k in range(3)), F(9, f[8])))
        elif m == "GE":
            d["ge"].append(_as_i32(F(1, f[0])) if f else 0)
        elif m in ("GM", "GR"):
            n = 9 if m == "GM" else 3
            _need(no, m, f, n)
            for k in range(n):
                F(k + 1, f[k])
            d["transforms"] = True
        elif m == "GN":
            _need(no, m, f, 1)
            if len(f) > 4:
                F(5, f[4])
            if len(f) > 5:
                F(6, f[5])
            d["gn"].append(_as_i32(F(1, f[0])))
        elif m == "EX":
            _need(no, m, f, 4)
            fl = [F(5 + k, f[4 + k]) if len(f) > 4 + k else 0.0 for k in range(6)]
            d["ex"].append([_as_u32(F(k + 1, f[k])) for k in range(4)] + fl)
        elif m == "FR":
            _need(no, m, f, 4)
            fi, si = (4, 5) if len(f) >= 6 else (2, 3)
            d["fr"].append((_as_u32(F(1, f[0])), _as_u32(F(2, f[1])), F(fi + 1, f[fi]), F(si + 1, f[si])))
        elif m == "RP":
            _need(no, m, f, 7)
            a = 4 if len(f) >= 8 else 3
            xnda = _as_u32(F(4, f[3])) if len(f) >= 8 else 0
            d["rp"].append((_as_u32(F(2, f[1])), _as_u32(F(3, f[2])), F(a + 1, f[a]), F(a + 2, f[a + 1]),
                            F(a + 3, f[a + 2]), F(a + 4, f[a + 3]), (xnda // 1000) % 10 != 0, xnda % 10 != 0))
        elif m == "LD":
            _need(no, m, f, 4)
            fl = [F(5 + k, f[4 + k]) if len(f) > 4 + k else 0.0 for k in range(3)]
            d["ld"].append((_as_i32(F(1, f[0])), _as_u32(F(2, f[1])), _as_u32(F(3, f[2])), _as_u32(F(4, f[3])), *fl))
        elif m == "TL":
            _need(no, m, f, 8)
            f3 = F(9, f[8]) if len(f) > 8 else 1.0
            d["tl"].append(tuple(_as_u32(F(k + 1, f[k])) for k in range(6)) + (F(7, f[6]), F(8, f[7]), f3))
        elif m == "NT":
            d["nt"].append(f)
        elif m == "PT":
            d["pt"].append(f)
        elif m in ("NE", "NH"):
            _need(no, m, f, 4)
            d["ne"].append((m, [_as_u32(F(k + 1, f[k])) for k in range(4)] +
                            [F(k + 1, f[k]) if len(f) > k else 0.0 for k in range(4, 10)]))
        elif m == "EN":
            break
        else:
            d["warnings"] += 1
    return d


def ground(d) -> int:
    if d["gn"]:
        return {-1: 0, 1: 1}.get(d["gn"][0], -99)
    return 1 if any(g == 1 for g in d["ge"]) else 0


def frequencies(d):
    if not d["fr"]:
        return []
    t, steps, f0, df = d["fr"][0]
    steps = max(steps, 1)
    if t == 0:
        return [(f0 + i * df) * 1e6 for i in range(steps)]
    if t == 1:
        return [f0 * _powi(df, i) * 1e6 for i in range(steps)]
    return [f0 * 1e6]


def rp_points(d):
    out = []
    for nt, nph, th0, ph0, dth, dph, _, _ in d["rp"]:
        for ip in range(max(nph, 1)):
            phi = ph0 + ip * dph
            for it in range(max(nt, 1)):
                out.append((th0 + it * dth, phi))
    return out


def nts(d):
    out = []
    for f in d["nt"]:
        if len(f) < 10:
            continue
        try:
            ends = [int(x) for x in f[:4]]
            if any(not (x.lstrip("+").isdigit()) for x in f[:4]):
                continue
            ys = [float(x) for x in f[4:10]]
        except ValueError:
            continue
        out.append(tuple(ends + ys))
    return out


# ---- report contract v1 formats (nec_report/src/lib.rs:307-484) -------------

def rfix(v, p):
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return f"{v:.{p}f}"


def rexp(v, p):
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    m, e = f"{v:.{p}e}".split("e")
    return f"{m}e{int(e)}"


def pt_filter(d):
    """solve_session.rs:781-826: the last PT card's (mode, tag, first, last)."""
    if not d["pt"]:
        return (0, 0, 0, 0)

    def g(i):
        f = d["pt"][-1]
        try:
            v = float(f[i].strip())
        except (IndexError, ValueError):
            return 0
        return 0 if v != v else int(v)
    return tuple(g(i) for i in range(4))


def ne_points(card):
    """solve_session.rs:645-688 near_field_grid_points."""
    coord, nx, ny, nz, x0, y0, z0, dx, dy, dz = card
    rad = math.pi / 180.0
    out = []
    if coord == 0:
        for ix in range(max(nx, 1)):
            for iy in range(max(ny, 1)):
                for iz in range(max(nz, 1)):
                    out.append((x0 + ix * dx, y0 + iy * dy, z0 + iz * dz))
    else:
        for it in range(max(nz, 1)):
            th = (z0 + it * dz) * rad
            for ip in range(max(ny, 1)):
                ph = (y0 + ip * dy) * rad
                for ir in range(max(nx, 1)):
                    r = x0 + ir * dx
                    out.append((r * math.sin(th) * math.cos(ph), r * math.sin(th) * math.sin(ph), r * math.cos(th)))
    return out


def render(d, freq_hz, mode, feeds, seg_tags, currents, pattern, receive, near_e, near_h):
    """nec_report::render_text_report (nec_report/src/lib.rs:307-484) of one
    frequency: feeds (tag, seg, V, I, Z complex), seg_tags (tag, index) per
    segment, currents per segment, pattern rows (theta, phi, g, gv, gh, ar),
    receive rows (theta, phi, dB), near rows (x, y, z, 3 complex)."""
    o = ["FNEC FEEDPOINT REPORT", "FORMAT_VERSION 1", f"FREQ_MHZ {rfix(freq_hz / 1e6, 6)}", f"SOLVER_MODE {mode}",
         "PULSE_RHS Nec2", "", "FEEDPOINTS", "TAG SEG V_RE V_IM I_RE I_IM Z_RE Z_IM"]
    for tag, seg, v, i, z in feeds:
        o.append(f"{tag} {seg} " + " ".join(rfix(x, 6) for x in (v.real, v.imag, i.real, i.imag, z.real, z.imag)))
    if d["ex"]:
        o += ["", "SOURCES", f"N_SOURCES {len(d['ex'])}", "TYPE TAG SEG I4 V_RE V_IM"]
        o += [f"{e[0]} {e[1]} {e[2]} {e[3]} {rfix(e[4], 6)} {rfix(e[5], 6)}" for e in d["ex"]]
    if d["ld"]:
        o += ["", "LOADS", f"N_LOADS {len(d['ld'])}", "TYPE TAG SEG_FIRST SEG_LAST F1 F2 F3"]
        o += [f"{l[0]} {l[1]} {l[2]} {l[3]} {rfix(l[4], 6)} {rfix(l[5], 6)} {rfix(l[6], 6)}" for l in d["ld"]]
    mode_pt, tag, first, last = pt_filter(d)
    rows = []
    if mode_pt > -1:
        for (t, s), c in zip(seg_tags, currents):
            if mode_pt != 0 and not ((tag == 0 or t == tag) and (first == 0 or (s >= first and (last == 0 or s <= last)))):
                continue
            ph = math.atan2(c.imag, c.real) * (180.0 / math.pi)
            rows.append(f"{t} {s} {rexp(c.real, 6)} {rexp(c.imag, 6)} {rexp(math.hypot(c.real, c.imag), 6)} "
                        f"{rfix(ph, 4)}")
    if rows:
        o += ["", "CURRENTS", "TAG SEG I_RE I_IM I_MAG I_PHASE"] + rows
    if pattern:
        o += ["", "RADIATION_PATTERN", f"N_POINTS {len(pattern)}", "THETA PHI GAIN_DB GAIN_V_DB GAIN_H_DB AXIAL_RATIO"]
        o += [" ".join(rfix(x, 4) for x in r) for r in pattern]
    if receive:
        o += ["", "RECEIVE_PATTERN", f"N_POINTS {len(receive)}", "THETA PHI RESPONSE_DB"]
        o += [" ".join(rfix(x, 4) for x in r) for r in receive]
    for title, head, rows_n in (("NEAR_FIELD", "X Y Z EX_RE EX_IM EY_RE EY_IM EZ_RE EZ_IM", near_e),
                                ("NEAR_H_FIELD", "X Y Z HX_RE HX_IM HY_RE HY_IM HZ_RE HZ_IM", near_h)):
        if rows_n:
            o += ["", title, f"N_POINTS {len(rows_n)}", head]
            for x, y, z, f in rows_n:
                o.append(" ".join(rfix(v, 4) for v in (x, y, z)) + " " +
                         " ".join(rexp(v, 6) for c in f for v in (c.real, c.imag)))
    if any(r[6] for r in d["rp"]) and pattern:
        peak = max([-math.inf] + [r[2] for r in pattern if r[2] == r[2]])
        o += ["", "NORMALIZED_PATTERN", f"N_POINTS {len(pattern)}", "THETA PHI GAIN_NORM_DB"]
        o += [f"{rfix(r[0], 4)} {rfix(r[1], 4)} {rfix(r[2] - peak if r[2] > -900.0 else r[2], 4)}" for r in pattern]
    if any(r[7] for r in d["rp"]) and pattern:
        num = den = 0.0
        for r in pattern:
            if r[2] <= -900.0:
                continue
            w = math.sin(r[0] * (math.pi / 180.0))
            num += math.pow(10.0, r[2] / 10.0) * w
            den += w
        if den > 0.0:
            o += ["", f"AVERAGE_POWER_GAIN {rfix(num / den, 4)}"]
    return "\n".join(o) + "\n"

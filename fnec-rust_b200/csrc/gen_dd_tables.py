"""Generate dd_tables.inc: double-double constants for the correctly rounded
sin/cos/log used by the exact-parity kernels.

Every entry is a mathematical constant evaluated with mpmath at 256 bits and
split into a (hi, lo) pair of doubles with hi = fl(v), lo = fl(v - hi):
  - pi/2 as three doubles (Cody-Waite reduction constant),
  - sin(i/64), cos(i/64) for i = 0..52,
  - 1/n! for n = 0..16,
  - ln 2, and ln(1 + j/64) for j = -32..32.
Run: python gen_dd_tables.py > dd_tables.inc
"""
import mpmath

mpmath.mp.prec = 256


def split(v):
    hi = float(v)
    lo = float(v - mpmath.mpf(hi))
    return hi, lo


def fmt(x):
    return float.hex(x)


def main():
    out = ["/* generated by gen_dd_tables.py -- do not edit */"]
    half_pi = mpmath.pi / 2
    p0 = float(half_pi)
    p1 = float(half_pi - p0)
    p2 = float(half_pi - p0 - p1)
    out.append(f"#define DD_PIO2_0 {fmt(p0)}")
    out.append(f"#define DD_PIO2_1 {fmt(p1)}")
    out.append(f"#define DD_PIO2_2 {fmt(p2)}")
    out.append(f"#define DD_TWO_OVER_PI {fmt(float(2 / mpmath.pi))}")
    ln2 = split(mpmath.log(2))
    out.append(f"#define DD_LN2_HI {fmt(ln2[0])}")
    out.append(f"#define DD_LN2_LO {fmt(ln2[1])}")
    out.append("FNEC_DD_TABLE double dd_sin_tab[53][2] = {")
    for i in range(53):
        h, l = split(mpmath.sin(mpmath.mpf(i) / 64))
        out.append(f"  {{{fmt(h)}, {fmt(l)}}},")
    out.append("};")
    out.append("FNEC_DD_TABLE double dd_cos_tab[53][2] = {")
    for i in range(53):
        h, l = split(mpmath.cos(mpmath.mpf(i) / 64))
        out.append(f"  {{{fmt(h)}, {fmt(l)}}},")
    out.append("};")
    out.append("FNEC_DD_TABLE double dd_inv_fact[17][2] = {")
    for n in range(17):
        h, l = split(1 / mpmath.factorial(n))
        out.append(f"  {{{fmt(h)}, {fmt(l)}}},")
    out.append("};")
    out.append("FNEC_DD_TABLE double dd_log_tab[65][2] = {  /* ln(1 + j/64), j = -32..32 */")
    for j in range(-32, 33):
        h, l = split(mpmath.log(1 + mpmath.mpf(j) / 64))
        out.append(f"  {{{fmt(h)}, {fmt(l)}}},")
    out.append("};")
    print("\n".join(out))


if __name__ == "__main__":
    main()

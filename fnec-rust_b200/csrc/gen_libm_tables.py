"""Generate libm_tables.inc: the sin/cos table of the FP64 libm restatement
in fnec_libm.cuh.

The reference evaluates f64::sin / f64::cos through the platform libm
(glibc on linux-gnu).  glibc's double sin/cos (sysdeps/ieee754/dbl-64/
s_sin.c, the IBM Accurate Mathematical Library design as simplified in
glibc 2.28) reduce |x| to a table point X_i = i/128 and a remainder of at
most 1/256 and combine sin(X_i), cos(X_i) -- each held as a double-double
(hi = fl(v), lo = fl(v - hi)) -- with short polynomials of the remainder.
The table entries are mathematical constants; they are evaluated here with
mpmath at 256 bits, for i = 0..109 (|x| < 0.85546875 = 109.5/128 is the
largest argument the table serves), in the layout sin hi, sin lo, cos hi,
cos lo per point (the file is the body of an array initialiser).
Run: python gen_libm_tables.py > libm_tables.inc
"""
import mpmath

mpmath.mp.prec = 256


def split(v):
    hi = float(v)
    lo = float(v - mpmath.mpf(hi))
    return hi, lo


def main():
    out = ["/* generated by gen_libm_tables.py -- do not edit; the 440 values of the",
           "   table, included inside an array initialiser */"]
    for i in range(110):
        x = mpmath.mpf(i) / 128
        sh, sl = split(mpmath.sin(x))
        ch, cl = split(mpmath.cos(x))
        out.append(f"  {float.hex(sh)}, {float.hex(sl)}, {float.hex(ch)}, {float.hex(cl)},")
    print("\n".join(out))


if __name__ == "__main__":
    main()

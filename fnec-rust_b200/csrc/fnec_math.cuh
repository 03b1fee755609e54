// fnec_math.cuh -- exact-parity arithmetic for the Hallen kernels.
//
// Three groups of functions:
//
//  1. Double-double (dd) arithmetic: Knuth/Dekker error-free transformations
//     (TwoSum, TwoProd via fma) and the usual dd add/mul built from them.
//
//  2. Correctly rounded sin/cos, ln and hypot.  The reference computes its
//     Z matrix with glibc's sin/cos/ln (Rust f64 methods on linux-gnu) and
//     picks pivots by glibc's hypot, which is correctly rounded.  The
//     regularised normal equations have cond(A) of 1e6..1e9, so 1-ulp
//     differences in a fraction of Z already move the solution by ~1e-9.
//     These functions evaluate in double-double (Cody-Waite reduction by
//     pi/2, a 1/64-step table of sin/cos/ln and Taylor/atanh series, all
//     constants from gen_dd_tables.py) and round once, so they return the
//     correctly rounded double except in the astronomically rare inputs
//     within ~2^-100 relative of a rounding midpoint.  They agree with glibc
//     wherever glibc is itself correctly rounded (all hypot calls; ~99.86 %
//     of sin/cos calls).
//
//  3. Complex arithmetic with the exact operation order of num-complex
//     0.4.6 and no FMA contraction (explicit _rn intrinsics on the device),
//     so sums and eliminations reproduce the reference bit for bit.
//
// The header compiles as CUDA device code under nvcc and as plain C++ under
// g++ (host unit tests of the correctly rounded functions).
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define FNEC_FN __device__ __forceinline__
#define FNEC_DD_TABLE static __device__ const
#define D_ADD(a, b) __dadd_rn((a), (b))
#define D_SUB(a, b) __dsub_rn((a), (b))
#define D_MUL(a, b) __dmul_rn((a), (b))
#define D_DIV(a, b) __ddiv_rn((a), (b))
#define D_SQRT(a) __dsqrt_rn((a))
#else
#define FNEC_FN static inline
#define FNEC_DD_TABLE static const
#define D_ADD(a, b) ((a) + (b))
#define D_SUB(a, b) ((a) - (b))
#define D_MUL(a, b) ((a) * (b))
#define D_DIV(a, b) ((a) / (b))
#define D_SQRT(a) sqrt((a))
#endif

#include "dd_tables.inc"

namespace fnec {

// ---------------------------------------------------------------------------
// double-double
// ---------------------------------------------------------------------------
struct dd {
    double hi, lo;
};

FNEC_FN dd two_sum(double a, double b) {
    double s = D_ADD(a, b);
    double bb = D_SUB(s, a);
    double e = D_ADD(D_SUB(a, D_SUB(s, bb)), D_SUB(b, bb));
    return {s, e};
}
FNEC_FN dd quick_two_sum(double a, double b) {
    double s = D_ADD(a, b);
    double e = D_SUB(b, D_SUB(s, a));
    return {s, e};
}
FNEC_FN dd two_prod(double a, double b) {
    double p = D_MUL(a, b);
    double e = fma(a, b, -p);
    return {p, e};
}
FNEC_FN dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    dd t = two_sum(a.lo, b.lo);
    s.lo = D_ADD(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = D_ADD(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}
FNEC_FN dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
FNEC_FN dd dd_sub(dd a, dd b) { return dd_add(a, dd_neg(b)); }
FNEC_FN dd dd_mul(dd a, dd b) {
    dd p = two_prod(a.hi, b.hi);
    p.lo = fma(a.hi, b.lo, p.lo);
    p.lo = fma(a.lo, b.hi, p.lo);
    return quick_two_sum(p.hi, p.lo);
}
FNEC_FN dd dd_mul_d(dd a, double b) {
    dd p = two_prod(a.hi, b);
    p.lo = fma(a.lo, b, p.lo);
    return quick_two_sum(p.hi, p.lo);
}
FNEC_FN dd dd_div(dd a, dd b) {
    double q1 = D_DIV(a.hi, b.hi);
    dd r = dd_sub(a, dd_mul_d(b, q1));
    double q2 = D_DIV(r.hi, b.hi);
    r = dd_sub(r, dd_mul_d(b, q2));
    double q3 = D_DIV(r.hi, b.hi);
    dd q = quick_two_sum(q1, q2);
    return dd_add(q, dd{q3, 0.0});
}
FNEC_FN dd dd_tab(const double (*t)[2], int i) { return {t[i][0], t[i][1]}; }
// Round a dd to the nearest double (hi + lo with a full TwoSum).
FNEC_FN double dd_round(dd a) { return two_sum(a.hi, a.lo).hi; }

// ---------------------------------------------------------------------------
// correctly rounded sin/cos
// ---------------------------------------------------------------------------

// sin(t), cos(t) for |t| <= 1/128 (plus rounding slack), t given as dd.
// Taylor series; the tail terms are small enough to run in double.
FNEC_FN void dd_sincos_small(dd t, dd *s, dd *c) {
    dd u = dd_mul(t, t);  // t^2
    double ud = u.hi;
    // sin: t * (1 - u/3! + u^2/5! - u^3/7! + u^4/9! - u^5/11!)
    double sv = fma(ud, dd_inv_fact[11][0], -dd_inv_fact[9][0]);  // -(1/9! - u/11!)
    sv = fma(ud, -sv, -dd_inv_fact[7][0]);                         // -1/7! + u(1/9! - u/11!)
    dd sw = dd_add(dd_tab(dd_inv_fact, 5), dd{D_MUL(ud, sv), 0.0});
    sw = dd_sub(dd_mul(u, sw), dd_tab(dd_inv_fact, 3));
    sw = dd_add(dd{1.0, 0.0}, dd_mul(u, sw));
    *s = dd_mul(t, sw);
    // cos: 1 - u/2! + u^2/4! - u^3/6! + u^4/8! - u^5/10! + u^6/12!
    double cv = fma(ud, dd_inv_fact[12][0], -dd_inv_fact[10][0]);
    cv = fma(ud, cv, dd_inv_fact[8][0]);
    cv = fma(ud, cv, -dd_inv_fact[6][0]);
    dd cw = dd_add(dd_tab(dd_inv_fact, 4), dd{D_MUL(ud, cv), 0.0});
    cw = dd_sub(dd_mul(u, cw), dd_tab(dd_inv_fact, 2));
    *c = dd_add(dd{1.0, 0.0}, dd_mul(u, cw));
}

// Correctly rounded (sin x, cos x) for |x| < 2^20; outside that range (never
// reached by the Hallen kernels: |x| = k*R with k <= 2pi*30 MHz/c) the
// platform sincos is used.
FNEC_FN void cr_sincos(double x, double *sn, double *cs) {
    if (x == 0.0) {
        *sn = x;
        *cs = 1.0;
        return;
    }
    if (!(fabs(x) < 1048576.0)) {
#ifdef __CUDACC__
        sincos(x, sn, cs);
#else
        *sn = sin(x);
        *cs = cos(x);
#endif
        return;
    }
    double q = rint(D_MUL(x, DD_TWO_OVER_PI));
    // x - q*pi/2 with pi/2 = P0 + P1 + P2; fma(-q, P0, x) is exact here.
    double r0 = fma(-q, DD_PIO2_0, x);
    dd p1 = two_prod(q, DD_PIO2_1);
    dd r = dd_sub(dd{r0, 0.0}, p1);
    r = dd_sub(r, dd{D_MUL(q, DD_PIO2_2), 0.0});
    // table step: r = a + t, a = i/64
    double ai = rint(D_MUL(r.hi, 64.0));
    int i = (int)ai;
    int ia = i < 0 ? -i : i;
    double a = D_MUL(ai, 0.015625);
    dd t = quick_two_sum(D_SUB(r.hi, a), r.lo);
    dd st, ct;
    dd_sincos_small(t, &st, &ct);
    dd sa = dd_tab(dd_sin_tab, ia);
    if (i < 0) sa = dd_neg(sa);
    dd ca = dd_tab(dd_cos_tab, ia);
    dd s = dd_add(dd_mul(sa, ct), dd_mul(ca, st));
    dd c = dd_sub(dd_mul(ca, ct), dd_mul(sa, st));
    int quad = (int)((long long)q & 3);
    double sv, cv;
    switch (quad) {
        case 0: sv = dd_round(s); cv = dd_round(c); break;
        case 1: sv = dd_round(c); cv = -dd_round(s); break;
        case 2: sv = -dd_round(s); cv = -dd_round(c); break;
        default: sv = -dd_round(c); cv = dd_round(s); break;
    }
    *sn = sv;
    *cs = cv;
}

// ---------------------------------------------------------------------------
// correctly rounded natural log (positive, finite, normal arguments)
// ---------------------------------------------------------------------------
FNEC_FN double cr_log(double x) {
    if (!(x > 0.0) || x == INFINITY || x < 2.2250738585072014e-308) return log(x);
    int e;
    double m = frexp(x, &e);  // m in [0.5, 1)
    m = D_MUL(m, 2.0);
    e -= 1;                   // x = m * 2^e, m in [1, 2)
    if (m > 1.4142135623730951) {
        m = D_MUL(m, 0.5);
        e += 1;
    }
    double jd = rint(D_MUL(D_SUB(m, 1.0), 64.0));
    int j = (int)jd;
    double c = D_ADD(1.0, D_MUL(jd, 0.015625));
    double num = D_SUB(m, c);          // exact
    dd den = two_sum(m, c);
    dd s = dd_div(dd{num, 0.0}, den);  // (m - c) / (m + c)
    dd s2 = dd_mul(s, s);
    double v = s2.hi;
    // 2*atanh(s) = 2 s (1 + s^2/3 + s^4/5 + s^6/7 + s^8/9 + s^10/11 + s^12/13)
    double tail = fma(v, 1.0 / 13.0, 1.0 / 11.0);
    tail = fma(v, tail, 1.0 / 9.0);
    tail = fma(v, tail, 1.0 / 7.0);
    tail = fma(v, tail, 1.0 / 5.0);
    dd third = dd_div(dd{1.0, 0.0}, dd{3.0, 0.0});
    dd w = dd_add(third, dd{D_MUL(v, tail), 0.0});
    w = dd_add(dd{1.0, 0.0}, dd_mul(s2, w));
    dd at = dd_mul_d(dd_mul(s, w), 2.0);
    dd ln2 = {DD_LN2_HI, DD_LN2_LO};
    dd res = dd_add(dd_mul_d(ln2, (double)e), dd_tab(dd_log_tab, j + 32));
    res = dd_add(res, at);
    return dd_round(res);
}

// ---------------------------------------------------------------------------
// correctly rounded hypot
// ---------------------------------------------------------------------------
// neighbours of a positive finite double
FNEC_FN double next_up_pos(double h) {
#ifdef __CUDACC__
    return __longlong_as_double(__double_as_longlong(h) + 1);
#else
    int64_t b;
    memcpy(&b, &h, sizeof b);
    b += 1;
    memcpy(&h, &b, sizeof b);
    return h;
#endif
}
FNEC_FN double next_down_pos(double h) {
#ifdef __CUDACC__
    return __longlong_as_double(__double_as_longlong(h) - 1);
#else
    int64_t b;
    memcpy(&b, &h, sizeof b);
    b -= 1;
    memcpy(&h, &b, sizeof b);
    return h;
#endif
}

FNEC_FN double cr_hypot(double a, double b) {
    a = fabs(a);
    b = fabs(b);
    if (!(a <= 1.0e300 && b <= 1.0e300)) return hypot(a, b);  // inf / nan / huge
    if (a == 0.0) return b;
    if (b == 0.0) return a;
    double big = a > b ? a : b;
    double scale = 1.0;
    if (big < 0x1p-450) {  // keep the squares (and their TwoProd errors) normal
        scale = 0x1p-600;
        a = D_MUL(a, 0x1p600);
        b = D_MUL(b, 0x1p600);
    } else if (big > 0x1p450) {
        scale = 0x1p600;
        a = D_MUL(a, 0x1p-600);
        b = D_MUL(b, 0x1p-600);
    }
    dd s = dd_add(two_prod(a, a), two_prod(b, b));  // a^2 + b^2 to ~2^-106
    double h = D_SQRT(s.hi);
    // residual s - h^2 (fma gives s.hi - h^2 exactly for the rounded sqrt)
    double rho = D_ADD(fma(-h, h, s.hi), s.lo);
    int ex;
    frexp(h, &ex);
    double ulp = ldexp(1.0, ex - 53);
    // true sqrt above the upper midpoint h + ulp/2 ?
    if (rho > fma(h, ulp, D_MUL(0.25, D_MUL(ulp, ulp)))) {
        h = next_up_pos(h);
    } else {
        double ulpd = (h == ldexp(1.0, ex - 1)) ? D_MUL(ulp, 0.5) : ulp;
        if (rho < -fma(h, ulpd, -D_MUL(0.25, D_MUL(ulpd, ulpd)))) h = next_down_pos(h);
    }
    return D_MUL(h, scale);
}

// ---------------------------------------------------------------------------
// num-complex 0.4.6 arithmetic, each operation separately rounded
// ---------------------------------------------------------------------------
struct cx {
    double re, im;
};
FNEC_FN cx cx_make(double re, double im) { return {re, im}; }
FNEC_FN cx cx_add(cx a, cx b) { return {D_ADD(a.re, b.re), D_ADD(a.im, b.im)}; }
FNEC_FN cx cx_sub(cx a, cx b) { return {D_SUB(a.re, b.re), D_SUB(a.im, b.im)}; }
// (ac - bd, ad + bc)
FNEC_FN cx cx_mul(cx a, cx b) {
    return {D_SUB(D_MUL(a.re, b.re), D_MUL(a.im, b.im)), D_ADD(D_MUL(a.re, b.im), D_MUL(a.im, b.re))};
}
// conj(a) * b exactly as num-complex evaluates it: (ar*br - (-ai)*bi,
// ar*bi + (-ai)*br), which IEEE makes equal to (ar*br + ai*bi, ar*bi - ai*br).
FNEC_FN cx cx_conj_mul(cx a, cx b) {
    return {D_ADD(D_MUL(a.re, b.re), D_MUL(a.im, b.im)), D_SUB(D_MUL(a.re, b.im), D_MUL(a.im, b.re))};
}
// ((ac + bd) / |b|^2, (bc - ad) / |b|^2)
FNEC_FN cx cx_div(cx a, cx b) {
    double ns = D_ADD(D_MUL(b.re, b.re), D_MUL(b.im, b.im));
    double re = D_ADD(D_MUL(a.re, b.re), D_MUL(a.im, b.im));
    double im = D_SUB(D_MUL(a.im, b.re), D_MUL(a.re, b.im));
    return {D_DIV(re, ns), D_DIV(im, ns)};
}
FNEC_FN double cx_norm(cx a) { return cr_hypot(a.re, a.im); }
FNEC_FN double cx_norm_sqr(cx a) { return D_ADD(D_MUL(a.re, a.re), D_MUL(a.im, a.im)); }

}  // namespace fnec

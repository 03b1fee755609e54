// FP64 sin, cos and hypot that return, bit for bit, what the reference's
// f64::sin, f64::cos and f64::hypot return on linux-gnu, where Rust calls
// the platform libm (hypot: at the end of this file).
//
// The reference's Z fill evaluates exp(-jkR) through num-complex's
// Complex64::exp (from_polar: cos and sin of -kR; matrix.rs:397 green_k),
// and its Hallen right-hand side takes cos(k s) and sin(k |s - s_src|)
// (excitation.rs:119-244).  Those values come from glibc 2.39 (the libm of
// this image), whose double sin/cos are not correctly rounded: about 0.1 %
// of arguments land 1 ulp away from the correctly rounded value.  The normal
// equations of ill-conditioned decks (cond(A) ~ 1e13 for linked-dipole TL
// decks) amplify such 1-ulp differences in Z to 1e-6 of Zin, so the exact
// form evaluates the same algorithm with the same roundings.
//
// The algorithm is glibc's sysdeps/ieee754/dbl-64/s_sin.c (IBM Accurate
// Mathematical Library, as simplified in glibc 2.28), restated here:
//  - |x| < 2^-26 (sin) / 2^-27 (cos): x / 1;
//  - |x| < 0.85546875: table point X = round(|x|*128)/128 (by adding
//    1.5*2^45), remainder r = |x| - X, and
//      sin(X + r) = sin X + [(sin_lo + s*cos_lo - sin X * c) + cos X * s]
//      cos(X + r) = cos X + [(cos_lo - s*sin_lo - cos X * c) - sin X * s]
//    with s = r + r^3 (sn3 + r^2 sn5) ~ sin r and c = r^2 (cs2 + ...) ~
//    1 - cos r; below 0.126, sin uses an odd Taylor polynomial (s1..s5);
//  - |x| < 2.426265: the argument is taken from pi/2 (hp0 + hp1) and the
//    other function is evaluated;
//  - |x| < 105414336: x - n*pi/2 in a double-double (pi/2 = mp1 + mp2 +
//    pp3 + pp4, n from x*2/pi rounded by adding 1.5*2^52), then the
//    quadrant's function.
// Larger arguments need glibc's multi-word reduction (branred.c) and are not
// restated: no wire geometry reaches k*R of 1e8.  Callers keep |x| below
// LIBM_SINCOS_MAX and the functions return NaN beyond it.
//
// Contraction: on x86-64 CPUs with FMA and AVX2, glibc selects the variant
// of s_sin.c compiled with -mfma -mavx2 (sysdeps/x86_64/fpu/multiarch), in
// which GCC fuses every multiply whose only uses are additions or
// subtractions into an FMA.  The fused operations are written out below as
// FMAs, the others as separately rounded multiplies and adds; the host test
// compares this code with the host libm on millions of arguments.
//
// Constants: the polynomial coefficients and the range-reduction splits of
// pi/2 and 2/pi are glibc's (usncs.h); the table of sin/cos at i/128 is
// evaluated with mpmath (gen_libm_tables.py).
//
// ln, the one other libm function of the exact fill, enters only through
// the per-segment self term; the host evaluates that term with the host
// libm (DevSeg::self_log), so no ln is restated here.
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define FNEC_LIBM_FN __host__ __device__ __forceinline__
#else
#define FNEC_LIBM_FN static inline
#endif

namespace fnec_libm {

// sin(i/128) hi, lo, cos(i/128) hi, lo for i = 0..109.  The device copy
// lives in global memory and is read through the read-only cache: the lanes
// of a warp index it with different points, which the constant cache would
// serialise.
#ifdef __CUDACC__
static __device__ const double libm_sincos_tab_dev[440] = {
#include "libm_tables.inc"
};
#endif
static const double libm_sincos_tab_host[440] = {
#include "libm_tables.inc"
};

#ifdef __CUDA_ARCH__
#define LM_FMA(a, b, c) __fma_rn((a), (b), (c))
#define LM_MUL(a, b) __dmul_rn((a), (b))
#define LM_ADD(a, b) __dadd_rn((a), (b))
#define LM_SUB(a, b) __dsub_rn((a), (b))
#define LM_TAB(i) __ldg(&libm_sincos_tab_dev[i])
#else
#define LM_FMA(a, b, c) fma((a), (b), (c))
#define LM_MUL(a, b) ((a) * (b))
#define LM_ADD(a, b) ((a) + (b))
#define LM_SUB(a, b) ((a) - (b))
#define LM_TAB(i) libm_sincos_tab_host[i]
#endif

// the largest |x| the restated branches serve: 0x1.921fbp+26 ~ 2^26 pi/2
#define LIBM_SINCOS_MAX 105414336.0

FNEC_LIBM_FN uint64_t lm_bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}

FNEC_LIBM_FN double lm_copysign(double a, double b) {
#ifdef __CUDA_ARCH__
    return copysign(a, b);
#else
    return copysign(a, b);
#endif
}

// polynomial coefficients (usncs.h)
#define LM_S1 (-0.16666666666666666)
#define LM_S2 0.0083333333333323288
#define LM_S3 (-0.00019841269834414642)
#define LM_S4 2.755729806860771e-06
#define LM_S5 (-2.5022014848318398e-08)
#define LM_SN3 (-1.66666666666664880952546298448555E-01)
#define LM_SN5 8.33333214285722277379541354343671E-03
#define LM_CS2 4.99999999999999999999950396842453E-01
#define LM_CS4 (-4.16666666666664434524222570944589E-02)
#define LM_CS6 1.38888874007937613028114285595617E-03
// 1.5 * 2^45: adding it rounds to a multiple of 1/128
#define LM_BIG 52776558133248.0
// pi/2 = hp0 + hp1
#define LM_HP0 0x1.921fb54442d18p+0
#define LM_HP1 0x1.1a62633145c07p-54
// pi/2 = mp1 + mp2 + pp3 + pp4 (mp1, mp2 short enough for exact n * mp)
#define LM_MP1 0x1.921fb58p+0
#define LM_MP2 (-0x1.dde973cp-27)
#define LM_PP3 (-0x1.cb3b398p-55)
#define LM_PP4 (-0x1.d747f23e32ed7p-83)
#define LM_HPINV 0x1.45f306dc9c883p-1
#define LM_TOINT 6755399441055744.0

// sin(a + da) for |a| < 0.126: odd Taylor polynomial
FNEC_LIBM_FN double lm_taylor_sin(double xx, double a, double da) {
    double p = LM_FMA(LM_S5, xx, LM_S4);
    p = LM_FMA(p, xx, LM_S3);
    p = LM_FMA(p, xx, LM_S2);
    p = LM_FMA(p, xx, LM_S1);
    double q = LM_FMA(p, a, -LM_MUL(0.5, da));
    double t = LM_FMA(q, xx, da);
    return LM_ADD(a, t);
}

// sin(x + dx), |x| < 0.855469
FNEC_LIBM_FN double lm_do_sin(double x, double dx) {
    double xold = x;
    if (fabs(x) < 0.126) return lm_taylor_sin(LM_MUL(x, x), x, dx);
    if (x <= 0) dx = -dx;
    double ax = fabs(x);
    double u = LM_ADD(LM_BIG, ax);
    x = LM_SUB(ax, LM_SUB(u, LM_BIG));
    int k = (int)(lm_bits(u) & 0xffffffffu) << 2;
    double xx = LM_MUL(x, x);
    double s = LM_ADD(x, LM_FMA(LM_MUL(x, xx), LM_FMA(xx, LM_SN5, LM_SN3), dx));
    double c = LM_FMA(x, dx, LM_MUL(xx, LM_FMA(xx, LM_FMA(xx, LM_CS6, LM_CS4), LM_CS2)));
    double sn = LM_TAB(k), ssn = LM_TAB(k + 1), cs = LM_TAB(k + 2), ccs = LM_TAB(k + 3);
    double cor = LM_FMA(s, ccs, ssn);
    cor = LM_FMA(-sn, c, cor);
    cor = LM_FMA(cs, s, cor);
    return lm_copysign(LM_ADD(sn, cor), xold);
}

// cos(x + dx), |x| < 0.855469
FNEC_LIBM_FN double lm_do_cos(double x, double dx) {
    if (x < 0) dx = -dx;
    double ax = fabs(x);
    double u = LM_ADD(LM_BIG, ax);
    x = LM_ADD(LM_SUB(ax, LM_SUB(u, LM_BIG)), dx);
    int k = (int)(lm_bits(u) & 0xffffffffu) << 2;
    double xx = LM_MUL(x, x);
    double s = LM_FMA(LM_MUL(x, xx), LM_FMA(xx, LM_SN5, LM_SN3), x);
    double c = LM_MUL(xx, LM_FMA(xx, LM_FMA(xx, LM_CS6, LM_CS4), LM_CS2));
    double sn = LM_TAB(k), ssn = LM_TAB(k + 1), cs = LM_TAB(k + 2), ccs = LM_TAB(k + 3);
    double cor = LM_FMA(-s, ssn, ccs);
    cor = LM_FMA(-cs, c, cor);
    cor = LM_FMA(-sn, s, cor);
    return LM_ADD(cs, cor);
}

// x - n*pi/2 as a + da; returns n mod 4
FNEC_LIBM_FN int lm_reduce(double x, double *a, double *da) {
    double t = LM_FMA(x, LM_HPINV, LM_TOINT);
    double xn = LM_SUB(t, LM_TOINT);
    double y = LM_FMA(-xn, LM_MP2, LM_FMA(-xn, LM_MP1, x));
    int n = (int)(lm_bits(t) & 3u);
    double t2 = LM_FMA(-xn, LM_PP3, y);
    double db = LM_FMA(-xn, LM_PP3, LM_SUB(y, t2));
    double b = LM_FMA(-xn, LM_PP4, t2);
    db = LM_ADD(db, LM_FMA(-xn, LM_PP4, LM_SUB(t2, b)));
    *a = b;
    *da = db;
    return n;
}

FNEC_LIBM_FN double lm_do_sincos(double a, double da, int n) {
    double r = (n & 1) ? lm_do_cos(a, da) : lm_do_sin(a, da);
    return (n & 2) ? -r : r;
}

// f64::sin on linux-gnu
FNEC_LIBM_FN double libm_sin(double x) {
    uint32_t k = (uint32_t)(lm_bits(x) >> 32) & 0x7fffffffu;
    if (k < 0x3e500000u) return x;
    if (k < 0x3feb6000u) return lm_do_sin(x, 0.0);
    if (k < 0x400368fdu) {
        double t = LM_SUB(LM_HP0, fabs(x));
        return lm_copysign(lm_do_cos(t, LM_HP1), x);
    }
    if (k < 0x419921fbu) {
        double a, da;
        int n = lm_reduce(x, &a, &da);
        return lm_do_sincos(a, da, n);
    }
    return x - x + NAN;  // outside the restated range (or inf/nan)
}

// f64::cos on linux-gnu
FNEC_LIBM_FN double libm_cos(double x) {
    uint32_t k = (uint32_t)(lm_bits(x) >> 32) & 0x7fffffffu;
    if (k < 0x3e400000u) return 1.0;
    if (k < 0x3feb6000u) return lm_do_cos(x, 0.0);
    if (k < 0x400368fdu) {
        double y = LM_SUB(LM_HP0, fabs(x));
        double a = LM_ADD(y, LM_HP1);
        double da = LM_ADD(LM_SUB(y, a), LM_HP1);
        return lm_do_sin(a, da);
    }
    if (k < 0x419921fbu) {
        double a, da;
        int n = lm_reduce(x, &a, &da);
        return lm_do_sincos(a, da, n + 1);
    }
    return x - x + NAN;
}

// (libm_sin(x), libm_cos(x)) with the branch and the reduction shared:
// glibc's sincos returns the same two values as sin and cos.  Every branch
// evaluates one do_sin and one do_cos; only their arguments differ, so the
// branch picks arguments and the two evaluations run once for all lanes of
// a warp whose arguments fall in different branches.
FNEC_LIBM_FN void libm_sincos(double x, double *s, double *c) {
    uint32_t k = (uint32_t)(lm_bits(x) >> 32) & 0x7fffffffu;
    double as, das, ac, dac;
    int mode, n = 0;
    if (k < 0x3feb6000u) {  // |x| < 0.855469: the table around x itself
        as = ac = x;
        das = dac = 0.0;
        mode = 0;
    } else if (k < 0x400368fdu) {  // |x| < 2.426265: taken from pi/2
        double y = LM_SUB(LM_HP0, fabs(x));
        ac = y;  // sin x = copysign(cos(y + hp1), x)
        dac = LM_HP1;
        as = LM_ADD(y, LM_HP1);  // cos x = sin(a + da)
        das = LM_ADD(LM_SUB(y, as), LM_HP1);
        mode = 1;
    } else if (k < 0x419921fbu) {  // x - n pi/2
        double a, da;
        n = lm_reduce(x, &a, &da);
        as = ac = a;
        das = dac = da;
        mode = 2;
    } else {
        *s = *c = x - x + NAN;
        return;
    }
    const double sp = lm_do_sin(as, das), cp = lm_do_cos(ac, dac);
    if (mode == 0) {
        *s = k < 0x3e500000u ? x : sp;
        *c = k < 0x3e400000u ? 1.0 : cp;
    } else if (mode == 1) {
        *s = lm_copysign(cp, x);
        *c = sp;
    } else {
        double sv = (n & 1) ? cp : sp, cv = (n & 1) ? sp : cp;
        *s = (n & 2) ? -sv : sv;
        *c = ((n + 1) & 2) ? -cv : cv;
    }
}

// f64::hypot on linux-gnu: glibc 2.35+ sysdeps/ieee754/dbl-64/e_hypot.c
// (Borges, "An Improved Algorithm for hypot(a, b)", the variant without
// FMA, which is what x86-64 builds of glibc run): the rounded sqrt of
// ax^2 + ay^2 followed by one correction step from the exact residual
// terms, with power-of-two scaling near overflow and underflow.  num-complex
// takes Complex64::norm from it, and the reference's pivot search compares
// those norms (linear.rs:1343-1352).
FNEC_LIBM_FN double lm_hypot_kernel(double ax, double ay) {
#ifdef __CUDA_ARCH__
    double h = __dsqrt_rn(LM_ADD(LM_MUL(ax, ax), LM_MUL(ay, ay)));
#else
    double h = sqrt(LM_ADD(LM_MUL(ax, ax), LM_MUL(ay, ay)));
#endif
    double t1, t2;
    if (h <= LM_MUL(2.0, ay)) {
        double delta = LM_SUB(h, ay);
        t1 = LM_MUL(ax, LM_SUB(LM_MUL(2.0, delta), ax));
        t2 = LM_MUL(LM_SUB(delta, LM_MUL(2.0, LM_SUB(ax, ay))), delta);
    } else {
        double delta = LM_SUB(h, ax);
        t1 = LM_MUL(LM_MUL(2.0, delta), LM_SUB(ax, LM_MUL(2.0, ay)));
        t2 = LM_ADD(LM_MUL(LM_SUB(LM_MUL(4.0, delta), ay), ay), LM_MUL(delta, delta));
    }
#ifdef __CUDA_ARCH__
    return LM_SUB(h, __ddiv_rn(LM_ADD(t1, t2), LM_MUL(2.0, h)));
#else
    return LM_SUB(h, LM_ADD(t1, t2) / LM_MUL(2.0, h));
#endif
}

FNEC_LIBM_FN double libm_hypot(double x, double y) {
    if (!isfinite(x) || !isfinite(y)) {
        if (isinf(x) || isinf(y)) return INFINITY;
        return x + y;
    }
    x = fabs(x);
    y = fabs(y);
    double ax = x < y ? y : x;
    double ay = x < y ? x : y;
    if (ax > 0x1p+511) {
        if (ay <= LM_MUL(ax, 0x1p-54)) return LM_ADD(ax, ay);
        return LM_MUL(lm_hypot_kernel(LM_MUL(ax, 0x1p-600), LM_MUL(ay, 0x1p-600)), 0x1p+600);
    }
    if (ay < 0x1p-459) {
        if (ax >= LM_MUL(ay, 0x1p+54)) return LM_ADD(ax, ay);
        return LM_MUL(lm_hypot_kernel(LM_MUL(ax, 0x1p+600), LM_MUL(ay, 0x1p+600)), 0x1p-600);
    }
    if (ay <= LM_MUL(ax, 0x1p-54)) return LM_ADD(ax, ay);
    return lm_hypot_kernel(ax, ay);
}

}  // namespace fnec_libm

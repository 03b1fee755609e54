// fnec_sincospi.cuh -- sin(pi x), cos(pi x) from a quadrant reduction and
// Taylor series, and 1/sqrt(x) by Newton's iteration (host and device), for
// the FMA-contracted kernels whose phases and distances need about 1e-16
// relative accuracy but not a particular libm's bits.
#pragma once
#include <cmath>
#include <cstring>

namespace fnec {

// sin(pi x) and cos(pi x) for 0 <= x < 2^50 (the phases of the mixed fill's
// samples and of the far field's wire runs).  Quadrant reduction in half-turns: adding 1.5 * 2^52 rounds 2x
// to the integer n (its low bits are n), and f = x - n / 2 is exact with
// |f| <= 1/4; then the Taylor series of sin and cos at theta = pi f
// (|theta| <= pi/4) to theta^15 and theta^16, whose truncation error is
// below 5e-17, in Horner form in theta^2, and the quadrant n mod 4 swaps
// and signs the pair.  About 22 FP64 operations and no table.
__host__ __device__ __forceinline__ void sincospi_taylor(double x, double &sn, double &cs) {
    const double big = 6755399441055744.0;  // 1.5 * 2^52
    const double t = fma(x, 2.0, big);
    const double nd = t - big;
#ifdef __CUDA_ARCH__
    const int q = __double2loint(t) & 3;
#else
    long long bits;
    memcpy(&bits, &t, sizeof(bits));
    const int q = (int)(bits & 3);
#endif
    const double th = fma(nd, -0.5, x) * 3.141592653589793;
    const double t2 = th * th;
    // sin: theta (1 + t2 (-1/3! + t2 (1/5! - ... - t2 / 15!)))
    double ps = -7.647163731819816e-13;  // -1/15!
    ps = fma(ps, t2, 1.6059043836821613e-10);   // 1/13!
    ps = fma(ps, t2, -2.505210838544172e-08);   // -1/11!
    ps = fma(ps, t2, 2.7557319223985893e-06);   // 1/9!
    ps = fma(ps, t2, -0.0001984126984126984);   // -1/7!
    ps = fma(ps, t2, 0.008333333333333333);    // 1/5!
    ps = fma(ps, t2, -0.16666666666666666);  // -1/3!
    const double s0 = fma(th * t2, ps, th);
    // cos: 1 + t2 (-1/2! + t2 (1/4! - ... + t2 / 16!))
    double pc = 4.779477332387385e-14;  // 1/16!
    pc = fma(pc, t2, -1.1470745597729725e-11);  // -1/14!
    pc = fma(pc, t2, 2.08767569878681e-09);     // 1/12!
    pc = fma(pc, t2, -2.755731922398589e-07);   // -1/10!
    pc = fma(pc, t2, 2.48015873015873e-05);     // 1/8!
    pc = fma(pc, t2, -0.001388888888888889);  // -1/6!
    pc = fma(pc, t2, 0.041666666666666664);   // 1/4!
    pc = fma(pc, t2, -0.5);                     // -1/2!
    const double c0 = fma(t2, pc, 1.0);
    const double a = (q & 1) ? c0 : s0, b = (q & 1) ? s0 : c0;
    sn = (q & 2) ? -a : a;
    cs = ((q + 1) & 2) ? -b : b;
}

// 1/sqrt(x) for normal, finite x > 0: a single-precision first guess
// (about 23 correct bits; the device's approximate reciprocal square root),
// then two Newton steps for f(y) = y^-2 - x in FP64,
// y <- y + (y / 2)(1 - x y^2), each doubling the correct bits: within about
// 3e-16 relative of the true value over the fill's range (R^2 from 1e-8 to
// 1e4 m^2).  Nine FP64 / conversion operations and no branch.
__host__ __device__ __forceinline__ double rsqrt_newton(double x) {
#ifdef __CUDA_ARCH__
    double y = (double)rsqrtf((float)x);
#else
    double y = (double)(1.0f / std::sqrt((float)x));
#endif
    double e = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, e, y);
    e = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, e, y);
    return y;
}

// Either sign: sin(pi x) is odd, cos(pi x) even.
__host__ __device__ __forceinline__ void sincospi_taylor_signed(double x, double &sn, double &cs) {
    sincospi_taylor(fabs(x), sn, cs);
    if (x < 0.0) sn = -sn;
}

}  // namespace fnec

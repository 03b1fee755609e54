// fnec_math.cuh -- exact-parity arithmetic for the Hallen kernels.
//
// Complex arithmetic with the exact operation order of num-complex 0.4.6
// and no FMA contraction (explicit _rn intrinsics on the device), so sums
// and eliminations reproduce the reference bit for bit.  The libm functions
// the reference calls (sin, cos, hypot) are restated in fnec_libm.cuh.
//
// The header compiles as CUDA device code under nvcc and as plain C++ under
// g++ (host unit tests).
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fnec_libm.cuh"

#ifdef __CUDACC__
#define FNEC_FN __device__ __forceinline__
#define D_ADD(a, b) __dadd_rn((a), (b))
#define D_SUB(a, b) __dsub_rn((a), (b))
#define D_MUL(a, b) __dmul_rn((a), (b))
#define D_DIV(a, b) __ddiv_rn((a), (b))
#define D_SQRT(a) __dsqrt_rn((a))
#else
#define FNEC_FN static inline
#define D_ADD(a, b) ((a) + (b))
#define D_SUB(a, b) ((a) - (b))
#define D_MUL(a, b) ((a) * (b))
#define D_DIV(a, b) ((a) / (b))
#define D_SQRT(a) sqrt((a))
#endif

namespace fnec {

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
// Complex64::norm = f64::hypot, as the platform libm evaluates it
FNEC_FN double cx_norm(cx a) { return fnec_libm::libm_hypot(a.re, a.im); }
FNEC_FN double cx_norm_sqr(cx a) { return D_ADD(D_MUL(a.re, a.re), D_MUL(a.im, a.im)); }

}  // namespace fnec

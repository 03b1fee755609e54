// Host build of the correctly rounded functions in fnec_math.cuh, exported
// for the CPU unit test (tests/test_cr_math.py) that compares them against
// 256-bit mpmath values.  Not part of libfnec_cuda.so.
#include "fnec_math.cuh"

extern "C" {
void probe_sincos(const double *x, double *s, double *c, long n) {
    for (long i = 0; i < n; ++i) fnec::cr_sincos(x[i], &s[i], &c[i]);
}
void probe_log(const double *x, double *y, long n) {
    for (long i = 0; i < n; ++i) y[i] = fnec::cr_log(x[i]);
}
void probe_hypot(const double *a, const double *b, double *y, long n) {
    for (long i = 0; i < n; ++i) y[i] = fnec::cr_hypot(a[i], b[i]);
}
}

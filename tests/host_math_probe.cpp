// Host build of the libm restatement in fnec_libm.cuh (the sin, cos and
// hypot the exact-parity kernels evaluate), exported for the CPU unit test
// tests/test_libm_restatement.py, which compares it bit for bit with the
// host's own libm -- the library the reference's f64 methods call on
// linux-gnu.  Test infrastructure; not part of libfnec_cuda.so.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fnec_libm.cuh"

static uint64_t bits(double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
}

extern "C" {
// the restatement's values
void probe_libm_sincos(const double *x, double *s, double *c, long n) {
    for (long i = 0; i < n; ++i) fnec_libm::libm_sincos(x[i], &s[i], &c[i]);
}
void probe_libm_hypot(const double *a, const double *b, double *y, long n) {
    for (long i = 0; i < n; ++i) y[i] = fnec_libm::libm_hypot(a[i], b[i]);
}
// the host libm's values
void probe_host_sincos(const double *x, double *s, double *c, long n) {
    for (long i = 0; i < n; ++i) {
        s[i] = sin(x[i]);
        c[i] = cos(x[i]);
    }
}
void probe_host_hypot(const double *a, const double *b, double *y, long n) {
    for (long i = 0; i < n; ++i) y[i] = hypot(a[i], b[i]);
}
// arguments where the restatement and the host libm differ in any bit
// (sin, cos, libm_sincos and the separate libm_sin / libm_cos); returns the
// count and stores up to cap of them in bad
long probe_sincos_mismatches(const double *x, long n, double *bad, long cap) {
    long k = 0;
    for (long i = 0; i < n; ++i) {
        double s, c;
        fnec_libm::libm_sincos(x[i], &s, &c);
        bool ok = bits(s) == bits(sin(x[i])) && bits(c) == bits(cos(x[i])) &&
                  bits(fnec_libm::libm_sin(x[i])) == bits(s) && bits(fnec_libm::libm_cos(x[i])) == bits(c);
        if (!ok) {
            if (k < cap) bad[k] = x[i];
            ++k;
        }
    }
    return k;
}
long probe_hypot_mismatches(const double *a, const double *b, long n, long *bad, long cap) {
    long k = 0;
    for (long i = 0; i < n; ++i)
        if (bits(fnec_libm::libm_hypot(a[i], b[i])) != bits(hypot(a[i], b[i]))) {
            if (k < cap) bad[k] = i;
            ++k;
        }
    return k;
}
}

// fnec_mixed.cu -- the chosen form: FP32 normal equations + FP32 GEPP as a
// preconditioner, FP64 GMRES iterative refinement on the true system.
//
// The answer is the same as the plain path's -- the solution of the
// regularised normal equations (M^H M + 1e-8 I) x = M^H y of
// linear.rs:672-797 -- but only the preconditioner is formed in FP32:
//
//   fill      FP64 (hardware sincos/log, FMA): Z must be FP64 because the
//             refinement residual is formed from it
//   Gram      A32 = fl32(M^H M) + lambda I, complex64 with FMA
//   factor    complex64 GEPP (full-row swaps, so P A32 = L U is reusable)
//   refine    GMRES(24) in FP64, left-preconditioned by (L U)^-1 P, with
//             matrix-vector products A v = M^H (M v) + lambda v taken from
//             the FP64 Z and the sparse cos / constraint columns -- the
//             residual of the regularised system itself
//
// cond(A) reaches 3e8 for the 5-wire array, so classical refinement with an
// FP32 factor (u32 * cond ~ 18) diverges; preconditioned GMRES converges in
// a handful of iterations because the FP32 factor's errors concentrate in
// few directions.  The error against the FP64 oracle is reported per unit
// (iterations and final residual are kept for inspection).
#include <algorithm>
#include <cstring>
#include <climits>
#include <vector>

#include "fnec_grid.cuh"
#include "fnec_mixed.h"
#include "fnec_sincospi.cuh"
#include "fnec_tc.h"

namespace fnec {

namespace {

constexpr int MNB = 32;          // FP32 panel width
constexpr int GM = 24;           // GMRES Krylov vectors per cycle
constexpr int MAX_OUTER = 4;     // GMRES cycles
// Stop when the preconditioned residual is 1e-9 of |P^-1 b|: the feedpoint
// then sits ~1e-8 from the FP64 oracle, 100x inside the 1e-6 gate.
constexpr double GMRES_TOL = 1e-9;

__device__ __forceinline__ float2 cf(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 cf_mul(float2 a, float2 b) {
    return cf(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cf_sub(float2 a, float2 b) { return cf(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cf_add(float2 a, float2 b) { return cf(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cf_div(float2 a, float2 b) {
    float inv = 1.0f / (b.x * b.x + b.y * b.y);
    return cf((a.x * b.x + a.y * b.y) * inv, (a.y * b.x - a.x * b.y) * inv);
}
// (fast FP64 complex, FMA allowed)
__device__ __forceinline__ cx zmul(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cx zcmul(cx a, cx b) { return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re}; }
__device__ __forceinline__ cx zadd(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cx zsub(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cx zscale(cx a, double s) { return {a.re * s, a.im * s}; }
// One Z entry as a single 16-byte read-only load (Z is read-only after the
// fill and its entries are 16-byte aligned); the struct's own copy would
// issue two 8-byte loads.
__device__ __forceinline__ cx ld_z(const cx *p) {
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return {v.x, v.y};
}
__device__ __forceinline__ cx zdiv(cx a, cx b) {
    double inv = 1.0 / (b.re * b.re + b.im * b.im);
    return {(a.re * b.re + a.im * b.im) * inv, (a.im * b.re - a.re * b.im) * inv};
}

__constant__ double m_gl_n4[4] = {-0.861136311594953, -0.339981043584856, 0.339981043584856,
                                  0.861136311594953};
__constant__ double m_gl_w4[4] = {0.347854845137454, 0.652145154862626, 0.652145154862626,
                                  0.347854845137454};
__constant__ double m_gl_n8[8] = {-0.960289856497536, -0.796666477413627, -0.525532409916329,
                                  -0.183434642495650, 0.183434642495650,  0.525532409916329,
                                  0.796666477413627,  0.960289856497536};
__constant__ double m_gl_w8[8] = {0.101228536290376, 0.222381034453374, 0.313706645877887,
                                  0.362683783378362, 0.362683783378362, 0.313706645877887,
                                  0.222381034453374, 0.101228536290376};

// ---------------------------------------------------------------------------
// fast FP64 fill (matrix.rs:297-331 with hardware sincos/log and FMA)
// ---------------------------------------------------------------------------
// Z element (obs midpoint om, source segment mid sm / unit direction sd /
// length slen / radius srad); the far form takes the midpoint difference
// d = om - sm and the half-length step hs = sd slen / 2 once per element,
// then per Gauss-Legendre sample r = d - x_m hs, R^2 = |r|^2 + a^2, one
// reciprocal square root (rsqrt_newton) for R and 1/R and
// sincospi_taylor(k R / pi).
__device__ __forceinline__ cx elem_fast(const double *om, const double *od, const double *sm, const double *sd,
                                        double slen, double srad, double k, bool is_self) {
    double cos_alpha = od[0] * sd[0] + od[1] * sd[1] + od[2] * sd[2];
    double half = slen * 0.5, a = srad;
    double ire = 0.0, iim = 0.0;
    if (is_self) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            double l = m_gl_n4[m] * half;
            double r = sqrt(l * l + a * a);
            double sn, cs;
            sincos(-k * r, &sn, &cs);
            double inv = 1.0 / r;
            ire += m_gl_w4[m] * (cs * inv - inv);
            iim += m_gl_w4[m] * (sn * inv);
        }
        ire *= half;
        iim *= half;
        double r_end = sqrt(half * half + a * a);
        ire += 2.0 * log((half + r_end) / a);
    } else {
        const double kpi = k * 0.31830988618379067;  // k / pi
        const double d0 = om[0] - sm[0], d1 = om[1] - sm[1], d2 = om[2] - sm[2];
        const double h0 = sd[0] * half, h1 = sd[1] * half, h2 = sd[2] * half;
        const double a2 = a * a;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const double xm = m_gl_n8[m];
            const double r0 = fma(-xm, h0, d0), r1 = fma(-xm, h1, d1), r2 = fma(-xm, h2, d2);
            const double r2s = fma(r0, r0, fma(r1, r1, fma(r2, r2, a2)));
            const double inv = rsqrt_newton(r2s);
            double sn, cs;
            sincospi_taylor(kpi * (r2s * inv), sn, cs);
            const double wr = m_gl_w8[m] * inv;
            ire = fma(wr, cs, ire);
            iim = fma(-wr, sn, iim);  // e^{-jkR}
        }
        ire *= half;
        iim *= half;
    }
    return {ire * cos_alpha, iim * cos_alpha};
}

// One CTA of 256 threads fills a 16x16 tile of one unit's Z.  With gu set
// it also writes the tile into the tensor-core Gram's operand stacks --
// T[2c+s][k] = (Re, Im) Z[k][c] as tf32 hi/lo pairs, K-blocked (k_split_gram's
// layout and rounding) -- through a shared-memory transpose, so the Gram
// does not read Z back for them.  The stacks' padding is zero from their
// allocation and never written.
__global__ void __launch_bounds__(256, 4) k_fill_fast(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                                                   const DevSeg *__restrict__ segs, const int4 *__restrict__ tiles,
                                                   cx *zbuf, const TcGramUnit *__restrict__ gu, float *ghi,
                                                   float *glo) {
    // the tile's segments field by field (structure of arrays): a warp's 16
    // source lanes read 16 consecutive doubles, one conflict-free wavefront
    __shared__ double s_o[6][16];  // observation midpoint, direction
    __shared__ double s_s[8][16];  // source midpoint, direction, length, radius
    __shared__ cx s_z[16][17];
    int4 t = tiles[blockIdx.x];
    UnitDesc u = units[t.x];
    AntDesc a = ants[u.ant];
    int n = a.n;
    const DevSeg *sg = segs + a.seg_off;
    int tid = threadIdx.x;
    if (tid < 6 * 16) {
        const int q = tid / 6, f = tid % 6;
        const DevSeg *g = sg + min(t.y + q, n - 1);
        s_o[f][q] = f < 3 ? g->mid[f] : g->dir[f - 3];
    } else if (tid < 6 * 16 + 8 * 16) {
        const int q = (tid - 96) / 8, f = (tid - 96) % 8;
        const DevSeg *g = sg + min(t.z + q, n - 1);
        s_s[f][q] = f < 3 ? g->mid[f] : (f < 6 ? g->dir[f - 3] : (f == 6 ? g->len : g->rad));
    }
    __syncthreads();
    int ii = tid / 16, jj = tid % 16;
    int i = t.y + ii, j = t.z + jj;
    if (i < n && j < n) {
        const double om[3] = {s_o[0][ii], s_o[1][ii], s_o[2][ii]}, od[3] = {s_o[3][ii], s_o[4][ii], s_o[5][ii]};
        const double sm[3] = {s_s[0][jj], s_s[1][jj], s_s[2][jj]}, sd[3] = {s_s[3][jj], s_s[4][jj], s_s[5][jj]};
        const double slen = s_s[6][jj], srad = s_s[7][jj];
        cx z = elem_fast(om, od, sm, sd, slen, srad, u.k_fill, i == j);
        if (a.ground == 1) {
            const double im_mid[3] = {sm[0], sm[1], -sm[2]};
            const double im_dir[3] = {-sd[0], -sd[1], sd[2]};
            cx g = elem_fast(om, od, im_mid, im_dir, slen, srad, u.k_fill, false);
            z = zadd(z, g);
        }
        zbuf[u.z_off + (int64_t)i * n + j] = z;
        s_z[ii][jj] = z;
    }
    if (!gu) return;  // block-uniform
    __syncthreads();
    const TcGramUnit g = gu[t.x];
    // 32 stack rows (2 jj + s) of 16 consecutive k = t.y + kk each
#pragma unroll
    for (int e = tid; e < 32 * 16; e += 256) {
        const int rr = e / 16, kk = e % 16;
        const int jc = t.z + rr / 2, ik = t.y + kk;
        if (ik >= n || jc >= n) continue;
        const cx v = s_z[kk][rr / 2];
        float h, l;
        split_tf32((float)((rr & 1) ? v.im : v.re), h, l);
        const int64_t o = ((int64_t)g.base + (int64_t)(ik / 32) * g.rpad + 2 * jc + (rr & 1)) * 32 + (ik % 32);
        ghi[o] = h;
        glo[o] = l;
    }
}

// ---------------------------------------------------------------------------
// FP32 normal equations A32 = M^H M + lambda I (S x S, row stride S)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_gram32_zz(const UnitDesc *__restrict__ units, const MixedUnit *__restrict__ mus,
                                                   const int4 *__restrict__ tiles, const cx *__restrict__ zbuf,
                                                   float2 *a32buf) {
    __shared__ float2 s_l[16][64];
    __shared__ float2 s_r[16][65];
    int4 t = tiles[blockIdx.x];
    UnitDesc u = units[t.x];
    int n = u.n, s = u.s;
    int i0 = t.y, j0 = t.z;
    if (j0 >= n) return;  // the RHS-column tile of the exact path
    const cx *z = zbuf + u.z_off;
    int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = cf(0.f, 0.f);
    for (int r0 = 0; r0 < n; r0 += 16) {
        for (int e = tid; e < 16 * 64; e += 256) {
            int rr = e / 64, cc = e % 64, r = r0 + rr;
            float2 lv = cf(0.f, 0.f), rv = cf(0.f, 0.f);
            if (r < n) {
                if (i0 + cc < n) {
                    cx v = z[(int64_t)r * n + i0 + cc];
                    lv = cf((float)v.re, (float)v.im);
                }
                if (j0 + cc < n) {
                    cx v = z[(int64_t)r * n + j0 + cc];
                    rv = cf((float)v.re, (float)v.im);
                }
            }
            s_l[rr][cc] = lv;
            s_r[rr][cc] = rv;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
            float2 lv[4], rv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) lv[a] = s_l[kk][ty + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) rv[b] = s_r[kk][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {  // conj(l) * r
                    acc[a][b].x = fmaf(lv[a].x, rv[b].x, fmaf(lv[a].y, rv[b].y, acc[a][b].x));
                    acc[a][b].y = fmaf(lv[a].x, rv[b].y, fmaf(-lv[a].y, rv[b].x, acc[a][b].y));
                }
        }
        __syncthreads();
    }
    float2 *A = a32buf + mus[t.x].a32_off;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int i = i0 + ty + 16 * a;
        if (i >= n) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int j = j0 + tx + 16 * b;
            if (j < n) A[(int64_t)i * s + j] = acc[a][b];
        }
    }
}

// cos columns (grid.x = wire column, grid.y = system)
__global__ void k_gram32_ccols(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                               const MixedUnit *__restrict__ mus, const int32_t *__restrict__ ibuf,
                               const cx *__restrict__ zbuf, const double *__restrict__ cos_buf, float2 *a32buf) {
    UnitDesc u = units[blockIdx.y];
    AntDesc a = ants[u.ant];
    int w = blockIdx.x;
    if (w >= a.w || mus[blockIdx.y].first_solve >= 0) return;  // the latter: k_gram32_ccols_mhy
    int n = u.n, s = u.s;
    const cx *z = zbuf + u.z_off;
    const double *cv = cos_buf + u.cos_off;
    const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
    float2 *A = a32buf + mus[blockIdx.y].a32_off;
    int b = wptr[w], e = wptr[w + 1];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double cr = 0, ci = 0;
        for (int q = b; q < e; ++q) {
            int r = wrow[q];
            cx zi = z[(int64_t)r * n + i];
            cr += -cv[r] * zi.re;
            ci += -cv[r] * zi.im;
        }
        A[(int64_t)i * s + n + w] = cf((float)cr, (float)-ci);   // conj(Z) * (-cos)
        A[(int64_t)(n + w) * s + i] = cf((float)cr, (float)ci);  // (-cos) * Z
    }
    for (int v = threadIdx.x; v < a.w; v += blockDim.x) {
        double d = 0;
        if (v == w)
            for (int q = b; q < e; ++q) d += cv[wrow[q]] * cv[wrow[q]];
        A[(int64_t)(n + w) * s + n + v] = cf((float)d, 0.f);
    }
}

// The cos columns of k_gram32_ccols and every solve's M^H y together, for
// a system of at most CM_MAX_W homogeneous columns and CM_MAX_RHS
// right-hand sides whose solves are consecutive (MixedUnit::first_solve,
// set at planning): one pass over Z instead of two, a thread per column c
// (grid.x: blocks of 256 columns, grid.y: system).  The thread walks the
// rows in order; the current wire's cos sum stays in registers and moves
// through shared memory when the wire changes, so each wire's sum runs
// over its rows in increasing order -- k_gram32_ccols's operations and
// order.  (M^H y)[c] = sum_r conj(Z[r][c]) y[r] runs in row order and the
// wire entries (M^H y)[n + q] over the wire's rows: the refinement
// kernel's own sums, written into each solve's work vector b, which the
// refinement then takes as it is.
// NRMAX: one instance for the systems of one right-hand side (the common
// case: fewer registers, so the next rows' loads fit beside the sums), one
// for 2 .. CM_MAX_RHS; each skips the other's systems.
constexpr int CM_MAX_W = 8, CM_MAX_RHS = 4;
template <int NRMAX>
__global__ void __launch_bounds__(256, 3) k_gram32_ccols_mhy(const UnitDesc *__restrict__ units,
                                                         const UnitDesc *__restrict__ solves,
                                                         const AntDesc *__restrict__ ants,
                                                         const MixedUnit *__restrict__ smu,
                                                         const MixedUnit *__restrict__ mus,
                                                         const int32_t *__restrict__ ibuf,
                                                         const cx *__restrict__ zbuf,
                                                         const double *__restrict__ cos_buf,
                                                         const cx *__restrict__ rhs, float2 *a32buf, cx *wbuf) {
    __shared__ cx s_acc[CM_MAX_W][256];
    const UnitDesc u = units[blockIdx.y];
    const int first = smu[blockIdx.y].first_solve;
    if (first < 0) return;
    const AntDesc a = ants[u.ant];
    const int n = u.n, s = u.s, W = a.w, nr = u.n_rhs;
    if ((NRMAX == 1) != (nr == 1)) return;  // the other instance's systems
    const int c0 = (int)blockIdx.x * 256;
    if (c0 >= n) return;
    const int tid = threadIdx.x, c = c0 + tid;
    const cx *z = zbuf + u.z_off;
    const double *cv = cos_buf + u.cos_off;
    const int32_t *rowwire = ibuf + a.rowwire_off;
    const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
    float2 *A = a32buf + smu[blockIdx.y].a32_off;
    const cx *y[NRMAX];
#pragma unroll
    for (int k = 0; k < NRMAX; ++k) y[k] = rhs + solves[first + min(k, nr - 1)].rhs_off;
    for (int w = 0; w < W; ++w) s_acc[w][tid] = {0, 0};  // a thread's own column: no barrier
    if (c < n) {
        cx bacc[NRMAX];
#pragma unroll
        for (int k = 0; k < NRMAX; ++k) bacc[k] = {0, 0};
        int cur = n > 0 ? rowwire[0] : 0;
        double cr = 0, ci = 0;
        constexpr int RB = 4;  // rows per batch; the next batch's loads are in flight meanwhile
        cx zb[RB], zn[RB];
#pragma unroll
        for (int j = 0; j < RB; ++j) zb[j] = j < n ? ld_z(z + (int64_t)j * n + c) : cx{0, 0};
        for (int r0 = 0; r0 < n; r0 += RB) {
#pragma unroll
            for (int j = 0; j < RB; ++j) {
                const int r = r0 + RB + j;
                zn[j] = r < n ? ld_z(z + (int64_t)r * n + c) : cx{0, 0};
            }
#pragma unroll
            for (int j = 0; j < RB; ++j) {
                const int r = r0 + j;
                if (r >= n) break;  // uniform over the block
                const int w = rowwire[r];
                if (w != cur) {  // uniform over the block
                    s_acc[cur][tid] = {cr, ci};
                    cur = w;
                    cr = s_acc[w][tid].re;
                    ci = s_acc[w][tid].im;
                }
                cr += -cv[r] * zb[j].re;
                ci += -cv[r] * zb[j].im;
#pragma unroll
                for (int k = 0; k < NRMAX; ++k)
                    if (k < nr) bacc[k] = zadd(bacc[k], zcmul(zb[j], y[k][r]));
            }
#pragma unroll
            for (int j = 0; j < RB; ++j) zb[j] = zn[j];
        }
        s_acc[cur][tid] = {cr, ci};
        for (int w = 0; w < W; ++w) {
            const cx v = s_acc[w][tid];
            A[(int64_t)c * s + n + w] = cf((float)v.re, (float)-v.im);   // conj(Z) * (-cos)
            A[(int64_t)(n + w) * s + c] = cf((float)v.re, (float)v.im);  // (-cos) * Z
        }
#pragma unroll
        for (int k = 0; k < NRMAX; ++k)
            if (k < nr) wbuf[mus[first + k].w_off + c] = bacc[k];
    }
    if (blockIdx.x == 0) {
        for (int e = tid; e < W * W; e += 256) {
            const int w = e / W, v = e % W;
            double d = 0;
            if (v == w)
                for (int q = wptr[w]; q < wptr[w + 1]; ++q) d += cv[wrow[q]] * cv[wrow[q]];
            A[(int64_t)(n + w) * s + n + v] = cf((float)d, 0.f);
        }
        for (int e = tid; e < nr * W; e += 256) {
            const int k = e / W, q = e % W;
            const cx *yk = rhs + solves[first + k].rhs_off;
            cx acc = {0, 0};
            for (int kk = wptr[q]; kk < wptr[q + 1]; ++kk) acc = zadd(acc, zscale(yk[wrow[kk]], -cv[wrow[kk]]));
            wbuf[mus[first + k].w_off + n + q] = acc;
        }
    }
}

// constraint rows (in row order) and lambda; one CTA per system
// Constraint rows and the regulariser: A[c][c'] += m_qc m_qc' over the
// constraint rows q touching column c (its CSR), then A[c][c] += 1e-8.
// One thread owns each row c of A, so the updates need no atomics.
__global__ void k_gram32_rest(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                              const MixedUnit *__restrict__ mus, const int32_t *__restrict__ ibuf,
                              const DevConRow *__restrict__ crows, float2 *a32buf) {
    UnitDesc u = units[blockIdx.x];
    AntDesc a = ants[u.ant];
    int s = u.s, n = u.n;
    float2 *A = a32buf + mus[blockIdx.x].a32_off;
    const DevConRow *cr = crows + a.crow_off;
    const int32_t *ccptr = ibuf + a.ccptr_off, *ccq = ibuf + a.ccq_off;
    for (int c = threadIdx.x; c < s; c += blockDim.x) {
        float2 *row = A + (int64_t)c * s;
        if (c < n)
            for (int k = ccptr[c]; k < ccptr[c + 1]; ++k) {
                DevConRow r = cr[ccq[k]];
                float v1 = (float)r.v1;
                float mc = (r.c0 == c ? 1.f : 0.f) + (r.c1 == c ? v1 : 0.f);
                row[r.c0].x += mc * (r.c1 == r.c0 ? 1.f + v1 : 1.f);
                if (r.c1 >= 0 && r.c1 != r.c0) row[r.c1].x += mc * v1;
            }
        row[c].x += 1e-8f;
    }
}

// ---------------------------------------------------------------------------
// complex64 GEPP (blocked, full-row swaps: P A32 = L U)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void piv_better32(float &bv, int &bi, float v, int i) {
    if (v > bv || (v == bv && i > bi)) {
        bv = v;
        bi = i;
    }
}

__global__ void __launch_bounds__(256) k_panel32(const UnitDesc *__restrict__ units, const MixedUnit *__restrict__ mus,
                                                 int c0, float2 *a32buf, int32_t *piv_buf, int32_t *status,
                                                 int skip_m, const int32_t *__restrict__ order, int base) {
    __shared__ float s_v[8];
    __shared__ int s_i[8];
    __shared__ int s_p;
    __shared__ float2 s_prow[MNB];
    int ui = order[base + blockIdx.x];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || s - c0 > skip_m || status[ui] != 0) return;  // skip_m: taller panels go grid-wide
    float2 *A = a32buf + mus[ui].a32_off;
    int32_t *piv = piv_buf + u.piv_off;
    int nb = min(MNB, s - c0);
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int c = c0; c < c0 + nb; ++c) {
        float bv = -1.f;
        int bi = -1;
        for (int r = c + tid; r < s; r += blockDim.x) {
            float2 v = A[(int64_t)r * s + c];
            piv_better32(bv, bi, v.x * v.x + v.y * v.y, r);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            float ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            piv_better32(bv, bi, ov, oi);
        }
        if (lane == 0) {
            s_v[wid] = bv;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            float v = s_v[0];
            int p = s_i[0];
            for (int q = 1; q < (int)(blockDim.x >> 5); ++q) piv_better32(v, p, s_v[q], s_i[q]);
            if (p < 0 || !(v > 0.f)) {
                status[ui] = -(c + 1);
                p = -1;
            }
            s_p = p;
            piv[c] = p;
        }
        __syncthreads();
        int p = s_p;
        if (p < 0) return;
        if (p != c && tid < nb) {
            int k = c0 + tid;
            float2 t0 = A[(int64_t)c * s + k];
            A[(int64_t)c * s + k] = A[(int64_t)p * s + k];
            A[(int64_t)p * s + k] = t0;
        }
        __syncthreads();
        if (tid < nb) s_prow[tid] = A[(int64_t)c * s + c0 + tid];
        __syncthreads();
        float2 diag = s_prow[c - c0];
        for (int r = c + 1 + tid; r < s; r += blockDim.x) {
            float2 *row = A + (int64_t)r * s;
            float2 f = cf_div(row[c], diag);
            row[c] = f;
            for (int k = c + 1; k < c0 + nb; ++k) row[k] = cf_sub(row[k], cf_mul(f, s_prow[k - c0]));
        }
        __syncthreads();
    }
}

// The FP32 panel held in shared memory (rows c0..s-1, MNB columns).
constexpr int PANEL32_SMEM_MAX = 200 * 1024;

// The FP32 panel of one unit (rows c0..s-1, MNB columns) factored from
// shared memory by a CTA of NT threads: pivot search, row swap, and
// elimination with the pivot's reciprocal, a warp per row.  The next
// column's pivot search is folded into each elimination pass (the tie rule
// is order-free).  Writes the panel and its pivots back to global memory;
// returns false (with the unit's status set) for a singular panel.
template <int NT>
__device__ bool panel32_body(float2 *A, int s, int c0, int32_t *piv, int32_t *status_u, float2 *s_pan32,
                             float *s_v, int *s_i, int *s_p) {
    // panel rows padded to PS = MNB + 1 entries: a column read by consecutive
    // rows then falls on distinct banks
    constexpr int PS = MNB + 1;
    constexpr int nw = NT / 32;
    int nb = min(MNB, s - c0), m = s - c0;
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int e = tid; e < m * nb; e += NT) {
        int rr = e / nb, q = e % nb;
        s_pan32[rr * PS + q] = A[(int64_t)(c0 + rr) * s + c0 + q];
    }
    __syncthreads();
    float bv = -1.f;
    int bi = -1;
    for (int r = c0 + tid; r < s; r += NT) {
        float2 v = s_pan32[(r - c0) * PS];
        piv_better32(bv, bi, v.x * v.x + v.y * v.y, r);
    }
    for (int c = c0; c < c0 + nb; ++c) {
        int lc = c - c0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            float ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            piv_better32(bv, bi, ov, oi);
        }
        if (lane == 0) {
            s_v[wid] = bv;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (wid == 0) {  // the per-warp candidates, reduced by warp 0
            float v = lane < nw ? s_v[lane] : -1.f;
            int p = lane < nw ? s_i[lane] : -1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                float ov = __shfl_down_sync(0xffffffffu, v, o);
                int oi = __shfl_down_sync(0xffffffffu, p, o);
                piv_better32(v, p, ov, oi);
            }
            if (lane == 0) {
                if (p < 0 || !(v > 0.f)) {
                    *status_u = -(c + 1);
                    p = -1;
                }
                *s_p = p;
                piv[c] = p;
            }
        }
        __syncthreads();
        int p = *s_p;
        if (p < 0) return false;
        if (p != c && tid < nb) {
            float2 t0 = s_pan32[lc * PS + tid];
            s_pan32[lc * PS + tid] = s_pan32[(p - c0) * PS + tid];
            s_pan32[(p - c0) * PS + tid] = t0;
        }
        __syncthreads();
        const float2 *prow = s_pan32 + lc * PS;  // the pivot row, read by broadcast
        const float2 diag = prow[lc];
        const float dn = 1.0f / (diag.x * diag.x + diag.y * diag.y);
        const float2 dinv = cf(diag.x * dn, -diag.y * dn);
        const int nx = lc + 1;
        bv = -1.f;
        bi = -1;
        // a thread per row: its multiplier, then its remaining panel entries
        // in column order (the row's entries sit 33 float2 apart from the
        // next row's, an odd stride: a warp's accesses are conflict-free)
        for (int r = c + 1 + tid; r < s; r += NT) {
            float2 *row = s_pan32 + (r - c0) * PS;
            const float2 f = cf_mul(row[lc], dinv);
            row[lc] = f;
            for (int k = lc + 1; k < nb; ++k) row[k] = cf_sub(row[k], cf_mul(f, prow[k]));
            if (nx < nb) {
                const float2 y = row[nx];
                piv_better32(bv, bi, y.x * y.x + y.y * y.y, r);
            }
        }
        // no barrier here: the next column's first barrier orders these
        // writes before its swap, and s_v is rewritten only after this
        // column's reads of it
    }
    __syncthreads();
    for (int e = tid; e < m * nb; e += NT) {
        int rr = e / nb, q = e % nb;
        A[(int64_t)(c0 + rr) * s + c0 + q] = s_pan32[rr * PS + q];
    }
    return true;
}

// The panel step of every unit of a size class, one CTA of NT threads per
// unit: 256, or 1024 for tall panels (fewer rows per warp on the
// column-serial critical path of the largest units).
template <int NT>
__global__ void __launch_bounds__(NT) k_panel32_smem(const UnitDesc *__restrict__ units,
                                                     const MixedUnit *__restrict__ mus, int c0, float2 *a32buf,
                                                     int32_t *piv_buf, int32_t *status, int skip_m, const int32_t *__restrict__ order, int base) {
    extern __shared__ float2 s_pan32[];
    __shared__ float s_v[NT / 32];
    __shared__ int s_i[NT / 32];
    __shared__ int s_p;
    int ui = order[base + blockIdx.x];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || s - c0 > skip_m || status[ui] != 0) return;  // skip_m: taller panels go grid-wide
    panel32_body<NT>(a32buf + mus[ui].a32_off, s, c0, piv_buf + u.piv_off, &status[ui], s_pan32, s_v, s_i, &s_p);
}

// The whole FP32 blocked GEPP of one small unit (S <= fu_max_s(level)) per CTA:
// the panel, swap/U12 and trailing steps of the per-step kernels
// (k_panel32_smem, k_swap_u12_32, k_trailing32) with the same per-element
// operations in the same order -- so the factor is bit-identical -- but
// without a kernel boundary or a global round trip between steps.
// unit_factor level 1, 2, 3: units with S <= 256, 384, 512 (0: none)
__host__ __device__ constexpr int fu_max_s(int level) { return level <= 0 ? 0 : 128 + 128 * level; }
constexpr int FU_MAX_S_ALL = 512;
// trailing blocks of at least this many rows go to the tensor cores
constexpr int TC_TRAIL_MIN_M = 192;
constexpr int FU_THREADS = 256;
constexpr size_t FU_SMEM = sizeof(float2) * (size_t)(MNB * (MNB + 1) + MNB * FU_THREADS);  // the swap stage
// dynamic shared memory of a launch whose largest unit has S = smax: the
// swap stage, or the panel (S rows of MNB + 1 entries) when taller
__host__ __device__ constexpr size_t fu_smem(int smax) {
    return FU_SMEM > sizeof(float2) * (size_t)smax * (MNB + 1) ? FU_SMEM : sizeof(float2) * (size_t)smax * (MNB + 1);
}

__global__ void __launch_bounds__(FU_THREADS, 3) k_factor32_unit(const UnitDesc *__restrict__ units,
                                                                const MixedUnit *__restrict__ mus, float2 *a32buf,
                                                                int32_t *piv_buf, int32_t *status,
                                                                const int32_t *__restrict__ order, int base) {
    extern __shared__ float2 s_fu[];
    __shared__ float s_v[FU_THREADS / 32];
    __shared__ int s_i[FU_THREADS / 32];
    __shared__ int s_p;
    const int ui = order[base + blockIdx.x];
    const UnitDesc u = units[ui];
    const int s = u.s;
    if (status[ui] != 0) return;
    float2 *A = a32buf + mus[ui].a32_off;
    int32_t *piv = piv_buf + u.piv_off;
    const int tid = threadIdx.x;
    for (int c0 = 0; c0 < s; c0 += MNB) {
        if (!panel32_body<FU_THREADS>(A, s, c0, piv, &status[ui], s_fu, s_v, s_i, &s_p)) return;
        __syncthreads();
        // row swaps on every column outside the panel, U12 = L11^-1 A12 on
        // the trailing ones (as k_swap_u12_32, a thread per column)
        const int nb = min(MNB, s - c0);
        float2(*s_L)[MNB + 1] = reinterpret_cast<float2(*)[MNB + 1]>(s_fu);
        float2(*s_c)[FU_THREADS] = reinterpret_cast<float2(*)[FU_THREADS]>(s_fu + MNB * (MNB + 1));
        for (int e = tid; e < nb * nb; e += FU_THREADS) s_L[e / nb][e % nb] = A[(int64_t)(c0 + e / nb) * s + c0 + e % nb];
        __syncthreads();
        for (int k0 = 0; k0 < s - nb; k0 += FU_THREADS) {
            const int idx = k0 + tid;
            const int K = idx < c0 ? idx : idx + nb;  // skip the panel columns
            if (K < s) {
                const bool trailing = K >= c0 + nb;
                for (int q = 0; q < nb; ++q) s_c[q][tid] = A[(int64_t)(c0 + q) * s + K];
                for (int q = 0; q < nb; ++q) {
                    int p = piv[c0 + q];
                    if (p == c0 + q) continue;
                    if (p < c0 + nb) {
                        float2 t0 = s_c[q][tid];
                        s_c[q][tid] = s_c[p - c0][tid];
                        s_c[p - c0][tid] = t0;
                    } else {
                        float2 t0 = s_c[q][tid];
                        s_c[q][tid] = A[(int64_t)p * s + K];
                        A[(int64_t)p * s + K] = t0;
                    }
                }
                if (trailing)
                    for (int q = 1; q < nb; ++q) {
                        float2 v = s_c[q][tid];
                        for (int c = 0; c < q; ++c) v = cf_sub(v, cf_mul(s_L[q][c], s_c[c][tid]));
                        s_c[q][tid] = v;
                    }
                for (int q = 0; q < nb; ++q) A[(int64_t)(c0 + q) * s + K] = s_c[q][tid];
            }
        }
        __syncthreads();
        // trailing update A22 -= L21 U12 (as k_trailing32, 64x64 tiles)
        if (c0 + MNB < s) {
            const int r0 = c0 + MNB, rows = s - r0;
            const int tiles = (rows + 63) / 64;
            float2(*s_l)[MNB + 1] = reinterpret_cast<float2(*)[MNB + 1]>(s_fu);
            float2(*s_u)[64] = reinterpret_cast<float2(*)[64]>(s_fu + 64 * (MNB + 1));
            const int ty = tid / 16, tx = tid % 16;
            for (int tile = 0; tile < tiles * tiles; ++tile) {
                const int R0 = r0 + (tile / tiles) * 64, K0 = r0 + (tile % tiles) * 64;
                for (int e = tid; e < 64 * MNB; e += FU_THREADS) {
                    int rr = e / MNB, q = e % MNB, R = R0 + rr;
                    s_l[rr][q] = (R < s) ? A[(int64_t)R * s + c0 + q] : cf(0.f, 0.f);
                }
                for (int e = tid; e < MNB * 64; e += FU_THREADS) {
                    int q = e / 64, cc = e % 64, K = K0 + cc;
                    s_u[q][cc] = (K < s) ? A[(int64_t)(c0 + q) * s + K] : cf(0.f, 0.f);
                }
                __syncthreads();
                float2 acc[4][4];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
                        acc[a][b] = (R < s && K < s) ? A[(int64_t)R * s + K] : cf(0.f, 0.f);
                    }
#pragma unroll 4
                for (int q = 0; q < MNB; ++q) {
                    float2 lv[4], uv[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) lv[a] = s_l[ty + 16 * a][q];
#pragma unroll
                    for (int b = 0; b < 4; ++b) uv[b] = s_u[q][tx + 16 * b];
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            acc[a][b].x = fmaf(-lv[a].x, uv[b].x, fmaf(lv[a].y, uv[b].y, acc[a][b].x));
                            acc[a][b].y = fmaf(-lv[a].x, uv[b].y, fmaf(-lv[a].y, uv[b].x, acc[a][b].y));
                        }
                }
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
                        if (R < s && K < s) A[(int64_t)R * s + K] = acc[a][b];
                    }
                __syncthreads();
            }
        }
    }
}

// Row swaps on every column outside the panel, then U12 for the trailing
// ones; 64 columns per CTA with their panel rows and the L block staged in
// shared memory.
// Panels taller than one CTA's shared memory, over many CTAs (fnec_grid.cuh).
struct MixedPanelOps {
    using E = float2;
    using V = float;
    static constexpr float V_NONE = -1.f;
    __device__ static float key(float2 a) { return a.x * a.x + a.y * a.y; }
    __device__ static void better(float &bv, int &bi, float v, int i) { piv_better32(bv, bi, v, i); }
    __device__ static float2 div(float2 a, float2 b) { return cf_div(a, b); }
    __device__ static float2 sub_mul(float2 acc, float2 f, float2 p) { return cf_sub(acc, cf_mul(f, p)); }
    __device__ static bool singular(float v) { return !(v > 0.f); }
    __device__ static float2 load_cg(const float2 *p) { return __ldcg(p); }
};

__global__ void __launch_bounds__(256) k_panel32_grid(const UnitDesc *__restrict__ units,
                                                      const MixedUnit *__restrict__ mus,
                                                      const int32_t *__restrict__ order, int c0, float2 *a32buf,
                                                      int32_t *piv_buf, int32_t *status, PanelXchg<float2> *xg,
                                                      GridSync *gs) {
    extern __shared__ float2 s_gpan32[];
    int ui = order[blockIdx.y];
    UnitDesc u = units[ui];
    if (status[ui] != 0) return;
    panel_grid_body<MixedPanelOps, MNB, 256>(a32buf + mus[ui].a32_off, (int64_t)u.s, u.s, c0, piv_buf + u.piv_off,
                                             &status[ui], xg + blockIdx.y, gs + blockIdx.y, (int)gridDim.x,
                                             (int)blockIdx.x, s_gpan32);
}

// defer: the previous step's update (columns c0 - 32 .. c0 of L, rows of
// U) is still owed by the trailing columns of this panel's rows (the
// second step of a two-step pair): it is applied to them after the swaps,
// before U12 is solved.
// Columns idx in [lo, hi) of the columns outside the panel (idx < c0: the
// column idx; else idx + nb), 64 per CTA: hi < 0 means all of them.
__global__ void __launch_bounds__(64) k_swap_u12_32(const UnitDesc *__restrict__ units,
                                                    const MixedUnit *__restrict__ mus, int c0, float2 *a32buf,
                                                    const int32_t *__restrict__ piv_buf,
                                                    const int32_t *__restrict__ status, const int32_t *__restrict__ order, int base,
                                                    int defer, int lo, int hi) {
    __shared__ float2 s_c[MNB][64];
    __shared__ float2 s_L[MNB][MNB + 1];
    __shared__ float2 s_D[MNB][MNB + 1];  // defer: the owed step's L rows of this panel (swapped)
    int ui = order[base + blockIdx.y];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || status[ui] != 0) return;
    int nb = min(MNB, s - c0);
    int t = threadIdx.x;
    const int end = hi < 0 ? s - nb : min(hi, s - nb);
    int idx = lo + blockIdx.x * 64 + t;
    if (lo + (int)blockIdx.x * 64 >= end) return;
    int K = idx < c0 ? idx : idx + nb;  // skip the panel columns
    bool live = idx < end;
    bool trailing = K >= c0 + nb;
    float2 *A = a32buf + mus[ui].a32_off;
    const int32_t *piv = piv_buf + u.piv_off;
    for (int e = t; e < nb * nb; e += 64) s_L[e / nb][e % nb] = A[(int64_t)(c0 + e / nb) * s + c0 + e % nb];
    if (defer)  // its L columns were swapped by the launch before this one
        for (int e = t; e < nb * MNB; e += 64) s_D[e / MNB][e % MNB] = A[(int64_t)(c0 + e / MNB) * s + c0 - MNB + e % MNB];
    for (int q = 0; q < nb; ++q) s_c[q][t] = live ? A[(int64_t)(c0 + q) * s + K] : cf(0.f, 0.f);
    __syncthreads();
    if (!live) return;
    for (int q = 0; q < nb; ++q) {
        int p = piv[c0 + q];
        if (p == c0 + q) continue;
        if (p < c0 + nb) {
            float2 t0 = s_c[q][t];
            s_c[q][t] = s_c[p - c0][t];
            s_c[p - c0][t] = t0;
        } else {
            float2 t0 = s_c[q][t];
            s_c[q][t] = A[(int64_t)p * s + K];
            A[(int64_t)p * s + K] = t0;
        }
    }
    if (trailing && defer) {
        // the deferred update, on the swapped rows: L rows from columns
        // c0 - 32 .. c0 of this panel's rows (s_D), U from rows c0 - 32 .. c0
        float2 uc[MNB];
#pragma unroll
        for (int c = 0; c < MNB; ++c) uc[c] = A[(int64_t)(c0 - MNB + c) * s + K];
        for (int q = 0; q < nb; ++q) {
            float2 v = s_c[q][t];
#pragma unroll
            for (int c = 0; c < MNB; ++c) {
                const float2 l = s_D[q][c];
                v.x = fmaf(-l.x, uc[c].x, fmaf(l.y, uc[c].y, v.x));
                v.y = fmaf(-l.x, uc[c].y, fmaf(-l.y, uc[c].x, v.y));
            }
            s_c[q][t] = v;
        }
    }
    if (trailing)
        for (int q = 1; q < nb; ++q) {
            float2 v = s_c[q][t];
            for (int c = 0; c < q; ++c) v = cf_sub(v, cf_mul(s_L[q][c], s_c[c][t]));
            s_c[q][t] = v;
        }
    for (int q = 0; q < nb; ++q) A[(int64_t)(c0 + q) * s + K] = s_c[q][t];
}

// A22 -= L21 U12 over kparts consecutive 32-column steps starting at c0
// (L21: columns c0 .. c0 + 32 kparts, U12: the same rows), on rows and
// columns from r0 = c0 + 32 kparts up to col_end (columns) and s (rows);
// 64x64 tiles, a 4x4 complex block per thread, the parts' products
// accumulated in registers so A22 is read and written once.  kparts 1,
// col_end s: the one-step update; kparts 1, col_end c0 + 64: the next
// panel's columns only (the look-ahead of a two-step pair); kparts 2: the
// pair's deferred update of everything to the right and below.  lower:
// only the tiles on and below the diagonal (the Hermitian factor; kparts
// 1, col_end s), T (T + 1) / 2 of them, row-major.
// Asynchronous 8-byte global -> shared copy (cp.async, no register
// staging); valid false writes zeros and reads nothing (src points into the
// matrix all the same).  cp_async_wait_all waits for this thread's copies.
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void lower_tile(int i, int &tr, int &tc) {
    int r = (int)((sqrtf(8.f * (float)i + 1.f) - 1.f) * 0.5f);
    while (r * (r + 1) / 2 > i) --r;
    while ((r + 1) * (r + 2) / 2 <= i) ++r;
    tr = r;
    tc = i - r * (r + 1) / 2;
}

// acc -= s_l s_u over the 32 panel columns for thread (ty, tx)'s 4 x 4
// entries of a 64 x 64 trailing tile (rows ty + 16 a, columns tx + 16 b).
// SKIP_UR: a diagonal tile of the Hermitian factor, whose upper-right 32 x
// 32 block (a < 2, b >= 2) is left alone -- those entries belong to a later
// step's U12, which that step's panel writes as its L21's mirror before
// anything reads them (every other entry gets the same operations).
template <bool SKIP_UR>
__device__ __forceinline__ void tile_fma(float2 (&acc)[4][4], const float2 (*s_l)[MNB + 1], const float2 (*s_u)[64],
                                         int ty, int tx) {
#pragma unroll 4
    for (int q = 0; q < MNB; ++q) {
        float2 lv[4], uv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) lv[a] = s_l[ty + 16 * a][q];
#pragma unroll
        for (int b = 0; b < 4; ++b) uv[b] = s_u[q][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (SKIP_UR && a < 2 && b >= 2) continue;
                acc[a][b].x = fmaf(-lv[a].x, uv[b].x, fmaf(lv[a].y, uv[b].y, acc[a][b].x));
                acc[a][b].y = fmaf(-lv[a].x, uv[b].y, fmaf(-lv[a].y, uv[b].x, acc[a][b].y));
            }
    }
}

__global__ void __launch_bounds__(256) k_trailing32(const UnitDesc *__restrict__ units, const MixedUnit *__restrict__ mus,
                                                    int c0, float2 *a32buf, const int32_t *__restrict__ status,
                                                    const int32_t *__restrict__ order, int base, int kparts,
                                                    int col_end, int lower) {
    __shared__ float2 s_l[64][MNB + 1];
    __shared__ float2 s_u[MNB][64];
    int ui = order[base + blockIdx.y];
    UnitDesc u = units[ui];
    int s = u.s;
    int r0 = c0 + MNB * kparts;
    if (r0 >= s || status[ui] != 0) return;
    const int ce = min(s, col_end);
    if (ce <= r0) return;
    int rows = s - r0, cols = ce - r0;
    int tiles_c = (cols + 63) / 64, tiles_r = (rows + 63) / 64;
    int tile = blockIdx.x;
    int R0, K0;
    if (lower) {
        if (tile >= tiles_r * (tiles_r + 1) / 2) return;
        int tr, tc;
        lower_tile(tile, tr, tc);
        R0 = r0 + tr * 64;
        K0 = r0 + tc * 64;
    } else {
        if (tile >= tiles_r * tiles_c) return;
        R0 = r0 + (tile / tiles_c) * 64;
        K0 = r0 + (tile % tiles_c) * 64;
    }
    float2 *A = a32buf + mus[ui].a32_off;
    int tid = threadIdx.x;
    int ty = tid / 16, tx = tid % 16;
    const bool skip_ur = lower && R0 == K0;  // a diagonal tile of the Hermitian factor (tile_fma)
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
            acc[a][b] = (R < s && K < ce && !(skip_ur && a < 2 && b >= 2)) ? A[(int64_t)R * s + K] : cf(0.f, 0.f);
        }
    for (int part = 0; part < kparts; ++part) {
        const int cp = c0 + MNB * part;
        if (part) __syncthreads();  // the previous part's reads of s_l / s_u are done
        for (int e = tid; e < 64 * MNB; e += 256) {
            const int rr = e / MNB, q = e % MNB, R = R0 + rr;
            cp_async8(&s_l[rr][q], A + (int64_t)min(R, s - 1) * s + cp + q, R < s);
        }
        for (int e = tid; e < MNB * 64; e += 256) {
            const int q = e / 64, cc = e % 64, K = K0 + cc;
            cp_async8(&s_u[q][cc], A + (int64_t)(cp + q) * s + min(K, ce - 1), K < ce);
        }
        cp_async_wait_all();
        __syncthreads();
        if (skip_ur) tile_fma<true>(acc, s_l, s_u, ty, tx);
        else tile_fma<false>(acc, s_l, s_u, ty, tx);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
            if (R < s && K < ce && !(skip_ur && a < 2 && b >= 2)) A[(int64_t)R * s + K] = acc[a][b];
        }
}

// ---------------------------------------------------------------------------
// Hermitian factor without row exchanges (schedule factor_pivoting 0)
// ---------------------------------------------------------------------------
// A32 = M^H M + lambda I is Hermitian positive definite, so Gaussian
// elimination needs no row exchanges, and its factor A = L U has
// U = D L^H (D: the pivots).  Two consequences: the trailing update
// A22 -= L21 U12 stays Hermitian, so only the tiles on and below the
// diagonal are computed (the 32x32 diagonal blocks always lie inside
// diagonal tiles, and nothing reads the stale entries above them); and
// each step's U12 is its L21 mirrored, U12[q][K] = d_q conj(L21[K][q]),
// written by the panel instead of a triangular solve.  The factor is
// stored in the GEPP layout (unit-lower L below the diagonal, U on and
// above it, identity pivots), so the refinement applies it unchanged.
// A zero or non-finite pivot fails the unit as a singular GEPP panel does.

// The nb x nb diagonal block at c0, factored in shared memory by all NT
// threads (sD[r][k]; one barrier per column).  On return sD holds L11
// (unit lower, below the diagonal) and U11, sDinv the pivots' reciprocals;
// *s_bad the first failing column + 1, or 0.
template <int NT>
__device__ void herm_diag_block(const float2 *A, int s, int c0, int nb, float2 (*sD)[MNB + 1], float2 *sDinv,
                                int *s_bad) {
    const int tid = threadIdx.x;
    for (int e = tid; e < nb * nb; e += NT) sD[e / nb][e % nb] = A[(int64_t)(c0 + e / nb) * s + c0 + e % nb];
    if (tid == 0) *s_bad = 0;
    for (int c = 0; c < nb; ++c) {
        __syncthreads();  // column c - 1's update is complete
        const float2 d = sD[c][c];
        const float dn = d.x * d.x + d.y * d.y;
        const float2 dinv = cf(d.x / dn, -d.y / dn);
        if (tid == 0) {
            sDinv[c] = dinv;
            if ((!(dn > 0.f) || !(dn < INFINITY)) && *s_bad == 0) *s_bad = c + 1;
        }
        // column c - 1's multipliers (nobody reads that column in this pass)
        if (c > 0 && tid >= c && tid < nb) sD[tid][c - 1] = cf_mul(sD[tid][c - 1], sDinv[c - 1]);
        const int m = nb - 1 - c;
        for (int e = tid; e < m * m; e += NT) {
            const int r = c + 1 + e / m, k = c + 1 + e % m;
            const float2 f = cf_mul(sD[r][c], dinv);
            sD[r][k] = cf_sub(sD[r][k], cf_mul(f, sD[c][k]));
        }
    }
    __syncthreads();
}

// Rows [r_begin, r_end) below a full (32-column) diagonal block: L21 row r
// solves l U11 = A[r][c0 .. c0 + 32) (a thread per row, U11 read by
// broadcast), then U12's column r is its mirror.  Two halves of 16
// columns keep the live row in 16 complex registers: the second half
// takes the first's contribution from its stored entries.
template <int NT>
__device__ void herm_rows(float2 *A, int s, int c0, int r_begin, int r_end, const float2 (*sD)[MNB + 1],
                          const float2 *sDinv) {
    constexpr int H = MNB / 2;
    for (int r = r_begin + (int)threadIdx.x; r < r_end; r += NT) {
        float2 *row = A + (int64_t)r * s + c0;
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const int o = h * H;
            float2 a[H];
#pragma unroll
            for (int q = 0; q < H; ++q) a[q] = row[o + q];
            if (h) {
#pragma unroll 4
                for (int c = 0; c < H; ++c) {
                    const float2 l = row[c];
#pragma unroll
                    for (int k = 0; k < H; ++k) a[k] = cf_sub(a[k], cf_mul(l, sD[c][o + k]));
                }
            }
#pragma unroll
            for (int c = 0; c < H; ++c) {
                a[c] = cf_mul(a[c], sDinv[o + c]);
#pragma unroll
                for (int k = c + 1; k < H; ++k) a[k] = cf_sub(a[k], cf_mul(a[c], sD[o + c][o + k]));
            }
#pragma unroll
            for (int q = 0; q < H; ++q) {
                row[o + q] = a[q];
                const float2 d = sD[o + q][o + q];
                A[(int64_t)(c0 + o + q) * s + r] = cf(d.x * a[q].x + d.y * a[q].y, d.y * a[q].x - d.x * a[q].y);
            }
        }
    }
}

// The inverses of a factored diagonal block for the refinement's
// preconditioner (sD: unit-lower L11 below the diagonal, U11 on and above
// it; sDinv: 1 / U11[i][i]), in FP32, by threads 0 .. 255: threads
// 0 .. 127 form L11^-1, 128 .. 255 U11^-1, four consecutive lanes per
// column j, each summing the terms k = q (mod 4) of the substitution; the
// quarter sums are added by two shuffles (a column's lanes share a warp).
// The columns live in X, column-major with a pitch of 36 entries per
// column (a warp's 8 columns x 4 quarters then read 2-way-spread banks:
// two wavefronts per 64-bit load, the minimum).  Stored row-major, L^-1
// then U^-1 (2 x 1024 entries), zero outside an nb < 32 block.
constexpr int BI_PITCH = 36;
__device__ void herm_block_inverse(const float2 (*sD)[MNB + 1], const float2 *sDinv, int nb, float2 *X,
                                   float2 *out) {
    const int t = threadIdx.x, w = t >> 7, j = (t & 127) >> 2, q = t & 3;
    float2 *Xj = X + (w * 32 + j) * BI_PITCH;  // column j of this triangle's inverse
    const bool live = j < nb;
    if (w == 0) {  // L^-1 e_j: forward, unit diagonal
        for (int i = 0; i < 32; ++i) {
            float2 p = cf(0.f, 0.f);
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int k = q + 4 * m;
                if (k < i && k < nb) p = cf_add(p, cf_mul(sD[i][k], Xj[k]));  // Xj[k] = 0 for k < j
            }
            p.x += __shfl_xor_sync(0xffffffffu, p.x, 1);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, 1);
            p.x += __shfl_xor_sync(0xffffffffu, p.x, 2);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, 2);
            if (q == 0) Xj[i] = (live && i >= j && i < nb) ? cf((i == j ? 1.f : 0.f) - p.x, -p.y) : cf(0.f, 0.f);
            __syncwarp();
        }
    } else {  // U^-1 e_j: backward
        for (int i = 31; i >= 0; --i) {
            float2 p = cf(0.f, 0.f);
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int k = q + 4 * m;
                if (k > i && k < nb) p = cf_add(p, cf_mul(sD[i][k], Xj[k]));  // Xj[k] = 0 for k > j
            }
            p.x += __shfl_xor_sync(0xffffffffu, p.x, 1);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, 1);
            p.x += __shfl_xor_sync(0xffffffffu, p.x, 2);
            p.y += __shfl_xor_sync(0xffffffffu, p.y, 2);
            if (q == 0)
                Xj[i] = (live && i <= j && i < nb) ? cf_mul(cf((i == j ? 1.f : 0.f) - p.x, -p.y), sDinv[i])
                                                   : cf(0.f, 0.f);
            __syncwarp();
        }
    }
    out += w * 1024;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int i = q + 4 * m;
        out[i * 32 + j] = Xj[i];
    }
}

// The panel step at c0 of every unit of a size class, one CTA of NT
// threads per unit (1024 for panels of more than 256 rows below the
// diagonal block): the diagonal block, then every row below it.
template <int NT>
__global__ void __launch_bounds__(NT) k_panel32_herm(const UnitDesc *__restrict__ units,
                                                    const MixedUnit *__restrict__ mus, int c0, float2 *a32buf,
                                                    int32_t *piv_buf, int32_t *status,
                                                    const int32_t *__restrict__ order, int base) {
    __shared__ float2 sD[MNB][MNB + 1];
    __shared__ float2 sDinv[MNB];
    __shared__ int s_bad;
    const int ui = order[base + blockIdx.x];
    const UnitDesc u = units[ui];
    const int s = u.s;
    if (c0 >= s || status[ui] != 0) return;
    const int nb = min(MNB, s - c0);
    float2 *A = a32buf + mus[ui].a32_off;
    herm_diag_block<NT>(A, s, c0, nb, sD, sDinv, &s_bad);
    const int tid = threadIdx.x;
    if (s_bad) {
        if (tid == 0) status[ui] = -(c0 + s_bad);
        return;
    }
    for (int e = tid; e < nb * nb; e += NT) A[(int64_t)(c0 + e / nb) * s + c0 + e % nb] = sD[e / nb][e % nb];
    if (tid < nb) piv_buf[u.piv_off + c0 + tid] = c0 + tid;
    if (nb == MNB) herm_rows<NT>(A, s, c0, c0 + MNB, s, sD, sDinv);
}

// Tall panels (more than HERM_SPLIT_ROWS rows below the diagonal block)
// in two launches, so that their rows spread over many CTAs: the diagonal
// block first (one CTA per unit, stored in place with its pivots), then
// the rows in chunks of HERM_ROWS_CHUNK, each CTA loading the stored block
// and recomputing the pivots' reciprocals with the same operations -- every
// stored entry is the one-CTA panel's.
constexpr int HERM_SPLIT_ROWS = 1024;
constexpr int HERM_ROWS_CHUNK = 256;

__global__ void __launch_bounds__(256) k_herm_diag(const UnitDesc *__restrict__ units,
                                                   const MixedUnit *__restrict__ mus, int c0, float2 *a32buf,
                                                   int32_t *piv_buf, int32_t *status,
                                                   const int32_t *__restrict__ order, int base) {
    __shared__ float2 sD[MNB][MNB + 1];
    __shared__ float2 sDinv[MNB];
    __shared__ int s_bad;
    const int ui = order[base + blockIdx.x];
    const UnitDesc u = units[ui];
    const int s = u.s;
    if (c0 >= s || status[ui] != 0) return;
    const int nb = min(MNB, s - c0);
    float2 *A = a32buf + mus[ui].a32_off;
    herm_diag_block<256>(A, s, c0, nb, sD, sDinv, &s_bad);
    const int tid = threadIdx.x;
    if (s_bad) {
        if (tid == 0) status[ui] = -(c0 + s_bad);
        return;
    }
    for (int e = tid; e < nb * nb; e += 256) A[(int64_t)(c0 + e / nb) * s + c0 + e % nb] = sD[e / nb][e % nb];
    if (tid < nb) piv_buf[u.piv_off + c0 + tid] = c0 + tid;
}

__global__ void __launch_bounds__(HERM_ROWS_CHUNK) k_herm_rows(const UnitDesc *__restrict__ units,
                                                               const MixedUnit *__restrict__ mus, int c0,
                                                               float2 *a32buf, const int32_t *__restrict__ status,
                                                               const int32_t *__restrict__ order, int base) {
    __shared__ float2 sD[MNB][MNB + 1];
    __shared__ float2 sDinv[MNB];
    const int ui = order[base + blockIdx.y];
    const UnitDesc u = units[ui];
    const int s = u.s;
    if (c0 + MNB >= s || status[ui] != 0) return;  // no rows below a full block (status: set before this launch)
    const int r_begin = c0 + MNB + (int)blockIdx.x * HERM_ROWS_CHUNK;
    if (r_begin >= s) return;
    float2 *A = a32buf + mus[ui].a32_off;
    const int tid = threadIdx.x;
    for (int e = tid; e < MNB * MNB; e += HERM_ROWS_CHUNK) sD[e / MNB][e % MNB] = A[(int64_t)(c0 + e / MNB) * s + c0 + e % MNB];
    __syncthreads();
    if (tid < MNB) {  // as herm_diag_block forms them from the same pivots
        const float2 d = sD[tid][tid];
        const float dn = d.x * d.x + d.y * d.y;
        sDinv[tid] = cf(d.x / dn, -d.y / dn);
    }
    __syncthreads();
    herm_rows<HERM_ROWS_CHUNK>(A, s, c0, r_begin, min(s, r_begin + HERM_ROWS_CHUNK), sD, sDinv);
}

// The whole Hermitian factor of one small unit (S <= fu_max_s(level)) per
// CTA: the per-step kernels' operations without a launch between steps.
__global__ void __launch_bounds__(FU_THREADS, 4) k_factor32_unit_herm(const UnitDesc *__restrict__ units,
                                                                     const MixedUnit *__restrict__ mus,
                                                                     float2 *a32buf, int32_t *piv_buf,
                                                                     int32_t *status,
                                                                     const int32_t *__restrict__ order, int base) {
    __shared__ float2 sD[MNB][MNB + 1];
    __shared__ float2 sDinv[MNB];
    __shared__ float2 s_l[64][MNB + 1];
    __shared__ float2 s_u[MNB][64];
    __shared__ int s_bad;
    const int ui = order[base + blockIdx.x];
    const UnitDesc u = units[ui];
    const int s = u.s;
    if (status[ui] != 0) return;
    float2 *A = a32buf + mus[ui].a32_off;
    const int tid = threadIdx.x;
    for (int c0 = 0; c0 < s; c0 += MNB) {
        const int nb = min(MNB, s - c0);
        herm_diag_block<FU_THREADS>(A, s, c0, nb, sD, sDinv, &s_bad);
        if (s_bad) {
            if (tid == 0) status[ui] = -(c0 + s_bad);
            return;
        }
        for (int e = tid; e < nb * nb; e += FU_THREADS) A[(int64_t)(c0 + e / nb) * s + c0 + e % nb] = sD[e / nb][e % nb];
        if (tid < nb) piv_buf[u.piv_off + c0 + tid] = c0 + tid;
        if (nb < MNB) break;  // the last block: nothing below it
        herm_rows<FU_THREADS>(A, s, c0, c0 + MNB, s, sD, sDinv);
        __syncthreads();  // L21 and U12 written (global, this CTA)
        // A22 -= L21 U12 on the tiles on and below the diagonal
        const int r0 = c0 + MNB, rows = s - r0;
        if (rows <= 0) continue;
        const int T = (rows + 63) / 64;
        const int ty = tid / 16, tx = tid % 16;
        int staged_tr = -1;  // the tile row whose L21 block s_l holds
        for (int tile = 0; tile < T * (T + 1) / 2; ++tile) {
            int tr, tc;
            lower_tile(tile, tr, tc);
            const int R0 = r0 + tr * 64, K0 = r0 + tc * 64;
            // the panel blocks copied asynchronously (L21 only when the tile
            // row changes: the tiles of a row share it) while this thread's
            // A22 entries load
            if (tr != staged_tr) {
                for (int e = tid; e < 64 * MNB; e += FU_THREADS) {
                    const int rr = e / MNB, q = e % MNB, R = R0 + rr;
                    cp_async8(&s_l[rr][q], A + (int64_t)min(R, s - 1) * s + c0 + q, R < s);
                }
                staged_tr = tr;
            }
            for (int e = tid; e < MNB * 64; e += FU_THREADS) {
                const int q = e / 64, cc = e % 64, K = K0 + cc;
                cp_async8(&s_u[q][cc], A + (int64_t)(c0 + q) * s + min(K, s - 1), K < s);
            }
            const bool diag = tr == tc;
            float2 acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
                    acc[a][b] = (R < s && K < s && !(diag && a < 2 && b >= 2)) ? A[(int64_t)R * s + K] : cf(0.f, 0.f);
                }
            cp_async_wait_all();
            __syncthreads();
            if (diag) tile_fma<true>(acc, s_l, s_u, ty, tx);
            else tile_fma<false>(acc, s_l, s_u, ty, tx);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
                    if (R < s && K < s && !(diag && a < 2 && b >= 2)) A[(int64_t)R * s + K] = acc[a][b];
                }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 GMRES iterative refinement, one CTA (256 threads) per unit
// ---------------------------------------------------------------------------
struct GmresCtx {
    int n, s, w, rows, nc;
    const cx *z;
    const cx *y;
    const double *cv;
    const int32_t *rowwire, *wptr, *wrow;
    const DevConRow *crows;
    const float2 *lu;
    const int32_t *piv;
    const int32_t *perm = nullptr;  // the row permutation of piv, if built (then P in = in[perm])
    const float2 *binv = nullptr;   // the factor's diagonal block inverses (FP32), if built
    cx *t;  // rows
};

__device__ __forceinline__ cx warp_sum(cx v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.re += __shfl_down_sync(0xffffffffu, v.re, o);
        v.im += __shfl_down_sync(0xffffffffu, v.im, o);
    }
    return v;
}

__device__ double block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
    __syncthreads();
    return s;
}

// out = M^H (M v) + lambda v   (v, out: S).  v and the row vector t are
// staged in shared memory (sv: S, st: rows; so: N accumulators).  Z is
// streamed once from HBM: each block of ARB rows is first reduced into
// t (a warp per row) and then, right away and still in L1/L2, folded into
// the column sums M^H t (a thread per column), so the second use of every
// row costs no HBM traffic.
constexpr int ARB = 16;  // rows per block (2 per warp)


__device__ void apply_A(const GmresCtx &g, const cx *v, cx *out, cx *sv, cx *st, cx *so) {
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n = g.n;
    for (int i = tid; i < g.s; i += blockDim.x) sv[i] = v[i];
    for (int c = tid; c < n; c += blockDim.x) so[c] = {0, 0};
    __syncthreads();
    for (int rb = 0; rb < n; rb += ARB) {
        // a warp's ARB / 8 rows of the block together: their loads are in
        // flight at once (each row's sum in the same order as alone)
        constexpr int RPW = ARB / 8;
        cx acc[RPW];
        const cx *zr[RPW];
        bool has[RPW];
#pragma unroll
        for (int q = 0; q < RPW; ++q) {
            const int r = rb + wid + 8 * q;
            acc[q] = {0, 0};
            has[q] = r < n;
            zr[q] = g.z + (int64_t)(has[q] ? r : 0) * n;
        }
#pragma unroll 4
        for (int c = lane; c < n; c += 32) {
            const cx x = sv[c];
#pragma unroll
            for (int q = 0; q < RPW; ++q)
                if (has[q]) acc[q] = zadd(acc[q], zmul(ld_z(zr[q] + c), x));
        }
#pragma unroll
        for (int q = 0; q < RPW; ++q) {
            const int r = rb + wid + 8 * q;
            const cx a = warp_sum(acc[q]);
            if (lane == 0 && has[q]) {
                cx cvv = sv[n + g.rowwire[r]];
                st[r] = {a.re - g.cv[r] * cvv.re, a.im - g.cv[r] * cvv.im};
            }
        }
        __syncthreads();
        const int re = min(rb + ARB, n);
        for (int c = tid; c < n; c += blockDim.x) {
            const cx *zc = g.z + (int64_t)rb * n + c;
            cx a0 = so[c], a1 = {0, 0};
            int r = rb;
#pragma unroll 4
            for (; r + 2 <= re; r += 2, zc += 2 * (int64_t)n) {
                a0 = zadd(a0, zcmul(ld_z(zc), st[r]));
                a1 = zadd(a1, zcmul(ld_z(zc + n), st[r + 1]));
            }
            if (r < re) a0 = zadd(a0, zcmul(ld_z(zc), st[r]));
            so[c] = zadd(a0, a1);
        }
        // no barrier: st rows of the next block are disjoint, and so[c] is
        // only ever touched by the thread that owns column c
    }
    for (int q = tid; q < g.nc; q += blockDim.x) {
        DevConRow c = g.crows[q];
        cx val = sv[c.c0];
        if (c.c1 >= 0) val = zadd(val, zscale(sv[c.c1], c.v1));
        st[n + q] = val;
    }
    __syncthreads();
    for (int c = tid; c < n; c += blockDim.x) out[c] = zadd(so[c], zscale(sv[c], 1e-8));
    for (int w = tid; w < g.w; w += blockDim.x) {
        cx acc = {0, 0};
        for (int q = g.wptr[w]; q < g.wptr[w + 1]; ++q) {
            int r = g.wrow[q];
            acc = zadd(acc, zscale(st[r], -g.cv[r]));
        }
        out[g.n + w] = zadd(acc, zscale(sv[g.n + w], 1e-8));
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < g.nc; ++q) {
            DevConRow c = g.crows[q];
            cx tq = st[g.n + q];
            out[c.c0] = zadd(out[c.c0], tq);
            if (c.c1 >= 0) out[c.c1] = zadd(out[c.c1], zscale(tq, c.v1));
        }
    __syncthreads();
}

// out = (L U)^-1 P in with the complex64 factor, blocked by 32 columns:
// one warp solves each 32x32 diagonal block from registers (each lane holds
// its row of the block), then all threads update the remaining rows with
// fully unrolled, independent loads.  The factor is stored in FP32 but the
// substitution runs in FP64: the preconditioner is then one fixed linear
// operator (the stored L U) to FP64 rounding, so the preconditioned
// residual GMRES minimises and tests is measured without an FP32 floor.
// in/out are FP64, sy is shared memory (S).
__device__ __forceinline__ cx f2z(float2 a) { return {(double)a.x, (double)a.y}; }

__device__ void apply_prec(const GmresCtx &g, const cx *in, cx *out, cx *sy) {
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int s = g.s;
    if (g.perm) {
        for (int i = tid; i < s; i += blockDim.x) sy[i] = in[g.perm[i]];
    } else {
        for (int i = tid; i < s; i += blockDim.x) sy[i] = in[i];
        __syncthreads();
        if (tid == 0)
            for (int c = 0; c < s; ++c) {
                int p = g.piv[c];
                if (p != c) {
                    cx t0 = sy[c];
                    sy[c] = sy[p];
                    sy[p] = t0;
                }
            }
    }
    __syncthreads();
    if (g.binv) {
        // block products with the diagonal blocks' inverses: every warp
        // takes rows of the 32x32 product (no serial substitution chain),
        // then all threads update the rows outside the block (the refinement
        // kernels run 256 threads: 8 warps x 4 rows of each block)
        __shared__ cx s_blk[32];
        // each warp's 4 rows of the next block's inverse are loaded one block
        // step ahead (blockDim 256: 8 warps x 4 rows = 32); entries outside
        // an nb < 32 block are stored as zeros
        float2 li[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) li[q] = g.binv[(wid + 8 * q) * 32 + lane];
        for (int c0 = 0; c0 < s; c0 += 32) {
            const int nb = min(32, s - c0);
            const cx xk = lane < nb ? sy[c0 + lane] : cx{0, 0};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = wid + 8 * q;
                cx p = warp_sum(lane < nb ? zmul(f2z(li[q]), xk) : cx{0, 0});
                if (lane == 0 && i < nb) s_blk[i] = p;
            }
            if (c0 + 32 < s) {
                const float2 *Ln = g.binv + (int64_t)(c0 / 32 + 1) * 2048;
#pragma unroll
                for (int q = 0; q < 4; ++q) li[q] = Ln[(wid + 8 * q) * 32 + lane];
            }
            __syncthreads();
            for (int i = tid; i < nb; i += blockDim.x) sy[c0 + i] = s_blk[i];
            if (nb == 32) {
                // threads per row: adjacent lanes split a short trailing
                // block's 32 columns (their partial sums meet by shuffles),
                // so a step takes fewer rounds of dependent loads
                const int rows = s - (c0 + 32);
                const int tpr = rows <= 64 ? 4 : (rows <= 128 ? 2 : 1);
                const int per = 256 / tpr, cols = 32 / tpr, part = tid % tpr;
                for (int base = 0; base < rows; base += per) {
                    const int r = c0 + 32 + base + tid / tpr;
                    cx acc = {0, 0};
                    if (r < s) {
                        const float2 *lrow = g.lu + (int64_t)r * s + c0 + part * cols;
                        const cx *sb = s_blk + part * cols;
                        for (int c8 = 0; c8 < cols; c8 += 8) {
                            float2 lr[8];
#pragma unroll
                            for (int c = 0; c < 8; ++c) lr[c] = lrow[c8 + c];
#pragma unroll
                            for (int c = 0; c < 8; ++c) acc = zadd(acc, zmul(f2z(lr[c]), sb[c8 + c]));
                        }
                    }
                    for (int o = tpr >> 1; o > 0; o >>= 1) {
                        acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
                        acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
                    }
                    if (r < s && part == 0) sy[r] = zsub(sy[r], acc);
                }
            }
            __syncthreads();
        }
        {
            const float2 *Ul = g.binv + (int64_t)((s - 1) / 32) * 2048 + 1024;
#pragma unroll
            for (int q = 0; q < 4; ++q) li[q] = Ul[(wid + 8 * q) * 32 + lane];
        }
        for (int c0 = ((s - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
            const int nb = min(32, s - c0);
            const cx xk = lane < nb ? sy[c0 + lane] : cx{0, 0};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int i = wid + 8 * q;
                cx p = warp_sum(lane < nb ? zmul(f2z(li[q]), xk) : cx{0, 0});
                if (lane == 0 && i < nb) s_blk[i] = p;
            }
            if (c0 > 0) {
                const float2 *Un = g.binv + (int64_t)(c0 / 32 - 1) * 2048 + 1024;
#pragma unroll
                for (int q = 0; q < 4; ++q) li[q] = Un[(wid + 8 * q) * 32 + lane];
            }
            __syncthreads();
            for (int i = tid; i < nb; i += blockDim.x) sy[c0 + i] = s_blk[i];
            if (nb == 32) {
                const int rows = c0;
                const int tpr = rows <= 64 ? 4 : (rows <= 128 ? 2 : 1);
                const int per = 256 / tpr, cols = 32 / tpr, part = tid % tpr;
                for (int base = 0; base < rows; base += per) {
                    const int r = base + tid / tpr;
                    cx acc = {0, 0};
                    if (r < c0) {
                        const float2 *urow = g.lu + (int64_t)r * s + c0 + part * cols;
                        const cx *sb = s_blk + part * cols;
                        for (int c8 = 0; c8 < cols; c8 += 8) {
                            float2 ur[8];
#pragma unroll
                            for (int c = 0; c < 8; ++c) ur[c] = urow[c8 + c];
#pragma unroll
                            for (int c = 0; c < 8; ++c) acc = zadd(acc, zmul(f2z(ur[c]), sb[c8 + c]));
                        }
                    }
                    for (int o = tpr >> 1; o > 0; o >>= 1) {
                        acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
                        acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
                    }
                    if (r < c0 && part == 0) sy[r] = zsub(sy[r], acc);
                }
            } else {
                for (int r = tid; r < c0; r += blockDim.x) {
                    const float2 *urow = g.lu + (int64_t)r * s + c0;
                    cx acc = sy[r];
                    for (int c = 0; c < nb; ++c) acc = zsub(acc, zmul(f2z(urow[c]), s_blk[c]));
                    sy[r] = acc;
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < s; i += blockDim.x) out[i] = sy[i];
        __syncthreads();
        return;
    }
    // forward: unit lower triangular (factor rows read 8 entries at a time
    // to keep the register footprint small enough for several CTAs per SM)
    for (int c0 = 0; c0 < s; c0 += 32) {
        int nb = min(32, s - c0);
        if (wid == 0) {
            cx yl = lane < nb ? sy[c0 + lane] : cx{0, 0};
            const float2 *lrow = g.lu + (int64_t)(c0 + (lane < nb ? lane : 0)) * s + c0;
#pragma unroll 1
            for (int c8 = 0; c8 < 32; c8 += 8) {
                float2 lr[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) lr[c] = (c8 + c < nb) ? lrow[c8 + c] : cf(0.f, 0.f);
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    double yr = __shfl_sync(0xffffffffu, yl.re, c8 + c), yi = __shfl_sync(0xffffffffu, yl.im, c8 + c);
                    if (lane > c8 + c && lane < nb) yl = zsub(yl, zmul(f2z(lr[c]), cx{yr, yi}));
                }
            }
            if (lane < nb) sy[c0 + lane] = yl;
        }
        __syncthreads();
        if (nb == 32) {
            for (int r = c0 + 32 + tid; r < s; r += blockDim.x) {
                const float2 *lrow = g.lu + (int64_t)r * s + c0;
                cx acc = sy[r];
#pragma unroll
                for (int c8 = 0; c8 < 32; c8 += 8) {
                    float2 lr[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) lr[c] = lrow[c8 + c];
#pragma unroll
                    for (int c = 0; c < 8; ++c) acc = zsub(acc, zmul(f2z(lr[c]), sy[c0 + c8 + c]));
                }
                sy[r] = acc;
            }
        }
        __syncthreads();
    }
    // backward: upper triangular with diagonal
    for (int c1 = s; c1 > 0; c1 -= 32) {
        int c0 = max(0, c1 - 32), nb = c1 - c0;
        if (wid == 0) {
            cx yl = lane < nb ? sy[c0 + lane] : cx{0, 0};
            const float2 *urow = g.lu + (int64_t)(c0 + (lane < nb ? lane : 0)) * s + c0;
#pragma unroll 1
            for (int c8 = 24; c8 >= 0; c8 -= 8) {
                float2 ur[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) ur[c] = (c8 + c < nb) ? urow[c8 + c] : cf(1.f, 0.f);
#pragma unroll
                for (int c = 7; c >= 0; --c) {
                    const int cc = c8 + c;
                    if (cc < nb) {
                        if (lane == cc) yl = zdiv(yl, f2z(ur[c]));
                        double yr = __shfl_sync(0xffffffffu, yl.re, cc), yi = __shfl_sync(0xffffffffu, yl.im, cc);
                        if (lane < cc) yl = zsub(yl, zmul(f2z(ur[c]), cx{yr, yi}));
                    }
                }
            }
            if (lane < nb) sy[c0 + lane] = yl;
        }
        __syncthreads();
        for (int r = tid; r < c0; r += blockDim.x) {
            const float2 *urow = g.lu + (int64_t)r * s + c0;
            cx acc = sy[r];
            if (nb == 32) {
#pragma unroll
                for (int c8 = 0; c8 < 32; c8 += 8) {
                    float2 ur[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) ur[c] = urow[c8 + c];
#pragma unroll
                    for (int c = 0; c < 8; ++c) acc = zsub(acc, zmul(f2z(ur[c]), sy[c0 + c8 + c]));
                }
            } else {
                for (int c = 0; c < nb; ++c) acc = zsub(acc, zmul(f2z(urow[c]), sy[c0 + c]));
            }
            sy[r] = acc;
        }
        __syncthreads();
    }
    for (int i = tid; i < s; i += blockDim.x) out[i] = sy[i];
    __syncthreads();
}

// Inverses, in FP64, of the FP32 factor's 32x32 diagonal blocks of one
// system: warp 0 forms L11^-1 (unit lower), warp 1 U11^-1 (upper), lane j
// column j by substitution on its own column.  Stored row-major per block:
// L^-1 then U^-1 (2 x 1024 complex128); entries outside an nb < 32 block
// are zero.  The refinement applies the preconditioner with them.
// The inverses of every system's 32x32 diagonal blocks of the factor (any
// factor: unit-lower L11, U11 on and above the diagonal), one CTA of 256
// threads per block (herm_block_inverse).
// One CTA per 32-row diagonal block of every system: tab[blockIdx.x] =
// (system, block), built at planning, so no CTA is launched for a block a
// system does not have.
__global__ void __launch_bounds__(256) k_block_inv32(const UnitDesc *__restrict__ units,
                                                     const MixedUnit *__restrict__ smu,
                                                     const float2 *__restrict__ a32buf, float2 *binvbuf,
                                                     const int32_t *__restrict__ status,
                                                     const int2 *__restrict__ tab) {
    __shared__ float2 sB[MNB][MNB + 1];
    __shared__ float2 sDinv[MNB];
    __shared__ float2 sX[2 * MNB * BI_PITCH];
    const int2 t = tab[blockIdx.x];
    const int ui = t.x;
    const UnitDesc u = units[ui];
    const int c0 = t.y * 32, s = u.s;
    if (c0 >= s || status[ui] != 0) return;
    const int nb = min(32, s - c0);
    const float2 *A = a32buf + smu[ui].a32_off;
    const int tid = threadIdx.x;
    for (int e = tid; e < 32 * 32; e += 256) {
        const int i = e / 32, k = e % 32;
        sB[i][k] = (i < nb && k < nb) ? A[(int64_t)(c0 + i) * s + c0 + k] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (tid < 32) {
        const float2 d = sB[tid][tid];
        const float dn = d.x * d.x + d.y * d.y;
        sDinv[tid] = tid < nb ? cf(d.x / dn, -d.y / dn) : cf(0.f, 0.f);
    }
    __syncthreads();
    herm_block_inverse(sB, sDinv, nb, sX, binvbuf + smu[ui].binv_off + (int64_t)t.y * 2048);
}

__device__ double vnorm(const cx *v, int s, double *red) {
    double a = 0;
    for (int i = threadIdx.x; i < s; i += blockDim.x) a += v[i].re * v[i].re + v[i].im * v[i].im;
    return sqrt(block_sum(a, red));
}

// MINB: CTAs per SM the registers are budgeted for (3: 80 registers, no
// spills; 4: 64 registers, a few spilled) -- more resident solves against
// cheaper ones, picked per batch by the tuner.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_gmres_ir(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                                                  MixedUnit *mus, const int32_t *__restrict__ ibuf,
                                                  const DevConRow *__restrict__ crows, const cx *__restrict__ zbuf,
                                                  const cx *__restrict__ rhs, const double *__restrict__ cosv,
                                                  const float2 *__restrict__ a32buf, const int32_t *__restrict__ pivbuf,
                                                  cx *xbuf, cx *vbuf, cx *wbuf, const int32_t *__restrict__ status,
                                                  int staged, int skip_s, int only, int min_s,
                                                  const int32_t *__restrict__ s_order, const float2 *__restrict__ binvbuf,
                                                  int use_b) {
    extern __shared__ unsigned char s_dyn[];
    __shared__ cx sH[(GM + 1) * GM];
    __shared__ double scs[GM];
    __shared__ cx ssn[GM];
    __shared__ cx sg[GM + 1];
    __shared__ cx sh[GM + 1];
    __shared__ double red[8];
    __shared__ int s_stop;
    int ui = s_order ? s_order[blockIdx.x] : (int)blockIdx.x;  // one solve (right-hand side)
    UnitDesc u = units[ui];
    if (status[u.sys] != 0 || u.s >= skip_s || u.s < min_s) return;  // refined grid-wide / by clusters
    if (only >= 0 && ui != only) return;
    AntDesc a = ants[u.ant];
    MixedUnit mu = mus[ui];
    GmresCtx g;
    g.n = u.n;
    g.s = u.s;
    g.w = a.w;
    g.nc = a.n_crow;
    g.rows = u.n + a.n_crow;
    g.z = zbuf + u.z_off;
    g.y = rhs + u.rhs_off;
    g.cv = cosv + u.cos_off;
    g.rowwire = ibuf + a.rowwire_off;
    g.wptr = ibuf + a.wptr_off;
    g.wrow = ibuf + a.wrow_off;
    g.crows = crows + a.crow_off;
    g.lu = a32buf + mu.a32_off;
    g.piv = pivbuf + u.piv_off;
    if (binvbuf) g.binv = binvbuf + mu.binv_off;
    int s = g.s;
    cx *W = wbuf + mu.w_off;
    cx *b = W, *x = W + s, *r = W + 2 * s, *w = W + 3 * s;
    g.t = W + 4 * s;
    cx *V = vbuf + mu.v_off;
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    // staging vectors: shared memory when they fit, else the solve's work area
    cx *sv = staged ? reinterpret_cast<cx *>(s_dyn) : W + 4 * s + g.rows;
    cx *stv = sv + s;
    cx *sy = stv + g.rows;
    if (staged) {
        // the pivots' row permutation, built once: each preconditioner
        // application then gathers in parallel instead of swapping serially
        int32_t *perm = reinterpret_cast<int32_t *>(sy + s);
        for (int i = tid; i < s; i += blockDim.x) perm[i] = i;
        __syncthreads();
        if (tid == 0)
            for (int c = 0; c < s; ++c) {
                int p = g.piv[c];
                if (p != c) {
                    int t0 = perm[c];
                    perm[c] = perm[p];
                    perm[p] = t0;
                }
            }
        __syncthreads();
        g.perm = perm;
    }

    // b = M^H y (y is zero on the constraint rows), unless the Gram phase
    // of this run formed it with the same sums (k_gram32_ccols_mhy; use_b:
    // the factor is fresh, not a resident re-solve with new sources)
    if (!(use_b && mu.b_ready)) {
        for (int i = tid; i < g.rows; i += blockDim.x) g.t[i] = i < g.n ? g.y[i] : cx{0, 0};
        __syncthreads();
        for (int c = tid; c < g.n; c += blockDim.x) {
            cx acc = {0, 0};
            for (int rr = 0; rr < g.n; ++rr) acc = zadd(acc, zcmul(ld_z(g.z + (int64_t)rr * g.n + c), g.t[rr]));
            b[c] = acc;
        }
        for (int q = tid; q < g.w; q += blockDim.x) {
            cx acc = {0, 0};
            for (int k = g.wptr[q]; k < g.wptr[q + 1]; ++k) acc = zadd(acc, zscale(g.t[g.wrow[k]], -g.cv[g.wrow[k]]));
            b[g.n + q] = acc;
        }
    }
    // x0 = 0: the first cycle's residual is b itself (no operator pass), and
    // its first Krylov vector P^-1 b is the classical first guess
    for (int i = tid; i < s; i += blockDim.x) x[i] = {0, 0};
    __syncthreads();
    double bnorm = 0.0;  // |P^-1 b|, the scale of the preconditioned residual
    int iters = 0;
    double rel = 1.0;
    for (int outer = 0; outer < MAX_OUTER; ++outer) {
        if (outer == 0) {
            apply_prec(g, b, V, sy);
        } else {
            apply_A(g, x, w, sv, stv, sy);
            for (int i = tid; i < s; i += blockDim.x) r[i] = zsub(b[i], w[i]);
            __syncthreads();
            apply_prec(g, r, V, sy);
        }
        double beta = vnorm(V, s, red);
        if (outer == 0) bnorm = beta;
        rel = bnorm > 0 ? beta / bnorm : 0.0;
        if (rel <= GMRES_TOL || beta == 0.0) break;
        for (int i = tid; i < s; i += blockDim.x) V[i] = zscale(V[i], 1.0 / beta);
        if (tid == 0) {
            sg[0] = {beta, 0};
            for (int q = 1; q <= GM; ++q) sg[q] = {0, 0};
            s_stop = 0;
        }
        __syncthreads();
        int jend = GM - 1;
        for (int j = 0; j < GM; ++j) {
            cx *vj = V + (int64_t)j * s, *vn = V + (int64_t)(j + 1) * s;
            apply_A(g, vj, w, sv, stv, sy);
            apply_prec(g, w, vn, sy);
            // classical Gram-Schmidt, twice
            if (tid <= j) sh[tid] = {0, 0};
            __syncthreads();
            for (int pass = 0; pass < 2; ++pass) {
                for (int i = wid; i <= j; i += nw) {
                    const cx *vi = V + (int64_t)i * s;
                    cx acc = {0, 0};
                    for (int k = lane; k < s; k += 32) acc = zadd(acc, zcmul(vi[k], vn[k]));
                    acc = warp_sum(acc);
                    if (lane == 0) sH[i * GM + j] = acc;  // this pass's coefficient
                }
                __syncthreads();
                for (int k = tid; k < s; k += blockDim.x) {
                    cx v = vn[k];
                    for (int i = 0; i <= j; ++i) v = zsub(v, zmul(sH[i * GM + j], V[(int64_t)i * s + k]));
                    vn[k] = v;
                }
                if (tid <= j) sh[tid] = zadd(sh[tid], sH[tid * GM + j]);
                __syncthreads();
            }
            if (tid <= j) sH[tid * GM + j] = sh[tid];
            double hn = vnorm(vn, s, red);
            if (tid == 0) {
                sH[(j + 1) * GM + j] = {hn, 0};
                // previous rotations
                for (int i = 0; i < j; ++i) {
                    cx h0 = sH[i * GM + j], h1 = sH[(i + 1) * GM + j];
                    cx t0 = zadd(zscale(h0, scs[i]), zmul(ssn[i], h1));
                    cx sc = {ssn[i].re, -ssn[i].im};
                    sH[(i + 1) * GM + j] = zsub(zscale(h1, scs[i]), zmul(sc, h0));
                    sH[i * GM + j] = t0;
                }
                cx aa = sH[j * GM + j];
                double bb = hn;
                double na = sqrt(aa.re * aa.re + aa.im * aa.im);
                double nu = sqrt(na * na + bb * bb);
                double c;
                cx sn;
                if (na == 0.0) {
                    c = 0.0;
                    sn = {1.0, 0.0};
                    sH[j * GM + j] = {bb, 0};
                } else {
                    c = na / nu;
                    cx ph = {aa.re / na, aa.im / na};
                    sn = zscale(ph, bb / nu);
                    sH[j * GM + j] = zscale(ph, nu);
                }
                scs[j] = c;
                ssn[j] = sn;
                cx gj = sg[j];
                cx sc = {sn.re, -sn.im};
                sg[j + 1] = zscale(zmul(sc, gj), -1.0);
                sg[j] = zscale(gj, c);
                double res = sqrt(sg[j + 1].re * sg[j + 1].re + sg[j + 1].im * sg[j + 1].im);
                s_stop = (res <= GMRES_TOL * bnorm || hn == 0.0) ? 1 : 0;
            }
            __syncthreads();
            if (hn > 0.0)
                for (int k = tid; k < s; k += blockDim.x) vn[k] = zscale(vn[k], 1.0 / hn);
            __syncthreads();
            ++iters;
            if (s_stop) {
                jend = j;
                break;
            }
        }
        // solve the (jend+1) upper triangular system, x += V y
        if (tid == 0) {
            for (int i = jend; i >= 0; --i) {
                cx acc = sg[i];
                for (int k = i + 1; k <= jend; ++k) acc = zsub(acc, zmul(sH[i * GM + k], sh[k]));
                sh[i] = zdiv(acc, sH[i * GM + i]);
            }
        }
        __syncthreads();
        for (int k = tid; k < s; k += blockDim.x) {
            cx v = x[k];
            for (int i = 0; i <= jend; ++i) v = zadd(v, zmul(sh[i], V[(int64_t)i * s + k]));
            x[k] = v;
        }
        __syncthreads();
        // a cycle that met the tolerance ends the refinement on GMRES's own
        // residual estimate (|g_{j+1}|, the preconditioned residual of x in
        // FP64 with twice-orthogonalised Krylov vectors); a cycle that ran
        // out of vectors restarts from the explicit residual b - A x
        if (s_stop) {
            const cx gl = sg[jend + 1];
            rel = bnorm > 0 ? sqrt(gl.re * gl.re + gl.im * gl.im) / bnorm : 0.0;
            break;
        }
    }
    for (int i = tid; i < s; i += blockDim.x) xbuf[u.x_off + i] = x[i];
    if (tid == 0) {
        mus[ui].iters = iters;
        mus[ui].resid = rel;
    }
}


// ---------------------------------------------------------------------------
// GMRES for large systems: the same iteration as k_gmres_ir, spread over
// the whole GPU (one cooperative launch per solve).  Every CTA runs the
// same control flow; scalars (inner products, norms, the Hessenberg
// column, the Givens rotations, the stopping test) are reduced in a fixed
// order and recomputed identically in every CTA, so all CTAs take the same
// branches.  Vectors are split element-wise over all threads; the phases
// that read another CTA's elements are separated by grid barriers
// (fnec_grid.cuh) and read through L2.
//   A v      row pass t = M v (a warp per row), then M^H t as column sums
//            over row chunks (a warp per 64 columns x GG_RC rows) reduced
//            in chunk order, plus the sparse constraint and cos columns
//   P^-1     gather through the factor's row permutation, then blocked
//            forward / backward substitution: the owner CTA of each 32-row
//            block solves its diagonal block, one barrier, every CTA
//            updates the blocks it owns
// ---------------------------------------------------------------------------
constexpr int GG_RC = 256;           // rows per column-sum chunk of M^H t
constexpr int GG_MIN_S = 1536;       // solves this large go grid-wide ...
constexpr int GG_MAX_SOLVES = 16;    // ... when there are at most this many
constexpr int GG_MAX_CTAS = 296;

__device__ __forceinline__ cx ldcg_cx(const cx *p) {
    double2 d = __ldcg(reinterpret_cast<const double2 *>(p));
    return {d.x, d.y};
}

struct GGrid {
    GmresCtx g;
    const int32_t *ccptr, *ccq, *perm;
    cx *part;
    cx *y;
    cx *red;
    GridSync *gs;
    int32_t *status;
    int G, cta, tid, lane, wid, gt, T, gw, TW;
    int rc;       // rows per column-sum chunk of M^H t
    int cluster;  // 1: the G CTAs are one thread-block cluster (hardware barrier)
    unsigned epoch, redk;
};

// Rows per column-sum chunk: enough (column block, row chunk) items to keep
// every warp busy, at least 32 rows and at most 256.
__host__ __device__ __forceinline__ int gg_row_chunk(int n, int total_warps) {
    int ncb = (n + 63) / 64;
    int rc = (int)(((int64_t)n * ncb + 4 * total_warps - 1) / (4 * total_warps));
    return rc < 32 ? 32 : (rc > 256 ? 256 : rc);
}

__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ bool gg_sync(GGrid &c) {
    if (c.cluster) {  // a hardware barrier: every CTA of the cluster takes the same path
        cluster_barrier();
        return true;
    }
    if (grid_barrier(c.gs, (unsigned)c.G, ++c.epoch)) return true;
    if (c.tid == 0) atomicExch(c.status, FNEC_STATUS_GRID_TIMEOUT);
    return false;
}
#define GG_SYNC(c)          \
    if (!gg_sync(c)) return false

// out = M^H (M v) + lambda v; with v == nullptr, out = M^H [y; 0] (the
// right-hand side b).
__device__ bool gg_apply(GGrid &c, const cx *v, cx *out) {
    const GmresCtx &g = c.g;
    if (v) {
        for (int r = c.gw; r < g.n; r += c.TW) {
            const cx *zr = g.z + (int64_t)r * g.n;
            cx acc = {0, 0};
#pragma unroll 4
            for (int col = c.lane; col < g.n; col += 32) acc = zadd(acc, zmul(zr[col], ldcg_cx(v + col)));
            acc = warp_sum(acc);
            if (c.lane == 0) {
                cx cvv = ldcg_cx(v + g.n + g.rowwire[r]);
                g.t[r] = {acc.re - g.cv[r] * cvv.re, acc.im - g.cv[r] * cvv.im};
            }
        }
        for (int q = c.gt; q < g.nc; q += c.T) {
            DevConRow cr = g.crows[q];
            cx val = ldcg_cx(v + cr.c0);
            if (cr.c1 >= 0) val = zadd(val, zscale(ldcg_cx(v + cr.c1), cr.v1));
            g.t[g.n + q] = val;
        }
    } else {
        for (int r = c.gt; r < g.n; r += c.T) g.t[r] = g.y[r];
        for (int q = c.gt; q < g.nc; q += c.T) g.t[g.n + q] = {0, 0};
    }
    GG_SYNC(c);
    const int ncb = (g.n + 63) / 64, nch = (g.n + c.rc - 1) / c.rc;
    for (int it = c.gw; it < ncb * nch; it += c.TW) {
        int cb = it % ncb, ch = it / ncb;
        int c0 = cb * 64 + c.lane, c1 = c0 + 32;
        int r0 = ch * c.rc, r1 = min(g.n, r0 + c.rc);
        cx a0 = {0, 0}, a1 = {0, 0};
        if (c1 < g.n) {
            for (int r = r0; r < r1; ++r) {
                cx tr = ldcg_cx(g.t + r);
                const cx *zr = g.z + (int64_t)r * g.n;
                a0 = zadd(a0, zcmul(zr[c0], tr));
                a1 = zadd(a1, zcmul(zr[c1], tr));
            }
        } else if (c0 < g.n) {
            for (int r = r0; r < r1; ++r) a0 = zadd(a0, zcmul(g.z[(int64_t)r * g.n + c0], ldcg_cx(g.t + r)));
        }
        if (c0 < g.n) c.part[(int64_t)ch * g.n + c0] = a0;
        if (c1 < g.n) c.part[(int64_t)ch * g.n + c1] = a1;
    }
    GG_SYNC(c);
    for (int col = c.gt; col < g.n; col += c.T) {
        cx acc = {0, 0};
        for (int ch = 0; ch < nch; ++ch) acc = zadd(acc, ldcg_cx(c.part + (int64_t)ch * g.n + col));
        for (int k = c.ccptr[col]; k < c.ccptr[col + 1]; ++k) {
            int q = c.ccq[k];
            DevConRow cr = g.crows[q];
            double coef = (cr.c0 == col ? 1.0 : 0.0) + (cr.c1 == col ? cr.v1 : 0.0);
            acc = zadd(acc, zscale(ldcg_cx(g.t + g.n + q), coef));
        }
        if (v) acc = zadd(acc, zscale(ldcg_cx(v + col), 1e-8));
        out[col] = acc;
    }
    for (int w = c.gt; w < g.w; w += c.T) {
        cx acc = {0, 0};
        for (int k = g.wptr[w]; k < g.wptr[w + 1]; ++k) {
            int r = g.wrow[k];
            acc = zadd(acc, zscale(ldcg_cx(g.t + r), -g.cv[r]));
        }
        if (v) acc = zadd(acc, zscale(ldcg_cx(v + g.n + w), 1e-8));
        out[g.n + w] = acc;
    }
    GG_SYNC(c);
    return true;
}

// out = (L U)^-1 P in (the caller has synchronised after writing in);
// FP64 substitution with the FP32 factor, as apply_prec.
__device__ bool gg_prec(GGrid &c, const cx *in, cx *out) {
    const GmresCtx &g = c.g;
    const int s = g.s, nblk = (s + 31) / 32;
    __shared__ cx s_yb[32];
    for (int i = c.gt; i < s; i += c.T) c.y[i] = ldcg_cx(in + c.perm[i]);
    GG_SYNC(c);
    // forward, unit lower triangular
    for (int bk = 0; bk < nblk; ++bk) {
        const int c0 = bk * 32, nb = min(32, s - c0);
        if (bk % c.G == c.cta && c.wid == 0) {
            cx yl = c.lane < nb ? ldcg_cx(c.y + c0 + c.lane) : cx{0, 0};
            const float2 *lrow = g.lu + (int64_t)(c0 + (c.lane < nb ? c.lane : 0)) * s + c0;
#pragma unroll 1
            for (int q8 = 0; q8 < 32; q8 += 8) {
                float2 lr[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) lr[q] = (q8 + q < nb) ? lrow[q8 + q] : cf(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    double yr = __shfl_sync(0xffffffffu, yl.re, q8 + q), yi = __shfl_sync(0xffffffffu, yl.im, q8 + q);
                    if (c.lane > q8 + q && c.lane < nb) yl = zsub(yl, zmul(f2z(lr[q]), cx{yr, yi}));
                }
            }
            if (c.lane < nb) c.y[c0 + c.lane] = yl;
        }
        GG_SYNC(c);
        if (c.tid < nb) s_yb[c.tid] = ldcg_cx(c.y + c0 + c.tid);
        __syncthreads();
        // owned blocks q > bk: q = bk+1+d with q % G == cta
        int q0 = bk + 1 + ((c.cta - (bk + 1)) % c.G + c.G) % c.G;
        int nown = q0 < nblk ? (nblk - 1 - q0) / c.G + 1 : 0;
        for (int e = c.tid; e < nown * 32; e += blockDim.x) {
            int r = (q0 + (e >> 5) * c.G) * 32 + (e & 31);
            if (r >= s) continue;
            const float2 *lrow = g.lu + (int64_t)r * s + c0;
            cx acc = ldcg_cx(c.y + r);
            if (nb == 32) {
#pragma unroll
                for (int k8 = 0; k8 < 32; k8 += 8) {
                    float2 lr[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) lr[k] = lrow[k8 + k];
#pragma unroll
                    for (int k = 0; k < 8; ++k) acc = zsub(acc, zmul(f2z(lr[k]), s_yb[k8 + k]));
                }
            } else {
                for (int k = 0; k < nb; ++k) acc = zsub(acc, zmul(f2z(lrow[k]), s_yb[k]));
            }
            c.y[r] = acc;
        }
        __syncthreads();
    }
    // backward, upper triangular with its diagonal
    for (int bk = nblk - 1; bk >= 0; --bk) {
        const int c0 = bk * 32, nb = min(32, s - c0);
        if (bk % c.G == c.cta && c.wid == 0) {
            cx yl = c.lane < nb ? ldcg_cx(c.y + c0 + c.lane) : cx{0, 0};
            const float2 *urow = g.lu + (int64_t)(c0 + (c.lane < nb ? c.lane : 0)) * s + c0;
#pragma unroll 1
            for (int q8 = 24; q8 >= 0; q8 -= 8) {
                float2 ur[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) ur[q] = (q8 + q < nb) ? urow[q8 + q] : cf(1.f, 0.f);
#pragma unroll
                for (int q = 7; q >= 0; --q) {
                    const int qq = q8 + q;
                    if (qq < nb) {
                        if (c.lane == qq) yl = zdiv(yl, f2z(ur[q]));
                        double yr = __shfl_sync(0xffffffffu, yl.re, qq), yi = __shfl_sync(0xffffffffu, yl.im, qq);
                        if (c.lane < qq) yl = zsub(yl, zmul(f2z(ur[q]), cx{yr, yi}));
                    }
                }
            }
            if (c.lane < nb) c.y[c0 + c.lane] = yl;
        }
        GG_SYNC(c);
        if (bk == 0) break;
        if (c.tid < nb) s_yb[c.tid] = ldcg_cx(c.y + c0 + c.tid);
        __syncthreads();
        // owned blocks q < bk: q = cta, cta + G, ...
        int nown = c.cta < bk ? (bk - 1 - c.cta) / c.G + 1 : 0;
        for (int e = c.tid; e < nown * 32; e += blockDim.x) {
            int r = (c.cta + (e >> 5) * c.G) * 32 + (e & 31);
            const float2 *urow = g.lu + (int64_t)r * s + c0;
            cx acc = ldcg_cx(c.y + r);
            if (nb == 32) {
#pragma unroll
                for (int k8 = 0; k8 < 32; k8 += 8) {
                    float2 ur[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) ur[k] = urow[k8 + k];
#pragma unroll
                    for (int k = 0; k < 8; ++k) acc = zsub(acc, zmul(f2z(ur[k]), s_yb[k8 + k]));
                }
            } else {
                for (int k = 0; k < nb; ++k) acc = zsub(acc, zmul(f2z(urow[k]), s_yb[k]));
            }
            c.y[r] = acc;
        }
        __syncthreads();
    }
    for (int i = c.gt; i < s; i += c.T) out[i] = ldcg_cx(c.y + i);
    GG_SYNC(c);
    return true;
}

// h[i] = <V_i, vn> for i <= j (h in shared memory, identical in every CTA)
__device__ bool gg_dots(GGrid &c, const cx *V, int j, const cx *vn, cx *h, cx (*s_wp)[GM + 1]) {
    const int s = c.g.s;
    cx *red = c.red + (size_t)(c.redk & 1) * c.G * (GM + 1);
    ++c.redk;
    for (int i = 0; i <= j; ++i) {
        const cx *vi = V + (int64_t)i * s;
        cx acc = {0, 0};
        for (int k = c.gt; k < s; k += c.T) acc = zadd(acc, zcmul(ldcg_cx(vi + k), ldcg_cx(vn + k)));
        acc = warp_sum(acc);
        if (c.lane == 0) s_wp[c.wid][i] = acc;
    }
    __syncthreads();
    if (c.tid <= j) {
        cx a = {0, 0};
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) a = zadd(a, s_wp[q][c.tid]);
        red[c.cta * (GM + 1) + c.tid] = a;
    }
    GG_SYNC(c);
    if (c.tid <= j) {
        cx a = {0, 0};
        for (int q = 0; q < c.G; ++q) a = zadd(a, ldcg_cx(red + q * (GM + 1) + c.tid));
        h[c.tid] = a;
    }
    __syncthreads();
    return true;
}

// |v| (identical in every CTA)
__device__ bool gg_norm(GGrid &c, const cx *v, double *out, double *s_red) {
    const int s = c.g.s;
    cx *red = c.red + (size_t)(c.redk & 1) * c.G * (GM + 1);
    ++c.redk;
    double a = 0;
    for (int k = c.gt; k < s; k += c.T) {
        cx x = ldcg_cx(v + k);
        a += x.re * x.re + x.im * x.im;
    }
    a = block_sum(a, s_red);
    if (c.tid == 0) red[c.cta * (GM + 1)] = {a, 0.0};
    GG_SYNC(c);
    if (c.tid == 0) {
        double t = 0;
        for (int q = 0; q < c.G; ++q) t += __ldcg(reinterpret_cast<const double *>(red + q * (GM + 1)));
        s_red[8] = sqrt(t);
    }
    __syncthreads();
    *out = s_red[8];
    __syncthreads();
    return true;
}

__device__ bool gmres_grid_body(GGrid &c, const UnitDesc &u, MixedUnit *mus, int ui, cx *xbuf, cx *W, cx *V) {
    __shared__ cx sH[(GM + 1) * GM];
    __shared__ double scs[GM];
    __shared__ cx ssn[GM];
    __shared__ cx sg[GM + 1];
    __shared__ cx sh[GM + 1];
    __shared__ cx shp[GM + 1];
    __shared__ cx s_wp[8][GM + 1];
    __shared__ double s_red[9];
    __shared__ int s_stop;
    const int s = c.g.s, tid = c.tid;
    cx *b = W, *x = W + s, *r = W + 2 * s, *w = W + 3 * s;
    if (!gg_apply(c, nullptr, b)) return false;
    if (!gg_prec(c, b, x)) return false;
    double bnorm;
    if (!gg_norm(c, x, &bnorm, s_red)) return false;
    int iters = 0;
    double rel = 1.0;
    for (int outer = 0; outer < MAX_OUTER; ++outer) {
        if (!gg_apply(c, x, w)) return false;
        for (int i = c.gt; i < s; i += c.T) r[i] = zsub(ldcg_cx(b + i), ldcg_cx(w + i));
        GG_SYNC(c);
        if (!gg_prec(c, r, V)) return false;
        double beta;
        if (!gg_norm(c, V, &beta, s_red)) return false;
        rel = bnorm > 0 ? beta / bnorm : 0.0;
        if (rel <= GMRES_TOL || beta == 0.0) break;
        for (int i = c.gt; i < s; i += c.T) V[i] = zscale(V[i], 1.0 / beta);
        if (tid == 0) {
            sg[0] = {beta, 0};
            for (int q = 1; q <= GM; ++q) sg[q] = {0, 0};
        }
        GG_SYNC(c);
        int jend = GM - 1;
        for (int j = 0; j < GM; ++j) {
            cx *vj = V + (int64_t)j * s, *vn = V + (int64_t)(j + 1) * s;
            if (!gg_apply(c, vj, w)) return false;
            if (!gg_prec(c, w, vn)) return false;
            if (tid <= j) sh[tid] = {0, 0};
            __syncthreads();
            for (int pass = 0; pass < 2; ++pass) {
                if (!gg_dots(c, V, j, vn, shp, s_wp)) return false;
                for (int k = c.gt; k < s; k += c.T) {
                    cx vv = vn[k];
                    for (int i = 0; i <= j; ++i) vv = zsub(vv, zmul(shp[i], V[(int64_t)i * s + k]));
                    vn[k] = vv;
                }
                if (tid <= j) sh[tid] = zadd(sh[tid], shp[tid]);
                __syncthreads();
            }
            if (tid <= j) sH[tid * GM + j] = sh[tid];
            double hn;
            if (!gg_norm(c, vn, &hn, s_red)) return false;
            if (tid == 0) {
                sH[(j + 1) * GM + j] = {hn, 0};
                for (int i = 0; i < j; ++i) {
                    cx h0 = sH[i * GM + j], h1 = sH[(i + 1) * GM + j];
                    cx t0 = zadd(zscale(h0, scs[i]), zmul(ssn[i], h1));
                    cx sc = {ssn[i].re, -ssn[i].im};
                    sH[(i + 1) * GM + j] = zsub(zscale(h1, scs[i]), zmul(sc, h0));
                    sH[i * GM + j] = t0;
                }
                cx aa = sH[j * GM + j];
                double bb = hn;
                double na = sqrt(aa.re * aa.re + aa.im * aa.im);
                double nu = sqrt(na * na + bb * bb);
                double cc;
                cx sn;
                if (na == 0.0) {
                    cc = 0.0;
                    sn = {1.0, 0.0};
                    sH[j * GM + j] = {bb, 0};
                } else {
                    cc = na / nu;
                    cx ph = {aa.re / na, aa.im / na};
                    sn = zscale(ph, bb / nu);
                    sH[j * GM + j] = zscale(ph, nu);
                }
                scs[j] = cc;
                ssn[j] = sn;
                cx gj = sg[j];
                cx sc = {sn.re, -sn.im};
                sg[j + 1] = zscale(zmul(sc, gj), -1.0);
                sg[j] = zscale(gj, cc);
                double res = sqrt(sg[j + 1].re * sg[j + 1].re + sg[j + 1].im * sg[j + 1].im);
                s_stop = (res <= GMRES_TOL * bnorm || hn == 0.0) ? 1 : 0;
            }
            __syncthreads();
            if (hn > 0.0)
                for (int k = c.gt; k < s; k += c.T) vn[k] = zscale(vn[k], 1.0 / hn);
            GG_SYNC(c);
            ++iters;
            if (s_stop) {
                jend = j;
                break;
            }
        }
        if (tid == 0) {
            for (int i = jend; i >= 0; --i) {
                cx acc = sg[i];
                for (int k = i + 1; k <= jend; ++k) acc = zsub(acc, zmul(sH[i * GM + k], sh[k]));
                sh[i] = zdiv(acc, sH[i * GM + i]);
            }
        }
        __syncthreads();
        for (int k = c.gt; k < s; k += c.T) {
            cx vv = x[k];
            for (int i = 0; i <= jend; ++i) vv = zadd(vv, zmul(sh[i], V[(int64_t)i * s + k]));
            x[k] = vv;
        }
        GG_SYNC(c);
    }
    for (int i = c.gt; i < s; i += c.T) xbuf[u.x_off + i] = x[i];
    if (c.cta == 0 && tid == 0) {
        mus[ui].iters = iters;
        mus[ui].resid = rel;
    }
    return true;
}

__global__ void __launch_bounds__(256) k_gmres_grid(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                                                    MixedUnit *mus, int ui, const int32_t *__restrict__ ibuf,
                                                    const DevConRow *__restrict__ crows, const cx *__restrict__ zbuf,
                                                    const cx *__restrict__ rhs, const double *__restrict__ cosv,
                                                    const float2 *__restrict__ a32buf, const int32_t *__restrict__ pivbuf,
                                                    cx *xbuf, cx *vbuf, cx *wbuf, int32_t *status,
                                                    const int32_t *__restrict__ perm, cx *part, cx *ybuf, cx *red,
                                                    GridSync *gs) {
    UnitDesc u = units[ui];
    if (status[u.sys] != 0) return;
    AntDesc a = ants[u.ant];
    MixedUnit mu = mus[ui];
    GGrid c;
    c.g.n = u.n;
    c.g.s = u.s;
    c.g.w = a.w;
    c.g.nc = a.n_crow;
    c.g.rows = u.n + a.n_crow;
    c.g.z = zbuf + u.z_off;
    c.g.y = rhs + u.rhs_off;
    c.g.cv = cosv + u.cos_off;
    c.g.rowwire = ibuf + a.rowwire_off;
    c.g.wptr = ibuf + a.wptr_off;
    c.g.wrow = ibuf + a.wrow_off;
    c.g.crows = crows + a.crow_off;
    c.g.lu = a32buf + mu.a32_off;
    c.g.piv = pivbuf + u.piv_off;
    cx *W = wbuf + mu.w_off;
    c.g.t = W + 4 * u.s;
    c.ccptr = ibuf + a.ccptr_off;
    c.ccq = ibuf + a.ccq_off;
    c.perm = perm;
    c.part = part;
    c.y = ybuf;
    c.red = red;
    c.gs = gs;
    c.status = &status[u.sys];
    c.G = gridDim.x;
    c.cta = blockIdx.x;
    c.tid = threadIdx.x;
    c.lane = threadIdx.x & 31;
    c.wid = threadIdx.x >> 5;
    c.gt = blockIdx.x * blockDim.x + threadIdx.x;
    c.T = gridDim.x * blockDim.x;
    c.gw = c.gt >> 5;
    c.TW = c.T >> 5;
    c.epoch = 0;
    c.redk = 0;
    c.rc = GG_RC;
    c.cluster = 0;
    gmres_grid_body(c, u, mus, ui, xbuf, W, vbuf + mu.v_off);
}

constexpr int GC_MAX_S = 8192;  // cluster GMRES: the permutation is built in shared memory

// Scratch (complex128 units) of one solve of the cluster GMRES: column-sum
// partials, the substitution vector, the reduction slots and the row
// permutation (int32).
__host__ __device__ __forceinline__ int64_t gc_scratch(int n, int s, int C) {
    int rc = gg_row_chunk(n, C * 8);
    int64_t nch = (n + rc - 1) / rc;
    return nch * n + s + 2LL * C * (GM + 1) + (s + 3) / 4;
}

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// The grid-wide GMRES iteration on one thread-block cluster per solve: the
// cluster's C CTAs split the vectors and the matrix passes, synchronise with
// the hardware cluster barrier and exchange through L2.  Solves with S at or
// above skip_s (refined grid-wide) or above GC_MAX_S are left to the others.
__global__ void __launch_bounds__(256, 2) k_gmres_cluster(
    const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants, MixedUnit *mus,
    const int32_t *__restrict__ ibuf, const DevConRow *__restrict__ crows, const cx *__restrict__ zbuf,
    const cx *__restrict__ rhs, const double *__restrict__ cosv, const float2 *__restrict__ a32buf,
    const int32_t *__restrict__ pivbuf, cx *xbuf, cx *vbuf, cx *wbuf, int32_t *status, cx *cscratch, int C,
    int skip_s) {
    extern __shared__ int32_t s_pperm[];
    const int ui = blockIdx.x / C;
    UnitDesc u = units[ui];
    if (status[u.sys] != 0 || u.s >= skip_s || u.s > GC_MAX_S) return;  // the whole cluster leaves
    AntDesc a = ants[u.ant];
    MixedUnit mu = mus[ui];
    GGrid c;
    c.g.n = u.n;
    c.g.s = u.s;
    c.g.w = a.w;
    c.g.nc = a.n_crow;
    c.g.rows = u.n + a.n_crow;
    c.g.z = zbuf + u.z_off;
    c.g.y = rhs + u.rhs_off;
    c.g.cv = cosv + u.cos_off;
    c.g.rowwire = ibuf + a.rowwire_off;
    c.g.wptr = ibuf + a.wptr_off;
    c.g.wrow = ibuf + a.wrow_off;
    c.g.crows = crows + a.crow_off;
    c.g.lu = a32buf + mu.a32_off;
    c.g.piv = pivbuf + u.piv_off;
    cx *W = wbuf + mu.w_off;
    c.g.t = W + 4 * u.s;
    c.ccptr = ibuf + a.ccptr_off;
    c.ccq = ibuf + a.ccq_off;
    c.G = C;
    c.cta = (int)cluster_rank();
    c.tid = threadIdx.x;
    c.lane = threadIdx.x & 31;
    c.wid = threadIdx.x >> 5;
    c.gt = c.cta * blockDim.x + threadIdx.x;
    c.T = C * blockDim.x;
    c.gw = c.gt >> 5;
    c.TW = c.T >> 5;
    c.epoch = 0;
    c.redk = 0;
    c.rc = gg_row_chunk(u.n, C * 8);
    c.cluster = 1;
    c.gs = nullptr;
    c.status = &status[u.sys];
    cx *cs = cscratch + mu.cs_off;
    const int64_t nch = (u.n + c.rc - 1) / c.rc;
    c.part = cs;
    c.y = cs + nch * u.n;
    c.red = c.y + u.s;
    int32_t *perm = reinterpret_cast<int32_t *>(c.red + 2 * C * (GM + 1));
    c.perm = perm;
    if (c.cta == 0) {  // the factor's row permutation, applied in order in shared memory
        for (int i = threadIdx.x; i < u.s; i += blockDim.x) s_pperm[i] = i;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < u.s; ++k) {
                int p = c.g.piv[k];
                if (p >= 0 && p != k) {
                    int t0 = s_pperm[k];
                    s_pperm[k] = s_pperm[p];
                    s_pperm[p] = t0;
                }
            }
        __syncthreads();
        for (int i = threadIdx.x; i < u.s; i += blockDim.x) perm[i] = s_pperm[i];
    }
    cluster_barrier();
    gmres_grid_body(c, u, mus, ui, xbuf, W, vbuf + mu.v_off);
}

// The row permutation of the factor: perm[i] = source row of row i after
// the swaps piv[0..s) (applied in order, in shared memory when it fits).
__global__ void k_perm_from_piv(const UnitDesc *__restrict__ units, int ui, const int32_t *__restrict__ pivbuf,
                                int32_t *perm, int staged) {
    extern __shared__ int32_t s_perm_dyn[];
    UnitDesc u = units[ui];
    const int32_t *piv = pivbuf + u.piv_off;
    int32_t *s_perm = staged ? s_perm_dyn : perm;
    for (int i = threadIdx.x; i < u.s; i += blockDim.x) s_perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int c = 0; c < u.s; ++c) {
            int p = piv[c];
            if (p >= 0 && p != c) {
                int t0 = s_perm[c];
                s_perm[c] = s_perm[p];
                s_perm[p] = t0;
            }
        }
    __syncthreads();
    if (!staged) return;
    for (int i = threadIdx.x; i < u.s; i += blockDim.x) perm[i] = s_perm[i];
}

}  // namespace

bool mixed_available() { return true; }

cudaError_t alloc_mixed(MixedWork &w, const std::vector<UnitDesc> &systems, const std::vector<UnitDesc> &solves,
                        const std::vector<AntDesc> &ants, int max_s, const DevAlloc &dev, bool allow_grid) {
    std::vector<int64_t> a32_of(systems.size()), binv_of(systems.size());
    int64_t a32 = 0, v = 0, wk = 0, binv = 0;
    for (size_t i = 0; i < systems.size(); ++i) {
        a32_of[i] = a32;
        a32 += (int64_t)systems[i].s * systems[i].s;
        binv_of[i] = binv;
        binv += (int64_t)((systems[i].s + 31) / 32) * 2048;
    }
    std::vector<MixedUnit> mu(solves.size());
    for (size_t i = 0; i < solves.size(); ++i) {
        const UnitDesc &u = solves[i];
        int rows = u.n + ants[u.ant].n_crow;
        mu[i].a32_off = a32_of[u.sys];
        mu[i].binv_off = binv_of[u.sys];
        mu[i].v_off = v;
        mu[i].w_off = wk;
        mu[i].rows = rows;
        mu[i].iters = 0;
        mu[i].resid = 0.0;
        mu[i].cs_off = -1;
        mu[i].b_ready = 0;
        mu[i].first_solve = -1;
        v += (int64_t)(GM + 1) * u.s;
        wk += 6 * (int64_t)u.s + 2 * (int64_t)rows;  // 4 vectors + rows, then the unstaged copies
    }
    // systems' descriptors index the factor through the first solve's entry
    std::vector<MixedUnit> sysmu(systems.size());
    for (size_t i = 0; i < systems.size(); ++i) {
        sysmu[i].a32_off = a32_of[i];
        sysmu[i].binv_off = binv_of[i];
        sysmu[i].first_solve = -1;
        sysmu[i].b_ready = 0;
    }
    // systems whose M^H y the Gram phase forms with its cos columns
    // (k_gram32_ccols_mhy): few homogeneous columns and right-hand sides,
    // solves numbered consecutively
    w.mhy_systems = 0;
    w.mhy_max_n = 0;
    {
        std::vector<int> first(systems.size(), -1), count(systems.size(), 0);
        std::vector<char> consecutive(systems.size(), 1);
        for (size_t i = 0; i < solves.size(); ++i) {
            const int sy = solves[i].sys;
            if (first[sy] < 0) first[sy] = (int)i;
            else if (first[sy] + count[sy] != (int)i) consecutive[sy] = 0;
            ++count[sy];
        }
        for (size_t i = 0; i < systems.size(); ++i) {
            const UnitDesc &u = systems[i];
            const AntDesc &a = ants[u.ant];
            if (first[i] < 0 || !consecutive[i] || count[i] != u.n_rhs || u.n_rhs > CM_MAX_RHS || a.w > CM_MAX_W ||
                a.hom2 != 0)
                continue;
            sysmu[i].first_solve = first[i];
            for (int k = 0; k < count[i]; ++k) mu[first[i] + k].b_ready = 1;
            ++w.mhy_systems;
            w.mhy_max_n = std::max(w.mhy_max_n, u.n);
        }
    }
    size_t b_mu = sizeof(MixedUnit) * (mu.size() + 1);
    size_t b_smu = sizeof(MixedUnit) * (sysmu.size() + 1);
    size_t b_a32 = sizeof(float2) * (size_t)(a32 + 1);
    size_t b_v = sizeof(cx) * (size_t)(v + 1);
    size_t b_w = sizeof(cx) * (size_t)(wk + 1);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    size_t b_ord = sizeof(int32_t) * (solves.size() + 1);
    size_t b_binv = sizeof(float2) * (size_t)(binv + 1);
    std::vector<int2> btab;  // (system, 32-row block) of every diagonal block
    for (size_t i = 0; i < systems.size(); ++i)
        for (int k = 0; k < (systems[i].s + 31) / 32; ++k) btab.push_back(make_int2((int)i, k));
    size_t b_btab = sizeof(int2) * (btab.size() + 1);
    size_t total = al(b_mu) + al(b_smu) + al(b_a32) + al(b_v) + al(b_w) + al(b_ord) + al(b_binv) + al(b_btab);
    cudaError_t e = dev.alloc(&w.base, total);
    if (e != cudaSuccess) return e;
    unsigned char *p = (unsigned char *)w.base;
    // refinement CTAs take the largest solves first (longest-first
    // scheduling shortens the tail of the one-launch refinement)
    std::vector<int32_t> lpt(solves.size());
    for (size_t i = 0; i < lpt.size(); ++i) lpt[i] = (int32_t)i;
    std::stable_sort(lpt.begin(), lpt.end(), [&](int32_t x, int32_t y) {
        return (int64_t)solves[x].n * solves[x].n > (int64_t)solves[y].n * solves[y].n;
    });
    w.mu = (MixedUnit *)p;
    p += al(b_mu);
    w.smu = (MixedUnit *)p;
    p += al(b_smu);
    w.a32 = (float2 *)p;
    p += al(b_a32);
    w.v = (cx *)p;
    p += al(b_v);
    w.w = (cx *)p;
    p += al(b_w);
    w.s_order = (int32_t *)p;
    p += al(b_ord);
    w.binv = (float2 *)p;
    p += al(b_binv);
    w.binv_tab = (int2 *)p;
    w.n_binv = (int)btab.size();
    w.bytes = total;
    w.n_units = (int)solves.size();
    w.max_s = max_s;
    w.host = mu;
    w.grid_solves.clear();
    w.grid_s.clear();
    for (size_t i = 0; i < solves.size(); ++i)
        if (solves[i].s >= GG_MIN_S) {
            w.grid_solves.push_back((int)i);
            w.grid_s.push_back(solves[i].s);
        }
    if (w.grid_solves.size() > (size_t)GG_MAX_SOLVES || !allow_grid) {
        w.grid_solves.clear();
        w.grid_s.clear();
    }
    if (!w.grid_solves.empty()) {
        int64_t smax = 0, partmax = 0;
        for (int i : w.grid_solves) {
            const UnitDesc &u = solves[i];
            smax = std::max<int64_t>(smax, u.s);
            partmax = std::max<int64_t>(partmax, (int64_t)((u.n + GG_RC - 1) / GG_RC) * u.n);
        }
        size_t b_perm = sizeof(int32_t) * (size_t)smax, b_part = sizeof(cx) * (size_t)partmax,
               b_y = sizeof(cx) * (size_t)smax, b_red = sizeof(cx) * 2 * GG_MAX_CTAS * (GM + 1),
               b_sync = sizeof(GridSync) * w.grid_solves.size();
        size_t gt = al(b_perm) + al(b_part) + al(b_y) + al(b_red) + al(b_sync);
        e = dev.alloc(&w.grid_base, gt);
        if (e != cudaSuccess) return e;
        unsigned char *q = (unsigned char *)w.grid_base;
        w.g_perm = (int32_t *)q;
        q += al(b_perm);
        w.g_part = (cx *)q;
        q += al(b_part);
        w.g_y = (cx *)q;
        q += al(b_y);
        w.g_red = (cx *)q;
        q += al(b_red);
        w.g_sync = q;
        w.bytes += gt;
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gmres_grid, 256, 0);
        w.grid_ctas = std::min(GG_MAX_CTAS, sms * std::min(per_sm, 1));
    }
    {
        // cluster GMRES when one CTA per solve cannot fill the GPU
        int device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int capacity = 3 * sms;  // one-CTA solves resident at once (3 CTAs per SM)
        int C = 1;
        while (C < 8 && (int64_t)solves.size() * C * 2 <= capacity) C *= 2;
        w.cluster_max = C;
        w.cluster_c = 1;  // one CTA per solve unless the tuner measures better
        if (C > 1) {
            int64_t tot = 0;
            for (size_t i = 0; i < solves.size(); ++i) {
                mu[i].cs_off = tot;
                tot += gc_scratch(solves[i].n, solves[i].s, C);
            }
            e = dev.alloc(&w.c_base, sizeof(cx) * (size_t)(tot + 1));
            if (e != cudaSuccess) return e;
            w.c_scratch = (cx *)w.c_base;
            w.bytes += sizeof(cx) * (size_t)(tot + 1);
        }
    }
    {
        // tensor-core Gram: operand stacks, per-unit layout and the tile list
        TcGramPlan *p = new TcGramPlan();
        tc_gram_plan(systems, *p);
        if (!p->units.empty()) {
            size_t b_st = sizeof(float) * 32 * (size_t)p->rows;
            size_t b_gu = sizeof(TcGramUnit) * p->units.size(), b_t = sizeof(TcTile) * p->tiles.size();
            size_t tot = 2 * al(b_st) + al(b_gu) + al(b_t);
            e = dev.alloc(&w.tc_base, tot);
            if (e != cudaSuccess) {
                delete p;
                return e;
            }
            unsigned char *q = (unsigned char *)w.tc_base;
            w.tc_hi = (float *)q;
            q += al(b_st);
            w.tc_lo = (float *)q;
            q += al(b_st);
            w.tc_gu = q;
            q += al(b_gu);
            w.tc_tiles = q;
            w.bytes += tot;
            e = dev.upload(w.tc_gu, p->units.data(), b_gu);
            if (e == cudaSuccess) e = dev.upload(w.tc_tiles, p->tiles.data(), b_t);
            if (e != cudaSuccess) {
                delete p;
                return e;
            }
            if (!tc_gram_maps(*p, w.tc_hi, w.tc_lo)) {
                delete p;
                return cudaErrorNotSupported;  // no tensor-map encoder in this driver
            }
            for (const UnitDesc &u : systems) w.tc_max_n = std::max(w.tc_max_n, u.n);
            // the fill may write the stacks (one gram entry per system, same
            // index); their padding must then be zero once and for all
            w.tc_fusable = p->units.size() == systems.size();
            for (size_t q = 0; w.tc_fusable && q < p->units.size(); ++q) w.tc_fusable = p->units[q].unit == (int)q;
            if (w.tc_fusable) e = cudaMemsetAsync(w.tc_hi, 0, 2 * al(b_st), dev.st);
            if (e != cudaSuccess) {
                delete p;
                return e;
            }
            w.tc = p;
        } else {
            delete p;
        }
    }
    {
        // tensor-core trailing updates: units whose first trailing block has
        // at least TC_TRAIL_MIN_M rows, while it still does
        std::vector<int32_t> ord(systems.size());
        for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int32_t)i;
        std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) { return systems[x].s > systems[y].s; });
        std::vector<int> sd(ord.size());
        for (size_t i = 0; i < ord.size(); ++i) sd[i] = systems[ord[i]].s;
        int n_tc = 0;
        while (n_tc < (int)sd.size() && sd[n_tc] - 32 >= TC_TRAIL_MIN_M) ++n_tc;
        if (n_tc > 0 && w.tc) {
            TcTrailPlan *p = new TcTrailPlan();
            tc_trail_plan(sd, ord, n_tc, TC_TRAIL_MIN_M, *p);
            size_t b_st = sizeof(float) * 32 * (size_t)p->rows, b_u = sizeof(TcTrailUnit) * (p->units.size() + 1);
            size_t tot = 2 * al(b_st) + al(b_u);
            e = dev.alloc(&w.trail_base, tot);
            if (e != cudaSuccess) {
                delete p;
                return e;
            }
            unsigned char *q = (unsigned char *)w.trail_base;
            w.tr_hi = (float *)q;
            q += al(b_st);
            w.tr_lo = (float *)q;
            q += al(b_st);
            w.d_trail = q;
            w.bytes += tot;
            e = dev.upload(w.d_trail, p->units.data(), sizeof(TcTrailUnit) * p->units.size());
            if (e != cudaSuccess || !tc_trail_maps(*p, w.tr_hi, w.tr_lo)) {
                delete p;
                return e != cudaSuccess ? e : cudaErrorNotSupported;
            }
            w.trail = p;
            w.trail_n = n_tc;
        }
    }
    if (systems.size() >= 4 && !w.fmade) {  // concurrent factor groups
        bool ok = true;
        for (int g = 0; g + 1 < MixedWork::MAX_FACTOR_STREAMS && ok; ++g)
            ok = cudaStreamCreateWithFlags(&w.fstream[g], cudaStreamNonBlocking) == cudaSuccess;
        for (int g = 0; g < MixedWork::MAX_FACTOR_STREAMS && ok; ++g)
            ok = cudaEventCreateWithFlags(&w.fevent[g], cudaEventDisableTiming) == cudaSuccess;
        w.fmade = ok;
        if (!ok) (void)cudaGetLastError();  // one stream: the groups run in sequence
    }
    e = dev.upload(w.s_order, lpt.data(), sizeof(int32_t) * lpt.size());
    if (e == cudaSuccess && !btab.empty()) e = dev.upload(w.binv_tab, btab.data(), sizeof(int2) * btab.size());
    if (e == cudaSuccess) e = dev.upload(w.mu, mu.data(), sizeof(MixedUnit) * mu.size());
    if (e == cudaSuccess)
        e = dev.upload(w.smu, sysmu.data(), sizeof(MixedUnit) * sysmu.size());
    return e;
}

void free_mixed(MixedWork &w, const DevAlloc &dev) {
    for (auto &s : w.fstream)
        if (s) cudaStreamDestroy(s), s = nullptr;
    for (auto &e : w.fevent)
        if (e) cudaEventDestroy(e), e = nullptr;
    w.fmade = false;
    dev.release(w.base);
    dev.release(w.grid_base);
    dev.release(w.tc_base);
    dev.release(w.c_base);
    dev.release(w.trail_base);
    w.trail_base = nullptr;
    delete w.trail;
    w.trail = nullptr;
    w.trail_n = 0;
    w.c_base = nullptr;
    w.c_scratch = nullptr;
    w.grid_base = nullptr;
    w.tc_base = nullptr;
    delete w.tc;
    w.tc = nullptr;
    w.base = nullptr;
    w.bytes = 0;
}

// The FP64 GMRES refinement of every solve on the stored FP32 factor (the
// last part of run_mixed; also a resident system's re-solve with new
// right-hand sides, where the factor and its block inverses are reused:
// fresh_factor false).
uint64_t refine_mixed(MixedWork &mw, const UnitDesc *d_units, int nu, const UnitDesc *d_solves, int ns,
                      const AntDesc *d_ants, const int32_t *ibuf, const DevConRow *crows, const cx *z, const cx *rhs,
                      const double *cosv, cx *x, int32_t *piv, int32_t *status, int max_s, MixedMarks &marks,
                      cudaStream_t st, bool fresh_factor) {
    uint64_t L = 0;
    int max_rows = 0;
    for (size_t i = 0; i < mw.host.size(); ++i) max_rows = max_rows > mw.host[i].rows ? max_rows : mw.host[i].rows;
    size_t smem = sizeof(cx) * (size_t)(2 * max_s + max_rows) + sizeof(int32_t) * (size_t)max_s;  // + perm
    int staged = smem <= 200 * 1024;
    if (staged && smem > 0) {  // static + dynamic above 48 KB needs the raised limit
        int lim = std::min(set_smem_limit_once(k_gmres_ir<3>, 200 * 1024), set_smem_limit_once(k_gmres_ir<4>, 200 * 1024));
        if (lim < 0 || (size_t)lim < smem) staged = 0;
    }
    if (!staged) smem = 0;
    const bool grid_refine = mw.grid_on && !mw.grid_solves.empty();
    const int skip_s = grid_refine ? GG_MIN_S : INT_MAX;
    if (fresh_factor && mw.use_binv && nu > 0) {  // the preconditioner's diagonal block inverses
        if (mw.n_binv > 0) {
            k_block_inv32<<<(unsigned)mw.n_binv, 256, 0, st>>>(d_units, mw.smu, mw.a32, mw.binv, status, mw.binv_tab);
            ++L;
        }
    }
    int min_s = 0;  // solves below this are refined by the cluster kernel
    if (ns > 0 && mw.cluster_c > 1) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(ns * mw.cluster_c));
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = sizeof(int32_t) * (size_t)std::min(max_s, GC_MAX_S);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)mw.cluster_c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        set_smem_limit_once(k_gmres_cluster, (int)(sizeof(int32_t) * GC_MAX_S));
        if (cudaLaunchKernelEx(&cfg, k_gmres_cluster, d_solves, d_ants, mw.mu, ibuf, crows, (const cx *)z, rhs, cosv,
                               (const float2 *)mw.a32, (const int32_t *)piv, x, mw.v, mw.w, status, mw.c_scratch,
                               mw.cluster_c, skip_s) == cudaSuccess) {
            min_s = GC_MAX_S + 1;
            ++L;
        } else {
            (void)cudaGetLastError();  // clusters not schedulable: one CTA per solve
        }
    }
    if (ns > 0) {
        auto gk = mw.gmres_minb == 4 ? k_gmres_ir<4> : k_gmres_ir<3>;
        gk<<<ns, 256, smem, st>>>(d_solves, d_ants, mw.mu, ibuf, crows, z, rhs, cosv, mw.a32, piv, x, mw.v, mw.w, status,
                                  staged, skip_s, -1, min_s, mw.s_order, mw.use_binv ? mw.binv : nullptr,
                                  fresh_factor ? 1 : 0);
        cudaError_t le = cudaPeekAtLastError();
        if (le != cudaSuccess && !marks.detail[0])
            std::snprintf(marks.detail, sizeof(marks.detail), "GMRES launch: %d solves, %zu B shared (%s), max_s %d, rows %d",
                          ns, smem, staged ? "staged" : "unstaged", max_s, max_rows);
    }
    ++L;
    if (grid_refine) {
        cudaMemsetAsync(mw.g_sync, 0, sizeof(GridSync) * mw.grid_solves.size(), st);
        for (size_t k = 0; k < mw.grid_solves.size(); ++k) {
            int ui = mw.grid_solves[k];
            size_t psm = sizeof(int32_t) * (size_t)mw.grid_s[k];
            int pst = psm <= 200 * 1024;
            if (pst && psm > 0) {
                int lim = set_smem_limit_once(k_perm_from_piv, 200 * 1024);
                if (lim < 0 || (size_t)lim < psm) pst = 0;
            }
            if (!pst) psm = 0;
            k_perm_from_piv<<<1, 256, psm, st>>>(d_solves, ui, piv, mw.g_perm, pst);
            GridSync *gs = static_cast<GridSync *>(mw.g_sync) + k;
            MixedUnit *mus = mw.mu;
            float2 *a32 = mw.a32;
            cx *vb = mw.v, *wb = mw.w;
            const int32_t *perm = mw.g_perm;
            void *args[] = {(void *)&d_solves, (void *)&d_ants, (void *)&mus, (void *)&ui, (void *)&ibuf,
                            (void *)&crows, (void *)&z, (void *)&rhs, (void *)&cosv, (void *)&a32,
                            (void *)&piv, (void *)&x, (void *)&vb, (void *)&wb, (void *)&status,
                            (void *)&perm, (void *)&mw.g_part, (void *)&mw.g_y, (void *)&mw.g_red, (void *)&gs};
            if (mw.grid_ctas <= 0 ||
                launch_cooperative((const void *)k_gmres_grid, dim3(mw.grid_ctas), dim3(256), args, 0, st) !=
                    cudaSuccess) {
                (void)cudaGetLastError();  // not co-resident: refine this solve in one CTA
                k_gmres_ir<3><<<ns, 256, smem, st>>>(d_solves, d_ants, mw.mu, ibuf, crows, z, rhs, cosv, mw.a32, piv, x,
                                                  mw.v, mw.w, status, staged, INT_MAX, ui, 0, mw.s_order,
                                                  mw.use_binv ? mw.binv : nullptr, fresh_factor ? 1 : 0);
            }
            L += 2;
        }
    }
    return L;
}

uint64_t run_mixed(MixedWork &mw, const UnitDesc *d_units, int nu, const UnitDesc *d_solves, int ns,
                   const AntDesc *d_ants, const DevSeg *d_segs, const int4 *fill_tiles, int n_fill,
                   const int4 *gram_tiles, int n_gram, const int32_t *ibuf, const DevConRow *crows, cx *z,
                   const cx *rhs, const double *cosv, cx *x, int32_t *piv, int32_t *status, int max_s,
                   bool do_fill, int max_w, const GridPlan &gp, MixedMarks &marks, cudaStream_t st,
                   const DevStamp *stamps, int n_stamps) {
    uint64_t L = 0;
    static const char *const phase_name[4] = {"fill", "gram", "factor", "refinement"};
    auto mark = [&](int k) {
        if (!marks.failed_phase && cudaPeekAtLastError() != cudaSuccess) marks.failed_phase = phase_name[k];
        if (marks.ev) cudaEventRecord(marks.ev[k], st);
    };
    // the fill writes the Gram's tf32 operand stacks itself when the Gram
    // runs on the tensor cores and no stamp changes Z after the fill
    const bool fused_split = do_fill && n_fill > 0 && mw.tc && mw.use_tc && mw.tc_fusable && n_stamps == 0;
    if (do_fill && n_fill > 0) {
        k_fill_fast<<<n_fill, 256, 0, st>>>(d_units, d_ants, d_segs, fill_tiles, z,
                                            fused_split ? static_cast<const TcGramUnit *>(mw.tc_gu) : nullptr,
                                            mw.tc_hi, mw.tc_lo);
        ++L;
        if (n_stamps > 0) {  // LD loads on the diagonal, before Z is used
            launch_stamps(stamps, n_stamps, z, st);
            ++L;
        }
    }
    mark(0);
    if (mw.tc && mw.use_tc) {
        tc_gram_run(*mw.tc, d_units, static_cast<const TcGramUnit *>(mw.tc_gu), static_cast<const TcTile *>(mw.tc_tiles),
                    mw.smu, z, mw.tc_hi, mw.tc_lo, mw.a32, status, mw.tc_max_n, st, !fused_split, !mw.pivoting);
        ++L;
    } else if (n_gram > 0) {
        k_gram32_zz<<<n_gram, 256, 0, st>>>(d_units, mw.smu, gram_tiles, z, mw.a32);
    }
    {
        dim3 g(max_w > 0 ? max_w : 1, nu);
        k_gram32_ccols<<<g, 256, 0, st>>>(d_units, d_ants, mw.smu, ibuf, z, cosv, mw.a32);
    }
    if (mw.mhy_systems > 0) {
        dim3 g((unsigned)((mw.mhy_max_n + 255) / 256), (unsigned)nu);
        k_gram32_ccols_mhy<1><<<g, 256, 0, st>>>(d_units, d_solves, d_ants, mw.smu, mw.mu, ibuf, z, cosv, rhs, mw.a32,
                                                 mw.w);
        k_gram32_ccols_mhy<CM_MAX_RHS><<<g, 256, 0, st>>>(d_units, d_solves, d_ants, mw.smu, mw.mu, ibuf, z, cosv, rhs,
                                                          mw.a32, mw.w);
        L += 2;
    }
    k_gram32_rest<<<nu, 256, 0, st>>>(d_units, d_ants, mw.smu, ibuf, crows, mw.a32);
    L += 3;
    mark(1);
    // raised once per device (set_smem_limit_once)
    set_smem_limit_once((const void *)k_panel32_smem<256>, PANEL32_SMEM_MAX);
    set_smem_limit_once((const void *)k_panel32_smem<1024>, PANEL32_SMEM_MAX);
    set_smem_limit_once((const void *)k_panel32_grid, 96 * 1024);
    const int thr_rows = PANEL32_SMEM_MAX / (int)((MNB + 1) * sizeof(float2));
    const int32_t *ord = gp.d_order;
    if (gp.d_sync) cudaMemsetAsync(gp.d_sync, 0, grid_sync_bytes(gp.steps), st);
    // Units (in decreasing s) are split into up to factor_streams groups of
    // about equal work (sum of s^3), each factored on its own stream: the
    // column-serial panel chain of the tallest units then overlaps the
    // many short units' work instead of leaving the GPU idle.
    const int nu_all = (int)gp.s_desc.size();
    // no row exchanges on the Hermitian normal equations (k_panel32_herm)
    const bool herm = !mw.pivoting;
    // units with S <= FU_MAX_S (the tail of the order) are factored whole,
    // one CTA each, in one launch on a stream of their own
    int i_unit = nu_all;
    if (gp.unit_factor > 0)
        while (i_unit > 0 && gp.s_desc[i_unit - 1] <= fu_max_s(gp.unit_factor)) --i_unit;
    const bool unit_launch = i_unit < nu_all;
    int G = std::max(1, std::min(gp.factor_streams, MixedWork::MAX_FACTOR_STREAMS) - (unit_launch ? 1 : 0));
    if (!mw.fmade || i_unit < 2 * G) G = 1;
    std::vector<int> gb(1, 0);
    if (G > 1) {
        // units whose panels outgrow one CTA (grid-wide or global-memory
        // panels, one exchange area) all stay in the first group
        int n_tall = 0;
        while (!herm && n_tall < i_unit && gp.s_desc[n_tall] > thr_rows) ++n_tall;
        if (mw.trail && mw.use_tc_trail) n_tall = std::max(n_tall, std::min(mw.trail_n, i_unit));  // one stack set
        double tot = 0, acc = 0;
        for (int i = 0; i < i_unit; ++i) tot += (double)gp.s_desc[i] * gp.s_desc[i] * gp.s_desc[i];
        for (int i = 0; i < i_unit && (int)gb.size() < G; ++i) {
            acc += (double)gp.s_desc[i] * gp.s_desc[i] * gp.s_desc[i];
            if (acc >= tot * (double)gb.size() / G && i + 1 < i_unit && i + 1 >= n_tall) gb.push_back(i + 1);
        }
    }
    gb.push_back(i_unit);
    G = (int)gb.size() - 1;
    // streams: the per-step groups on st, fstream[0..G-2]; the whole-unit
    // launch on the next one (or st when there is no stream to spare)
    const bool unit_own = unit_launch && mw.fmade && G - 1 < MixedWork::MAX_FACTOR_STREAMS - 1 && i_unit > 0;
    const int n_side = (G - 1) + (unit_own ? 1 : 0);
    if (n_side > 0) {
        cudaEventRecord(mw.fevent[0], st);
        for (int g = 0; g < n_side; ++g) cudaStreamWaitEvent(mw.fstream[g], mw.fevent[0], 0);
    }
    if (unit_launch) {
        cudaStream_t us = unit_own ? mw.fstream[G - 1] : st;
        if (herm) {
            k_factor32_unit_herm<<<nu_all - i_unit, FU_THREADS, 0, us>>>(d_units, mw.smu, mw.a32, piv, status, ord,
                                                                         i_unit);
        } else {
            set_smem_limit_once((const void *)k_factor32_unit, (int)fu_smem(FU_MAX_S_ALL));
            const size_t fsm = fu_smem(gp.s_desc[i_unit]);  // the launch's largest unit
            k_factor32_unit<<<nu_all - i_unit, FU_THREADS, fsm, us>>>(d_units, mw.smu, mw.a32, piv, status, ord,
                                                                      i_unit);
        }
        ++L;
    }
    std::vector<StepClass> cls;
    const bool two_step = mw.two_step && !(mw.trail && mw.use_tc_trail);
    for (int grp = 0; grp < G && i_unit > 0; ++grp) {
    const int gi0 = gb[grp], gi1 = gb[grp + 1];
    cudaStream_t fs = grp == 0 ? st : mw.fstream[grp - 1];
    for (int c0 = 0; herm && gi0 < gi1 && c0 < gp.s_desc[gi0]; c0 += MNB) {
        // Hermitian factor: panel (diagonal block, L21, mirrored U12), then
        // the trailing tiles on and below the diagonal, per size class: the
        // largest units' on the tensor cores when tensor_trailing is on (a
        // prefix of the order, in the first group), the rest as SIMT tiles
        step_classes(gp, c0, gi0, cls, gi1);
        for (const StepClass &c : cls) {
            const int rows = c.m_max - MNB;
            if (rows > HERM_SPLIT_ROWS) {  // tall: the diagonal block, then the rows over many CTAs
                k_herm_diag<<<c.i1 - c.i0, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0);
                dim3 gr((unsigned)((rows + HERM_ROWS_CHUNK - 1) / HERM_ROWS_CHUNK), (unsigned)(c.i1 - c.i0));
                k_herm_rows<<<gr, HERM_ROWS_CHUNK, 0, fs>>>(d_units, mw.smu, c0, mw.a32, status, ord, c.i0);
                L += 2;
            } else if (rows > 256) {
                k_panel32_herm<1024><<<c.i1 - c.i0, 1024, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0);
                ++L;
            } else {
                k_panel32_herm<256><<<c.i1 - c.i0, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0);
                ++L;
            }
        }
        const int k_tc =
            (grp == 0 && mw.trail && mw.use_tc_trail) ? std::min(mw.trail->active(c0 / MNB), i_unit) : 0;
        step_classes(gp, c0, std::max(gi0, k_tc), cls, gi1);
        for (const StepClass &c : cls) {
            const int rows = c.m_max - MNB;
            if (rows <= 0) continue;
            const int T = (rows + 63) / 64;
            dim3 g2(T * (T + 1) / 2, c.i1 - c.i0);
            k_trailing32<<<g2, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, status, ord, c.i0, 1, INT_MAX, 1);
            ++L;
        }
        if (k_tc > 0) {
            tc_trail_run(*mw.trail, c0 / MNB, k_tc, static_cast<const TcTrailUnit *>(mw.d_trail), d_units, mw.smu, mw.a32,
                         mw.tr_hi, mw.tr_lo, status, fs, true);
            L += 3;
        }
    }
    for (int c0 = 0; !herm && gi0 < gi1 && c0 < gp.s_desc[gi0]; c0 += MNB) {
        // panels as in the plain path: tallest grid-wide (or one CTA from
        // global memory), the rest one CTA from shared memory per size class
        int n_thr = gi0;
        while (n_thr < gi1 && gp.s_desc[n_thr] - c0 > thr_rows) ++n_thr;
        n_thr -= gi0;  // only the first group (the tallest units) can have any
        if (n_thr > 0) {
            int Gp = 0;
            size_t gsm = 0;
            bool done = false;
            if (plan_grid_panel(gp, c0, thr_rows, MNB, sizeof(float2), (const void *)k_panel32_grid, &Gp, &gsm) ==
                n_thr) {
                PanelXchg<float2> *xg = static_cast<PanelXchg<float2> *>(gp.d_xchg);
                GridSync *gs = static_cast<GridSync *>(gp.d_sync) + (size_t)(c0 / MNB) * GRID_PANEL_MAX_UNITS;
                const MixedUnit *smu = mw.smu;
                float2 *a32 = mw.a32;
                void *args[] = {(void *)&d_units, (void *)&smu, (void *)&ord, (void *)&c0, (void *)&a32,
                                (void *)&piv, (void *)&status, (void *)&xg, (void *)&gs};
                done = launch_cooperative((const void *)k_panel32_grid, dim3(Gp, n_thr), dim3(256), args, gsm, fs) ==
                       cudaSuccess;
                if (!done) (void)cudaGetLastError();
            }
            if (!done) k_panel32<<<n_thr, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, INT_MAX, ord, gi0);
            ++L;
        }
        step_classes(gp, c0, gi0 + n_thr, cls, gi1);
        for (const StepClass &c : cls) {
            const size_t psm = sizeof(float2) * (size_t)c.m_max * (MNB + 1);
            if (c.m_max > 256)
                k_panel32_smem<1024><<<c.i1 - c.i0, 1024, psm, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, INT_MAX,
                                                                   ord, c.i0);
            else
                k_panel32_smem<256><<<c.i1 - c.i0, 256, psm, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, INT_MAX,
                                                                 ord, c.i0);
            ++L;
        }
        // Two-step pairs (two_step): the first step of a pair updates only
        // the next panel's 32 columns (look-ahead); the second step's swaps
        // run first on the L columns, then its trailing columns take the
        // owed update of the first step before U12 is solved, and one
        // trailing pass applies both steps (K = 64), reading and writing
        // A22 once per pair instead of once per step.
        const bool pair_first = two_step && (c0 / MNB) % 2 == 0;
        const bool pair_second = two_step && (c0 / MNB) % 2 == 1;
        step_classes(gp, c0, gi0, cls, gi1);
        for (const StepClass &c : cls) {
            int m = c.m_max;
            if (pair_second) {
                // the L columns first (the owed update reads them swapped) ...
                dim3 ga((c0 + 63) / 64, c.i1 - c.i0);
                k_swap_u12_32<<<ga, 64, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0, 0, 0, c0);
                // ... then the trailing columns with the owed update and U12
                dim3 gt((m + 63) / 64, c.i1 - c.i0);
                k_swap_u12_32<<<gt, 64, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0, 1, c0, -1);
                L += 2;
            } else {
                dim3 g1((m + c0 + 63) / 64, c.i1 - c.i0);  // every column outside the panel
                k_swap_u12_32<<<g1, 64, 0, fs>>>(d_units, mw.smu, c0, mw.a32, piv, status, ord, c.i0, 0, 0, -1);
                ++L;
            }
        }
        // trailing updates: the largest units' on the tensor cores (a prefix
        // of the order, in the first group), the rest as FP32 SIMT tiles
        // (never a unit factored whole: those are the order's tail from i_unit)
        const int k_tc =
            (grp == 0 && mw.trail && mw.use_tc_trail) ? std::min(mw.trail->active(c0 / MNB), i_unit) : 0;
        step_classes(gp, c0, std::max(gi0, k_tc), cls, gi1);
        for (const StepClass &c : cls) {
            int rows = c.m_max - MNB;
            if (rows <= 0) continue;
            if (pair_first) {  // the next panel's columns only
                dim3 g2((rows + 63) / 64, c.i1 - c.i0);
                k_trailing32<<<g2, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, status, ord, c.i0, 1, c0 + 2 * MNB, 0);
            } else if (pair_second) {  // both steps of the pair, from the pair's first column
                int t = ((rows + 63) / 64) * ((rows + 63) / 64);
                dim3 g2(t, c.i1 - c.i0);
                k_trailing32<<<g2, 256, 0, fs>>>(d_units, mw.smu, c0 - MNB, mw.a32, status, ord, c.i0, 2, INT_MAX, 0);
            } else {
                int t = ((rows + 63) / 64) * ((rows + 63) / 64);
                dim3 g2(t, c.i1 - c.i0);
                k_trailing32<<<g2, 256, 0, fs>>>(d_units, mw.smu, c0, mw.a32, status, ord, c.i0, 1, INT_MAX, 0);
            }
            ++L;
        }
        if (k_tc > 0) {
            tc_trail_run(*mw.trail, c0 / MNB, k_tc, static_cast<const TcTrailUnit *>(mw.d_trail), d_units, mw.smu, mw.a32,
                         mw.tr_hi, mw.tr_lo, status, fs);
            L += 3;
        }
    }
    }
    for (int g = 0; g < n_side; ++g) {  // join the side streams back into the batch stream
        cudaEventRecord(mw.fevent[g + 1], mw.fstream[g]);
        cudaStreamWaitEvent(st, mw.fevent[g + 1], 0);
    }
    mark(2);
    L += refine_mixed(mw, d_units, nu, d_solves, ns, d_ants, ibuf, crows, z, rhs, cosv, x, piv, status, max_s, marks,
                      st, true);
    mark(3);
    return L;
}

cudaError_t read_mixed_stats(MixedWork &mw, int32_t *iters, double *resid, cudaStream_t st) {
    if (!mw.base) return cudaSuccess;
    std::vector<MixedUnit> h(mw.n_units);
    cudaError_t e = cudaMemcpyAsync(h.data(), mw.mu, sizeof(MixedUnit) * h.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < mw.n_units; ++i) {
        if (iters) iters[i] = h[i].iters;
        if (resid) resid[i] = h[i].resid;
    }
    return cudaSuccess;
}

}  // namespace fnec

namespace {
__global__ void k_test_rsqrt(const double *x, int n, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = fnec::rsqrt_newton(x[i]);
}
}  // namespace

// The fill's reciprocal square root on the device (n <= 2^20 values, each
// normal, finite and > 0): staged through device memory of its own.
extern "C" int fnec_test_fill_rsqrt(const double *x, uint64_t n, double *out) {
    if (n && (!x || !out)) return FNEC_ERR_BAD_ARG;
    if (n > ((uint64_t)1 << 20)) return FNEC_ERR_TOO_LARGE;
    for (uint64_t i = 0; i < n; ++i)
        if (!(x[i] >= 2.2250738585072014e-308 && x[i] < INFINITY)) return FNEC_ERR_BAD_ARG;
    if (n == 0) return FNEC_OK;
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * 2 * n) != cudaSuccess) {
        (void)cudaGetLastError();
        return FNEC_ERR_OUT_OF_MEMORY;
    }
    cudaError_t e = cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_test_rsqrt<<<(unsigned)((n + 255) / 256), 256>>>(d, (int)n, d + n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? FNEC_OK : FNEC_ERR_CUDA;
}

extern "C" int fnec_test_fill_sincospi(const double *x, uint64_t n, double *sin_out, double *cos_out) {
    if ((n && (!x || !sin_out || !cos_out))) return FNEC_ERR_BAD_ARG;
    for (uint64_t i = 0; i < n; ++i) {
        if (!(x[i] >= 0.0 && x[i] < 1125899906842624.0)) return FNEC_ERR_BAD_ARG;  // [0, 2^50)
        fnec::sincospi_taylor(x[i], sin_out[i], cos_out[i]);
    }
    return FNEC_OK;
}

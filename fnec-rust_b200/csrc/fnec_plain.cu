// fnec_plain.cu -- plain FP64 Hallen kernels with bit-exact operation order.
//
// Every arithmetic operation below is one separately rounded IEEE
// operation (explicit _rn intrinsics; the file is also built with
// -fmad=false), issued in the order the reference issues it, and sin, cos
// and hypot return the platform libm's values (fnec_libm.cuh restates
// glibc's algorithms; the self term's ln comes from the host libm, see
// DevSeg::self_log).  Given the
// same inputs the Gram matrix, the elimination and the back substitution
// therefore reproduce the reference CPU path bit for bit; pivot order is
// chosen with the reference's "last maximum by hypot" rule.
//
// Kernels (one launch each, all units of a batch at once):
//   k_expand_segments  geometry.rs:710-754     one CTA per GW wire
//   k_hallen_rhs       excitation.rs:119-244   one CTA per unit
//   k_fill_exact       matrix.rs:186-331       16x16 tiles of Z, tile list
//   k_gram_zz          linear.rs:765-780       64x64 tiles of Z^H [Z | y]
//   k_gram_ccols       linear.rs:765-780       the -cos(k s) columns (sparse)
//   k_gram_finish      linear.rs:757-785       constraint rows, then +1e-8 I
//   k_panel            linear.rs:1343-1370     NB columns, one CTA per unit
//   k_panel_grid       linear.rs:1343-1370     NB columns of a tall panel, many CTAs
//   k_swap_u12         linear.rs:1358-1369     deferred swaps + U block row
//   k_trailing         linear.rs:1362-1369     A22 -= L21 U12, 64x64 tiles
//   k_backsub          linear.rs:1372-1381     one warp per unit
//   k_feedpoints       solve_session.rs:846-947
#include <algorithm>
#include <cstdio>
#include <climits>
#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>

#include "fnec_grid.cuh"
#include "fnec_kernels.h"
#include "fnec_libm.cuh"
#include "fnec_math.cuh"

namespace fnec {

// Gauss-Legendre tables as written in matrix.rs:39-72 (15 decimal digits).
__constant__ double c_gl_n4[4] = {-0.861136311594953, -0.339981043584856, 0.339981043584856,
                                  0.861136311594953};
__constant__ double c_gl_w4[4] = {0.347854845137454, 0.652145154862626, 0.652145154862626,
                                  0.347854845137454};
__constant__ double c_gl_n8[8] = {-0.960289856497536, -0.796666477413627, -0.525532409916329,
                                  -0.183434642495650, 0.183434642495650,  0.525532409916329,
                                  0.796666477413627,  0.960289856497536};
__constant__ double c_gl_w8[8] = {0.101228536290376, 0.222381034453374, 0.313706645877887,
                                  0.362683783378362, 0.362683783378362, 0.313706645877887,
                                  0.222381034453374, 0.101228536290376};

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
__global__ void k_expand_segments(const DevWire *__restrict__ wires, int nw, DevSeg *segs) {
    int w = blockIdx.x;
    if (w >= nw) return;
    DevWire gw = wires[w];
    double dx = D_SUB(gw.end[0], gw.start[0]);
    double dy = D_SUB(gw.end[1], gw.start[1]);
    double dz = D_SUB(gw.end[2], gw.start[2]);
    double wl = D_SQRT(D_ADD(D_ADD(D_MUL(dx, dx), D_MUL(dy, dy)), D_MUL(dz, dz)));
    double dir0 = D_DIV(dx, wl), dir1 = D_DIV(dy, wl), dir2 = D_DIV(dz, wl);
    double nn = (double)gw.nseg;
    double seg_len = D_DIV(wl, nn);
    for (uint32_t i = threadIdx.x; i < gw.nseg; i += blockDim.x) {
        double t0 = D_DIV((double)i, nn);
        double t1 = D_DIV(D_ADD((double)i, 1.0), nn);
        double tm = D_MUL(D_ADD(t0, t1), 0.5);
        DevSeg s;
        s.start[0] = D_ADD(gw.start[0], D_MUL(dx, t0));
        s.start[1] = D_ADD(gw.start[1], D_MUL(dy, t0));
        s.start[2] = D_ADD(gw.start[2], D_MUL(dz, t0));
        s.end[0] = D_ADD(gw.start[0], D_MUL(dx, t1));
        s.end[1] = D_ADD(gw.start[1], D_MUL(dy, t1));
        s.end[2] = D_ADD(gw.start[2], D_MUL(dz, t1));
        s.mid[0] = D_ADD(gw.start[0], D_MUL(dx, tm));
        s.mid[1] = D_ADD(gw.start[1], D_MUL(dy, tm));
        s.mid[2] = D_ADD(gw.start[2], D_MUL(dz, tm));
        s.dir[0] = dir0;
        s.dir[1] = dir1;
        s.dir[2] = dir2;
        s.len = seg_len;
        s.rad = gw.radius;
        s.tag = gw.tag;
        s.tag_index = i + 1;
        s.self_log = gw.self_log;
        segs[gw.seg_off + i] = s;
    }
}

// ---------------------------------------------------------------------------
// Hallen RHS: cos(k s_local) per merged conductor and the delta-gap term
// -j (2 pi / eta0) V sin(k |s - s_src|) on the source's conductor.
// ---------------------------------------------------------------------------
__global__ void k_hallen_rhs(const UnitDesc *__restrict__ solves, const AntDesc *__restrict__ ants,
                             const DevSeg *__restrict__ segs, const int32_t *__restrict__ ibuf,
                             const DevSource *__restrict__ srcs, const double *__restrict__ dtab,
                             cx *rhs_buf, double *cos_buf, double scale) {
    UnitDesc u = solves[blockIdx.x];  // one right-hand side
    AntDesc a = ants[u.ant];
    if (a.hom2) return;  // a receiving antenna: k_planewave_field / k_planewave_rhs
    const DevSeg *sg = segs + a.seg_off;
    const int32_t *comp = ibuf + a.comp_off;
    const int32_t *sptr = ibuf + a.sptr_off;
    const DevSource *src = srcs + a.src_off + sptr[u.rhs];
    int n_src = sptr[u.rhs + 1] - sptr[u.rhs];
    double k = u.k_fill;
    if (a.paths) {
        // build_hallen_rhs_paths (excitation.rs:264-341): cos(k s) and the
        // source terms along each path's signed arc length s, times the
        // traversal signs; every EX card drives its whole path
        const double *s_mid = dtab + a.arc_off, *sgn = s_mid + a.n;
        const int32_t *col = ibuf + a.rowwire_off;
        for (int m = threadIdx.x; m < a.n; m += blockDim.x) {
            if (u.rhs == 0) {
                double sn, cs;
                fnec_libm::libm_sincos(D_MUL(k, s_mid[m]), &sn, &cs);
                cos_buf[u.cos_off + m] = D_MUL(sgn[m], cs);
            }
            cx r = cx_make(0.0, 0.0);
            for (int q = 0; q < n_src; ++q) {
                DevSource s = src[q];
                if (col[m] != col[s.feed]) continue;
                double ds = fabs(D_SUB(s_mid[m], s_mid[s.feed]));
                double ss, sc;
                fnec_libm::libm_sincos(D_MUL(k, ds), &ss, &sc);
                cx t = cx_mul(cx_make(0.0, D_MUL(-scale, ss)), cx_make(s.v_re, s.v_im));
                double f = D_MUL(sgn[m], sgn[s.feed]);
                r = cx_add(r, cx_make(D_MUL(t.re, f), D_MUL(t.im, f)));
            }
            rhs_buf[u.rhs_off + m] = r;
        }
        return;
    }
    for (int m = threadIdx.x; m < a.n; m += blockDim.x) {
        int first = comp[2 * m], last = comp[2 * m + 1];
        const double *wd = sg[first].dir;
        double wm0 = D_DIV(D_ADD(sg[first].mid[0], sg[last].mid[0]), 2.0);
        double wm1 = D_DIV(D_ADD(sg[first].mid[1], sg[last].mid[1]), 2.0);
        double wm2 = D_DIV(D_ADD(sg[first].mid[2], sg[last].mid[2]), 2.0);
        double dl0 = D_SUB(sg[m].mid[0], wm0);
        double dl1 = D_SUB(sg[m].mid[1], wm1);
        double dl2 = D_SUB(sg[m].mid[2], wm2);
        double s_local = D_ADD(D_ADD(D_MUL(dl0, wd[0]), D_MUL(dl1, wd[1])), D_MUL(dl2, wd[2]));
        if (u.rhs == 0) {  // cos(k s) belongs to the system: written once
            double sn, cs;
            fnec_libm::libm_sincos(D_MUL(k, s_local), &sn, &cs);
            cos_buf[u.cos_off + m] = cs;
        }
        cx r = cx_make(0.0, 0.0);
        for (int q = 0; q < n_src; ++q) {
            DevSource s = src[q];
            if (m < s.comp_first || m > s.comp_last) continue;
            const DevSeg &f = sg[s.feed];
            double d0 = D_SUB(sg[m].mid[0], f.mid[0]);
            double d1 = D_SUB(sg[m].mid[1], f.mid[1]);
            double d2 = D_SUB(sg[m].mid[2], f.mid[2]);
            double sd = D_ADD(D_ADD(D_MUL(d0, f.dir[0]), D_MUL(d1, f.dir[1])), D_MUL(d2, f.dir[2]));
            double ss, sc;
            fnec_libm::libm_sincos(D_MUL(k, fabs(sd)), &ss, &sc);
            cx t = cx_mul(cx_make(0.0, D_MUL(-scale, ss)), cx_make(s.v_re, s.v_im));
            r = cx_add(r, t);
        }
        rhs_buf[u.rhs_off + m] = r;
    }
}

// ---------------------------------------------------------------------------
// Plane-wave forcing (planewave.rs:162-254 per wire, :278-348 per path).
// k_planewave_field: the tangential incident field of every segment for
// every incidence direction, E_p = sign_p (e . d_p) exp(+j k r_hat . r_p)
// with d_p the direction of the wire's first segment (per-wire form) or of
// the segment itself (path form); the solve's x vector holds it until the
// solve overwrites x.  Solve 0 of each system also writes cos(k s) and
// sin(k s), times the sign, as the two homogeneous columns.
// It also tabulates sin(k |s_m - s_p|) for the rows p of m's wire or path
// (ascending), which no incidence direction changes, after the two columns.
// k_planewave_rhs: rhs_m = sign_m (-j 2 pi / eta0) sum_p E_p sin(k |s_m -
// s_p|) dl_p over those rows in ascending order, reading the table.
// Every operation is the reference's, in its order; sign = 1 in the
// per-wire form, where multiplying by it is exact.
// ---------------------------------------------------------------------------
__global__ void k_planewave_field(const UnitDesc *__restrict__ solves, int ns, const AntDesc *__restrict__ ants,
                                  const DevSeg *__restrict__ segs, const int32_t *__restrict__ ibuf,
                                  const double *__restrict__ dtab, cx *xbuf, double *cos_buf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    for (int si = blockIdx.y; si < ns; si += gridDim.y) {  // solves beyond the grid's y limit
        UnitDesc u = solves[si];
        AntDesc a = ants[u.ant];
        if (!a.hom2 || p >= a.n) continue;
        const DevSeg *sg = segs + a.seg_off;
        const double *wv = dtab + a.wave_off + 10 * (int64_t)u.rhs;  // r_hat[3], pol re[3], pol im[3]
        const double *dir = a.paths ? sg[p].dir : sg[ibuf[a.comp_off + 2 * p]].dir;
        const double s = dtab[a.arc_off + p], sgn = dtab[a.arc_off + a.n + p];
        const double k = u.k_fill;
        cx coup = cx_make(0.0, 0.0);
        for (int c = 0; c < 3; ++c) coup = cx_add(coup, cx_make(D_MUL(wv[3 + c], dir[c]), D_MUL(wv[6 + c], dir[c])));
        const double phase = D_MUL(
            k, D_ADD(D_ADD(D_MUL(wv[0], sg[p].mid[0]), D_MUL(wv[1], sg[p].mid[1])), D_MUL(wv[2], sg[p].mid[2])));
        double sn, cs;
        fnec_libm::libm_sincos(phase, &sn, &cs);
        const cx e = cx_mul(coup, cx_make(D_MUL(1.0, cs), D_MUL(1.0, sn)));  // from_polar(1, phase)
        xbuf[u.x_off + p] = cx_make(D_MUL(e.re, sgn), D_MUL(e.im, sgn));
        if (u.rhs == 0) {
            double ss, sc;
            fnec_libm::libm_sincos(D_MUL(k, s), &ss, &sc);
            cos_buf[u.cos_off + p] = D_MUL(sgn, sc);
            cos_buf[u.cos_off + a.n + p] = D_MUL(sgn, ss);
            const int32_t col = ibuf[a.rowwire_off + p];
            const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
            double *kt = cos_buf + u.cos_off + 2 * (int64_t)a.n + ibuf[a.koff_off + p];
            for (int q = wptr[col]; q < wptr[col + 1]; ++q) {
                double ks, kc;
                fnec_libm::libm_sincos(D_MUL(k, fabs(D_SUB(s, dtab[a.arc_off + wrow[q]]))), &ks, &kc);
                kt[q - wptr[col]] = ks;
            }
        }
    }
}

__global__ void k_planewave_rhs(const UnitDesc *__restrict__ solves, int ns, const AntDesc *__restrict__ ants,
                                const DevSeg *__restrict__ segs, const int32_t *__restrict__ ibuf,
                                const double *__restrict__ dtab, const double *__restrict__ cos_buf,
                                const cx *__restrict__ xbuf, cx *rhs_buf, double scale) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    for (int si = blockIdx.y; si < ns; si += gridDim.y) {
        UnitDesc u = solves[si];
        AntDesc a = ants[u.ant];
        if (!a.hom2 || m >= a.n) continue;
        const DevSeg *sg = segs + a.seg_off;
        const double *s_mid = dtab + a.arc_off, *sgn = s_mid + a.n;
        const int32_t col = ibuf[a.rowwire_off + m];  // the wire's cos column
        const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
        const cx *e = xbuf + u.x_off;
        const double *kt = cos_buf + u.cos_off + 2 * (int64_t)a.n + ibuf[a.koff_off + m];
        cx acc = cx_make(0.0, 0.0);
        for (int q = wptr[col]; q < wptr[col + 1]; ++q) {
            const int p = wrow[q];
            const double ks = kt[q - wptr[col]];
            const cx ep = e[p];
            const double len = sg[p].len;
            acc = cx_add(acc, cx_make(D_MUL(D_MUL(ep.re, ks), len), D_MUL(D_MUL(ep.im, ks), len)));
        }
        const cx r = cx_mul(cx_make(0.0, -scale), acc);
        rhs_buf[u.rhs_off + m] = cx_make(D_MUL(r.re, sgn[m]), D_MUL(r.im, sgn[m]));
    }
}

// Peak |I| of each plane-wave solve (solve_session.rs:354): the largest
// hypot over the segment currents, NaN when the solve failed.
__global__ void k_receive_peaks(const UnitDesc *__restrict__ solves, const AntDesc *__restrict__ ants,
                                const cx *__restrict__ xbuf, const int32_t *__restrict__ status, double *peak) {
    UnitDesc u = solves[blockIdx.x];
    if (!ants[u.ant].hom2) return;
    double v = 0.0;
    for (int m = threadIdx.x; m < u.n; m += 32) v = fmax(v, cx_norm(xbuf[u.x_off + m]));
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) peak[blockIdx.x] = status[u.sys] != 0 ? __longlong_as_double(0x7ff8000000000000ll) : v;
}

// ---------------------------------------------------------------------------
// Z fill
// ---------------------------------------------------------------------------
// G(R) = exp(-jkR)/R with exp(0 + jt) = (cos t, sin t) (num-complex exp)
__device__ __forceinline__ cx green_k_exact(double r, double k) {
    double sn, cs;
    fnec_libm::libm_sincos(D_MUL(-k, r), &sn, &cs);
    return cx_make(D_DIV(cs, r), D_DIV(sn, r));
}

// matrix.rs:297-331 elem(obs, src, k, is_self); self_log is the source
// segment's 2 ln((h + sqrt(h^2 + a^2)) / a), evaluated on the host
__device__ __forceinline__ cx elem_exact(const double *om, const double *od, const double *sm,
                                         const double *sd, double slen, double srad, double self_log, double k,
                                         bool is_self) {
    double cos_alpha = D_ADD(D_ADD(D_MUL(od[0], sd[0]), D_MUL(od[1], sd[1])), D_MUL(od[2], sd[2]));
    double half = D_MUL(slen, 0.5);
    double a = srad;
    double ire, iim;
    if (is_self) {
        double sre = 0.0, sim = 0.0;
#pragma unroll 1
        for (int m = 0; m < 4; ++m) {
            double l = D_MUL(c_gl_n4[m], half);
            double r_eff = D_SQRT(D_ADD(D_MUL(l, l), D_MUL(a, a)));
            cx g = green_k_exact(r_eff, k);
            double dre = D_SUB(g.re, D_DIV(1.0, r_eff));
            sre = D_ADD(sre, D_MUL(c_gl_w4[m], dre));
            sim = D_ADD(sim, D_MUL(c_gl_w4[m], g.im));
        }
        sre = D_MUL(sre, half);
        sim = D_MUL(sim, half);
        ire = D_ADD(sre, self_log);
        iim = sim;
    } else {
        double sre = 0.0, sim = 0.0;
#pragma unroll 1
        for (int m = 0; m < 8; ++m) {
            double sc = D_MUL(c_gl_n8[m], half);
            double rs0 = D_ADD(sm[0], D_MUL(sc, sd[0]));
            double rs1 = D_ADD(sm[1], D_MUL(sc, sd[1]));
            double rs2 = D_ADD(sm[2], D_MUL(sc, sd[2]));
            double r0 = D_SUB(om[0], rs0), r1 = D_SUB(om[1], rs1), r2 = D_SUB(om[2], rs2);
            double r_sq = D_ADD(D_ADD(D_MUL(r0, r0), D_MUL(r1, r1)), D_MUL(r2, r2));
            double r_eff = D_SQRT(D_ADD(r_sq, D_MUL(a, a)));
            cx g = green_k_exact(r_eff, k);
            sre = D_ADD(sre, D_MUL(c_gl_w8[m], g.re));
            sim = D_ADD(sim, D_MUL(c_gl_w8[m], g.im));
        }
        ire = D_MUL(sre, half);
        iim = D_MUL(sim, half);
    }
    return cx_make(D_MUL(ire, cos_alpha), D_MUL(iim, cos_alpha));
}

__device__ __forceinline__ cx z_entry_exact(const DevSeg &o, const DevSeg &s, double k, int ground,
                                            bool is_self) {
    cx direct = elem_exact(o.mid, o.dir, s.mid, s.dir, s.len, s.rad, s.self_log, k, is_self);
    cx img = cx_make(0.0, 0.0);
    if (ground == 1) {
        // matrix.rs:265-279 image: position (x, y, -z), current (-Jx, -Jy, +Jz)
        double im_mid[3] = {s.mid[0], s.mid[1], -s.mid[2]};
        double im_dir[3] = {-s.dir[0], -s.dir[1], s.dir[2]};
        img = elem_exact(o.mid, o.dir, im_mid, im_dir, s.len, s.rad, 0.0, k, false);
    }
    return cx_add(direct, img);
}

// One CTA of 256 threads fills a 16x16 tile of one unit's Z.
__global__ void __launch_bounds__(256) k_fill_exact(const UnitDesc *__restrict__ units,
                                                    const AntDesc *__restrict__ ants,
                                                    const DevSeg *__restrict__ segs,
                                                    const int4 *__restrict__ tiles, cx *zbuf) {
    __shared__ DevSeg s_obs[16];
    __shared__ DevSeg s_src[16];
    int4 t = tiles[blockIdx.x];  // (unit, row0, col0, -)
    UnitDesc u = units[t.x];
    AntDesc a = ants[u.ant];
    int n = a.n;
    const DevSeg *sg = segs + a.seg_off;
    int tid = threadIdx.x;
    if (tid < 16 && t.y + tid < n) s_obs[tid] = sg[t.y + tid];
    if (tid >= 32 && tid < 48 && t.z + tid - 32 < n) s_src[tid - 32] = sg[t.z + tid - 32];
    __syncthreads();
    int ii = tid / 16, jj = tid % 16;
    int i = t.y + ii, j = t.z + jj;
    if (i >= n || j >= n) return;
    cx z = z_entry_exact(s_obs[ii], s_src[jj], u.k_fill, a.ground, i == j);
    zbuf[u.z_off + (int64_t)i * n + j] = z;
}

// Fill for caller-provided segments (ZSegmentInput): same arithmetic.
__global__ void __launch_bounds__(256) k_fill_exact_flat(const DevSeg *__restrict__ sg, int n,
                                                         double k, int ground, cx *z) {
    int i = blockIdx.y * 16 + threadIdx.x / 16;
    int j = blockIdx.x * 16 + threadIdx.x % 16;
    if (i >= n || j >= n) return;
    z[(int64_t)i * n + j] = z_entry_exact(sg[i], sg[j], k, ground, i == j);
}

// ---------------------------------------------------------------------------
// Gram:  A[i][j] = sum_r conj(M[r][i]) M[r][j]  (r ascending, no FMA)
// ---------------------------------------------------------------------------
// Part 1: i < N, j <= N over the Z rows r < N, where column j == N is the
// RHS y (aty).  64x64 output tile per CTA, 4x4 per thread, k-chunks of 16.
__global__ void __launch_bounds__(256) k_gram_zz(const UnitDesc *__restrict__ units,
                                                 const int4 *__restrict__ tiles,
                                                 const cx *__restrict__ zbuf,
                                                 const cx *__restrict__ rhs_buf, cx *abuf) {
    __shared__ cx s_l[16][64];  // conj side: Z[r][i0 + ii]
    __shared__ cx s_r[16][65];  // right side: B[r][j0 + jj], B = [Z | y]
    int4 t = tiles[blockIdx.x];
    UnitDesc u = units[t.x];
    int n = u.n;
    int i0 = t.y, j0 = t.z;
    const cx *z = zbuf + u.z_off;
    const cx *y = rhs_buf + u.rhs_off;
    int tid = threadIdx.x;
    int ty = tid / 16, tx = tid % 16;
    cx acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = cx_make(0.0, 0.0);
    for (int r0 = 0; r0 < n; r0 += 16) {
        // load 16 x 64 of each side (4 elements per thread per side)
        for (int e = tid; e < 16 * 64; e += 256) {
            int rr = e / 64, cc = e % 64;
            int r = r0 + rr;
            int ci = i0 + cc, cj = j0 + cc;
            cx lv = cx_make(0.0, 0.0), rv = cx_make(0.0, 0.0);
            if (r < n) {
                if (ci < n) lv = z[(int64_t)r * n + ci];
                if (cj < n) rv = z[(int64_t)r * n + cj];
                else if (cj == n) rv = y[r];
            }
            s_l[rr][cc] = lv;
            s_r[rr][cc] = rv;
        }
        __syncthreads();
        int kmax = min(16, n - r0);
        for (int kk = 0; kk < kmax; ++kk) {
            cx lv[4], rv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) lv[a] = s_l[kk][ty + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) rv[b] = s_r[kk][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = cx_add(acc[a][b], cx_conj_mul(lv[a], rv[b]));
        }
        __syncthreads();
    }
    int w1 = u.s + 1;
    cx *A = abuf + u.a_off;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int i = i0 + ty + 16 * a;
        if (i >= n) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int j = j0 + tx + 16 * b;
            if (j < n) A[(int64_t)i * w1 + j] = acc[a][b];
            else if (j == n) A[(int64_t)i * w1 + u.s] = acc[a][b];
        }
    }
}

// Part 2: the homogeneous columns N+w (M[r][N+w] = -cos_r for rows of wire
// w, zero elsewhere; zero products change neither value nor sign of a sum
// that starts at +0, so only the wire's rows are visited, in ascending r).
// grid.x = wire column w, grid.y = unit; threads stride over i in [0, N]
// (i == N is the y column).
__global__ void k_gram_ccols(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                             const int32_t *__restrict__ ibuf, const cx *__restrict__ zbuf,
                             const cx *__restrict__ rhs_buf, const double *__restrict__ cos_buf,
                             cx *abuf) {
    UnitDesc u = units[blockIdx.y];
    AntDesc a = ants[u.ant];
    int w = blockIdx.x;
    if (w >= a.w) return;
    int n = u.n, s = u.s, w1 = s + 1;
    const cx *z = zbuf + u.z_off;
    const cx *y = rhs_buf + u.rhs_off;
    // the plane-wave form's odd columns hold -sin(k s): the second half
    const double *cv = cos_buf + u.cos_off + ((a.hom2 && (w & 1)) ? n : 0);
    const int32_t *wptr = ibuf + a.wptr_off;
    const int32_t *wrow = ibuf + a.wrow_off;
    cx *A = abuf + u.a_off;
    int b = wptr[w], e = wptr[w + 1];
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        cx col = cx_make(0.0, 0.0);  // A[i][N+w]  (i < N)
        cx row = cx_make(0.0, 0.0);  // A[N+w][i]  (i < N), or A[N+w][S] for i == N
        for (int q = b; q < e; ++q) {
            int r = wrow[q];
            cx c = cx_make(-cv[r], 0.0);
            cx zi = (i < n) ? z[(int64_t)r * n + i] : y[r];
            if (i < n) col = cx_add(col, cx_conj_mul(zi, c));
            row = cx_add(row, cx_conj_mul(c, zi));
        }
        if (i < n) {
            A[(int64_t)i * w1 + n + w] = col;
            A[(int64_t)(n + w) * w1 + i] = row;
        } else {
            A[(int64_t)(n + w) * w1 + s] = row;
        }
    }
    // the W x W block row of this column: the sum of squares on the
    // diagonal, and in the plane-wave form the cos-sin cross sum of the same
    // wire (its rows ascending, as the reference's sum over all rows); exact
    // zeros elsewhere
    for (int v = threadIdx.x; v < a.w; v += blockDim.x) {
        cx d = cx_make(0.0, 0.0);
        if (v == w || (a.hom2 && v == (w ^ 1))) {
            const double *cw = cos_buf + u.cos_off + ((a.hom2 && (v & 1)) ? n : 0);
            for (int q = b; q < e; ++q) {
                const int r = wrow[q];
                d = cx_add(d, cx_conj_mul(cx_make(-cv[r], 0.0), cx_make(-cw[r], 0.0)));
            }
        }
        A[(int64_t)(n + w) * w1 + n + v] = d;
    }
}

// Part 3: constraint rows (free-end I = 0 rows, then junction rows, in
// row order), then the Tikhonov term +1e-8 on the diagonal.
__global__ void k_gram_finish(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                              const DevConstraint *__restrict__ cons,
                              const int32_t *__restrict__ codes, cx *abuf) {
    UnitDesc u = units[blockIdx.x];
    AntDesc a = ants[u.ant];
    int w1 = u.s + 1;
    cx *A = abuf + u.a_off;
    const DevConstraint *cg = cons + a.con_off;
    const int32_t *cc = codes + a.conv_off;
    for (int g = threadIdx.x; g < a.n_con; g += blockDim.x) {
        DevConstraint c = cg[g];
        cx e = A[(int64_t)c.i * w1 + c.j];
        for (int t = 0; t < c.count; ++t) {
            int code = cc[c.begin + t];
            cx uv = cx_make((code & 2) ? -1.0 : 1.0, 0.0);
            cx vv = cx_make((code & 1) ? -1.0 : 1.0, 0.0);
            e = cx_add(e, cx_conj_mul(uv, vv));
        }
        A[(int64_t)c.i * w1 + c.j] = e;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < u.s; i += blockDim.x) {
        cx d = A[(int64_t)i * w1 + i];
        A[(int64_t)i * w1 + i] = cx_add(d, cx_make(1e-8, 0.0));
    }
}

// ---------------------------------------------------------------------------
// Blocked GEPP with the reference's per-element operation order.
// Panel columns c0 .. c0+NB-1 are factored right-looking inside the panel;
// the row swaps are applied to the trailing columns afterwards, and every
// trailing element then receives its updates in the same column order as
// the unblocked loop, so the result is identical to linear.rs:1343-1370.
// The multipliers f = a[r][c] / a[c][c] are stored in place of a[r][c]
// (the reference leaves a[r][c] - f*a[c][c] there, which it never reads).
// ---------------------------------------------------------------------------
constexpr int NB = 32;

// Pivot reduction: largest hypot, ties resolved to the larger row index
// (Iterator::max_by keeps the last maximum).
__device__ __forceinline__ void piv_better(double &bv, int &bi, double v, int i) {
    if (v > bv || (v == bv && i > bi)) {
        bv = v;
        bi = i;
    }
}

__global__ void __launch_bounds__(256) k_panel(const UnitDesc *__restrict__ units, int c0,
                                               cx *abuf, int32_t *piv_buf, int32_t *status, int skip_m, const int32_t *__restrict__ order, int base) {
    __shared__ double s_v[8];
    __shared__ int s_i[8];
    __shared__ int s_p;
    __shared__ cx s_prow[NB];
    int ui = order[base + blockIdx.x];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || s - c0 > skip_m || status[ui] != 0) return;  // skip_m: taller panels go grid-wide
    int w1 = s + 1;
    cx *A = abuf + u.a_off;
    int32_t *piv = piv_buf + u.piv_off;
    int nb = min(NB, s - c0);
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int c = c0; c < c0 + nb; ++c) {
        // --- pivot search over rows c..s-1 of column c
        double bv = -1.0;
        int bi = -1;
        for (int r = c + tid; r < s; r += blockDim.x) piv_better(bv, bi, cx_norm(A[(int64_t)r * w1 + c]), r);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            piv_better(bv, bi, ov, oi);
        }
        if (lane == 0) {
            s_v[wid] = bv;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double v = s_v[0];
            int p = s_i[0];
            for (int q = 1; q < (int)(blockDim.x >> 5); ++q) piv_better(v, p, s_v[q], s_i[q]);
            // linear.rs:1354 singular test on the chosen pivot (NaN never passes <)
            if (p < 0 || v < 1e-30) {
                status[ui] = -(c + 1);
                p = -1;
            }
            s_p = p;
            piv[c] = p;
        }
        __syncthreads();
        int p = s_p;
        if (p < 0) return;
        // --- swap rows c and p inside the panel columns
        if (p != c && tid < nb) {
            int k = c0 + tid;
            cx t0 = A[(int64_t)c * w1 + k];
            A[(int64_t)c * w1 + k] = A[(int64_t)p * w1 + k];
            A[(int64_t)p * w1 + k] = t0;
        }
        __syncthreads();
        if (tid < nb) s_prow[tid] = A[(int64_t)c * w1 + c0 + tid];
        __syncthreads();
        cx diag = s_prow[c - c0];
        // --- eliminate below the pivot inside the panel
        for (int r = c + 1 + tid; r < s; r += blockDim.x) {
            cx *row = A + (int64_t)r * w1;
            cx f = cx_div(row[c], diag);
            row[c] = f;
            for (int k = c + 1; k < c0 + nb; ++k) row[k] = cx_sub(row[k], cx_mul(f, s_prow[k - c0]));
        }
        __syncthreads();
    }
}

// The same panel factorisation with the panel (rows c0..s-1, NB columns)
// held in shared memory for the whole kernel: identical operations on
// identical values, without an L2 round trip in the sequential column loop.
// Used when (s - c0) * NB * 16 bytes fits in PANEL_SMEM_MAX.
constexpr int PANEL_SMEM_MAX = 200 * 1024;

__global__ void __launch_bounds__(256) k_panel_smem(const UnitDesc *__restrict__ units, int c0, cx *abuf,
                                                    int32_t *piv_buf, int32_t *status, int skip_m, const int32_t *__restrict__ order, int base) {
    // rows padded to PS = NB + 1 entries (distinct banks down a column); the
    // elimination runs a warp per row and a lane per panel column.  Each
    // element still receives f = a_rc / a_cc and a_rk -= f a_ck in column
    // order, as in k_panel.
    constexpr int PS = NB + 1;
    extern __shared__ cx s_pan[];  // [m][PS], m = s - c0
    __shared__ double s_v[8];
    __shared__ int s_i[8];
    __shared__ int s_p;
    int ui = order[base + blockIdx.x];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || s - c0 > skip_m || status[ui] != 0) return;  // skip_m: taller panels go grid-wide
    int w1 = s + 1;
    cx *A = abuf + u.a_off;
    int32_t *piv = piv_buf + u.piv_off;
    int nb = min(NB, s - c0);
    int m = s - c0;
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nw = blockDim.x >> 5;
    for (int e = tid; e < m * nb; e += blockDim.x) {
        int rr = e / nb, q = e % nb;
        s_pan[rr * PS + q] = A[(int64_t)(c0 + rr) * w1 + c0 + q];
    }
    __syncthreads();
    for (int c = c0; c < c0 + nb; ++c) {
        int lc = c - c0;
        double bv = -1.0;
        int bi = -1;
        for (int r = c + tid; r < s; r += blockDim.x) piv_better(bv, bi, cx_norm(s_pan[(r - c0) * PS + lc]), r);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            piv_better(bv, bi, ov, oi);
        }
        if (lane == 0) {
            s_v[wid] = bv;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double v = s_v[0];
            int p = s_i[0];
            for (int q = 1; q < nw; ++q) piv_better(v, p, s_v[q], s_i[q]);
            if (p < 0 || v < 1e-30) {
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
            cx t0 = s_pan[lc * PS + tid];
            s_pan[lc * PS + tid] = s_pan[(p - c0) * PS + tid];
            s_pan[(p - c0) * PS + tid] = t0;
        }
        __syncthreads();
        const cx pj = lane < nb ? s_pan[lc * PS + lane] : cx_make(0.0, 0.0);
        const cx diag = s_pan[lc * PS + lc];
#pragma unroll 2
        for (int r = c + 1 + wid; r < s; r += nw) {
            cx *row = s_pan + (r - c0) * PS;
            cx x = lane < nb ? row[lane] : cx_make(0.0, 0.0);
            cx f = lane == lc ? cx_div(x, diag) : x;  // one division, then broadcast
            f = cx_make(__shfl_sync(0xffffffffu, f.re, lc), __shfl_sync(0xffffffffu, f.im, lc));
            if (lane == lc) row[lc] = f;
            else if (lane > lc && lane < nb) row[lane] = cx_sub(x, cx_mul(f, pj));
        }
        __syncthreads();
    }
    for (int e = tid; e < m * nb; e += blockDim.x) {
        int rr = e / nb, q = e % nb;
        A[(int64_t)(c0 + rr) * w1 + c0 + q] = s_pan[rr * PS + q];
    }
}

// Panels taller than one CTA's shared memory: the grid-wide panel of
// fnec_grid.cuh over gridDim.x CTAs per unit (gridDim.y units, the tallest
// first), launched cooperatively.  Bit-identical to k_panel.
struct ExactPanelOps {
    using E = cx;
    using V = double;
    static constexpr double V_NONE = -1.0;
    __device__ static double key(cx a) { return cx_norm(a); }
    __device__ static void better(double &bv, int &bi, double v, int i) { piv_better(bv, bi, v, i); }
    __device__ static cx div(cx a, cx b) { return cx_div(a, b); }
    __device__ static cx sub_mul(cx acc, cx f, cx p) { return cx_sub(acc, cx_mul(f, p)); }
    __device__ static bool singular(double v) { return v < 1e-30; }  // linear.rs:1354
    __device__ static cx load_cg(const cx *p) {
        double2 d = __ldcg(reinterpret_cast<const double2 *>(p));
        return cx_make(d.x, d.y);
    }
};

__global__ void __launch_bounds__(256) k_panel_grid(const UnitDesc *__restrict__ units,
                                                    const int32_t *__restrict__ order, int c0, cx *abuf,
                                                    int32_t *piv_buf, int32_t *status, PanelXchg<cx> *xg,
                                                    GridSync *gs) {
    extern __shared__ cx s_gpan[];
    int ui = order[blockIdx.y];
    UnitDesc u = units[ui];
    if (status[ui] != 0) return;
    panel_grid_body<ExactPanelOps, NB, 256>(abuf + u.a_off, (int64_t)u.s + 1, u.s, c0, piv_buf + u.piv_off,
                                            &status[ui], xg + blockIdx.y, gs + blockIdx.y, (int)gridDim.x,
                                            (int)blockIdx.x, s_gpan);
}

// Deferred swaps and the U12 block row.  A CTA of 64 threads owns 64
// trailing columns; their NB panel rows and the panel's L block are staged
// in shared memory, the swaps are applied in pivot order (rows inside the
// panel swap in shared memory, rows below it swap with global memory), and
// row c0+q then receives the updates of panel columns c0..c0+q-1 in order.
__global__ void __launch_bounds__(64) k_swap_u12(const UnitDesc *__restrict__ units, int c0, cx *abuf,
                                                 const int32_t *__restrict__ piv_buf,
                                                 const int32_t *__restrict__ status, const int32_t *__restrict__ order, int base) {
    __shared__ cx s_c[NB][64];
    __shared__ cx s_L[NB][NB];  // read as broadcasts: no padding needed
    int ui = order[base + blockIdx.y];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 >= s || status[ui] != 0) return;
    int nb = min(NB, s - c0);
    int w1 = s + 1;
    cx *A = abuf + u.a_off;
    const int32_t *piv = piv_buf + u.piv_off;
    int t = threadIdx.x;
    if (blockIdx.x >= gridDim.x - (c0 + 63) / 64) {
        // columns left of the panel (earlier panels' multipliers): swaps
        // only, so that every row of L ends up with the row it belongs to
        int K = (blockIdx.x - (gridDim.x - (c0 + 63) / 64)) * 64 + t;
        if (K >= c0) return;
        for (int q = 0; q < nb; ++q) {
            int p = piv[c0 + q];
            if (p == c0 + q) continue;
            cx t0 = A[(int64_t)(c0 + q) * w1 + K];
            A[(int64_t)(c0 + q) * w1 + K] = A[(int64_t)p * w1 + K];
            A[(int64_t)p * w1 + K] = t0;
        }
        return;
    }
    int K = c0 + nb + blockIdx.x * 64 + t;  // column s is the right-hand side
    if (c0 + nb + blockIdx.x * 64 > s) return;
    bool live = K <= s;
    for (int e = t; e < nb * nb; e += 64) s_L[e / nb][e % nb] = A[(int64_t)(c0 + e / nb) * w1 + c0 + e % nb];
    for (int q = 0; q < nb; ++q) s_c[q][t] = live ? A[(int64_t)(c0 + q) * w1 + K] : cx_make(0.0, 0.0);
    __syncthreads();
    if (live) {
        for (int q = 0; q < nb; ++q) {
            int p = piv[c0 + q];
            if (p == c0 + q) continue;
            if (p < c0 + nb) {
                cx t0 = s_c[q][t];
                s_c[q][t] = s_c[p - c0][t];
                s_c[p - c0][t] = t0;
            } else {
                cx t0 = s_c[q][t];
                s_c[q][t] = A[(int64_t)p * w1 + K];
                A[(int64_t)p * w1 + K] = t0;
            }
        }
        for (int q = 1; q < nb; ++q) {
            cx v = s_c[q][t];
            for (int c = 0; c < q; ++c) v = cx_sub(v, cx_mul(s_L[q][c], s_c[c][t]));
            s_c[q][t] = v;
        }
        for (int q = 0; q < nb; ++q) A[(int64_t)(c0 + q) * w1 + K] = s_c[q][t];
    }
}

// A22 -= L21 * U12 with per-element in-order accumulation over the panel.
// grid.x = tiles of 64x64 over the trailing block, grid.y = unit.
__global__ void __launch_bounds__(256) k_trailing(const UnitDesc *__restrict__ units, int c0,
                                                  cx *abuf, const int32_t *__restrict__ status, const int32_t *__restrict__ order, int base) {
    extern __shared__ cx s_dyn[];
    cx(*s_l)[NB + 1] = reinterpret_cast<cx(*)[NB + 1]>(s_dyn);
    cx(*s_u)[64] = reinterpret_cast<cx(*)[64]>(s_dyn + 64 * (NB + 1));
    int ui = order[base + blockIdx.y];
    UnitDesc u = units[ui];
    int s = u.s;
    if (c0 + NB >= s || status[ui] != 0) return;  // no trailing block (or a failed unit)
    int r0 = c0 + NB;  // first trailing row/column
    int rows = s - r0, cols = s + 1 - r0;
    int tiles_c = (cols + 63) / 64;
    int tiles_r = (rows + 63) / 64;
    int tile = blockIdx.x;
    if (tile >= tiles_r * tiles_c) return;
    int R0 = r0 + (tile / tiles_c) * 64;
    int K0 = r0 + (tile % tiles_c) * 64;
    int w1 = s + 1;
    cx *A = abuf + u.a_off;
    int tid = threadIdx.x;
    for (int e = tid; e < 64 * NB; e += 256) {
        int rr = e / NB, q = e % NB;
        int R = R0 + rr;
        s_l[rr][q] = (R < s) ? A[(int64_t)R * w1 + c0 + q] : cx_make(0.0, 0.0);
    }
    for (int e = tid; e < NB * 64; e += 256) {
        int q = e / 64, cc = e % 64;
        int K = K0 + cc;
        s_u[q][cc] = (K <= s) ? A[(int64_t)(c0 + q) * w1 + K] : cx_make(0.0, 0.0);
    }
    __syncthreads();
    int ty = tid / 16, tx = tid % 16;
    cx acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
            acc[a][b] = (R < s && K <= s) ? A[(int64_t)R * w1 + K] : cx_make(0.0, 0.0);
        }
    for (int q = 0; q < NB; ++q) {
        cx lv[4], uv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) lv[a] = s_l[ty + 16 * a][q];
#pragma unroll
        for (int b = 0; b < 4; ++b) uv[b] = s_u[q][tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = cx_sub(acc[a][b], cx_mul(lv[a], uv[b]));
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int R = R0 + ty + 16 * a, K = K0 + tx + 16 * b;
            if (R < s && K <= s) A[(int64_t)R * w1 + K] = acc[a][b];
        }
}

// Back substitution x_i = (b_i - sum_{j>i} a_ij x_j) / a_ii, j ascending.
// One warp per unit.  The subtraction chain is sequential in the reference
// and stays sequential here; what is parallel is the memory stream.  The
// products a_ij x_j of a 32-wide chunk are formed one per lane, every lane
// runs the same in-order chain over the chunk through shuffles, and the U
// entries of the next BS_DEPTH chunks (in exactly the order the chain will
// consume them, across row boundaries) are already in flight while a chunk
// is consumed.  b_i and a_ii are fetched one row ahead.  x lives in shared
// memory and may alias b: b_i is read before x_i is written, and only
// x_j, j > i, is read after.
constexpr int BS_DEPTH = 8;
constexpr size_t BS_SMEM_MAX = 220 * 1024;  // x staged in shared memory up to S = 14080

struct ChunkCursor {  // (row i, first column j0) of the next 32-wide chunk
    int i, j0;
    __device__ void next(int s) {
        j0 += 32;
        while (i >= 0 && j0 >= s) {
            --i;
            j0 = i + 1;
        }
    }
};

__device__ __forceinline__ cx ld_cx(const cx *p) { return *p; }

__device__ __forceinline__ void backsub_rows(const cx *A, int s, int w1, const cx *bv, int64_t b_stride,
                                             cx *s_x) {
    int lane = threadIdx.x & 31;
    ChunkCursor pf{s - 1, s - 32};  // positioned before the first chunk
    pf.next(s);
    cx u[BS_DEPTH];
#pragma unroll
    for (int q = 0; q < BS_DEPTH; ++q) {
        int j = pf.j0 + lane;
        u[q] = (pf.i >= 0 && j < s) ? A[(int64_t)pf.i * w1 + j] : cx_make(0.0, 0.0);
        if (pf.i >= 0) pf.next(s);
    }
    cx b_next = ld_cx(bv + (int64_t)(s - 1) * b_stride);
    cx d_next = A[(int64_t)(s - 1) * w1 + (s - 1)];
    for (int i = s - 1; i >= 0; --i) {
        cx sum = b_next, di = d_next;
        if (i > 0) {
            b_next = ld_cx(bv + (int64_t)(i - 1) * b_stride);
            d_next = A[(int64_t)(i - 1) * w1 + (i - 1)];
        }
        for (int j0 = i + 1; j0 < s; j0 += 32) {
            cx uv = u[0];
#pragma unroll
            for (int q = 0; q < BS_DEPTH - 1; ++q) u[q] = u[q + 1];
            {
                int j = pf.j0 + lane;
                u[BS_DEPTH - 1] = (pf.i >= 0 && j < s) ? A[(int64_t)pf.i * w1 + j] : cx_make(0.0, 0.0);
                if (pf.i >= 0) pf.next(s);
            }
            // Lanes past the row end contribute +0: sum - (+0) == sum
            // exactly for every sum (-0, infinities and NaN included), so
            // the chain needs no predicate.
            int j = j0 + lane;
            cx p = (j < s) ? cx_mul(uv, s_x[j]) : cx_make(0.0, 0.0);
            double pr[32], pim[32];
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                pr[q] = __shfl_sync(0xffffffffu, p.re, q);
                pim[q] = __shfl_sync(0xffffffffu, p.im, q);
            }
#pragma unroll
            for (int q = 0; q < 32; ++q) sum = cx_sub(sum, cx_make(pr[q], pim[q]));
        }
        cx xi = cx_div(sum, di);
        __syncwarp();
        if (lane == 0) s_x[i] = xi;
        __syncwarp();
    }
}

// staged == 0 (systems whose x does not fit in shared memory): x is built
// in place in global memory; __syncwarp orders the warp's accesses there too.
__global__ void k_backsub(const UnitDesc *__restrict__ units, const cx *__restrict__ abuf, cx *xbuf,
                          const int32_t *__restrict__ status, int staged) {
    extern __shared__ cx s_xs[];
    int ui = blockIdx.x;
    UnitDesc u = units[ui];
    if (status[ui] != 0) return;
    int s = u.s, w1 = s + 1;
    const cx *A = abuf + u.a_off;
    cx *xs = staged ? s_xs : xbuf + u.x_off;
    backsub_rows(A, s, w1, A + s, w1, xs);
    if (staged)
        for (int i = threadIdx.x; i < s; i += 32) xbuf[u.x_off + i] = s_xs[i];
}

// Feedpoint rows: v_source = v_vec[idx] * dl, Zin = v_source / I[idx] when
// |I| > 1e-60 (solve_session.rs:911-917).  One CTA per solve; its rows are
// the feed rows of its right-hand side.
__global__ void k_feedpoints(const UnitDesc *__restrict__ solves, const AntDesc *__restrict__ ants,
                             const DevSeg *__restrict__ segs, const int32_t *__restrict__ ibuf,
                             const DevFeed *__restrict__ feeds, const cx *__restrict__ xbuf,
                             const int32_t *__restrict__ status, double *feed_out,
                             const int64_t *__restrict__ feed_row_off) {
    int si = blockIdx.x;
    UnitDesc u = solves[si];
    AntDesc a = ants[u.ant];
    const int32_t *fptr = ibuf + a.fptr_off;
    int f0 = fptr[u.rhs], nf = fptr[u.rhs + 1] - f0;
    for (int q = threadIdx.x; q < nf; q += blockDim.x) {
        DevFeed f = feeds[a.feed_off + f0 + q];
        double *o = feed_out + 7 * (feed_row_off[si] + q);
        if (status[u.sys] != 0) {
            for (int t = 0; t < 7; ++t) o[t] = 0.0;
            continue;
        }
        double dl = segs[a.seg_off + f.seg].len;
        cx vs = cx_make(D_MUL(f.vdl_re, dl), D_MUL(f.vdl_im, dl));
        cx cur = xbuf[u.x_off + f.seg];
        cx zin = cx_norm(cur) > 1e-60 ? cx_div(vs, cur) : vs;
        o[0] = (double)f.seg;
        o[1] = vs.re;
        o[2] = vs.im;
        o[3] = cur.re;
        o[4] = cur.im;
        o[5] = zin.re;
        o[6] = zin.im;
    }
}

// ---------------------------------------------------------------------------
// Further right-hand sides on the factored system (solves with rhs >= 1).
// The reference re-runs the whole elimination for another source; A does
// not depend on the source, so its operations on A repeat exactly and only
// the b column differs.  b = M^H y is formed in the Gram's order; the row
// swaps, the multipliers (stored in L with all later swaps applied, so row
// r of L is the row that ends at position r) and the back substitution then
// give b exactly the sequence of operations the reference's augmented
// column receives.
// ---------------------------------------------------------------------------
__global__ void k_extra_rhs_b(const UnitDesc *__restrict__ solves, const AntDesc *__restrict__ ants,
                              const int32_t *__restrict__ ibuf, const cx *__restrict__ zbuf,
                              const cx *__restrict__ rhs_buf, const double *__restrict__ cos_buf, cx *xbuf,
                              int first_rhs) {
    UnitDesc u = solves[blockIdx.y];
    if (u.rhs < first_rhs) return;
    AntDesc a = ants[u.ant];
    int n = u.n;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const cx *z = zbuf + u.z_off;
    const cx *y = rhs_buf + u.rhs_off;
    cx *b = xbuf + u.x_off;
    if (i < n) {
        cx acc = cx_make(0.0, 0.0);
        for (int r = 0; r < n; ++r) acc = cx_add(acc, cx_conj_mul(z[(int64_t)r * n + i], y[r]));
        b[i] = acc;
    } else if (i < n + a.w) {
        int w = i - n;
        const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
        const double *cv = cos_buf + u.cos_off + ((a.hom2 && (w & 1)) ? n : 0);
        cx acc = cx_make(0.0, 0.0);
        for (int q = wptr[w]; q < wptr[w + 1]; ++q) {
            int r = wrow[q];
            acc = cx_add(acc, cx_conj_mul(cx_make(-cv[r], 0.0), y[r]));
        }
        b[i] = acc;
    }
}

__global__ void k_extra_rhs_solve(const UnitDesc *__restrict__ solves, const cx *__restrict__ abuf,
                                  const int32_t *__restrict__ piv_buf, cx *xbuf,
                                  const int32_t *__restrict__ status, int staged, int first_rhs) {
    extern __shared__ cx s_bs[];
    UnitDesc u = solves[blockIdx.x];
    if (u.rhs < first_rhs || status[u.sys] != 0) return;
    int s = u.s, w1 = s + 1;
    const cx *A = abuf + u.a_off;
    const int32_t *piv = piv_buf + u.piv_off;
    cx *x = xbuf + u.x_off;
    cx *s_b = staged ? s_bs : x;  // unstaged: work in place in global memory
    int lane = threadIdx.x;
    if (staged)
        for (int i = lane; i < s; i += 32) s_b[i] = x[i];
    __syncwarp();
    if (lane == 0)
        for (int c = 0; c < s; ++c) {
            int p = piv[c];
            if (p != c) {
                cx t0 = s_b[c];
                s_b[c] = s_b[p];
                s_b[p] = t0;
            }
        }
    __syncwarp();
    // forward: row r receives b[r] -= f[r][c] * b[c] for c = 0..r-1 in order
    for (int c = 0; c < s; ++c) {
        cx bc = s_b[c];
        for (int r = c + 1 + lane; r < s; r += 32) s_b[r] = cx_sub(s_b[r], cx_mul(A[(int64_t)r * w1 + c], bc));
        __syncwarp();
    }
    // back substitution, j ascending, as k_backsub (x overwrites b in place)
    backsub_rows(A, s, w1, s_b, 1, s_b);
    if (staged)
        for (int i = lane; i < s; i += 32) x[i] = s_b[i];
}

// ---------------------------------------------------------------------------
// Many right-hand sides on one factorisation (a receive sweep's incidence
// directions), in groups of up to 32 solves of one system: group g =
// (system, first solve, count).  k_extra_rhs_b_group forms M^H y of every
// solve of the group with Z read once per group: thread i keeps the 32
// accumulators of row i, each summed over r ascending exactly as
// k_extra_rhs_b sums it.  k_extra_rhs_solve_group gives each solve one lane
// (16 per block): its right-hand side lives in a shared [s][16] tile, the row swaps, the
// forward elimination (b[r] -= f[r][c] b[c], c ascending) and the back
// substitution (j ascending, then the division) are k_extra_rhs_solve's
// operations in its order, with the factor read warp-uniformly.
// ---------------------------------------------------------------------------
constexpr int RG = 32;  // solves per group
constexpr int SG = 16;  // solves per substitution block: a [s][16] tile, several blocks per SM

__global__ void __launch_bounds__(64) k_extra_rhs_b_group(const UnitDesc *__restrict__ solves,
                                                          const int4 *__restrict__ groups,
                                                          const AntDesc *__restrict__ ants,
                                                          const int32_t *__restrict__ ibuf,
                                                          const cx *__restrict__ zbuf,
                                                          const cx *__restrict__ rhs_buf,
                                                          const double *__restrict__ cos_buf, cx *xbuf) {
    __shared__ cx Y[RG][RG];  // [row in chunk][solve]
    const int4 g = groups[blockIdx.y];
    const UnitDesc u0 = solves[g.y];
    const int n = u0.n, s = u0.s;
    if ((int)(blockIdx.x * blockDim.x) >= s) return;  // the whole block: no barrier is skipped
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const cx *z = zbuf + u0.z_off;
    cx acc[RG];
#pragma unroll
    for (int d = 0; d < RG; ++d) acc[d] = cx_make(0.0, 0.0);
    for (int r0 = 0; r0 < n; r0 += RG) {
        __syncthreads();
        for (int t = threadIdx.x; t < RG * RG; t += blockDim.x) {
            const int d = t / RG, rr = t % RG;
            Y[rr][d] = (d < g.z && r0 + rr < n) ? rhs_buf[solves[g.y + d].rhs_off + r0 + rr] : cx_make(0.0, 0.0);
        }
        __syncthreads();
        if (i < n) {
            const int rmax = min(RG, n - r0);
            for (int rr = 0; rr < rmax; ++rr) {
                const cx zz = z[(int64_t)(r0 + rr) * n + i];
#pragma unroll
                for (int d = 0; d < RG; ++d) acc[d] = cx_add(acc[d], cx_conj_mul(zz, Y[rr][d]));
            }
        }
    }
    if (i < n) {
#pragma unroll
        for (int d = 0; d < RG; ++d)  // static indices keep acc in registers
            if (d < g.z) xbuf[solves[g.y + d].x_off + i] = acc[d];
    } else if (i < s) {  // a homogeneous column: its rows' -cos (or -sin) values
        const AntDesc a = ants[u0.ant];
        const int w = i - n;
        const int32_t *wptr = ibuf + a.wptr_off, *wrow = ibuf + a.wrow_off;
        const double *cv = cos_buf + u0.cos_off + ((a.hom2 && (w & 1)) ? n : 0);
        for (int d = 0; d < g.z; ++d) {
            const cx *y = rhs_buf + solves[g.y + d].rhs_off;
            cx b = cx_make(0.0, 0.0);
            for (int q = wptr[w]; q < wptr[w + 1]; ++q) {
                const int r = wrow[q];
                b = cx_add(b, cx_conj_mul(cx_make(-cv[r], 0.0), y[r]));
            }
            xbuf[solves[g.y + d].x_off + i] = b;
        }
    }
}

// The factor streams through the lanes in 16-wide row chunks, PD chunks
// ahead of the arithmetic: lane k loads entry c0 + k of a chunk (one
// coalesced access), and the chain receives the entries in column order
// by shuffles.  Forward chunks: rows 1 .. s-1, columns 0 .. r-1; back
// chunks: rows s-1 .. 0, columns i+1 .. s-1 (rows without any skipped).
constexpr int PD = 8;
struct FwdChunks {
    int r, c0;
    __device__ void next(int s) {
        c0 += SG;
        if (c0 >= r) {
            ++r;
            c0 = 0;
        }
        (void)s;
    }
    __device__ bool valid(int s) const { return r < s; }
    __device__ int end(int s) const { return r; }
};
struct BackChunks {
    int r, c0;
    __device__ void norm(int s) {
        while (r >= 0 && c0 >= s) {
            --r;
            c0 = r + 1;
        }
    }
    __device__ void next(int s) {
        c0 += SG;
        norm(s);
    }
    __device__ bool valid(int s) const { return r >= 0; }
    __device__ int end(int s) const { return s; }
};

template <typename Cur>
__device__ __forceinline__ cx chunk_entry(const cx *A, int w1, int s, const Cur &pf, int l) {
    const int c = pf.c0 + l;
    return (pf.valid(s) && c < pf.end(s)) ? A[(int64_t)pf.r * w1 + c] : cx_make(0.0, 0.0);
}

__global__ void __launch_bounds__(SG) k_extra_rhs_solve_group(const UnitDesc *__restrict__ solves,
                                                             const int4 *__restrict__ groups,
                                                             const cx *__restrict__ abuf,
                                                             const int32_t *__restrict__ piv_buf, cx *xbuf,
                                                             const int32_t *__restrict__ status) {
    extern __shared__ cx B[];  // [s][SG], then the diagonal [s], then the pivots (int32 [s])
    const int4 g = groups[blockIdx.x];
    const UnitDesc u0 = solves[g.y];
    if (status[u0.sys] != 0 || (int)(blockIdx.y * SG) >= g.z) return;
    const int s = u0.s, w1 = s + 1, d = blockIdx.y * SG + threadIdx.x, l = threadIdx.x;
    const unsigned mask = (1u << SG) - 1u;
    cx *diag = B + (size_t)s * SG;
    int32_t *pv = reinterpret_cast<int32_t *>(diag + s);
    const cx *A = abuf + u0.a_off;
    const int32_t *piv = piv_buf + u0.piv_off;
    for (int i = l; i < s; i += SG) {
        diag[i] = A[(int64_t)i * w1 + i];
        pv[i] = piv[i];
    }
    const bool live = d < g.z;
    cx *x = xbuf + solves[g.y + (live ? d : 0)].x_off;
    for (int j = 0; j < s; ++j) B[j * SG + l] = live ? x[j] : cx_make(0.0, 0.0);
    __syncwarp(mask);
    for (int c = 0; c < s; ++c) {
        const int p = pv[c];
        if (p != c) {
            const cx t = B[c * SG + l];
            B[c * SG + l] = B[p * SG + l];
            B[p * SG + l] = t;
        }
    }
    // forward elimination row by row: row r receives b[r] -= f[r][c] b[c]
    // for c ascending -- the operations and order of the column sweep, as
    // every b[c] with c < r is final when row r starts
    {
        FwdChunks pf{1, 0};
        cx u[PD];
#pragma unroll
        for (int q = 0; q < PD; ++q) {
            u[q] = chunk_entry(A, w1, s, pf, l);
            if (pf.valid(s)) pf.next(s);
        }
        for (int r = 1; r < s; ++r) {
            cx sum = B[r * SG + l];
            for (int c0 = 0; c0 < r; c0 += SG) {
                const cx uv = u[0];
#pragma unroll
                for (int q = 0; q < PD - 1; ++q) u[q] = u[q + 1];
                u[PD - 1] = chunk_entry(A, w1, s, pf, l);
                if (pf.valid(s)) pf.next(s);
                const int cnt = min(SG, r - c0);
#pragma unroll
                for (int q = 0; q < SG; ++q) {
                    const cx a = cx_make(__shfl_sync(mask, uv.re, q, SG), __shfl_sync(mask, uv.im, q, SG));
                    if (q < cnt) sum = cx_sub(sum, cx_mul(a, B[(c0 + q) * SG + l]));
                }
            }
            B[r * SG + l] = sum;
        }
    }
    // back substitution: j ascending, then the division by the diagonal
    {
        BackChunks pf{s - 1, s};
        pf.norm(s);
        cx u[PD];
#pragma unroll
        for (int q = 0; q < PD; ++q) {
            u[q] = chunk_entry(A, w1, s, pf, l);
            if (pf.valid(s)) pf.next(s);
        }
        for (int i = s - 1; i >= 0; --i) {
            cx sum = B[i * SG + l];
            for (int j0 = i + 1; j0 < s; j0 += SG) {
                const cx uv = u[0];
#pragma unroll
                for (int q = 0; q < PD - 1; ++q) u[q] = u[q + 1];
                u[PD - 1] = chunk_entry(A, w1, s, pf, l);
                if (pf.valid(s)) pf.next(s);
                const int cnt = min(SG, s - j0);
#pragma unroll
                for (int q = 0; q < SG; ++q) {
                    const cx a = cx_make(__shfl_sync(mask, uv.re, q, SG), __shfl_sync(mask, uv.im, q, SG));
                    if (q < cnt) sum = cx_sub(sum, cx_mul(a, B[(j0 + q) * SG + l]));
                }
            }
            B[i * SG + l] = cx_div(sum, diag[i]);
        }
    }
    if (live)
        for (int j = 0; j < s; ++j) x[j] = B[j * SG + l];
}

// Four warps per group of 32 solves (lane = solve): the forward elimination
// as the column sweep (every row r > c receives b[r] -= f[r][c] b[c] at step
// c, rows spread over the warps, the factor staged PC columns at a time in
// shared memory, a barrier per column), the back substitution with each
// 32-column chunk's products formed by all warps and subtracted in ascending
// j by warp 0.  Same operations in the same order per element as
// k_extra_rhs_solve; used while [s][32] + the panel + one product chunk fit.
constexpr int PC = 8;   // factor columns per staged panel
constexpr int CH = 32;  // back-substitution product chunk
constexpr int GW4 = 4;  // warps per block
constexpr int RB = 3;   // row-buffer loads per thread: S <= 3 * 128

size_t solve_group4_smem(int s) { return sizeof(cx) * ((size_t)s * (RG + PC + 2) + (size_t)CH * RG); }

__global__ void __launch_bounds__(GW4 * 32) k_extra_rhs_solve_group4(const UnitDesc *__restrict__ solves,
                                                                    const int4 *__restrict__ groups,
                                                                    const cx *__restrict__ abuf,
                                                                    const int32_t *__restrict__ piv_buf, cx *xbuf,
                                                                    const int32_t *__restrict__ status) {
    extern __shared__ cx sm[];
    const int4 g = groups[blockIdx.x];
    const UnitDesc u0 = solves[g.y];
    if (status[u0.sys] != 0) return;  // uniform over the block
    const int s = u0.s, w1 = s + 1;
    const int d = threadIdx.x & 31, w = threadIdx.x >> 5;
    cx *B = sm;                        // [s][RG]
    cx *Ap = B + (size_t)s * RG;       // [s][PC]: rows of the staged columns
    cx *P = Ap + (size_t)s * PC;       // [CH][RG]
    const cx *A = abuf + u0.a_off;
    const int32_t *piv = piv_buf + u0.piv_off;
    const bool live = d < g.z;
    cx *x = xbuf + solves[g.y + (live ? d : 0)].x_off;
    for (int j = w; j < s; j += GW4) B[j * RG + d] = live ? x[j] : cx_make(0.0, 0.0);
    __syncthreads();
    if (w == 0)
        for (int c = 0; c < s; ++c) {
            const int p = piv[c];
            if (p != c) {
                const cx t = B[c * RG + d];
                B[c * RG + d] = B[p * RG + d];
                B[p * RG + d] = t;
            }
        }
    // forward elimination, column by column
    for (int c0 = 0; c0 < s; c0 += PC) {
        const int pc_n = min(PC, s - c0);
        __syncthreads();  // the previous panel is no longer read
        for (int t = threadIdx.x; t < (s - c0 - 1) * PC; t += blockDim.x) {
            const int r = c0 + 1 + t / PC, q = t % PC;
            if (q < pc_n) Ap[r * PC + q] = A[(int64_t)r * w1 + c0 + q];
        }
        __syncthreads();
        for (int q = 0; q < pc_n; ++q) {
            const int c = c0 + q;
            const cx bc = B[c * RG + d];
            int r = c + 1;
            r += (w - r % GW4 + GW4) % GW4;  // this warp's first row after c
            for (; r < s; r += GW4) B[r * RG + d] = cx_sub(B[r * RG + d], cx_mul(Ap[r * PC + q], bc));
            __syncthreads();
        }
    }
    // back substitution; the factor rows pass through two shared row
    // buffers, row i-1 loaded while row i is processed
    cx *Ar = P + (size_t)CH * RG;  // [2][s]
    for (int t = threadIdx.x; t < s; t += blockDim.x)
        if (t >= s - 1) Ar[t] = A[(int64_t)(s - 1) * w1 + t];
    __syncthreads();
    cx sum = cx_make(0.0, 0.0);
    int cur = 0;
    for (int i = s - 1; i >= 0; --i) {
        cx nxt[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            const int t = threadIdx.x + k * GW4 * 32;
            nxt[k] = (i > 0 && t >= i - 1 && t < s) ? A[(int64_t)(i - 1) * w1 + t] : cx_make(0.0, 0.0);
        }
        const cx *ar = Ar + (size_t)cur * s;
        if (w == 0) sum = B[i * RG + d];
        for (int j0 = i + 1; j0 < s; j0 += CH) {
            const int cnt = min(CH, s - j0);
            __syncthreads();  // P is free; x[j] for j > i is final
            for (int q = w; q < cnt; q += GW4) P[q * RG + d] = cx_mul(ar[j0 + q], B[(j0 + q) * RG + d]);
            __syncthreads();
            if (w == 0)
                for (int q = 0; q < cnt; ++q) sum = cx_sub(sum, P[q * RG + d]);
        }
        if (w == 0) B[i * RG + d] = cx_div(sum, ar[i]);
        // row i+1's buffer was last read before this row's barriers
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            const int t = threadIdx.x + k * GW4 * 32;
            if (i > 0 && t >= i - 1 && t < s) Ar[(size_t)(cur ^ 1) * s + t] = nxt[k];
        }
        cur ^= 1;
        if (i == s - 1) __syncthreads();  // row s-1 has no chunk barrier before row s-2 reads its buffer
    }
    __syncthreads();
    if (live)
        for (int j = w; j < s; j += GW4) x[j] = B[j * RG + d];
}

// ---------------------------------------------------------------------------
// launch wrappers (host)
// ---------------------------------------------------------------------------
void launch_expand_segments(const DevWire *wires, int nw, DevSeg *segs, cudaStream_t st) {
    if (nw > 0) k_expand_segments<<<nw, 64, 0, st>>>(wires, nw, segs);
}
void launch_hallen_rhs(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevSource *srcs, const double *dtab, cx *rhs, double *cosv,
                       double scale, cudaStream_t st) {
    if (ns > 0) k_hallen_rhs<<<ns, 128, 0, st>>>(solves, ants, segs, ibuf, srcs, dtab, rhs, cosv, scale);
}
void launch_planewave_rhs(const UnitDesc *solves, int ns, int max_n, const AntDesc *ants, const DevSeg *segs,
                          const int32_t *ibuf, const double *dtab, cx *x, cx *rhs, double *cosv, double scale,
                          cudaStream_t st) {
    if (ns <= 0 || max_n <= 0) return;
    dim3 g((max_n + 127) / 128, ns < 65535 ? ns : 65535);
    k_planewave_field<<<g, 128, 0, st>>>(solves, ns, ants, segs, ibuf, dtab, x, cosv);
    k_planewave_rhs<<<g, 128, 0, st>>>(solves, ns, ants, segs, ibuf, dtab, cosv, x, rhs, scale);
}
void launch_receive_peaks(const UnitDesc *solves, int ns, const AntDesc *ants, const cx *x, const int32_t *status,
                          double *peak, cudaStream_t st) {
    if (ns > 0) k_receive_peaks<<<ns, 32, 0, st>>>(solves, ants, x, status, peak);
}
void launch_fill_exact(const UnitDesc *units, const AntDesc *ants, const DevSeg *segs,
                       const int4 *tiles, int ntiles, cx *z, cudaStream_t st) {
    if (ntiles > 0) k_fill_exact<<<ntiles, 256, 0, st>>>(units, ants, segs, tiles, z);
}
void launch_fill_exact_flat(const DevSeg *segs, int n, double k, int ground, cx *z, cudaStream_t st) {
    dim3 g((n + 15) / 16, (n + 15) / 16);
    if (n > 0) k_fill_exact_flat<<<g, 256, 0, st>>>(segs, n, k, ground, z);
}
void launch_gram_exact(const UnitDesc *units, int nu, int max_w, const AntDesc *ants, const int4 *gtiles,
                       int ngtiles, const int32_t *ibuf, const DevConstraint *cons,
                       const int32_t *codes, const cx *z, const cx *rhs, const double *cosv, cx *A,
                       cudaStream_t st) {
    if (ngtiles > 0) k_gram_zz<<<ngtiles, 256, 0, st>>>(units, gtiles, z, rhs, A);
    if (nu > 0) {
        dim3 g(max_w > 0 ? max_w : 1, nu);
        k_gram_ccols<<<g, 256, 0, st>>>(units, ants, ibuf, z, rhs, cosv, A);
        k_gram_finish<<<nu, 256, 0, st>>>(units, ants, cons, codes, A);
    }
}
constexpr size_t TRAILING_SMEM = sizeof(cx) * (64 * (NB + 1) + NB * 64);

// Raises a kernel's dynamic shared-memory limit once per device: the
// attribute belongs to the kernel in the current device's context, so a
// second GPU needs its own call.  Returns the limit in effect.
int set_smem_limit_once(const void *kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1;
    }
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(dev, kernel);
    auto it = done.find(key);
    if (it != done.end()) return it->second;
    int got = -1;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) {
        got = bytes;
    } else {
        (void)cudaGetLastError();  // leave no error behind for the launch checks
        std::fprintf(stderr, "fnec: shared-memory limit %d B refused (%s); kernels fall back to global staging\n",
                     bytes, cudaGetErrorString(e));
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess) got = fa.maxDynamicSharedSizeBytes;
        else (void)cudaGetLastError();
    }
    done[key] = got;
    return got;
}

size_t grid_xchg_bytes() { return sizeof(PanelXchg<cx>) * GRID_PANEL_MAX_UNITS; }
size_t grid_sync_bytes(int steps) { return sizeof(GridSync) * GRID_PANEL_MAX_UNITS * (size_t)(steps > 0 ? steps : 1); }

// Chooses how the panel at column c0 is factored.  Units whose panel
// (s - c0 rows) exceeds one CTA's shared memory (thr_rows) go to the
// grid-wide kernel when they are few enough to be co-resident; the rest use
// the one-CTA shared-memory kernel.  Returns the number of grid units
// (0: none; -1: not possible, every unit takes the one-CTA global kernel)
// and the CTAs per grid unit and their shared memory.
int plan_grid_panel(const GridPlan &gp, int c0, int thr_rows, int pnb, size_t elem, const void *kernel,
                    int *G_out, size_t *smem_out) {
    int nl = 0;
    while (nl < (int)gp.s_desc.size() && gp.s_desc[nl] - c0 > thr_rows) ++nl;
    if (nl == 0) return 0;
    if (!gp.grid_on || nl > GRID_PANEL_MAX_UNITS || !gp.d_xchg || !gp.d_sync || gp.sms <= 0) return -1;
    const int m_max = gp.s_desc[0] - c0;
    const size_t cta_cap = 96 * 1024;  // two CTAs per SM
    const int r_cap = (int)(cta_cap / (pnb * elem));
    int G = std::max(1, gp.sms / nl);
    G = std::min(G, (m_max + 31) / 32);
    G = std::max(G, (m_max + r_cap - 1) / r_cap);
    if (G > GRID_PANEL_MAX_CTAS) return -1;
    int R = (m_max + G - 1) / G;
    size_t smem = (size_t)R * pnb * elem;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem) != cudaSuccess) return -1;
    if ((int64_t)G * nl > (int64_t)per_sm * gp.sms) return -1;
    *G_out = G;
    *smem_out = smem;
    return nl;
}

cudaError_t launch_cooperative(const void *kernel, dim3 grid, dim3 block, void **args, size_t smem,
                               cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, kernel, args);
}

void step_classes(const GridPlan &gp, int c0, int i_begin, std::vector<StepClass> &out, int i_end) {
    out.clear();
    int i = i_begin, n = i_end < 0 ? (int)gp.s_desc.size() : std::min(i_end, (int)gp.s_desc.size());
    while (i < n && gp.s_desc[i] > c0) {
        const int f = 1 << gp.class_shift;
        int m = gp.s_desc[i] - c0, hi = 64;
        while (hi < m) hi *= f;
        int lo = hi == 64 ? 0 : hi / f;  // the class holds heights (lo, hi]
        StepClass c{i, i, m};
        while (i < n && gp.s_desc[i] - c0 > lo) ++i;  // s descending: the class is a run
        c.i1 = i;
        out.push_back(c);
    }
}

uint64_t launch_factor_exact(const UnitDesc *units, int nu, int max_s, const GridPlan &gp, cx *A,
                             int32_t *piv, int32_t *status, cudaStream_t st) {
    uint64_t L = 0;
    set_smem_limit_once(k_trailing, (int)TRAILING_SMEM);  // once per device
    set_smem_limit_once(k_panel_smem, PANEL_SMEM_MAX);
    set_smem_limit_once(k_panel_grid, 96 * 1024);
    (void)nu;
    const int thr_rows = PANEL_SMEM_MAX / (int)((NB + 1) * sizeof(cx));
    const int32_t *ord = gp.d_order;
    if (gp.d_sync) cudaMemsetAsync(gp.d_sync, 0, grid_sync_bytes(gp.steps), st);
    std::vector<StepClass> cls;
    for (int c0 = 0; c0 < max_s; c0 += NB) {
        // panels: the tallest units (m > thr_rows) grid-wide or one CTA each
        // from global memory, the rest one CTA each from shared memory, in
        // size classes so that short panels do not reserve tall panels' memory
        int n_thr = 0;
        while (n_thr < (int)gp.s_desc.size() && gp.s_desc[n_thr] - c0 > thr_rows) ++n_thr;
        if (n_thr > 0) {
            int G = 0;
            size_t gsm = 0;
            bool done = false;
            if (plan_grid_panel(gp, c0, thr_rows, NB, sizeof(cx), (const void *)k_panel_grid, &G, &gsm) == n_thr) {
                PanelXchg<cx> *xg = static_cast<PanelXchg<cx> *>(gp.d_xchg);
                GridSync *gs = static_cast<GridSync *>(gp.d_sync) + (size_t)(c0 / NB) * GRID_PANEL_MAX_UNITS;
                void *args[] = {(void *)&units, (void *)&ord, (void *)&c0, (void *)&A, (void *)&piv,
                                (void *)&status, (void *)&xg, (void *)&gs};
                done = launch_cooperative((const void *)k_panel_grid, dim3(G, n_thr), dim3(256), args, gsm, st) ==
                       cudaSuccess;
                if (!done) (void)cudaGetLastError();  // not co-resident after all
            }
            if (!done) k_panel<<<n_thr, 256, 0, st>>>(units, c0, A, piv, status, INT_MAX, ord, 0);
            ++L;
        }
        step_classes(gp, c0, n_thr, cls);
        for (const StepClass &c : cls) {
            k_panel_smem<<<c.i1 - c.i0, 256, sizeof(cx) * (size_t)c.m_max * (NB + 1), st>>>(units, c0, A, piv, status,
                                                                                      INT_MAX, ord, c.i0);
            ++L;
        }
        // deferred swaps + U12, then the trailing update, by size class
        step_classes(gp, c0, 0, cls);
        for (const StepClass &c : cls) {
            int m = c.m_max;
            int rest = m + 1 - NB;  // columns right of the panel, at least the right-hand side
            if (rest < 1) rest = 1;
            dim3 g1((rest + 63) / 64 + (c0 + 63) / 64, c.i1 - c.i0);
            k_swap_u12<<<g1, 64, 0, st>>>(units, c0, A, piv, status, ord, c.i0);
            ++L;
            int rows = m - NB;
            if (rows > 0) {
                int t = ((rows + 63) / 64) * ((rest + 63) / 64);
                dim3 g2(t, c.i1 - c.i0);
                k_trailing<<<g2, 256, TRAILING_SMEM, st>>>(units, c0, A, status, ord, c.i0);
                ++L;
            }
        }
    }
    return L;
}
void launch_backsub(const UnitDesc *units, int nu, int max_s, const cx *A, cx *x,
                    const int32_t *status, cudaStream_t st) {
    size_t smem = sizeof(cx) * (size_t)max_s;
    int staged = smem <= BS_SMEM_MAX;
    if (staged && smem > 0) {  // static + dynamic above 48 KB needs the raised limit
        int lim = set_smem_limit_once(k_backsub, (int)BS_SMEM_MAX);
        if (lim < 0 || (size_t)lim < smem) staged = 0;
    }
    if (!staged) smem = 0;
    if (nu > 0) k_backsub<<<nu, 32, smem, st>>>(units, A, x, status, staged);
}
// matrix.rs:131-139 add_to_diagonal / add_to_entry: each stamp one
// separately rounded complex add, an entry's stamps in their order (the
// thread at the first stamp of each run applies the run).
__global__ void k_stamps(const DevStamp *__restrict__ stamps, int n, cx *z) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n || !stamps[q].first) return;
    const DevStamp d = stamps[q];
    cx v = z[d.index];
    for (int t = 0; t < d.count; ++t) v = cx_add(v, cx_make(stamps[q + t].re, stamps[q + t].im));
    z[d.index] = v;
}
void launch_stamps(const DevStamp *stamps, int n, cx *z, cudaStream_t st) {
    if (n > 0) k_stamps<<<(n + 255) / 256, 256, 0, st>>>(stamps, n, z);
}
void launch_feedpoints(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevFeed *feeds, const cx *x, const int32_t *status,
                       double *feed_out, const int64_t *feed_row_off, cudaStream_t st) {
    if (ns > 0)
        k_feedpoints<<<ns, 32, 0, st>>>(solves, ants, segs, ibuf, feeds, x, status, feed_out, feed_row_off);
}
void launch_extra_rhs_exact(const UnitDesc *solves, int ns, int max_s, const AntDesc *ants, const int32_t *ibuf,
                            const cx *z, const cx *rhs, const double *cosv, const cx *A, const int32_t *piv,
                            cx *x, const int32_t *status, cudaStream_t st, const int4 *groups, int n_groups,
                            int first_rhs) {
    if (ns <= 0) return;
    if (groups && n_groups > 0 && first_rhs == 1) {
        dim3 gb((max_s + 63) / 64, n_groups);
        k_extra_rhs_b_group<<<gb, 64, 0, st>>>(solves, groups, ants, ibuf, z, rhs, cosv, x);
        const size_t smem4 = solve_group4_smem(max_s);
        int lim4 = (smem4 <= BS_SMEM_MAX && max_s <= RB * GW4 * 32)
                       ? set_smem_limit_once(k_extra_rhs_solve_group4, (int)BS_SMEM_MAX)
                       : -1;
        if (lim4 >= 0 && (size_t)lim4 >= smem4) {
            k_extra_rhs_solve_group4<<<n_groups, GW4 * 32, smem4, st>>>(solves, groups, A, piv, x, status);
            return;
        }
        const size_t smem = (sizeof(cx) * (SG + 1) + sizeof(int32_t)) * (size_t)max_s;
        int lim = smem <= BS_SMEM_MAX ? set_smem_limit_once(k_extra_rhs_solve_group, (int)BS_SMEM_MAX) : -1;
        if (lim >= 0 && (size_t)lim >= smem) {
            k_extra_rhs_solve_group<<<dim3(n_groups, RG / SG), SG, smem, st>>>(solves, groups, A, piv, x, status);
            return;
        }
        // a factor too tall for the shared tile: one warp per solve on the b vectors formed above
        k_extra_rhs_solve<<<ns, 32, 0, st>>>(solves, A, piv, x, status, 0, 1);
        return;
    }
    dim3 g((max_s + 127) / 128, ns);
    k_extra_rhs_b<<<g, 128, 0, st>>>(solves, ants, ibuf, z, rhs, cosv, x, first_rhs);
    size_t smem = sizeof(cx) * (size_t)max_s;
    int staged = smem <= BS_SMEM_MAX;
    if (staged && smem > 0) {  // static + dynamic above 48 KB needs the raised limit
        int lim = set_smem_limit_once(k_extra_rhs_solve, (int)BS_SMEM_MAX);
        if (lim < 0 || (size_t)lim < smem) staged = 0;
    }
    if (!staged) smem = 0;
    k_extra_rhs_solve<<<ns, 32, smem, st>>>(solves, A, piv, x, status, staged, first_rhs);
}

}  // namespace fnec

// ---------------------------------------------------------------------------
// Self-test of the bounded grid barrier's timeout path
// (fnec_selftest_wait_timeout): every CTA but `absent` takes the barrier;
// the absent CTA returns without arriving, so the others' waits run out
// after wait_ns and each marks the status word FNEC_UNIT_TIMEOUT.  With
// absent < 0 every CTA arrives and the status stays 0.
// ---------------------------------------------------------------------------
namespace fnec {
__global__ void k_grid_barrier_probe(GridSync *gs, int32_t *status, int absent, unsigned long long wait_ns) {
    if ((int)blockIdx.x == absent) return;
    if (!grid_barrier(gs, gridDim.x, 1, wait_ns)) {
        if (threadIdx.x == 0) atomicExch(status, FNEC_UNIT_TIMEOUT);
        return;
    }
}

int selftest_grid_timeout(int32_t device, int32_t ctas, int32_t absent, uint64_t wait_ns, int32_t *unit_status,
                          double *elapsed_ms) {
    if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    if (ctas < 2 || ctas > 148 || absent >= ctas) return FNEC_ERR_BAD_ARG;
    GridSync *gs = nullptr;
    int32_t *st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = FNEC_OK;
    do {
        if (cudaMalloc(&gs, sizeof(GridSync)) != cudaSuccess || cudaMalloc(&st, sizeof(int32_t)) != cudaSuccess) {
            rc = FNEC_ERR_OUT_OF_MEMORY;
            break;
        }
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            rc = FNEC_ERR_CUDA;
            break;
        }
        cudaMemset(gs, 0, sizeof(GridSync));
        cudaMemset(st, 0, sizeof(int32_t));
        unsigned long long w = wait_ns;
        void *args[] = {(void *)&gs, (void *)&st, (void *)&absent, (void *)&w};
        cudaEventRecord(e0, 0);
        if (launch_cooperative((const void *)k_grid_barrier_probe, dim3(ctas), dim3(64), args, 0, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            rc = FNEC_ERR_UNSUPPORTED;
            break;
        }
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = FNEC_ERR_CUDA;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (elapsed_ms) *elapsed_ms = ms;
        if (unit_status) cudaMemcpy(unit_status, st, sizeof(int32_t), cudaMemcpyDeviceToHost);
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(gs);
    cudaFree(st);
    return rc;
}
}  // namespace fnec

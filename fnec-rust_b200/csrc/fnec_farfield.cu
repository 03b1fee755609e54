// fnec_farfield.cu -- RP far-field gain grid (farfield.rs:265-291, :422-464,
// :514-546, :563-667) for every unit of a batch in two launches.
//
// Reference algorithm: for every direction, F = sum_n I_n L_n exp(jk r.r_n)
// projected on theta-hat and phi-hat (plus the PEC image), normalised by
// the radiated power integrated over a 1-degree grid (181x360 in free space,
// 91x360 over ground) with trapezoid weights in theta.
//
// B200 restatement: the segments of one GW wire share direction and length
// and their midpoints advance by a constant step, so along a wire
//   sum_n I_n exp(jk r.(m0 + n d)) = exp(jk r.m0) * P(z),  z = exp(jk r.d),
// with P(z) = sum_n I_n z^n evaluated by Horner's rule.  Each direction
// costs two sincos per wire run (sincospi_taylor on the phase in half-turns)
// and 4 FP64 FMAs per segment instead of one sincos per segment; the rounding difference to the reference's direct sum
// is O(n eps), i.e. ~1e-14 relative for runs of 100 segments (the parity
// bar for gains is 1e-6 dB).  The integral is a fixed-order block tree
// reduction (deterministic), and the gains, the Stokes axial ratio and the
// -999.99 clamps are formed on the device.
#include "fnec_kernels.h"
#include "fnec_libm.cuh"
#include "fnec_math.cuh"
#include "fnec_sincospi.cuh"

namespace fnec {

constexpr double RADS_PER_DEG = 3.14159265358979323846 / 180.0;  // Rust to_radians
constexpr int FF_THREADS = 128;

// Requested point p of an antenna: explicit list or RP card grid.
__device__ __forceinline__ void req_point(const DevRp &rp, const double *pts, int p, double &th,
                                          double &ph) {
    if (rp.pts_off >= 0) {
        th = pts[2 * (rp.pts_off + p)];
        ph = pts[2 * (rp.pts_off + p) + 1];
    } else {
        int ip = p / rp.n_theta, it = p % rp.n_theta;
        th = rp.theta0 + (double)it * rp.d_theta;
        ph = rp.phi0 + (double)ip * rp.d_phi;
    }
}

__device__ __forceinline__ void unit_vectors_dev(double th_deg, double ph_deg, double *rh,
                                                 double *thh, double *phh) {
    double th = th_deg * RADS_PER_DEG, ph = ph_deg * RADS_PER_DEG;
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    rh[0] = st * cp;
    rh[1] = st * sp;
    rh[2] = ct;
    thh[0] = ct * cp;
    thh[1] = ct * sp;
    thh[2] = -st;
    phh[0] = -sp;
    phh[1] = cp;
    phh[2] = 0.0;
}

// The same vectors with sin / cos of theta given (sincos(th * RADS_PER_DEG)
// of the direction's integration row, shared by the block).
__device__ __forceinline__ void unit_vectors_row(double st, double ct, double ph_deg, double *rh, double *thh,
                                                 double *phh) {
    double sp, cp;
    sincos(ph_deg * RADS_PER_DEG, &sp, &cp);
    rh[0] = st * cp;
    rh[1] = st * sp;
    rh[2] = ct;
    thh[0] = ct * cp;
    thh[1] = ct * sp;
    thh[2] = -st;
    phh[0] = -sp;
    phh[1] = cp;
    phh[2] = 0.0;
}

// Fields of two directions at once: Horner sums over the antenna's runs
// (+ images).  The two recurrences are independent, so each current load
// from shared memory feeds 8 FMAs on two dependency chains.
__device__ __forceinline__ void field_dir2(const DevRun *runs, int n_run, const cx *cur, double k, bool pec,
                                           const double *rh0, const double *th0, const double *ph0,
                                           const double *rh1, const double *th1, const double *ph1, cx &ft0,
                                           cx &fp0, cx &ft1, cx &fp1) {
    double a_tr = 0, a_ti = 0, a_pr = 0, a_pi = 0;
    double b_tr = 0, b_ti = 0, b_pr = 0, b_pi = 0;
    const double kpi = k * 0.31830988618379067;  // k / pi
    for (int q = 0; q < n_run; ++q) {
        const DevRun &R = runs[q];
        for (int img = 0; img < (pec ? 2 : 1); ++img) {
            double m0 = R.mid0[0], m1 = R.mid0[1], m2 = img ? -R.mid0[2] : R.mid0[2];
            double s0 = R.step[0], s1 = R.step[1], s2 = img ? -R.step[2] : R.step[2];
            double d0 = img ? -R.dir[0] : R.dir[0], d1 = img ? -R.dir[1] : R.dir[1], d2 = R.dir[2];
            // phases in half-turns (k / pi): sincospi_taylor needs no Cody-Waite reduction
            double pa = kpi * (m0 * rh0[0] + m1 * rh0[1] + m2 * rh0[2]);
            double da = kpi * (s0 * rh0[0] + s1 * rh0[1] + s2 * rh0[2]);
            double pb = kpi * (m0 * rh1[0] + m1 * rh1[1] + m2 * rh1[2]);
            double db = kpi * (s0 * rh1[0] + s1 * rh1[1] + s2 * rh1[2]);
            double eas, eac, zas, zac, ebs, ebc, zbs, zbc;
            sincospi_taylor_signed(pa, eas, eac);
            sincospi_taylor_signed(da, zas, zac);
            sincospi_taylor_signed(pb, ebs, ebc);
            sincospi_taylor_signed(db, zbs, zbc);
            const cx *I = cur + R.first;
            int c = R.count;
            cx last = I[c - 1];
            double ar = last.re, ai = last.im, br = last.re, bi = last.im;
            for (int n = c - 2; n >= 0; --n) {
                cx v = I[n];
                double nar = fma(ar, zac, fma(-ai, zas, v.re));
                double nai = fma(ar, zas, fma(ai, zac, v.im));
                double nbr = fma(br, zbc, fma(-bi, zbs, v.re));
                double nbi = fma(br, zbs, fma(bi, zbc, v.im));
                ar = nar;
                ai = nai;
                br = nbr;
                bi = nbi;
            }
            // F = exp(j p0) * acc * L, projected on theta-hat and phi-hat
            double fr = (eac * ar - eas * ai) * R.len, fi = (eac * ai + eas * ar) * R.len;
            double gr = (ebc * br - ebs * bi) * R.len, gi = (ebc * bi + ebs * br) * R.len;
            double pta = d0 * th0[0] + d1 * th0[1] + d2 * th0[2];
            double ppa = d0 * ph0[0] + d1 * ph0[1] + d2 * ph0[2];
            double ptb = d0 * th1[0] + d1 * th1[1] + d2 * th1[2];
            double ppb = d0 * ph1[0] + d1 * ph1[1] + d2 * ph1[2];
            a_tr = fma(fr, pta, a_tr);
            a_ti = fma(fi, pta, a_ti);
            a_pr = fma(fr, ppa, a_pr);
            a_pi = fma(fi, ppa, a_pi);
            b_tr = fma(gr, ptb, b_tr);
            b_ti = fma(gi, ptb, b_ti);
            b_pr = fma(gr, ppb, b_pr);
            b_pi = fma(gi, ppb, b_pi);
        }
    }
    ft0 = cx_make(a_tr, a_ti);
    fp0 = cx_make(a_pr, a_pi);
    ft1 = cx_make(b_tr, b_ti);
    fp1 = cx_make(b_pr, b_pi);
}

// Runs along z (every run of the antenna with zero x and y direction and
// step -- z-parallel wires): their Horner polynomial P(z) depends on the
// direction only through cos(theta), so along a theta row of the
// integration grid it is the same for all 360 phi.  A block evaluates it
// once per (row, run, image) into a shared table and each direction only
// forms exp(j k r.m0) P L and its projections -- the operations of
// field_dir2 on the same values (contraction choices aside), with one
// sincos per (direction, run) instead of two and no per-direction Horner.
constexpr int FF_VMAX = 32;  // largest run count of the per-row table

__device__ __forceinline__ bool run_is_vertical(const DevRun &R) {
    return R.dir[0] == 0.0 && R.dir[1] == 0.0 && R.step[0] == 0.0 && R.step[1] == 0.0;
}

// P of run R (image if img) for the direction of unit vector rh: Horner
// over its currents, as in field_dir2
__device__ __forceinline__ cx run_poly(const DevRun &R, const cx *cur, double k, int img, const double *rh) {
    double s0 = R.step[0], s1 = R.step[1], s2 = img ? -R.step[2] : R.step[2];
    double da = k * 0.31830988618379067 * (s0 * rh[0] + s1 * rh[1] + s2 * rh[2]);  // half-turns
    double zas, zac;
    sincospi_taylor_signed(da, zas, zac);
    const cx *I = cur + R.first;
    int c = R.count;
    cx last = I[c - 1];
    double ar = last.re, ai = last.im;
    for (int n = c - 2; n >= 0; --n) {
        cx v = I[n];
        double nar = fma(ar, zac, fma(-ai, zas, v.re));
        double nai = fma(ar, zas, fma(ai, zac, v.im));
        ar = nar;
        ai = nai;
    }
    return cx_make(ar, ai);
}

// The field of one direction from the per-row table P[run * 2 + img].
__device__ __forceinline__ void field_vert(const DevRun *runs, int n_run, const cx *P, double k, bool pec,
                                           const double *rh, const double *th, const double *ph, cx &ft, cx &fp) {
    double a_tr = 0, a_ti = 0, a_pr = 0, a_pi = 0;
    for (int q = 0; q < n_run; ++q) {
        const DevRun &R = runs[q];
        for (int img = 0; img < (pec ? 2 : 1); ++img) {
            double m0 = R.mid0[0], m1 = R.mid0[1], m2 = img ? -R.mid0[2] : R.mid0[2];
            double d0 = img ? -R.dir[0] : R.dir[0], d1 = img ? -R.dir[1] : R.dir[1], d2 = R.dir[2];
            double pa = k * 0.31830988618379067 * (m0 * rh[0] + m1 * rh[1] + m2 * rh[2]);  // half-turns
            double eas, eac;
            sincospi_taylor_signed(pa, eas, eac);
            const cx acc = P[q * 2 + img];
            double fr = (eac * acc.re - eas * acc.im) * R.len, fi = (eac * acc.im + eas * acc.re) * R.len;
            double pta = d0 * th[0] + d1 * th[1] + d2 * th[2];
            double ppa = d0 * ph[0] + d1 * ph[1] + d2 * ph[2];
            a_tr = fma(fr, pta, a_tr);
            a_ti = fma(fi, pta, a_ti);
            a_pr = fma(fr, ppa, a_pr);
            a_pi = fma(fi, ppa, a_pi);
        }
    }
    ft = cx_make(a_tr, a_ti);
    fp = cx_make(a_pr, a_pi);
}

// One direction's role: an integration direction (weight, and possibly the
// requested point that coincides with it) or a requested point of its own.
struct FfDir {
    bool live;       // a field is needed
    bool integ;      // contributes to the power integral with weight wgt
    double wgt;
    int req;         // requested point written with this field (-1: none)
    bool below;      // requested point below a PEC ground: zeros
    double th, ph;   // degrees
};

// sin_t_row: sin(theta) of the integration rows row_lo and row_lo + 1, as
// sin(th * RADS_PER_DEG) gives it (null: computed here)
__device__ __forceinline__ FfDir ff_dir(int d, int n_int, int n_xr, int n_th, double th_max, bool pec,
                                        const DevRp &rp, const double *pts, const int32_t *ibuf,
                                        const double *sin_t_row = nullptr, int row_lo = 0) {
    FfDir r{false, false, 0.0, -1, false, 0.0, 0.0};
    if (d < n_int) {
        int it = d / 360, ip = d % 360;
        r.th = (double)it * th_max / ((double)n_th - 1.0);
        r.ph = (double)ip;
        double sin_t = sin_t_row ? sin_t_row[it - row_lo] : sin(r.th * RADS_PER_DEG);
        double d_theta = (th_max * RADS_PER_DEG) / ((double)n_th - 1.0);
        double d_phi = 2.0 * 3.14159265358979323846 / 360.0;
        double w_t = (it == 0 || it == n_th - 1) ? 0.5 * d_theta : d_theta;
        // farfield.rs:441 skips sin(theta) == 0 rows
        if (sin_t != 0.0) {
            r.live = r.integ = true;
            r.wgt = sin_t * w_t * d_phi;
            r.req = rp.i2r_off >= 0 ? ibuf[rp.i2r_off + d] : -1;
        }
    } else if (d < n_int + n_xr) {
        int p = rp.i2r_off >= 0 ? ibuf[rp.xr_off + (d - n_int)] : d - n_int;
        req_point(rp, pts, p, r.th, r.ph);
        r.req = p;
        r.below = pec && r.th > 90.0;
        r.live = !r.below;
    }
    return r;
}

__device__ __forceinline__ void ff_store(double *fld_out, const UnitDesc &u, const FfDir &r, cx ft, cx fp) {
    if (r.req < 0) return;
    double *o = fld_out + 4 * (u.pat_off + r.req);
    if (r.below) {
        o[0] = o[1] = o[2] = o[3] = 0.0;
        return;
    }
    o[0] = ft.re;
    o[1] = ft.im;
    o[2] = fp.re;
    o[3] = fp.im;
}

// grid.x: direction blocks, grid.y: solve (status is per system).  Each
// thread takes directions d and d + FF_THREADS of its block's 2*FF_THREADS.
// Directions [0, n_int) are the power-integration grid (theta outer, phi
// inner, as integrate_power_for_ground iterates); [n_int, n_int + n_xr)
// the requested points not already covered by an integration direction.
// Requested fields go to fld_out (4 doubles per point); each block writes
// one partial integral.
__global__ void __launch_bounds__(FF_THREADS, 5) k_farfield(
    const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
    const DevRun *__restrict__ runs_all, const DevRp *__restrict__ rps, const double *__restrict__ pts,
    const int32_t *__restrict__ ibuf, const cx *__restrict__ xbuf, const int32_t *__restrict__ status,
    double *fld_out, double *partials, int max_blocks, int staged) {
    extern __shared__ unsigned char s_raw[];
    __shared__ double s_red[FF_THREADS / 32];
    int ui = blockIdx.y;
    UnitDesc u = units[ui];
    AntDesc a = ants[u.ant];
    DevRp rp = rps[u.ant];
    bool pec = a.ground == 1;
    int n_th = pec ? 91 : 181;
    double th_max = pec ? 90.0 : 180.0;
    int n_int = rp.skip_integral ? 0 : n_th * 360;
    int n_req = rp.pts_off >= 0 ? rp.n_pts : rp.n_theta * rp.n_phi;
    int n_xr = rp.i2r_off >= 0 ? rp.n_xr : n_req;
    int total = n_int + n_xr;
    int nblocks = (total + 2 * FF_THREADS - 1) / (2 * FF_THREADS);
    if ((int)blockIdx.x >= nblocks) return;
    if (status[u.sys] != 0) {
        if (threadIdx.x == 0) partials[(int64_t)ui * max_blocks + blockIdx.x] = 0.0;
        return;
    }
    // stage runs and currents in shared memory when they fit (else read L2)
    const DevRun *s_runs = runs_all + a.run_off;
    const cx *s_cur = xbuf + u.x_off;
    if (staged) {
        DevRun *sr = reinterpret_cast<DevRun *>(s_raw);
        cx *sc = reinterpret_cast<cx *>(s_raw + sizeof(DevRun) * a.n_run);
        for (int q = threadIdx.x; q < a.n_run; q += blockDim.x) sr[q] = runs_all[a.run_off + q];
        for (int q = threadIdx.x; q < a.n; q += blockDim.x) sc[q] = xbuf[u.x_off + q];
        s_runs = sr;
        s_cur = sc;
    }
    // the block's (at most two) integration rows: sin / cos of theta once per
    // block, as each direction would form them
    __shared__ double s_row_st[2], s_row_ct[2], s_row_sin[2];
    const int row_lo = (int)(blockIdx.x * 2 * FF_THREADS) / 360;
    if (threadIdx.x < 2) {
        const double th = (double)(row_lo + threadIdx.x) * th_max / ((double)n_th - 1.0);
        double st, ct;
        sincos(th * RADS_PER_DEG, &st, &ct);
        s_row_st[threadIdx.x] = st;
        s_row_ct[threadIdx.x] = ct;
        s_row_sin[threadIdx.x] = sin(th * RADS_PER_DEG);
    }
    __shared__ int s_vert;
    if (threadIdx.x == 32) {
        int v = a.n_run <= FF_VMAX && n_int > 0;
        for (int q = 0; v && q < a.n_run; ++q) v = run_is_vertical(runs_all[a.run_off + q]);
        s_vert = v;
    }
    __syncthreads();

    const int d0 = blockIdx.x * 2 * FF_THREADS + threadIdx.x, d1 = d0 + FF_THREADS;
    FfDir r0 = ff_dir(d0, n_int, n_xr, n_th, th_max, pec, rp, pts, ibuf, s_row_sin, row_lo);
    FfDir r1 = ff_dir(d1, n_int, n_xr, n_th, th_max, pec, rp, pts, ibuf, s_row_sin, row_lo);
    double rh0[3], th0[3], ph0[3], rh1[3], th1[3], ph1[3];
    if (d0 < n_int) unit_vectors_row(s_row_st[d0 / 360 - row_lo], s_row_ct[d0 / 360 - row_lo], r0.ph, rh0, th0, ph0);
    else unit_vectors_dev(r0.th, r0.ph, rh0, th0, ph0);
    if (d1 < n_int) unit_vectors_row(s_row_st[d1 / 360 - row_lo], s_row_ct[d1 / 360 - row_lo], r1.ph, rh1, th1, ph1);
    else unit_vectors_dev(r1.th, r1.ph, rh1, th1, ph1);
    // z-parallel antennas: the run polynomials of the block's (at most two)
    // integration rows, once per block
    __shared__ cx s_rowp[2][FF_VMAX * 2];
    const bool vert = s_vert != 0;
    if (vert) {
        const int nimg = pec ? 2 : 1;
        for (int t = threadIdx.x; t < 2 * a.n_run * nimg; t += blockDim.x) {
            const int rr = t / (a.n_run * nimg), q = (t / nimg) % a.n_run, img = t % nimg;
            const int row = row_lo + rr;
            if (row >= n_th) continue;
            double rh[3], th[3], ph[3];
            unit_vectors_row(s_row_st[rr], s_row_ct[rr], 0.0, rh, th, ph);
            s_rowp[rr][q * 2 + img] = run_poly(s_runs[q], s_cur, u.k_rp, img, rh);
        }
        __syncthreads();
    }
    double contrib = 0.0;
    if (r0.live || r1.live) {
        cx ft0, fp0, ft1, fp1;
        if (vert && d0 < n_int && d1 < n_int) {
            field_vert(s_runs, a.n_run, s_rowp[d0 / 360 - row_lo], u.k_rp, pec, rh0, th0, ph0, ft0, fp0);
            field_vert(s_runs, a.n_run, s_rowp[d1 / 360 - row_lo], u.k_rp, pec, rh1, th1, ph1, ft1, fp1);
        } else {
            field_dir2(s_runs, a.n_run, s_cur, u.k_rp, pec, rh0, th0, ph0, rh1, th1, ph1, ft0, fp0, ft1, fp1);
        }
        if (r0.integ) contrib += (ft0.re * ft0.re + ft0.im * ft0.im + fp0.re * fp0.re + fp0.im * fp0.im) * r0.wgt;
        if (r1.integ) contrib += (ft1.re * ft1.re + ft1.im * ft1.im + fp1.re * fp1.re + fp1.im * fp1.im) * r1.wgt;
        ff_store(fld_out, u, r0, ft0, fp0);
        ff_store(fld_out, u, r1, ft1, fp1);
    } else {
        ff_store(fld_out, u, r0, cx_make(0.0, 0.0), cx_make(0.0, 0.0));
        ff_store(fld_out, u, r1, cx_make(0.0, 0.0), cx_make(0.0, 0.0));
    }
    // deterministic block reduction of the integral contributions
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = contrib;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < FF_THREADS / 32; ++q) s += s_red[q];
        partials[(int64_t)ui * max_blocks + blockIdx.x] = s;
    }
}

// Per unit (blockIdx.y): total radiated power (fixed-order sum of block
// partials, formed by every block of the unit), then gains in dBi and the
// Stokes axial ratio for the requested points of this block's slice
// (blockIdx.x of gridDim.x).
__global__ void k_gains(const UnitDesc *__restrict__ units, const AntDesc *__restrict__ ants,
                        const DevRp *__restrict__ rps, const double *__restrict__ pts,
                        const int32_t *__restrict__ status,
                        const double *__restrict__ fld, const double *__restrict__ partials,
                        int max_blocks, double *pat_out, double *total_out) {
    __shared__ double s_total;
    int ui = blockIdx.y;
    UnitDesc u = units[ui];
    AntDesc a = ants[u.ant];
    DevRp rp = rps[u.ant];
    bool pec = a.ground == 1;
    int n_int = rp.skip_integral ? 0 : (pec ? 91 : 181) * 360;
    int n_req = rp.pts_off >= 0 ? rp.n_pts : rp.n_theta * rp.n_phi;
    int n_xr = rp.i2r_off >= 0 ? rp.n_xr : n_req;
    int nblocks = (n_int + n_xr + 2 * FF_THREADS - 1) / (2 * FF_THREADS);
    if (threadIdx.x == 0) {
        double t = 0.0;
        if (rp.skip_integral) t = rp.total_given;
        else
            for (int b = 0; b < nblocks; ++b) t += partials[(int64_t)ui * max_blocks + b];
        s_total = t;
        if (blockIdx.x == 0) total_out[ui] = status[u.sys] == 0 ? t : 0.0;
    }
    __syncthreads();
    double total = s_total;
    double norm = total > 0.0 ? 4.0 * 3.14159265358979323846 / total : 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_req; p += gridDim.x * blockDim.x) {
        double *o = pat_out + PAT_STRIDE * (u.pat_off + p);
        double th_deg, ph_deg;
        req_point(rp, pts, p, th_deg, ph_deg);
        if (status[u.sys] != 0 || (pec && th_deg > 90.0)) {
            o[0] = o[1] = o[2] = -999.99;
            o[3] = o[4] = o[5] = 0.0;
            continue;
        }
        const double *f = fld + 4 * (u.pat_off + p);
        cx ft = cx_make(f[0], f[1]), fp = cx_make(f[2], f[3]);
        double uth = ft.re * ft.re + ft.im * ft.im;
        double uph = fp.re * fp.re + fp.im * fp.im;
        double ut = uth + uph;
        o[0] = ut * norm > 1e-20 ? 10.0 * log10(ut * norm) : -999.99;
        o[1] = uth * norm > 1e-20 ? 10.0 * log10(uth * norm) : -999.99;
        o[2] = uph * norm > 1e-20 ? 10.0 * log10(uph * norm) : -999.99;
        // farfield.rs:659-667 Stokes axial ratio
        double s0 = ut;
        double ar = 0.0;
        if (s0 > 1e-30) {
            double s3 = 2.0 * (ft.im * fp.re - ft.re * fp.im);
            double q = s3 / s0;
            q = q < -1.0 ? -1.0 : (q > 1.0 ? 1.0 : q);
            ar = tan(0.5 * asin(q));
        }
        o[3] = ar;
        o[4] = uth;
        o[5] = uph;
    }
}

int farfield_max_blocks(int n_int_max, int n_req_max) {
    return (n_int_max + n_req_max + 2 * FF_THREADS - 1) / (2 * FF_THREADS);
}

void launch_farfield(const UnitDesc *units, int nu, const AntDesc *ants, const DevRun *runs,
                     const DevRp *rps, const double *pts, const int32_t *ibuf, const cx *x, const int32_t *status,
                     double *fld,
                     double *partials, int max_blocks, size_t smem, double *pat_out,
                     double *total_out, cudaStream_t st) {
    if (nu <= 0 || max_blocks <= 0) return;
    int staged = smem <= 200 * 1024;
    if (staged && smem > 0) {  // static + dynamic above 48 KB needs the raised limit
        int lim = set_smem_limit_once(k_farfield, 200 * 1024);
        if (lim < 0 || (size_t)lim < smem) staged = 0;
    }
    if (!staged) smem = 0;
    dim3 g(max_blocks, nu);
    k_farfield<<<g, FF_THREADS, smem, st>>>(units, ants, runs, rps, pts, ibuf, x, status, fld, partials,
                                            max_blocks, staged);
    // slices per unit: about one per 8 far-field blocks, at most 16
    const int gx = max_blocks / 8 < 1 ? 1 : (max_blocks / 8 > 16 ? 16 : max_blocks / 8);
    k_gains<<<dim3(gx, nu), 256, 0, st>>>(units, ants, rps, pts, status, fld, partials, max_blocks, pat_out,
                                          total_out);
}

// ---------------------------------------------------------------------------
// Near fields (farfield.rs:154-261 near_e_field / near_h_field): each
// segment is a Hertzian element of moment I_n L_n at its midpoint, and the
// field at P is the sum over segments in index order of
//   E += eta/(4 pi) I L e^{-jkr} [ rh 2c/r^2 (1 + 1/jkr)
//                                  + (c rh - u) jk/r^2 (1 + 1/jkr - 1/(kr)^2) ]
//   H += 1/(4 pi) I L e^{-jkr} jk/r^2 (1 + 1/jkr) (u x rh),
// c = u.rh, skipping segments whose midpoint is within 1e-9 m of P.  Every
// operation is a separately rounded FP64 op in the reference's order and
// sin/cos(kr) are the platform libm's values (fnec_libm.cuh), so a point's
// field is the CPU sum bit for bit.  One thread per point; the segment list is staged through shared
// memory in tiles that every thread of the block reads by broadcast.
// ---------------------------------------------------------------------------
constexpr int NF_THREADS = 128;
constexpr int NF_TILE = 128;
constexpr int NF_SEG_DOUBLES = 9;  // midpoint, direction, length, current (re, im)

__device__ __forceinline__ cx nf_scale(double s, cx a) { return cx_make(D_MUL(a.re, s), D_MUL(a.im, s)); }

__global__ void __launch_bounds__(NF_THREADS) k_near_field(const double *__restrict__ segs, int64_t n,
                                                           const cx *__restrict__ cur, double k, double coeff_e,
                                                           double coeff_h, const double *__restrict__ pts,
                                                           int64_t p, cx *e_out, cx *h_out) {
    __shared__ double tile[NF_TILE * NF_SEG_DOUBLES];
    const int64_t q = (int64_t)blockIdx.x * NF_THREADS + threadIdx.x;
    const bool live = q < p;
    double P[3] = {0.0, 0.0, 0.0};
    if (live)
        for (int c = 0; c < 3; ++c) P[c] = pts[3 * q + c];
    cx e[3], h[3];
    for (int a = 0; a < 3; ++a) e[a] = h[a] = cx_make(0.0, 0.0);
    const cx one = cx_make(1.0, 0.0);
    for (int64_t base = 0; base < n; base += NF_TILE) {
        const int cnt = (int)min((int64_t)NF_TILE, n - base);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt * NF_SEG_DOUBLES; t += NF_THREADS) {
            const int m = t / NF_SEG_DOUBLES, f = t % NF_SEG_DOUBLES;
            const int64_t g = base + m;
            tile[t] = f < 7 ? segs[7 * g + f] : (f == 7 ? cur[g].re : cur[g].im);
        }
        __syncthreads();
        if (!live) continue;
        for (int m = 0; m < cnt; ++m) {
            const double *s = &tile[m * NF_SEG_DOUBLES];
            const double d[3] = {D_SUB(P[0], s[0]), D_SUB(P[1], s[1]), D_SUB(P[2], s[2])};
            const double r = D_SQRT(D_ADD(D_ADD(D_MUL(d[0], d[0]), D_MUL(d[1], d[1])), D_MUL(d[2], d[2])));
            if (r < 1e-9) continue;
            const double rh[3] = {D_DIV(d[0], r), D_DIV(d[1], r), D_DIV(d[2], r)};
            const double *u = &s[3];
            const double len = s[6];
            const cx I = cx_make(s[7], s[8]);
            const double kr = D_MUL(k, r);
            double sn, cs;
            fnec_libm::libm_sincos(kr, &sn, &cs);
            const cx phase = cx_make(cs, -sn);
            const cx jkr = cx_make(0.0, kr);
            const cx one_p = cx_add(one, cx_div(one, jkr));
            const double rr = D_MUL(r, r);
            const cx jk_rr = cx_make(D_DIV(jkr.re, rr), D_DIV(jkr.im, rr));
            if (e_out) {
                const double c = D_ADD(D_ADD(D_MUL(u[0], rh[0]), D_MUL(u[1], rh[1])), D_MUL(u[2], rh[2]));
                const cx pref = cx_mul(nf_scale(D_MUL(len, coeff_e), I), phase);
                const double inv_kr2 = D_DIV(1.0, D_MUL(D_MUL(D_MUL(k, r), k), r));
                const cx rad = nf_scale(D_DIV(D_MUL(2.0, c), rr), one_p);
                const cx th = cx_mul(jk_rr, cx_sub(one_p, cx_make(inv_kr2, 0.0)));
                for (int a = 0; a < 3; ++a) {
                    const double tan_a = D_SUB(D_MUL(c, rh[a]), u[a]);
                    e[a] = cx_add(e[a], cx_mul(pref, cx_add(nf_scale(rh[a], rad), nf_scale(tan_a, th))));
                }
            }
            if (h_out) {
                const double cr[3] = {D_SUB(D_MUL(u[1], rh[2]), D_MUL(u[2], rh[1])),
                                      D_SUB(D_MUL(u[2], rh[0]), D_MUL(u[0], rh[2])),
                                      D_SUB(D_MUL(u[0], rh[1]), D_MUL(u[1], rh[0]))};
                const cx factor = cx_mul(jk_rr, one_p);
                const cx pref = cx_mul(cx_mul(nf_scale(D_MUL(len, coeff_h), I), phase), factor);
                for (int a = 0; a < 3; ++a) h[a] = cx_add(h[a], nf_scale(cr[a], pref));
            }
        }
    }
    if (!live) return;
    for (int a = 0; a < 3; ++a) {
        if (e_out) e_out[3 * q + a] = e[a];
        if (h_out) h_out[3 * q + a] = h[a];
    }
}

void launch_near_field(const double *segs, int64_t n, const cx *cur, double k, double coeff_e, double coeff_h,
                       const double *pts, int64_t p, cx *e_out, cx *h_out, cudaStream_t st) {
    if (p <= 0) return;
    const int64_t blocks = (p + NF_THREADS - 1) / NF_THREADS;
    k_near_field<<<(unsigned)blocks, NF_THREADS, 0, st>>>(segs, n, cur, k, coeff_e, coeff_h, pts, p, e_out, h_out);
}

}  // namespace fnec

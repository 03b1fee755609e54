// fnec_grid.cuh -- grid-wide pieces for systems too large for one CTA.
//
// 1. A bounded grid barrier for kernels launched cooperatively (all CTAs
//    co-resident).  Every wait has a wall-clock limit; a CTA that runs out
//    raises the shared error word, every other waiter sees it and leaves,
//    so a fault in the protocol ends the kernel instead of hanging it.
// 2. The panel factorisation of one 32-column panel spread over many CTAs
//    (row slices in shared memory, one barrier per column).  It performs the
//    same per-element operations as the one-CTA panel kernels:
//    - the pivot is the maximum of (norm, row) under the same total order
//      (larger norm, then larger row: the last-max rule of
//      linear.rs:1337-1352), which any reduction order reproduces;
//    - each row below the pivot gets f = a_rc / a_cc and then
//      a_rk -= f a_ck for the panel columns k > c, in column order.
//    So the factors are bit-identical to the unsplit kernel's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fnec_cuda.h"

namespace fnec {

constexpr int GRID_PANEL_MAX_CTAS = 320;  // CTAs per unit in a grid panel
constexpr int GRID_PANEL_MAX_UNITS = 16; // units per grid-panel launch
constexpr int32_t FNEC_STATUS_GRID_TIMEOUT = FNEC_UNIT_TIMEOUT;  // a grid barrier gave up

struct GridSync {
    unsigned int count;  // arrivals, monotonic within one launch
    int err;             // nonzero: a CTA timed out, everyone leaves
    unsigned int pad[2];
};

constexpr unsigned long long GRID_WAIT_NS = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ unsigned long long gtimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Barrier number `epoch` (1, 2, ...) of a launch whose GridSync was zeroed
// before the launch; nblocks CTAs take part; each CTA waits at most wait_ns.
// Returns false (in every thread of the CTA) when the barrier failed: the
// caller returns at once.
__device__ __forceinline__ bool grid_barrier(GridSync *gs, unsigned int nblocks, unsigned int epoch,
                                             unsigned long long wait_ns = GRID_WAIT_NS) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&gs->count, 1u);
        const unsigned int target = epoch * nblocks;
        volatile unsigned int *cnt = &gs->count;
        volatile int *err = &gs->err;
        int ok = 1;
        unsigned long long t0 = gtimer_ns();
        while (*cnt < target) {
            if (*err) {
                ok = 0;
                break;
            }
            if (gtimer_ns() - t0 > wait_ns) {
                atomicExch(&gs->err, 1);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Exchange area of one unit's grid panel: per CTA its pivot candidate and
// that candidate's panel row; plus the current row c.  Double-buffered by
// column parity: a CTA may write column c+1's candidate while a slower one
// still reads column c's.
template <class E>
struct PanelXchg {
    double cand_v[2][GRID_PANEL_MAX_CTAS];
    int cand_i[2][GRID_PANEL_MAX_CTAS];
    E cand_row[2][GRID_PANEL_MAX_CTAS][32];
    E row_c[2][32];
};

// Ops: E (element), V (pivot key), key(E) -> V, better(V&, int&, V, int),
// div(E, E), sub_mul(E acc, E f, E p) = acc - f p, singular(V), V_NONE,
// load_cg(const E*) (an L2 load: other CTAs' writes are read past L1).
template <class Ops, int PNB, int NT>
__device__ void panel_grid_body(typename Ops::E *A, int64_t ld, int s, int c0, int32_t *piv, int32_t *status_word,
                                PanelXchg<typename Ops::E> *xg, GridSync *gs, int G, int g,
                                typename Ops::E *s_pan /* [R][PNB] */) {
    using E = typename Ops::E;
    using V = typename Ops::V;
    __shared__ V s_v[NT / 32];
    __shared__ int s_i[NT / 32];
    __shared__ int s_p;
    __shared__ E s_prow[PNB];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int m = s - c0;
    if (m <= 0) return;
    const int nb = min(PNB, m);
    const int R = (m + G - 1) / G;
    const int r_lo = c0 + g * R;
    const int r_hi = min(s, r_lo + R);
    const int nl = max(0, r_hi - r_lo);  // local rows
    for (int e = tid; e < nl * nb; e += NT) {
        int rr = e / nb, q = e % nb;
        s_pan[rr * PNB + q] = A[(int64_t)(r_lo + rr) * ld + c0 + q];
    }
    __syncthreads();
    unsigned int epoch = 0;
    for (int c = c0; c < c0 + nb; ++c) {
        const int lc = c - c0, par = lc & 1;
        // local pivot candidate over owned rows >= c
        V bv = Ops::V_NONE;
        int bi = -1;
        for (int r = max(c, r_lo) + tid; r < r_hi; r += NT) Ops::better(bv, bi, Ops::key(s_pan[(r - r_lo) * PNB + lc]), r);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            V ov = __shfl_down_sync(0xffffffffu, bv, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            Ops::better(bv, bi, ov, oi);
        }
        if (lane == 0) {
            s_v[wid] = bv;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            V v = s_v[0];
            int p = s_i[0];
            for (int q = 1; q < NT / 32; ++q) Ops::better(v, p, s_v[q], s_i[q]);
            xg->cand_v[par][g] = (double)v;
            xg->cand_i[par][g] = p;
            s_p = p;
        }
        __syncthreads();
        {
            int p = s_p;
            if (p >= 0 && tid < nb) xg->cand_row[par][g][tid] = s_pan[(p - r_lo) * PNB + tid];
            if (c >= r_lo && c < r_hi && tid < nb) xg->row_c[par][tid] = s_pan[(c - r_lo) * PNB + tid];
        }
        if (!grid_barrier(gs, (unsigned)G, ++epoch)) {
            if (tid == 0) atomicExch(status_word, FNEC_STATUS_GRID_TIMEOUT);
            return;
        }
        // global pivot: the same maximum in every CTA
        {
            V v = Ops::V_NONE;
            int p = -1;
            for (int q = tid; q < G; q += NT) {
                int qi = __ldcg(&xg->cand_i[par][q]);
                if (qi >= 0) Ops::better(v, p, (V)__ldcg(&xg->cand_v[par][q]), qi);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                V ov = __shfl_down_sync(0xffffffffu, v, o);
                int oi = __shfl_down_sync(0xffffffffu, p, o);
                Ops::better(v, p, ov, oi);
            }
            if (lane == 0) {
                s_v[wid] = v;
                s_i[wid] = p;
            }
            __syncthreads();
            if (tid == 0) {
                V vv = s_v[0];
                int pp = s_i[0];
                for (int q = 1; q < NT / 32; ++q) Ops::better(vv, pp, s_v[q], s_i[q]);
                if (pp < 0 || Ops::singular(vv)) pp = -1;
                if (g == 0) {
                    piv[c] = pp;
                    if (pp < 0) *status_word = -(c + 1);
                }
                s_p = pp;
            }
            __syncthreads();
        }
        const int p = s_p;
        if (p < 0) return;
        const int wg = (p - c0) / R;  // rows are dealt out in contiguous slices
        if (tid < nb) s_prow[tid] = Ops::load_cg(&xg->cand_row[par][wg][tid]);
        __syncthreads();
        if (tid < nb) {
            if (c >= r_lo && c < r_hi) s_pan[(c - r_lo) * PNB + tid] = s_prow[tid];
            if (p != c && p >= r_lo && p < r_hi) s_pan[(p - r_lo) * PNB + tid] = Ops::load_cg(&xg->row_c[par][tid]);
        }
        __syncthreads();
        const E diag = s_prow[lc];
        const int first = max(c + 1, r_lo);
        for (int r = first + tid; r < r_hi; r += NT) {
            E *row = s_pan + (r - r_lo) * PNB;
            row[lc] = Ops::div(row[lc], diag);
        }
        __syncthreads();
        const int ncol = nb - lc - 1;
        if (ncol > 0 && first < r_hi) {
            const int nrow = r_hi - first;
            for (int e = tid; e < nrow * ncol; e += NT) {
                int rr = e / ncol, k = lc + 1 + e % ncol;
                E *row = s_pan + (first + rr - r_lo) * PNB;
                row[k] = Ops::sub_mul(row[k], row[lc], s_prow[k]);
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < nl * nb; e += NT) {
        int rr = e / nb, q = e % nb;
        A[(int64_t)(r_lo + rr) * ld + c0 + q] = s_pan[rr * PNB + q];
    }
}

}  // namespace fnec

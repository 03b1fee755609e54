// fnec_kernels.h -- host-side launch wrappers of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "fnec_math.cuh"
#include "fnec_types.h"

namespace fnec {

constexpr int PAT_STRIDE = 6;  // gain_total, gain_theta, gain_phi, axial_ratio, u_theta, u_phi

// Raise a kernel's dynamic shared-memory limit to its largest use, once per
// device.  The limit is a per-function attribute of the device's context,
// shared by every thread and stream there: setting it to each launch's own
// size would let a concurrent launch (another server lane) lower it under a
// larger one.
// Returns the kernel's resulting limit (bytes), or -1 if it could not be raised.
int set_smem_limit_once(const void *kernel, int bytes);  // fnec_plain.cu
// self-tests of the bounded waits (fnec_selftest_wait_timeout)
int selftest_grid_timeout(int32_t device, int32_t ctas, int32_t absent, uint64_t wait_ns, int32_t *unit_status,
                          double *elapsed_ms);                   // fnec_plain.cu
int selftest_tc_timeout(int32_t device, uint64_t wait_ns, int32_t *unit_status);  // fnec_tc.cu
template <class K>
inline int set_smem_limit_once(K kernel, int bytes) {
    return set_smem_limit_once(reinterpret_cast<const void *>(kernel), bytes);
}

// Device allocations of a batch: plain cudaMalloc, or the stream-ordered
// pool (cudaMallocAsync on the batch's stream) for server lanes.
struct DevAlloc {
    cudaStream_t st;
    bool pooled;
    // optional page-locked staging for uploads (a server lane's): copies go
    // through it asynchronously instead of from pageable memory
    unsigned char *stage = nullptr;
    size_t stage_cap = 0;
    size_t *stage_used = nullptr;
    cudaError_t alloc(void **p, size_t bytes) const {
        return pooled ? cudaMallocAsync(p, bytes, st) : cudaMalloc(p, bytes);
    }
    cudaError_t upload(void *dst, const void *src, size_t bytes) const {
        if (bytes == 0) return cudaSuccess;
        if (stage && stage_used && *stage_used + bytes <= stage_cap) {
            unsigned char *s = stage + *stage_used;
            std::memcpy(s, src, bytes);
            *stage_used += (bytes + 255) / 256 * 256;
            return cudaMemcpyAsync(dst, s, bytes, cudaMemcpyHostToDevice, st);
        }
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    }
    void release(void *p) const {
        if (!p) return;
        if (pooled) cudaFreeAsync(p, st);
        else cudaFree(p);
    }
};

// Units whose panels are too tall for one CTA's shared memory are factored
// by the grid-wide panel kernel (fnec_grid.cuh).  Built once per batch.
struct GridPlan {
    int32_t *d_order = nullptr;  // unit indices, s descending
    std::vector<int> s_desc;     // their s (host copy)
    void *d_xchg = nullptr;      // GRID_PANEL_MAX_UNITS exchange areas (complex128-sized)
    void *d_sync = nullptr;      // GridSync words: panel steps x GRID_PANEL_MAX_UNITS
    int steps = 0;               // panel steps the sync words cover
    int sms = 0;                 // SMs of the device
    // schedule (set per batch, the autotuner's choices)
    bool grid_on = true;         // tall panels grid-wide (else one CTA from global memory)
    int class_shift = 1;         // size classes of panel heights: (2^k x lo, hi]
    int factor_streams = 1;      // mixed factor: groups of units factored on concurrent streams
    int unit_factor = 1;         // mixed factor: units with S <= 256 / 384 / 512 (1 / 2 / 3) factored
                                 // whole, one CTA each; 0: none
};
size_t grid_xchg_bytes();        // bytes of d_xchg
size_t grid_sync_bytes(int steps);
// The units still active at panel step c0 (s > c0), in ranges [i0, i1) of
// the s-descending order whose panel heights m = s - c0 share a size class
// (<= 64, then powers of 2^class_shift above it); m_max is the range's
// tallest.  Starts at i_begin.
struct StepClass {
    int i0, i1, m_max;
};
// i_end >= 0 stops at that position of the order.
void step_classes(const GridPlan &gp, int c0, int i_begin, std::vector<StepClass> &out, int i_end = -1);
// A cooperative launch (every CTA co-resident) issued through
// cudaLaunchKernelExC so that stream capture records it as a cooperative
// kernel node.
cudaError_t launch_cooperative(const void *kernel, dim3 grid, dim3 block, void **args, size_t smem,
                               cudaStream_t st);
// How the panel at column c0 is factored (fnec_plain.cu): the number of
// units that take the grid-wide kernel (0 none, -1 infeasible) and its shape.
int plan_grid_panel(const GridPlan &gp, int c0, int thr_rows, int pnb, size_t elem, const void *kernel,
                    int *G_out, size_t *smem_out);

// fnec_plain.cu
void launch_expand_segments(const DevWire *wires, int nw, DevSeg *segs, cudaStream_t st);
// dtab: the batch's double table (path arc lengths and signs, AntDesc::arc_off)
void launch_hallen_rhs(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevSource *srcs, const double *dtab, cx *rhs, double *cosv,
                       double scale, cudaStream_t st);
void launch_fill_exact(const UnitDesc *units, const AntDesc *ants, const DevSeg *segs,
                       const int4 *tiles, int ntiles, cx *z, cudaStream_t st);
void launch_fill_exact_flat(const DevSeg *segs, int n, double k, int ground, cx *z, cudaStream_t st);
void launch_gram_exact(const UnitDesc *units, int nu, int max_w, const AntDesc *ants, const int4 *gtiles,
                       int ngtiles, const int32_t *ibuf, const DevConstraint *cons,
                       const int32_t *codes, const cx *z, const cx *rhs, const double *cosv, cx *A,
                       cudaStream_t st);
// returns the number of kernel launches issued
uint64_t launch_factor_exact(const UnitDesc *units, int nu, int max_s, const GridPlan &gp, cx *A,
                             int32_t *piv, int32_t *status, cudaStream_t st);
void launch_backsub(const UnitDesc *units, int nu, int max_s, const cx *A, cx *x,
                    const int32_t *status, cudaStream_t st);
// plane-wave forcing and homogeneous columns of the hom2 solves (x holds
// the incident field until the solve overwrites it)
void launch_planewave_rhs(const UnitDesc *solves, int ns, int max_n, const AntDesc *ants, const DevSeg *segs,
                          const int32_t *ibuf, const double *dtab, cx *x, cx *rhs, double *cosv, double scale,
                          cudaStream_t st);
// peak |I| per plane-wave solve (NaN for a failed system)
void launch_receive_peaks(const UnitDesc *solves, int ns, const AntDesc *ants, const cx *x, const int32_t *status,
                          double *peak, cudaStream_t st);
// Z[index] += (re, im) for every stamp (LD loads on the diagonal)
void launch_stamps(const DevStamp *stamps, int n, cx *z, cudaStream_t st);
void launch_feedpoints(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevFeed *feeds, const cx *x, const int32_t *status,
                       double *feed_out, const int64_t *feed_row_off, cudaStream_t st);
// groups (system, first solve, count <= 32): grouped kernels for many right-hand sides
void launch_extra_rhs_exact(const UnitDesc *solves, int ns, int max_s, const AntDesc *ants, const int32_t *ibuf,
                            const cx *z, const cx *rhs, const double *cosv, const cx *A, const int32_t *piv,
                            cx *x, const int32_t *status, cudaStream_t st, const int4 *groups = nullptr,
                            int n_groups = 0, int first_rhs = 1);  // first_rhs 0: every right-hand side
                                                                   // (a resident system's re-solve)

// fnec_farfield.cu
int farfield_max_blocks(int n_int_max, int n_req_max);
// ibuf: the int32 buffer the DevRp coverage maps index (may be null when
// every DevRp has i2r_off < 0)
void launch_farfield(const UnitDesc *units, int nu, const AntDesc *ants, const DevRun *runs,
                     const DevRp *rps, const double *pts, const int32_t *ibuf, const cx *x, const int32_t *status,
                     double *fld, double *partials, int max_blocks, size_t smem, double *pat_out,
                     double *total_out, cudaStream_t st);
// near E and H (either may be null) at p points from n segments given as
// fnec_gpu_segment records (7 doubles each) and their currents
void launch_near_field(const double *segs, int64_t n, const cx *cur, double k, double coeff_e, double coeff_h,
                       const double *pts, int64_t p, cx *e_out, cx *h_out, cudaStream_t st);

}  // namespace fnec

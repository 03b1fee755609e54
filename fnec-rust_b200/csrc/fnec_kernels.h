// fnec_kernels.h -- host-side launch wrappers of the device kernels.
#pragma once
#include <cuda_runtime.h>

#include "fnec_math.cuh"
#include "fnec_types.h"

namespace fnec {

constexpr int PAT_STRIDE = 6;  // gain_total, gain_theta, gain_phi, axial_ratio, u_theta, u_phi

// fnec_plain.cu
void launch_expand_segments(const DevWire *wires, int nw, DevSeg *segs, cudaStream_t st);
void launch_hallen_rhs(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevSource *srcs, cx *rhs, double *cosv,
                       double scale, cudaStream_t st);
void launch_fill_exact(const UnitDesc *units, const AntDesc *ants, const DevSeg *segs,
                       const int4 *tiles, int ntiles, cx *z, cudaStream_t st);
void launch_fill_exact_flat(const DevSeg *segs, int n, double k, int ground, cx *z, cudaStream_t st);
void launch_gram_exact(const UnitDesc *units, int nu, int max_w, const AntDesc *ants, const int4 *gtiles,
                       int ngtiles, const int32_t *ibuf, const DevConstraint *cons,
                       const int32_t *codes, const cx *z, const cx *rhs, const double *cosv, cx *A,
                       cudaStream_t st);
void launch_factor_exact(const UnitDesc *units, int nu, int max_s, int max_trailing_tiles, cx *A,
                         int32_t *piv, int32_t *status, cudaStream_t st);
void launch_backsub(const UnitDesc *units, int nu, int max_s, const cx *A, cx *x,
                    const int32_t *status, cudaStream_t st);
void launch_feedpoints(const UnitDesc *solves, int ns, const AntDesc *ants, const DevSeg *segs,
                       const int32_t *ibuf, const DevFeed *feeds, const cx *x, const int32_t *status,
                       double *feed_out, const int64_t *feed_row_off, cudaStream_t st);
void launch_extra_rhs_exact(const UnitDesc *solves, int ns, int max_s, const AntDesc *ants, const int32_t *ibuf,
                            const cx *z, const cx *rhs, const double *cosv, const cx *A, const int32_t *piv,
                            cx *x, const int32_t *status, cudaStream_t st);

// fnec_farfield.cu
int farfield_max_blocks(int n_int_max, int n_req_max);
void launch_farfield(const UnitDesc *units, int nu, const AntDesc *ants, const DevRun *runs,
                     const DevRp *rps, const double *pts, const cx *x, const int32_t *status,
                     double *fld, double *partials, int max_blocks, size_t smem, double *pat_out,
                     double *total_out, cudaStream_t st);

}  // namespace fnec

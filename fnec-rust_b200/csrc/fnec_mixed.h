// fnec_mixed.h -- the mixed-precision (FP32 factor + FP64 refinement) path.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "fnec_kernels.h"

namespace fnec {

struct MixedWork {
    size_t bytes = 0;
    void *base = nullptr;
};

// Phase events the mixed path records after its fill, Gram, factor and
// refinement phases (ev[0..3]); null when profiling is off.
struct MixedMarks {
    cudaEvent_t *ev;
};

bool mixed_available();
cudaError_t alloc_mixed(MixedWork &w, const std::vector<UnitDesc> &units, int max_s);
void free_mixed(MixedWork &w);
// Enqueue fill + Gram + factor + refinement for all units; returns the
// number of kernel launches issued.
uint64_t run_mixed(MixedWork &w, const UnitDesc *d_units, int nu, const std::vector<UnitDesc> &units,
                   const AntDesc *d_ants, const DevSeg *d_segs, const int4 *fill_tiles, int n_fill,
                   const int4 *gram_tiles, int n_gram, const int32_t *ibuf, const DevConstraint *cons,
                   const int32_t *codes, cx *z, const cx *rhs, const double *cosv, cx *A, cx *x,
                   int32_t *piv, int32_t *status, int max_s, bool do_fill, MixedMarks marks,
                   cudaStream_t st);

}  // namespace fnec

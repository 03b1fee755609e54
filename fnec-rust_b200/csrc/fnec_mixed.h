// fnec_mixed.h -- the mixed-precision (FP32 factor + FP64 refinement) path.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "fnec_kernels.h"

namespace fnec {

// defined in fnec_plain.cu (declared with its template wrapper in fnec_kernels.h)
int set_smem_limit_once(const void *kernel, int bytes);

struct TcGramPlan;
struct TcTrailPlan;

// Per-unit offsets into the mixed path's work buffers, and its refinement
// statistics (written by the GMRES kernel).
struct MixedUnit {
    int64_t a32_off;  // complex64 S*S factor
    int64_t v_off;    // complex128 Krylov basis
    int64_t w_off;    // complex128 work vectors
    int32_t rows;     // N + constraint rows
    int32_t iters;    // GMRES iterations used
    double resid;     // final preconditioned relative residual
    int64_t cs_off;   // complex128 scratch of the cluster GMRES (-1: none)
    int64_t binv_off; // complex64 inverses of the factor's 32x32 diagonal blocks (per system)
    int32_t b_ready;     // per solve: the Gram phase writes M^H y into the work vector b
    int32_t first_solve; // per system: its first solve when the Gram phase forms M^H y, else -1
};

struct MixedWork {
    size_t bytes = 0;
    void *base = nullptr;
    MixedUnit *mu = nullptr;   // per solve
    MixedUnit *smu = nullptr;  // per system (a32_off only)
    float2 *a32 = nullptr;
    float2 *binv = nullptr;      // per system: ceil(S/32) x (L11^-1, U11^-1), 32x32 each
    int2 *binv_tab = nullptr;    // (system, block) of every diagonal block: k_block_inv32's grid
    int n_binv = 0;
    int32_t *s_order = nullptr;  // solves by decreasing N^2 (refinement launch order)
    cx *v = nullptr;
    cx *w = nullptr;
    int n_units = 0;
    int max_s = 0;
    int mhy_systems = 0;  // systems whose M^H y the Gram phase forms (k_gram32_ccols_mhy)
    int mhy_max_n = 0;    // and their largest N
    std::vector<MixedUnit> host;
    // large solves refined by the grid-wide GMRES, one cooperative launch each
    std::vector<int> grid_solves;
    std::vector<int> grid_s;       // their s
    void *grid_base = nullptr;     // scratch shared by those launches
    int32_t *g_perm = nullptr;
    cx *g_part = nullptr;
    cx *g_y = nullptr;
    cx *g_red = nullptr;
    void *g_sync = nullptr;
    int grid_ctas = 0;
    // GMRES spread over thread-block clusters of cluster_c CTAs per solve
    // (when there are too few solves to fill the GPU one CTA each)
    int cluster_c = 1;    // in use (1: one CTA per solve); the tuner picks it
    int cluster_max = 1;  // largest cluster the scratch was sized for
    bool use_tc = true;   // Gram on the tensor cores (else the FP32 SIMT kernel); the tuner picks it
    bool grid_on = true;  // grid_solves refine grid-wide (else one CTA each); the tuner picks it
    bool use_binv = true; // the refinement applies the factor with diagonal block inverses
    int gmres_minb = 3;   // refinement CTAs per SM its registers are budgeted for (3 or 4)
    // concurrent factor groups: the batch stream plus these, forked and
    // joined with events (parallel branches of a captured graph)
    static constexpr int MAX_FACTOR_STREAMS = 4;
    cudaStream_t fstream[MAX_FACTOR_STREAMS - 1] = {};
    cudaEvent_t fevent[MAX_FACTOR_STREAMS] = {};
    bool fmade = false;
    cx *c_scratch = nullptr;
    void *c_base = nullptr;
    // the Gram block Z^H Z on the tensor cores (fnec_tc.cu)
    TcGramPlan *tc = nullptr;
    void *tc_base = nullptr;
    float *tc_hi = nullptr, *tc_lo = nullptr;
    void *tc_gu = nullptr, *tc_tiles = nullptr;
    int tc_max_n = 0;
    bool tc_fusable = false;  // the fill can write the Gram's operand stacks (k_fill_fast)
    // the factor's trailing updates of the largest units on the tensor cores
    TcTrailPlan *trail = nullptr;
    void *trail_base = nullptr;
    float *tr_hi = nullptr, *tr_lo = nullptr;
    void *d_trail = nullptr;  // TcTrailUnit per (step, unit)
    int trail_n = 0;          // units (a prefix of the s-descending order) it covers
    bool use_tc_trail = false; // the tuner picks it
    bool two_step = false;     // SIMT trailing updates once per two steps (look-ahead of the next panel)
    bool pivoting = false;     // GEPP with row exchanges; else the Hermitian factor without them
};

// Phase events the mixed path records after its fill, Gram, factor and
// refinement phases (ev[0..3]); null when profiling is off.
struct MixedMarks {
    cudaEvent_t *ev;
    const char *failed_phase = nullptr;  // set by run_mixed: the first phase whose launches failed
    char detail[160] = {0};               // the failed launch's shape, when known
};

bool mixed_available();
// systems: one per factorisation; solves: one per right-hand side.
// allow_grid: large solves may take the grid-wide (cooperative) GMRES
cudaError_t alloc_mixed(MixedWork &w, const std::vector<UnitDesc> &systems, const std::vector<UnitDesc> &solves,
                        const std::vector<AntDesc> &ants, int max_s, const DevAlloc &dev, bool allow_grid);
void free_mixed(MixedWork &w, const DevAlloc &dev);
// Enqueue fill + Gram + factor + refinement for all units; returns the
// number of kernel launches issued.
uint64_t run_mixed(MixedWork &w, const UnitDesc *d_units, int nu, const UnitDesc *d_solves, int ns,
                   const AntDesc *d_ants, const DevSeg *d_segs, const int4 *fill_tiles, int n_fill,
                   const int4 *gram_tiles, int n_gram, const int32_t *ibuf, const DevConRow *crows, cx *z,
                   const cx *rhs, const double *cosv, cx *x, int32_t *piv, int32_t *status, int max_s,
                   bool do_fill, int max_w, const GridPlan &gp, MixedMarks &marks, cudaStream_t st,
                   const DevStamp *stamps = nullptr, int n_stamps = 0);
// The refinement alone on the stored factor (run_mixed's last phase; a
// resident system's re-solve passes fresh_factor = false).
uint64_t refine_mixed(MixedWork &w, const UnitDesc *d_units, int nu, const UnitDesc *d_solves, int ns,
                      const AntDesc *d_ants, const int32_t *ibuf, const DevConRow *crows, const cx *z, const cx *rhs,
                      const double *cosv, cx *x, int32_t *piv, int32_t *status, int max_s, MixedMarks &marks,
                      cudaStream_t st, bool fresh_factor);
cudaError_t read_mixed_stats(MixedWork &w, int32_t *iters, double *resid, cudaStream_t st);

}  // namespace fnec

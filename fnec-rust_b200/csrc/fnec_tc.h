// fnec_tc.h -- the 3xTF32 tensor-core GEMM (fnec_tc.cu) and its Gram plan.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "fnec_mixed.h"

namespace fnec {

// x = hi + lo with both parts tf32 values, each rounded to nearest: the
// tensor core then uses lo as given (it would otherwise drop lo's low 13
// bits), so x is carried to ~2^-23 relative instead of ~2^-22.
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
    lo = __uint_as_float(l);
}

constexpr int TC_EPI_STORE = 0;  // C[R][C] = D (row-major FP32), bounds m x n
constexpr int TC_EPI_GRAM = 1;   // complex Gram combine into the unit's A32
constexpr int TC_EPI_TRAIL = 2;  // A22 -= L21 U12 of one factor step, into the unit's A32

// One unit's trailing update at one factor step (TC_EPI_TRAIL).  The
// complex product L21 U12 (m x 32 times 32 x m) runs as one real GEMM of
// K = 64 whose output columns interleave (Re, Im) like A32 itself:
//   A[i][k] = Re L(i,k), A[i][32+k] = Im L(i,k)
//   B[2j][k] = Re U(k,j), B[2j][32+k] = -Im U(k,j)
//   B[2j+1][k] = Im U(k,j), B[2j+1][32+k] = Re U(k,j)
// so D[i][2j+s] = (Re, Im) of (L U)(i,j).
struct TcTrailUnit {
    int32_t unit;    // system index
    int32_t m;       // trailing rows (= columns) at this step: s - c0 - 32
    int32_t m_pad;   // m rounded up to 128: A rows per k-block
    int32_t n2_pad;  // 2m rounded up to 128: B rows per k-block
    int64_t a_base, b_base;  // first rows of the unit's A and B in the stacks
};

// One 128x128 output tile.  Operand rows of k-block kb start at
// a_row + kb * a_kstride (A) and b_row + kb * b_kstride (B) of the
// K-blocked [rows][32] float stacks.
struct TcTile {
    int32_t a_row, b_row;
    int32_t a_kstride, b_kstride;
    int32_t kblocks;
    int32_t unit;
    int32_t ti, tj;
};

struct TcEpilogue {
    // TC_EPI_STORE
    float *c;
    int64_t ldc, m, n;
    // TC_EPI_GRAM
    const UnitDesc *units;
    const MixedUnit *mus;
    float2 *a32;
    int32_t lower_only;  // off-diagonal tiles write only their mirrored (lower) entries
    // both: a CTA whose waits ran out marks status[unit] (or status[0])
    int32_t *status;
    int32_t status_of_tile;
    // TC_EPI_TRAIL: the step and its units (blockIdx.y), tiles from blockIdx.x;
    // trail_lower: only tiles reaching the diagonal or below it (the
    // Hermitian factor), the others leave at once
    int32_t c0;
    const TcTrailUnit *trail;
    int32_t trail_lower;
    // limit of every mbarrier wait (0: TC_WAIT_NS, 2 s)
    uint64_t wait_ns;
    // self-test of the timeout path only: the producer stops issuing loads
    // at this k-block (-1 or 0 fields of a zeroed struct: never; see
    // fnec_selftest_wait_timeout)
    int32_t test_stop_kb;
    int32_t test_stop_on;
};

// Gram operand layout of one unit: T (2N x N) as kblocks k-blocks of rpad
// rows (2N rounded up to 128), starting at row `base` of the stacks.
struct TcGramUnit {
    int32_t unit;
    int32_t kblocks;
    int32_t rpad;
    int32_t pad;
    int64_t base;
};

struct TcGramPlan {
    std::vector<TcGramUnit> units;
    std::vector<TcTile> tiles;
    int64_t rows = 0;  // rows of each stack (hi, lo)
    CUtensorMap m_hi, m_lo;
    bool ready = false;
};

// The tensor-core trailing updates of the mixed factor: the units at
// positions [0, n) of the s-descending order, at every step where their
// trailing block has at least min_m rows.  Each unit owns operand rows in
// the stacks sized for its first step; later steps reuse them.
struct TcTrailPlan {
    std::vector<TcTrailUnit> units;  // every step's units, concatenated
    std::vector<int32_t> u_off;      // per step: first entry (steps + 1 values)
    std::vector<int32_t> max_tiles, max_mpad, max_n2pad;  // per step
    int64_t rows = 0;                // rows of each stack (hi, lo)
    CUtensorMap m_hi, m_lo;          // 128-row boxes (the A operand)
    CUtensorMap m_hi_b, m_lo_b;      // 64-row boxes (the B operand of 128 x 64 output tiles)
    bool ready = false;
    int steps() const { return (int)u_off.size() - 1; }
    int active(int step) const { return step < steps() ? u_off[step + 1] - u_off[step] : 0; }
};
cudaError_t tc_trail_plan(const std::vector<int> &s_desc, const std::vector<int32_t> &order, int n, int min_m,
                          TcTrailPlan &p);
bool tc_trail_maps(TcTrailPlan &p, const float *hi, const float *lo);
// Step `step` (c0 = 32 step): split L21 / U12 of the step's first `count`
// units (<= active(step)) into the stacks, then the GEMM subtracting
// L21 U12 from each one's A22.
// lower: the Hermitian factor's update, tiles on and below the diagonal
// only; persistent: one CTA per SM over the step's tiles with the
// accumulator double-buffered in TMEM (else one 128 x 64 tile per CTA)
cudaError_t tc_trail_run(const TcTrailPlan &p, int step, int count, const TcTrailUnit *d_trail, const UnitDesc *d_systems,
                         const MixedUnit *d_smu, float2 *a32, float *hi, float *lo, int32_t *status, cudaStream_t st,
                         bool lower = false, bool persistent = true);

cudaError_t tc_gram_plan(const std::vector<UnitDesc> &systems, TcGramPlan &p);
// Tensor maps over the hi / lo stacks (rows x 32 floats each); false when
// the driver's tensor-map encoder is unavailable.
bool tc_gram_maps(TcGramPlan &p, const float *hi, const float *lo);
// Z -> hi/lo stacks, then the tile GEMM writing Z^H Z into each unit's A32
// (its N x N block).
// lower_only: write only the tiles' lower-triangle entries (and the
// diagonal tiles whole), enough for the Hermitian factor
cudaError_t tc_gram_run(const TcGramPlan &p, const UnitDesc *d_units, const TcGramUnit *d_gu, const TcTile *d_tiles,
                        const MixedUnit *d_mus, const cx *z, float *hi, float *lo, float2 *a32, int32_t *status,
                        int max_n, cudaStream_t st, bool split = true,  // split false: the fill wrote the stacks
                        bool lower_only = false);

}  // namespace fnec

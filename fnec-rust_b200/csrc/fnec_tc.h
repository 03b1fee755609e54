// fnec_tc.h -- the 3xTF32 tensor-core GEMM (fnec_tc.cu) and its Gram plan.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "fnec_mixed.h"

namespace fnec {

constexpr int TC_EPI_STORE = 0;  // C[R][C] = D (row-major FP32), bounds m x n
constexpr int TC_EPI_GRAM = 1;   // complex Gram combine into the unit's A32

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
    // both: a CTA whose waits ran out marks status[unit] (or status[0])
    int32_t *status;
    int32_t status_of_tile;
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

cudaError_t tc_gram_plan(const std::vector<UnitDesc> &systems, TcGramPlan &p);
// Tensor maps over the hi / lo stacks (rows x 32 floats each); false when
// the driver's tensor-map encoder is unavailable.
bool tc_gram_maps(TcGramPlan &p, const float *hi, const float *lo);
// Z -> hi/lo stacks, then the tile GEMM writing Z^H Z into each unit's A32
// (its N x N block).
cudaError_t tc_gram_run(const TcGramPlan &p, const UnitDesc *d_units, const TcGramUnit *d_gu, const TcTile *d_tiles,
                        const MixedUnit *d_mus, const cx *z, float *hi, float *lo, float2 *a32, int32_t *status,
                        int max_n, cudaStream_t st);

}  // namespace fnec

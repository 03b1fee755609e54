// fnec_tc.cu -- 3xTF32 tensor-core GEMM on the 5th-generation tensor cores.
//
// D = A B^T over K, both operands K-major FP32, each split once into
// hi = tf32(x) and lo = x - hi; D = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
// recovers FP32-level accuracy (the dropped A_lo B_lo^T term is ~2^-22 of
// the product) at tensor-core rate.  One CTA computes one 128x128 tile:
//   warp 0   TMA producer: 4 boxes (A_hi, A_lo, B_hi, B_lo) of 128 rows x
//            32 floats (128 B, SWIZZLE_128B) per k-block, 3-stage ring
//   warp 1   MMA issuer: tcgen05.mma.cta_group::1.kind::tf32, M=128 N=128
//            K=8, 12 per k-block, accumulator in TMEM (128 columns)
//   warps 2-5  epilogue: tcgen05.ld of their TMEM lane quarter, then the
//            caller's epilogue (store, or the complex Gram combine)
// Operands live in "K-blocked" stacks: a [rows][32] float array where
// k-block kb of an operand row block starts kb * kstride rows after the
// first, so one tensor map serves every unit of an uneven batch.
// Every wait is bounded (2 s of global time); a CTA that gives up marks
// its unit FNEC_UNIT_TIMEOUT, drains its copies and MMAs and frees TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>

#include "fnec_cuda.h"
#include "fnec_grid.cuh"
#include "fnec_tc.h"

namespace fnec {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int STAGES = 3;
constexpr int BOX_BYTES = BM * BK * 4;         // 16 KB
constexpr int STAGE_BYTES = 4 * BOX_BYTES;    // A_hi, A_lo, B_hi, B_lo
constexpr int TRAIL_NT = 64;  // output tile width of the trailing update
constexpr int TC_THREADS = 192;
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait.  false: the CTA is aborting (abort word set by another role)
// or this wait ran out of time (it then sets the abort word).
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_word,
                          unsigned long long limit_ns = TC_WAIT_NS) {
    unsigned long long t0 = gtimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_word) return false;
        if ((it & 63) == 0 && gtimer_ns() - t0 > limit_ns) {
            *abort_word = 1;
            return false;
        }
    }
}
// Bounded wait that ignores the abort word (draining after an abort).
__device__ void mbar_drain(uint32_t bar, uint32_t parity, unsigned long long limit_ns = TC_WAIT_NS) {
    unsigned long long t0 = gtimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return;
        if ((it & 63) == 0 && gtimer_ns() - t0 > limit_ns) return;
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major operand tile written by TMA
// with SWIZZLE_128B: rows of 128 B, 8-row groups 1024 B apart (SBO), the
// swizzle applied on absolute address bits, so a K step inside the 128 B
// row is a plain start-address offset.
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address, 16 B units
    d |= (uint64_t)1 << 16;                    // leading byte offset (unused here)
    d |= (uint64_t)(1024 >> 4) << 32;          // stride byte offset
    d |= (uint64_t)1 << 46;                    // descriptor version
    d |= (uint64_t)2 << 61;                    // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D f32, A and B tf32, both K-major, M=128, N=NT.
template <int NT>
__host__ __device__ constexpr uint32_t idesc_tf32() {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <int NT>
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc_tf32<NT>()), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// -- epilogues ------------------------------------------------------------
// row: 0..127 inside the tile; v: 32 consecutive columns starting at col.
__device__ __forceinline__ void epi_store(const TcTile &t, const TcEpilogue &ep, int row, int col, const float (&v)[32]) {
    int64_t R = (int64_t)t.ti * BM + row;
    if (R >= ep.m) return;
    float *c = ep.c + R * ep.ldc;
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        int64_t C = (int64_t)t.tj * BN + col + j;
        if (C < ep.n) c[C] = v[j];
    }
}

// The complex Gram A = Z^H Z from D = T T^T with T[2c+s][k] = (Re, Im) Z[k][c]:
//   A[c][c'] = (D[2c][2c'] + D[2c+1][2c'+1], D[2c][2c'+1] - D[2c+1][2c']).
// Lanes 2i and 2i+1 hold rows 2c and 2c+1; the even lane writes complex
// columns 0..7 of the chunk, the odd lane 8..15.  Off-diagonal tiles also
// write the mirrored entries A[c'][c] = conj(A[c][c']).
__device__ __forceinline__ void epi_gram(const TcTile &t, const TcEpilogue &ep, int row, int col, const float (&v)[32],
                                         int lane) {
    float p[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) p[j] = __shfl_xor_sync(0xffffffffu, v[j], 1);
    const bool odd = lane & 1;
    const UnitDesc u = ep.units[t.unit];
    const int n = u.n, s = u.s;
    float2 *A = ep.a32 + ep.mus[t.unit].a32_off;
    const int c = (t.ti * BM + row) >> 1;
    const int c1 = ((t.tj * BN + col) >> 1) + (odd ? 8 : 0);
    if (c >= n) return;
    float2 out[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        float e0 = odd ? p[16 + 2 * q] : v[2 * q];
        float e1 = odd ? p[17 + 2 * q] : v[2 * q + 1];
        float o0 = odd ? v[16 + 2 * q] : p[2 * q];
        float o1 = odd ? v[17 + 2 * q] : p[2 * q + 1];
        out[q] = make_float2(e0 + o1, e1 - o0);
    }
    // tiles lie on and above the diagonal (ti <= tj): the entry at (c, c1 + q)
    // is the upper one; lower_only keeps diagonal tiles whole
    if (!ep.lower_only || t.ti == t.tj) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (c1 + q < n) A[(int64_t)c * s + c1 + q] = out[q];
    }
    if (t.ti != t.tj) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (c1 + q < n) A[(int64_t)(c1 + q) * s + c] = make_float2(out[q].x, -out[q].y);
    }
}

// A22 -= D for one factor step: rows c0 + 32 + tile row, float columns
// 2 (c0 + 32) + tile column of the unit's interleaved complex A32.  The
// warp's 32 x 32 block (a row per lane from TMEM) is transposed through
// shared memory (stg: 32 x 33 floats of the warp) so that each
// read-modify-write covers 32 consecutive floats of one row.
template <int NT>
__device__ __forceinline__ void epi_trail(const TcTile &t, const TcEpilogue &ep, int row0, int col, const float (&v)[32],
                                          int lane, float *stg) {
#pragma unroll
    for (int j = 0; j < 32; ++j) stg[lane * 33 + j] = v[j];
    __syncwarp();
    const int s = ep.units[t.unit].s;
    float *A = reinterpret_cast<float *>(ep.a32 + ep.mus[t.unit].a32_off);
    const int64_t F = 2 * ((int64_t)ep.c0 + 32) + (int64_t)t.tj * NT + col + lane;
    const int64_t R0 = (int64_t)ep.c0 + 32 + (int64_t)t.ti * BM + row0;
    // all reads (the transposed block, then A22) before any write, so no
    // load waits behind a store it might alias
    float d[32], a[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) d[r] = stg[r * 33 + lane];
    __syncwarp();
    const bool col_ok = F < 2 * (int64_t)s;
#pragma unroll
    for (int r = 0; r < 32; ++r) a[r] = (col_ok && R0 + r < s) ? A[(R0 + r) * 2 * s + F] : 0.f;
#pragma unroll
    for (int r = 0; r < 32; ++r)
        if (col_ok && R0 + r < s) A[(R0 + r) * 2 * s + F] = a[r] - d[r];
}

// NT: output tile width (B rows) -- 128, or 64 for the trailing update,
// whose smaller stages (ST of them) let two CTAs share an SM so that one
// CTA's read-modify-write epilogue overlaps the other's loads and MMAs.
template <int EPI, int NT = BN, int ST = STAGES>
__global__ void __launch_bounds__(TC_THREADS, (NT == BN ? 1 : 2))
    k_tc_gemm(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
              const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
              const TcTile *__restrict__ tiles, TcEpilogue ep) {
    constexpr int B_BOX = NT * BK * 4;
    constexpr int STG = 2 * BOX_BYTES + 2 * B_BOX;  // A_hi, A_lo, B_hi, B_lo
    constexpr int TCOLS = NT;                       // TMEM columns (power of 2, >= 32)
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2 * ST + 1];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    TcTile t;
    if (EPI == TC_EPI_TRAIL) {  // the tile from (unit of the step, tile index)
        const TcTrailUnit tu = ep.trail[blockIdx.y];
        const int ntj = tu.n2_pad / NT, ti = (int)blockIdx.x / ntj, tj = (int)blockIdx.x % ntj;
        if (ti >= tu.m_pad / BM) return;  // the whole CTA, before any barrier or TMEM allocation
        // complex columns [NT/2 tj, NT/2 (tj + 1)) against rows [128 ti, 128 ti + 128):
        // wholly above the diagonal when (NT/2) tj > 128 ti + 127
        if (ep.trail_lower && (NT / 2) * tj > BM * ti + BM - 1) return;
        t.a_row = (int32_t)(tu.a_base + (int64_t)ti * BM);
        t.b_row = (int32_t)(tu.b_base + (int64_t)tj * NT);
        t.a_kstride = tu.m_pad;
        t.b_kstride = tu.n2_pad;
        t.kblocks = 2;
        t.unit = tu.unit;
        t.ti = ti;
        t.tj = tj;
    } else {
        t = tiles[blockIdx.x];
    }
    const uint32_t sbase = smem_u32(smem);
    auto full = [&](int st) { return smem_u32(&s_bar[st]); };
    auto empty = [&](int st) { return smem_u32(&s_bar[ST + st]); };
    const uint32_t tfull = smem_u32(&s_bar[2 * ST]);
    volatile int *abort_word = &s_abort;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2 * ST + 1; ++i) mbar_init(smem_u32(&s_bar[i]), 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const unsigned long long wlim = ep.wait_ns ? (unsigned long long)ep.wait_ns : TC_WAIT_NS;
    const int stop_kb = ep.test_stop_on ? ep.test_stop_kb : INT_MAX;

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < t.kblocks && kb < stop_kb; ++kb) {
                const int st = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (kb >= ST && !mbar_wait(empty(st), ph ^ 1u, abort_word, wlim)) break;
                const uint32_t dst = sbase + st * STG;
                mbar_expect_tx(full(st), STG);
                const int ya = t.a_row + kb * t.a_kstride, yb = t.b_row + kb * t.b_kstride;
                tma_load_2d(dst, &mAh, 0, ya, full(st));
                tma_load_2d(dst + BOX_BYTES, &mAl, 0, ya, full(st));
                tma_load_2d(dst + 2 * BOX_BYTES, &mBh, 0, yb, full(st));
                tma_load_2d(dst + 2 * BOX_BYTES + B_BOX, &mBl, 0, yb, full(st));
                issued = kb + 1;
            }
            if (*abort_word || issued < t.kblocks)  // let the copies already issued land before the CTA exits
                for (int kb = issued - 1; kb >= 0 && kb >= issued - ST; --kb)
                    mbar_drain(full(kb % ST), (uint32_t)(kb / ST) & 1u, wlim);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int kb = 0; kb < t.kblocks; ++kb) {
                const int st = kb % ST;
                const uint32_t ph = (uint32_t)(kb / ST) & 1u;
                if (!mbar_wait(full(st), ph, abort_word, wlim)) break;
                tc_fence_after();
                const uint32_t a_hi = sbase + st * STG, a_lo = a_hi + BOX_BYTES;
                const uint32_t b_hi = a_hi + 2 * BOX_BYTES, b_lo = b_hi + B_BOX;
#pragma unroll
                for (int kk = 0; kk < BK / 8; ++kk) {
                    const uint32_t off = kk * 32;  // 8 tf32 = 32 B along the swizzled row
                    const uint64_t dah = sw128_kmajor_desc(a_hi + off), dal = sw128_kmajor_desc(a_lo + off);
                    const uint64_t dbh = sw128_kmajor_desc(b_hi + off), dbl = sw128_kmajor_desc(b_lo + off);
                    mma_tf32<NT>(tmem, dah, dbh, (kb | kk) != 0);
                    mma_tf32<NT>(tmem, dah, dbl, 1u);
                    mma_tf32<NT>(tmem, dal, dbh, 1u);
                }
                mma_commit(empty(st));
            }
            mma_commit(tfull);  // arrives once every MMA issued above has completed
            if (*abort_word) mbar_drain(tfull, 0, wlim);
        }
    } else {
        const bool ok = mbar_wait(tfull, 0, abort_word, wlim);
        tc_fence_after();
        if (ok) {
            const int q = warp & 3;  // TMEM lane quarter this warp may access
            const int row = q * 32 + lane;
            // every MMA has completed: the stage buffers are free for staging
            float *stg = reinterpret_cast<float *>(smem) + q * 32 * 33;
#pragma unroll 1
            for (int cc = 0; cc < NT / 32; ++cc) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cc * 32), v);
                if (EPI == TC_EPI_STORE) epi_store(t, ep, row, cc * 32, v);
                else if (EPI == TC_EPI_GRAM) epi_gram(t, ep, row, cc * 32, v, lane);
                else epi_trail<NT>(t, ep, q * 32, cc * 32, v, lane, stg);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
    if (threadIdx.x == 0 && *abort_word && ep.status) atomicExch(&ep.status[ep.status_of_tile ? t.unit : 0],
                                                                 FNEC_UNIT_TIMEOUT);
}

// -- the trailing update as a persistent kernel --------------------------------
//
// One CTA per SM walks the step's 128 x 64 output tiles (every unit of the
// step; with lower, the tiles wholly above the diagonal are skipped by all
// roles alike), so that nothing is set up per tile, and the accumulator is
// double-buffered in TMEM (2 x 64 columns): the MMA warp fills one buffer
// while the four epilogue warps read-modify-write A22 from the other, and
// the TMA producer runs PT_ST stages ahead across tile boundaries.  Barriers:
// full / empty per stage (k-blocks counted over the CTA's whole sequence),
// tfull per buffer (the MMA warp's commit) and tempty per buffer (one
// arrival from each epilogue warp after its TMEM reads).  Every wait is
// bounded; a CTA that gives up drains its copies and MMAs, frees TMEM and
// marks the unit of the tile it was on.
constexpr int PT_ST = 3;
constexpr int PT_EPI_WARPS = 8;  // two per TMEM lane quarter, one per 32-column chunk
constexpr int PT_THREADS = 32 * (2 + PT_EPI_WARPS);
constexpr int PT_MAX_UNITS = 1024;  // units per step it takes
// shared memory of a launch: PT_ST stages of A_hi, A_lo, B_hi, B_lo (+ the
// trailing update's epilogue staging, a 32 x 33 block per epilogue warp)
template <int EPI, int NT>
constexpr size_t pt_smem() {
    return (size_t)PT_ST * (2 * BOX_BYTES + 2 * NT * BK * 4) +
           (EPI == TC_EPI_TRAIL ? PT_EPI_WARPS * 32 * 33 * sizeof(float) : 0) + 1024;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Tile g of the step's sequence: its unit entry and grid position (false:
// g is past the end or, with lower, the tile lies wholly above the diagonal)
__device__ __forceinline__ bool pt_tile(const TcTrailUnit *tl, const int32_t *pre, int na, int g, bool lower,
                                        TcTile &t) {
    if (g >= pre[na]) return false;
    int lo = 0, hi = na;  // pre[lo] <= g < pre[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= g) lo = mid;
        else hi = mid;
    }
    const TcTrailUnit tu = tl[lo];
    const int ntj = tu.n2_pad / TRAIL_NT, x = g - pre[lo], ti = x / ntj, tj = x % ntj;
    if (lower && (TRAIL_NT / 2) * tj > BM * ti + BM - 1) return false;
    t.a_row = (int32_t)(tu.a_base + (int64_t)ti * BM);
    t.b_row = (int32_t)(tu.b_base + (int64_t)tj * TRAIL_NT);
    t.a_kstride = tu.m_pad;
    t.b_kstride = tu.n2_pad;
    t.kblocks = 2;
    t.unit = tu.unit;
    t.ti = ti;
    t.tj = tj;
    return true;
}

// The next tile of the sequence: the trailing update's tile g (decoded from
// the step's units), or entry g of the Gram's tile list.
template <int EPI>
__device__ __forceinline__ bool pt_next(const TcTrailUnit *tl, const TcTile *tiles, const int32_t *pre, int na,
                                        int g, bool lower, TcTile &t) {
    if (EPI == TC_EPI_TRAIL) return pt_tile(tl, pre, na, g, lower, t);
    t = tiles[g];
    return true;
}

// EPI TC_EPI_TRAIL (NT 64, na units of the step) or TC_EPI_GRAM (NT 128, na
// tiles in `tiles`)
template <int EPI, int NT>
__global__ void __launch_bounds__(PT_THREADS, 1)
    k_tc_persist(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                 const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                 const TcTile *__restrict__ tiles, int na, TcEpilogue ep) {
    constexpr int B_BOX = NT * BK * 4;
    constexpr int PT_STG = 2 * BOX_BYTES + 2 * B_BOX;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t s_bar[2 * PT_ST + 5];
    __shared__ int32_t s_pre[PT_MAX_UNITS + 1];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort, s_abort_unit;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    float *stage_out = reinterpret_cast<float *>(smem + PT_ST * PT_STG);  // TRAIL: epilogue warps x 32 x 33
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TcTrailUnit *tl = ep.trail;
    const bool lower = ep.trail_lower != 0;
    if (threadIdx.x == 0) {
        if (EPI == TC_EPI_TRAIL) {
            int acc = 0;
            for (int q = 0; q < na; ++q) {
                s_pre[q] = acc;
                acc += (tl[q].m_pad / BM) * (tl[q].n2_pad / NT);
            }
            s_pre[na] = acc;
        } else {
            s_pre[0] = na;
        }
        for (int i = 0; i < 2 * PT_ST; ++i) mbar_init(smem_u32(&s_bar[i]), 1);
        mbar_init(smem_u32(&s_bar[2 * PT_ST + 0]), 1);  // tfull 0
        mbar_init(smem_u32(&s_bar[2 * PT_ST + 1]), 1);  // tfull 1
        mbar_init(smem_u32(&s_bar[2 * PT_ST + 2]), PT_EPI_WARPS);  // tempty 0: one arrival per epilogue warp
        mbar_init(smem_u32(&s_bar[2 * PT_ST + 3]), PT_EPI_WARPS);  // tempty 1
        mbar_init(smem_u32(&s_bar[2 * PT_ST + 4]), 1);  // tdone: every MMA the issuer started
        s_abort = 0;
        s_abort_unit = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(2 * NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t sbase = smem_u32(smem);
    auto full = [&](int st) { return smem_u32(&s_bar[st]); };
    auto empty = [&](int st) { return smem_u32(&s_bar[PT_ST + st]); };
    auto tfull = [&](int b) { return smem_u32(&s_bar[2 * PT_ST + b]); };
    auto tempty = [&](int b) { return smem_u32(&s_bar[2 * PT_ST + 2 + b]); };
    volatile int *abort_word = &s_abort;
    const unsigned long long wlim = ep.wait_ns ? (unsigned long long)ep.wait_ns : TC_WAIT_NS;
    const int total = EPI == TC_EPI_TRAIL ? s_pre[na] : s_pre[0];
    TcTile t;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int kq = 0;   // k-blocks issued over the sequence
            for (int g = blockIdx.x; g < total && !*abort_word; g += gridDim.x) {
                if (!pt_next<EPI>(tl, tiles, s_pre, na, g, lower, t)) continue;
                for (int kb = 0; kb < t.kblocks; ++kb, ++kq) {
                    const int st = kq % PT_ST;
                    const uint32_t ph = (uint32_t)(kq / PT_ST) & 1u;
                    if (kq >= PT_ST && !mbar_wait(empty(st), ph ^ 1u, abort_word, wlim)) {
                        s_abort_unit = t.unit;
                        break;
                    }
                    const uint32_t dst = sbase + st * PT_STG;
                    mbar_expect_tx(full(st), PT_STG);
                    const int ya = t.a_row + kb * t.a_kstride, yb = t.b_row + kb * t.b_kstride;
                    tma_load_2d(dst, &mAh, 0, ya, full(st));
                    tma_load_2d(dst + BOX_BYTES, &mAl, 0, ya, full(st));
                    tma_load_2d(dst + 2 * BOX_BYTES, &mBh, 0, yb, full(st));
                    tma_load_2d(dst + 2 * BOX_BYTES + B_BOX, &mBl, 0, yb, full(st));
                }
            }
            if (*abort_word)  // let the copies already issued land before the CTA exits
                for (int q = kq - 1; q >= 0 && q >= kq - PT_ST; --q) mbar_drain(full(q % PT_ST), (uint32_t)(q / PT_ST) & 1u, wlim);
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            int kq = 0, i = 0;
            bool ok = true;
            for (int g = blockIdx.x; ok && g < total; g += gridDim.x) {
                if (!pt_next<EPI>(tl, tiles, s_pre, na, g, lower, t)) continue;
                const int b = i & 1;
                if (i >= 2 && !mbar_wait(tempty(b), (uint32_t)((i >> 1) - 1) & 1u, abort_word, wlim)) {
                    s_abort_unit = t.unit;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * NT);
                for (int kb = 0; kb < t.kblocks; ++kb, ++kq) {
                    const int st = kq % PT_ST;
                    if (!mbar_wait(full(st), (uint32_t)(kq / PT_ST) & 1u, abort_word, wlim)) {
                        s_abort_unit = t.unit;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_hi = sbase + st * PT_STG, a_lo = a_hi + BOX_BYTES;
                    const uint32_t b_hi = a_hi + 2 * BOX_BYTES, b_lo = b_hi + B_BOX;
#pragma unroll
                    for (int kk = 0; kk < BK / 8; ++kk) {
                        const uint32_t off = kk * 32;
                        const uint64_t dah = sw128_kmajor_desc(a_hi + off), dal = sw128_kmajor_desc(a_lo + off);
                        const uint64_t dbh = sw128_kmajor_desc(b_hi + off), dbl = sw128_kmajor_desc(b_lo + off);
                        mma_tf32<NT>(acc, dah, dbh, (kb | kk) != 0);
                        mma_tf32<NT>(acc, dah, dbl, 1u);
                        mma_tf32<NT>(acc, dal, dbh, 1u);
                    }
                    mma_commit(empty(st));
                }
                if (!ok) break;
                mma_commit(tfull(b));  // arrives once this tile's MMAs have completed
                ++i;
            }
            // a last commit tracks every MMA issued above (a tile cut short by an
            // abort included): TMEM is freed only after they complete
            mma_commit(smem_u32(&s_bar[2 * PT_ST + 4]));
            mbar_drain(smem_u32(&s_bar[2 * PT_ST + 4]), 0, wlim);
        }
    } else {  // epilogue warps 2..9: TMEM lane quarter q, every other 32-column chunk from c0
        const int q = warp & 3, c0 = (warp - 2) >> 2;
        float *stg = stage_out + (warp - 2) * 32 * 33;
        int i = 0;
        for (int g = blockIdx.x; g < total; g += gridDim.x) {
            if (!pt_next<EPI>(tl, tiles, s_pre, na, g, lower, t)) continue;
            const int b = i & 1;
            if (!mbar_wait(tfull(b), (uint32_t)(i >> 1) & 1u, abort_word, wlim)) {
                if (lane == 0) s_abort_unit = t.unit;
                break;
            }
            tc_fence_after();
#pragma unroll 1
            for (int cc = c0; cc < NT / 32; cc += 2) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * NT + cc * 32), v);
                if (EPI == TC_EPI_TRAIL) epi_trail<NT>(t, ep, q * 32, cc * 32, v, lane, stg);
                else epi_gram(t, ep, q * 32 + lane, cc * 32, v, lane);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty(b));
            ++i;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT));
    if (threadIdx.x == 0 && *abort_word && ep.status)
        atomicExch(&ep.status[s_abort_unit >= 0 ? s_abort_unit : 0], FNEC_UNIT_TIMEOUT);
}

// -- operand preparation (split_tf32: fnec_tc.h) -----------------------------

// Row-major FP32 [rows][k] -> K-blocked hi/lo stacks (zero padded to
// kblocks * 32 columns and rpad rows per k-block).
__global__ void k_split_rows(const float *__restrict__ src, int rows, int k, int rpad, float *hi, float *lo) {
    int kb = blockIdx.y, r = blockIdx.x * 8 + (threadIdx.x >> 5), j = threadIdx.x & 31;
    if (r >= rpad) return;
    int kk = kb * 32 + j;
    float x = (r < rows && kk < k) ? src[(int64_t)r * k + kk] : 0.f;
    float h, l;
    split_tf32(x, h, l);
    int64_t o = ((int64_t)kb * rpad + r) * 32 + j;
    hi[o] = h;
    lo[o] = l;
}

// Z (FP64 complex, N x N, row-major) -> the Gram operand T[2c+s][k] =
// (Re, Im) Z[k][c] as K-blocked hi/lo stacks, one unit per blockIdx.z.
// A 32 (k) x 16 (c) tile of Z is transposed through shared memory.
__global__ void k_split_gram(const UnitDesc *__restrict__ units, const TcGramUnit *__restrict__ gu,
                             const cx *__restrict__ zbuf, float *hi, float *lo) {
    __shared__ float s_t[32][33];  // [2c+s local][k local]
    const int ui = blockIdx.z;
    const TcGramUnit g = gu[ui];
    const UnitDesc u = units[g.unit];
    const int n = u.n;
    const int k0 = blockIdx.y * 32, c0 = blockIdx.x * 16;
    if (k0 >= g.kblocks * 32 || 2 * c0 >= g.rpad) return;
    const cx *z = zbuf + u.z_off;
    const int tid = threadIdx.x;  // 256 threads
    for (int e = tid; e < 32 * 16; e += 256) {
        int kk = e / 16, cc = e % 16, k = k0 + kk, c = c0 + cc;
        cx v = (k < n && c < n) ? z[(int64_t)k * n + c] : cx{0.0, 0.0};
        s_t[2 * cc][kk] = (float)v.re;
        s_t[2 * cc + 1][kk] = (float)v.im;
    }
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += 256) {
        int rr = e / 32, kk = e % 32;
        float h, l;
        split_tf32(s_t[rr][kk], h, l);
        int64_t o = ((int64_t)g.base + (int64_t)blockIdx.y * g.rpad + 2 * c0 + rr) * 32 + kk;
        hi[o] = h;
        lo[o] = l;
    }
}

// L21 of one factor step -> the trailing A operand (K-blocked hi/lo):
// k-block 0 the real parts, k-block 1 the imaginary parts, a warp per row.
__global__ void k_split_trail_a(const TcTrailUnit *__restrict__ tu_list, const UnitDesc *__restrict__ systems,
                                const MixedUnit *__restrict__ smu, const float2 *__restrict__ a32buf, int c0,
                                float *hi, float *lo) {
    const TcTrailUnit tu = tu_list[blockIdx.y];
    const int i = blockIdx.x * 8 + (threadIdx.x >> 5), k = threadIdx.x & 31;
    if (i >= tu.m_pad) return;
    const int s = systems[tu.unit].s;
    float2 v = make_float2(0.f, 0.f);
    if (i < tu.m) v = a32buf[smu[tu.unit].a32_off + (int64_t)(c0 + 32 + i) * s + c0 + k];
    float h, l;
    const int64_t o0 = (tu.a_base + i) * 32 + k, o1 = (tu.a_base + tu.m_pad + i) * 32 + k;
    split_tf32(v.x, h, l);
    hi[o0] = h;
    lo[o0] = l;
    split_tf32(v.y, h, l);
    hi[o1] = h;
    lo[o1] = l;
}

// U12 of one factor step -> the trailing B operand: rows 2j (Re U, -Im U)
// and 2j+1 (Im U, Re U) over k-blocks 0 / 1.  A 32 (k) x 32 (j) block of
// U is transposed through shared memory.
__global__ void k_split_trail_b(const TcTrailUnit *__restrict__ tu_list, const UnitDesc *__restrict__ systems,
                                const MixedUnit *__restrict__ smu, const float2 *__restrict__ a32buf, int c0,
                                float *hi, float *lo) {
    __shared__ float2 s_u[32][33];  // [j local][k]
    const TcTrailUnit tu = tu_list[blockIdx.y];
    const int j0 = blockIdx.x * 32;
    if (2 * j0 >= tu.n2_pad) return;
    const int s = systems[tu.unit].s;
    const float2 *A = a32buf + smu[tu.unit].a32_off;
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int k = e / 32, jj = e % 32, j = j0 + jj;
        s_u[jj][k] = j < tu.m ? A[(int64_t)(c0 + k) * s + c0 + 32 + j] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * 32; e += blockDim.x) {  // 64 B rows (2j + sgn) x 32 k
        const int rr = e / 32, k = e % 32, jj = rr >> 1, sg = rr & 1;
        const int64_t row = 2 * (int64_t)j0 + rr;
        if (row >= tu.n2_pad) continue;
        const float2 u = s_u[jj][k];
        const float x0 = sg ? u.y : u.x;   // k-block 0
        const float x1 = sg ? u.x : -u.y;  // k-block 1
        float h, l;
        const int64_t o0 = (tu.b_base + row) * 32 + k, o1 = (tu.b_base + tu.n2_pad + row) * 32 + k;
        split_tf32(x0, h, l);
        hi[o0] = h;
        lo[o0] = l;
        split_tf32(x1, h, l);
        hi[o1] = h;
        lo[o1] = l;
    }
}

// -- host --------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

bool make_map(CUtensorMap *m, const float *base, int64_t rows, int box_rows = BM) {
    std::call_once(g_encode_once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode || rows <= 0) return false;
    cuuint64_t dims[2] = {32, (cuuint64_t)rows};
    cuuint64_t strides[1] = {32 * sizeof(float)};
    cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t tc_smem_bytes() { return (size_t)STAGES * STAGE_BYTES + 1024; }

template <int EPI>
cudaError_t launch_tc(const CUtensorMap &ah, const CUtensorMap &al, const CUtensorMap &bh, const CUtensorMap &bl,
                      const TcTile *tiles, int ntiles, const TcEpilogue &ep, cudaStream_t st) {
    if (set_smem_limit_once((const void *)k_tc_gemm<EPI>, (int)tc_smem_bytes()) < (int)tc_smem_bytes())
        return cudaErrorInvalidConfiguration;
    if (ntiles <= 0) return cudaSuccess;
    k_tc_gemm<EPI><<<ntiles, TC_THREADS, tc_smem_bytes(), st>>>(ah, al, bh, bl, tiles, ep);
    return cudaGetLastError();
}

}  // namespace

// Gram plan: per unit the operand base row, padded rows and k-blocks; the
// tile list (upper triangle of 128x128 real tiles).
cudaError_t tc_gram_plan(const std::vector<UnitDesc> &systems, TcGramPlan &p) {
    p.units.clear();
    p.tiles.clear();
    int64_t rows = 0;
    for (size_t i = 0; i < systems.size(); ++i) {
        const int n = systems[i].n;
        if (n <= 0) continue;
        TcGramUnit g;
        g.unit = (int)i;
        g.kblocks = (n + 31) / 32;
        g.rpad = ((2 * n + BM - 1) / BM) * BM;
        g.base = rows;
        rows += (int64_t)g.kblocks * g.rpad;
        const int nt = g.rpad / BM;
        for (int ti = 0; ti < nt; ++ti)
            for (int tj = ti; tj < nt; ++tj) {
                TcTile t;
                t.a_row = (int32_t)(g.base + ti * BM);
                t.b_row = (int32_t)(g.base + tj * BM);
                t.a_kstride = t.b_kstride = g.rpad;
                t.kblocks = g.kblocks;
                t.unit = (int)i;
                t.ti = ti;
                t.tj = tj;
                p.tiles.push_back(t);
            }
        p.units.push_back(g);
    }
    p.rows = rows;
    return cudaSuccess;
}

cudaError_t tc_trail_plan(const std::vector<int> &s_desc, const std::vector<int32_t> &order, int n, int min_m,
                          TcTrailPlan &p) {
    p.units.clear();
    p.u_off.assign(1, 0);
    p.max_tiles.clear();
    p.max_mpad.clear();
    p.max_n2pad.clear();
    auto pad = [](int64_t x) { return (int32_t)((x + BM - 1) / BM * BM); };
    std::vector<int64_t> a_base(n), b_base(n);
    int64_t rows = 0;
    for (int q = 0; q < n; ++q) {  // stack rows sized for the unit's first step
        const int64_t m0 = std::max(0, s_desc[q] - 32);
        a_base[q] = rows;
        rows += 2 * (int64_t)pad(m0);
        b_base[q] = rows;
        rows += 2 * (int64_t)pad(2 * m0);
    }
    p.rows = rows;
    const int max_s = n > 0 ? s_desc[0] : 0;
    for (int c0 = 0; c0 < max_s; c0 += 32) {
        int32_t mt = 0, mm = 0, mn = 0;
        for (int q = 0; q < n && s_desc[q] - c0 - 32 >= min_m; ++q) {
            TcTrailUnit t;
            t.unit = order[q];
            t.m = s_desc[q] - c0 - 32;
            t.m_pad = pad(t.m);
            t.n2_pad = pad(2 * (int64_t)t.m);
            t.a_base = a_base[q];
            t.b_base = b_base[q];
            p.units.push_back(t);
            mt = std::max(mt, (t.m_pad / BM) * (t.n2_pad / BN));
            mm = std::max(mm, t.m_pad);
            mn = std::max(mn, t.n2_pad);
        }
        p.u_off.push_back((int32_t)p.units.size());
        p.max_tiles.push_back(mt);
        p.max_mpad.push_back(mm);
        p.max_n2pad.push_back(mn);
    }
    return cudaSuccess;
}

bool tc_trail_maps(TcTrailPlan &p, const float *hi, const float *lo) {
    p.ready = make_map(&p.m_hi, hi, p.rows) && make_map(&p.m_lo, lo, p.rows) &&
              make_map(&p.m_hi_b, hi, p.rows, TRAIL_NT) && make_map(&p.m_lo_b, lo, p.rows, TRAIL_NT);
    return p.ready;
}

cudaError_t tc_trail_run(const TcTrailPlan &p, int step, int count, const TcTrailUnit *d_trail, const UnitDesc *d_systems,
                         const MixedUnit *d_smu, float2 *a32, float *hi, float *lo, int32_t *status, cudaStream_t st,
                         bool lower, bool persistent) {
    const int na = std::min(count, p.active(step));
    if (na <= 0) return cudaSuccess;
    const TcTrailUnit *tl = d_trail + p.u_off[step];
    const int c0 = 32 * step;
    k_split_trail_a<<<dim3((unsigned)(p.max_mpad[step] / 8), (unsigned)na), 256, 0, st>>>(tl, d_systems, d_smu, a32,
                                                                                         c0, hi, lo);
    k_split_trail_b<<<dim3((unsigned)((p.max_n2pad[step] / 2 + 31) / 32), (unsigned)na), 256, 0, st>>>(
        tl, d_systems, d_smu, a32, c0, hi, lo);
    TcEpilogue ep{};
    ep.units = d_systems;
    ep.mus = d_smu;
    ep.a32 = a32;
    ep.status = status;
    ep.status_of_tile = 1;
    ep.c0 = c0;
    ep.trail = tl;
    ep.trail_lower = lower ? 1 : 0;
    constexpr size_t psm = pt_smem<TC_EPI_TRAIL, TRAIL_NT>();
    if (persistent && na <= PT_MAX_UNITS &&
        set_smem_limit_once((const void *)k_tc_persist<TC_EPI_TRAIL, TRAIL_NT>, (int)psm) >= (int)psm) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int64_t tiles = (int64_t)p.max_tiles[step] * (BN / TRAIL_NT) * na;  // bound on the sequence
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sms, tiles));
        k_tc_persist<TC_EPI_TRAIL, TRAIL_NT><<<grid, PT_THREADS, psm, st>>>(p.m_hi, p.m_lo, p.m_hi_b, p.m_lo_b,
                                                                          nullptr, na, ep);
        return cudaGetLastError();
    }
    // 128 x 64 output tiles in two 48 KB stages: two CTAs per SM
    constexpr size_t smem = (size_t)2 * (2 * BOX_BYTES + 2 * TRAIL_NT * BK * 4) + 1024;
    auto kern = k_tc_gemm<TC_EPI_TRAIL, TRAIL_NT, 2>;
    if (set_smem_limit_once((const void *)kern, (int)smem) < (int)smem) return cudaErrorInvalidConfiguration;
    kern<<<dim3((unsigned)(p.max_tiles[step] * (BN / TRAIL_NT)), (unsigned)na), TC_THREADS, smem, st>>>(
        p.m_hi, p.m_lo, p.m_hi_b, p.m_lo_b, nullptr, ep);
    return cudaGetLastError();
}

bool tc_gram_maps(TcGramPlan &p, const float *hi, const float *lo) {
    p.ready = make_map(&p.m_hi, hi, p.rows) && make_map(&p.m_lo, lo, p.rows);
    return p.ready;
}

cudaError_t tc_gram_run(const TcGramPlan &p, const UnitDesc *d_units, const TcGramUnit *d_gu, const TcTile *d_tiles,
                        const MixedUnit *d_mus, const cx *z, float *hi, float *lo, float2 *a32, int32_t *status,
                        int max_n, cudaStream_t st, bool split, bool lower_only) {
    if (p.units.empty()) return cudaSuccess;
    if (split) {  // else the fill has written the stacks
        int max_kb = (max_n + 31) / 32, max_cb = (max_n + 15) / 16;
        dim3 g(max_cb, max_kb, (unsigned)p.units.size());
        k_split_gram<<<g, 256, 0, st>>>(d_units, d_gu, z, hi, lo);
    }
    TcEpilogue ep{};
    ep.units = d_units;
    ep.mus = d_mus;
    ep.a32 = a32;
    ep.status = status;
    ep.status_of_tile = 1;
    ep.lower_only = lower_only ? 1 : 0;
    const int nt = (int)p.tiles.size();
    constexpr size_t psm = pt_smem<TC_EPI_GRAM, BN>();
    if (nt > 0 && set_smem_limit_once((const void *)k_tc_persist<TC_EPI_GRAM, BN>, (int)psm) >= (int)psm) {
        // persistent: one CTA per SM over the tile list, epilogue overlapping the next tile's MMAs
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_tc_persist<TC_EPI_GRAM, BN><<<std::max(1, std::min(sms, nt)), PT_THREADS, psm, st>>>(
            p.m_hi, p.m_lo, p.m_hi, p.m_lo, d_tiles, nt, ep);
        return cudaGetLastError();
    }
    return launch_tc<TC_EPI_GRAM>(p.m_hi, p.m_lo, p.m_hi, p.m_lo, d_tiles, nt, ep, st);
}

}  // namespace fnec

using namespace fnec;

// The GEMM self-test; stop_kb >= 0 makes the producer stop issuing loads
// at that k-block, so the MMA warp's wait on the next one runs out after
// wait_ns and the CTAs take the timeout path (drain, free TMEM, mark the
// status word), which *unit_status reports.
static int tc_selftest(int32_t device, uint64_t m, uint64_t n, uint64_t k, const float *a, const float *b, float *c,
                       int32_t stop_kb, uint64_t wait_ns, int32_t *unit_status) {
    if (!a || !b || !c || m == 0 || n == 0 || k == 0) return FNEC_ERR_BAD_ARG;
    if (m > (1u << 16) || n > (1u << 16) || k > (1u << 16)) return FNEC_ERR_TOO_LARGE;
    if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    const int kb = (int)((k + 31) / 32);
    const int mp = (int)((m + BM - 1) / BM) * BM, np = (int)((n + BN - 1) / BN) * BN;
    float *da = nullptr, *db = nullptr, *dc = nullptr, *ops = nullptr;
    TcTile *dt = nullptr;
    int32_t *dst = nullptr;
    size_t opa = (size_t)kb * mp * 32, opb = (size_t)kb * np * 32;
    int rc = FNEC_OK;
    std::vector<TcTile> tiles;
    for (int ti = 0; ti < mp / BM; ++ti)
        for (int tj = 0; tj < np / BN; ++tj) {
            TcTile t;
            t.a_row = ti * BM;
            t.b_row = tj * BN;
            t.a_kstride = mp;
            t.b_kstride = np;
            t.kblocks = kb;
            t.unit = 0;
            t.ti = ti;
            t.tj = tj;
            tiles.push_back(t);
        }
    do {
        if (cudaMalloc(&da, sizeof(float) * m * k) != cudaSuccess || cudaMalloc(&db, sizeof(float) * n * k) != cudaSuccess ||
            cudaMalloc(&dc, sizeof(float) * m * n) != cudaSuccess ||
            cudaMalloc(&ops, sizeof(float) * 2 * (opa + opb)) != cudaSuccess ||
            cudaMalloc(&dt, sizeof(TcTile) * tiles.size()) != cudaSuccess || cudaMalloc(&dst, sizeof(int32_t)) != cudaSuccess) {
            rc = FNEC_ERR_OUT_OF_MEMORY;
            break;
        }
        cudaMemcpy(da, a, sizeof(float) * m * k, cudaMemcpyHostToDevice);
        cudaMemcpy(db, b, sizeof(float) * n * k, cudaMemcpyHostToDevice);
        cudaMemcpy(dt, tiles.data(), sizeof(TcTile) * tiles.size(), cudaMemcpyHostToDevice);
        cudaMemset(dst, 0, sizeof(int32_t));
        float *ah = ops, *al = ops + opa, *bh = ops + 2 * opa, *bl = ops + 2 * opa + opb;
        k_split_rows<<<dim3(mp / 8, kb), 256>>>(da, (int)m, (int)k, mp, ah, al);
        k_split_rows<<<dim3(np / 8, kb), 256>>>(db, (int)n, (int)k, np, bh, bl);
        CUtensorMap mah, mal, mbh, mbl;
        if (!make_map(&mah, ah, (int64_t)kb * mp) || !make_map(&mal, al, (int64_t)kb * mp) ||
            !make_map(&mbh, bh, (int64_t)kb * np) || !make_map(&mbl, bl, (int64_t)kb * np)) {
            rc = FNEC_ERR_UNSUPPORTED;
            break;
        }
        TcEpilogue ep{};
        ep.c = dc;
        ep.ldc = (int64_t)n;
        ep.m = (int64_t)m;
        ep.n = (int64_t)n;
        ep.status = dst;
        ep.status_of_tile = 0;
        ep.wait_ns = wait_ns;
        ep.test_stop_on = stop_kb >= 0 ? 1 : 0;
        ep.test_stop_kb = stop_kb;
        if (launch_tc<TC_EPI_STORE>(mah, mal, mbh, mbl, dt, (int)tiles.size(), ep, 0) != cudaSuccess) {
            rc = FNEC_ERR_CUDA;
            break;
        }
        if (cudaDeviceSynchronize() != cudaSuccess) {
            rc = FNEC_ERR_CUDA;
            break;
        }
        int32_t stv = 0;
        cudaMemcpy(&stv, dst, sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (unit_status) *unit_status = stv;
        if (stv != 0) {
            rc = FNEC_ERR_TIMEOUT;
            break;
        }
        cudaMemcpy(c, dc, sizeof(float) * m * n, cudaMemcpyDeviceToHost);
    } while (0);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dc);
    cudaFree(ops);
    cudaFree(dt);
    cudaFree(dst);
    return rc;
}

extern "C" int fnec_selftest_tf32x3_gemm(int32_t device, uint64_t m, uint64_t n, uint64_t k, const float *a,
                                         const float *b, float *c) {
    return tc_selftest(device, m, n, k, a, b, c, -1, 0, nullptr);
}

namespace fnec {
// The timeout path of the tensor-core GEMM (fnec_selftest_wait_timeout):
// a 128 x 128 x 256 product whose loads stop after two of its eight
// k-blocks.  FNEC_OK when the CTA gave up within its limit and marked the
// status word; *unit_status is that word.
int selftest_tc_timeout(int32_t device, uint64_t wait_ns, int32_t *unit_status) {
    std::vector<float> a(128 * 256, 0.5f), b(128 * 256, 0.25f), c(128 * 128);
    int rc = tc_selftest(device, 128, 128, 256, a.data(), b.data(), c.data(), 2, wait_ns, unit_status);
    return rc == FNEC_ERR_TIMEOUT ? FNEC_OK : (rc == FNEC_OK ? FNEC_ERR_CUDA : rc);
}
}  // namespace fnec

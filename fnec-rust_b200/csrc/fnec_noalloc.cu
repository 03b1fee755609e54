// fnec_noalloc.cu -- radiation pattern that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc -- code that runs while
// a host framework owns all device memory through its own pool (the raw
// allocator is off limits there), plugins held to a fixed memory budget,
// and real-time loops that cannot afford the implicit device
// synchronisation of cudaMalloc/cudaFree.  They already hold their inputs
// and outputs in device memory and only need the pattern computed.
//
// How: the far-field kernels of fnec_farfield.cu need scratch (descriptors,
// the wire-run table, per-block partial integrals, per-point fields and
// gains).  Here that scratch is one file-scope static __device__ array of
// fixed size, so every GPU that loads the library holds it until the
// process exits.  Host code cannot use the array's name as a device address
// (the symbol is only a host-side stand-in): the first call on each device,
// with that device current, looks the address up with cudaGetSymbolAddress
// and caches it.  Every call shares the array and leaves its contents
// behind; everything a call reads is written or cleared by the same call
// first, and calls whose kernels overlap on the GPU race on the array.
#include <cuda_runtime.h>

#include <mutex>

#include "fnec_cuda.h"
#include "fnec_kernels.h"

namespace fnec {
namespace {

constexpr int NA_MAX_SEGMENTS = FNEC_NOALLOC_MAX_SEGMENTS;
constexpr int NA_MAX_POINTS = FNEC_NOALLOC_MAX_POINTS;
constexpr int NA_MAX_BLOCKS = 1024;  // >= (181*360 + NA_MAX_POINTS + 255) / 256 far-field blocks

struct NoallocScratch {
    UnitDesc unit;
    AntDesc ant;
    DevRp rp;
    int32_t status;  // the solve status the far-field kernels read: 0, the caller's currents are a solution
    int32_t pad;
    double total;
    DevRun runs[NA_MAX_SEGMENTS];
    double partials[NA_MAX_BLOCKS];
    double fld[4 * NA_MAX_POINTS];
    double pat[PAT_STRIDE * NA_MAX_POINTS];
};

// The scratch: about 5.6 MB per device, alive until the process exits.
static __device__ __align__(256) unsigned char g_pattern_scratch[sizeof(NoallocScratch)];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_mu;
NoallocScratch *g_addr[NA_MAX_DEVICES] = {};

// Device address of the scratch on the current device (looked up once).
int scratch_for_current_device(NoallocScratch **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_pattern_scratch);
        if (e != cudaSuccess || p == nullptr) return FNEC_ERR_CUDA;
        g_addr[dev] = static_cast<NoallocScratch *>(p);
    }
    *out = g_addr[dev];
    return FNEC_OK;
}

// Descriptors and the wire-run table of the caller's segments (one thread:
// consecutive segments with equal direction and length whose midpoints
// advance by a constant step share a run, as build_runs does on the host).
__global__ void k_na_setup(NoallocScratch *S, const fnec_gpu_segment *__restrict__ sg, int n, int p,
                           double k_rp, int ground) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int nr = 0;
    int i = 0;
    while (i < n) {
        int j = i + 1;
        double step[3] = {0, 0, 0};
        if (j < n)
            for (int c = 0; c < 3; ++c) step[c] = sg[j].midpoint[c] - sg[i].midpoint[c];
        double sl = sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]);
        while (j < n) {
            bool same = sg[j].direction[0] == sg[i].direction[0] && sg[j].direction[1] == sg[i].direction[1] &&
                        sg[j].direction[2] == sg[i].direction[2] && sg[j].length == sg[i].length;
            double e = 0, sc = 0;
            for (int c = 0; c < 3; ++c) {
                double pred = sg[i].midpoint[c] + step[c] * (double)(j - i);
                e = fmax(e, fabs(pred - sg[j].midpoint[c]));
                sc += fabs(sg[j].midpoint[c]);
            }
            if (!same || sl == 0.0 || e > 1e-12 * fmax(1.0, sc)) break;
            ++j;
        }
        DevRun r;
        for (int c = 0; c < 3; ++c) {
            r.mid0[c] = sg[i].midpoint[c];
            r.step[c] = (j - i > 1) ? step[c] : 0.0;
            r.dir[c] = sg[i].direction[c];
        }
        r.len = sg[i].length;
        r.first = i;
        r.count = j - i;
        S->runs[nr++] = r;
        i = j;
    }
    AntDesc a = {};
    a.n = n;
    a.w = 0;
    a.ground = ground;
    a.run_off = 0;
    a.n_run = nr;
    S->ant = a;
    UnitDesc u = {};
    u.ant = 0;
    u.n = n;
    u.s = n;
    u.k_rp = k_rp;
    u.x_off = 0;
    u.pat_off = 0;
    S->unit = u;
    DevRp rp = {};
    rp.pts_off = 0;
    rp.n_pts = p;
    rp.skip_integral = 0;
    rp.i2r_off = -1;  // no coverage maps: every requested point on its own
    rp.n_xr = p;
    S->rp = rp;
    S->status = 0;
    S->total = 0.0;
}

// gains rows (6 doubles) -> the caller's 4-double rows, and the integral
__global__ void k_na_repack(const NoallocScratch *__restrict__ S, int p, double *out, double *total) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < p)
        for (int c = 0; c < 4; ++c) out[4 * q + c] = S->pat[PAT_STRIDE * q + c];
    if (q == 0 && total) *total = S->total;
}

}  // namespace
}  // namespace fnec

using namespace fnec;

extern "C" int fnec_radiation_pattern_noalloc(const fnec_gpu_segment *d_segments, uint64_t n,
                                              const double *d_currents, double freq_hz, int32_t ground,
                                              const double *d_points, uint64_t p, double *d_out,
                                              double *d_total, void *stream) {
    if (!d_segments || !d_currents || n == 0) return FNEC_ERR_BAD_ARG;
    if (p > 0 && (!d_points || !d_out)) return FNEC_ERR_BAD_ARG;
    if (ground != FNEC_GROUND_FREE && ground != FNEC_GROUND_PEC) return FNEC_ERR_BAD_ARG;
    if (!(freq_hz > 0.0)) return FNEC_ERR_BAD_ARG;
    if (n > (uint64_t)NA_MAX_SEGMENTS || p > (uint64_t)NA_MAX_POINTS) return FNEC_ERR_TOO_LARGE;
    // A CUDA error still pending on this thread belongs to earlier work: it
    // is reported and left in place (not cleared), and nothing is launched,
    // so the launch check below sees this call's launches only.
    if (cudaPeekAtLastError() != cudaSuccess) return FNEC_ERR_CUDA;
    NoallocScratch *S = nullptr;
    int st = scratch_for_current_device(&S);
    if (st != FNEC_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double k_rp = 2.0 * 3.14159265358979323846 / (299792458.0 / freq_hz);  // farfield.rs:570-571
    k_na_setup<<<1, 32, 0, s>>>(S, d_segments, (int)n, (int)p, k_rp, ground);
    int n_int = (ground == FNEC_GROUND_PEC ? 91 : 181) * 360;
    int max_blocks = farfield_max_blocks(n_int, (int)p);
    // n_run <= n bounds the staged run table
    size_t smem = sizeof(DevRun) * (size_t)n + sizeof(cx) * (size_t)n;
    launch_farfield(&S->unit, 1, &S->ant, S->runs, &S->rp, d_points, nullptr, reinterpret_cast<const cx *>(d_currents),
                    &S->status, S->fld, S->partials, max_blocks, smem, S->pat, &S->total, s);
    int rb = (int)((p + 255) / 256);
    k_na_repack<<<rb > 0 ? rb : 1, 256, 0, s>>>(S, (int)p, d_out, d_total);
    if (cudaGetLastError() != cudaSuccess) return FNEC_ERR_CUDA;
    return FNEC_OK;
}

// fnec_peaks.cu -- FP64 pipe throughput microbenchmark.
//
// The exact-parity kernels are FP64-pipe bound and are built without FMA
// contraction; the roofline denominators for them are measured here on the
// same GPU: (a) fused DFMA throughput, (b) separately rounded DMUL + DADD
// throughput (what a no-FMA complex multiply-add issues).  Each thread runs
// 8 independent dependency chains so the pipe, not latency, is the limit.
#include <cuda_runtime.h>

#include "fnec_cuda.h"

namespace {

__global__ void k_dfma(double *out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-9 + q;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 12345.678) out[0] = s;
}

__global__ void k_dmuladd(double *out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-9 + q;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = __dadd_rn(__dmul_rn(x[q], a), b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 12345.678) out[0] = s;
}

__global__ void k_ffma(float *out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-6f + q;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = fmaf(x[q], a, b);
    }
    float s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 12345.678f) out[0] = s;
}

}  // namespace

extern "C" int fnec_measure_fp64_peak(int device, double *fma_tflops, double *muladd_tflops) {
    if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, device);
    double *d = nullptr;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return FNEC_ERR_OUT_OF_MEMORY;
    int blocks = p.multiProcessorCount * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best_f = 0, best_m = 0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        k_dfma<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        double fl = 2.0 * 8.0 * iters * (double)blocks * threads;  // 2 flops per FMA
        if (rep > 0) best_f = fl / (ms * 1e-3) / 1e12 > best_f ? fl / (ms * 1e-3) / 1e12 : best_f;
        cudaEventRecord(e0);
        k_dmuladd<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        double fm = 2.0 * 8.0 * iters * (double)blocks * threads;  // one mul + one add
        if (rep > 0) best_m = fm / (ms * 1e-3) / 1e12 > best_m ? fm / (ms * 1e-3) / 1e12 : best_m;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    if (cudaGetLastError() != cudaSuccess) return FNEC_ERR_CUDA;
    if (fma_tflops) *fma_tflops = best_f;
    if (muladd_tflops) *muladd_tflops = best_m;
    return FNEC_OK;
}

// FP32 FFMA throughput (the mixed form's FP32 factor runs on this pipe).
extern "C" int fnec_measure_fp32_peak(int device, double *ffma_tflops) {
    if (!ffma_tflops) return FNEC_ERR_BAD_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, device);
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float)) != cudaSuccess) return FNEC_ERR_OUT_OF_MEMORY;
    int blocks = p.multiProcessorCount * 8, threads = 256, iters = 8192;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        k_ffma<<<blocks, threads>>>(d, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        double fl = 2.0 * 8.0 * iters * (double)blocks * threads;
        if (rep > 0 && fl / (ms * 1e-3) / 1e12 > best) best = fl / (ms * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    *ffma_tflops = best;
    return cudaGetLastError() == cudaSuccess ? FNEC_OK : FNEC_ERR_CUDA;
}

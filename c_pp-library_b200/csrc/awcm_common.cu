// Library-wide C-ABI helpers: per-thread last-error text and the version string.
#include <cstdio>
#include <cstring>

#include "awcm_b200.h"
#include "awcm_common.cuh"

namespace awcm {

static thread_local char g_last_error[512] = "";

void set_last_error(const char* msg, const char* file, int line)
{
    const char* base = std::strrchr(file, '/');
    std::snprintf(g_last_error, sizeof(g_last_error), "%s (%s:%d)", msg, base ? base + 1 : file, line);
}

// FP64 peak probe: independent DFMA chains on every SM (2 flops per DFMA).
__global__ void k_dfma_probe(double* out, int iters)
{
    double a[8];
    for (int k = 0; k < 8; ++k) a[k] = (threadIdx.x + k) * 1e-9;
    const double b = 1.0000001, c = 1e-9;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0;
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == -1.0) out[threadIdx.x] = s;  // never true; keeps the chains live
}

}  // namespace awcm

extern "C" {

// Measures the dense FP64 FMA throughput of the current device (TFLOP/s, 2 flops per DFMA),
// best of `repeats` timed launches.
int awcm_measure_fp64_peak(int iters, int repeats, double* tflops)
{
    if (!tflops || iters <= 0 || repeats <= 0) return awcm::kErrArg;
    int dev = 0, sms = 0;
    AWCM_CUDA_TRY(cudaGetDevice(&dev));
    AWCM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double* out = nullptr;
    AWCM_CUDA_TRY(cudaMalloc(&out, 1024 * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256;
    awcm::k_dfma_probe<<<blocks, threads>>>(out, iters / 10 + 1);
    float best = 1e30f;
    for (int r = 0; r < repeats; ++r) {
        cudaEventRecord(e0);
        awcm::k_dfma_probe<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    AWCM_CUDA_TRY(cudaGetLastError());
    const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return awcm::kOk;
}


const char* awcm_last_error(void) { return awcm::g_last_error; }

const char* awcm_version(void) { return "awcm-b200 0.1 (sm_100a, fp64)"; }

}  // extern "C"

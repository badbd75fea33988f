// Shared host/device definitions of the AWCM B200 library: status codes, the interpolating-
// wavelet weight table, stencil clamping of the lifted transform and the block-wide compaction
// used to build the active-point worklists.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "awcm_numerics.cuh"

namespace awcm {

// Status codes of the C-ABI (also declared in include/awcm_b200.h).
enum Status : int {
    kOk = 0,
    kErrArg = 1,
    kErrOom = 2,
    kErrCuda = 3,
    kErrTimeout = 4,
    kErrNonFinite = 5,
    kErrState = 6,
};

// Mask bits of the per-point mask byte: 0..3 = mask0..mask3, 4 = the previous step's mask0
// (the reference's mask_temp), 5 = interpolation work mask, 6 = copy read by pushing passes.
// Ghost bytes follow the reference: mask0 starts true on the ghost ring, the other masks false,
// and the whole-field copies (mask_temp = mask0, mask_{k+1} = mask_k) carry the ghosts along.
constexpr int kBitTemp = 4, kBitInterp = 5, kBitCopy = 6;

// Lifted 4-point (N = 2) interpolating-wavelet weights w[i][j+1] = l_i(j + 1/2): Lagrange basis on
// nodes 0..3 evaluated halfway between nodes, built by the running product of WAVELET_1D::Initialize
// (Wavelet/WAVELET_1D.h:26-42).  Column k of a transform stencil (k = 0 left edge, 1 interior,
// 2 right edge) is w[.][k+1].
struct Weights {
    double w[4][5];
};

inline Weights make_weights()
{
    Weights W;
    for (int j = -1; j < 4; ++j)
        for (int i = 0; i < 4; ++i) {
            double v = 1;
            for (int k = 0; k < 4; ++k) {
                if (k == i) continue;
                v *= (j + 0.5 - k) / (i - k);
            }
            W.w[i][j + 1] = v;
        }
    return W;
}

// Predict stencil of a detail point c of level spacing D on [0, N1]: the coarse nodes
// c-3D/2 .. c+3D/2, shifted one-sided at the ends (WAVELET_1D.h:298-302).
__host__ __device__ __forceinline__ void predict_stencil(int c, int D, int N1, int& s, int& k)
{
    const int h = D >> 1;
    s = c - D - h;
    k = 1;
    if (s < 0) s = 0, k = 0;
    else if (c + D + h > N1) s = N1 - 3 * D, k = 2;
}

// Update (lifting) stencil of an even point: the four nearest detail points (WAVELET_1D.h:320-327).
__host__ __device__ __forceinline__ void update_stencil(int c, int D, int N1, int& s, int& k)
{
    const int h = D >> 1;
    s = c - D - h;
    k = 1;
    if (s < 0) s = h, k = 0;
    else if (c + D + h > N1) s = N1 - 3 * D - h, k = 2;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v)
{
    // Non-negative doubles order like their bit patterns.
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = maxd(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

#define AWCM_CUDA_TRY(expr)                                                                        \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            awcm::set_last_error(cudaGetErrorString(_e), __FILE__, __LINE__);                      \
            return _e == cudaErrorMemoryAllocation ? awcm::kErrOom : awcm::kErrCuda;               \
        }                                                                                          \
    } while (0)

void set_last_error(const char* msg, const char* file, int line);

}  // namespace awcm

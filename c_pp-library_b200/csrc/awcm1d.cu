// 1D AWCM compressible-Euler path on one B200 (sm_100a), FP64: single instances and batches.
//
// A 1D instance is small (Nx = (nx_coarse-1) 2^(L-1) + 1 points, 1025 for the Sod case, up to
// 8193 in the uneven batch), so one CTA advances one instance through a whole RK3 step --
// PrepareEuler, CFL, three stages, residue removal -- separating the level-sequential phases with
// block barriers instead of kernel launches.  A batch is one persistent launch: CTAs pull instance
// ids from a queue (largest first), so hundreds of uneven instances share the GPU in one kernel;
// a single instance is the same launch with one queue entry.  Each step is captured once into a
// CUDA graph (queue reset + step kernel) and replayed.
//
// Per-instance layout in the pool (w = Nx + 6, ghost ring 3): doubles q[3][w] (conserved),
// qc[3][w] (stage-start copy), qt[3][w] (coarse-point flux derivatives of a stage), fl[3][w] (face
// fluxes, face i+1/2 at point i), then w + 32 doubles holding the stage worklists of an instance
// too large to stage in shared memory (2 (w + 32) indices); bytes mask[w] (bits 0..3 mask0..3,
// 4 previous mask0, 5/6 work bits), then 16-byte aligned level[4][w].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "awcm_b200.h"
#include "awcm_common.cuh"

namespace awcm {
namespace {

struct Inst1 {
    int nx, maxl, scheme, pad0;
    double x_min, dx, gamma, tol, cfl, t, t_end, dt_fixed;
    long long q_off;  // in doubles
    long long m_off;  // in bytes
    // results of the last step
    double dt, mv, alpha[3];
    int do_print, done, steps, err;
    unsigned mask_cnt[4];
    unsigned long long upd;
    // the enum-driven BOUNDARY_MANAGER_1D<T> when bc_generic: BOUNDARY_CONDITION of the ghost cells
    // -1, -2, -3 (bcg[0..2]) and N1+1, N1+2, N1+3 (bcg[3..5])
    int8_t bcg[6];
    int8_t bc_generic, pad1;
};

// BOUNDARY_CONDITION values of the generic manager (BOUNDARY_MANAGER_1D.h:4-13).
constexpr int kBcPeriodic1 = -3, kBcExtrapolation1 = -2;

struct Pool {
    double* q;
    uint8_t* m;
    Weights W;
};

__device__ __forceinline__ double block_max(double v, double* red)
{
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double r = 0;
    const int nw = (blockDim.x + 31) >> 5;
    for (int k = 0; k < nw; ++k) r = maxd(r, red[k]);
    __syncthreads();
    return r;
}

// Sums of four per-thread counts over the block (one shared-memory round for all four).
__device__ __forceinline__ void block_sum4(unsigned (&v)[4], unsigned* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < 4; ++k) red[4 * warp + k] = v[k];
    __syncthreads();
    for (int k = 0; k < 4; ++k) {
        unsigned r = 0;
        for (int q = 0; q < nw; ++q) r += red[4 * q + k];
        v[k] = r;
    }
    __syncthreads();
}

// Exclusive prefix of v over the threads of the block (thread order); *total = the block sum.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* red, unsigned* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) red[warp] = x;
    __syncthreads();
    unsigned before = 0, all = 0;
    for (int k = 0; k < nw; ++k) {
        const unsigned r = red[k];
        before += k < warp ? r : 0u;
        all += r;
    }
    *total = all;
    return before + x - v;
}

// The same over 64-bit values (three packed 21-bit counts); red holds one 64-bit word per warp.
__device__ __forceinline__ unsigned long long block_exclusive_scan64(unsigned long long v, unsigned long long* red,
                                                                     unsigned long long* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) red[warp] = x;
    __syncthreads();
    unsigned long long before = 0, all = 0;
    for (int k = 0; k < nw; ++k) {
        const unsigned long long r = red[k];
        before += k < warp ? r : 0ull;
        all += r;
    }
    *total = all;
    return before + x - v;
}

// Block-wide stream compaction of the indices lo..hi whose predicate holds into `list` (order
// preserved).  Returns the count.  Each thread owns a contiguous chunk of the range: it counts its
// hits, one block-wide exclusive scan gives its output offset, and it writes its hits in order
// (two evaluations of the predicate, three barriers in all, whatever the range).
template <class Pred>
__device__ int block_compact(int lo, int hi, Pred pred, uint32_t* list, unsigned* red)
{
    const int n = hi - lo + 1;
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int a0 = lo + (int)threadIdx.x * per;
    const int a1 = min(a0 + per, hi + 1);
    unsigned cnt = 0;
    for (int i = a0; i < a1; ++i) cnt += pred(i) ? 1u : 0u;
    unsigned total;
    unsigned off = block_exclusive_scan(cnt, red, &total);
    for (int i = a0; i < a1; ++i)
        if (pred(i)) list[off++] = (uint32_t)i;
    __syncthreads();
    return (int)total;
}

// Views of one instance for a step or a pass.  Pointers are generic: in the step kernel the mask
// bytes, the levels and the density plane point into the CTA's shared memory (staged in and out
// around the step), elsewhere into the instance's global buffers.
struct Ctx {
    const Inst1& I;
    double* q;   // q[p*w + i + 3] (plane 0 is read through q0)
    double* qc;
    double* qt;
    double* fl;
    uint8_t* m;  // m[i + 3]
    int8_t* lv;  // lv[l*w + i + 3]
    const Weights& W;
    int w, nx, N1, maxl;
    double* q0;  // density plane: q0[i + 3]
    __device__ double& Q(int p, int i) const { return (p == 0 ? q0 : q + p * w)[i + kGhost]; }
    __device__ double& QT(int p, int i) const { return qt[p * w + i + kGhost]; }
    __device__ double& QC(int p, int i) const { return qc[p * w + i + kGhost]; }
    __device__ uint8_t& M(int i) const { return m[i + kGhost]; }
    __device__ int8_t& L(int l, int i) const { return lv[l * w + i + kGhost]; }
    __device__ bool bit(int i, int b) const { return (m[i + kGhost] >> b) & 1u; }
    // Mask push; pushes off the ghosted line (only reachable from inconsistent user-set
    // masks/levels, where the reference writes out of bounds) are dropped.
    // atomicOr on the containing 32-bit word: no dependent round trip per push.
    __device__ void set(int i, int b) const
    {
        if (i < -kGhost || i >= nx + kGhost) return;
        const uintptr_t a = reinterpret_cast<uintptr_t>(m + i + kGhost);
        atomicOr(reinterpret_cast<unsigned*>(a & ~(uintptr_t)3), 1u << (8 * (unsigned)(a & 3) + b));
    }
    // The push of the bits `bits` (one byte's worth) of point i in one atomicOr.
    __device__ void set_bits(int i, unsigned bits) const
    {
        if (i < -kGhost || i >= nx + kGhost) return;
        const uintptr_t a = reinterpret_cast<uintptr_t>(m + i + kGhost);
        atomicOr(reinterpret_cast<unsigned*>(a & ~(uintptr_t)3), bits << (8 * (unsigned)(a & 3)));
    }
    // The same push on the n <= 8 consecutive points i0 .. i0+n-1: one atomicOr per 32-bit word.
    __device__ void set_run(int i0, int n, int b) const
    {
        const int lo = i0 < -kGhost ? -kGhost : i0, hi = min(i0 + n - 1, nx + kGhost - 1);
        if (lo > hi) return;
        uintptr_t a = reinterpret_cast<uintptr_t>(m + lo + kGhost);
        const uintptr_t e = reinterpret_cast<uintptr_t>(m + hi + kGhost);
        while (a <= e) {
            const uintptr_t wb = a & ~(uintptr_t)3;
            const uintptr_t we = wb + 3 < e ? wb + 3 : e;
            unsigned bits = 0;
            for (uintptr_t x = a; x <= we; ++x) bits |= 1u << (8 * (unsigned)(x & 3) + b);
            atomicOr(reinterpret_cast<unsigned*>(wb), bits);
            a = we + 1;
        }
    }
    __device__ int D(int lev) const { return 1 << (maxl - lev); }
    __device__ double w_(int cnt, int k) const { return W.w[cnt][k + 1]; }
};

// ------------------------------------------------------------------ PrepareEuler building blocks
// ForwardWaveletTransformEuler (Wavelet/WAVELET_1D.h:282-335).
__device__ void fwt1(const Ctx& c)
{
    for (int lev = c.maxl - 1; lev >= 0; --lev) {
        const int D = c.D(lev), h = D >> 1, nd = c.N1 / D;
        for (int a = threadIdx.x; a < nd; a += blockDim.x) {
            const int i = h + a * D;
            if (!c.bit(i, 0)) continue;
            int s, k;
            predict_stencil(i, D, c.N1, s, k);
            double v = c.Q(0, i);
            for (int cnt = 0; cnt < 4; ++cnt) v -= c.w_(cnt, k) * c.Q(0, s + cnt * D);
            v *= 0.5;
            c.Q(0, i) = v;
            if (absd(v) < c.I.tol) c.M(i) &= (uint8_t)~1u;
        }
        __syncthreads();
        for (int a = threadIdx.x; a < nd - 1; a += blockDim.x) {
            const int i = D + a * D;
            if (!c.bit(i, 0)) continue;
            int s, k;
            update_stencil(i, D, c.N1, s, k);
            double v = c.Q(0, i);
            for (int cnt = 0; cnt < 4; ++cnt) v += c.w_(cnt, k) * c.Q(0, s + cnt * D);
            c.Q(0, i) = v;
        }
        __syncthreads();
    }
}

// InverseWaveletTransformEuler (Wavelet/WAVELET_1D.h:337-391).
__device__ void iwt1(const Ctx& c, int b)
{
    for (int lev = 0; lev < c.maxl; ++lev) {
        const int D = c.D(lev), h = D >> 1, nd = c.N1 / D;
        for (int a = threadIdx.x; a < nd - 1; a += blockDim.x) {
            const int i = D + a * D;
            if (!c.bit(i, b)) {
                c.Q(0, i) = 0;
                continue;
            }
            int s, k;
            update_stencil(i, D, c.N1, s, k);
            double v = c.Q(0, i);
            for (int cnt = 0; cnt < 4; ++cnt) v -= c.w_(cnt, k) * c.Q(0, s + cnt * D);
            c.Q(0, i) = v;
        }
        __syncthreads();
        for (int a = threadIdx.x; a < nd; a += blockDim.x) {
            const int i = h + a * D;
            if (!c.bit(i, b)) {
                c.Q(0, i) = 0;
                continue;
            }
            int s, k;
            predict_stencil(i, D, c.N1, s, k);
            double v = c.Q(0, i);
            v *= 2;
            for (int cnt = 0; cnt < 4; ++cnt) v += c.w_(cnt, k) * c.Q(0, s + cnt * D);
            c.Q(0, i) = v;
        }
        __syncthreads();
    }
}

// AWCM_MANAGER_1D::CheckReconstruction (Wavelet/AWCM_MANAGER_1D.h:45-71), fine to coarse.
__device__ void cr1(const Ctx& c, int b)
{
    for (int lev = c.maxl - 1; lev >= 0; --lev) {
        const int D = c.D(lev), h = D >> 1, nd = c.N1 / D;
        for (int a = threadIdx.x; a < nd; a += blockDim.x) {
            const int i = h + a * D;
            if (!c.bit(i, b)) continue;
            int s, k;
            predict_stencil(i, D, c.N1, s, k);
            for (int cnt = 0; cnt < 4; ++cnt) c.set(s + cnt * D, b);
        }
        __syncthreads();
    }
}

// AWCM_MANAGER_1D::AddAdjacentZone (Wavelet/AWCM_MANAGER_1D.h:14-43): detail points whose `src`
// bit is set mark their finer neighbours in `b` (and in `b2` too when it is given, in the same
// atomic).  i = odd * 2^t is a detail of level maxl-1-t.
__device__ void aaz1(const Ctx& c, int b, int src, int b2 = -1)
{
    const unsigned bits = (1u << b) | (b2 >= 0 ? 1u << b2 : 0u);
    for (int i = 1 + threadIdx.x; i <= c.N1 - 1; i += blockDim.x) {
        const int t = __ffs(i) - 1;
        if (t >= c.maxl || !c.bit(i, src)) continue;
        const int off = t == 0 ? 1 : (1 << (t - 1));
        c.set_bits(i - off, bits);
        c.set_bits(i + off, bits);
    }
    __syncthreads();
}

// BadingBoundary (AWCM_1D.h:73-80: mask0 set on the three points at each end, i < 3 and
// i > N1 - 3), then mask0 copied into the copy bit on the points [0, N1], one word at a time.
__device__ void band_copy1(const Ctx& c)
{
    unsigned* mw = reinterpret_cast<unsigned*>(c.m);
    for (int wi = (kGhost >> 2) + (int)threadIdx.x; wi <= ((c.N1 + kGhost) >> 2); wi += blockDim.x) {
        unsigned pts = 0, band = 0;  // bit 0 of the bytes of points [0, N1] / of the banded ones
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const int i = 4 * wi + L - kGhost;
            if (i < 0 || i > c.N1) continue;
            pts |= 1u << (8 * L);
            if (!(3 <= i && i <= c.N1 - 3)) band |= 1u << (8 * L);
        }
        const unsigned v0 = mw[wi], v = v0 | band;
        const unsigned nv = (v & ~(pts << kBitCopy)) | ((v & pts) << kBitCopy);
        if (nv != v0) mw[wi] = nv;
    }
    __syncthreads();
}

// AWCM_MANAGER_1D::AddPointForDifferentiation (Wavelet/AWCM_MANAGER_1D.h:73-107), reading the
// copy bit and level set l.
__device__ void apd1(const Ctx& c, int b, int l)
{
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        if (!c.bit(i, kBitCopy)) continue;
        const int lev = c.L(l, i);
        const int D = c.D(lev);
        const int is = i - 2 * D, ie = i + 2 * D;
        if (lev == c.maxl) {
            c.set_run(i - 3, 7, b);
        } else if (is <= 0) {
            for (int cnt = 0; cnt < 6; ++cnt) c.set(cnt * D, b);
        } else if (ie >= c.N1) {
            for (int cnt = 0; cnt < 6; ++cnt) c.set(c.N1 - cnt * D, b);
        } else {
            for (int cnt = 0; cnt < 5; ++cnt) c.set(is + cnt * D, b);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ bool mask_or_ghost1(const Ctx& c, int i, int b)
{
    if (i < -kGhost || i >= c.nx + kGhost) return true;
    return c.bit(i, b);
}

// AWCM_MANAGER_1D::ComputeLevel (Wavelet/AWCM_MANAGER_1D.h:109-133), with the optional copy
// mask_{k+1} = mask_k of the own point.  One 32-bit mask word (four points) per iteration: the copy
// is one word operation and the level search runs for the mask's points only.  The search reads
// bit b of other bytes, which no thread changes here (the copy writes bit copy_to, and bit
// copy_to2 too when it is given).
__device__ void cl1(const Ctx& c, int l, int b, int copy_to, int copy_to2 = -1)
{
    unsigned* mw = reinterpret_cast<unsigned*>(c.m);
    const int nw = (c.w + 3) >> 2;
    for (int wi = threadIdx.x; wi < nw; wi += blockDim.x) {
        const unsigned v = mw[wi];
        unsigned lanes = 0;  // the bytes of the word that are points of the line (ghosts included)
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const int i = 4 * wi + L - kGhost;
            if (i > c.N1 + kGhost) continue;
            lanes |= 1u << (8 * L);
            if (i < 0 || i > c.N1) continue;  // ghost byte: only the copy (the reference copies whole fields)
            if (i == 0 || i == c.N1) {
                c.L(l, i) = (int8_t)c.maxl;
            } else if (!((v >> (8 * L + b)) & 1u)) {
                c.L(l, i) = 0;
            } else {
                int dx = 1;
                for (int lev = c.maxl; lev >= 0; --lev) {
                    if (mask_or_ghost1(c, i - dx, b) || mask_or_ghost1(c, i + dx, b)) {
                        c.L(l, i) = (int8_t)lev;
                        break;
                    }
                    dx *= 2;
                }
            }
        }
        if (copy_to >= 0) {
            unsigned nv = (v & ~(lanes << copy_to)) | (((v >> b) & lanes) << copy_to);
            if (copy_to2 >= 0) nv = (nv & ~(lanes << copy_to2)) | (((v >> b) & lanes) << copy_to2);
            if (nv != v) mw[wi] = nv;
        }
    }
    __syncthreads();
}

// Copies bit `from` into bit `to` on the points [0, N1] (ghosts: [-3, N1+3]), a word at a time.
__device__ void copy_bit1(const Ctx& c, int from, int to, bool ghosts)
{
    const int x0 = ghosts ? 0 : kGhost, x1 = ghosts ? c.N1 + 2 * kGhost : c.N1 + kGhost;  // byte range
    unsigned* mw = reinterpret_cast<unsigned*>(c.m);
    for (int wi = (x0 >> 2) + (int)threadIdx.x; wi <= (x1 >> 2); wi += blockDim.x) {
        unsigned lanes = 0;
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const int x = 4 * wi + L;
            if (x >= x0 && x <= x1) lanes |= 1u << (8 * L);
        }
        const unsigned v = mw[wi];
        const unsigned nv = (v & ~(lanes << to)) | (((v >> from) & lanes) << to);
        if (nv != v) mw[wi] = nv;
    }
    __syncthreads();
}

// WAVELET_1D::InterpolateEuler(q, mra, from, to) (Wavelet/WAVELET_1D.h:393-431).
__device__ void interp1(const Ctx& c, int from, int to)
{
    // work bit = to and not from, on the points [0, N1], a word at a time
    unsigned* mw = reinterpret_cast<unsigned*>(c.m);
    for (int wi = (kGhost >> 2) + (int)threadIdx.x; wi <= ((c.N1 + kGhost) >> 2); wi += blockDim.x) {
        unsigned lanes = 0;
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const int x = 4 * wi + L;
            if (x >= kGhost && x <= c.N1 + kGhost) lanes |= 1u << (8 * L);
        }
        const unsigned v = mw[wi];
        const unsigned on = (v >> to) & ~(v >> from) & lanes;
        const unsigned nv = (v & ~(lanes << kBitInterp)) | (on << kBitInterp);
        if (nv != v) mw[wi] = nv;
    }
    __syncthreads();
    cr1(c, kBitInterp);
    for (int lev = 0; lev < c.maxl; ++lev) {
        const int D = c.D(lev), h = D >> 1, nd = c.N1 / D;
        for (int a = threadIdx.x; a < nd; a += blockDim.x) {
            const int i = h + a * D;
            if (!c.bit(i, kBitInterp) || c.bit(i, from)) continue;
            int s, k;
            predict_stencil(i, D, c.N1, s, k);
            for (int p = 1; p < 3; ++p) {
                double v = 0;
                for (int cnt = 0; cnt < 4; ++cnt) v += c.w_(cnt, k) * c.Q(p, s + cnt * D);
                c.Q(p, i) = v;
            }
        }
        __syncthreads();
    }
}

// AWCM_1D::PrepareEuler (Wavelet/AWCM_1D.h:86-120).
__device__ void prepare1(const Ctx& c)
{
    copy_bit1(c, 0, kBitTemp, true);
    fwt1(c);
    band_copy1(c);
    aaz1(c, 0, kBitCopy);
    cr1(c, 0);
    for (int k = 1; k <= 3; ++k) {
        // level_{k-1} of mask_{k-1}; mask_k = mask_{k-1}, and the copy bit too
        cl1(c, k - 1, k - 1, k, kBitCopy);
        // AddAdjacentZone(mask_k) reads bit k-1 (== mask_k before it) and marks bit k and the copy
        // bit, so the copy bit is mask_k after it: the input of AddPointForDifferentiation
        aaz1(c, k, k - 1, kBitCopy);
        apd1(c, k, k - 1);            // AddPointForDifferentiation(mask_k, level_{k-1})
        cr1(c, k);
    }
    cl1(c, 3, 3, -1);
    iwt1(c, 3);
    interp1(c, kBitTemp, 3);
}

// --------------------------------------------------------------------------------- RK3 stages
__device__ void bc1(const Ctx& c)
{
    if (threadIdx.x < 3 * kGhost) {
        const int p = threadIdx.x / kGhost, g = threadIdx.x % kGhost + 1;
        if (!c.I.bc_generic) {
            // BOUNDARY_MANAGER::SetBoundaryCondition (Problems/1D/PROBLEM_SHOCKTUBE.h:86-107).
            c.Q(p, -g) = c.Q(p, 0);
            c.Q(p, c.N1 + g) = c.Q(p, c.N1);
        } else {
            // BOUNDARY_MANAGER_1D<T>::SetBoundaryCondition (BOUNDARY_MANAGER_1D.h:47-75): zero-order
            // extrapolation or the periodic image (ghost -g <- N1-(g-1), N1+g <- g-1) by the
            // condition of each ghost cell; other conditions leave it.
            const int kl = c.I.bcg[g - 1], kr = c.I.bcg[kGhost + g - 1];
            if (kl == kBcExtrapolation1) c.Q(p, -g) = c.Q(p, 0);
            else if (kl == kBcPeriodic1) c.Q(p, -g) = c.Q(p, c.N1 - (g - 1));
            if (kr == kBcExtrapolation1) c.Q(p, c.N1 + g) = c.Q(p, c.N1);
            else if (kr == kBcPeriodic1) c.Q(p, c.N1 + g) = c.Q(p, g - 1);
        }
    }
    __syncthreads();
}

// nf: set when a speed is NaN or infinite (NaN/Inf state, negative pressure or density).
__device__ double lf_speed1(const Ctx& c, int b, int l, double* red, bool& nf)
{
    // main_1d_euler.cpp:86-95: max |u|+c over the finest-level points of mask b.
    double a = 0;
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        if (!c.bit(i, b) || c.L(l, i) != c.maxl) continue;
        const double q0 = c.Q(0, i), q1 = c.Q(1, i), q2 = c.Q(2, i);
        const double u = q1 / q0;
        const double s = sound1(q0, q1, q2, c.I.gamma);
        nf |= !isfinite(absd(u) + s);
        a = maxd(a, absd(u) + s);
    }
    return block_max(a, red);
}

// Coarse-level flux derivative (AWCM_1D::DifferentiateEuler*, Wavelet/AWCM_1D.h:142-189) with the
// driver's branch selection (main_1d_euler.cpp:111-133); right-boundary forms mirror the left ones.
// Reads the stage input Q, which no point update has touched yet when it runs.
__device__ void coarse_dF1(const Ctx& c, int i, int d, double* dF)
{
    const double g = 1.4;  // EULER_EQUATION_1D euler_eqn(1.4) in the reference helpers
    auto F = [&](int ii, double* f) {
        const double s[3] = {c.Q(0, ii), c.Q(1, ii), c.Q(2, ii)};
        flux1(s, g, f);
    };
    const int iend = c.N1;
    double a[3], b[3], e[3], f[3], h[3];
    if (i - 2 * d > 0 && i + 2 * d < iend) {
        F(i - 2 * d, a), F(i - d, b), F(i + d, e), F(i + 2 * d, f);
        for (int p = 0; p < 3; ++p) dF[p] = kD1 * (e[p] - b[p]) + kD2 * (f[p] - a[p]);
    } else if (i - 2 * d < 0) {
        F(i - d, a), F(i, b), F(i + d, e), F(i + 2 * d, f);
        for (int p = 0; p < 3; ++p) dF[p] = kD01 * a[p] + kD11 * b[p] + kD21 * e[p] + kD31 * f[p];
    } else if (i == 2 * d) {
        F(i - 2 * d, a), F(i - d, b), F(i, e), F(i + d, f), F(i + 2 * d, h);
        for (int p = 0; p < 3; ++p) dF[p] = kD02 * a[p] + kD12 * b[p] + kD22 * e[p] + kD32 * f[p] + kD2 * h[p];
    } else if (i > iend - 2 * d) {
        F(i + d, a), F(i, b), F(i - d, e), F(i - 2 * d, f);
        for (int p = 0; p < 3; ++p) dF[p] = kD01 * a[p] + kD11 * b[p] + kD21 * e[p] + kD31 * f[p];
    } else {
        F(i + 2 * d, a), F(i + d, b), F(i, e), F(i - d, f), F(i - 2 * d, h);
        for (int p = 0; p < 3; ++p) dF[p] = kD02 * a[p] + kD12 * b[p] + kD22 * e[p] + kD32 * f[p] + kD2 * h[p];
    }
}

// Lists of one stage, from one pass over the points: faces f in [-1, N1] (face f+1/2 is needed when a
// finest-level point of the stage's mask lies on either side) into fl_list[0, nf), finest-level
// points into pl[0, nfin), coarse points (valid level, derivative stencil inside the ghosted line)
// into pl[cap - ncrs, cap).  copy_qc: also the stage-start copy QC of every mask1 point (the only
// points whose QC stages 2 and 3 read; mask0 is inside mask1).  Each thread owns a contiguous
// chunk of positions and keeps its hits as bit sets (chunks of up to 64 positions; longer chunks
// evaluate again), one block scan of the three packed counts places them; order is preserved.
struct StageLists {
    int nf, nfin, ncrs;
};
// Stage class of a point whose mask bit is set: 1 finest level, 2 coarse point with its derivative
// stencil inside the ghosted line, 0 neither (main_1d_euler.cpp:111-133).
__device__ __forceinline__ int stage_class(const Ctx& c, int l, int i)
{
    const int lev = c.L(l, i);
    if (lev == c.maxl) return 1;
    if (lev < 0 || lev > c.maxl) return 0;
    const int d = c.D(lev);
    return (i - 2 * d < -kGhost || i + 2 * d > c.N1 + kGhost) ? 0 : 2;
}
__device__ __forceinline__ bool fin_byte(const Ctx& c, int b, int l, int x)
{
    return x >= kGhost && x <= c.N1 + kGhost && ((c.m[x] >> b) & 1u) && c.L(l, x - kGhost) == c.maxl;
}

// Word-level form of stage_lists for instances whose per-thread share is at most 16 mask words:
// each thread reads its run of 32-bit mask words (four points each), looks up levels for the
// stage's points only, and keeps its hits as bit sets over the run.
__device__ StageLists stage_lists_words(const Ctx& c, int b, int l, bool copy_qc, uint32_t* fl_list, uint32_t* pl,
                                        int cap, unsigned long long* red, int w0, int w1)
{
    const int xlo = kGhost - 1, xhi = c.N1 + kGhost;  // faces x in [xlo, xhi], points x in [kGhost, xhi]
    const unsigned* mw = reinterpret_cast<const unsigned*>(c.m);
    const int base = 4 * w0;
    unsigned long long mf = 0, mp = 0, mc = 0;
    bool fprev = w0 < w1 && fin_byte(c, b, l, base - 1);
    for (int wi = w0; wi < w1; ++wi) {
        const unsigned v = mw[wi];
#pragma unroll
        for (int L = 0; L < 4; ++L) {
            const int x = 4 * wi + L;
            int k = 0;
            if (x >= kGhost && x <= xhi) {
                if ((v >> (8 * L + b)) & 1u) k = stage_class(c, l, x - kGhost);
                if (copy_qc && ((v >> (8 * L + 1)) & 1u))
                    for (int q = 0; q < 3; ++q) c.QC(q, x - kGhost) = c.Q(q, x - kGhost);
            }
            const unsigned long long bit = 1ull << (x - base);
            if (k == 1) mp |= bit;
            else if (k == 2) mc |= bit;
            // face x - 1 needs a finest-level point at x - 1 or x
            if (x - 1 >= base && x - 1 >= xlo && (fprev || k == 1)) mf |= bit >> 1;
            fprev = k == 1;
        }
    }
    if (w0 < w1) {
        const int xl = 4 * w1 - 1;
        if (xl >= xlo && xl <= xhi && (fprev || fin_byte(c, b, l, xl + 1))) mf |= 1ull << (xl - base);
    }
    constexpr unsigned long long M21 = (1ull << 21) - 1;
    unsigned long long tot;
    const unsigned long long off = block_exclusive_scan64(
        (unsigned long long)__popcll(mf) | ((unsigned long long)__popcll(mp) << 21) | ((unsigned long long)__popcll(mc) << 42),
        red, &tot);
    StageLists o{(int)(tot & M21), (int)((tot >> 21) & M21), (int)((tot >> 42) & M21)};
    unsigned of = (unsigned)(off & M21), op = (unsigned)((off >> 21) & M21), oc = (unsigned)((off >> 42) & M21);
    uint32_t* crs = pl + cap - o.ncrs;
    for (; mf; mf &= mf - 1) fl_list[of++] = (uint32_t)(base + __ffsll(mf) - 1 - kGhost);
    for (; mp; mp &= mp - 1) pl[op++] = (uint32_t)(base + __ffsll(mp) - 1 - kGhost);
    for (; mc; mc &= mc - 1) crs[oc++] = (uint32_t)(base + __ffsll(mc) - 1 - kGhost);
    __syncthreads();
    return o;
}

__device__ StageLists stage_lists(const Ctx& c, int b, int l, bool copy_qc, uint32_t* fl_list, uint32_t* pl, int cap,
                                  unsigned long long* red)
{
    {
        const int wlo = (kGhost - 1) >> 2, whi = (c.N1 + kGhost) >> 2;
        const int pw = (whi - wlo + (int)blockDim.x) / (int)blockDim.x;
        if (pw <= 16) {
            const int w0 = wlo + (int)threadIdx.x * pw;
            return stage_lists_words(c, b, l, copy_qc, fl_list, pl, cap, red, w0, min(w0 + pw, whi + 1));
        }
    }
    const int lo = -1, hi = c.N1;
    const int n = hi - lo + 1;
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int a0 = lo + (int)threadIdx.x * per;
    const int a1 = min(a0 + per, hi + 1);
    // 0: not a stage point, 1: finest-level point, 2: coarse point (main_1d_euler.cpp:111-133)
    auto cls = [&](int i) -> int {
        if (i < 0 || i > c.N1 || !c.bit(i, b)) return 0;
        const int lev = c.L(l, i);
        if (lev == c.maxl) return 1;
        if (lev < 0 || lev > c.maxl) return 0;
        const int d = c.D(lev);
        return (i - 2 * d < -kGhost || i + 2 * d > c.N1 + kGhost) ? 0 : 2;
    };
    const bool bits = per <= 64;
    unsigned long long mf = 0, mp = 0, mc = 0;
    unsigned cf = 0, cp = 0, cc = 0;
    int k_i = a0 < a1 ? cls(a0) : 0;
    for (int i = a0; i < a1; ++i) {
        const int k_n = cls(i + 1);
        const unsigned long long bit = 1ull << ((i - a0) & 63);
        if (k_i == 1 || k_n == 1) {
            ++cf;
            if (bits) mf |= bit;
        }
        if (k_i == 1) {
            ++cp;
            if (bits) mp |= bit;
        } else if (k_i == 2) {
            ++cc;
            if (bits) mc |= bit;
        }
        if (copy_qc && i >= 0 && c.bit(i, 1))
            for (int k = 0; k < 3; ++k) c.QC(k, i) = c.Q(k, i);
        k_i = k_n;
    }
    constexpr unsigned long long M21 = (1ull << 21) - 1;
    unsigned long long tot;
    const unsigned long long off =
        block_exclusive_scan64((unsigned long long)cf | ((unsigned long long)cp << 21) | ((unsigned long long)cc << 42),
                               red, &tot);
    StageLists o{(int)(tot & M21), (int)((tot >> 21) & M21), (int)((tot >> 42) & M21)};
    unsigned of = (unsigned)(off & M21), op = (unsigned)((off >> 21) & M21), oc = (unsigned)((off >> 42) & M21);
    uint32_t* crs = pl + cap - o.ncrs;
    if (bits) {
        for (; mf; mf &= mf - 1) fl_list[of++] = (uint32_t)(a0 + __ffsll(mf) - 1);
        for (; mp; mp &= mp - 1) pl[op++] = (uint32_t)(a0 + __ffsll(mp) - 1);
        for (; mc; mc &= mc - 1) crs[oc++] = (uint32_t)(a0 + __ffsll(mc) - 1);
    } else {
        k_i = a0 < a1 ? cls(a0) : 0;
        for (int i = a0; i < a1; ++i) {
            const int k_n = cls(i + 1);
            if (k_i == 1 || k_n == 1) fl_list[of++] = (uint32_t)i;
            if (k_i == 1) pl[op++] = (uint32_t)i;
            else if (k_i == 2) crs[oc++] = (uint32_t)i;
            k_i = k_n;
        }
    }
    __syncthreads();
    return o;
}

// One stage over mask bit b / level set l (main_1d_euler.cpp:97-245).  Faces are computed once
// (face i+1/2 is shared by points i and i+1; the reference evaluates it for both, identically).
// The faces and the coarse derivatives read the stage input Q and run in one phase (the coarse
// derivatives are parked in qt); the point updates follow in a second phase, so Q is never read
// after a point of this stage has been written and no copy of the stage input is needed.
template <int SCHEME>
__device__ void stage1(const Ctx& c, int b, int l, double alpha, double dt, int kind, uint32_t* list,
                       unsigned long long* red)
{
    const int cap = c.w + 32;
    uint32_t* pl = list + cap;
    const StageLists L = stage_lists(c, b, l, kind == 1, list, pl, cap, red);
    const uint32_t* crs = pl + cap - L.ncrs;
    for (int e = threadIdx.x; e < L.nf + L.ncrs; e += blockDim.x) {
        if (e < L.nf) {
            const int f = (int)list[e];
            double s[6][3];
#pragma unroll
            for (int p = 0; p < 6; ++p)
#pragma unroll
                for (int k = 0; k < 3; ++k) s[p][k] = c.Q(k, f - 2 + p);
            double o[3];
            face_flux_1d<SCHEME>(s, alpha, c.I.gamma, o);
#pragma unroll
            for (int k = 0; k < 3; ++k) c.fl[k * c.w + f + kGhost] = o[k];
        } else {
            const int i = (int)crs[e - L.nf];
            double dF[3];
            coarse_dF1(c, i, c.D(c.L(l, i)), dF);
#pragma unroll
            for (int k = 0; k < 3; ++k) c.QT(k, i) = dF[k];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < L.nfin + L.ncrs; e += blockDim.x) {
        int i, d;
        double dF[3];
        if (e < L.nfin) {
            i = (int)pl[e];
            d = 1;
            for (int k = 0; k < 3; ++k) dF[k] = c.fl[k * c.w + i + kGhost] - c.fl[k * c.w + i - 1 + kGhost];
        } else {
            i = (int)crs[e - L.nfin];
            d = c.D(c.L(l, i));
            for (int k = 0; k < 3; ++k) dF[k] = c.QT(k, i);
        }
        const double sc = dt / (c.I.dx * d);
        for (int k = 0; k < 3; ++k) {
            double& Qv = c.Q(k, i);
            if (kind == 1) Qv = Qv - sc * dF[k];
            else if (kind == 2) Qv = 0.75 * c.QC(k, i) + 0.25 * (Qv - sc * dF[k]);
            else Qv = (c.QC(k, i) + 2.0 * (Qv - sc * dF[k])) / 3.0;
        }
    }
    __syncthreads();
}

// One RK3 step of one instance on the context's buffers (q, stage copies, faces, mask bytes, levels).
template <int SCHEME>
__device__ void step_ctx(Inst1& I, const Ctx& c, uint32_t* list, double* dred, unsigned* ured)
{
    unsigned long long* red64 = reinterpret_cast<unsigned long long*>(ured);
    prepare1(c);

    // CFL (main_1d_euler.cpp:67-81)
    double mv = 0;
    bool nf = false;  // a NaN or infinite wave speed in the CFL or LF scans
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        if (!c.bit(i, 3)) continue;
        const double q0 = c.Q(0, i), q1 = c.Q(1, i), q2 = c.Q(2, i);
        const double s = sound1(q0, q1, q2, I.gamma);
        const double u = q1 / q0;
        nf |= !isfinite(absd(u) + s);
        mv = maxd(mv, absd(u) + s);
    }
    mv = block_max(mv, dred);
    double dt = I.cfl * I.dx / mv;
    if (I.dt_fixed > 0) dt = I.dt_fixed;
    int do_print = 0;
    if (I.t + dt > I.t_end) {
        dt = I.t_end - I.t;
        do_print = 1;
    }
    unsigned cnt[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        const unsigned v = c.M(i);
        for (int k = 0; k < 4; ++k) cnt[k] += (v >> k) & 1u;
    }
    block_sum4(cnt, ured);

    bc1(c);
    const double a1 = lf_speed1(c, 3, 3, dred, nf);
    // the stage-start copy QC is taken inside stage 1's list pass
    stage1<SCHEME>(c, 2, 2, a1, dt, 1, list, red64);
    bc1(c);
    const double a2 = lf_speed1(c, 2, 2, dred, nf);
    stage1<SCHEME>(c, 1, 1, a2, dt, 2, list, red64);
    bc1(c);
    const double a3 = lf_speed1(c, 1, 1, dred, nf);
    stage1<SCHEME>(c, 0, 0, a3, dt, 3, list, red64);
    const bool any_nf = __syncthreads_or(nf);
    // RemoveResidue (AWCM_MANAGER_1D.h:135-157)
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
        if (!c.bit(i, 0)) c.Q(0, i) = c.Q(1, i) = c.Q(2, i) = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        I.dt = dt;
        I.mv = mv;
        I.alpha[0] = a1;
        I.alpha[1] = a2;
        I.alpha[2] = a3;
        I.do_print = do_print;
        for (int k = 0; k < 4; ++k) I.mask_cnt[k] = cnt[k];
        I.upd += cnt[0];
        I.steps += 1;
        I.t += dt;
        I.done = I.t >= I.t_end;
        if (any_nf) {
            // not a valid gas state: the instance stops and reports it (the reference carries
            // the NaN on)
            I.err = kErrNonFinite;
            I.done = 1;
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------- scalar AWCM (advection)
// The scalar path of Wavelet/main_1d_advect.cpp:48-224: one field q advected with unit speed at a
// fixed dt, on the same masks and levels.  q lives in plane 0 of the instance's field; the stage
// outputs q_2, q_1, q_0 in the three planes of the stage-start copy.

// AWCM_1D::Prepare (Wavelet/AWCM_1D.h:45-72): WAVELET_1D::ForwardWaveletTransform
// (WAVELET_1D.h:90-144, the arithmetic of the Euler form on its density), banding, then the
// mask/level chain without PrepareEuler's adjacent zones on mask1..mask3, the inverse transform
// (WAVELET_1D.h:146-196) and no interpolation of new points.
__device__ void prepare1_scalar(const Ctx& c)
{
    fwt1(c);
    band_copy1(c);
    aaz1(c, 0, kBitCopy);
    cr1(c, 0);
    for (int k = 1; k <= 3; ++k) {
        cl1(c, k - 1, k - 1, k, kBitCopy);  // level_{k-1} of mask_{k-1}; mask_k = the copy bit = mask_{k-1}
        apd1(c, k, k - 1);                  // AddPointForDifferentiation(mask_k, level_{k-1})
        cr1(c, k);
    }
    cl1(c, 3, 3, -1);
    iwt1(c, 3);
}

// Coarse-level derivative of the field with the driver's branch selection (main_1d_advect.cpp:
// 62-83): AWCM_1D::Differentiate and the 4-point DifferentiateAtLeftBoundary (Wavelet/AWCM_1D.h:
// 127-135), the right edge by the left form on the mirrored stencil as the driver calls it.  The
// driver's two 6-argument DifferentiateAtLeftBoundary calls (i == 2 dx_, i + 2 dx_ == i_end) name
// no scalar overload of AWCM_1D (the driver does not compile as shipped); they take the 5-point
// form of the vector counterpart, DifferentiateEulerAtLeftBoundary (AWCM_1D.h:174-185), with the
// identity flux of unit-speed advection.
__device__ double coarse_d1_scalar(const Ctx& c, const double* in, int i, int d)
{
    auto Q = [&](int ii) { return in[ii + kGhost]; };
    const int iend = c.N1;
    if (i - 2 * d > 0 && i + 2 * d < iend) return kD1 * (Q(i + d) - Q(i - d)) + kD2 * (Q(i + 2 * d) - Q(i - 2 * d));
    if (i - 2 * d < 0) return kD1 * (Q(i + d) - Q(i - d)) + kD2 * (Q(i + 2 * d) - Q(i - d));
    if (i == 2 * d)
        return kD02 * Q(i - 2 * d) + kD12 * Q(i - d) + kD22 * Q(i) + kD32 * Q(i + d) + kD2 * Q(i + 2 * d);
    if (i + 2 * d > iend) return kD1 * (Q(i - d) - Q(i + d)) + kD2 * (Q(i - 2 * d) - Q(i + d));
    return kD02 * Q(i + 2 * d) + kD12 * Q(i + d) + kD22 * Q(i) + kD32 * Q(i - d) + kD2 * Q(i - 2 * d);
}

// One scalar stage (main_1d_advect.cpp:50-99, :100-155, :164-212): out = in (the whole line),
// then at the points of mask b (level set l) out(i) -= dt (F_r - F_l) / (dx dx_) on the finest
// level, F_r = WENO5::ReconstructRight(in(i-2..i+2)) (WENO.h:101-104; the face i+1/2 is shared by
// points i and i+1, which the reference evaluates twice identically), or out(i) -= dt / (dx dx_)
// dF below it; then the driver's ghost copies of the end points.
__device__ void stage1_scalar(const Ctx& c, const double* in, double* out, int b, int l, double dt, uint32_t* list,
                              unsigned* ured)
{
    for (int t = threadIdx.x; t < c.w; t += blockDim.x) out[t] = in[t];
    __syncthreads();
    auto fin = [&](int i) { return i >= 0 && i <= c.N1 && c.bit(i, b) && c.L(l, i) == c.maxl; };
    const int nf = block_compact(-1, c.N1, [&](int f) { return fin(f) || fin(f + 1); }, list, ured);
    for (int e = threadIdx.x; e < nf; e += blockDim.x) {
        const int f = (int)list[e];
        const double* v = in + f + kGhost;
        c.fl[f + kGhost] = recon_left<kWeno5>(v[2], v[1], v[0], v[-1], v[-2]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        if (!c.bit(i, b)) continue;
        const int lev = c.L(l, i);
        if (lev < 0 || lev > c.maxl) continue;
        const int d = c.D(lev);
        if (lev != c.maxl && (i - 2 * d < -kGhost || i + 2 * d > c.N1 + kGhost)) continue;
        double& o = out[i + kGhost];
        if (lev == c.maxl) o = o - dt * (c.fl[i + kGhost] - c.fl[i - 1 + kGhost]) / (c.I.dx * d);
        else o = o - dt / (c.I.dx * d) * coarse_d1_scalar(c, in, i, d);
    }
    __syncthreads();
    if (threadIdx.x < kGhost) {
        const int g = threadIdx.x + 1;
        out[kGhost - g] = out[kGhost];
        out[kGhost + c.N1 + g] = out[kGhost + c.N1];
    }
    __syncthreads();
}

// One pass of the scalar driver loop: Prepare, the three stages at dt = dt_fixed (the driver's
// 0.5 dx is the caller's choice), the combinations q_1 = 3/4 q + 1/4 q_1 on mask1 (after q_1's
// ghost copies) and q = 1/3 q + 2/3 q_0 on mask0, and PostProcess (RemoveResidue on mask0).  The
// ghosts of q itself are never rewritten, as in the driver.
__device__ void step_ctx_scalar(Inst1& I, const Ctx& c, uint32_t* list, unsigned* ured)
{
    prepare1_scalar(c);
    const double dt = I.dt_fixed;
    unsigned cnt[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x) {
        const unsigned v = c.M(i);
        for (int k = 0; k < 4; ++k) cnt[k] += (v >> k) & 1u;
    }
    block_sum4(cnt, ured);
    double* q = c.q;
    double* q2 = c.qc;
    double* q1 = c.qc + c.w;
    double* q0 = c.qc + 2 * c.w;
    stage1_scalar(c, q, q2, 2, 2, dt, list, ured);
    stage1_scalar(c, q2, q1, 1, 1, dt, list, ured);
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
        if (c.bit(i, 1)) q1[i + kGhost] = 0.75 * q[i + kGhost] + 0.25 * q1[i + kGhost];
    __syncthreads();
    stage1_scalar(c, q1, q0, 0, 0, dt, list, ured);
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
        if (c.bit(i, 0)) q[i + kGhost] = kC1_3 * q[i + kGhost] + kD1 * q0[i + kGhost];
    __syncthreads();
    for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
        if (!c.bit(i, 0)) q[i + kGhost] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        I.dt = dt;
        I.mv = 0;
        I.alpha[0] = I.alpha[1] = I.alpha[2] = 0;
        I.do_print = 0;
        for (int k = 0; k < 4; ++k) I.mask_cnt[k] = cnt[k];
        I.upd += cnt[0];
        I.steps += 1;
        I.t += dt;
        I.done = I.t >= I.t_end;
    }
    __syncthreads();
}

// Byte offset of the level planes behind the mask bytes of an instance's state block.
__host__ __device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// The stage worklists of an instance of w ghosted points: faces, then finest and coarse points.
__host__ __device__ __forceinline__ size_t list_bytes(int w) { return sizeof(uint32_t) * 2 * (size_t)(w + 32); }

// What a step keeps in the CTA's shared memory (the rest stays in the instance's global buffers):
// kStageAll: mask bytes, the four level planes, the three conserved planes and the worklists;
// kStagePlanes: mask bytes and the three conserved planes (levels and worklists global, for an
// instance too large for kStageAll: a Jmax-13 tube needs 205 KB this way against 303 KB);
// kStageDensity: mask bytes, levels, the density plane and the worklists (the scalar path stages
// no plane); kStageNone: nothing.
enum StageLayout : int { kStageNone = 0, kStageDensity = 1, kStagePlanes = 2, kStageAll = 3 };
__host__ __device__ __forceinline__ size_t stage_bytes(int layout, int w)
{
    const size_t m = align16((size_t)w), l = align16((size_t)4 * w), d = sizeof(double) * (size_t)w;
    switch (layout) {
        case kStageAll: return m + l + 3 * d + list_bytes(w);
        case kStagePlanes: return m + 3 * d;
        case kStageDensity: return m + l + d + list_bytes(w);
        default: return 0;
    }
}
// The fullest layout that fits `avail` bytes; pool_lists: the instance has worklist space in the
// pool (the batch; the allocation-free step has none).
__host__ __device__ __forceinline__ int pick_layout(int w, size_t avail, bool scalar, bool pool_lists)
{
    if (!scalar && stage_bytes(kStageAll, w) <= avail) return kStageAll;
    if (!scalar && pool_lists && stage_bytes(kStagePlanes, w) <= avail) return kStagePlanes;
    if (stage_bytes(kStageDensity, w) <= avail) return kStageDensity;
    return kStageNone;
}
// Shared memory of the allocation-free step (kStageDensity).
__host__ __device__ __forceinline__ size_t step_smem_bytes(int w) { return stage_bytes(kStageDensity, w); }

// Copy of n bytes by all threads of the block; 16-byte words where both ends allow it.
__device__ __forceinline__ void block_copy_bytes(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, int n)
{
    int head = 0;
    if ((((uintptr_t)dst | (uintptr_t)src) & 15) == 0) {
        const int nv = n >> 4;
        for (int t = threadIdx.x; t < nv; t += blockDim.x)
            reinterpret_cast<int4*>(dst)[t] = reinterpret_cast<const int4*>(src)[t];
        head = nv << 4;
    }
    for (int t = head + threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}

__device__ __forceinline__ void block_copy_doubles(double* __restrict__ dst, const double* __restrict__ src, int n)
{
    int head = 0;
    if ((((uintptr_t)dst | (uintptr_t)src) & 15) == 0) {
        const int nv = n >> 1;
        for (int t = threadIdx.x; t < nv; t += blockDim.x)
            reinterpret_cast<double2*>(dst)[t] = reinterpret_cast<const double2*>(src)[t];
        head = nv << 1;
    }
    for (int t = head + threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
}

// One RK3 step of an instance, with the part of its state that `layout` names staged in the CTA's
// shared memory (smem: stage_bytes(layout, w) bytes): the ~100 level-sequential mask and transform
// phases of PrepareEuler and the stages then run on shared memory, with one global round trip in
// and one out per step.  q: the three conserved planes (global); qc, qt, fl: stage-start copy,
// coarse derivatives, face fluxes; mg: w mask bytes, lg: four planes of w levels (global); glist:
// worklist space in the pool (layouts that keep the worklists global).  One call site for every
// layout keeps the step kernel's code to one copy of each scheme.
// Up to nsteps RK3 steps of instance I (the caller has checked that it is not done), staged into
// shared memory once around them; the steps stop when the instance is done.
__device__ void step_inst(Inst1& I, double* q, double* qc, double* qt, double* fl, uint8_t* mg, int8_t* lg,
                          const Weights& W, uint8_t* smem, int layout, uint32_t* glist, double* dred, unsigned* ured,
                          int nsteps = 1)
{
    const int w = I.nx + 2 * kGhost;
    // the scalar path reads and writes its field planes directly; only its masks are staged
    const bool scalar = I.scheme == kScalarAdvection;
    const bool st_lv = layout == kStageDensity || layout == kStageAll;
    const bool st_q0 = layout == kStageDensity && !scalar;
    const bool st_q = layout == kStagePlanes || layout == kStageAll;
    uint8_t* ms = mg;
    int8_t* ls = lg;
    double* qp = q;   // plane p at qp + p w
    double* q0 = q;   // plane 0
    uint32_t* list = glist;
    if (layout != kStageNone) {
        uint8_t* p = smem;
        ms = p;
        p += align16((size_t)w);
        if (st_lv) {
            ls = reinterpret_cast<int8_t*>(p);
            p += align16((size_t)4 * w);
        }
        if (layout == kStageDensity) {
            if (st_q0) q0 = reinterpret_cast<double*>(p);
            p += sizeof(double) * (size_t)w;
        }
        if (st_q) {
            qp = q0 = reinterpret_cast<double*>(p);
            p += 3 * sizeof(double) * (size_t)w;
        }
        if (st_lv) list = reinterpret_cast<uint32_t*>(p);
        block_copy_bytes(ms, mg, w);
        if (st_lv) block_copy_bytes(reinterpret_cast<uint8_t*>(ls), reinterpret_cast<const uint8_t*>(lg), 4 * w);
        if (st_q0) block_copy_doubles(q0, q, w);
        if (st_q) block_copy_doubles(qp, q, 3 * w);
        __syncthreads();
    }
    const Ctx c{I, qp, qc, qt, fl, ms, ls, W, w, I.nx, I.nx - 1, I.maxl, q0};
    for (int s = 0; s < nsteps; ++s) {
        // the step's end (thread 0, then a block barrier) sets done at t_end or on an error
        if (s > 0 && *reinterpret_cast<volatile int*>(&I.done)) break;
        if (scalar) step_ctx_scalar(I, c, list, ured);
        else if (I.scheme == kWeno5) step_ctx<kWeno5>(I, c, list, dred, ured);
        else step_ctx<kWenoZ>(I, c, list, dred, ured);
    }
    if (layout != kStageNone) {
        block_copy_bytes(mg, ms, w);
        if (st_lv) block_copy_bytes(reinterpret_cast<uint8_t*>(lg), reinterpret_cast<const uint8_t*>(ls), 4 * w);
        if (st_q0) block_copy_doubles(q, q0, w);
        if (st_q) block_copy_doubles(q, qp, 3 * w);
        __syncthreads();
    }
}

// Global views of instance I in the pool.
__device__ __forceinline__ Ctx make_ctx(Inst1& I, const Pool& P)
{
    const int w = I.nx + 2 * kGhost;
    double* base = P.q + I.q_off;
    uint8_t* mb = P.m + I.m_off;
    return Ctx{I, base, base + 3 * w, base + 6 * w, base + 9 * w, mb, (int8_t*)(mb + align16((size_t)w)), P.W,
               w, I.nx, I.nx - 1, I.maxl, base};
}

// nsteps RK3 steps of every queued instance (fewer for an instance that reaches t_end).  CTAs pull
// queue slots until the queue is exhausted, and run each instance's steps back to back before
// taking the next: nsteps = 1 is one step of the whole batch (the per-step graph); a large
// nsteps runs every instance to its end in one launch, each CTA independently of the others.
// smem_bytes: the launch's dynamic shared memory; an instance whose staged step does not fit in
// it runs on its global buffers (its worklists in the pool too).
// Up to 768 threads per CTA (80 registers a thread, some of the face computation spilled to L1):
// a CTA advances one instance through ~150 block-barrier phases per step, latency-bound, so more
// warps per instance pay for the spills (Jmax-13 tail step 0.312 -> 0.255 ms against 384 threads
// and 162 registers; the step-synchronous batched whole run 3.48e7 -> 4.20e7 updates/s).
__global__ void __launch_bounds__(768, 1) k_step1d(Inst1* insts, int n, const int* __restrict__ order, unsigned* queue, Pool P,
                         unsigned smem_bytes, int nsteps)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ double dred[32];
    __shared__ __align__(8) unsigned ured[128];
    __shared__ int cur;
    for (;;) {
        if (threadIdx.x == 0) cur = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int k = cur;
        __syncthreads();
        if (k >= n) break;
        Inst1& I = insts[order[k]];
        if (I.t >= I.t_end || I.err) {
            if (threadIdx.x == 0) I.done = 1;
        } else {
            const int w = I.nx + 2 * kGhost;
            double* base = P.q + I.q_off;
            uint8_t* mb = P.m + I.m_off;
            step_inst(I, base, base + 3 * w, base + 6 * w, base + 9 * w, mb, (int8_t*)(mb + align16((size_t)w)), P.W,
                      smem, pick_layout(w, smem_bytes, I.scheme == kScalarAdvection, true),
                      reinterpret_cast<uint32_t*>(base + 12 * (size_t)w), dred, ured, nsteps);
        }
        __syncthreads();
    }
}

// Single passes for the C-ABI manager surface (one CTA per instance).
__global__ void k_pass1d(Inst1* insts, int inst, Pool P, int op, int bit, int level_id)
{
    Inst1& I = insts[inst];
    const Ctx c = make_ctx(I, P);
    switch (op) {
        case 0:  // AddAdjacentZone
            copy_bit1(c, bit, kBitCopy, true);
            aaz1(c, bit, kBitCopy);
            break;
        case 1: cr1(c, bit); break;
        case 2:
            copy_bit1(c, bit, kBitCopy, true);
            apd1(c, bit, level_id);
            break;
        case 3: cl1(c, level_id, bit, -1); break;
        case 4:
            for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
                if (!c.bit(i, bit)) c.Q(0, i) = c.Q(1, i) = c.Q(2, i) = 0;
            break;
        case 5:
            for (int i = threadIdx.x; i <= c.N1; i += blockDim.x)
                if (!(3 <= i && i <= c.N1 - 3)) c.set(i, bit);
            break;
        case 10:
            if (I.scheme == kScalarAdvection) prepare1_scalar(c);
            else prepare1(c);
            break;
        case 11: fwt1(c); break;
        case 12: iwt1(c, bit); break;
        case 13: interp1(c, bit, level_id); break;  // InterpolateEuler(from = bit, to = level_id as a bit)
        case 14: bc1(c); break;
        default: break;
    }
}

// EULER_EQUATION_1D batch entry points (EULER_EQUATION.h:16-26, 42-47): n states of 3 doubles.
__global__ void k_euler1d_flux(const double* __restrict__ q, double* __restrict__ f, int n, double gamma)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double s[3] = {q[3 * t], q[3 * t + 1], q[3 * t + 2]};
    double o[3];
    flux1(s, gamma, o);
    for (int k = 0; k < 3; ++k) f[3 * t + k] = o[k];
}

__global__ void k_euler1d_sr(const double* __restrict__ q, double* __restrict__ out, int n, double gamma)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double q0 = q[3 * t], q1 = q[3 * t + 1], q2 = q[3 * t + 2];
    const double u = q1 / q0;
    out[t] = absd(u) + sound1(q0, q1, q2, gamma);
}

}  // namespace

// ====================================================================================== Batch1D
struct Batch1D {
    std::vector<Inst1> host;
    Inst1* d_inst = nullptr;
    int* d_order = nullptr;
    unsigned* d_queue = nullptr;
    double* d_q = nullptr;
    uint8_t* d_m = nullptr;
    size_t q_doubles = 0, m_bytes = 0;
    int max_w = 0;
    Pool P{};
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int device = 0;
    int block = 256;
    int grid = 0;
    int n = 0;

    ~Batch1D()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (d_inst) cudaFree(d_inst);
        if (d_order) cudaFree(d_order);
        if (d_queue) cudaFree(d_queue);
        if (d_q) cudaFree(d_q);
        if (d_m) cudaFree(d_m);
        if (stream) cudaStreamDestroy(stream);
    }

    int create(int count, const int* num_levels, const int* nx_coarse, const double* x_min, const double* x_max,
               double gamma, int scheme)
    {
        if (count <= 0 || !num_levels || !nx_coarse || !x_min || !x_max) return kErrArg;
        if (scheme != kWenoZ && scheme != kWeno5 && scheme != kScalarAdvection) return kErrArg;
        AWCM_CUDA_TRY(cudaGetDevice(&device));
        n = count;
        host.assign(n, Inst1{});
        size_t qo = 0, mo = 0;
        for (int k = 0; k < n; ++k) {
            if (num_levels[k] < 2 || num_levels[k] > 20 || nx_coarse[k] < 5) return kErrArg;
            Inst1& I = host[k];
            I.nx = (nx_coarse[k] - 1) * (1 << (num_levels[k] - 1)) + 1;
            I.maxl = num_levels[k] - 1;
            I.scheme = scheme;
            I.x_min = x_min[k];
            I.dx = (x_max[k] - x_min[k]) / (I.nx - 1);
            I.gamma = gamma;
            I.t = 0;
            I.t_end = 0;
            const int w = I.nx + 2 * kGhost;
            max_w = std::max(max_w, w);
            I.q_off = (long long)qo;
            I.m_off = (long long)mo;
            qo += (size_t)12 * w + (size_t)(w + 32);
            qo = (qo + 31) & ~(size_t)31;
            mo += align16((size_t)w) + (size_t)4 * w;  // mask bytes, then the levels 16-byte aligned
            mo = (mo + 255) & ~(size_t)255;
        }
        q_doubles = qo;
        m_bytes = mo;
        AWCM_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        AWCM_CUDA_TRY(cudaMalloc(&d_inst, sizeof(Inst1) * n));
        AWCM_CUDA_TRY(cudaMalloc(&d_order, sizeof(int) * n));
        AWCM_CUDA_TRY(cudaMalloc(&d_queue, sizeof(unsigned)));
        AWCM_CUDA_TRY(cudaMalloc(&d_q, sizeof(double) * q_doubles));
        AWCM_CUDA_TRY(cudaMalloc(&d_m, m_bytes));
        AWCM_CUDA_TRY(cudaMemsetAsync(d_q, 0, sizeof(double) * q_doubles, stream));
        // AWCM_1D's constructor: mask0 true everywhere incl. ghosts, mask_temp and mask1..mask3
        // false everywhere, levels 0 (Wavelet/AWCM_1D.h:23-34).  Ghost bytes also carry the work
        // bits, which are never read there.
        std::vector<uint8_t> hm(m_bytes, 0);
        for (int k = 0; k < n; ++k) {
            const int w = host[k].nx + 2 * kGhost;
            uint8_t* mk = hm.data() + host[k].m_off;
            for (int a = 0; a < w; ++a) {
                const bool ghost = a < kGhost || a >= w - kGhost;
                mk[a] = ghost ? 0xe1 : 0x01;
            }
        }
        AWCM_CUDA_TRY(cudaMemcpy(d_m, hm.data(), m_bytes, cudaMemcpyHostToDevice));
        // Largest instances first in the queue.
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return host[a].nx > host[b].nx; });
        AWCM_CUDA_TRY(cudaMemcpy(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
        AWCM_CUDA_TRY(upload_inst());
        P.q = d_q;
        P.m = d_m;
        P.W = make_weights();
        // Default width: measured alone, lines of up to ~1000 points step 2-3 % faster with 512
        // threads, longer ones fastest with 768 (the batch's critical path is its longest line).
        int nx_max = 0;
        for (int k = 0; k < n; ++k) nx_max = std::max(nx_max, host[k].nx);
        return set_launch(nx_max <= 1100 ? 512 : 768, 0);
    }

    cudaError_t upload_inst()
    {
        return cudaMemcpy(d_inst, host.data(), sizeof(Inst1) * n, cudaMemcpyHostToDevice);
    }
    cudaError_t download_inst()
    {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(host.data(), d_inst, sizeof(Inst1) * n, cudaMemcpyDeviceToHost);
    }

    // Dynamic shared memory of the step kernel: the fullest staging layout of the largest instance
    // that fits the per-CTA limit, else the limit (the largest instances then run on their global
    // buffers, the smaller ones still staged).  Smaller instances take the fullest layout that fits.
    size_t smem_cap = 227 * 1024;
    size_t smem_bytes() const
    {
        const size_t e = stage_bytes(pick_layout(max_w, smem_cap, false, true), max_w);
        const size_t sc = stage_bytes(pick_layout(max_w, smem_cap, true, true), max_w);
        const size_t b = std::max(e, sc);
        return b ? b : smem_cap;
    }

    // Launch shape: threads per CTA and CTAs per SM (0 = as many as fit).
    int set_launch(int threads, int ctas_per_sm)
    {
        if (threads < 64 || threads > 1024 || threads % 32) return kErrArg;
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, k_step1d) == cudaSuccess && threads > fa.maxThreadsPerBlock) {
            set_last_error("launch shape exceeds the step kernel's register budget", __FILE__, __LINE__);
            return kErrArg;
        }
        block = threads;
        int sms = 148, occ = 1, optin = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) == cudaSuccess && optin > 0)
            smem_cap = (size_t)optin - 1024;  // leave room for the kernel's static shared arrays
        cudaFuncSetAttribute(k_step1d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_step1d, block, smem_bytes());
        if (occ < 1) occ = 1;
        if (ctas_per_sm > 0) occ = std::min(occ, ctas_per_sm);
        grid = std::min(n, sms * occ);
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        return kOk;
    }

    void enq_step(int nsteps = 1)
    {
        cudaMemsetAsync(d_queue, 0, sizeof(unsigned), stream);
        k_step1d<<<grid, block, smem_bytes(), stream>>>(d_inst, n, d_order, d_queue, P, (unsigned)smem_bytes(), nsteps);
    }

    int build_graph()
    {
        if (graph) return kOk;
        cudaGraph_t gr;
        AWCM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        enq_step();
        cudaError_t e = cudaStreamEndCapture(stream, &gr);
        if (e != cudaSuccess) {
            set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
            return kErrCuda;
        }
        e = cudaGraphInstantiate(&graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
            return kErrCuda;
        }
        return kOk;
    }

    int set_run(const double* tol, const double* cfl, const double* t, const double* t_end, double dt_fixed)
    {
        AWCM_CUDA_TRY(download_inst());
        for (int k = 0; k < n; ++k) {
            Inst1& I = host[k];
            I.tol = tol[k];
            I.cfl = cfl[k];
            I.t = t[k];
            I.t_end = t_end[k];
            I.dt_fixed = dt_fixed;
            I.err = 0;
            I.done = I.t >= I.t_end;
        }
        AWCM_CUDA_TRY(upload_inst());
        return kOk;
    }

    int steps(int n_steps)
    {
        int rc = build_graph();
        if (rc) return rc;
        for (int s = 0; s < n_steps; ++s) AWCM_CUDA_TRY(cudaGraphLaunch(graph, stream));
        AWCM_CUDA_TRY(cudaGetLastError());
        return kOk;
    }

    // Every unfinished instance to its end time, at most max_steps steps each, in one launch.
    int run(int max_steps)
    {
        enq_step(max_steps);
        AWCM_CUDA_TRY(cudaGetLastError());
        return kOk;
    }

    // Attaches the enum-driven BOUNDARY_MANAGER_1D to instance k: bc = Nx+6 BOUNDARY_CONDITION
    // values in the FIELD_UNIFORM_1D layout (only the six ghost cells are read).
    int set_bc_field(int k, const int* bc)
    {
        const int nx = host[k].nx;
        const int idx[6] = {2, 1, 0, nx + 3, nx + 4, nx + 5};  // ghosts -1, -2, -3, N1+1, N1+2, N1+3
        for (int q = 0; q < 6; ++q)
            if (bc[idx[q]] < -4 || bc[idx[q]] > 0) {
                set_last_error("BOUNDARY_CONDITION values are -4 (SOLID_WALL) .. 0 (FLUID)", __FILE__, __LINE__);
                return kErrArg;
            }
        AWCM_CUDA_TRY(download_inst());
        for (int q = 0; q < 6; ++q) host[k].bcg[q] = (int8_t)bc[idx[q]];
        host[k].bc_generic = 1;
        AWCM_CUDA_TRY(upload_inst());
        return kOk;
    }

    // Threshold of instance k for a single-pass call (the step takes it from set_run).
    int set_tol(int k, double tol)
    {
        AWCM_CUDA_TRY(download_inst());
        host[k].tol = tol;
        AWCM_CUDA_TRY(upload_inst());
        return kOk;
    }

    int pass(int inst, int op, int bit, int level_id)
    {
        if (inst < 0 || inst >= n) return kErrArg;
        k_pass1d<<<1, 256, 0, stream>>>(d_inst, inst, P, op, bit, level_id);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int w_of(int k) const { return host[k].nx + 2 * kGhost; }

    int set_q(int k, const double* aos)
    {
        const int w = w_of(k);
        std::vector<double> soa(3 * (size_t)w);
        for (int a = 0; a < w; ++a)
            for (int p = 0; p < 3; ++p) soa[p * w + a] = aos[a * 3 + p];
        AWCM_CUDA_TRY(cudaMemcpy(d_q + host[k].q_off, soa.data(), sizeof(double) * 3 * w, cudaMemcpyHostToDevice));
        return kOk;
    }

    int get_q(int k, double* aos)
    {
        const int w = w_of(k);
        std::vector<double> soa(3 * (size_t)w);
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        AWCM_CUDA_TRY(cudaMemcpy(soa.data(), d_q + host[k].q_off, sizeof(double) * 3 * w, cudaMemcpyDeviceToHost));
        for (int a = 0; a < w; ++a)
            for (int p = 0; p < 3; ++p) aos[a * 3 + p] = soa[p * w + a];
        return kOk;
    }

    int get_masks(int k, uint8_t* planes)
    {
        const int w = w_of(k);
        std::vector<uint8_t> mb(w);
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        AWCM_CUDA_TRY(cudaMemcpy(mb.data(), d_m + host[k].m_off, w, cudaMemcpyDeviceToHost));
        const int bits[5] = {kBitTemp, 0, 1, 2, 3};
        for (int r = 0; r < 5; ++r)
            for (int a = 0; a < w; ++a) planes[r * w + a] = (mb[a] >> bits[r]) & 1u;
        return kOk;
    }

    int set_masks(int k, const uint8_t* planes)
    {
        const int w = w_of(k);
        std::vector<uint8_t> mb(w);
        const int bits[5] = {kBitTemp, 0, 1, 2, 3};
        for (int a = 0; a < w; ++a) {
            const bool ghost = a < kGhost || a >= w - kGhost;
            unsigned v = ghost ? 0xe0u : 0u;
            for (int r = 0; r < 5; ++r) v |= (unsigned)(planes[r * w + a] != 0) << bits[r];
            mb[a] = (uint8_t)v;
        }
        AWCM_CUDA_TRY(cudaMemcpy(d_m + host[k].m_off, mb.data(), w, cudaMemcpyHostToDevice));
        return kOk;
    }

    int get_levels(int k, int* lv)
    {
        const int w = w_of(k), nx = host[k].nx;
        std::vector<int8_t> l(4 * (size_t)w);
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        AWCM_CUDA_TRY(cudaMemcpy(l.data(), d_m + host[k].m_off + align16((size_t)w), 4 * (size_t)w,
                                 cudaMemcpyDeviceToHost));
        for (int r = 0; r < 4; ++r)
            for (int i = 0; i < nx; ++i) lv[r * nx + i] = l[r * w + i + kGhost];
        return kOk;
    }

    int set_levels(int k, const int* lv)
    {
        const int w = w_of(k), nx = host[k].nx;
        std::vector<int8_t> l(4 * (size_t)w, 0);
        for (int r = 0; r < 4; ++r)
            for (int i = 0; i < nx; ++i) l[r * w + i + kGhost] = (int8_t)lv[r * nx + i];
        AWCM_CUDA_TRY(cudaMemcpy(d_m + host[k].m_off + align16((size_t)w), l.data(), 4 * (size_t)w,
                                 cudaMemcpyHostToDevice));
        return kOk;
    }

    // Sod-type states on the cell-centred grid x_min + i dx (SHOCKTUBE::Initialize,
    // Problems/1D/PROBLEM_SHOCKTUBE.h:14-54, with the interface and states as arguments).
    int init_riemann(int k, double x_interface, const double* left, const double* right)
    {
        const Inst1& I = host[k];
        const int w = w_of(k);
        std::vector<double> aos(3 * (size_t)w);
        for (int i = -kGhost; i < I.nx + kGhost; ++i) {
            const double x = I.x_min + I.dx * i;
            const double* s = x <= x_interface ? left : right;
            const double rho = s[0], u = s[1], p = s[2];
            double* o = &aos[3 * (size_t)(i + kGhost)];
            o[0] = rho;
            o[1] = rho * u;
            o[2] = p / (I.gamma - 1) + 0.5 * rho * (u * u);
        }
        return set_q(k, aos.data());
    }
};

// =========================================================================== allocation-free step
// One RK3 step of a single 1D instance whose conserved field and mask/level state live in device
// buffers the caller owns, with every other buffer the step needs -- the stage-start and stage-input
// copies of the field, the face fluxes and the instance descriptor -- placed in the file-scope
// array below instead of memory allocated per instance.  It is sized for instances of up to
// kNoAllocMaxNx points (Jmax 13 with 17 coarse points): 9 x 8199 doubles plus a 256-byte
// descriptor, about 577 KiB, which every GPU that loads this library holds until the process exits.
constexpr int kNoAllocMaxNx = 8193;
constexpr int kNoAllocMaxW = kNoAllocMaxNx + 2 * kGhost;
constexpr int kNoAllocHeader = 32;  // doubles reserved for the descriptor (Inst1 fits in 256 bytes)
constexpr size_t kNoAllocDoubles = kNoAllocHeader + (size_t)9 * kNoAllocMaxW;
static_assert(sizeof(Inst1) <= kNoAllocHeader * sizeof(double), "descriptor does not fit the reserved header");

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {

// scratch: the device address of g_noalloc_scratch (resolved on the host once per device).
__global__ void k_step1d_noalloc(Inst1 param, double* q, uint8_t* state, double* scratch, double* out, Weights W)
{
    extern __shared__ __align__(16) uint8_t smem[];  // step_smem_bytes(w)
    __shared__ double dred[32];
    __shared__ __align__(8) unsigned ured[128];
    Inst1& I = *reinterpret_cast<Inst1*>(scratch);
    if (threadIdx.x == 0) I = param;  // the descriptor is rewritten by every call
    __syncthreads();
    const int w = param.nx + 2 * kGhost;
    double* qc = scratch + kNoAllocHeader;
    double* qt = qc + 3 * w;
    double* fl = qt + 3 * w;
    if (I.t < I.t_end) {
        step_inst(I, q, qc, qt, fl, state, (int8_t*)(state + w), W, smem, kStageDensity, nullptr, dred, ured);
    } else if (threadIdx.x == 0) {
        I.done = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = I.t;
        out[1] = I.dt;
        out[2] = I.do_print;
        out[3] = I.done;
        out[4] = I.steps;
        for (int k = 0; k < 4; ++k) out[5 + k] = I.mask_cnt[k];
        out[9] = I.mv;
        out[10] = I.alpha[0];
        out[11] = I.alpha[1];
        out[12] = I.alpha[2];
        out[13] = (double)I.upd;
        out[14] = I.err;
        out[15] = 0;
    }
}

// Device address of the scratch array, resolved once per device (host code must not use the
// symbol itself: on the host it is only a stand-in for the device copy).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

int noalloc_scratch(int dev, double** ptr)
{
    if (dev < 0 || dev >= kMaxDevices) return kErrArg;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
            return kErrCuda;
        }
        g_noalloc_addr[dev] = p;
    }
    *ptr = static_cast<double*>(g_noalloc_addr[dev]);
    return kOk;
}

}  // namespace

}  // namespace awcm

// ======================================================================================== C-ABI
using awcm::Batch1D;

struct awcm1d_batch_s {
    Batch1D b;
};

extern "C" {

int awcm1d_batch_create(int count, const int* num_levels, const int* nx_coarse, const double* x_min,
                        const double* x_max, double gamma, int scheme, awcm1d_batch_t* out)
{
    if (!out) return awcm::kErrArg;
    *out = nullptr;
    awcm1d_batch_s* h = new (std::nothrow) awcm1d_batch_s();
    if (!h) return awcm::kErrOom;
    const int rc = h->b.create(count, num_levels, nx_coarse, x_min, x_max, gamma, scheme);
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return awcm::kOk;
}

int awcm1d_batch_destroy(awcm1d_batch_t h)
{
    delete h;
    return awcm::kOk;
}

#define AWCM_B(h, k)                                                   \
    if (!(h) || (k) < 0 || (k) >= (h)->b.n) return awcm::kErrArg;     \
    cudaSetDevice((h)->b.device)

int awcm1d_batch_count(awcm1d_batch_t h, int* n)
{
    if (!h || !n) return awcm::kErrArg;
    *n = h->b.n;
    return awcm::kOk;
}
int awcm1d_batch_nx(awcm1d_batch_t h, int k, int* nx)
{
    AWCM_B(h, k);
    if (!nx) return awcm::kErrArg;
    *nx = h->b.host[k].nx;
    return awcm::kOk;
}
int awcm1d_batch_set_q(awcm1d_batch_t h, int k, const double* q)
{
    AWCM_B(h, k);
    return q ? h->b.set_q(k, q) : awcm::kErrArg;
}
int awcm1d_batch_get_q(awcm1d_batch_t h, int k, double* q)
{
    AWCM_B(h, k);
    return q ? h->b.get_q(k, q) : awcm::kErrArg;
}
int awcm1d_batch_get_masks(awcm1d_batch_t h, int k, uint8_t* m)
{
    AWCM_B(h, k);
    return m ? h->b.get_masks(k, m) : awcm::kErrArg;
}
int awcm1d_batch_set_masks(awcm1d_batch_t h, int k, const uint8_t* m)
{
    AWCM_B(h, k);
    return m ? h->b.set_masks(k, m) : awcm::kErrArg;
}
int awcm1d_batch_get_levels(awcm1d_batch_t h, int k, int* lv)
{
    AWCM_B(h, k);
    return lv ? h->b.get_levels(k, lv) : awcm::kErrArg;
}
int awcm1d_batch_set_levels(awcm1d_batch_t h, int k, const int* lv)
{
    AWCM_B(h, k);
    return lv ? h->b.set_levels(k, lv) : awcm::kErrArg;
}
int awcm1d_batch_init_riemann(awcm1d_batch_t h, int k, double x_interface, const double* left3,
                              const double* right3)
{
    AWCM_B(h, k);
    if (!left3 || !right3) return awcm::kErrArg;
    return h->b.init_riemann(k, x_interface, left3, right3);
}
int awcm1d_batch_set_run(awcm1d_batch_t h, const double* tol, const double* cfl, const double* t,
                         const double* t_end, double dt_fixed)
{
    if (!h || !tol || !cfl || !t || !t_end) return awcm::kErrArg;
    cudaSetDevice(h->b.device);
    return h->b.set_run(tol, cfl, t, t_end, dt_fixed);
}
int awcm1d_batch_steps(awcm1d_batch_t h, int n_steps)
{
    if (!h || n_steps < 0) return awcm::kErrArg;
    cudaSetDevice(h->b.device);
    return h->b.steps(n_steps);
}
int awcm1d_batch_run(awcm1d_batch_t h, int max_steps)
{
    if (!h || max_steps < 1) return awcm::kErrArg;
    cudaSetDevice(h->b.device);
    return h->b.run(max_steps);
}
int awcm1d_batch_sync(awcm1d_batch_t h)
{
    if (!h) return awcm::kErrArg;
    AWCM_CUDA_TRY(cudaStreamSynchronize(h->b.stream));
    return awcm::kOk;
}
// out[16]: t, dt, do_print, done, steps, |mask0..3|, max speed, alpha1..3, sum|mask0|, err, 0
int awcm1d_batch_status(awcm1d_batch_t h, int k, double* out)
{
    AWCM_B(h, k);
    if (!out) return awcm::kErrArg;
    AWCM_CUDA_TRY(h->b.download_inst());
    const auto& I = h->b.host[k];
    out[0] = I.t;
    out[1] = I.dt;
    out[2] = I.do_print;
    out[3] = I.done;
    out[4] = I.steps;
    for (int q = 0; q < 4; ++q) out[5 + q] = I.mask_cnt[q];
    out[9] = I.mv;
    out[10] = I.alpha[0];
    out[11] = I.alpha[1];
    out[12] = I.alpha[2];
    out[13] = (double)I.upd;
    out[14] = I.err;
    out[15] = 0;
    if (I.err == awcm::kErrNonFinite) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "instance %d: non-finite state: a CFL or Lax-Friedrichs wave speed was NaN or infinite in "
                      "the step ending at t = %.17g (NaN/Inf values, negative pressure or density)",
                      k, I.t);
        awcm::set_last_error(msg, __FILE__, __LINE__);
        return I.err;
    }
    return awcm::kOk;
}
int awcm1d_batch_totals(awcm1d_batch_t h, double* out)
{
    if (!h || !out) return awcm::kErrArg;
    cudaSetDevice(h->b.device);
    AWCM_CUDA_TRY(h->b.download_inst());
    double upd = 0, steps = 0, done = 0;
    for (const auto& I : h->b.host) {
        upd += (double)I.upd;
        steps += I.steps;
        done += I.done;
    }
    out[0] = upd;
    out[1] = steps;
    out[2] = done;
    return awcm::kOk;
}
int awcm1d_batch_pass(awcm1d_batch_t h, int k, int op, int mask_id, int level_id)
{
    AWCM_B(h, k);
    const int bit = mask_id >= 0 && mask_id <= 3 ? mask_id : awcm::kBitTemp;
    if (level_id < 0 || level_id > 3) return awcm::kErrArg;
    return h->b.pass(k, op, bit, level_id);
}
static int bit_of_mask(int mask_id) { return mask_id >= 0 && mask_id <= 3 ? mask_id : awcm::kBitTemp; }
static bool mask_id_ok(int mask_id) { return mask_id >= 0 && mask_id <= 4; }

int awcm1d_batch_prepare(awcm1d_batch_t h, int k, double tol)
{
    AWCM_B(h, k);
    const int rc = h->b.set_tol(k, tol);
    return rc ? rc : h->b.pass(k, 10, 0, 0);
}
int awcm1d_batch_fwt(awcm1d_batch_t h, int k, double tol)
{
    AWCM_B(h, k);
    const int rc = h->b.set_tol(k, tol);
    return rc ? rc : h->b.pass(k, 11, 0, 0);
}
int awcm1d_batch_iwt(awcm1d_batch_t h, int k, int mask_id)
{
    AWCM_B(h, k);
    if (!mask_id_ok(mask_id)) return awcm::kErrArg;
    return h->b.pass(k, 12, bit_of_mask(mask_id), 0);
}
int awcm1d_batch_interpolate(awcm1d_batch_t h, int k, int from_id, int to_id)
{
    AWCM_B(h, k);
    if (!mask_id_ok(from_id) || !mask_id_ok(to_id)) return awcm::kErrArg;
    return h->b.pass(k, 13, bit_of_mask(from_id), bit_of_mask(to_id));
}
int awcm1d_batch_manager(awcm1d_batch_t h, int k, int op, int mask_id, int level_id)
{
    AWCM_B(h, k);
    if (op < AWCM_OP_ADD_ADJACENT_ZONE || op > AWCM_OP_BANDING || !mask_id_ok(mask_id) || level_id < 0 ||
        level_id > 3)
        return awcm::kErrArg;
    return h->b.pass(k, op, bit_of_mask(mask_id), level_id);
}
int awcm1d_batch_set_bc_field(awcm1d_batch_t h, int k, const int* bc)
{
    AWCM_B(h, k);
    if (!bc) return awcm::kErrArg;
    return h->b.set_bc_field(k, bc);
}
int awcm1d_batch_apply_bc(awcm1d_batch_t h, int k)
{
    AWCM_B(h, k);
    return h->b.pass(k, 14, 0, 0);
}

int euler1d_flux(const double* q_dev, double* f_dev, int n, double gamma, void* stream)
{
    if (n < 0 || (n && (!q_dev || !f_dev))) return awcm::kErrArg;
    if (!n) return awcm::kOk;
    awcm::k_euler1d_flux<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(q_dev, f_dev, n, gamma);
    AWCM_CUDA_TRY(cudaGetLastError());
    return awcm::kOk;
}
int euler1d_spectral_radius(const double* q_dev, double* s_dev, int n, double gamma, void* stream)
{
    if (n < 0 || (n && (!q_dev || !s_dev))) return awcm::kErrArg;
    if (!n) return awcm::kOk;
    awcm::k_euler1d_sr<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(q_dev, s_dev, n, gamma);
    AWCM_CUDA_TRY(cudaGetLastError());
    return awcm::kOk;
}

int awcm1d_batch_set_launch(awcm1d_batch_t h, int threads, int ctas_per_sm)
{
    if (!h) return awcm::kErrArg;
    cudaSetDevice(h->b.device);
    return h->b.set_launch(threads, ctas_per_sm);
}
int awcm1d_batch_stream(awcm1d_batch_t h, void** stream)
{
    if (!h || !stream) return awcm::kErrArg;
    *stream = (void*)h->b.stream;
    return awcm::kOk;
}

int awcm1d_step_noalloc(int num_levels, int nx_coarse, double x_min, double x_max, double gamma, int scheme,
                        double tol, double cfl, double t, double t_end, double* q_dev, uint8_t* state_dev,
                        double* out_dev, void* stream)
{
    using namespace awcm;
    if (num_levels < 2 || num_levels > 20 || nx_coarse < 5 || !q_dev || !state_dev || !out_dev) {
        set_last_error("awcm1d_step_noalloc: bad argument", __FILE__, __LINE__);
        return kErrArg;
    }
    if (scheme != kWenoZ && scheme != kWeno5) {
        set_last_error("awcm1d_step_noalloc: scheme must be 0 (WENO-Z) or 1 (WENO5)", __FILE__, __LINE__);
        return kErrArg;
    }
    const long long nx = (long long)(nx_coarse - 1) * (1LL << (num_levels - 1)) + 1;
    if (nx > kNoAllocMaxNx) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "awcm1d_step_noalloc: Nx = %lld exceeds the static scratch limit of %d points", nx,
                      kNoAllocMaxNx);
        set_last_error(msg, __FILE__, __LINE__);
        return kErrArg;
    }
    int dev = 0;
    AWCM_CUDA_TRY(cudaGetDevice(&dev));
    double* scratch = nullptr;
    const int rc = noalloc_scratch(dev, &scratch);
    if (rc) return rc;
    Inst1 I{};
    I.nx = (int)nx;
    I.maxl = num_levels - 1;
    I.scheme = scheme;
    I.x_min = x_min;
    I.dx = (x_max - x_min) / (double)(nx - 1);
    I.gamma = gamma;
    I.tol = tol;
    I.cfl = cfl;
    I.t = t;
    I.t_end = t_end;
    const int w = (int)nx + 2 * kGhost;
    const size_t smem = step_smem_bytes(w);  // 172 KB at the 8193-point limit
    AWCM_CUDA_TRY(cudaFuncSetAttribute(k_step1d_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_step1d_noalloc<<<1, 256, smem, (cudaStream_t)stream>>>(I, q_dev, state_dev, scratch, out_dev, make_weights());
    AWCM_CUDA_TRY(cudaGetLastError());
    return kOk;
}

}  // extern "C"

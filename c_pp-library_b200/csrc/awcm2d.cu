// 2D AWCM compressible-Euler path on one B200 (sm_100a), FP64.
//
// Layout in HBM (one instance):
//   conserved field Q and the RK stage fields Q2, Q1: four structure-of-arrays planes each
//     (rho, rho u, rho v, E), row pitch `pitch` doubles, ghost ring of 3, point (i,j) at
//     (j+3)*pitch + (i+3);
//   face fluxes Fx (face i+1/2 stored at point i) and Fy (face j+1/2 at point j), four planes each;
//   one mask byte per point: bits 0..3 = mask0..mask3, 4 = previous mask0, 5/6 = work bits;
//   one int8 level plane per level set (level0..level3);
//   per stage compacted worklists (row-ordered uint32 point indices) of finest-level points,
//   coarse points, needed x faces and needed y faces, built by block ballot/prefix compaction.
//
// One RK3 step = PrepareEuler (level-by-level transform and mask kernels) + CFL/LF reductions +
// three stages (boundary fill, face-flux kernels, point-update kernels) + residue removal.  All
// scalars the step needs (t, dt, CFL speed, per-level dt/dx) stay on the device, so a step is a
// fixed launch sequence captured once into a CUDA graph and replayed.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "awcm_b200.h"
#include "awcm_common.cuh"
#include "awcm2d_types.cuh"

namespace awcm {
namespace {

// Device-resident step scalars.
struct StepState {
    double t, t_end, dt, cfl, dt_fixed, tol, mv;
    double sc[kMaxLevels];        // dt / (dx * 2^(maxl-lev)) per level
    int do_print, done, steps, full_zero;
    unsigned cnt[4 * kStages];     // per stage: finest points, coarse points, x faces, y faces
    unsigned mask_cnt[4];          // |mask0..mask3| over the grid points
    unsigned long long upd;        // sum over steps of |mask0|
    unsigned long long stage_pts;  // sum over steps of |mask2|+|mask1|+|mask0|
    unsigned bar[2];               // grid barrier of the persistent prepare: arrivals, generation
    int bar_err;                   // set when a barrier wait ran out (or another CTA failed)
    int error;                     // first error of the run (reported by the host API)
    int nonfinite;                 // set when a CFL or LF wave speed of the step is NaN or infinite
    unsigned spin_limit;           // polls before a grid-barrier wait gives up (0 = kSpinLimit)
};

__device__ __forceinline__ int ctz_or(int v, int big) { return v == 0 ? big : __ffs(v) - 1; }

// Sub-band geometry of level lev: which 0 = d1 (half x, coarse y), 1 = d2 (coarse x, half y),
// 2 = d3 (half, half), 3 = c (coarse interior); extents of MRA_GRID_INT_2D::Initialize
// (Wavelet/MRA_GRID_UNIFORM_2D.h:101-131).
struct Band {
    int i0, j0, cx, cy, D;
};
__host__ __device__ __forceinline__ Band band_of(const Grid2& g, int lev, int which)
{
    const int D = g.D(lev), h = D >> 1;
    const int MX = (g.nx - 1) / D, MY = (g.ny - 1) / D;
    Band b;
    b.D = D;
    switch (which) {
        case 0: b.i0 = h, b.cx = MX, b.j0 = D, b.cy = MY - 1; break;
        case 1: b.i0 = D, b.cx = MX - 1, b.j0 = h, b.cy = MY; break;
        case 2: b.i0 = h, b.cx = MX, b.j0 = h, b.cy = MY; break;
        default: b.i0 = D, b.cx = MX - 1, b.j0 = D, b.cy = MY - 1; break;
    }
    if (b.cx < 0) b.cx = 0;
    if (b.cy < 0) b.cy = 0;
    return b;
}

// Global thread index (all grids here are far below 2^32 threads; 32-bit index arithmetic avoids
// the emulated 64-bit division).
__device__ __forceinline__ unsigned gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// Programmatic dependent launch: the kernels of a step are launched with programmatic stream
// serialisation, so the next kernel's CTAs are scheduled once every CTA of the current one is
// running and then wait in griddepcontrol.wait (a hardware wait on the predecessor grid's
// completion and memory flush, not a software spin) before their first access.  This hides the
// launch latency between the ~100 short dependent kernels of a step.  Launched without the
// attribute, both instructions are no-ops.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Push of a mask bit at (i,j).  Under the reference's mask invariants every push lands on the
// ghosted grid; pushes that would leave it (possible only for inconsistent user-set masks/levels,
// where the reference itself writes out of bounds) are dropped.
// The push is an atomicOr on the 32-bit word holding the byte: fire-and-forget (no dependent
// round trip per push, unlike a byte read-modify-write) and race-free next to other pushes.
__device__ __forceinline__ void push_bit(const Grid2& g, uint8_t* m, int i, int j, int bit)
{
    if (i < -kGhost || i >= g.nx + kGhost || j < -kGhost || j >= g.ny + kGhost) return;
    const size_t a = g.at(i, j);
    atomicOr(reinterpret_cast<unsigned*>(m + (a & ~(size_t)3)), 1u << (8 * (unsigned)(a & 3) + bit));
}

// Point t of the concatenation of the listed sub-bands of level lev (see band_of).
template <int NB>
__device__ __forceinline__ bool union_point(const Grid2& g, int lev, const int (&which)[NB], unsigned t, int& i,
                                            int& j, int& w)
{
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const Band b = band_of(g, lev, which[k]);
        const unsigned n = (unsigned)b.cx * (unsigned)b.cy;
        if (t < n) {
            i = b.i0 + (int)(t % (unsigned)b.cx) * b.D;
            j = b.j0 + (int)(t / (unsigned)b.cx) * b.D;
            w = which[k];
            return true;
        }
        t -= n;
    }
    return false;
}

// Mask words: the plane-wide passes and the fine-level row scans work one 32-bit word of the mask
// plane (four consecutive points of one row: the pitch is a multiple of 32) per virtual thread,
// test the word's bits of interest at once and skip empty words, which is most of them.
constexpr unsigned kLaneBits = 0x01010101u;  // bit 0 of each of the four bytes

// Pushes onto points that lie on the ghosted plane by construction (no bounds test).
__device__ __forceinline__ void push_bit_in(const Grid2& g, uint8_t* m, int i, int j, int bit)
{
    const size_t a = g.at(i, j);
    atomicOr(reinterpret_cast<unsigned*>(m + (a & ~(size_t)3)), 1u << (8 * (unsigned)(a & 3) + bit));
}
// `bit` onto the n points i0, i0 + s, .., i0 + (n-1) s of row j (s = 1 or 2, span at most 8 bytes,
// all on the ghosted plane): one atomicOr per 32-bit word they touch, its lane mask built by shifts.
__device__ __forceinline__ void push_run(const Grid2& g, uint8_t* m, int i0, int n, int s, int j, int bit)
{
    const size_t a0 = g.at(i0, j), a1 = a0 + (size_t)((n - 1) * s);
    unsigned* w = reinterpret_cast<unsigned*>(m + (a0 & ~(size_t)3));
    const unsigned lanes = (s == 1 ? kLaneBits : ((a0 & 1) ? 0x01000100u : 0x00010001u)) << bit;
    const unsigned head = lanes & (0xFFFFFFFFu << (8u * (unsigned)(a0 & 3)));         // bytes >= a0's
    const unsigned tail = lanes & (0xFFFFFFFFu >> (8u * (3u - (unsigned)(a1 & 3))));  // bytes <= a1's
    const int nw = (int)((a1 >> 2) - (a0 >> 2));
    if (nw == 0) {
        atomicOr(w, head & tail);
        return;
    }
    atomicOr(w, head);
    if (nw == 2) atomicOr(w + 1, lanes);
    atomicOr(w + nw, tail);
}

struct MaskWord {
    unsigned w;  // word index; bytes 4w .. 4w+3 of the plane
    int i0, j;   // grid coordinates of byte 0 (ghosts negative / beyond the grid)
};
__device__ __forceinline__ MaskWord mask_word(const Grid2& g, unsigned w)
{
    const unsigned a = 4u * w, row = a / (unsigned)g.pitch;
    return MaskWord{w, (int)(a - row * (unsigned)g.pitch) - kGhost, (int)row - kGhost};
}
__device__ __forceinline__ unsigned plane_words(const Grid2& g) { return (unsigned)g.pitch * (unsigned)g.rows / 4u; }
// Lanes (bit L = byte L) whose column i0 + L lies in [lo, hi].
__device__ __forceinline__ unsigned lanes_in(int i0, int lo, int hi)
{
    unsigned r = 0;
#pragma unroll
    for (int L = 0; L < 4; ++L) r |= (unsigned)(i0 + L >= lo && i0 + L <= hi) << L;
    return r;
}
// Lane set -> bit 0 of each selected byte.
__device__ __forceinline__ unsigned lane_bits(unsigned lanes)
{
    return (lanes & 1u) | ((lanes & 2u) << 7) | ((lanes & 4u) << 14) | ((lanes & 8u) << 21);
}
// Lanes that are grid points (0 <= i < nx, 0 <= j < ny).
__device__ __forceinline__ unsigned grid_lanes(const Grid2& g, const MaskWord& mw)
{
    return (mw.j >= 0 && mw.j < g.ny) ? lanes_in(mw.i0, 0, g.nx - 1) : 0u;
}

// ------------------------------------------------------------------------------- phase bodies
// Every PrepareEuler pass is a device function over a virtual thread range (t0, stride), so the
// same body runs as a standalone kernel (one thread per point) or inside the persistent prepare
// kernel (grid-stride over the phase's points between grid barriers).
struct Span {
    unsigned t0, stride;
};
__device__ __forceinline__ Span grid_span() { return Span{gtid(), gridDim.x * blockDim.x}; }

__device__ __forceinline__ unsigned band_n(const Grid2& g, int lev, int which)
{
    const Band b = band_of(g, lev, which);
    return (unsigned)b.cx * (unsigned)b.cy;
}

// Forward transform of one level (ForwardWaveletTransformationEuler, WAVELET_2D.h:478-624) in two
// phases.  The reference orders d3 -> d1 -> d2 -> c because d3 must see untransformed d1/d2
// values; phase A computes all three detail sub-bands at once with the d1/d2 results staged in
// the scratch plane `tb`, and phase B applies the c update (reading d1/d2 from `tb`) and moves the
// staged details into q.  Same operations on the same operands: identical results.
// idle: kBitTemp holds the mask0 of the start of the pass (PrepareEuler copies it there first);
// the d1/d2 points outside it are then left in q instead of going through the staging plane.
// Forward predict of one detail point of a level (w: 2 = d3 into q, 0/1 = d1/d2 into the staging
// plane tb); on: the point is in mask0 (its detail is computed and thresholded).
__device__ __forceinline__ void fwt_a_point(const Grid2& g, double* __restrict__ q, double* __restrict__ tb,
                                            uint8_t* __restrict__ m, int i, int j, size_t a, int D, int w, double tol,
                                            bool on)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    if (w == 2) {
        if (!on) return;
        int is, k1, js, k2;
        predict_stencil(i, D, NX, is, k1);
        predict_stencil(j, D, NY, js, k2);
        double v = q[a];
        for (int c = 0; c < 4; ++c) v -= q[g.at(is + c * D, j)] * g.w(c, k1);
        for (int c = 0; c < 4; ++c) v -= q[g.at(i, js + c * D)] * g.w(c, k2);
        for (int c2 = 0; c2 < 4; ++c2)
            for (int c1 = 0; c1 < 4; ++c1) v += q[g.at(is + c1 * D, js + c2 * D)] * g.w(c1, k1) * g.w(c2, k2);
        v *= 0.25;
        q[a] = v;
        if (absd(v) < tol) m[a] &= (uint8_t)~1u;
        return;
    }
    double v = q[a];
    if (on) {
        int s0, k;
        if (w == 0) {
            predict_stencil(i, D, NX, s0, k);
            for (int c = 0; c < 4; ++c) v -= q[g.at(s0 + c * D, j)] * g.w(c, k);
        } else {
            predict_stencil(j, D, NY, s0, k);
            for (int c = 0; c < 4; ++c) v -= q[g.at(i, s0 + c * D)] * g.w(c, k);
        }
        v *= 0.5;
        if (absd(v) < tol) m[a] &= (uint8_t)~1u;
    }
    tb[a] = v;
}

// idle: kBitTemp holds the mask0 of the start of the pass (PrepareEuler copies it there first);
// the d1/d2 points outside it are then left in q instead of going through the staging plane.
__device__ void ph_fwt_a(const Grid2& g, double* __restrict__ q, double* __restrict__ tb, uint8_t* __restrict__ m,
                         int lev, double tol, bool idle, Span sp)
{
    const int which[3] = {2, 0, 1};
    const unsigned n = band_n(g, lev, 0) + band_n(g, lev, 1) + band_n(g, lev, 2);
    const int D = g.D(lev);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        int i, j, w;
        union_point(g, lev, which, t, i, j, w);
        const size_t a = g.at(i, j);
        const bool on = m[a] & 1u;
        if (idle && !on) continue;  // d1/d2: q[a] stays, ph_fwt_b reads it from q; d3: nothing to do
        fwt_a_point(g, q, tb, m, i, j, a, D, w, tol, on);
    }
}

// Forward update of one c point of mask0 (the d1/d2 neighbours: the staged detail of a point of the
// pass's mask0, else q itself, which this pass does not write; without idle all come from tb).
__device__ __forceinline__ void fwt_b_point(const Grid2& g, double* __restrict__ q, const double* __restrict__ tb,
                                            const uint8_t* __restrict__ m, int i, int j, size_t a, int D, bool idle)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    int is, k1, js, k2;
    update_stencil(i, D, NX, is, k1);
    update_stencil(j, D, NY, js, k2);
    auto d12 = [&](size_t b) { return (!idle || ((m[b] >> kBitTemp) & 1u)) ? tb[b] : q[b]; };
    double v = q[a];
    for (int c = 0; c < 4; ++c) v += d12(g.at(is + c * D, j)) * g.w(c, k1);
    for (int c = 0; c < 4; ++c) v += d12(g.at(i, js + c * D)) * g.w(c, k2);
    for (int c2 = 0; c2 < 4; ++c2)
        for (int c1 = 0; c1 < 4; ++c1) v += q[g.at(is + c1 * D, js + c2 * D)] * g.w(c1, k1) * g.w(c2, k2);
    q[a] = v;
}

__device__ void ph_fwt_b(const Grid2& g, double* __restrict__ q, const double* __restrict__ tb,
                         const uint8_t* __restrict__ m, int lev, bool idle, Span sp)
{
    const int which[3] = {3, 0, 1};
    const unsigned n = band_n(g, lev, 3) + band_n(g, lev, 0) + band_n(g, lev, 1);
    const int D = g.D(lev);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        int i, j, w;
        union_point(g, lev, which, t, i, j, w);
        const size_t a = g.at(i, j);
        if (w != 3) {
            if (!idle || ((m[a] >> kBitTemp) & 1u)) q[a] = tb[a];
            continue;
        }
        if (!(m[a] & 1u)) continue;
        fwt_b_point(g, q, tb, m, i, j, a, D, idle);
    }
}

// Inverse transform, one phase of one level (InverseWaveletTransformationEuler, WAVELET_2D.h:626-782):
// PH 0 = c, PH 1 = d2 and d1, PH 2 = d3; points outside the mask get density 0.
// zero_all false: the density outside mask_temp (the step's starting mask0) is zero already (the
// previous step's residue removal), so only the points of mask_temp outside `bit` are zeroed.
// Inverse transform of one point of the mask (w: 3 = c update, 1 = d2, 0 = d1, 2 = d3 predict).
__device__ __forceinline__ void iwt_point(const Grid2& g, double* __restrict__ q, int i, int j, size_t a, int D, int w)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    if (w == 3) {
        int is, k1, js, k2;
        update_stencil(i, D, NX, is, k1);
        update_stencil(j, D, NY, js, k2);
        double v = q[a];
        for (int c = 0; c < 4; ++c) v -= q[g.at(is + c * D, j)] * g.w(c, k1);
        for (int c = 0; c < 4; ++c) v -= q[g.at(i, js + c * D)] * g.w(c, k2);
        for (int c2 = 0; c2 < 4; ++c2)
            for (int c1 = 0; c1 < 4; ++c1) v -= q[g.at(is + c1 * D, js + c2 * D)] * g.w(c1, k1) * g.w(c2, k2);
        q[a] = v;
    } else if (w == 1) {
        int s0, k;
        predict_stencil(j, D, NY, s0, k);
        double v = q[a];
        v *= 2.0;
        for (int c = 0; c < 4; ++c) v += q[g.at(i, s0 + c * D)] * g.w(c, k);
        q[a] = v;
    } else if (w == 0) {
        int s0, k;
        predict_stencil(i, D, NX, s0, k);
        double v = q[a];
        v *= 2.0;
        for (int c = 0; c < 4; ++c) v += q[g.at(s0 + c * D, j)] * g.w(c, k);
        q[a] = v;
    } else {
        int is, k1, js, k2;
        predict_stencil(i, D, NX, is, k1);
        predict_stencil(j, D, NY, js, k2);
        double v = q[a];
        v *= 4.0;
        for (int c = 0; c < 4; ++c) v += q[g.at(is + c * D, j)] * g.w(c, k1);
        for (int c = 0; c < 4; ++c) v += q[g.at(i, js + c * D)] * g.w(c, k2);
        for (int c2 = 0; c2 < 4; ++c2)
            for (int c1 = 0; c1 < 4; ++c1) v -= q[g.at(is + c1 * D, js + c2 * D)] * g.w(c1, k1) * g.w(c2, k2);
        q[a] = v;
    }
}

template <int PH>
__device__ void ph_iwt(const Grid2& g, double* __restrict__ q, const uint8_t* __restrict__ m, int lev, int bit,
                       bool zero_all, Span sp)
{
    const int D = g.D(lev);
    unsigned n;
    if (PH == 0) n = band_n(g, lev, 3);
    else if (PH == 1) n = band_n(g, lev, 0) + band_n(g, lev, 1);
    else n = band_n(g, lev, 2);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        int i, j, w;
        if (PH == 0) {
            const int wh[1] = {3};
            union_point(g, lev, wh, t, i, j, w);
        } else if (PH == 1) {
            const int wh[2] = {0, 1};
            union_point(g, lev, wh, t, i, j, w);
        } else {
            const int wh[1] = {2};
            union_point(g, lev, wh, t, i, j, w);
        }
        const size_t a = g.at(i, j);
        if (!((m[a] >> bit) & 1u)) {
            if (zero_all || ((m[a] >> kBitTemp) & 1u)) q[a] = 0;
            continue;
        }
        iwt_point(g, q, i, j, a, D, w);
    }
}

// The finest level (point spacing 1) of the step's transforms as a row scan: word t of the grid rows
// is tested for the two mask bits that can make one of its points need work before its row and
// column are decoded (most words have neither), and the set lanes are classified by parity:
// 2 = d3 (odd, odd), 0 = d1 (odd, even; not the top or bottom row), 1 = d2 (even, odd; not the left
// or right column), 3 = c (even, even; not on the boundary), -1 = none -- the extents of band_of.
__device__ __forceinline__ int fine_band(const Grid2& g, int i, int j)
{
    const bool io = i & 1, jo = j & 1;
    if (io && jo) return 2;
    if (io) return (j == 0 || j == g.ny - 1) ? -1 : 0;
    if (jo) return (i == 0 || i == g.nx - 1) ? -1 : 1;
    return (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1) ? -1 : 3;
}
// f(i, j, a, byte) for the grid points of the scanned words whose byte has bit b1 or b2.
template <class F>
__device__ __forceinline__ void fine_rows(const Grid2& g, const uint8_t* m, int b1, int b2, Span sp, F&& f)
{
    const unsigned wpr = (unsigned)g.pitch / 4u, row0 = (unsigned)kGhost * wpr;
    const unsigned n = (unsigned)g.ny * wpr;
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        const unsigned v = mp[row0 + t];
        unsigned hit = ((v >> b1) | (v >> b2)) & kLaneBits;
        if (!hit) continue;
        const unsigned r = t / wpr, wi = t - r * wpr;
        const int j = (int)r, i0 = 4 * (int)wi - kGhost;
        hit &= lane_bits(lanes_in(i0, 0, g.nx - 1));
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            f(i0 + L, j, 4u * (row0 + t) + (unsigned)L, (v >> (8 * L)) & 0xffu);
        }
    }
}
// Row-scan forms of the finest level (idle mode / sparse zeroing, see ph_fwt_a and ph_iwt).
__device__ void ph_fwt_a_fine(const Grid2& g, double* __restrict__ q, double* __restrict__ tb,
                              uint8_t* __restrict__ m, double tol, Span sp)
{
    fine_rows(g, m, 0, 0, sp, [&](int i, int j, size_t a, unsigned) {
        const int w = fine_band(g, i, j);
        if (w >= 0 && w != 3) fwt_a_point(g, q, tb, m, i, j, a, 2, w, tol, true);
    });
}
__device__ void ph_fwt_b_fine(const Grid2& g, double* __restrict__ q, const double* __restrict__ tb,
                              const uint8_t* __restrict__ m, Span sp)
{
    fine_rows(g, m, 0, kBitTemp, sp, [&](int i, int j, size_t a, unsigned byte) {
        const int w = fine_band(g, i, j);
        if (w == 3) {
            if (byte & 1u) fwt_b_point(g, q, tb, m, i, j, a, 2, true);
        } else if (w == 0 || w == 1) {
            if ((byte >> kBitTemp) & 1u) q[a] = tb[a];
        }
    });
}
template <int PH>
__device__ void ph_iwt_fine(const Grid2& g, double* __restrict__ q, const uint8_t* __restrict__ m, int bit, Span sp)
{
    fine_rows(g, m, bit, kBitTemp, sp, [&](int i, int j, size_t a, unsigned byte) {
        const int w = fine_band(g, i, j);
        if (PH == 0 ? w != 3 : PH == 1 ? (w != 0 && w != 1) : w != 2) return;
        if ((byte >> bit) & 1u) iwt_point(g, q, i, j, a, 2, w);
        else q[a] = 0;  // in mask_temp, not in the mask
    });
}

// CheckReconstruction of one level (AWCM_MANAGER_2D.h:63-158) in one phase.  The reference runs
// d3 -> d1 -> d2 so that d1/d2 points switched on by a d3 point also mark their stencils; those
// stencils ((is..is+3D, n) for a d1 point (i, n), (m, js..js+3D) for a d2 point (m, j)) lie inside
// the d3 point's own 4x4 block of marks, so all three sub-bands can run concurrently.
// The stencil points lie in [0, NX] x [0, NY] (predict_stencil clamps them), so the pushes need no
// bounds test; at spacing D = 2 the four points of a row span 7 bytes and go in 2-3 word ORs.
__device__ __forceinline__ void cr_push(const Grid2& g, uint8_t* m, int i, int j, int D, int w, int bit)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    int is, js, k;
    auto row4 = [&](int jr) {
        if (D == 2) {
            push_run(g, m, is, 4, 2, jr, bit);
        } else {
            for (int c = 0; c < 4; ++c) push_bit_in(g, m, is + c * D, jr, bit);
        }
    };
    if (w == 2) {
        predict_stencil(i, D, NX, is, k);
        predict_stencil(j, D, NY, js, k);
        row4(j);
        for (int c = 0; c < 4; ++c) push_bit_in(g, m, i, js + c * D, bit);
        for (int c2 = 0; c2 < 4; ++c2) row4(js + c2 * D);
    } else if (w == 0) {
        predict_stencil(i, D, NX, is, k);
        row4(j);
    } else {
        predict_stencil(j, D, NY, js, k);
        for (int c = 0; c < 4; ++c) push_bit_in(g, m, i, js + c * D, bit);
    }
}

__device__ void ph_cr(const Grid2& g, uint8_t* __restrict__ m, int lev, int bit, Span sp)
{
    const int which[3] = {2, 0, 1};
    const unsigned n = band_n(g, lev, 0) + band_n(g, lev, 1) + band_n(g, lev, 2);
    const int D = g.D(lev);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        int i, j, w;
        union_point(g, lev, which, t, i, j, w);
        if (!((m[g.at(i, j)] >> bit) & 1u)) continue;
        cr_push(g, m, i, j, D, w, bit);
    }
}

// Row-scan form of a fine level (point spacing h = D/2 <= kRowScanMaxH): the rows j = 0, h, 2h ..
// of the level are scanned one mask word (four columns) per virtual thread and the set lanes are
// classified by position: d1 = (odd, even) multiples of h off the top/bottom rows, d2 = (even,
// odd) off the left/right columns, d3 = (odd, odd) -- exactly the sub-band extents of band_of.
// Rows with parity `rows` (0 even, 1 odd, 2 both) in units of h.
constexpr int kRowScanMaxH = 2;
__device__ __forceinline__ unsigned rowscan_n(const Grid2& g, int lev, int rows)
{
    const int h = g.D(lev) >> 1;
    const unsigned nr = (unsigned)((g.ny - 1) / h) + 1u;  // rows 0, h, .., NY
    const unsigned wpr = (unsigned)g.pitch / 4u;
    return (rows == 2 ? nr : (rows == 0 ? (nr + 1u) / 2u : nr / 2u)) * wpr;
}
// Decodes virtual thread t of a row scan into the row j and the word (its first column i0, its
// mask bits v) ; returns the set of lanes that are points of this level (columns multiple of h in
// [0, NX]).
__device__ __forceinline__ unsigned rowscan_word(const Grid2& g, int lev, int rows, unsigned t, int& j, int& i0,
                                                 unsigned& widx)
{
    const int h = g.D(lev) >> 1;
    const unsigned wpr = (unsigned)g.pitch / 4u;
    const unsigned r = t / wpr, wi = t - r * wpr;
    const unsigned rr = rows == 2 ? r : 2u * r + (unsigned)rows;
    j = (int)rr * h;
    i0 = 4 * (int)wi - kGhost;
    widx = (unsigned)(j + kGhost) * wpr + wi;
    unsigned lanes = lanes_in(i0, 0, g.nx - 1);
    if (h == 2) lanes &= (i0 & 1) ? 0xAu : 0x5u;  // even columns
    return lanes;
}
// Sub-band of the level point (i, j) (h = spacing): 2 = d3, 0 = d1, 1 = d2, -1 = none.
__device__ __forceinline__ int rowscan_band(const Grid2& g, int i, int j, int h)
{
    const bool io = (i / h) & 1, jo = (j / h) & 1;
    if (io && jo) return 2;
    if (io) return (j == 0 || j == g.ny - 1) ? -1 : 0;
    if (jo) return (i == 0 || i == g.nx - 1) ? -1 : 1;
    return -1;
}

__device__ void ph_cr_rows(const Grid2& g, uint8_t* __restrict__ m, int lev, int bit, Span sp)
{
    const int D = g.D(lev), h = D >> 1;
    const unsigned n = rowscan_n(g, lev, 2);
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    const unsigned row0 = (unsigned)kGhost * ((unsigned)g.pitch / 4u);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        // on the finest detail level (h = 1) every row is scanned and word t is word t of the
        // plane's grid rows: test it before decoding its row and column
        if (h == 1 && !((mp[row0 + t] >> bit) & kLaneBits)) continue;
        int j, i0;
        unsigned wdx;
        const unsigned lanes = rowscan_word(g, lev, 2, t, j, i0, wdx);
        unsigned hit = (mp[wdx] >> bit) & lane_bits(lanes);
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const int i = i0 + L;
            const int w = rowscan_band(g, i, j, h);
            if (w >= 0) cr_push(g, m, i, j, D, w, bit);
        }
    }
}

// InterpolateEuler, one phase of one level (WAVELET_2D.h:784-907): PH 0 = d1 and d2, PH 1 = d3;
// components 1..3 at points of the work mask that were not active before (`from_bit`).  All
// components are computed before any is stored: a store of one component plane could alias the
// stencil loads of the next as far as the compiler knows, which would serialize their gathers.
__device__ __forceinline__ void interp_point(const Grid2& g, Field4 q, int i, int j, size_t a, int D, int w, int p0)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    double out[4] = {0, 0, 0, 0};
    if (w == 0) {
        int s0, k;
        predict_stencil(i, D, NX, s0, k);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (p < p0) continue;
            const double* qp = q.p[p];
            double v = 0.0;
            for (int c = 0; c < 4; ++c) v += qp[g.at(s0 + c * D, j)] * g.w(c, k);
            out[p] = v;
        }
    } else if (w == 1) {
        int s0, k;
        predict_stencil(j, D, NY, s0, k);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (p < p0) continue;
            const double* qp = q.p[p];
            double v = 0.0;
            for (int c = 0; c < 4; ++c) v += qp[g.at(i, s0 + c * D)] * g.w(c, k);
            out[p] = v;
        }
    } else {
        int is, k1, js, k2;
        predict_stencil(i, D, NX, is, k1);
        predict_stencil(j, D, NY, js, k2);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (p < p0) continue;
            const double* qp = q.p[p];
            double v = 0.0;
            for (int c = 0; c < 4; ++c) v += qp[g.at(is + c * D, j)] * g.w(c, k1);
            for (int c = 0; c < 4; ++c) v += qp[g.at(i, js + c * D)] * g.w(c, k2);
            for (int c2 = 0; c2 < 4; ++c2)
                for (int c1 = 0; c1 < 4; ++c1) v -= qp[g.at(is + c1 * D, js + c2 * D)] * g.w(c1, k1) * g.w(c2, k2);
            out[p] = v;
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
        if (p >= p0) q.p[p][a] = out[p];
}

template <int PH>
__device__ void ph_interp(const Grid2& g, Field4 q, const uint8_t* __restrict__ m, int lev, int from_bit, int p0,
                          Span sp)
{
    const int D = g.D(lev);
    const unsigned n = PH == 0 ? band_n(g, lev, 0) + band_n(g, lev, 1) : band_n(g, lev, 2);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        int i, j, w;
        if (PH == 0) {
            const int wh[2] = {0, 1};
            union_point(g, lev, wh, t, i, j, w);
        } else {
            const int wh[1] = {2};
            union_point(g, lev, wh, t, i, j, w);
        }
        const size_t a = g.at(i, j);
        const unsigned mb = m[a];
        if (!((mb >> kBitInterp) & 1u) || ((mb >> from_bit) & 1u)) continue;
        interp_point(g, q, i, j, a, D, w, p0);
    }
}

// Row-scan form of ph_interp for the fine levels: PH 0 scans every row of the level (d1 on the
// even ones, d2 on the odd ones), PH 1 only the odd rows (d3).
template <int PH>
__device__ void ph_interp_rows(const Grid2& g, Field4 q, const uint8_t* __restrict__ m, int lev, int from_bit, int p0,
                               Span sp)
{
    const int D = g.D(lev), h = D >> 1;
    const int rows = PH == 0 ? 2 : 1;
    const unsigned n = rowscan_n(g, lev, rows);
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    const unsigned row0 = (unsigned)kGhost * ((unsigned)g.pitch / 4u);
    for (unsigned t = sp.t0; t < n; t += sp.stride) {
        // every row of the finest detail level (h = 1, PH 0): word t of the grid rows
        if (PH == 0 && h == 1 && !((mp[row0 + t] >> kBitInterp) & kLaneBits)) continue;
        int j, i0;
        unsigned wdx;
        const unsigned lanes = rowscan_word(g, lev, rows, t, j, i0, wdx);
        const unsigned v = mp[wdx];
        unsigned hit = (v >> kBitInterp) & ~(v >> from_bit) & lane_bits(lanes);
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const int i = i0 + L;
            const int w = rowscan_band(g, i, j, h);
            if (w < 0 || (PH == 0) == (w == 2)) continue;
            interp_point(g, q, i, j, 4u * wdx + L, D, w, p0);
        }
    }
}

// ------------------------------------------------------------------------------- dense mask passes
// Bits 1..3 (mask1..mask3) of the four bytes of a mask word.
constexpr unsigned kMask123 = (kLaneBits << 1) | (kLaneBits << 2) | (kLaneBits << 3);
// Copies bit `from` into bit `to` on every byte; `clear` (lane-replicated bits) is cleared too.
__device__ void ph_copy_bit_all(uint8_t* m, size_t n, int from, int to, Span sp, unsigned clear = 0)
{
    unsigned* mw = reinterpret_cast<unsigned*>(m);
    const unsigned nw = (unsigned)(n / 4);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const unsigned v = mw[w];
        const unsigned nv = ((v & ~(kLaneBits << to)) | (((v >> from) & kLaneBits) << to)) & ~clear;
        if (nv != v) mw[w] = nv;
    }
}

// BandingMask (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:205-213) on `bit`, then copies the
// result into the work bit read by the following add-adjacent-zone pass (grid points only).
__device__ void ph_band_copy(const Grid2& g, uint8_t* m, int bit, int copy_to, Span sp)
{
    unsigned* mp = reinterpret_cast<unsigned*>(m);
    const unsigned nw = plane_words(g);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const MaskWord mw = mask_word(g, w);
        const unsigned G = grid_lanes(g, mw);
        if (!G) continue;
        unsigned inner = (mw.j >= 2 && mw.j <= g.ny - 3) ? lanes_in(mw.i0, 2, g.nx - 3) : 0u;
        if (g.bc_kind == AWCM_BC_WIND_TUNNEL) {
            // BOUNDARY_MANAGER_WT::BandingMask (Problems/2D/PROBLEM_WINDTUNNEL.h:202-220): also the
            // band around the step's top and front face
            if (abs(mw.j - g.wt_j) <= 2) inner &= ~lanes_in(mw.i0, g.wt_i - 2, g.nx - 1);
            if (mw.j <= g.wt_j + 2) inner &= ~lanes_in(mw.i0, g.wt_i - 2, g.wt_i + 2);
        }
        const unsigned v = mp[w];
        unsigned nv = v | (lane_bits(G & ~inner) << bit);
        if (copy_to >= 0) {
            const unsigned gb = lane_bits(G);
            nv = (nv & ~(gb << copy_to)) | (((nv >> bit) & gb) << copy_to);
        }
        if (nv != v) mp[w] = nv;
    }
}

// AddAdjacentZone (AWCM_MANAGER_2D.h:14-61): every detail point whose copy bit is set marks its
// finer neighbours in `bit`.  A point (i,j) = (odd*2^a, odd*2^b) is a detail of level
// maxl-1-min(a,b): d1 if a < b, d2 if a > b, d3 if a == b (boundary rows/columns excluded as in
// the sub-grids).
__device__ void ph_aaz(const Grid2& g, uint8_t* m, int bit, int src, Span sp)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    const unsigned nw = plane_words(g);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const unsigned v = mp[w];
        if (!((v >> src) & kLaneBits)) continue;  // no detail of `src` in this word
        const MaskWord mw = mask_word(g, w);
        const unsigned G = grid_lanes(g, mw);
        if (!G) continue;
        unsigned hit = (v >> src) & lane_bits(G);
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const int i = mw.i0 + L, j = mw.j;
            const int ti = ctz_or(i, 64), tj = ctz_or(j, 64);
            const int mn = ti < tj ? ti : tj;
            if (mn >= g.maxl) continue;
            if (ti < tj && (j == 0 || j == NY)) continue;
            if (tj < ti && (i == 0 || i == NX)) continue;
            const int lev = g.maxl - 1 - mn;
            if (lev == g.maxl - 1) {
                push_bit(g, m, i - 1, j, bit);
                push_bit(g, m, i + 1, j, bit);
                push_bit(g, m, i, j - 1, bit);
                push_bit(g, m, i, j + 1, bit);
            } else {
                const int D = g.D(lev), h = D / 2, q4 = D / 4;
                push_bit(g, m, i - q4, j, bit);
                push_bit(g, m, i + q4, j, bit);
                push_bit(g, m, i, j - q4, bit);
                push_bit(g, m, i, j + q4, bit);
                push_bit(g, m, i - h, j, bit);
                push_bit(g, m, i + h, j, bit);
                push_bit(g, m, i, j - h, bit);
                push_bit(g, m, i, j + h, bit);
            }
        }
    }
}

__device__ __forceinline__ bool mask_or_ghost(const Grid2& g, const uint8_t* m, int i, int j, int bit)
{
    // Beyond the ghost ring a mask reads as set, like the ghosts themselves.
    if (i < -kGhost || i >= g.nx + kGhost || j < -kGhost || j >= g.ny + kGhost) return true;
    return (m[g.at(i, j)] >> bit) & 1u;
}

// ComputeLevel (AWCM_MANAGER_2D.h:215-241) of mask `bit` into `lvl`; a level is left unchanged when
// no neighbour is found.  When copy_to >= 0 the pass also performs `mask_{k+1} = mask_k` on every
// byte of the plane, ghost ring included (the reference copies whole fields).  The level search
// runs for grid points only.
__device__ void ph_cl(const Grid2& g, uint8_t* m, int8_t* lvl, int bit, int copy_to, size_t plane, Span sp)
{
    unsigned* mp = reinterpret_cast<unsigned*>(m);
    unsigned* lp = reinterpret_cast<unsigned*>(lvl);
    const unsigned nw = (unsigned)(plane / 4);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const MaskWord mw = mask_word(g, w);
        const unsigned v = mp[w];
        const unsigned G = grid_lanes(g, mw);
        if (G) {
            const unsigned lv0 = lp[w];
            unsigned lv = lv0;
            const unsigned on = (v >> bit) & kLaneBits;
#pragma unroll
            for (int L = 0; L < 4; ++L) {
                if (!((G >> L) & 1u)) continue;
                const unsigned sh = 8u * L;
                if (!((on >> sh) & 1u)) {
                    lv &= ~(0xffu << sh);
                    continue;
                }
                const int i = mw.i0 + L, j = mw.j;
                int dx = 1;
                for (int lev = g.maxl; lev >= 0; --lev) {
                    if (mask_or_ghost(g, m, i - dx, j, bit) || mask_or_ghost(g, m, i + dx, j, bit) ||
                        mask_or_ghost(g, m, i, j - dx, bit) || mask_or_ghost(g, m, i, j + dx, bit)) {
                        lv = (lv & ~(0xffu << sh)) | ((unsigned)(uint8_t)(int8_t)lev << sh);
                        break;
                    }
                    dx *= 2;
                }
            }
            if (lv != lv0) lp[w] = lv;
        }
        if (copy_to >= 0) {
            const unsigned nv = (v & ~(kLaneBits << copy_to)) | (((v >> bit) & kLaneBits) << copy_to);
            if (nv != v) mp[w] = nv;
        }
    }
}

// AddPointForDifferentiation (AWCM_MANAGER_2D.h:160-213): points of mask `src` mark their flux
// stencil in `bit` (finest level: the +-3 cross; coarser: +-2 spacings, shifted at the edges).
__device__ void ph_apd(const Grid2& g, uint8_t* m, const int8_t* lvl, int bit, int src, Span sp)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    const unsigned nw = plane_words(g);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const MaskWord mw = mask_word(g, w);
        if (mw.j < 1 || mw.j > NY - 1) continue;
        const unsigned I = lanes_in(mw.i0, 1, NX - 1);
        if (!I) continue;
        unsigned hit = (mp[w] >> src) & lane_bits(I);
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const int i = mw.i0 + L, j = mw.j;
            const int lev = lvl[4u * w + L];
            if (lev == g.maxl) {
                for (int c = -3; c <= 3; ++c) {
                    push_bit(g, m, i + c, j, bit);
                    push_bit(g, m, i, j + c, bit);
                }
                continue;
            }
            const int D = g.D(lev);
            int lo = -2, hi = 2;
            if (i - 2 * D < 0) lo = -1;
            else if (i + 2 * D > NX) hi = 1;
            for (int c = lo; c <= hi; ++c) push_bit(g, m, i + D * c, j, bit);
            lo = -2, hi = 2;
            if (j - 2 * D < 0) lo = -1;
            else if (j + 2 * D > NY) hi = 1;
            for (int c = lo; c <= hi; ++c) push_bit(g, m, i, j + D * c, bit);
        }
    }
}

// ComputeLevel of mask k-1 into lvl, mask_k = mask_{k-1} and AddPointForDifferentiation(mask_k,
// level_{k-1}) in one pass, for bit k cleared beforehand on every byte: the copy and the pushes
// both only set bit k (atomic ORs), nothing in the pass reads bit k, bit k-1 does not change,
// and each point's level is computed by the thread that then reads it.  The same results as
// ph_cl followed by ph_apd.
__device__ void ph_cl_apd(const Grid2& g, uint8_t* m, int8_t* lvl, int k, size_t plane, Span sp)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const int src = k - 1;
    unsigned* mp = reinterpret_cast<unsigned*>(m);
    unsigned* lp = reinterpret_cast<unsigned*>(lvl);
    const unsigned nw = (unsigned)(plane / 4);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const unsigned v = mp[w];
        // most words hold no point of mask k-1 and no non-zero level: nothing to write or push
        if (!((v >> src) & kLaneBits) && !lp[w]) continue;
        const MaskWord mw = mask_word(g, w);
        const unsigned G = grid_lanes(g, mw);
        unsigned lv = 0;
        if (G) {
            const unsigned lv0 = lp[w];
            lv = lv0;
            const unsigned on = (v >> src) & kLaneBits;
#pragma unroll
            for (int L = 0; L < 4; ++L) {
                if (!((G >> L) & 1u)) continue;
                const unsigned sh = 8u * L;
                if (!((on >> sh) & 1u)) {
                    lv &= ~(0xffu << sh);
                    continue;
                }
                const int i = mw.i0 + L, j = mw.j;
                int dx = 1;
                for (int lev = g.maxl; lev >= 0; --lev) {
                    if (mask_or_ghost(g, m, i - dx, j, src) || mask_or_ghost(g, m, i + dx, j, src) ||
                        mask_or_ghost(g, m, i, j - dx, src) || mask_or_ghost(g, m, i, j + dx, src)) {
                        lv = (lv & ~(0xffu << sh)) | ((unsigned)(uint8_t)(int8_t)lev << sh);
                        break;
                    }
                    dx *= 2;
                }
            }
            if (lv != lv0) lp[w] = lv;
        }
        const unsigned cp = ((v >> src) & kLaneBits) << k;
        if (cp) atomicOr(&mp[w], cp);
        if (mw.j < 1 || mw.j > NY - 1) continue;
        const unsigned I = lanes_in(mw.i0, 1, NX - 1);
        unsigned hit = (v >> src) & lane_bits(I);
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const int i = mw.i0 + L, j = mw.j;
            const int lev = (int)(int8_t)(uint8_t)(lv >> (8 * L));
            if (lev == g.maxl) {
                // i, j in [1, N-1]: the cross i-3..i+3, j-3..j+3 lies on the ghosted plane
                push_run(g, m, i - 3, 7, 1, j, k);
                for (int c = -3; c <= 3; ++c)
                    if (c) push_bit_in(g, m, i, j + c, k);
                continue;
            }
            const int D = g.D(lev);
            int lo = -2, hi = 2;
            if (i - 2 * D < 0) lo = -1;
            else if (i + 2 * D > NX) hi = 1;
            for (int c = lo; c <= hi; ++c) push_bit(g, m, i + D * c, j, k);
            lo = -2, hi = 2;
            if (j - 2 * D < 0) lo = -1;
            else if (j + 2 * D > NY) hi = 1;
            for (int c = lo; c <= hi; ++c) push_bit(g, m, i, j + D * c, k);
        }
    }
}

// Work mask of InterpolateEuler: `to` minus `from` over the grid points (ghost bits untouched);
// to < 0 stands for every grid point (InterpolateAllGridEuler).
__device__ void ph_interp_init(const Grid2& g, uint8_t* m, int from, int to, Span sp)
{
    unsigned* mp = reinterpret_cast<unsigned*>(m);
    const unsigned nw = plane_words(g);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const unsigned v = mp[w];
        // no point of `to` and no work bit to clear: the word stays as it is
        if (to >= 0 && !(((v >> to) | (v >> kBitInterp)) & kLaneBits)) continue;
        const MaskWord mw = mask_word(g, w);
        const unsigned G = grid_lanes(g, mw);
        if (!G) continue;
        const unsigned gb = lane_bits(G);
        const unsigned on = (to >= 0 ? (v >> to) : ~0u) & ~(v >> from) & gb;
        const unsigned nv = (v & ~(gb << kBitInterp)) | (on << kBitInterp);
        if (nv != v) mp[w] = nv;
    }
}

// RemoveResidueEuler (AWCM_MANAGER_2D.h:267-280): zero interior points outside `bit`.  In the
// step only points that can hold non-zero values (in mask3 or in the previous mask0) are written.
__device__ void ph_remove_residue(const Grid2& g, Field4 q, const uint8_t* m, int bit, bool full, Span sp)
{
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    const unsigned nw = plane_words(g);
    for (unsigned w = sp.t0; w < nw; w += sp.stride) {
        const unsigned v = mp[w];
        if (!full && !(((v >> 3) | (v >> kBitTemp)) & kLaneBits)) continue;  // nothing non-zero here
        const MaskWord mw = mask_word(g, w);
        if (mw.j < 1 || mw.j > g.ny - 2) continue;
        const unsigned I = lanes_in(mw.i0, 1, g.nx - 2);
        if (!I) continue;
        unsigned hit = ~(v >> bit) & lane_bits(I);
        if (!full) hit &= (v >> 3) | (v >> kBitTemp);
        hit &= kLaneBits;
        while (hit) {
            const int L = (__ffs(hit) - 1) >> 3;
            hit &= hit - 1;
            const size_t a = 4u * w + L;
            q.p[0][a] = 0.0;
            q.p[1][a] = 0.0;
            q.p[2][a] = 0.0;
            q.p[3][a] = 0.0;
        }
    }
}

// ------------------------------------------------------------------------ standalone kernels
#define AWCM_SKIP_IF_DONE(st) \
    if ((st) && (st)->done) return

__global__ void k_fwt_a(Grid2 g, double* q, double* tb, uint8_t* m, int lev, int idle, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    if (idle && lev == g.maxl - 1) ph_fwt_a_fine(g, q, tb, m, st->tol, grid_span());
    else ph_fwt_a(g, q, tb, m, lev, st->tol, idle != 0, grid_span());
}
__global__ void k_fwt_b(Grid2 g, double* q, const double* tb, const uint8_t* m, int lev, int idle, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    if (idle && lev == g.maxl - 1) ph_fwt_b_fine(g, q, tb, m, grid_span());
    else ph_fwt_b(g, q, tb, m, lev, idle != 0, grid_span());
}
template <int PH>
__global__ void k_iwt(Grid2 g, double* q, const uint8_t* m, int lev, int bit, int sparse, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    const bool zero_all = !sparse || !st || st->full_zero;
    if (!zero_all && lev == g.maxl - 1) ph_iwt_fine<PH>(g, q, m, bit, grid_span());
    else ph_iwt<PH>(g, q, m, lev, bit, zero_all, grid_span());
}
__global__ void k_cr(Grid2 g, uint8_t* m, int lev, int bit, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_cr(g, m, lev, bit, grid_span());
}
__global__ void k_cr_rows(Grid2 g, uint8_t* m, int lev, int bit, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_cr_rows(g, m, lev, bit, grid_span());
}
template <int PH>
__global__ void k_interp(Grid2 g, Field4 q, const uint8_t* m, int lev, int from_bit, int p0, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_interp<PH>(g, q, m, lev, from_bit, p0, grid_span());
}
template <int PH>
__global__ void k_interp_rows(Grid2 g, Field4 q, const uint8_t* m, int lev, int from_bit, int p0,
                              const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_interp_rows<PH>(g, q, m, lev, from_bit, p0, grid_span());
}
__global__ void k_copy_bit_all(uint8_t* m, size_t n, int from, int to, const StepState* st, unsigned clear)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_copy_bit_all(m, n, from, to, grid_span(), clear);
}
__global__ void k_band_copy(Grid2 g, uint8_t* m, int bit, int copy_to, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_band_copy(g, m, bit, copy_to, grid_span());
}
__global__ void k_aaz(Grid2 g, uint8_t* m, int bit, int src, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_aaz(g, m, bit, src, grid_span());
}
__global__ void k_cl(Grid2 g, uint8_t* m, int8_t* lvl, int bit, int copy_to, size_t plane, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_cl(g, m, lvl, bit, copy_to, plane, grid_span());
}
__global__ void k_apd(Grid2 g, uint8_t* m, const int8_t* lvl, int bit, int src, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_apd(g, m, lvl, bit, src, grid_span());
}
__global__ void k_cl_apd(Grid2 g, uint8_t* m, int8_t* lvl, int k, size_t plane, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_cl_apd(g, m, lvl, k, plane, grid_span());
}
// The coarsest level's first inverse-transform phase (CTAs [0, nb)) and the interpolation work mask
// `to` minus `from` (the other CTAs) in one launch: the mask pass rewrites only the work bit.
__global__ void k_iwt0_interp_init(Grid2 g, double* q, uint8_t* m, int lev, int to, int from, int sparse,
                                   const StepState* st, unsigned nb)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    if (blockIdx.x < nb)
        ph_iwt<0>(g, q, m, lev, to, !sparse || !st || st->full_zero,
                  Span{blockIdx.x * blockDim.x + threadIdx.x, nb * blockDim.x});
    else
        ph_interp_init(g, m, from, to, Span{(blockIdx.x - nb) * blockDim.x + threadIdx.x, (gridDim.x - nb) * blockDim.x});
}
__global__ void k_interp_init(Grid2 g, uint8_t* m, int from, int to, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    ph_interp_init(g, m, from, to, grid_span());
}
__global__ void k_remove_residue(Grid2 g, Field4 q, const uint8_t* m, int bit, int sparse, const StepState* st)
{
    pdl_begin();
    AWCM_SKIP_IF_DONE(st);
    const bool full = !sparse || (st && st->full_zero);
    ph_remove_residue(g, q, m, bit, full, grid_span());
}

// ------------------------------------------------------------------- persistent PrepareEuler
// Grid-wide barrier for the persistent prepare kernel (all CTAs co-resident: cooperative launch).
// Arrive = device-scope acq_rel increment of `count`; the last CTA resets `count` and bumps the
// generation; the others spin on the generation with a bounded number of polls.  A spin that
// runs out, or an error already raised by another CTA, sets `err` and every CTA leaves at its
// next barrier: the step then reports a timeout instead of hanging.
constexpr unsigned kSpinLimit = 1u << 22;  // polls of >= 64 ns: well over a second

struct GridSync {
    unsigned* count;
    unsigned* gen;
    int* err;
    unsigned nb;
    unsigned limit;  // polls before a wait gives up
    __device__ bool sync() const
    {
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile int* ve = err;
            if (*ve == 0) {
                cuda::atomic_ref<unsigned, cuda::thread_scope_device> G(*gen), C(*count);
                const unsigned my = G.load(cuda::memory_order_acquire);
                __threadfence();
                if (C.fetch_add(1u, cuda::memory_order_acq_rel) == nb - 1) {
                    C.store(0u, cuda::memory_order_relaxed);
                    G.fetch_add(1u, cuda::memory_order_release);
                } else {
                    unsigned spins = 0;
                    while (G.load(cuda::memory_order_acquire) == my) {
                        if (++spins > limit || *ve) {
                            atomicCAS(err, 0, (int)kErrTimeout);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                __threadfence();
            }
        }
        __syncthreads();
        return *(volatile int*)err == 0;
    }
};

struct PrepArgs {
    Grid2 g;
    Field4 q;
    double* tb;
    uint8_t* m;
    int8_t* lvl[4];
    const StepState* st;
    unsigned* sync;  // [0] arrival count, [1] generation
    int* err;
    size_t plane;
};


constexpr int kPrepThreads = 1024;

// AWCM_2D::PrepareEuler (Wavelet/AWCM_2D.h:114-147) as one persistent kernel: the reference's
// level-sequential passes run back to back, separated by grid barriers instead of launches.
__global__ void __launch_bounds__(kPrepThreads, 1) k_prepare(PrepArgs A)
{
    if (A.st->done) return;
    const Grid2& g = A.g;
    const Span sp = grid_span();
    const GridSync gs{A.sync, A.sync + 1, A.err, gridDim.x, A.st->spin_limit ? A.st->spin_limit : kSpinLimit};
    const double tol = A.st->tol;
#define SYNC_OR_LEAVE \
    if (!gs.sync()) return
    ph_copy_bit_all(A.m, A.plane, 0, kBitTemp, sp);
    SYNC_OR_LEAVE;
    for (int lev = g.maxl - 1; lev >= 0; --lev) {
        ph_fwt_a(g, A.q.p[0], A.tb, A.m, lev, tol, true, sp);
        SYNC_OR_LEAVE;
        ph_fwt_b(g, A.q.p[0], A.tb, A.m, lev, true, sp);
        SYNC_OR_LEAVE;
    }
    ph_band_copy(g, A.m, 0, kBitCopy, sp);
    SYNC_OR_LEAVE;
    ph_aaz(g, A.m, 0, kBitCopy, sp);
    SYNC_OR_LEAVE;
    for (int lev = g.maxl - 1; lev >= 0; --lev) {
        ph_cr(g, A.m, lev, 0, sp);
        SYNC_OR_LEAVE;
    }
    for (int k = 1; k <= 3; ++k) {
        ph_cl(g, A.m, A.lvl[k - 1], k - 1, k, A.plane, sp);
        SYNC_OR_LEAVE;
        ph_apd(g, A.m, A.lvl[k - 1], k, k - 1, sp);
        SYNC_OR_LEAVE;
        for (int lev = g.maxl - 1; lev >= 0; --lev) {
            ph_cr(g, A.m, lev, k, sp);
            SYNC_OR_LEAVE;
        }
    }
    for (int lev = 0; lev < g.maxl; ++lev) {
        ph_iwt<0>(g, A.q.p[0], A.m, lev, 3, A.st->full_zero != 0, sp);
        SYNC_OR_LEAVE;
        ph_iwt<1>(g, A.q.p[0], A.m, lev, 3, A.st->full_zero != 0, sp);
        SYNC_OR_LEAVE;
        ph_iwt<2>(g, A.q.p[0], A.m, lev, 3, A.st->full_zero != 0, sp);
        SYNC_OR_LEAVE;
    }
    ph_interp_init(g, A.m, kBitTemp, 3, sp);
    SYNC_OR_LEAVE;
    for (int lev = g.maxl - 1; lev >= 0; --lev) {
        ph_cr(g, A.m, lev, kBitInterp, sp);
        SYNC_OR_LEAVE;
    }
    for (int lev = 0; lev < g.maxl; ++lev) {
        ph_interp<0>(g, A.q, A.m, lev, kBitTemp, 1, sp);
        SYNC_OR_LEAVE;
        ph_interp<1>(g, A.q, A.m, lev, kBitTemp, 1, sp);
        if (lev + 1 < g.maxl) SYNC_OR_LEAVE;
    }
#undef SYNC_OR_LEAVE
}

// ------------------------------------------------------------------------------------ boundaries
__device__ __forceinline__ double euler_E(double g, double rho, double u, double v, double p)
{
    return p / (g - 1) + 0.5 * rho * (u * u + v * v);
}

// Ghost fill of the edge strips (corners are never read by the axis-aligned stencils):
// transmissive BOUNDARY_MANAGER_QUAD (Problems/2D/PROBLEM_QUADRANTS.h:123-203), double Mach
// BOUNDARY_MANAGER_DMACH(t) (Problems/2D/PROBLEM_DOUBLEMACH.h:106-245), periodic
// BOUNDARY_MANAGER_ISENVORTEX (Problems/2D/PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h:107-171) and
// BOUNDARY_MANAGER_SHOCK_VORTEX (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:118-201:
// transmissive left/right, bottom/top walls reflecting rho v).
// BOUNDARY_CONDITION values of the generic manager (BOUNDARY_MANAGER_2D.h:7-13).
constexpr int kBcPeriodic = -3, kBcExtrapolation = -2;

// The enum-driven BOUNDARY_MANAGER_2D<TT>::SetBoundaryCondition(field) (BOUNDARY_MANAGER_2D.h:
// 61-158): each ghost cell of the left/right strips (interior rows), the bottom/top strips
// (interior columns) and the four corner blocks takes, by its own BOUNDARY_CONDITION, the zero-order
// extrapolation of the nearest edge (corner) point or, on the strips, the periodic image
// (ghost -1-c <- end-c, end+1+c <- start+c); any other kind leaves the cell as it is.  Every read is
// of a grid point, every write of a ghost cell: the reference's sequence of five passes is
// order-free, so one thread per ghost cell computes it.
__device__ void bc_fill_generic(const Grid2& g, Field4 f, long tid)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const long nside = (long)kGhost * g.ny, nbt = (long)kGhost * g.nx, ncorner = 4L * kGhost * kGhost;
    int i, j, si, sj;
    if (tid < 2 * nside) {
        const bool right = tid >= nside;
        const long r = right ? tid - nside : tid;
        j = (int)(r / kGhost);
        const int c = (int)(r % kGhost);
        i = right ? NX + 1 + c : -1 - c;
        const int k = g.bcf[g.at(i, j)];
        if (k == kBcExtrapolation) si = right ? NX : 0;
        else if (k == kBcPeriodic) si = right ? c : NX - c;
        else return;
        sj = j;
    } else if (tid < 2 * nside + 2 * nbt) {
        const long r0 = tid - 2 * nside;
        const bool top = r0 >= nbt;
        const long r = top ? r0 - nbt : r0;
        i = (int)(r / kGhost);
        const int c = (int)(r % kGhost);
        j = top ? NY + 1 + c : -1 - c;
        const int k = g.bcf[g.at(i, j)];
        if (k == kBcExtrapolation) sj = top ? NY : 0;
        else if (k == kBcPeriodic) sj = top ? c : NY - c;
        else return;
        si = i;
    } else if (tid < 2 * nside + 2 * nbt + ncorner) {
        const int r = (int)(tid - 2 * nside - 2 * nbt);
        const int corner = r / (kGhost * kGhost), cell = r % (kGhost * kGhost);
        const bool right = corner & 1, top = corner >> 1;
        i = right ? NX + 1 + cell % kGhost : -1 - cell % kGhost;
        j = top ? NY + 1 + cell / kGhost : -1 - cell / kGhost;
        if (g.bcf[g.at(i, j)] != kBcExtrapolation) return;
        si = right ? NX : 0;
        sj = top ? NY : 0;
    } else {
        return;
    }
    const size_t a = g.at(i, j), s = g.at(si, sj);
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
    for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
}

// BOUNDARY_MANAGER_WT::SetBoundaryCondition (Problems/2D/PROBLEM_WINDTUNNEL.h:94-199, "except bottom"):
// Mach 3 inflow (rho 1.4, u 3, v 0, p 1) in the left ghost columns and zero-order extrapolation in
// the right ones (interior rows), rho v reflected in the top ghost rows (interior columns).
__device__ void bc_fill_wind_tunnel(const Grid2& g, Field4 f, long tid)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const long nside = (long)kGhost * g.ny, nbt = (long)kGhost * g.nx;
    if (tid < 2 * nside) {
        const bool right = tid >= nside;
        const long r = right ? tid - nside : tid;
        const int j = (int)(r / kGhost), c = (int)(r % kGhost);
        const size_t a = g.at(right ? NX + 1 + c : -1 - c, j);
        if (!right) {
            const double rho = 1.4, u = 3, v = 0, p = 1;
            f.p[0][a] = rho;
            f.p[1][a] = rho * u;
            f.p[2][a] = rho * v;
            f.p[3][a] = p / (1.4 - 1) + 0.5 * rho * (u * u + v * v);
        } else {
            const size_t s = g.at(NX, j);
            double v[4];
            for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
            for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
        }
        return;
    }
    const long r0 = tid - 2 * nside;
    if (r0 < nbt || r0 >= 2 * nbt) return;  // bottom: per sweep direction (k_wt_bottom_*)
    const long r = r0 - nbt;
    const int i = (int)(r / kGhost), c = (int)(r % kGhost);
    const size_t a = g.at(i, NY + 1 + c), s = g.at(i, NY);
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
    v[2] = -v[2];
    for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
}

__device__ void bc_fill(const Grid2& g, Field4 f, const StepState* st, double t_host, double* zx, double* zy,
                        long tid)
{
    const double t = st ? st->t : t_host;
    // zero the LF-speed accumulators of the stage this fill feeds (the grid covers nx and ny)
    if (zx && tid < g.ny) zx[tid] = 0.0;
    if (zy && tid < g.nx) zy[tid] = 0.0;
    if (g.bc_kind == AWCM_BC_GENERIC) {
        bc_fill_generic(g, f, tid);
        return;
    }
    if (g.bc_kind == AWCM_BC_WIND_TUNNEL) {
        bc_fill_wind_tunnel(g, f, tid);
        return;
    }
    const int NX = g.nx - 1, NY = g.ny - 1;
    const long nside = (long)kGhost * g.ny, nbt = (long)kGhost * g.nx;
    int i, j, si, sj;  // ghost point and source point
    const double g14 = 1.4;
    if (tid < 2 * nside) {
        const bool right = tid >= nside;
        const long r = right ? tid - nside : tid;
        j = (int)(r / kGhost);
        const int c = (int)(r % kGhost);
        if (!right) {
            i = -1 - c;
            si = g.bc_kind == AWCM_BC_PERIODIC ? NX - c : 0;
        } else {
            i = NX + 1 + c;
            si = g.bc_kind == AWCM_BC_PERIODIC ? c : NX;
        }
        sj = j;
        const size_t a = g.at(i, j);
        if (!right && g.bc_kind == AWCM_BC_DOUBLE_MACH) {
            const double rho = 8, u = 8.25 * sqrt(3.0) * 0.5, v = -8.25 * 0.5, p = 116.5;
            f.p[0][a] = rho;
            f.p[1][a] = rho * u;
            f.p[2][a] = rho * v;
            f.p[3][a] = euler_E(g.gamma, rho, u, v, p);
            return;
        }
        const size_t s = g.at(si, sj);
        double v[4];
        for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
        for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
        return;
    }
    const long r0 = tid - 2 * nside;
    if (r0 >= 2 * nbt) return;
    const bool top = r0 >= nbt;
    const long r = top ? r0 - nbt : r0;
    i = (int)(r / kGhost);
    const int c = (int)(r % kGhost);
    if (!top) {
        j = -1 - c;
        sj = g.bc_kind == AWCM_BC_PERIODIC ? NY - c : 0;
    } else {
        j = NY + 1 + c;
        sj = g.bc_kind == AWCM_BC_PERIODIC ? c : NY;
    }
    const size_t a = g.at(i, j);
    if (g.bc_kind == AWCM_BC_DOUBLE_MACH) {
        const double sqrt3 = sqrt(3.0);
        const double x = g.x_min + i * g.dx;
        const double post[4] = {8, 8 * 8.25 * sqrt3 * 0.5, -8 * 8.25 * 0.5,
                                euler_E(g14, 8, 8.25 * sqrt3 * 0.5, -8.25 * 0.5, 116.5)};
        if (!top) {
            if (x > 1.0 / 6.0) {
                const size_t s = g.at(i, 0);
                f.p[0][a] = f.p[0][s];
                f.p[1][a] = f.p[1][s];
                f.p[2][a] = -f.p[2][s];
                f.p[3][a] = f.p[3][s];
            } else {
                for (int k = 0; k < 4; ++k) f.p[k][a] = post[k];
            }
        } else {
            const double pre[4] = {1.4, 1.4 * 0, 1.4 * 0, euler_E(g14, 1.4, 0, 0, 1)};
            const bool behind = x < 1.0 / 6.0 + (1 + 20 * t) / sqrt3;
            for (int k = 0; k < 4; ++k) f.p[k][a] = behind ? post[k] : pre[k];
        }
        return;
    }
    const size_t s = g.at(i, sj);
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
    if (g.bc_kind == AWCM_BC_SHOCK_VORTEX) v[2] = -v[2];
    for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
}

__global__ void k_bc(Grid2 g, Field4 f, const StepState* st, double t_host, double* zx, double* zy)
{
    pdl_begin();
    if (st && st->done) return;
    bc_fill(g, f, st, t_host, zx, zy, gtid());
}

// BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition(true, false) (PROBLEM_WINDTUNNEL.h:129-141) on f
// and, when f2.p[0] is set, on f2 too: the three columns i_bdry .. i_bdry+2 of rows -3 .. j_bdry
// take column i_bdry-1 with rho u reflected.  One thread per written cell (and field).
__global__ void k_wt_bottom_x(Grid2 g, Field4 f, Field4 f2, const StepState* st)
{
    pdl_begin();
    if (st && st->done) return;
    const unsigned t = gtid(), rows = (unsigned)(g.wt_j + kGhost + 1), per = 3u * rows;
    if (t >= (f2.p[0] ? 2u : 1u) * per) return;
    const Field4 F = t < per ? f : f2;
    const unsigned r = t % per;
    const int j = (int)(r / 3u) - kGhost, c = (int)(r % 3u);
    const size_t a = g.at(g.wt_i + c, j), s = g.at(g.wt_i - 1, j);
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = F.p[k][s];
    v[1] = -v[1];
    for (int k = 0; k < 4; ++k) F.p[k][a] = v[k];
}

// SetBottomBoundaryCondition(false, true) (PROBLEM_WINDTUNNEL.h:143-167), its two loops in order:
// part 0, the bottom ghost rows of columns -3 .. Nx+1 from row 0; part 1, the rows j_bdry-2 ..
// j_bdry of columns i_bdry .. Nx+2 from row j_bdry+1; rho v reflected.
__global__ void k_wt_bottom_y(Grid2 g, Field4 f, int part, const StepState* st)
{
    pdl_begin();
    if (st && st->done) return;
    const unsigned t = gtid();
    const int i0 = part == 0 ? -kGhost : g.wt_i;
    const int i1 = part == 0 ? g.nx - 1 + kGhost - 1 : g.nx - 1 + kGhost;  // inclusive
    if (t >= 3u * (unsigned)(i1 - i0 + 1)) return;
    const int i = i0 + (int)(t / 3u), c = (int)(t % 3u);
    const size_t a = part == 0 ? g.at(i, -1 - c) : g.at(i, g.wt_j - c);
    const size_t s = part == 0 ? g.at(i, 0) : g.at(i, g.wt_j + 1);
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = f.p[k][s];
    v[2] = -v[2];
    for (int k = 0; k < 4; ++k) f.p[k][a] = v[k];
}

// ------------------------------------------------------------------------- CFL and LF reductions
// Per-row alpha_x[j] = max |u|+c and per-column alpha_y[i] = max |v|+c over the points of mask
// `bit` (main_2d_euler(quad).cpp:86-104); with mv != null also the CFL speed
// max (|u|+c)+(|v|+c) (:61-76).  A CTA covers 128 columns (one mask word of four points per
// lane) x 32 rows (four per warp); empty words cost one load.  Maxima are order-independent.
constexpr int kAlphaRows = 4;
__global__ void __launch_bounds__(256) k_alpha(Grid2 g, Field4 f, const uint8_t* __restrict__ m, int bit,
                                               double* ax, double* ay, double* mv, const StepState* st,
                                               int* nonfinite)
{
    pdl_begin();
    if (st && st->done) return;
    __shared__ double col[8][128];
    __shared__ double cfl[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned wpr = (unsigned)g.pitch / 4u;  // mask words per plane row
    const unsigned wi = blockIdx.x * 32u + lane;
    const int i0 = 4 * (int)wi - kGhost;
    const unsigned* mp = reinterpret_cast<const unsigned*>(m);
    double cm[4] = {0, 0, 0, 0};
    double vmax = 0;
    bool nf = false;  // a NaN or infinite speed (NaN/Inf state, negative pressure or density)
    for (int r = 0; r < kAlphaRows; ++r) {
        const int j = (int)blockIdx.y * (8 * kAlphaRows) + warp * kAlphaRows + r;
        double sx_row = 0;
        if (j < g.ny && wi < wpr) {
            const unsigned lanes = lanes_in(i0, 0, g.nx - 1);
            const unsigned hit = (mp[(size_t)(j + kGhost) * wpr + wi] >> bit) & lane_bits(lanes);
#pragma unroll
            for (int L = 0; L < 4; ++L) {
                if (!((hit >> (8 * L)) & 1u)) continue;
                const size_t a = g.at(i0 + L, j);
                const double q[4] = {f.p[0][a], f.p[1][a], f.p[2][a], f.p[3][a]};
                const double c = sound2(q, g.gamma);
                const double sx = absd(q[1] / q[0]) + c;
                const double sy = absd(q[2] / q[0]) + c;
                nf |= !(isfinite(sx) && isfinite(sy));
                sx_row = maxd(sx_row, sx);
                cm[L] = maxd(cm[L], sy);
                vmax = maxd(vmax, sx + sy);
            }
        }
        const double rowmax = warp_max(sx_row);
        if (ax && lane == 0 && j < g.ny && rowmax > 0) atomic_max_nonneg(&ax[j], rowmax);
    }
    if (nonfinite && __any_sync(0xffffffffu, nf) && lane == 0) atomicOr(nonfinite, 1);
#pragma unroll
    for (int L = 0; L < 4; ++L) col[warp][4 * lane + L] = cm[L];
    vmax = warp_max(vmax);
    if (lane == 0) cfl[warp] = vmax;
    __syncthreads();
    if (threadIdx.x < 128) {
        double c = col[0][threadIdx.x];
        for (int y = 1; y < 8; ++y) c = maxd(c, col[y][threadIdx.x]);
        const int i = 4 * ((int)blockIdx.x * 32) - kGhost + (int)threadIdx.x;
        if (ay && i >= 0 && i < g.nx && c > 0) atomic_max_nonneg(&ay[i], c);
        if (mv && threadIdx.x == 0) {
            double v = cfl[0];
            for (int y = 1; y < 8; ++y) v = maxd(v, cfl[y]);
            if (v > 0) atomic_max_nonneg(mv, v);
        }
    }
}

// The same LF speeds over a mask whose points are already listed: the union of a stage's
// finest-level and coarse point lists is exactly the grid points of that stage's mask, so stage 2
// (mask2) reads the lists of stage 1's update and stage 3 (mask1) those of stage 2's.  One point
// per lane; the row maximum is a segmented max-scan over runs of equal rows in the warp (lists
// are row-ordered within each warp segment) with one atomic per run, the column maximum one
// atomic per point.  Maxima are order-independent, so the result equals k_alpha's.
// first: this CTA's first thread in the launch's range of LF-speed threads, stride: that range's size.
__device__ void alpha_list_run(const Grid2& g, Field4 f, const uint32_t* __restrict__ la,
                               const unsigned* __restrict__ na, const uint32_t* __restrict__ lb,
                               const unsigned* __restrict__ nb, double* ax, double* ay, unsigned first,
                               unsigned stride, int* nonfinite)
{
    const unsigned n0 = *na, n = n0 + *nb;
    const int lane = threadIdx.x & 31;
    bool nf = false;
    for (unsigned base = first + (threadIdx.x & ~31u); base < n; base += stride) {
        const unsigned e = base + (unsigned)lane;
        const bool on = e < n;
        int j = -1;
        double sx = 0;
        if (on) {
            const uint32_t idx = e < n0 ? la[e] : lb[e - n0];
            const int i = (int)(idx % (uint32_t)g.pitch) - kGhost;
            j = (int)(idx / (uint32_t)g.pitch) - kGhost;
            const double q[4] = {f.p[0][idx], f.p[1][idx], f.p[2][idx], f.p[3][idx]};
            const double c = sound2(q, g.gamma);
            sx = absd(q[1] / q[0]) + c;
            const double sy = absd(q[2] / q[0]) + c;
            nf |= !(isfinite(sx) && isfinite(sy));
            if (sy > 0) atomic_max_nonneg(&ay[i], sy);
        }
        const int jp = __shfl_up_sync(0xffffffffu, j, 1);
        const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || j != jp);
        const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
        double v = sx;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double o = __shfl_up_sync(0xffffffffu, v, off);
            if (lane - off >= start) v = maxd(v, o);
        }
        const int jn = __shfl_down_sync(0xffffffffu, j, 1);
        if (on && (lane == 31 || jn != j) && v > 0) atomic_max_nonneg(&ax[j], v);
    }
    if (nonfinite && __any_sync(0xffffffffu, nf) && lane == 0) atomicOr(nonfinite, 1);
}

__global__ void __launch_bounds__(256) k_alpha_list(Grid2 g, Field4 f, const uint32_t* __restrict__ la,
                                                    const unsigned* __restrict__ na,
                                                    const uint32_t* __restrict__ lb,
                                                    const unsigned* __restrict__ nb, double* ax, double* ay,
                                                    const StepState* st, int* nonfinite)
{
    pdl_begin();
    if (st->done) return;
    alpha_list_run(g, f, la, na, lb, nb, ax, ay, blockIdx.x * blockDim.x, gridDim.x * blockDim.x, nonfinite);
}

// Boundary fill and LF speeds of stage 2 or 3 in one launch: the fill writes only ghost cells and
// the speeds read only listed grid points, so neither waits for the other (the accumulators were
// zeroed by the worklist builder).  CTAs [0, bc_blocks) fill, the others compute the speeds.
__global__ void __launch_bounds__(256) k_bc_alpha(Grid2 g, Field4 f, const uint32_t* __restrict__ la,
                                                  const unsigned* __restrict__ na,
                                                  const uint32_t* __restrict__ lb,
                                                  const unsigned* __restrict__ nb, double* ax, double* ay,
                                                  const StepState* st, unsigned bc_blocks, int* nonfinite)
{
    pdl_begin();
    if (st->done) return;
    if (blockIdx.x < bc_blocks) {
        bc_fill(g, f, st, 0.0, nullptr, nullptr, (long)blockIdx.x * blockDim.x + threadIdx.x);
        return;
    }
    alpha_list_run(g, f, la, na, lb, nb, ax, ay, (blockIdx.x - bc_blocks) * blockDim.x,
                   (gridDim.x - bc_blocks) * blockDim.x, nonfinite);
}

// dt = cfl dx / max speed, clipped to the output time (main_2d_euler(quad).cpp:76-83), and the
// per-level stage factor dt / (dx 2^(maxl-lev)) of the RK updates.
__device__ void compute_dt(const Grid2& g, StepState* st)
{
    double dt = st->cfl * g.dx / st->mv;
    if (st->dt_fixed > 0) dt = st->dt_fixed;
    st->do_print = 0;
    if (st->t + dt > st->t_end) {
        dt = st->t_end - st->t;
        st->do_print = 1;
    }
    st->dt = dt;
    for (int lev = 0; lev <= g.maxl; ++lev) {
        const double dxl = g.dx * g.D(lev);
        st->sc[lev] = dt / dxl;
    }
}
__global__ void k_dt(Grid2 g, StepState* st)
{
    pdl_begin();
    if (st->done) return;
    compute_dt(g, st);
}

// keep_lists: the step reuses the worklists (and mask counts) of the previous one (frozen masks).
__global__ void k_begin(StepState* st, int keep_lists)
{
    pdl_begin();
    st->done = (st->t >= st->t_end || st->error) ? 1 : 0;
    if (st->done) return;
    st->bar[0] = 0;
    st->bar_err = 0;
    st->nonfinite = 0;
    st->mv = 0;
    if (keep_lists) return;
    for (int k = 0; k < 4 * kStages; ++k) st->cnt[k] = 0;
    for (int k = 0; k < 4; ++k) st->mask_cnt[k] = 0;
}

__global__ void k_copy4(Field4 dst, Field4 src, size_t n)
{
    pdl_begin();
    for (size_t a = gtid(); a < n; a += (size_t)gridDim.x * blockDim.x) {
        double v[4];
        for (int k = 0; k < 4; ++k) v[k] = src.p[k][a];
        for (int k = 0; k < 4; ++k) dst.p[k][a] = v[k];
    }
}

__global__ void k_finish(StepState* st)
{
    pdl_begin();
    if (st->done) return;
    if (st->bar_err) {
        st->error = st->bar_err;
        st->done = 1;
        return;
    }
    st->t += st->dt;
    st->steps += 1;
    st->upd += st->mask_cnt[0];
    st->stage_pts += (unsigned long long)st->mask_cnt[2] + st->mask_cnt[1] + st->mask_cnt[0];
    st->full_zero = 0;
    if (st->nonfinite) {
        // a NaN or infinite wave speed: the state is not a valid gas state; stop and report
        st->error = kErrNonFinite;
        st->done = 1;
    }
}

// ------------------------------------------------------------------------------------ worklists
// Builds, for the three stages (mask2/level2, mask1/level1, mask0/level0), row-ordered lists of
// finest-level points, coarse points, x faces (i+1/2, j) and y faces (i, j+1/2) whose flux a
// finest-level point needs.  A CTA covers 256 consecutive columns of kListRows rows of the grid
// extended by one row/column on the low side (faces -1/2); compaction is a warp ballot, a
// per-block prefix over warps and one atomicAdd per list per block.
constexpr int kListRows = 4;  // rows per CTA: 4 measured fastest (8: +0.8 % step time, 2: +0.1 %, 16: +2 %)
constexpr int kNumLists = 4 * kStages;

struct ListArgs {
    uint32_t* list[kNumLists];
    // optional: LF-speed accumulators of stages 2 and 3 to zero, and the dt computation (both need
    // only to happen after stage 1's speeds and before their own use)
    double *zx1 = nullptr, *zy1 = nullptr, *zx2 = nullptr, *zy2 = nullptr;
    int with_dt = 0;
};

// Stage predicates of the point (i, j) (i from -1, j from -1): per stage s (bits 4s..4s+3):
// finest-level point, coarse point, x face (i+1/2, j) needed, y face (i, j+1/2) needed.
__device__ __forceinline__ unsigned list_preds(const Grid2& g, const uint8_t* __restrict__ m,
                                               const int8_t* const (&lvls)[kStages], int i, int j, unsigned& mbits)
{
    const bool row_in = j >= 0 && j < g.ny, col_in = i >= 0 && i < g.nx;
    const bool inside = row_in && col_in;
    const bool right_in = row_in && i + 1 >= 0 && i + 1 < g.nx;
    const bool up_in = col_in && j + 1 >= 0 && j + 1 < g.ny;
    const unsigned here = inside ? m[g.at(i, j)] : 0u;
    const unsigned right = right_in ? m[g.at(i + 1, j)] : 0u;
    const unsigned up = up_in ? m[g.at(i, j + 1)] : 0u;
    mbits = here & 15u;
    if (!((here | right | up) & 7u)) return 0u;
    const bool xface = row_in && i <= g.nx - 1, yface = col_in && j <= g.ny - 1;
    unsigned p = 0;
#pragma unroll
    for (int s = 0; s < kStages; ++s) {
        const int bit = 2 - s;
        const int8_t* lvl = lvls[s];
        const bool act = (here >> bit) & 1u;
        const bool fin = act && lvl[g.at(i, j)] == g.maxl;
        const bool fin_r = ((right >> bit) & 1u) && lvl[g.at(i + 1, j)] == g.maxl;
        const bool fin_u = ((up >> bit) & 1u) && lvl[g.at(i, j + 1)] == g.maxl;
        p |= ((unsigned)fin | ((unsigned)(act && !fin) << 1) | ((unsigned)(xface && (fin || fin_r)) << 2) |
              ((unsigned)(yface && (fin || fin_u)) << 3))
             << (4 * s);
    }
    return p;
}

__global__ void __launch_bounds__(256) k_lists(Grid2 g, const uint8_t* __restrict__ m, const int8_t* __restrict__ l2,
                                               const int8_t* __restrict__ l1, const int8_t* __restrict__ l0,
                                               ListArgs la, StepState* st)
{
    pdl_begin();
    if (st->done) return;
    {
        const unsigned lin = (blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
        if (la.zx1 && lin < (unsigned)g.ny) la.zx1[lin] = la.zx2[lin] = 0.0;
        if (la.zy1 && lin < (unsigned)g.nx) la.zy1[lin] = la.zy2[lin] = 0.0;
        if (la.with_dt && lin == 0) compute_dt(g, st);
    }
    __shared__ unsigned wcnt[8][kNumLists];
    __shared__ unsigned woff[8][kNumLists];
    __shared__ unsigned mcnt[4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = (int)blockIdx.x * 256 + threadIdx.x - 1;  // -1 .. nx-1 (+ padding)
    const int8_t* const lvls[kStages] = {l2, l1, l0};
    if (threadIdx.x < kNumLists)
        for (int w = 0; w < 8; ++w) wcnt[w][threadIdx.x] = 0;
    if (threadIdx.x < 4) mcnt[threadIdx.x] = 0;
    __syncthreads();

    // predicates of the kListRows rows, kept in registers for the write pass
    const int j0 = (int)blockIdx.y * kListRows - 1;
    unsigned pm[kListRows];
    unsigned mloc[4] = {0, 0, 0, 0};
    unsigned any = 0;
#pragma unroll
    for (int r = 0; r < kListRows; ++r) {
        unsigned mb;
        pm[r] = list_preds(g, m, lvls, i, j0 + r, mb);
        any |= pm[r];
        if (j0 + r >= 0 && i >= 0)
            for (int k = 0; k < 4; ++k) mloc[k] += (mb >> k) & 1u;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const unsigned v = __reduce_add_sync(0xffffffffu, mloc[k]);
        if (lane == 0 && v) atomicAdd(&mcnt[k], v);
    }
    const bool warp_any = __any_sync(0xffffffffu, any != 0);
    if (warp_any) {
#pragma unroll
        for (int r = 0; r < kListRows; ++r) {
            if (!__any_sync(0xffffffffu, pm[r] != 0)) continue;
#pragma unroll
            for (int L = 0; L < kNumLists; ++L) {
                const unsigned bal = __ballot_sync(0xffffffffu, (pm[r] >> L) & 1u);
                if (lane == 0) wcnt[warp][L] += __popc(bal);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < kNumLists) {
        const int L = threadIdx.x;
        unsigned tot = 0;
        for (int w = 0; w < 8; ++w) {
            woff[w][L] = tot;
            tot += wcnt[w][L];
        }
        const unsigned base = tot ? atomicAdd(&st->cnt[L], tot) : 0;
        for (int w = 0; w < 8; ++w) woff[w][L] += base;
    }
    if (threadIdx.x < 4 && mcnt[threadIdx.x]) atomicAdd(&st->mask_cnt[threadIdx.x], mcnt[threadIdx.x]);
    __syncthreads();
    if (!warp_any) return;
    unsigned run[kNumLists];
#pragma unroll
    for (int L = 0; L < kNumLists; ++L) run[L] = woff[warp][L];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kListRows; ++r) {
        if (!__any_sync(0xffffffffu, pm[r] != 0)) continue;
        const int j = j0 + r;
        const uint32_t idx = (uint32_t)((size_t)(j + kGhost) * g.pitch + (size_t)(i + kGhost));
#pragma unroll
        for (int L = 0; L < kNumLists; ++L) {
            const bool p = (pm[r] >> L) & 1u;
            const unsigned bal = __ballot_sync(0xffffffffu, p);
            if (p) la.list[L][run[L] + __popc(bal & lt)] = idx;
            run[L] += __popc(bal);
        }
    }
}

// --------------------------------------------------------------------------------- stage kernels
// Face flux from the compacted face list: x faces (DIR 0) read cells i-2..i+3 of row j, y faces
// (DIR 1) cells j-2..j+3 of column i (WENOZ_EULER_SOLVER_2D::ComputeFluxX/Y, WENOZ.h:236-320).
// CUSTOM false: the reference's WENO-Z parameters as compile-time constants (eps 1e-40, exact
// |b0 - b2|); true: the instance's runtime parameters (the differentiable mode).
#ifndef AWCM_FACE_MIN_CTAS
#define AWCM_FACE_MIN_CTAS 4
#endif
template <int DIR, bool CUSTOM>
__global__ void __launch_bounds__(128, AWCM_FACE_MIN_CTAS)
    k_face(Grid2 g, Field4 f, Field4 out, const uint32_t* __restrict__ list, const unsigned* __restrict__ count,
           const double* __restrict__ alpha, const StepState* st, StepState* dt_st)
{
    pdl_begin();
    if (st->done) return;
    // dt_st: this launch also computes the step's dt (from the CFL speed of the scan before it);
    // the faces do not read it, the point updates after them do
    if (dt_st && blockIdx.x == 0 && threadIdx.x == 0) compute_dt(g, dt_st);
    const unsigned n = *count;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long e = gtid(); e < n; e += stride) {
        const uint32_t idx = list[e];
        const int ii = (int)(idx % (uint32_t)g.pitch) - kGhost;
        const int jj = (int)(idx / (uint32_t)g.pitch) - kGhost;
        const long step = DIR == 0 ? 1 : g.pitch;
        double s[6][4];
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            const long a = (long)idx + (p - 2) * step;
#pragma unroll
            for (int k = 0; k < 4; ++k) s[p][k] = f.p[k][a];
        }
        const double al = DIR == 0 ? alpha[jj] : alpha[ii];
        double o[4];
        if (CUSTOM) face_flux_2d<DIR>(s, al, g.gamma, o, g.wz_eps, g.wz_delta);
        else face_flux_2d<DIR>(s, al, g.gamma, o);
#pragma unroll
        for (int k = 0; k < 4; ++k) out.p[k][idx] = o[k];
    }
}

// RK combinations of the three stages (main_2d_euler(quad).cpp:162, 242, 321 and 325-332):
// KIND 1: out = in - sc (dF+dG); KIND 2: out = 0.75 qn + 0.25 (in - sc (dF+dG));
// KIND 3: qn = (qn + 2 (in - sc (dF+dG))) / 3.
// All four components are loaded before any is stored (a store to one plane could alias the
// next plane's load as far as the compiler knows, which would serialize the round trips).
template <int KIND>
__device__ __forceinline__ void rk_store(Field4 in, Field4 out, Field4 qn, size_t a, const double* dF,
                                         const double* dG, double sc)
{
    double x[4], y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x[k] = in.p[k][a];
        y[k] = KIND == 1 ? 0.0 : qn.p[k][a];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double r = x[k] - sc * (dF[k] + dG[k]);
        if (KIND == 1) y[k] = r;
        else if (KIND == 2) y[k] = 0.75 * y[k] + 0.25 * r;
        else y[k] = (y[k] + 2.0 * r) / 3.0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (KIND == 3) qn.p[k][a] = y[k];
        else out.p[k][a] = y[k];
    }
}

// Finest-level point: dF = F(i+1/2) - F(i-1/2), dG likewise, from the face planes.
template <int KIND>
__device__ __forceinline__ void update_fin_point(const Grid2& g, Field4 in, Field4 out, Field4 qn, Field4 fx,
                                                 Field4 fy, size_t a, double sc)
{
    double dF[4], dG[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        dF[k] = fx.p[k][a] - fx.p[k][a - 1];
        dG[k] = fy.p[k][a] - fy.p[k][a - g.pitch];
    }
    rk_store<KIND>(in, out, qn, a, dF, dG, sc);
}


// Coarse-level points: 4th-order central differences of F and G at spacing d = 2^(maxl-lev), with
// the reference's one-sided forms next to the boundary (AWCM_2D::Differentiate*, Wavelet/AWCM_2D.h:154-187,
// branch selection main_2d_euler(quad).cpp:132-160).
// inx: the field of the x-direction fluxes (the wind tunnel's x-sweep copy of the stage input, else in).
template <int KIND>
__device__ __forceinline__ void update_crs_point(const Grid2& g, Field4 in, Field4 inx, Field4 out, Field4 qn,
                                                 const int8_t* __restrict__ lvl, size_t a, const StepState* st)
{
    const int NX = g.nx - 1, NY = g.ny - 1;
    const int i = (int)((unsigned)a % (unsigned)g.pitch) - kGhost;
    const int j = (int)((unsigned)a / (unsigned)g.pitch) - kGhost;
    const int lev = lvl[a];
    if (lev < 0 || lev > g.maxl) return;
    const int d = g.D(lev);
    // Coarse stencils stay on the ghosted grid whenever the levels come from ComputeLevel on
    // a reconstruction-closed mask; any other point is skipped rather than read out of bounds.
    const int lo_x = i <= d ? i - d : i - 2 * d, hi_x = i >= NX - d && !(i <= d) ? i + d : i + 2 * d;
    const int lo_y = j <= d ? j - d : j - 2 * d, hi_y = j >= NY - d && !(j <= d) ? j + d : j + 2 * d;
    if (lo_x < -kGhost || hi_x > NX + kGhost || lo_y < -kGhost || hi_y > NY + kGhost) return;
    double dF[4], dG[4];
    {
        double fl[4], fr[4], fo[4], q[4];
        auto load = [&](long off, double* o) {
            for (int k = 0; k < 4; ++k) q[k] = inx.p[k][(long)a + off];
            flux2<0>(q, g.gamma, o);
        };
        load(-d, fl);
        load(d, fr);
        if (i <= d) {
            load(2 * d, fo);
            for (int k = 0; k < 4; ++k) dF[k] = kD1 * (fr[k] - fl[k]) + kD2 * (fo[k] - fl[k]);
        } else if (i >= NX - d) {
            load(-2 * d, fo);
            for (int k = 0; k < 4; ++k) dF[k] = kD1 * (fr[k] - fl[k]) + kD2 * (fr[k] - fo[k]);
        } else {
            double fll[4];
            load(-2 * d, fll);
            load(2 * d, fo);
            for (int k = 0; k < 4; ++k) dF[k] = kD1 * (fr[k] - fl[k]) + kD2 * (fo[k] - fll[k]);
        }
    }
    {
        const long P = g.pitch;
        double gb[4], gt[4], go[4], q[4];
        auto load = [&](long off, double* o) {
            for (int k = 0; k < 4; ++k) q[k] = in.p[k][(long)a + off * P];
            flux2<1>(q, g.gamma, o);
        };
        load(-d, gb);
        load(d, gt);
        if (j <= d) {
            load(2 * d, go);
            for (int k = 0; k < 4; ++k) dG[k] = kD1 * (gt[k] - gb[k]) + kD2 * (go[k] - gb[k]);
        } else if (j >= NY - d) {
            load(-2 * d, go);
            for (int k = 0; k < 4; ++k) dG[k] = kD1 * (gt[k] - gb[k]) + kD2 * (gt[k] - go[k]);
        } else {
            double gbb[4];
            load(-2 * d, gbb);
            load(2 * d, go);
            for (int k = 0; k < 4; ++k) dG[k] = kD1 * (gt[k] - gb[k]) + kD2 * (go[k] - gbb[k]);
        }
    }
    rk_store<KIND>(in, out, qn, a, dF, dG, st->sc[lev]);
}

// The finest-level and the coarse points of a stage in one launch: the two sets are disjoint and
// neither reads what the other writes (the stage output, or qn at the point itself).
template <int KIND>
__global__ void __launch_bounds__(256) k_update(Grid2 g, Field4 in, Field4 inx, Field4 out, Field4 qn, Field4 fx,
                                                Field4 fy, const int8_t* __restrict__ lvl,
                                                const uint32_t* __restrict__ lf, const unsigned* __restrict__ nf,
                                                const uint32_t* __restrict__ lc, const unsigned* __restrict__ nc,
                                                const StepState* st)
{
    pdl_begin();
    if (st->done) return;
    const unsigned n0 = *nf, n = n0 + *nc;
    const double sc = st->sc[g.maxl];
    const long stride = (long)gridDim.x * blockDim.x;
    for (long e = gtid(); e < n; e += stride) {
        if (e < n0) update_fin_point<KIND>(g, in, out, qn, fx, fy, lf[e], sc);
        else update_crs_point<KIND>(g, in, inx, out, qn, lvl, lc[e - n0], st);
    }
}

// ------------------------------------------------------------------------- layout conversions
// ------------------------------------------------------------------- scalar AWCM (advection)
// The scalar path of Wavelet/main_2d_advect.cpp:33-205 (AWCM_2D::Prepare on FIELD_UNIFORM_2D<double>,
// linear advection with unit velocity in x and y): finest-level points take the upwind WENO5 face
// values F(i+1/2) = WENO5::ReconstructRight(q[i-2..i+2]) (WENO.h:101-104) and dF = F(i+1/2) -
// F(i-1/2); coarser points the 4th-order central differences of q itself
// (AWCM_2D::Differentiate*, Wavelet/AWCM_2D.h:95-109) with the same edge forms as the Euler path.
template <int DIR>
__global__ void __launch_bounds__(256) k_face_scalar(Grid2 g, const double* __restrict__ f, double* __restrict__ out,
                                                     const uint32_t* __restrict__ list,
                                                     const unsigned* __restrict__ count, const StepState* st)
{
    pdl_begin();
    if (st->done) return;
    const unsigned n = *count;
    const long step = DIR == 0 ? 1 : g.pitch;
    for (unsigned e = gtid(); e < n; e += gridDim.x * blockDim.x) {
        const long a = list[e];
        out[a] = recon_left<kWeno5>(f[a + 2 * step], f[a + step], f[a], f[a - step], f[a - 2 * step]);
    }
}

// Stage combinations of main_2d_advect.cpp:65, 121, 177 and 183-189: KIND 1: out = in - sc (dF+dG);
// KIND 2: out = 0.75 qn + 0.25 (in - sc (dF+dG)); KIND 4: qn = 1/3 qn + 2/3 (in - sc (dF+dG)).
template <int KIND>
__device__ __forceinline__ void rk_store_scalar(const double* in, double* out, double* qn, size_t a, double d,
                                                double sc)
{
    const double r = in[a] - sc * d;
    if (KIND == 1) out[a] = r;
    else if (KIND == 2) out[a] = 0.75 * qn[a] + 0.25 * r;
    else qn[a] = kC1_3 * qn[a] + kD1 * r;
}

template <int KIND>
__global__ void __launch_bounds__(256) k_update_fin_scalar(Grid2 g, const double* in, double* out, double* qn,
                                                           const double* fx, const double* fy,
                                                           const uint32_t* __restrict__ list,
                                                           const unsigned* __restrict__ count, const StepState* st)
{
    pdl_begin();
    if (st->done) return;
    const unsigned n = *count;
    const double sc = st->sc[g.maxl];
    for (unsigned e = gtid(); e < n; e += gridDim.x * blockDim.x) {
        const size_t a = list[e];
        const double dF = fx[a] - fx[a - 1];
        const double dG = fy[a] - fy[a - g.pitch];
        rk_store_scalar<KIND>(in, out, qn, a, dF + dG, sc);
    }
}

template <int KIND>
__global__ void __launch_bounds__(256) k_update_crs_scalar(Grid2 g, const double* in, double* out, double* qn,
                                                           const int8_t* __restrict__ lvl,
                                                           const uint32_t* __restrict__ list,
                                                           const unsigned* __restrict__ count, const StepState* st)
{
    pdl_begin();
    if (st->done) return;
    const unsigned n = *count;
    const int NX = g.nx - 1, NY = g.ny - 1;
    for (unsigned e = gtid(); e < n; e += gridDim.x * blockDim.x) {
        const size_t a = list[e];
        const int i = (int)((unsigned)a % (unsigned)g.pitch) - kGhost;
        const int j = (int)((unsigned)a / (unsigned)g.pitch) - kGhost;
        const int lev = lvl[a];
        if (lev < 0 || lev > g.maxl) continue;
        const int d = g.D(lev);
        const int lo_x = i <= d ? i - d : i - 2 * d, hi_x = i >= NX - d && !(i <= d) ? i + d : i + 2 * d;
        const int lo_y = j <= d ? j - d : j - 2 * d, hi_y = j >= NY - d && !(j <= d) ? j + d : j + 2 * d;
        if (lo_x < -kGhost || hi_x > NX + kGhost || lo_y < -kGhost || hi_y > NY + kGhost) continue;
        auto X = [&](long o) { return in[(long)a + o]; };
        auto Y = [&](long o) { return in[(long)a + o * g.pitch]; };
        double dF, dG;
        if (i <= d) dF = kD1 * (X(d) - X(-d)) + kD2 * (X(2 * d) - X(-d));
        else if (i >= NX - d) dF = kD1 * (X(d) - X(-d)) + kD2 * (X(d) - X(-2 * d));
        else dF = kD1 * (X(d) - X(-d)) + kD2 * (X(2 * d) - X(-2 * d));
        if (j <= d) dG = kD1 * (Y(d) - Y(-d)) + kD2 * (Y(2 * d) - Y(-d));
        else if (j >= NY - d) dG = kD1 * (Y(d) - Y(-d)) + kD2 * (Y(d) - Y(-2 * d));
        else dG = kD1 * (Y(d) - Y(-d)) + kD2 * (Y(2 * d) - Y(-2 * d));
        rk_store_scalar<KIND>(in, out, qn, a, dF + dG, st->sc[lev]);
    }
}

__global__ void k_aos_to_soa(Grid2 g, const double* __restrict__ aos, Field4 f)
{
    pdl_begin();
    const long t = gtid();
    const int w = g.nx + 2 * kGhost;
    if (t >= (long)w * (g.ny + 2 * kGhost)) return;
    const int ii = (int)(t % w), jj = (int)(t / w);
    const size_t a = (size_t)jj * g.pitch + ii;
    for (int k = 0; k < 4; ++k) f.p[k][a] = aos[t * 4 + k];
}

__global__ void k_soa_to_aos(Grid2 g, Field4 f, double* __restrict__ aos)
{
    pdl_begin();
    const long t = gtid();
    const int w = g.nx + 2 * kGhost;
    if (t >= (long)w * (g.ny + 2 * kGhost)) return;
    const int ii = (int)(t % w), jj = (int)(t / w);
    const size_t a = (size_t)jj * g.pitch + ii;
    for (int k = 0; k < 4; ++k) aos[t * 4 + k] = f.p[k][a];
}

// masks: 5 planes (mask_temp, mask0..mask3) of (ny+6) x (nx+6) bytes <-> bit byte per point.
__global__ void k_pack_masks(Grid2 g, const uint8_t* __restrict__ planes, uint8_t* m)
{
    pdl_begin();
    const long t = gtid();
    const int w = g.nx + 2 * kGhost;
    const long n = (long)w * (g.ny + 2 * kGhost);
    if (t >= n) return;
    const int ii = (int)(t % w), jj = (int)(t / w);
    const int bits[5] = {kBitTemp, 0, 1, 2, 3};
    unsigned v = (1u << kBitInterp) | (1u << kBitCopy) | (1u << 7);
    for (int r = 0; r < 5; ++r) v |= (unsigned)(planes[r * n + t] != 0) << bits[r];
    const bool ghost = ii < kGhost || ii >= g.nx + kGhost || jj < kGhost || jj >= g.ny + kGhost;
    if (!ghost) v &= ~((1u << kBitInterp) | (1u << kBitCopy) | (1u << 7));
    m[(size_t)jj * g.pitch + ii] = (uint8_t)v;
}

__global__ void k_unpack_masks(Grid2 g, const uint8_t* m, uint8_t* __restrict__ planes)
{
    pdl_begin();
    const long t = gtid();
    const int w = g.nx + 2 * kGhost;
    const long n = (long)w * (g.ny + 2 * kGhost);
    if (t >= n) return;
    const int ii = (int)(t % w), jj = (int)(t / w);
    const int bits[5] = {kBitTemp, 0, 1, 2, 3};
    const unsigned v = m[(size_t)jj * g.pitch + ii];
    for (int r = 0; r < 5; ++r) planes[r * n + t] = (v >> bits[r]) & 1u;
}

__global__ void k_levels_in(Grid2 g, const int* __restrict__ lv, int8_t* l0, int8_t* l1, int8_t* l2, int8_t* l3)
{
    pdl_begin();
    const long t = gtid();
    const long n = (long)g.nx * g.ny;
    if (t >= n) return;
    const size_t a = g.at((int)(t % g.nx), (int)(t / g.nx));
    l0[a] = (int8_t)lv[t];
    l1[a] = (int8_t)lv[n + t];
    l2[a] = (int8_t)lv[2 * n + t];
    l3[a] = (int8_t)lv[3 * n + t];
}

__global__ void k_levels_out(Grid2 g, const int8_t* l0, const int8_t* l1, const int8_t* l2, const int8_t* l3,
                             int* __restrict__ lv)
{
    pdl_begin();
    const long t = gtid();
    const long n = (long)g.nx * g.ny;
    if (t >= n) return;
    const size_t a = g.at((int)(t % g.nx), (int)(t / g.nx));
    lv[t] = l0[a];
    lv[n + t] = l1[a];
    lv[2 * n + t] = l2[a];
    lv[3 * n + t] = l3[a];
}

__global__ void k_fill_u8(uint8_t* p, size_t n, uint8_t v)
{
    pdl_begin();
    const size_t a = (size_t)gtid();
    if (a < n) p[a] = v;
}

__global__ void k_fill_i8(int8_t* p, size_t n, int8_t v)
{
    pdl_begin();
    const size_t a = (size_t)gtid();
    if (a < n) p[a] = v;
}

// EULER_EQUATION_2D batch entry points.
__global__ void k_euler_flux(const double* q, double* f, int n, int dir, double gamma)
{
    pdl_begin();
    const long t = gtid();
    if (t >= n) return;
    double s[4] = {q[4 * t], q[4 * t + 1], q[4 * t + 2], q[4 * t + 3]}, o[4];
    if (dir == 0) flux2<0>(s, gamma, o);
    else flux2<1>(s, gamma, o);
    for (int k = 0; k < 4; ++k) f[4 * t + k] = o[k];
}

__global__ void k_euler_sr(const double* q, double* out, int n, int dir, double gamma)
{
    pdl_begin();
    const long t = gtid();
    if (t >= n) return;
    const double s[4] = {q[4 * t], q[4 * t + 1], q[4 * t + 2], q[4 * t + 3]};
    const double c = sound2(s, gamma);
    out[t] = absd((dir == 0 ? s[1] : s[2]) / s[0]) + c;
}

inline unsigned blocks_for(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ===================================================================================== Solver2D
struct Solver2D {
    Grid2 g{};
    size_t plane = 0;
    Field4 q{}, q2{}, q1{}, fx{}, fy{};
    Field4 qx{};  // wind tunnel: the x-sweep copy of the stage input
    uint8_t* m = nullptr;
    int8_t* lvl[4] = {nullptr, nullptr, nullptr, nullptr};
    double* ax[kStages] = {};
    double* ay[kStages] = {};
    StepState* st = nullptr;
    uint32_t* lists[kNumLists] = {};
    void* staging = nullptr;
    size_t staging_bytes = 0;
    int8_t* bcf_dev = nullptr;  // BOUNDARY_CONDITION plane of the generic manager
    cudaStream_t stream = nullptr;
    // Second branch of the step graph: PrepareEuler's interpolation of the momenta and energy runs
    // beside the density's inverse transform, and the x faces beside the y faces.  `cur` is the
    // stream the launch helper enqueues on (null = `stream`).
    cudaStream_t side = nullptr, side2 = nullptr;
    cudaStream_t cur = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
    // a finely profiled step keeps one stream: its per-kernel events time the launches in order
    bool fork_ok() const { return side && !fine; }
    void fork(cudaStream_t to)
    {
        cudaEventRecord(ev_fork, stream);
        cudaStreamWaitEvent(to, ev_fork, 0);
        cur = to;
    }
    void join(cudaStream_t from, cudaEvent_t ev)
    {
        cur = nullptr;
        cudaEventRecord(ev, from);
        cudaStreamWaitEvent(stream, ev, 0);
    }
    cudaGraphExec_t graph = nullptr;
    int launches = 0;
    int device = 0;
    int list_rows_blocks = 0;
    int face_blocks = 0;
    // Grid of a grid-stride phase kernel: at most two waves (16 CTAs of 256 threads per SM).  The
    // passes are short and latency-bound: fewer CTAs leave too few warps in flight (8 per SM:
    // +1.2 % step time, 4: +7 %), while the uncapped grids of up to 12k CTAs spend microseconds
    // per launch on block scheduling (+2.6 %; measured on the 2049^2 four-quadrant step).
#ifndef AWCM_PHASE_CTAS_PER_SM
#define AWCM_PHASE_CTAS_PER_SM 16
#endif
    unsigned pb(long n) const
    {
        return std::min(blocks_for(n, 256), (unsigned)(face_blocks / 8 * AWCM_PHASE_CTAS_PER_SM));
    }
    // Phase marks of a profiled step (null while capturing the graph).
    cudaEvent_t* prof_ev = nullptr;
    int prof_n = 0;
    void mark()
    {
        if (prof_ev) cudaEventRecord(prof_ev[prof_n++], stream);
    }
    // Per-launch marks of a finely profiled step: an event after every kernel.
    std::vector<std::pair<const char*, cudaEvent_t>>* fine = nullptr;
    void after(const char* name)
    {
        if (!fine) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, cur ? cur : stream);
        fine->emplace_back(name, e);
    }

    // Kernel launch on the instance's stream with programmatic stream serialisation (see
    // pdl_begin); `pdl` false gives plain launches.
    bool pdl = true;
    template <typename... P, typename... A>
    void launch(void (*kern)(P...), dim3 grid, dim3 block, A&&... args)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = 0;
        cfg.stream = cur ? cur : stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = pdl ? 1 : 0;
        cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
    }

    ~Solver2D() { release(); }

    void release()
    {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        auto fr = [](void* p) {
            if (p) cudaFree(p);
        };
        for (int k = 0; k < 4; ++k) {
            fr(q.p[k]);
            fr(q2.p[k]);
            fr(q1.p[k]);
            fr(fx.p[k]);
            fr(fy.p[k]);
            fr(qx.p[k]);
            fr(lvl[k]);
        }
        fr(m);
        for (int s = 0; s < kStages; ++s) {
            fr(ax[s]);
            fr(ay[s]);
        }
        fr(st);
        for (auto& l : lists) fr(l);
        fr(staging);
        fr(bcf_dev);
        bcf_dev = nullptr;
        free_adj();
        fr(tape);
        tape = nullptr;
        tape_steps = 0;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        if (side) cudaStreamDestroy(side);
        if (side2) cudaStreamDestroy(side2);
        side = side2 = nullptr;
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_join2) cudaEventDestroy(ev_join2);
        ev_fork = ev_join = ev_join2 = nullptr;
    }

    awcm2d_geometry geo{};

    int create(int num_levels, int nxc, int nyc, double x_min, double x_max, double y_min, double y_max, int bc)
    {
        if (num_levels < 2 || num_levels > kMaxLevels - 1 || nxc < 5 || nyc < 5) return kErrArg;
        // the generic manager (kind 4) is attached by set_bc_field
        if (bc < 0 || bc > 5 || bc == AWCM_BC_GENERIC) return kErrArg;
        geo = awcm2d_geometry{num_levels, nxc, nyc, bc, x_min, x_max, y_min, y_max, 1.4};
        const long nx = (long)(nxc - 1) * (1L << (num_levels - 1)) + 1;
        const long ny = (long)(nyc - 1) * (1L << (num_levels - 1)) + 1;
        const long pitch = ((nx + 2 * kGhost + 31) / 32) * 32;
        if ((pitch * (ny + 2 * kGhost)) >= (1L << 32)) return kErrArg;
        AWCM_CUDA_TRY(cudaGetDevice(&device));
        g.nx = (int)nx;
        g.ny = (int)ny;
        g.maxl = num_levels - 1;
        g.pitch = (int)pitch;
        g.rows = (int)(ny + 2 * kGhost);
        g.bc_kind = bc;
        g.x_min = x_min;
        g.y_min = y_min;
        g.dx = (x_max - x_min) / (nx - 1);
        g.dy = (y_max - y_min) / (ny - 1);
        g.gamma = 1.4;
        g.wz_eps = 1e-40;
        g.wz_delta = 0.0;
        g.bcf = nullptr;
        // BOUNDARY_MANAGER_WT's corner of the step, int(0.6/dx) and int(0.2/dy) (PROBLEM_WINDTUNNEL.h:75-76)
        g.wt_i = int(0.6 / g.dx);
        g.wt_j = int(0.2 / g.dy);
        if (bc == AWCM_BC_WIND_TUNNEL && (g.wt_i < 1 || g.wt_i + 2 > g.nx - 1 + kGhost || g.wt_j + 1 > g.ny - 1)) {
            set_last_error("wind tunnel: the step corner (0.6, 0.2) must lie inside the grid", __FILE__, __LINE__);
            return kErrArg;
        }
        g.W = make_weights();
        plane = (size_t)g.pitch * g.rows;
        AWCM_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        AWCM_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        AWCM_CUDA_TRY(cudaStreamCreateWithFlags(&side2, cudaStreamNonBlocking));
        AWCM_CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        AWCM_CUDA_TRY(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        AWCM_CUDA_TRY(cudaEventCreateWithFlags(&ev_join2, cudaEventDisableTiming));
        for (int k = 0; k < 4; ++k) {
            AWCM_CUDA_TRY(cudaMalloc(&q.p[k], plane * sizeof(double)));
            AWCM_CUDA_TRY(cudaMalloc(&q2.p[k], plane * sizeof(double)));
            AWCM_CUDA_TRY(cudaMalloc(&q1.p[k], plane * sizeof(double)));
            AWCM_CUDA_TRY(cudaMalloc(&fx.p[k], plane * sizeof(double)));
            AWCM_CUDA_TRY(cudaMalloc(&fy.p[k], plane * sizeof(double)));
            AWCM_CUDA_TRY(cudaMalloc(&lvl[k], plane));
            if (bc == AWCM_BC_WIND_TUNNEL) {
                AWCM_CUDA_TRY(cudaMalloc(&qx.p[k], plane * sizeof(double)));
                AWCM_CUDA_TRY(cudaMemsetAsync(qx.p[k], 0, plane * sizeof(double), stream));
            }
            AWCM_CUDA_TRY(cudaMemsetAsync(q.p[k], 0, plane * sizeof(double), stream));
            AWCM_CUDA_TRY(cudaMemsetAsync(q2.p[k], 0, plane * sizeof(double), stream));
            AWCM_CUDA_TRY(cudaMemsetAsync(q1.p[k], 0, plane * sizeof(double), stream));
            AWCM_CUDA_TRY(cudaMemsetAsync(fx.p[k], 0, plane * sizeof(double), stream));
            AWCM_CUDA_TRY(cudaMemsetAsync(fy.p[k], 0, plane * sizeof(double), stream));
        }
        AWCM_CUDA_TRY(cudaMalloc(&m, plane));
        for (int s = 0; s < kStages; ++s) {
            AWCM_CUDA_TRY(cudaMalloc(&ax[s], sizeof(double) * g.ny));
            AWCM_CUDA_TRY(cudaMalloc(&ay[s], sizeof(double) * g.nx));
        }
        AWCM_CUDA_TRY(cudaMalloc(&st, sizeof(StepState)));
        AWCM_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(StepState), stream));
        const size_t cap = (size_t)(g.nx + 2) * (g.ny + 2);
        for (auto& l : lists) AWCM_CUDA_TRY(cudaMalloc(&l, cap * sizeof(uint32_t)));
        // AWCM_2D's constructor: every mask byte all ones on the ghosts, mask0 true inside, all
        // levels at the finest level (Wavelet/AWCM_2D.h:26-41).
        launch(k_fill_u8, blocks_for((long)plane, 256), 256, m, plane, 0xff);
        for (int k = 0; k < 4; ++k) launch(k_fill_i8, blocks_for((long)plane, 256), 256, lvl[k], plane, (int8_t)g.maxl);
        AWCM_CUDA_TRY(cudaGetLastError());
        {
            // AWCM_2D's constructor (Wavelet/AWCM_2D.h:26-37): mask0 true on every point, ghosts
            // included; mask_temp and mask1..mask3 false everywhere.
            const size_t n = (size_t)(g.nx + 6) * (g.ny + 6);
            std::vector<uint8_t> planes(5 * n, 0);
            for (size_t t = 0; t < n; ++t) planes[n + t] = 1;
            int rc = set_masks(planes.data());
            if (rc) return rc;
        }
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
        face_blocks = dev_sms * 8;
        {
            int per_sm = 0;
            AWCM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_prepare, kPrepThreads, 0));
            int coop = 0;
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
            prep_blocks = (coop && per_sm > 0) ? dev_sms : 0;  // one CTA per SM; 0 = per-phase launches
        }
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int ensure_staging(size_t bytes)
    {
        if (bytes <= staging_bytes) return kOk;
        if (staging) cudaFree(staging);
        staging = nullptr;
        staging_bytes = 0;
        AWCM_CUDA_TRY(cudaMalloc(&staging, bytes));
        staging_bytes = bytes;
        return kOk;
    }

    size_t ghosted_points() const { return (size_t)(g.nx + 6) * (g.ny + 6); }

    int set_q(const double* host)
    {
        const size_t n = ghosted_points();
        int rc = ensure_staging(n * 4 * sizeof(double));
        if (rc) return rc;
        AWCM_CUDA_TRY(cudaMemcpyAsync(staging, host, n * 4 * sizeof(double), cudaMemcpyHostToDevice, stream));
        launch(k_aos_to_soa, blocks_for((long)n, 256), 256, g, (const double*)staging, q);
        AWCM_CUDA_TRY(cudaGetLastError());
        mark_full_zero();
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int get_q(double* host)
    {
        const size_t n = ghosted_points();
        int rc = ensure_staging(n * 4 * sizeof(double));
        if (rc) return rc;
        launch(k_soa_to_aos, blocks_for((long)n, 256), 256, g, q, (double*)staging);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaMemcpyAsync(host, staging, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int set_masks(const uint8_t* host)
    {
        const size_t n = ghosted_points();
        int rc = ensure_staging(5 * n);
        if (rc) return rc;
        AWCM_CUDA_TRY(cudaMemcpyAsync(staging, host, 5 * n, cudaMemcpyHostToDevice, stream));
        launch(k_pack_masks, blocks_for((long)n, 256), 256, g, (const uint8_t*)staging, m);
        AWCM_CUDA_TRY(cudaGetLastError());
        mark_full_zero();
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int get_masks(uint8_t* host)
    {
        const size_t n = ghosted_points();
        int rc = ensure_staging(5 * n);
        if (rc) return rc;
        launch(k_unpack_masks, blocks_for((long)n, 256), 256, g, m, (uint8_t*)staging);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaMemcpyAsync(host, staging, 5 * n, cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int set_levels(const int* host)
    {
        const size_t n = (size_t)g.nx * g.ny;
        int rc = ensure_staging(4 * n * sizeof(int));
        if (rc) return rc;
        AWCM_CUDA_TRY(cudaMemcpyAsync(staging, host, 4 * n * sizeof(int), cudaMemcpyHostToDevice, stream));
        launch(k_levels_in, blocks_for((long)n, 256), 256, g, (const int*)staging, lvl[0], lvl[1], lvl[2], lvl[3]);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int get_levels(int* host)
    {
        const size_t n = (size_t)g.nx * g.ny;
        int rc = ensure_staging(4 * n * sizeof(int));
        if (rc) return rc;
        launch(k_levels_out, blocks_for((long)n, 256), 256, g, lvl[0], lvl[1], lvl[2], lvl[3], (int*)staging);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaMemcpyAsync(host, staging, 4 * n * sizeof(int), cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    void mark_full_zero()
    {
        // After an external write (or a frozen run) the invariant of the sparse residue removal and
        // of the sparse inverse-transform zeroing (values only inside mask3 or the previous mask0)
        // is not known to hold: the next step zeroes densely.
        const int one = 1;
        cudaMemcpyAsync(&st->full_zero, &one, sizeof(int), cudaMemcpyHostToDevice, stream);
    }

    // ---------------------------------------------------------------- enqueue helpers
    long grid_points() const { return (long)g.nx * g.ny; }
    // Threads of a ghost fill: the four edge strips and the four corner blocks (the corners are
    // filled by the generic manager only).
    long bc_threads() const { return 2L * kGhost * g.ny + 2L * kGhost * g.nx + 4L * kGhost * kGhost; }
    long words() const { return (long)(plane / 4); }  // 32-bit words of a mask/level plane

    long band_count(int lev, int which) const
    {
        const Band b = band_of(g, lev, which);
        return (long)b.cx * b.cy;
    }
    long details(int lev) const { return band_count(lev, 0) + band_count(lev, 1) + band_count(lev, 2); }

    // Fine levels (point spacing <= kRowScanMaxH) scan mask words row by row and skip empty words;
    // coarser levels enumerate their sub-band points.
    bool row_scan(int lev) const { return (g.D(lev) >> 1) <= kRowScanMaxH; }
    long rowscan_threads(int lev, int rows) const
    {
        const int h = g.D(lev) >> 1;
        const long nr = (g.ny - 1) / h + 1, wpr = g.pitch / 4;
        return (rows == 2 ? nr : (rows == 0 ? (nr + 1) / 2 : nr / 2)) * wpr;
    }

    void enq_cr(int bit, const StepState* s)
    {
        for (int lev = g.maxl - 1; lev >= 0; --lev) {
            if (row_scan(lev)) {
                launch(k_cr_rows, pb(rowscan_threads(lev, 2)), 256, g, m, lev, bit, s);
                after("k_cr_rows");
            } else {
                launch(k_cr, pb(details(lev)), 256, g, m, lev, bit, s);
                after("k_cr");
            }
            launches += 1;
        }
    }

    // The forward transform's scratch plane is the first x-face flux plane (faces are not live
    // during PrepareEuler).
    // idle: kBitTemp holds mask0 (PrepareEuler's first pass copied it), so the points outside it
    // skip the staging plane.
    void enq_fwt(const StepState* s, bool idle = false)
    {
        const int id = idle ? 1 : 0;
        for (int lev = g.maxl - 1; lev >= 0; --lev) {
            launch(k_fwt_a, pb(details(lev)), 256, g, q.p[0], fx.p[0], m, lev, id, s);
            after("k_fwt_a");
            const long nb = band_count(lev, 3) + band_count(lev, 0) + band_count(lev, 1);
            launch(k_fwt_b, pb(nb), 256, g, q.p[0], fx.p[0], m, lev, id, s);
            after("k_fwt_b");
            launches += 2;
        }
    }

    // init_from >= 0: the first launch also builds the work mask of the interpolation that follows
    // (ph_interp_init from init_from to bit), which the inverse transform does not read.
    // sparse: in PrepareEuler (mask_temp = the starting mask0), see ph_iwt.
    void enq_iwt(int bit, const StepState* s, int init_from = -1, bool sparse = false)
    {
        const int sp = sparse ? 1 : 0;
        for (int lev = 0; lev < g.maxl; ++lev) {
            const Band b3 = band_of(g, lev, 2), b1 = band_of(g, lev, 0), b2 = band_of(g, lev, 1), bc = band_of(g, lev, 3);
            if (lev == 0 && init_from >= 0) {
                const unsigned nb = pb((long)bc.cx * bc.cy);
                launch(k_iwt0_interp_init, nb + pb(words()), 256, g, q.p[0], m, lev, bit, init_from, sp, s, nb);
                after("k_iwt0_interp_init");
            } else {
                launch(k_iwt<0>, pb((long)bc.cx * bc.cy), 256, g, q.p[0], m, lev, bit, sp, s);
                after("k_iwt<0>");
            }
            launch(k_iwt<1>, pb((long)b1.cx * b1.cy + (long)b2.cx * b2.cy), 256, g, q.p[0], m, lev, bit, sp, s);
            after("k_iwt<1>");
            launch(k_iwt<2>, pb((long)b3.cx * b3.cy), 256, g, q.p[0], m, lev, bit, sp, s);
            after("k_iwt<2>");
            launches += 3;
        }
    }

    // init_done: the work mask was built by the inverse transform's first launch.
    void enq_interp(int from, int to, const StepState* s, int p0 = 1, bool init_done = false)
    {
        if (!init_done) {
            launch(k_interp_init, pb(words()), 256, g, m, from, to, s);
            after("k_interp_init");
            launches += 1;
        }
        enq_cr(kBitInterp, s);
        for (int lev = 0; lev < g.maxl; ++lev) {
            if (row_scan(lev)) {
                launch(k_interp_rows<0>, pb(rowscan_threads(lev, 2)), 256, g, q, m, lev, from, p0, s);
                after("k_interp_rows<0>");
                launch(k_interp_rows<1>, pb(rowscan_threads(lev, 1)), 256, g, q, m, lev, from, p0, s);
                after("k_interp_rows<1>");
            } else {
                launch(k_interp<0>, pb(band_count(lev, 0) + band_count(lev, 1)), 256, g, q, m, lev, from, p0, s);
                after("k_interp<0>");
                launch(k_interp<1>, pb(band_count(lev, 2)), 256, g, q, m, lev, from, p0, s);
                after("k_interp<1>");
            }
            launches += 2;
        }
    }

    void enq_aaz(int bit, const StepState* s)
    {
        launch(k_copy_bit_all, pb(words()), 256, m, plane, bit, kBitCopy, s, 0u);
        after("k_copy_bit_all");
        launch(k_aaz, pb(words()), 256, g, m, bit, kBitCopy, s);
        after("k_aaz");
        launches += 2;
    }

    // AWCM_2D::PrepareEuler (Wavelet/AWCM_2D.h:114-147): one launch per phase (prep_mode 1, the
    // default: the phases are latency-bound and run at full occupancy as separate kernels), or
    // (prep_mode 0) the persistent cooperative kernel with grid barriers.
    int prep_mode = 1;
    int prep_blocks = 0;
    // Scalar AWCM instance (Wavelet/main_2d_advect.cpp): plane 0 of q, q2, q1 carries the field.
    bool scalar = false;

    // Worklists of the step's three stages and the mask counts; with_dt also computes dt (from the
    // CFL speed, so after the stage-1 scan).
    void enq_lists(int with_dt)
    {
        ListArgs la;
        for (int L = 0; L < kNumLists; ++L) la.list[L] = lists[L];
        la.zx1 = ax[1];
        la.zy1 = ay[1];
        la.zx2 = ax[2];
        la.zy2 = ay[2];
        la.with_dt = with_dt;
        dim3 grid((g.nx + 1 + 255) / 256, (g.ny + 1 + kListRows - 1) / kListRows);
        launch(k_lists, grid, 256, g, m, lvl[2], lvl[1], lvl[0], la, st);
        after("k_lists");
        launches += 1;
    }

    // lists: the step's worklists are built too (without dt), as soon as the masks and levels are
    // final.
    void enq_prepare(const StepState* s, bool lists = false)
    {
        if (prep_mode == 0 && s == st && prep_blocks > 0) {
            PrepArgs A;
            A.g = g;
            A.q = q;
            A.tb = fx.p[0];
            A.m = m;
            for (int k = 0; k < 4; ++k) A.lvl[k] = lvl[k];
            A.st = st;
            A.sync = st->bar;
            A.err = &st->bar_err;
            A.plane = plane;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(prep_blocks);
            cfg.blockDim = dim3(kPrepThreads);
            cfg.stream = stream;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            cudaLaunchKernelEx(&cfg, k_prepare, A);
            after("k_prepare");
            launches += 1;
            if (lists) enq_lists(0);
            return;
        }
        // mask_temp = mask0; also clears mask1..3, which the merged ComputeLevel +
        // AddPointForDifferentiation passes below rebuild by ORs
        if (!scalar) launch(k_copy_bit_all, pb(words()), 256, m, plane, 0, kBitTemp, s, kMask123);
        after("k_copy_bit_all");
        launches += 1;
        enq_fwt(s, !scalar);
        launch(k_band_copy, pb(words()), 256, g, m, 0, kBitCopy, s);
        after("k_band_copy");
        launch(k_aaz, pb(words()), 256, g, m, 0, kBitCopy, s);
        after("k_aaz");
        launches += 2;
        enq_cr(0, s);
        for (int k = 1; k <= 3; ++k) {
            if (!scalar) {
                launch(k_cl_apd, pb(words()), 256, g, m, lvl[k - 1], k, plane, s);
                after("k_cl_apd");
                launches += 1;
            } else {
                launch(k_cl, pb(words()), 256, g, m, lvl[k - 1], k - 1, k, plane, s);
                after("k_cl");
                launch(k_apd, pb(words()), 256, g, m, lvl[k - 1], k, k - 1, s);
                after("k_apd");
                launches += 2;
            }
            enq_cr(k, s);
        }
        // AWCM_2D::Prepare (the scalar form, Wavelet/AWCM_2D.h:52-79) ends with the inverse transform
        if (scalar) {
            enq_iwt(3, s);
            if (lists) enq_lists(0);
        } else if (!fork_ok()) {
            enq_iwt(3, s, kBitTemp, true);
            enq_interp(kBitTemp, 3, s, 1, true);
            if (lists) enq_lists(0);
        } else {
            // The inverse transform writes the density only and reads mask3; the interpolation
            // reads and writes components 1..3 and the interpolation work bit; the worklist build
            // reads the mask bits 0..3 and the level planes and writes the lists: disjoint, so the
            // three run as parallel branches of the graph.
            cudaEventRecord(ev_fork, stream);
            cudaStreamWaitEvent(side, ev_fork, 0);
            if (lists) cudaStreamWaitEvent(side2, ev_fork, 0);
            cur = side;
            enq_interp(kBitTemp, 3, s, 1, false);
            if (lists) {
                cur = side2;
                enq_lists(0);
            }
            cur = nullptr;
            enq_iwt(3, s, -1, true);
            join(side, ev_join);
            if (lists) join(side2, ev_join2);
        }
    }

    // Boundary fill of a stage input; with zero_stage >= 0 it also zeroes that stage's LF-speed
    // accumulators for the k_alpha that follows.
    void enq_bc(Field4 f, const StepState* s, int zero_stage = -1, double* zx_in = nullptr, double* zy_in = nullptr)
    {
        const long n = bc_threads();
        double* zx = zx_in ? zx_in : (zero_stage >= 0 ? ax[zero_stage] : nullptr);
        double* zy = zy_in ? zy_in : (zero_stage >= 0 ? ay[zero_stage] : nullptr);
        launch(k_bc, blocks_for(n, 256), 256, g, f, s, 0.0, zx, zy);
        after("k_bc");
        launches += 1;
    }

    // Accumulates into ax[stage] / ay[stage], or into (axp, ayp) when given; the accumulators were
    // zeroed by the boundary fill before this launch.
    void enq_alpha(Field4 f, int bit, int stage, bool with_cfl, double* axp = nullptr, double* ayp = nullptr)
    {
        dim3 grid((unsigned)(g.pitch / 4 + 31) / 32, (unsigned)(g.ny + 8 * kAlphaRows - 1) / (8 * kAlphaRows));
        launch(k_alpha, grid, 256, g, f, m, bit, axp ? axp : ax[stage], ayp ? ayp : ay[stage],
               with_cfl ? &st->mv : nullptr, st, with_cfl ? &st->nonfinite : nullptr);
        after("k_alpha");
        launches += 1;
    }
    // Boundary fill of stage `stage`'s input (1 or 2) and its LF speeds over the previous stage's
    // update lists, in one launch; the speeds' accumulators are zeroed by k_lists.
    void enq_bc_alpha(Field4 f, int stage)
    {
        const int ls = stage - 1;
        const unsigned* C = st->cnt + 4 * ls;
        const unsigned bcb = blocks_for(bc_threads(), 256);
        launch(k_bc_alpha, bcb + face_blocks / 2, 256, g, f, lists[4 * ls], C, lists[4 * ls + 1], C + 1, ax[stage],
               ay[stage], st, bcb, &st->nonfinite);
        after("k_bc_alpha");
        launches += 1;
    }
    // Stage `stage` (1 or 2) over the points of the previous stage's update lists (its mask).
    void enq_alpha_listed(Field4 f, int stage, double* axp = nullptr, double* ayp = nullptr, int* nonfinite = nullptr)
    {
        const int ls = stage - 1;
        const unsigned* C = st->cnt + 4 * ls;
        launch(k_alpha_list, face_blocks / 2, 256, g, f, lists[4 * ls], C, lists[4 * ls + 1], C + 1,
               axp ? axp : ax[stage], ayp ? ayp : ay[stage], st, nonfinite);
        after("k_alpha_list");
        launches += 1;
    }

    // The field the x-direction fluxes of a stage read: the wind tunnel's x-sweep copy, else the input.
    Field4 xin(Field4 in) const { return g.bc_kind == AWCM_BC_WIND_TUNNEL ? qx : in; }

    // The wind tunnel's stage input after its standard fill: the x-sweep copy qx with the
    // x-direction bottom fill, and the input itself with the x- and then the y-direction one
    // (BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition, Problems/2D/PROBLEM_WINDTUNNEL.h:124-168).
    void enq_wt_input(Field4 f)
    {
        launch(k_copy4, pb((long)plane), 256, qx, f, plane);
        after("k_copy4");
        launch(k_wt_bottom_x, blocks_for(2L * 3 * (g.wt_j + kGhost + 1), 256), 256, g, f, qx, (const StepState*)st);
        after("k_wt_bottom_x");
        const long ny0 = 3L * (g.nx + 2 * kGhost - 1), ny1 = 3L * (g.nx - 1 + kGhost - g.wt_i + 1);
        launch(k_wt_bottom_y, blocks_for(ny0, 256), 256, g, f, 0, (const StepState*)st);
        after("k_wt_bottom_y");
        launch(k_wt_bottom_y, blocks_for(ny1, 256), 256, g, f, 1, (const StepState*)st);
        after("k_wt_bottom_y");
        launches += 4;
    }

    // Face fluxes and point updates of one stage; the LF speeds come from ax[stage] / ay[stage],
    // or from (axp, ayp) when given.
    void enq_faces_update(int stage, Field4 in, Field4 out, const double* axp = nullptr, const double* ayp = nullptr,
                          bool with_dt = false)
    {
        StepState* dts = with_dt ? st : nullptr;
        uint32_t* const* L = lists + 4 * stage;
        const unsigned* C = st->cnt + 4 * stage;
        const double* sx = axp ? axp : ax[stage];
        // face kernels: 16 CTAs of 128 per SM over the face list (4 resident, so four waves); 8 or 4
        // per SM measured 1.3 % and 7 % slower faces
        const double* sy = ayp ? ayp : ay[stage];
        mark();
        // the x faces (fx) and the y faces (fy) read the same stage input: parallel branches
        const bool par = fork_ok();
        if (par) fork(side);
        if (g.wz_eps == 1e-40 && g.wz_delta == 0.0)
            launch(k_face<0, false>, 2 * face_blocks, 128, g, xin(in), fx, L[2], C + 2, sx, st, (StepState*)nullptr);
        else
            launch(k_face<0, true>, 2 * face_blocks, 128, g, xin(in), fx, L[2], C + 2, sx, st, (StepState*)nullptr);
        after("k_face<0>");
        cur = nullptr;
        if (g.wz_eps == 1e-40 && g.wz_delta == 0.0)
            launch(k_face<1, false>, 2 * face_blocks, 128, g, in, fy, L[3], C + 3, sy, st, dts);
        else
            launch(k_face<1, true>, 2 * face_blocks, 128, g, in, fy, L[3], C + 3, sy, st, dts);
        after("k_face<1>");
        if (par) join(side, ev_join);
        launches += 2;
        mark();
        const int ub = face_blocks / 2;
        if (stage == 0) {
            launch(k_update<1>, ub, 256, g, in, xin(in), out, q, fx, fy, lvl[2], L[0], C + 0, L[1], C + 1, st);
            after("k_update<1>");
        } else if (stage == 1) {
            launch(k_update<2>, ub, 256, g, in, xin(in), out, q, fx, fy, lvl[1], L[0], C + 0, L[1], C + 1, st);
            after("k_update<2>");
        } else {
            launch(k_update<3>, ub, 256, g, in, xin(in), out, q, fx, fy, lvl[0], L[0], C + 0, L[1], C + 1, st);
            after("k_update<3>");
        }
        launches += 1;
        mark();
    }

    // One pass of the driver loop (main_2d_euler(quad).cpp:58-334).
    void enq_step()
    {
        launches = 0;
        mark();
        launch(k_begin, 1, 1, st, 0);
        after("k_begin");
        launches += 1;
        // the worklists (and the zeroing of stage 2/3's speed accumulators) are built beside the
        // last PrepareEuler passes; dt is computed by the first stage's y-face launch
        enq_prepare(st, true);
        mark();
        const bool wt = g.bc_kind == AWCM_BC_WIND_TUNNEL;
        enq_bc(q, st, 0);
        // The wind tunnel's bottom fills write solid cells of mask3 that PrepareEuler leaves in
        // non-physical states, so the CFL scan (with the LF speeds) reads the filled stage input;
        // the other managers write ghost cells only, outside the scan.
        if (wt) enq_wt_input(q);
        enq_alpha(q, 3, 0, true);
        enq_faces_update(0, q, q2, nullptr, nullptr, true);
        // RemoveResidue zeroes q off mask0.  After the second stage's update (the last reader of q
        // off mask0: its combination reads q on mask1) nothing else touches those points: the third
        // stage reads q1 and reads and writes q on mask0 only.  So it runs as a graph branch beside
        // the third stage.
        const bool rr_par = fork_ok() && side2;
        for (int stage = 1; stage <= 2; ++stage) {
            Field4 in = stage == 1 ? q2 : q1;
            if (stage == 2 && rr_par) {
                cudaEventRecord(ev_fork, stream);
                cudaStreamWaitEvent(side2, ev_fork, 0);
                cur = side2;
                launch(k_remove_residue, pb(words()), 256, g, q, m, 0, 1, st);
                after("k_remove_residue");
                cur = nullptr;
            }
            if (!wt) {
                enq_bc_alpha(in, stage);
            } else {
                // the wind tunnel's bottom fills write interior (solid) cells the speeds read
                enq_bc(in, st);
                enq_wt_input(in);
                enq_alpha_listed(in, stage, nullptr, nullptr, &st->nonfinite);
            }
            enq_faces_update(stage, in, q1);
        }
        if (rr_par) {
            join(side2, ev_join2);
        } else {
            launch(k_remove_residue, pb(words()), 256, g, q, m, 0, 1, st);
            after("k_remove_residue");
        }
        launch(k_finish, 1, 1, st);
        after("k_finish");
        launches += 2;
        mark();
    }

    // One pass of the scalar driver loop (Wavelet/main_2d_advect.cpp:48-190): Prepare (no
    // interpolation), periodic fill, three SSP-RK3 stages at the fixed dt with WENO5 upwind faces
    // on the finest level and central differences below, PostProcess.
    static Field4 alias(double* p) { return Field4{{p, p, p, p}}; }
    void enq_stage_scalar(int stage, const double* in, double* out)
    {
        uint32_t* const* L = lists + 4 * stage;
        const unsigned* C = st->cnt + 4 * stage;
        launch(k_face_scalar<0>, face_blocks, 256, g, in, fx.p[0], L[2], C + 2, st);
        after("k_face_scalar<0>");
        launch(k_face_scalar<1>, face_blocks, 256, g, in, fy.p[0], L[3], C + 3, st);
        after("k_face_scalar<1>");
        const int ub = face_blocks / 2;
        double* qn = q.p[0];
        if (stage == 0) {
            launch(k_update_fin_scalar<1>, ub, 256, g, in, out, qn, fx.p[0], fy.p[0], L[0], C + 0, st);
            launch(k_update_crs_scalar<1>, ub, 256, g, in, out, qn, lvl[2], L[1], C + 1, st);
        } else if (stage == 1) {
            launch(k_update_fin_scalar<2>, ub, 256, g, in, out, qn, fx.p[0], fy.p[0], L[0], C + 0, st);
            launch(k_update_crs_scalar<2>, ub, 256, g, in, out, qn, lvl[1], L[1], C + 1, st);
        } else {
            launch(k_update_fin_scalar<4>, ub, 256, g, in, out, qn, fx.p[0], fy.p[0], L[0], C + 0, st);
            launch(k_update_crs_scalar<4>, ub, 256, g, in, out, qn, lvl[0], L[1], C + 1, st);
        }
        after("k_update_scalar");
        launches += 4;
    }

    void enq_step_scalar()
    {
        launches = 0;
        launch(k_begin, 1, 1, st, 0);
        launches += 1;
        enq_prepare(st);
        enq_bc(alias(q.p[0]), st);
        launch(k_dt, 1, 1, g, st);
        {
            ListArgs la;
            for (int L = 0; L < kNumLists; ++L) la.list[L] = lists[L];
            dim3 grid((g.nx + 1 + 255) / 256, (g.ny + 1 + kListRows - 1) / kListRows);
            launch(k_lists, grid, 256, g, m, lvl[2], lvl[1], lvl[0], la, st);
        }
        launches += 2;
        enq_stage_scalar(0, q.p[0], q2.p[0]);
        enq_bc(alias(q2.p[0]), st);
        enq_stage_scalar(1, q2.p[0], q1.p[0]);
        enq_bc(alias(q1.p[0]), st);
        enq_stage_scalar(2, q1.p[0], q1.p[0]);
        launch(k_remove_residue, pb(words()), 256, g, q, m, 0, 1, st);
        launch(k_finish, 1, 1, st);
        launches += 2;
    }

    int build_graph()
    {
        if (graph) return kOk;
        cudaGraph_t gr;
        AWCM_CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        if (scalar) enq_step_scalar();
        else enq_step();
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

    int write_params(double tol, double cfl, double t, double t_end, double dt_fixed)
    {
        StepState h;
        AWCM_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(StepState), cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        h.tol = tol;
        h.cfl = cfl;
        h.t = t;
        h.t_end = t_end;
        h.dt_fixed = dt_fixed;
        h.done = 0;
        h.error = 0;
        h.bar_err = 0;
        h.nonfinite = 0;
        h.bar[0] = 0;
        AWCM_CUDA_TRY(cudaMemcpyAsync(st, &h, sizeof(StepState), cudaMemcpyHostToDevice, stream));
        return kOk;
    }

    // Status of a run whose device-side error word is set, with its text.
    static int report_error(const StepState& h)
    {
        if (h.error == kErrNonFinite) {
            char msg[200];
            std::snprintf(msg, sizeof(msg),
                          "non-finite state: a CFL or Lax-Friedrichs wave speed was NaN or infinite in the "
                          "step ending at t = %.17g (NaN/Inf values, negative pressure or density)",
                          h.t);
            set_last_error(msg, __FILE__, __LINE__);
        } else {
            set_last_error("grid barrier wait ran out in the prepare kernel", __FILE__, __LINE__);
        }
        return h.error;
    }

    // Test-only: polls before a grid-barrier wait of the persistent prepare kernel gives up
    // (0 restores the default).
    int set_spin_limit(unsigned polls)
    {
        StepState h;
        int rc = read_state(&h);
        if (rc) return rc;
        h.spin_limit = polls;
        AWCM_CUDA_TRY(cudaMemcpyAsync(st, &h, sizeof(StepState), cudaMemcpyHostToDevice, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int read_state(StepState* h)
    {
        AWCM_CUDA_TRY(cudaMemcpyAsync(h, st, sizeof(StepState), cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int step(double tol, double cfl, double t, double t_next, double dt_fixed, double* out)
    {
        int rc = build_graph();
        if (rc) return rc;
        rc = write_params(tol, cfl, t, t_next, dt_fixed);
        if (rc) return rc;
        AWCM_CUDA_TRY(cudaGraphLaunch(graph, stream));
        StepState h;
        rc = read_state(&h);
        if (rc) return rc;
        if (h.error) return report_error(h);
        if (out) {
            out[0] = h.dt;
            out[1] = h.do_print;
            for (int k = 0; k < 4; ++k) out[2 + k] = h.mask_cnt[k];
            out[6] = h.mv;
            out[7] = 0;
        }
        return kOk;
    }

    int advance(double tol, double cfl, double t_start, double t_end, int n_steps, double* out)
    {
        int rc = build_graph();
        if (rc) return rc;
        rc = write_params(tol, cfl, t_start, t_end, 0.0);
        if (rc) return rc;
        StepState h0;
        rc = read_state(&h0);
        if (rc) return rc;
        for (int s = 0; s < n_steps; ++s) AWCM_CUDA_TRY(cudaGraphLaunch(graph, stream));
        StepState h;
        rc = read_state(&h);
        if (rc) return rc;
        if (h.error) return report_error(h);
        if (out) {
            out[0] = h.t;
            out[1] = h.steps - h0.steps;
            out[2] = (double)(h.upd - h0.upd);
            out[3] = (double)(h.stage_pts - h0.stage_pts);
        }
        return kOk;
    }

    // One step with the same kernels launched eagerly and CUDA events at the phase boundaries.
    // out[0] prepare ms (with the worklist build beside its last passes), [1] boundary fill and
    // CFL/LF speeds ms, [2..4] face kernels ms per stage,
    // [5..7] point-update kernels ms per stage, [8] boundary fills + LF speeds of stages 2-3 ms,
    // [9] residue removal ms, [10] total ms, [11..13] faces per stage, [14..16] stage points,
    // [17] |mask0|, [18] dt.
    int profile_step(double tol, double cfl, double t, double t_end, double* out)
    {
        int rc = write_params(tol, cfl, t, t_end, 0.0);
        if (rc) return rc;
        cudaEvent_t ev[16];
        for (auto& e : ev) AWCM_CUDA_TRY(cudaEventCreate(&e));
        prof_ev = ev;
        prof_n = 0;
        enq_step();
        prof_ev = nullptr;
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        // marks: 0 start, 1 after prepare, then per stage (faces begin, faces end, updates end), last = end
        float ms[16] = {};
        for (int k = 1; k < prof_n; ++k) cudaEventElapsedTime(&ms[k], ev[k - 1], ev[k]);
        out[0] = ms[1];
        out[1] = ms[2];  // mark 2 = faces begin of stage 0
        double between = 0;
        for (int s2 = 0; s2 < kStages; ++s2) {
            out[2 + s2] = ms[3 + 3 * s2];
            out[5 + s2] = ms[4 + 3 * s2];
            if (s2 > 0) between += ms[2 + 3 * s2];
        }
        out[8] = between;
        out[9] = ms[prof_n - 1];
        float tot = 0;
        cudaEventElapsedTime(&tot, ev[0], ev[prof_n - 1]);
        out[10] = tot;
        StepState h;
        rc = read_state(&h);
        for (auto& e : ev) cudaEventDestroy(e);
        if (rc) return rc;
        for (int s2 = 0; s2 < kStages; ++s2) {
            out[11 + s2] = (double)h.cnt[4 * s2 + 2] + h.cnt[4 * s2 + 3];
            out[14 + s2] = (double)h.cnt[4 * s2 + 0] + h.cnt[4 * s2 + 1];
        }
        out[17] = h.mask_cnt[0];
        out[18] = h.dt;
        return kOk;
    }

    // One step with an event after every kernel: per-launch device times (ms) in launch order.
    int profile_fine(double tol, double cfl, double t, double t_end, std::vector<std::pair<const char*, float>>& out)
    {
        int rc = write_params(tol, cfl, t, t_end, 0.0);
        if (rc) return rc;
        std::vector<std::pair<const char*, cudaEvent_t>> evs;
        cudaEvent_t e0;
        cudaEventCreate(&e0);
        cudaEventRecord(e0, stream);
        fine = &evs;
        enq_step();
        fine = nullptr;
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        cudaEvent_t prev = e0;
        out.clear();
        for (auto& pe : evs) {
            float ms = 0;
            cudaEventElapsedTime(&ms, prev, pe.second);
            out.emplace_back(pe.first, ms);
            prev = pe.second;
        }
        for (auto& pe : evs) cudaEventDestroy(pe.second);
        cudaEventDestroy(e0);
        return kOk;
    }

    int prepare(double tol)
    {
        int rc = write_params(tol, 0, 0, 1, 0);
        if (rc) return rc;
        launch(k_begin, 1, 1, st, 0);
        enq_prepare(st);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int fwt(double tol)
    {
        int rc = write_params(tol, 0, 0, 1, 0);
        if (rc) return rc;
        launch(k_begin, 1, 1, st, 0);
        enq_fwt(st);
        mark_full_zero();  // standalone passes: the next step zeroes densely
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    static int bit_of(int mask_id) { return mask_id >= 0 && mask_id <= 3 ? mask_id : kBitTemp; }

    int iwt(int mask_id)
    {
        enq_iwt(bit_of(mask_id), nullptr);
        mark_full_zero();
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    int interpolate(int from_id, int to_id)
    {
        enq_interp(bit_of(from_id), bit_of(to_id), nullptr);
        mark_full_zero();
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    // WAVELET_2D::InterpolateAllGridEuler (Wavelet/WAVELET_2D.h:912-1044): every grid point outside
    // mask `from_id` gets all four components interpolated, coarse to fine, from the active ones:
    // the dense field.  Same work mask (all points minus `from`, closed by CheckReconstruction) and
    // the same interpolation bodies as InterpolateEuler, with density included.  The field then
    // holds values off mask0, so the next step zeroes densely.
    int interpolate_all(int from_id)
    {
        enq_interp(bit_of(from_id), -1, nullptr, 0);
        AWCM_CUDA_TRY(cudaGetLastError());
        mark_full_zero();
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    // Scalar field in the reference's FIELD_UNIFORM_2D<double> layout ((Ny+6) x (Nx+6) doubles).
    int scalar_set_q(const double* host)
    {
        const size_t w = (size_t)g.nx + 2 * kGhost;
        AWCM_CUDA_TRY(cudaMemcpy2DAsync(q.p[0], (size_t)g.pitch * sizeof(double), host, w * sizeof(double),
                                        w * sizeof(double), (size_t)g.rows, cudaMemcpyHostToDevice, stream));
        mark_full_zero();
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }
    int scalar_get_q(double* host)
    {
        const size_t w = (size_t)g.nx + 2 * kGhost;
        AWCM_CUDA_TRY(cudaMemcpy2DAsync(host, w * sizeof(double), q.p[0], (size_t)g.pitch * sizeof(double),
                                        w * sizeof(double), (size_t)g.rows, cudaMemcpyDeviceToHost, stream));
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }
    // n scalar steps at the fixed dt from t (graph replays); out[3]: t, steps, sum |mask0|.
    int scalar_advance(double tol, double dt, double t, int n, double* out)
    {
        if (!(dt > 0) || n < 0) return kErrArg;
        int rc = build_graph();
        if (rc) return rc;
        if ((rc = write_params(tol, 1.0, t, 1e300, dt))) return rc;
        StepState h0;
        if ((rc = read_state(&h0))) return rc;
        for (int k = 0; k < n; ++k) AWCM_CUDA_TRY(cudaGraphLaunch(graph, stream));
        StepState h;
        if ((rc = read_state(&h))) return rc;
        if (out) {
            out[0] = h.t;
            out[1] = h.steps - h0.steps;
            out[2] = (double)(h.upd - h0.upd);
        }
        return kOk;
    }

    int manager(int op, int mask_id, int level_id)
    {
        const int b = bit_of(mask_id);
        if (level_id < 0 || level_id > 3) return kErrArg;
        mark_full_zero();
        switch (op) {
            case 0: enq_aaz(b, nullptr); break;
            case 1: enq_cr(b, nullptr); break;
            case 2:
                launch(k_copy_bit_all, pb(words()), 256, m, plane, b, kBitCopy, nullptr, 0u);
                launch(k_apd, pb(words()), 256, g, m, lvl[level_id], b, kBitCopy, nullptr);
                break;
            case 3: launch(k_cl, pb(words()), 256, g, m, lvl[level_id], b, -1, plane, nullptr); break;
            case 4: launch(k_remove_residue, pb(words()), 256, g, q, m, b, 0, nullptr); break;
            case 5: launch(k_band_copy, pb(words()), 256, g, m, b, -1, nullptr); break;
            default: return kErrArg;
        }
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    // BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition(x_direction, y_direction) on the conserved field.
    int wt_bottom(int x_direction, int y_direction)
    {
        if (g.bc_kind != AWCM_BC_WIND_TUNNEL || (x_direction != 0) == (y_direction != 0)) {
            set_last_error("SetBottomBoundaryCondition: a wind-tunnel instance and exactly one direction", __FILE__,
                           __LINE__);
            return kErrArg;
        }
        if (x_direction) {
            launch(k_wt_bottom_x, blocks_for(3L * (g.wt_j + kGhost + 1), 256), 256, g, q, Field4{},
                   (const StepState*)nullptr);
        } else {
            launch(k_wt_bottom_y, blocks_for(3L * (g.nx + 2 * kGhost - 1), 256), 256, g, q, 0, (const StepState*)nullptr);
            launch(k_wt_bottom_y, blocks_for(3L * (g.nx - 1 + kGhost - g.wt_i + 1), 256), 256, g, q, 1,
                   (const StepState*)nullptr);
        }
        mark_full_zero();  // writes interior (solid) cells
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    // Attaches the enum-driven manager: bc holds (Ny+6) x (Nx+6) BOUNDARY_CONDITION values in the
    // FIELD_UNIFORM_2D layout; every later ghost fill of this instance applies it.
    int set_bc_field(const int* bc)
    {
        const int w = g.nx + 6;
        std::vector<int8_t> plane(this->plane, 0);
        for (int j = -kGhost; j < g.ny + kGhost; ++j)
            for (int i = -kGhost; i < g.nx + kGhost; ++i) {
                const int v = bc[(size_t)(j + kGhost) * w + (i + kGhost)];
                if (v < -4 || v > 0) {
                    set_last_error("BOUNDARY_CONDITION values are -4 (SOLID_WALL) .. 0 (FLUID)", __FILE__, __LINE__);
                    return kErrArg;
                }
                plane[g.at(i, j)] = (int8_t)v;
            }
        if (!bcf_dev) AWCM_CUDA_TRY(cudaMalloc(&bcf_dev, this->plane));
        AWCM_CUDA_TRY(cudaMemcpy(bcf_dev, plane.data(), this->plane, cudaMemcpyHostToDevice));
        g.bcf = bcf_dev;
        g.bc_kind = AWCM_BC_GENERIC;
        geo.bc_kind = AWCM_BC_GENERIC;
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        return kOk;
    }

    int apply_bc(double t)
    {
        const long n = bc_threads();
        launch(k_bc, blocks_for(n, 256), 256, g, q, nullptr, t, nullptr, nullptr);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }

    // ---------------------------------------------------------- frozen-mask run and its adjoint
    // Frozen-mask step (the gradient configuration): the driver loop of main_2d_euler(quad).cpp
    // without PrepareEuler and without residue removal, at a fixed dt, on the masks and levels of
    // the last PrepareEuler.  The per-stage LF speeds are computed (and written to `tout` when
    // given) or, with `tin`, replayed; tape layout per step: stage 0..2 x (alpha_x[Ny], alpha_y[Nx]).
    // With `save`, the three stage inputs after their boundary fill (Q, Q2, Q1) are copied out.
    size_t tape_stride() const { return (size_t)kStages * (g.nx + g.ny); }

    void copy_field(Field4 dst, Field4 src)
    {
        launch(k_copy4, blocks_for((long)plane, 256), 256, dst, src, plane);
    }

    // One frozen step.  The LF speeds of stage k live in the tape row itself: recorded there by
    // k_alpha (zeroed by the boundary fill before it), or read from it when replaying, so neither
    // way copies them.  The worklists are built by the first step of a run (masks and levels are
    // frozen) and kept by the later ones.
    void enq_frozen_step(const double* tin, double* tout, const Field4* save, bool build_lists)
    {
        launch(k_begin, 1, 1, st, build_lists ? 0 : 1);
        const size_t stride = (size_t)g.nx + g.ny;
        Field4 ins[3] = {q, q2, q1};
        for (int fs = 0; fs < kStages; ++fs) {
            const double* rin = tin ? tin + fs * stride : nullptr;
            double* rout = tout ? tout + fs * stride : nullptr;
            double* rx = rout ? rout : ax[fs];
            double* ry = rout ? rout + g.ny : ay[fs];
            if (tin) enq_bc(ins[fs], st);
            else enq_bc(ins[fs], st, -1, rx, ry);
            if (save) copy_field(save[fs], ins[fs]);
            if (!tin) {
                if (fs == 0) enq_alpha(ins[fs], 3, fs, false, rx, ry);
                else enq_alpha_listed(ins[fs], fs, rx, ry);
            }
            if (fs == 0) {
                launch(k_dt, 1, 1, g, st);
                if (build_lists) {
                    ListArgs la;
                    for (int L = 0; L < kNumLists; ++L) la.list[L] = lists[L];
                    dim3 grid((g.nx + 1 + 255) / 256, (g.ny + 1 + kListRows - 1) / kListRows);
                    launch(k_lists, grid, 256, g, m, lvl[2], lvl[1], lvl[0], la, st);
                }
            }
            const double* fx_a = tin ? rin : rx;
            const double* fy_a = tin ? rin + g.ny : ry;
            enq_faces_update(fs, ins[fs], fs == 0 ? q2 : q1, fx_a, fy_a);
        }
        launch(k_finish, 1, 1, st);
    }

    // Device buffers of the frozen run and the adjoint, grown on demand and kept.
    double* tape = nullptr;
    size_t tape_steps = 0;
    std::vector<void*> adj_mem;
    size_t adj_key[3] = {0, 0, 0};
    Field4 lam{}, lam1{}, lam2{}, nu{}, qkeep{};
    std::vector<Field4> ckpt, seg;
    double* target = nullptr;
    double* rowsum = nullptr;
    double* loss_dev = nullptr;

    int alloc_plane(double** p)
    {
        AWCM_CUDA_TRY(cudaMalloc(p, plane * sizeof(double)));
        adj_mem.push_back(*p);
        return kOk;
    }
    int alloc_field(Field4& f)
    {
        for (int k = 0; k < 4; ++k) {
            const int rc = alloc_plane(&f.p[k]);
            if (rc) return rc;
        }
        return kOk;
    }
    void free_adj()
    {
        for (void* p : adj_mem) cudaFree(p);
        adj_mem.clear();
        ckpt.clear();
        seg.clear();
        adj_key[0] = adj_key[1] = adj_key[2] = 0;
    }
    int ensure_tape(size_t steps)
    {
        if (steps <= tape_steps) return kOk;
        if (tape) cudaFree(tape);
        tape = nullptr;
        tape_steps = 0;
        AWCM_CUDA_TRY(cudaMalloc(&tape, std::max<size_t>(steps, 1) * tape_stride() * sizeof(double)));
        tape_steps = steps;
        return kOk;
    }
    int ensure_adj(size_t n_ckpt, size_t seg_len)
    {
        if (adj_key[0] && n_ckpt <= adj_key[1] && seg_len <= adj_key[2]) return kOk;
        free_adj();
        int rc;
        for (Field4* f : {&lam, &lam1, &lam2, &nu, &qkeep})
            if ((rc = alloc_field(*f))) return rc;
        ckpt.resize(n_ckpt);
        for (auto& f : ckpt)
            if ((rc = alloc_field(f))) return rc;
        seg.resize(3 * seg_len);
        for (auto& f : seg)
            if ((rc = alloc_field(f))) return rc;
        AWCM_CUDA_TRY(cudaMalloc(&target, sizeof(double) * g.nx * g.ny));
        adj_mem.push_back(target);
        AWCM_CUDA_TRY(cudaMalloc(&rowsum, sizeof(double) * g.ny));
        adj_mem.push_back(rowsum);
        AWCM_CUDA_TRY(cudaMalloc(&loss_dev, sizeof(double)));
        adj_mem.push_back(loss_dev);
        adj_key[0] = 1;
        adj_key[1] = n_ckpt;
        adj_key[2] = seg_len;
        return kOk;
    }

    // n frozen steps from t0 at fixed dt.  mode 1: LF speeds computed and recorded into the
    // solver's tape; mode 2: replayed from the tape of the last recording run.
    // out[0] = t, out[1] = device ms, out[2] = sum |mask0| over the steps.
    int frozen_run(double t0, double dt, int n, int mode, double* out)
    {
        if (n < 0 || !(dt > 0) || (mode != 1 && mode != 2)) return kErrArg;
        if (mode == 2 && (size_t)n > tape_steps) {
            set_last_error("frozen replay longer than the recorded LF-speed tape", __FILE__, __LINE__);
            return kErrState;
        }
        if (mode == 1) {
            const int rc = ensure_tape((size_t)n);
            if (rc) return rc;
        }
        int rc = write_params(0.0, 1.0, t0, 1e300, dt);
        if (rc) return rc;
        StepState h0;
        if ((rc = read_state(&h0))) return rc;
        cudaEvent_t e0, e1;
        AWCM_CUDA_TRY(cudaEventCreate(&e0));
        AWCM_CUDA_TRY(cudaEventCreate(&e1));
        cudaEventRecord(e0, stream);
        for (int s = 0; s < n; ++s) {
            double* row = tape + (size_t)s * tape_stride();
            enq_frozen_step(mode == 2 ? row : nullptr, mode == 1 ? row : nullptr, nullptr, s == 0);
        }
        cudaEventRecord(e1, stream);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        StepState h;
        if ((rc = read_state(&h))) return rc;
        // frozen steps leave values outside mask0 (no residue removal)
        mark_full_zero();
        if (out) {
            out[0] = h.t;
            out[1] = ms;
            out[2] = (double)(h.upd - h0.upd);
        }
        return kOk;
    }

    // Reverse sweep of one frozen step: stage inputs sv[0..2] = Q, Q2, Q1 (boundary-filled), LF
    // speeds of the step `ts`; lam holds the adjoint of the step's output on entry and of its
    // input on exit.
    void enq_adjoint_step(const Field4* sv, const double* ts)
    {
        const double* sc = st->sc;
        Field4 lam_out[3] = {lam, lam2, lam1};  // adjoint receiving the VJP of stage fs
        for (int fs = kStages - 1; fs >= 0; --fs) {
            const int bit = 2 - fs;
            const int8_t* lv = lvl[bit];
            if (fs == 2) adj_launch_rk(3, g, plane, m, lv, sc, lam, lam, lam1, nu, stream);
            else if (fs == 1) adj_launch_rk(2, g, plane, m, lv, sc, lam1, lam, lam2, nu, stream);
            else adj_launch_rk(1, g, plane, m, lv, sc, lam2, lam, lam2, nu, stream);
            AdjStage A;
            A.g = g;
            A.qin = sv[fs];
            A.lam = lam_out[fs];
            A.nu = nu;
            A.m = m;
            A.lvl = lv;
            A.bit = bit;
            A.xf = lists[4 * fs + 2];
            A.nxf = st->cnt + 4 * fs + 2;
            A.yf = lists[4 * fs + 3];
            A.nyf = st->cnt + 4 * fs + 3;
            A.crs = lists[4 * fs + 1];
            A.ncrs = st->cnt + 4 * fs + 1;
            A.ax = ts + (size_t)fs * (g.nx + g.ny);
            A.ay = A.ax + g.ny;
            adj_launch_stage(A, face_blocks, stream);
            adj_launch_fold(g, lam_out[fs], stream);
        }
    }

    // Loss L = 1/2 sum over the mask0 points of (rho(t0 + n dt) - target)^2 of the frozen run from
    // the current state, and dL/dQ(t0) by the discrete adjoint.  The forward run records the LF speeds
    // (mode 1) or replays the tape (mode 2); the reverse sweep recomputes the stage inputs segment
    // by segment from checkpoints of Q taken every `every` steps (every >= n: one segment, all
    // stage inputs kept from the forward run, no recomputation).  The state is left at the end of
    // the forward run.  out[0] = loss, [1] forward ms, [2] reverse ms (recomputation included),
    // [3] checkpoint interval, [4] device bytes of checkpoints + stage inputs + adjoint fields.
    int adjoint(double t0, double dt, int n, int every, int mode, const double* target_host, double* grad_host,
                double* out)
    {
        if (n <= 0 || !(dt > 0) || !target_host || (mode != 1 && mode != 2)) return kErrArg;
        if (every <= 0) every = std::max(1, (int)std::ceil(std::sqrt((double)n)));
        every = std::min(every, n);
        const int n_seg = (n + every - 1) / every;
        const bool keep_all = n_seg == 1;
        int rc = ensure_adj(keep_all ? 0 : (size_t)n_seg, (size_t)every);
        if (rc) return rc;
        if (mode == 1 && (rc = ensure_tape((size_t)n))) return rc;
        if (mode == 2 && (size_t)n > tape_steps) {
            set_last_error("adjoint replay longer than the recorded LF-speed tape", __FILE__, __LINE__);
            return kErrState;
        }
        AWCM_CUDA_TRY(cudaMemcpyAsync(target, target_host, sizeof(double) * g.nx * g.ny, cudaMemcpyHostToDevice, stream));
        if ((rc = write_params(0.0, 1.0, t0, 1e300, dt))) return rc;
        cudaEvent_t ev[3];
        for (auto& e : ev) AWCM_CUDA_TRY(cudaEventCreate(&e));
        // forward: checkpoints (or every stage input) and the LF-speed tape
        cudaEventRecord(ev[0], stream);
        for (int s = 0; s < n; ++s) {
            if (!keep_all && s % every == 0) copy_field(ckpt[s / every], q);
            double* row = tape + (size_t)s * tape_stride();
            enq_frozen_step(mode == 2 ? row : nullptr, mode == 1 ? row : nullptr, keep_all ? &seg[3 * s] : nullptr,
                            s == 0);
        }
        adj_launch_seed(g, q, m, target, lam, rowsum, loss_dev, stream);
        cudaEventRecord(ev[1], stream);
        // reverse
        if (!keep_all) copy_field(qkeep, q);
        for (int k = n_seg - 1; k >= 0; --k) {
            const int s0 = k * every, s1 = std::min(n, s0 + every);
            if (!keep_all) {
                copy_field(q, ckpt[k]);
                // the segment's start time, for the time-dependent boundary fill
                const double tk = t0 + s0 * dt;
                cudaMemcpyAsync(&st->t, &tk, sizeof(double), cudaMemcpyHostToDevice, stream);
                for (int s = s0; s < s1; ++s)
                    enq_frozen_step(tape + (size_t)s * tape_stride(), nullptr, &seg[3 * (s - s0)], false);
            }
            for (int s = s1 - 1; s >= s0; --s)
                enq_adjoint_step(&seg[3 * (s - s0)], tape + (size_t)s * tape_stride());
        }
        cudaEventRecord(ev[2], stream);
        if (!keep_all) copy_field(q, qkeep);
        AWCM_CUDA_TRY(cudaGetLastError());
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        float f_ms = 0, r_ms = 0;
        cudaEventElapsedTime(&f_ms, ev[0], ev[1]);
        cudaEventElapsedTime(&r_ms, ev[1], ev[2]);
        for (auto& e : ev) cudaEventDestroy(e);
        // the state's clock at the end of the forward run
        {
            const double tn = t0 + n * dt;
            AWCM_CUDA_TRY(cudaMemcpyAsync(&st->t, &tn, sizeof(double), cudaMemcpyHostToDevice, stream));
        }
        double loss = 0;
        AWCM_CUDA_TRY(cudaMemcpyAsync(&loss, loss_dev, sizeof(double), cudaMemcpyDeviceToHost, stream));
        if (grad_host) {
            const size_t np = ghosted_points();
            if ((rc = ensure_staging(np * 4 * sizeof(double)))) return rc;
            launch(k_soa_to_aos, blocks_for((long)np, 256), 256, g, lam, (double*)staging);
            AWCM_CUDA_TRY(cudaGetLastError());
            AWCM_CUDA_TRY(cudaMemcpyAsync(grad_host, staging, np * 4 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        }
        AWCM_CUDA_TRY(cudaStreamSynchronize(stream));
        if (out) {
            out[0] = loss;
            out[1] = f_ms;
            out[2] = r_ms;
            out[3] = every;
            out[4] = (double)((keep_all ? 0 : n_seg) + 3 * every + 5) * 4 * plane * sizeof(double) +
                     (double)n * tape_stride() * sizeof(double);
        }
        mark_full_zero();  // the frozen forward leaves values outside mask0
        return kOk;
    }

    int init_problem(int kind, double a, double b)
    {
        // Problem initial states (Problems/2D/PROBLEM_QUADRANTS.h:34-80, PROBLEM_DOUBLEMACH.h:34-62,
        // PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h:38-64), evaluated on the host with the grid's node
        // coordinates x_min + i dx, ghosts included.
        const int w = g.nx + 6;
        std::vector<double> h((size_t)w * (g.ny + 6) * 4);
        const double gam = g.gamma;
        const double PI = 4. * std::atan(1.);
        auto E = [&](double rho, double u, double v, double p) { return p / (gam - 1) + 0.5 * rho * (u * u + v * v); };
        for (int j = -3; j < g.ny + 3; ++j)
            for (int i = -3; i < g.nx + 3; ++i) {
                const double x = g.x_min + i * g.dx, y = g.y_min + j * g.dy;
                double rho, u, v, p, Q[4];
                if (kind == AWCM_PROBLEM_QUADRANTS) {
                    if (x >= a && y >= b) rho = 1.5, u = 0, v = 0, p = 1.5;
                    else if (x < a && y >= b) rho = 0.532258064516129, u = 1.206045378311055, v = 0, p = 0.3;
                    else if (x < a && y < b)
                        rho = 0.137992831541219, u = 1.206045378311055, v = 1.206045378311055, p = 0.029032258064516;
                    else rho = 0.532258064516129, u = 0, v = 1.206045378311055, p = 0.3;
                    Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = E(rho, u, v, p);
                } else if (kind == AWCM_PROBLEM_DOUBLE_MACH) {
                    if (y > std::sqrt(3.0) * (x - 1.0 / 6.0)) rho = 8, u = 8.25 * std::sqrt(3.0) * 0.5, v = -8.25 * 0.5, p = 116.5;
                    else rho = a, u = 0, v = 0, p = 1;
                    Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = E(rho, u, v, p);
                } else if (kind == AWCM_PROBLEM_VORTEX) {
                    const double rr = (x - a) * (x - a) + (y - b) * (y - b);
                    const double beta = 5;
                    rho = 1 - (gam - 1) * (beta * beta) / (8 * gam * PI * PI) * std::exp(1 - rr);
                    rho = std::pow(rho, 1.0 / (gam - 1.0));
                    double rhou = 0 - beta / (2 * PI) * std::exp((1 - rr) * 0.5) * (y - b);
                    rhou *= rho;
                    double rhov = 1 + beta / (2 * PI) * std::exp((1 - rr) * 0.5) * (x - a);
                    rhov *= rho;
                    p = std::pow(rho, gam);
                    Q[0] = rho, Q[1] = rhou, Q[2] = rhov, Q[3] = E(rho, rhou / rho, rhov / rho, p);
                } else if (kind == AWCM_PROBLEM_WIND_TUNNEL) {
                    // WINDTUNNEL::Initialize (Problems/2D/PROBLEM_WINDTUNNEL.h:14-47): Mach 3 uniform flow
                    rho = 1.4, u = 3, v = 0, p = 1;
                    Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = E(rho, u, v, p);
                } else if (kind == AWCM_PROBLEM_SHOCK_VORTEX) {
                    // SHOCK_VORTEX::Initialize (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:32-66):
                    // post-shock state for x <= 0, vortex of Mach 0.5 centred at (a, b) ahead of it.
                    const double Mv = 0.5;
                    const double r = std::sqrt((x - a) * (x - a) + (y - b) * (y - b));
                    if (x <= 0) {
                        rho = 1.394708041144614, u = -0.860403729339060, v = 0, p = 1.121834000000000;
                    } else {
                        rho = 1 - (gam - 1) / 2 * (Mv * Mv) * std::exp(1 - r * r);
                        rho = std::pow(rho, 1 / (gam - 1));
                        p = 1 - (gam - 1) / 2 * (Mv * Mv) * std::exp(1 - r * r);
                        p = std::pow(p, gam / (gam - 1));
                        p = 1 / gam * p;
                        u = Mv * std::exp(0.5 * (1 - r * r)) * (-y) - 1.200011999940001;
                        v = Mv * std::exp(0.5 * (1 - r * r)) * (x - a);
                    }
                    Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = E(rho, u, v, p);
                } else {
                    return kErrArg;
                }
                for (int k = 0; k < 4; ++k) h[((size_t)(j + 3) * w + (i + 3)) * 4 + k] = Q[k];
            }
        return set_q(h.data());
    }
};

}  // namespace awcm

// ======================================================================================== C-ABI
using awcm::Solver2D;

struct awcm2d_s {
    Solver2D s;
};

extern "C" {

int awcm2d_create(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                  double y_max, int bc_kind, awcm2d_t* out)
{
    if (!out) return awcm::kErrArg;
    *out = nullptr;
    awcm2d_s* h = new (std::nothrow) awcm2d_s();
    if (!h) return awcm::kErrOom;
    const int rc = h->s.create(num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, bc_kind);
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return awcm::kOk;
}

int awcm2d_create_scalar(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                         double y_max, awcm2d_t* out)
{
    const int rc = awcm2d_create(num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, AWCM_BC_PERIODIC, out);
    if (rc) return rc;
    (*out)->s.scalar = true;
    return awcm::kOk;
}

int awcm2d_destroy(awcm2d_t h)
{
    delete h;
    return awcm::kOk;
}

#define AWCM_H(h)                         \
    if (!(h)) return awcm::kErrArg;       \
    cudaSetDevice((h)->s.device)

#define AWCM_EULER_ONLY(h)                                                                  \
    if ((h)->s.scalar) {                                                                    \
        awcm::set_last_error("Euler entry point called on a scalar instance", __FILE__, __LINE__); \
        return awcm::kErrState;                                                             \
    }
#define AWCM_SCALAR_ONLY(h)                                                                 \
    if (!(h)->s.scalar) {                                                                   \
        awcm::set_last_error("scalar entry point called on an Euler instance", __FILE__, __LINE__); \
        return awcm::kErrState;                                                             \
    }


int awcm2d_dims(awcm2d_t h, int* nx, int* ny)
{
    if (!h || !nx || !ny) return awcm::kErrArg;
    *nx = h->s.g.nx;
    *ny = h->s.g.ny;
    return awcm::kOk;
}

int awcm2d_get_geometry(awcm2d_t h, awcm2d_geometry* out)
{
    if (!h || !out) return awcm::kErrArg;
    *out = h->s.geo;
    return awcm::kOk;
}
int awcm2d_set_q(awcm2d_t h, const double* q)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    return q ? h->s.set_q(q) : awcm::kErrArg;
}
int awcm2d_get_q(awcm2d_t h, double* q)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    return q ? h->s.get_q(q) : awcm::kErrArg;
}
int awcm2d_get_masks(awcm2d_t h, uint8_t* m)
{
    AWCM_H(h);
    return m ? h->s.get_masks(m) : awcm::kErrArg;
}
int awcm2d_set_masks(awcm2d_t h, const uint8_t* m)
{
    AWCM_H(h);
    return m ? h->s.set_masks(m) : awcm::kErrArg;
}
int awcm2d_get_levels(awcm2d_t h, int* lv)
{
    AWCM_H(h);
    return lv ? h->s.get_levels(lv) : awcm::kErrArg;
}
int awcm2d_set_levels(awcm2d_t h, const int* lv)
{
    AWCM_H(h);
    return lv ? h->s.set_levels(lv) : awcm::kErrArg;
}
int awcm2d_init_problem(awcm2d_t h, int kind, double a, double b)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    return h->s.init_problem(kind, a, b);
}
int awcm2d_prepare(awcm2d_t h, double tol)
{
    AWCM_H(h);
    return h->s.prepare(tol);
}
int awcm2d_fwt(awcm2d_t h, double tol)
{
    AWCM_H(h);
    return h->s.fwt(tol);
}
int awcm2d_iwt(awcm2d_t h, int mask_id)
{
    AWCM_H(h);
    return h->s.iwt(mask_id);
}
int awcm2d_interpolate(awcm2d_t h, int from_id, int to_id)
{
    AWCM_H(h);
    return h->s.interpolate(from_id, to_id);
}
int awcm2d_interpolate_all(awcm2d_t h, int from_id)
{
    AWCM_H(h);
    if (from_id < 0 || from_id > 4) return awcm::kErrArg;
    return h->s.interpolate_all(from_id);
}
int awcm2d_manager(awcm2d_t h, int op, int mask_id, int level_id)
{
    AWCM_H(h);
    return h->s.manager(op, mask_id, level_id);
}
int awcm2d_wt_set_bottom(awcm2d_t h, int x_direction, int y_direction)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    return h->s.wt_bottom(x_direction, y_direction);
}
int awcm2d_set_bc_field(awcm2d_t h, const int* bc)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    if (!bc) return awcm::kErrArg;
    return h->s.set_bc_field(bc);
}
int awcm2d_apply_bc(awcm2d_t h, double t)
{
    AWCM_H(h);
    return h->s.apply_bc(t);
}
int awcm2d_scalar_set_q(awcm2d_t h, const double* q)
{
    AWCM_H(h);
    AWCM_SCALAR_ONLY(h);
    return q ? h->s.scalar_set_q(q) : awcm::kErrArg;
}
int awcm2d_scalar_get_q(awcm2d_t h, double* q)
{
    AWCM_H(h);
    AWCM_SCALAR_ONLY(h);
    return q ? h->s.scalar_get_q(q) : awcm::kErrArg;
}
int awcm2d_scalar_advance(awcm2d_t h, double tol, double dt, double t, int n_steps, double* out)
{
    AWCM_H(h);
    AWCM_SCALAR_ONLY(h);
    return h->s.scalar_advance(tol, dt, t, n_steps, out);
}
int awcm2d_step(awcm2d_t h, double tol, double cfl, double t, double t_next, double dt_fixed, double* out)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    return h->s.step(tol, cfl, t, t_next, dt_fixed, out);
}
int awcm2d_advance(awcm2d_t h, double tol, double cfl, double t_start, double t_end, int n_steps, double* out)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    if (n_steps < 0) return awcm::kErrArg;
    return h->s.advance(tol, cfl, t_start, t_end, n_steps, out);
}
int awcm2d_step_io_bytes(awcm2d_t h, long long* h2d, long long* d2h)
{
    if (!h || !h2d || !d2h) return awcm::kErrArg;
    // awcm2d_step: the step scalars are read back, updated and written (one copy each way), and
    // the step's results read after the graph (a second copy back)
    *h2d = (long long)sizeof(awcm::StepState);
    *d2h = 2LL * (long long)sizeof(awcm::StepState);
    return awcm::kOk;
}
int awcm2d_launches_per_step(awcm2d_t h, int* n)
{
    AWCM_H(h);
    if (!n) return awcm::kErrArg;
    int rc = h->s.build_graph();
    *n = h->s.launches;
    return rc;
}
int awcm2d_profile_step(awcm2d_t h, double tol, double cfl, double t, double t_end, double* out)
{
    AWCM_H(h);
    if (!out) return awcm::kErrArg;
    return h->s.profile_step(tol, cfl, t, t_end, out);
}
int awcm2d_profile_kernels(awcm2d_t h, double tol, double cfl, double t, double t_end, int cap, char* names,
                           double* ms, int* n)
{
    AWCM_H(h);
    if (!names || !ms || !n || cap <= 0) return awcm::kErrArg;
    std::vector<std::pair<const char*, float>> v;
    const int rc = h->s.profile_fine(tol, cfl, t, t_end, v);
    if (rc) return rc;
    *n = (int)std::min<size_t>(v.size(), (size_t)cap);
    for (int k = 0; k < *n; ++k) {
        std::strncpy(names + 32 * k, v[k].first, 31);
        names[32 * k + 31] = 0;
        ms[k] = v[k].second;
    }
    return awcm::kOk;
}
int awcm2d_set_prepare_mode(awcm2d_t h, int mode)
{
    AWCM_H(h);
    if (mode != 0 && mode != 1) return awcm::kErrArg;
    h->s.prep_mode = mode;
    if (h->s.graph) cudaGraphExecDestroy(h->s.graph);
    h->s.graph = nullptr;
    return awcm::kOk;
}
int awcm2d_set_spin_limit(awcm2d_t h, unsigned polls)
{
    AWCM_H(h);
    return h->s.set_spin_limit(polls);
}
int awcm2d_frozen_run(awcm2d_t h, double t0, double dt, int n_steps, int mode, double* out)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    if (h->s.g.bc_kind == AWCM_BC_WIND_TUNNEL) {
        awcm::set_last_error("the frozen-mask run has no per-direction wind-tunnel fills", __FILE__, __LINE__);
        return awcm::kErrArg;
    }
    return h->s.frozen_run(t0, dt, n_steps, mode, out);
}
int awcm2d_adjoint(awcm2d_t h, double t0, double dt, int n_steps, int checkpoint_every, int mode,
                   const double* target, double* grad, double* out)
{
    AWCM_H(h);
    AWCM_EULER_ONLY(h);
    if (h->s.g.bc_kind == AWCM_BC_GENERIC || h->s.g.bc_kind == AWCM_BC_WIND_TUNNEL) {
        awcm::set_last_error("the adjoint's boundary transposes cover the fixed edge managers only, not the generic "
                             "or the wind-tunnel one",
                             __FILE__, __LINE__);
        return awcm::kErrArg;
    }
    return h->s.adjoint(t0, dt, n_steps, checkpoint_every, mode, target, grad, out);
}
int awcm2d_set_wenoz(awcm2d_t h, double eps, double tau_delta)
{
    AWCM_H(h);
    if (!(eps > 0) || !std::isfinite(eps) || !(tau_delta >= 0) || !std::isfinite(tau_delta)) return awcm::kErrArg;
    h->s.g.wz_eps = eps;
    h->s.g.wz_delta = tau_delta;
    if (h->s.graph) cudaGraphExecDestroy(h->s.graph);
    h->s.graph = nullptr;
    return awcm::kOk;
}
int awcm2d_get_alpha_tape(awcm2d_t h, int n_steps, double* tape)
{
    AWCM_H(h);
    if (!tape || n_steps < 0 || (size_t)n_steps > h->s.tape_steps) return awcm::kErrArg;
    AWCM_CUDA_TRY(cudaMemcpy(tape, h->s.tape, (size_t)n_steps * h->s.tape_stride() * sizeof(double),
                             cudaMemcpyDeviceToHost));
    return awcm::kOk;
}
int awcm2d_set_alpha_tape(awcm2d_t h, int n_steps, const double* tape)
{
    AWCM_H(h);
    if (!tape || n_steps < 0) return awcm::kErrArg;
    const int rc = h->s.ensure_tape((size_t)n_steps);
    if (rc) return rc;
    AWCM_CUDA_TRY(cudaMemcpy(h->s.tape, tape, (size_t)n_steps * h->s.tape_stride() * sizeof(double),
                             cudaMemcpyHostToDevice));
    return awcm::kOk;
}
int awcm2d_stream(awcm2d_t h, void** stream)
{
    if (!h || !stream) return awcm::kErrArg;
    *stream = (void*)h->s.stream;
    return awcm::kOk;
}

int euler2d_flux(const double* q_dev, double* f_dev, int n, int dir, double gamma, void* stream)
{
    if (n < 0 || (n && (!q_dev || !f_dev)) || (dir != 0 && dir != 1)) return awcm::kErrArg;
    if (!n) return awcm::kOk;
    awcm::k_euler_flux<<<awcm::blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(q_dev, f_dev, n, dir, gamma);
    AWCM_CUDA_TRY(cudaGetLastError());
    return awcm::kOk;
}

int euler2d_spectral_radius(const double* q_dev, double* s_dev, int n, int dir, double gamma, void* stream)
{
    if (n < 0 || (n && (!q_dev || !s_dev)) || (dir != 0 && dir != 1)) return awcm::kErrArg;
    if (!n) return awcm::kOk;
    awcm::k_euler_sr<<<awcm::blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(q_dev, s_dev, n, dir, gamma);
    AWCM_CUDA_TRY(cudaGetLastError());
    return awcm::kOk;
}

}  // extern "C"

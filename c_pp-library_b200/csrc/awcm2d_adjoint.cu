// Hand-written discrete adjoint of the 2D AWCM RK3 step on a frozen active mask.
//
// The forward map of one frozen step (masks, levels, per-stage LF speeds and dt fixed; no
// PrepareEuler, no residue removal) is
//   Q2 = Q  - s R(Q)              on mask2          (stage 1, main_2d_euler(quad).cpp:162)
//   Q1 = 3/4 Q + 1/4 (Q2 - s R(Q2)) on mask1        (stage 2, :242)
//   Q' = (Q + 2 (Q1 - s R(Q1))) / 3 on mask0, Q elsewhere   (stage 3 and :325-332)
// with R = dF + dG: WENO-Z/Roe face-flux differences at finest-level points
// (WENOZ_EULER_SOLVER_2D::ComputeFluxX/Y, WENOZ.h:236-320) and 4th-order central differences of
// the physical fluxes at coarser points (AWCM_2D::Differentiate*, Wavelet/AWCM_2D.h:154-187), each
// stage reading its input through the boundary fill.  This file holds the reverse-mode pieces:
// the vector-Jacobian product of the face flux (recompute the face's forward values, then sweep
// back through the WENO-Z weights, the Lax-Friedrichs split, the characteristic projection, the
// physical fluxes and the Roe average), of the coarse differences, of the RK combinations and of
// the boundary fill.  Built with FMA contraction: the adjoint is checked against finite
// differences, not bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

#include "awcm_b200.h"
#include "awcm2d_types.cuh"

namespace awcm {
namespace {

__device__ __forceinline__ unsigned gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// Programmatic dependent launch, as for the forward kernels: the successor's CTAs are scheduled
// once all of this kernel's CTAs run and wait in griddepcontrol.wait (a hardware wait on the
// predecessor's completion) before their first access; no-ops without the launch attribute.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... P, typename... A>
void launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, cudaStream_t s, A&&... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

__device__ __forceinline__ void atomic_sub(double* p, double v)
{
    if (v != 0.0) atomicAdd(p, -v);
}
__device__ __forceinline__ void atomic_add(double* p, double v)
{
    if (v != 0.0) atomicAdd(p, v);
}

// ---------------------------------------------------------------------------- WENO-Z reverse
// Reverse of recon_left<kWenoZ> (WENOZ5::ReconstructLeft, WENOZ.h:75-104): adds d(out)/d(input)
// times ob to g[0..4] for the inputs (ll, l, c, r, rr) and returns out itself.  tau = |b0 - b2| is differentiated as
// sign(b0 - b2); with delta > 0, tau = sqrt((b0 - b2)^2 + delta^2) and dtau = (b0 - b2) / tau.
__device__ __forceinline__ double recon_left_vjp(double ll, double l, double c, double r, double rr, double ob,
                                                 double eps, double delta, double* g)
{
    const double A0 = c - 2 * r + rr, B0 = 3 * c - 4 * r + rr;
    const double A1 = l - 2 * c + r, B1 = l - r;
    const double A2 = ll - 2 * l + c, B2 = ll - 4 * l + 3 * c;
    const double b0 = kC13_12 * A0 * A0 + 0.25 * B0 * B0;
    const double b1 = kC13_12 * A1 * A1 + 0.25 * B1 * B1;
    const double b2 = kC13_12 * A2 * A2 + 0.25 * B2 * B2;
    const double dl = b0 - b2;
    double tau, sg;
    if (delta > 0) {
        tau = sqrt(dl * dl + delta * delta);
        sg = dl / tau;
    } else {
        tau = fabs(dl);
        sg = dl > 0 ? 1.0 : (dl < 0 ? -1.0 : 0.0);
    }
    const double ie0 = 1.0 / (b0 + eps), ie1 = 1.0 / (b1 + eps), ie2 = 1.0 / (b2 + eps);
    const double a0 = 0.1 * (1 + tau * ie0), a1 = 0.6 * (1 + tau * ie1), a2 = 0.3 * (1 + tau * ie2);
    const double iS = 1.0 / (a0 + a1 + a2);
    const double w0 = a0 * iS, w1 = a1 * iS, w2 = a2 * iS;
    const double P0 = kC11_6 * c + kCm7_6 * r + kC1_3 * rr;
    const double P1 = kC1_3 * l + kC5_6 * c + kCm1_6 * r;
    const double P2 = kCm1_6 * ll + kC5_6 * l + kC1_3 * c;
    // out = w0 P0 + w1 P1 + w2 P2
    const double wb0 = ob * P0, wb1 = ob * P1, wb2 = ob * P2;
    const double Pb0 = ob * w0, Pb1 = ob * w1, Pb2 = ob * w2;
    const double Sb = -(wb0 * w0 + wb1 * w1 + wb2 * w2) * iS;
    const double ab0 = wb0 * iS + Sb, ab1 = wb1 * iS + Sb, ab2 = wb2 * iS + Sb;
    const double taub = 0.1 * ab0 * ie0 + 0.6 * ab1 * ie1 + 0.3 * ab2 * ie2;
    double bb0 = -0.1 * ab0 * tau * ie0 * ie0;
    const double bb1 = -0.6 * ab1 * tau * ie1 * ie1;
    double bb2 = -0.3 * ab2 * tau * ie2 * ie2;
    bb0 += taub * sg;
    bb2 -= taub * sg;
    const double Ab0 = 2 * kC13_12 * A0 * bb0, Bb0 = 0.5 * B0 * bb0;
    const double Ab1 = 2 * kC13_12 * A1 * bb1, Bb1 = 0.5 * B1 * bb1;
    const double Ab2 = 2 * kC13_12 * A2 * bb2, Bb2 = 0.5 * B2 * bb2;
    g[0] += Ab2 + Bb2 + kCm1_6 * Pb2;
    g[1] += Ab1 + Bb1 - 2 * Ab2 - 4 * Bb2 + kC1_3 * Pb1 + kC5_6 * Pb2;
    g[2] += Ab0 + 3 * Bb0 - 2 * Ab1 + Ab2 + 3 * Bb2 + kC11_6 * Pb0 + kC5_6 * Pb1 + kC1_3 * Pb2;
    g[3] += -2 * Ab0 - 4 * Bb0 + Ab1 - Bb1 + kCm7_6 * Pb0 + kCm1_6 * Pb1;
    g[4] += Ab0 + Bb0 + kC1_3 * Pb0;
    return w0 * P0 + w1 * P1 + w2 * P2;  // the forward value (FMA-contracted: a derivative input only)
}

// ---------------------------------------------------------------------- physical flux reverse
// Reverse of flux2<DIR> (EULER_EQUATION_2D::ComputeFu/ComputeGu, EULER_EQUATION.h:74-99):
// adds (dF/dq)^T fb to qb.
template <int DIR>
__device__ __forceinline__ void flux2_vjp(const double* q, double g, const double* fb, double* qb)
{
    const double gm1 = g - 1;
    const double iq0 = 1.0 / q[0];
    const double u = q[1] * iq0, v = q[2] * iq0;
    const double p = gm1 * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) * iq0);
    double pb = 0;
    if (DIR == 0) {
        // f0 = q1, f1 = q1^2/q0 + p, f2 = q1 q2/q0, f3 = (q3 + p) q1/q0
        qb[1] += fb[0];
        qb[1] += fb[1] * 2 * u;
        qb[0] -= fb[1] * u * u;
        pb += fb[1];
        qb[2] += fb[2] * u;
        qb[1] += fb[2] * v;
        qb[0] -= fb[2] * u * v;
        const double h = (q[3] + p) * iq0;
        qb[3] += fb[3] * u;
        pb += fb[3] * u;
        qb[1] += fb[3] * h;
        qb[0] -= fb[3] * h * u;
    } else {
        qb[2] += fb[0];
        qb[2] += fb[2] * 2 * v;
        qb[0] -= fb[2] * v * v;
        pb += fb[2];
        qb[1] += fb[1] * v;
        qb[2] += fb[1] * u;
        qb[0] -= fb[1] * u * v;
        const double h = (q[3] + p) * iq0;
        qb[3] += fb[3] * v;
        pb += fb[3] * v;
        qb[2] += fb[3] * h;
        qb[0] -= fb[3] * h * v;
    }
    // p = gm1 (q3 - (q1^2 + q2^2) / (2 q0))
    qb[0] += pb * 0.5 * gm1 * (u * u + v * v);
    qb[1] -= pb * gm1 * u;
    qb[2] -= pb * gm1 * v;
    qb[3] += pb * gm1;
}

struct RoeAdj {
    double u, v, H, c, kc;
};

// Reverse of inv2<DIR> (ROE_SOLVER_2D::Inversion_X/_Y, ROESOLVER.h:73-96): adds (dx/db)^T xb to
// bb and the parameter adjoints to P.
template <int DIR>
__device__ __forceinline__ void inv2_vjp(const RoeAdj& R, const double* b, const double* xb, double* bb, RoeAdj& P)
{
    const double u = R.u, v = R.v, H = R.H, c = R.c, kc = R.kc;
    const double A = H - u * u - v * v;
    const double y3 = DIR == 0 ? A * b[0] + u * b[1] + v * b[2] - b[3] : A * b[0] + v * b[2] + u * b[1] - b[3];
    const double x3 = y3 * kc;
    const double i2c = 0.5 / c;
    const double y4 = DIR == 0 ? b[1] + (c - u) * b[0] - c * x3 : b[2] + (c - v) * b[0] - c * x3;
    const double x4 = y4 * i2c;
    // x1 = b0 - x3 - x4
    bb[0] += xb[0];
    double x3b = xb[2] - xb[0];
    const double x4b = xb[3] - xb[0];
    // x4 = y4 / (2c)
    const double y4b = x4b * i2c;
    P.c -= x4b * x4 / c;
    if (DIR == 0) {
        bb[1] += y4b;
        bb[0] += y4b * (c - u);
        P.u -= y4b * b[0];
        // x2 = b2 - v b0
        bb[2] += xb[1];
        bb[0] -= xb[1] * v;
        P.v -= xb[1] * b[0];
    } else {
        bb[2] += y4b;
        bb[0] += y4b * (c - v);
        P.v -= y4b * b[0];
        // x2 = b1 - u b0
        bb[1] += xb[1];
        bb[0] -= xb[1] * u;
        P.u -= xb[1] * b[0];
    }
    P.c += y4b * (b[0] - x3);
    x3b -= y4b * c;
    // x3 = y3 kc
    const double y3b = x3b * kc;
    P.kc += x3b * y3;
    bb[0] += y3b * A;
    bb[1] += y3b * u;
    bb[2] += y3b * v;
    bb[3] -= y3b;
    P.u += y3b * b[1];
    P.v += y3b * b[2];
    const double Ab = y3b * b[0];
    P.H += Ab;
    P.u -= 2 * u * Ab;
    P.v -= 2 * v * Ab;
}

// d(face flux)/d(six cells)^T ob (WENOZ_EULER_SOLVER_2D::ComputeFluxX/Y, WENOZ.h:236-320).
// Forward values are recomputed here; alpha (the frozen LF speed) has no adjoint.  The 6 x 4
// characteristic states and fluxes (and, in place, their adjoints) live in shared memory:
// `sh` points at this thread's slot, element e at sh[e * kAdjThreads].
constexpr int kAdjThreads = 128;
template <int DIR>
__device__ void face_flux_2d_vjp(const double (&s)[6][4], double alpha, double g, const double* ob, double eps,
                                 double delta, double (&gs)[6][4], double* sh)
{
    auto RQs = [&](int p, int k) -> double& { return sh[(p * 4 + k) * kAdjThreads]; };
    auto RFs = [&](int p, int k) -> double& { return sh[(24 + p * 4 + k) * kAdjThreads]; };
    // ---- forward: Roe average of the face states s[2], s[3] (ROESOLVER.h:49-70)
    const double* L = s[2];
    const double* Rr = s[3];
    const double gm1 = g - 1;
    const double iL0 = 1.0 / L[0], iR0 = 1.0 / Rr[0];
    const double KL = L[1] * L[1] + L[2] * L[2], KR = Rr[1] * Rr[1] + Rr[2] * Rr[2];
    const double pL = gm1 * (L[3] - 0.5 * KL * iL0), pR = gm1 * (Rr[3] - 0.5 * KR * iR0);
    const double HL = (L[3] + pL) * iL0, HR = (Rr[3] + pR) * iR0;
    const double uL = L[1] * iL0, uR = Rr[1] * iR0, vL = L[2] * iL0, vR = Rr[2] * iR0;
    const double sL = sqrt(L[0]), sR = sqrt(Rr[0]);
    const double iden = 1.0 / (sL + sR);
    RoeAdj R;
    R.u = (sL * uL + sR * uR) * iden;
    R.v = (sL * vL + sR * vR) * iden;
    R.H = (sL * HL + sR * HR) * iden;
    const double q2 = R.u * R.u + R.v * R.v;
    R.c = sqrt(0.4 * (R.H - 0.5 * q2));
    R.kc = 0.4 / (R.c * R.c);
    // ---- forward: characteristic variables and LF split of the six cells
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        double f[4], rq[4], rf[4];
        flux2<DIR>(s[p], g, f);
        inv2<DIR>(R.u, R.v, R.H, R.c, R.kc, s[p], rq);
        inv2<DIR>(R.u, R.v, R.H, R.c, R.kc, f, rf);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            RQs(p, k) = rq[k];
            RFs(p, k) = rf[k];
        }
    }
    // ---- reverse: back-projection out = sum_k S_k r_k.  The adjoints of S depend only on ob
    // and the Roe state; S itself (needed for the Roe-state adjoints) comes out of the WENO-Z
    // reverse below, which recomputes the reconstructions anyway.
    const double u = R.u, v = R.v, H = R.H, c = R.c;
    double Sb[4];
    if (DIR == 0) {
        Sb[0] = ob[0] + ob[1] * (u - c) + ob[2] * v + ob[3] * (H - u * c);
        Sb[1] = ob[2] + ob[3] * v;
        Sb[2] = ob[0] + ob[1] * u + ob[2] * v + ob[3] * 0.5 * q2;
        Sb[3] = ob[0] + ob[1] * (u + c) + ob[2] * v + ob[3] * (H + u * c);
    } else {
        Sb[0] = ob[0] + ob[1] * u + ob[2] * (v - c) + ob[3] * (H - v * c);
        Sb[1] = ob[1] + ob[3] * u;
        Sb[2] = ob[0] + ob[1] * u + ob[2] * v + ob[3] * 0.5 * q2;
        Sb[3] = ob[0] + ob[1] * u + ob[2] * (v + c) + ob[3] * (H + v * c);
    }
    // ---- reverse: WENO-Z reconstructions and the LF split, per characteristic field
    double S[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double fp[6], fm[6], fpb[6] = {0, 0, 0, 0, 0, 0}, fmb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            fp[p] = 0.5 * (RFs(p, k) + alpha * RQs(p, k));
            fm[p] = 0.5 * (RFs(p, k) - alpha * RQs(p, k));
        }
        // left_r = ReconstructLeft(fp4, fp3, fp2, fp1, fp0); right_l = ReconstructLeft(fm1..fm5)
        double gl[5] = {0, 0, 0, 0, 0}, gr[5] = {0, 0, 0, 0, 0};
        S[k] = recon_left_vjp(fp[4], fp[3], fp[2], fp[1], fp[0], Sb[k], eps, delta, gl) +
               recon_left_vjp(fm[1], fm[2], fm[3], fm[4], fm[5], Sb[k], eps, delta, gr);
        fpb[4] += gl[0], fpb[3] += gl[1], fpb[2] += gl[2], fpb[1] += gl[3], fpb[0] += gl[4];
        fmb[1] += gr[0], fmb[2] += gr[1], fmb[3] += gr[2], fmb[4] += gr[3], fmb[5] += gr[4];
#pragma unroll
        for (int p = 0; p < 6; ++p) {  // column k is not read again: its adjoints replace it
            RFs(p, k) = 0.5 * (fpb[p] + fmb[p]);
            RQs(p, k) = 0.5 * alpha * (fpb[p] - fmb[p]);
        }
    }
    RoeAdj P{0, 0, 0, 0, 0};
    if (DIR == 0) {
        P.u += ob[1] * (S[0] + S[2] + S[3]) + ob[3] * (-S[0] * c + S[2] * u + S[3] * c);
        P.v += ob[2] * (S[0] + S[2] + S[3]) + ob[3] * (S[1] + S[2] * v);
        P.c += ob[1] * (S[3] - S[0]) + ob[3] * u * (S[3] - S[0]);
    } else {
        P.u += ob[1] * (S[0] + S[2] + S[3]) + ob[3] * (S[1] + S[2] * u);
        P.v += ob[2] * (S[0] + S[2] + S[3]) + ob[3] * (-S[0] * c + S[2] * v + S[3] * c);
        P.c += ob[2] * (S[3] - S[0]) + ob[3] * v * (S[3] - S[0]);
    }
    P.H += ob[3] * (S[0] + S[3]);
    // ---- reverse: characteristic projections and physical fluxes
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        double f[4], fb[4] = {0, 0, 0, 0}, rqb[4], rfb[4];
        flux2<DIR>(s[p], g, f);  // recomputed rather than kept live across the WENO-Z reverse
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            rqb[k] = RQs(p, k);
            rfb[k] = RFs(p, k);
        }
        inv2_vjp<DIR>(R, s[p], rqb, gs[p], P);
        inv2_vjp<DIR>(R, f, rfb, fb, P);
        flux2_vjp<DIR>(s[p], g, fb, gs[p]);
    }
    // ---- reverse: Roe average (kc = 0.4 / c^2, c = sqrt(0.4 (H - q2/2)))
    P.c += P.kc * (-2.0 * R.kc / R.c);
    const double ccb = P.c * 0.5 / R.c;
    P.H += 0.4 * ccb;
    const double q2b = -0.2 * ccb;
    P.u += 2 * R.u * q2b;
    P.v += 2 * R.v * q2b;
    const double Ub = P.u * iden, Vb = P.v * iden, HHb = P.H * iden;
    const double denb = -(P.u * R.u + P.v * R.v + P.H * R.H) * iden;
    double sLb = Ub * uL + Vb * vL + HHb * HL + denb;
    double sRb = Ub * uR + Vb * vR + HHb * HR + denb;
    const double uLb = Ub * sL, uRb = Ub * sR, vLb = Vb * sL, vRb = Vb * sR, HLb = HHb * sL, HRb = HHb * sR;
    // H = (q3 + p)/q0, u = q1/q0, v = q2/q0, p = gm1 (q3 - K/(2 q0)), s = sqrt(q0)
    auto side = [&](const double* q, double iq0, double K, double Hs, double us, double vs, double sq, double sb,
                    double ub, double vb, double hb, double* qb) {
        qb[0] += sb * 0.5 / sq;
        qb[1] += ub * iq0;
        qb[0] -= ub * us * iq0;
        qb[2] += vb * iq0;
        qb[0] -= vb * vs * iq0;
        qb[3] += hb * iq0;
        const double pb = hb * iq0;
        qb[0] -= hb * Hs * iq0;
        qb[3] += gm1 * pb;
        const double Kb = -0.5 * gm1 * pb * iq0;
        qb[0] += 0.5 * gm1 * pb * K * iq0 * iq0;
        qb[1] += 2 * q[1] * Kb;
        qb[2] += 2 * q[2] * Kb;
    };
    side(L, iL0, KL, HL, uL, vL, sL, sLb, uLb, vLb, HLb, gs[2]);
    side(Rr, iR0, KR, HR, uR, vR, sR, sRb, uRb, vRb, HRb, gs[3]);
}

__device__ __forceinline__ bool fin_point(const Grid2& g, const uint8_t* m, const int8_t* lvl, int i, int j, int bit)
{
    if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) return false;
    const size_t a = g.at(i, j);
    return ((m[a] >> bit) & 1u) && lvl[a] == g.maxl;
}

// Face VJP over the stage's face list: the weight of face f (between f and f+1 along DIR) is
// nu(f) for a finest-level point f (R_f += F_f) minus nu(f+1) for a finest point f+1
// (R_{f+1} -= F_f); lam -= weight . dF_f/dcells.
#ifndef AWCM_ADJ_MIN_CTAS
#define AWCM_ADJ_MIN_CTAS 1  // 255 registers and 2 CTAs per SM; forcing more CTAs spills and runs slower
#endif
template <int DIR>
__global__ void __launch_bounds__(kAdjThreads, AWCM_ADJ_MIN_CTAS) k_adj_face(AdjStage A, const uint32_t* __restrict__ list,
                                                  const unsigned* __restrict__ count,
                                                  const double* __restrict__ alpha)
{
    pdl_begin();
    __shared__ double sh[48 * kAdjThreads];
    const Grid2& g = A.g;
    const unsigned n = *count;
    const unsigned stride = gridDim.x * blockDim.x;
    const long step = DIR == 0 ? 1 : g.pitch;
    for (unsigned e = gtid(); e < n; e += stride) {
        const uint32_t idx = list[e];
        const int ii = (int)(idx % (uint32_t)g.pitch) - kGhost;
        const int jj = (int)(idx / (uint32_t)g.pitch) - kGhost;
        const int i1 = DIR == 0 ? ii + 1 : ii, j1 = DIR == 0 ? jj : jj + 1;
        double w[4] = {0, 0, 0, 0};
        bool any = false;
        if (fin_point(g, A.m, A.lvl, ii, jj, A.bit)) {
            for (int k = 0; k < 4; ++k) w[k] += A.nu.p[k][idx];
            any = true;
        }
        if (fin_point(g, A.m, A.lvl, i1, j1, A.bit)) {
            const size_t b = (size_t)idx + step;
            for (int k = 0; k < 4; ++k) w[k] -= A.nu.p[k][b];
            any = true;
        }
        if (!any || (w[0] == 0 && w[1] == 0 && w[2] == 0 && w[3] == 0)) continue;
        double s[6][4], gs[6][4];
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            const long a = (long)idx + (p - 2) * step;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                s[p][k] = A.qin.p[k][a];
                gs[p][k] = 0;
            }
        }
        const double al = DIR == 0 ? alpha[jj] : alpha[ii];
        face_flux_2d_vjp<DIR>(s, al, g.gamma, w, g.wz_eps, g.wz_delta, gs, sh + threadIdx.x);
#pragma unroll
        for (int p = 0; p < 6; ++p) {
            const long a = (long)idx + (p - 2) * step;
#pragma unroll
            for (int k = 0; k < 4; ++k) atomic_sub(&A.lam.p[k][a], gs[p][k]);
        }
    }
}

// Coarse points: R = dF + dG from physical fluxes at spacing d (central, or the reference's
// one-sided forms at the edges; same branch selection as the forward).
__global__ void __launch_bounds__(256) k_adj_coarse(AdjStage A)
{
    pdl_begin();
    const Grid2& g = A.g;
    const unsigned n = *A.ncrs;
    const unsigned stride = gridDim.x * blockDim.x;
    const int NX = g.nx - 1, NY = g.ny - 1;
    for (unsigned e = gtid(); e < n; e += stride) {
        const size_t a = A.crs[e];
        const int i = (int)((unsigned)a % (unsigned)g.pitch) - kGhost;
        const int j = (int)((unsigned)a / (unsigned)g.pitch) - kGhost;
        const int lev = A.lvl[a];
        if (lev < 0 || lev >= g.maxl) continue;
        const int d = g.D(lev);
        // same skip as the forward: stencils that would leave the ghosted grid
        const int lo_x = i <= d ? i - d : i - 2 * d, hi_x = i >= NX - d && !(i <= d) ? i + d : i + 2 * d;
        const int lo_y = j <= d ? j - d : j - 2 * d, hi_y = j >= NY - d && !(j <= d) ? j + d : j + 2 * d;
        if (lo_x < -kGhost || hi_x > NX + kGhost || lo_y < -kGhost || hi_y > NY + kGhost) continue;
        double nu[4];
        for (int k = 0; k < 4; ++k) nu[k] = A.nu.p[k][a];
        if (nu[0] == 0 && nu[1] == 0 && nu[2] == 0 && nu[3] == 0) continue;
        for (int dir = 0; dir < 2; ++dir) {
            const int pos = dir == 0 ? i : j, N1 = dir == 0 ? NX : NY;
            const long st = dir == 0 ? 1 : g.pitch;
            // weights of F at offsets -2d, -d, +d, +2d
            double wm2 = 0, wm1 = -kD1, wp1 = kD1, wp2 = 0;
            if (pos <= d) {
                wp2 += kD2;
                wm1 -= kD2;
            } else if (pos >= N1 - d) {
                wp1 += kD2;
                wm2 -= kD2;
            } else {
                wp2 += kD2;
                wm2 -= kD2;
            }
            const int offs[4] = {-2, -1, 1, 2};
            const double ws[4] = {wm2, wm1, wp1, wp2};
            for (int o = 0; o < 4; ++o) {
                if (ws[o] == 0) continue;
                const long b = (long)a + offs[o] * d * st;
                double q[4], fb[4], qb[4] = {0, 0, 0, 0};
                for (int k = 0; k < 4; ++k) {
                    q[k] = A.qin.p[k][b];
                    fb[k] = ws[o] * nu[k];
                }
                if (dir == 0) flux2_vjp<0>(q, g.gamma, fb, qb);
                else flux2_vjp<1>(q, g.gamma, fb, qb);
                for (int k = 0; k < 4; ++k) atomic_sub(&A.lam.p[k][b], qb[k]);
            }
        }
    }
}

// RK combination adjoints, one dense pass per stage over the plane (points off the grid are
// ghosts and carry no state).  stage 3: lam_n = lam_next (1/3 on mask0), lam_in = 2/3 lam_next
// on mask0, nu = s lam_in; stage 2: lam_n += 3/4 lam_in' on mask1, lam_in = 1/4 lam_in', nu = s
// lam_in (lam_in' = the adjoint of Q1 from stage 3, passed as lam_next); stage 1: lam_n += lam_Q2
// on mask2, nu = s lam_Q2.
__global__ void k_adj_rk(int stage, Grid2 g, size_t plane, const uint8_t* __restrict__ m,
                         const int8_t* __restrict__ lvl, const double* __restrict__ sc, Field4 lam_next, Field4 lam_n,
                         Field4 lam_in, Field4 nu)
{
    pdl_begin();
    const unsigned a = gtid();
    if (a >= plane) return;
    const int i = (int)(a % (unsigned)g.pitch) - kGhost, j = (int)(a / (unsigned)g.pitch) - kGhost;
    const bool grid = i >= 0 && i < g.nx && j >= 0 && j < g.ny;
    const int bit = stage == 3 ? 0 : (stage == 2 ? 1 : 2);
    const bool on = grid && ((m[a] >> bit) & 1u);
    const int lv = on ? lvl[a] : -1;
    const double s = (lv >= 0 && lv <= g.maxl) ? sc[lv] : 0.0;
    // every plane is read before any is written (the round trips of the four components overlap)
    double x[4], ln[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = grid ? lam_next.p[k][a] : 0.0;
    if (stage != 3 && on)
#pragma unroll
        for (int k = 0; k < 4; ++k) ln[k] = lam_n.p[k][a];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (stage == 3) {
            lam_n.p[k][a] = on ? x[k] / 3.0 : x[k];
            const double y = on ? 2.0 * x[k] / 3.0 : 0.0;
            lam_in.p[k][a] = y;
            nu.p[k][a] = s * y;
        } else if (stage == 2) {
            if (on) lam_n.p[k][a] = ln[k] + 0.75 * x[k];
            const double y = on ? 0.25 * x[k] : 0.0;
            lam_in.p[k][a] = y;
            nu.p[k][a] = s * y;
        } else {
            if (on) lam_n.p[k][a] = ln[k] + x[k];
            nu.p[k][a] = on ? s * x[k] : 0.0;
        }
    }
}

// Adjoint of the boundary fill: every ghost's adjoint moves to the interior point it was copied
// from (transmissive: the edge point; periodic: the wrapped point; double Mach: the transmissive
// right edge and the reflecting bottom for x > 1/6, sign flip on rho v; shock-vortex: the
// reflecting bottom and top, sign flip on rho v; prescribed states carry no adjoint).  One thread
// per ghost cell of the edge strips; several ghosts share a source (and the corner points are the
// source of a row ghost and a column ghost), so sources are updated atomically.
__global__ void k_adj_fold(Grid2 g, Field4 lam)
{
    pdl_begin();
    const long t = (long)gtid();
    const int NX = g.nx - 1, NY = g.ny - 1;
    const bool per = g.bc_kind == AWCM_BC_PERIODIC, dm = g.bc_kind == AWCM_BC_DOUBLE_MACH;
    const bool sv = g.bc_kind == AWCM_BC_SHOCK_VORTEX;  // walls at the bottom and top: rho v flips
    const long nside = (long)kGhost * g.ny, nbt = (long)kGhost * g.nx;
    size_t gh, src;
    bool take = true;    // false: a prescribed state, the adjoint is dropped
    double sg2 = 1.0;    // sign applied to component 2 (rho v)
    if (t < 2 * nside) {
        const bool right = t >= nside;
        const long r = right ? t - nside : t;
        const int j = (int)(r / kGhost), c = (int)(r % kGhost);
        if (!right) {
            gh = g.at(-1 - c, j);
            src = g.at(per ? NX - c : 0, j);
            take = !dm;
        } else {
            gh = g.at(NX + 1 + c, j);
            src = g.at(per ? c : NX, j);
        }
    } else if (t < 2 * nside + 2 * nbt) {
        const long r0 = t - 2 * nside;
        const bool top = r0 >= nbt;
        const long r = top ? r0 - nbt : r0;
        const int i = (int)(r / kGhost), c = (int)(r % kGhost);
        if (!top) {
            gh = g.at(i, -1 - c);
            src = g.at(i, per ? NY - c : 0);
            if (dm) take = g.x_min + i * g.dx > 1.0 / 6.0;
            if (dm || sv) sg2 = -1.0;
        } else {
            gh = g.at(i, NY + 1 + c);
            src = g.at(i, per ? c : NY);
            take = !dm;
            if (sv) sg2 = -1.0;
        }
    } else {
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double v = lam.p[k][gh];
        if (take) atomic_add(&lam.p[k][src], (k == 2 ? sg2 : 1.0) * v);
        lam.p[k][gh] = 0;
    }
}

// Loss and seed over the active points (mask0; the other points carry no solution value):
// lam = rho - target on mask0 points (component 0), 0 elsewhere on the grid; the loss
// 1/2 sum (rho - target)^2 is reduced in a fixed order (one CTA per row: strided partial sums, then
// a shared-memory tree; the rows likewise), so it is reproducible from run to run.
constexpr int kSeedThreads = 256;
__device__ __forceinline__ double block_sum_fixed(double v, double* sh)
{
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = kSeedThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    return sh[0];
}

__global__ void __launch_bounds__(kSeedThreads) k_adj_seed(Grid2 g, Field4 q, const uint8_t* __restrict__ m,
                                                            const double* __restrict__ target, Field4 lam,
                                                            double* rowsum)
{
    pdl_begin();
    __shared__ double sh[kSeedThreads];
    const int j = (int)blockIdx.x;
    double acc = 0;
    for (int i = threadIdx.x; i < g.nx; i += kSeedThreads) {
        const size_t a = g.at(i, j);
        const double d = (m[a] & 1u) ? q.p[0][a] - target[(size_t)j * g.nx + i] : 0.0;
        acc += 0.5 * d * d;
        lam.p[0][a] = d;
        lam.p[1][a] = lam.p[2][a] = lam.p[3][a] = 0;
    }
    const double r = block_sum_fixed(acc, sh);
    if (threadIdx.x == 0) rowsum[j] = r;
}

__global__ void __launch_bounds__(kSeedThreads) k_sum_rows(const double* rowsum, int n, double* loss)
{
    pdl_begin();
    __shared__ double sh[kSeedThreads];
    double acc = 0;
    for (int j = threadIdx.x; j < n; j += kSeedThreads) acc += rowsum[j];
    const double r = block_sum_fixed(acc, sh);
    if (threadIdx.x == 0) *loss = r;
}

}  // namespace

void adj_launch_stage(const AdjStage& a, int face_blocks, cudaStream_t s)
{
    // 16 CTAs per SM over the face list (2 resident): 0.9 % faster reverse sweep than 8
    launch_pdl(k_adj_face<0>, 2 * face_blocks, kAdjThreads, s, a, a.xf, a.nxf, a.ax);
    launch_pdl(k_adj_face<1>, 2 * face_blocks, kAdjThreads, s, a, a.yf, a.nyf, a.ay);
    launch_pdl(k_adj_coarse, face_blocks / 2, 256, s, a);
}

void adj_launch_rk(int stage, const Grid2& g, size_t plane, const uint8_t* m, const int8_t* lvl, const double* sc,
                   Field4 lam_next, Field4 lam_n, Field4 lam_in, Field4 nu, cudaStream_t s)
{
    launch_pdl(k_adj_rk, (unsigned)((plane + 255) / 256), 256, s, stage, g, plane, m, lvl, sc, lam_next, lam_n, lam_in, nu);
}

void adj_launch_fold(const Grid2& g, Field4 lam, cudaStream_t s)
{
    const long n = 2L * kGhost * (g.nx + g.ny);
    launch_pdl(k_adj_fold, (unsigned)((n + 255) / 256), 256, s, g, lam);
}

void adj_launch_seed(const Grid2& g, Field4 q, const uint8_t* m, const double* target, Field4 lam, double* rowsum,
                     double* loss, cudaStream_t s)
{
    launch_pdl(k_adj_seed, (unsigned)g.ny, kSeedThreads, s, g, q, m, target, lam, rowsum);
    launch_pdl(k_sum_rows, 1, kSeedThreads, s, (const double*)rowsum, g.ny, loss);
}

}  // namespace awcm

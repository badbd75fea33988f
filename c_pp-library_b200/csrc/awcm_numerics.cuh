// Device numerics of the AWCM compressible-Euler path: ideal-gas relations, physical fluxes,
// Roe-averaged characteristic projection, WENO-Z / WENO5 reconstruction and the Lax-Friedrichs
// split face flux.  Every expression keeps the reference's operation order (doseongju/C_pp-library),
// and the library is compiled with --fmad=false, so each result is bit-identical to the
// reference's IEEE double arithmetic: division and square root are the correctly rounded ones.
#pragma once
#include <cstdint>

namespace awcm {

constexpr int kGhost = 3;  // ghost width of every field (FIELD_UNIFORM_1D/2D ghost_width 3)

// 11/6, -7/6, 1/3, 5/6, -1/6, 13/12 correctly rounded (the reference builds them as 11.0/6.0, ...).
constexpr double kC11_6 = 0x1.d555555555555p+0;
constexpr double kCm7_6 = -0x1.2aaaaaaaaaaabp+0;
constexpr double kC1_3 = 0x1.5555555555555p-2;
constexpr double kC5_6 = 0x1.aaaaaaaaaaaabp-1;
constexpr double kCm1_6 = -0x1.5555555555555p-3;
constexpr double kC13_12 = 0x1.1555555555555p+0;
// Coarse-level derivative weights of AWCM_1D/AWCM_2D (Wavelet/AWCM_1D.h:21, 36-39).
constexpr double kD1 = 0x1.5555555555555p-1;    // 2/3
constexpr double kD2 = -0x1.5555555555555p-4;   // -1/12
constexpr double kD01 = -0x1.5555555555555p-2;  // -1/3
constexpr double kD11 = -0.5;
constexpr double kD21 = 1.0;
constexpr double kD31 = -0x1.5555555555555p-3;  // -1/6
constexpr double kD02 = 0x1.5555555555555p-4;   // 1/12
constexpr double kD12 = -0x1.5555555555555p-1;  // -2/3
constexpr double kD22 = 0.0;
constexpr double kD32 = 0x1.5555555555555p-1;   // 2/3

enum Scheme : int { kWenoZ = 0, kWeno5 = 1, kScalarAdvection = 2 };  // 2: the 1D scalar path only

__device__ __forceinline__ double sqr(double x) { return x * x; }
__device__ __forceinline__ double absd(double x) { return x < 0 ? -x : x; }
__device__ __forceinline__ double maxd(double a, double b) { return a > b ? a : b; }

// WENOZ5::ReconstructLeft (WENOZ.h:75-104): tau = |b0 - b2|, alpha_k = d_k (1 + tau/(b_k + eps)),
// eps = 1e-40.  WENO5::ReconstructLeft (WENO.h:71-99): alpha_k = d_k / (eps + b_k)^2, eps = 1e-6.
// wz_eps: WENOZ5::eps (WENOZ.h:13-18), a public member of the reference solver, 1e-40 by default.
// wz_delta > 0 replaces tau = |b0 - b2| by sqrt((b0 - b2)^2 + wz_delta^2) (the differentiable
// mode of the gradient checks; the reference has only |.|).
template <int SCHEME>
__device__ __forceinline__ double recon_left(double ll, double l, double c, double r, double rr,
                                             double wz_eps = 1e-40, double wz_delta = 0.0)
{
    const double b0 = kC13_12 * sqr(c - 2 * r + rr) + 0.25 * sqr(3 * c - 4 * r + rr);
    const double b1 = kC13_12 * sqr(l - 2 * c + r) + 0.25 * sqr(l - r);
    const double b2 = kC13_12 * sqr(ll - 2 * l + c) + 0.25 * sqr(ll - 4 * l + 3 * c);
    double w0, w1, w2;
    if (SCHEME == kWeno5) {
        const double eps = 1e-6;
        const double a0 = 0.1 / sqr(eps + b0);
        const double a1 = 0.6 / sqr(eps + b1);
        const double a2 = 0.3 / sqr(eps + b2);
        const double s = a0 + a1 + a2;
        w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
    } else {
        const double eps = wz_eps;
        const double tau = wz_delta > 0 ? sqrt(sqr(b0 - b2) + sqr(wz_delta)) : absd(b0 - b2);
        const double d0 = b0 + eps, d1 = b1 + eps, d2 = b2 + eps;
        if (tau == 0 && d0 > 0 && d1 > 0 && d2 > 0) {
            // tau / d_k is a signed zero and 1 + (+-0) = 1, so alpha_k = d_k exactly; their sum
            // 0.1 + 0.6 + 0.3 rounds to exactly 1.0 in IEEE double, so the normalised weights are
            // the d_k themselves.  All six divisions are skipped (a zero quotient sends IEEE
            // division down its slow path, and piecewise-constant stencils make tau = 0 common).
            w0 = 0.1, w1 = 0.6, w2 = 0.3;
        } else {
            const double a0 = 0.1 * (1 + tau / d0);
            const double a1 = 0.6 * (1 + tau / d1);
            const double a2 = 0.3 * (1 + tau / d2);
            const double s = a0 + a1 + a2;
            w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
        }
    }
    double left = w0 * (kC11_6 * c + kCm7_6 * r + kC1_3 * rr);
    left += w1 * (kC1_3 * l + kC5_6 * c + kCm1_6 * r);
    left += w2 * (kCm1_6 * ll + kC5_6 * l + kC1_3 * c);
    return left;
}

// ------------------------------------------------------------------------------------ 1D gas
// IDEAL_GAS_1D (IDEAL_GAS_EQUATIONS.h:8-58), EULER_EQUATION_1D::ComputeFu (EULER_EQUATION.h:16-26).
__device__ __forceinline__ double pressure1(double q0, double q1, double q2, double g)
{
    return (g - 1) * (q2 - 0.5 * sqr(q1) / q0);
}
__device__ __forceinline__ double sound1(double q0, double q1, double q2, double g)
{
    return sqrt(g * pressure1(q0, q1, q2, g) / q0);
}
__device__ __forceinline__ void flux1(const double* q, double g, double* f)
{
    const double rho = q[0], u = q[1] / q[0], E = q[2], p = pressure1(q[0], q[1], q[2], g);
    f[0] = rho * u;
    f[1] = rho * u * u + p;
    f[2] = (E + p) * u;
}

// ROE_SOLVER_1D::Inversion (ROESOLVER.h:27-36), with 0.4/(c*c) precomputed as kc (same value).
__device__ __forceinline__ void inv1(double u, double H, double c, double kc, const double* b, double* x)
{
    double x2 = (H - u * u) * b[0] + u * b[1] - b[2];
    x2 *= kc;
    double x3 = b[1] + (c - u) * b[0] - c * x2;
    x3 /= 2 * c;
    x[0] = b[0] - x2 - x3;
    x[1] = x2;
    x[2] = x3;
}

// WENOZ_EULER_SOLVER_1D::ComputeFlux (WENOZ.h:160-205) / WENO_EULER_SOLVER_1D::ComputeFlux
// (WENO.h:129-174).  s[p] are the six cells -3..+2 of the face, alpha the LF speed.
template <int SCHEME>
__device__ __forceinline__ void face_flux_1d(const double (&s)[6][3], double alpha, double g, double* out)
{
    const double* l = s[2];
    const double* r = s[3];
    const double rho_l = l[0], rho_r = r[0];
    const double u_l = l[1] / l[0], u_r = r[1] / r[0];
    const double H_l = (l[2] + pressure1(l[0], l[1], l[2], g)) / l[0];
    const double H_r = (r[2] + pressure1(r[0], r[1], r[2], g)) / r[0];
    const double sl = sqrt(rho_l), sr = sqrt(rho_r);
    const double den = sl + sr;
    double u = sl * u_l + sr * u_r;
    u /= den;
    double H = sl * H_l + sr * H_r;
    H /= den;
    const double c = sqrt((g - 1) * (H - 0.5 * u * u));
    const double kc = 0.4 / (c * c);
    double fp[6][3], fm[6][3];
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        double f[3], RQ[3], RF[3];
        flux1(s[p], g, f);
        inv1(u, H, c, kc, s[p], RQ);
        inv1(u, H, c, kc, f, RF);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            fp[p][k] = 0.5 * (RF[k] + alpha * RQ[k]);
            fm[p][k] = 0.5 * (RF[k] - alpha * RQ[k]);
        }
    }
    double S[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double lr = recon_left<SCHEME>(fp[4][k], fp[3][k], fp[2][k], fp[1][k], fp[0][k]);
        const double rl = recon_left<SCHEME>(fm[1][k], fm[2][k], fm[3][k], fm[4][k], fm[5][k]);
        S[k] = lr + rl;
    }
    const double r1[3] = {1, u - c, H - u * c};
    const double r2[3] = {1, u, 0.5 * (u * u)};
    const double r3[3] = {1, u + c, H + u * c};
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = S[0] * r1[k] + S[1] * r2[k] + S[2] * r3[k];
}

// ------------------------------------------------------------------------------------ 2D gas
// IDEAL_GAS_2D (IDEAL_GAS_EQUATIONS.h:60-111), EULER_EQUATION_2D (EULER_EQUATION.h:64-156).
__device__ __forceinline__ double pressure2(double q0, double q1, double q2, double q3, double g)
{
    return (g - 1) * (q3 - 0.5 * (sqr(q1) + sqr(q2)) / q0);
}
__device__ __forceinline__ double sound2(const double* q, double g)
{
    return sqrt(g * pressure2(q[0], q[1], q[2], q[3], g) / q[0]);
}
// DIR 0: ComputeFu (F), DIR 1: ComputeGu (G).
template <int DIR>
__device__ __forceinline__ void flux2(const double* q, double g, double* f)
{
    const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
    const double p = pressure2(q[0], q[1], q[2], q[3], g);
    if (DIR == 0) {
        f[0] = rho * u;
        f[1] = rho * u * u + p;
        f[2] = rho * v * u;
        f[3] = (E + p) * u;
    } else {
        f[0] = rho * v;
        f[1] = rho * u * v;
        f[2] = rho * v * v + p;
        f[3] = (E + p) * v;
    }
}

// ROE_SOLVER_2D::Inversion_X / Inversion_Y (ROESOLVER.h:73-96); kc = 0.4 / c / c, same value.
template <int DIR>
__device__ __forceinline__ void inv2(double u, double v, double H, double c, double kc, const double* b, double* x)
{
    double x3;
    if (DIR == 0) x3 = (H - u * u - v * v) * b[0] + u * b[1] + v * b[2] - b[3];
    else x3 = (H - u * u - v * v) * b[0] + v * b[2] + u * b[1] - b[3];
    x3 *= kc;
    const double x2 = DIR == 0 ? b[2] - v * b[0] : b[1] - u * b[0];
    double x4 = DIR == 0 ? b[1] + (c - u) * b[0] - c * x3 : b[2] + (c - v) * b[0] - c * x3;
    x4 /= 2 * c;
    x[0] = b[0] - x3 - x4;
    x[1] = x2;
    x[2] = x3;
    x[3] = x4;
}

// Roe average of the two face states (ROE_SOLVER_2D::RoeAverage, ROESOLVER.h:49-70).
struct Roe2 {
    double u, v, H, c, kc;
};
__device__ __forceinline__ Roe2 roe2(const double* l, const double* r, double g)
{
    Roe2 o;
    const double rho_l = l[0], rho_r = r[0];
    const double H_l = (l[3] + pressure2(l[0], l[1], l[2], l[3], g)) / l[0];
    const double H_r = (r[3] + pressure2(r[0], r[1], r[2], r[3], g)) / r[0];
    const double u_l = l[1] / l[0], u_r = r[1] / r[0];
    const double v_l = l[2] / l[0], v_r = r[2] / r[0];
    const double sl = sqrt(rho_l), sr = sqrt(rho_r);
    const double den = sl + sr;
    double u = sl * u_l + sr * u_r;
    u /= den;
    double v = sl * v_l + sr * v_r;
    v /= den;
    double H = sl * H_l + sr * H_r;
    H /= den;
    o.u = u;
    o.v = v;
    o.H = H;
    o.c = sqrt(0.4 * (H - 0.5 * (u * u + v * v)));
    o.kc = 0.4 / o.c / o.c;
    return o;
}

// WENOZ_EULER_SOLVER_2D::ComputeFluxX (DIR 0) / ComputeFluxY (DIR 1), WENOZ.h:236-320.
// s[p] = cells -3..+2 across the face along DIR.
template <int DIR>
__device__ __forceinline__ void face_flux_2d(const double (&s)[6][4], double alpha, double g, double* out,
                                             double wz_eps = 1e-40, double wz_delta = 0.0)
{
    const Roe2 R = roe2(s[2], s[3], g);
    double fp[6][4], fm[6][4];
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        double f[4], RQ[4], RF[4];
        flux2<DIR>(s[p], g, f);
        inv2<DIR>(R.u, R.v, R.H, R.c, R.kc, s[p], RQ);
        inv2<DIR>(R.u, R.v, R.H, R.c, R.kc, f, RF);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            fp[p][k] = 0.5 * (RF[k] + alpha * RQ[k]);
            fm[p][k] = 0.5 * (RF[k] - alpha * RQ[k]);
        }
    }
    double S[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double lr = recon_left<kWenoZ>(fp[4][k], fp[3][k], fp[2][k], fp[1][k], fp[0][k], wz_eps, wz_delta);
        const double rl = recon_left<kWenoZ>(fm[1][k], fm[2][k], fm[3][k], fm[4][k], fm[5][k], wz_eps, wz_delta);
        S[k] = lr + rl;
    }
    const double u = R.u, v = R.v, H = R.H, c = R.c;
    double r1[4], r2[4], r3[4], r4[4];
    if (DIR == 0) {
        r1[0] = 1, r2[0] = 0, r3[0] = 1, r4[0] = 1;
        r1[1] = u - c, r2[1] = 0, r3[1] = u, r4[1] = u + c;
        r1[2] = v, r2[2] = 1, r3[2] = v, r4[2] = v;
        r1[3] = H - u * c, r2[3] = v, r3[3] = 0.5 * (u * u + v * v), r4[3] = H + u * c;
    } else {
        r1[0] = 1, r2[0] = 0, r3[0] = 1, r4[0] = 1;
        r1[1] = u, r2[1] = 1, r3[1] = u, r4[1] = u;
        r1[2] = v - c, r2[2] = 0, r3[2] = v, r4[2] = v + c;
        r1[3] = H - v * c, r2[3] = u, r3[3] = 0.5 * (u * u + v * v), r4[3] = H + v * c;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = S[0] * r1[k] + S[1] * r2[k] + S[2] * r3[k] + S[3] * r4[k];
}

}  // namespace awcm

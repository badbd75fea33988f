// TEST INFRASTRUCTURE ONLY -- CPU restatement (the "oracle") of the reference's adaptive
// wavelet collocation (AWCM) compressible-Euler path, doseongju/C_pp-library.
//
// Written from the reference's algorithm, not copied: dense structure-of-arrays fields with a
// ghost ring of 3, one byte per point holding the significance masks as bits, and the same
// floating-point operation order as the reference so results are bit-identical to it (pinned by
// tests/test_oracle_vs_reference.py against the reference itself, compiled by oracle/Makefile).
// Build flags: -O2 -ffp-contract=off (no FMA), no fast-math.
//
// Mask bits per point: 0..3 = mask0..mask3, 4 = mask_temp (the previous step's mask0),
// 5 = interpolation work mask, 6 = copy read by the add-adjacent-zone / differentiation passes.
#include "awcm_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <omp.h>
#include <vector>

namespace {

constexpr int G = 3;  // ghost width of every field (FIELD_UNIFORM_1D/2D ghost_width 3)
constexpr double C11_6 = 11.0 / 6.0, CM7_6 = -7.0 / 6.0, C1_3 = 1.0 / 3.0, C5_6 = 5.0 / 6.0, CM1_6 = -1.0 / 6.0;
constexpr double C13_12 = 13.0 / 12.0;

// ---------------------------------------------------------------------------------------------
// Lifted 4-point interpolating-wavelet weights: w[i][j+1] = l_i(j + 1/2), the Lagrange basis on
// nodes 0..3 evaluated between nodes, built by the same running product as WAVELET_1D::Initialize
// (Wavelet/WAVELET_1D.h:26-42) and WAVELET_2D's constructor (Wavelet/WAVELET_2D.h:17-33).
// Column k = 0, 1, 2 of the transforms is j = 0, 1, 2, i.e. w[cnt][k + 1].
struct Weights {
    double w[4][5];
    Weights()
    {
        for (int j = -1; j < 4; ++j)
            for (int i = 0; i < 4; ++i) {
                double v = 1;
                for (int k = 0; k < 4; ++k) {
                    if (k == i) continue;
                    v *= (j + 0.5 - k) / (i - k);
                }
                w[i][j + 1] = v;
            }
    }
    double operator()(int cnt, int k) const { return w[cnt][k + 1]; }
};
const Weights W;

inline double sqr(double x) { return x * x; }
inline double absd(double x) { return x < 0 ? -x : x; }
inline double maxd(double a, double b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------------------------
// Reconstruction.  WENOZ5::ReconstructLeft (WENOZ.h:75-104): Z weights with tau = |b0 - b2| and
// exponent 1, eps 1e-40.  WENO5::ReconstructLeft (WENO.h:71-99): classic weights, eps 1e-6.
// ReconstructRight(a,b,c,d,e) is ReconstructLeft(e,d,c,b,a) in both (WENOZ.h:106-108, WENO.h:101-104).
inline double recon_left(double ll, double l, double c, double r, double rr, int scheme, double wz_eps = 1e-40,
                          double wz_delta = 0.0)
{
    const double b0 = C13_12 * sqr(c - 2 * r + rr) + 0.25 * sqr(3 * c - 4 * r + rr);
    const double b1 = C13_12 * sqr(l - 2 * c + r) + 0.25 * sqr(l - r);
    const double b2 = C13_12 * sqr(ll - 2 * l + c) + 0.25 * sqr(ll - 4 * l + 3 * c);
    double a0, a1, a2;
    if (scheme == 1) {
        const double eps = 1e-6;
        a0 = 0.1 / sqr(eps + b0);
        a1 = 0.6 / sqr(eps + b1);
        a2 = 0.3 / sqr(eps + b2);
    } else {
        const double eps = wz_eps;
        const double tau = wz_delta > 0 ? std::sqrt(sqr(b0 - b2) + sqr(wz_delta)) : absd(b0 - b2);
        a0 = 0.1 * (1 + tau / (b0 + eps));
        a1 = 0.6 * (1 + tau / (b1 + eps));
        a2 = 0.3 * (1 + tau / (b2 + eps));
    }
    const double s = a0 + a1 + a2;
    const double w0 = a0 / s, w1 = a1 / s, w2 = a2 / s;
    double left = w0 * (C11_6 * c + CM7_6 * r + C1_3 * rr);
    left += w1 * (C1_3 * l + C5_6 * c + CM1_6 * r);
    left += w2 * (CM1_6 * ll + C5_6 * l + C1_3 * c);
    return left;
}

// =============================================================================================
// 1D physics: IDEAL_GAS_1D (IDEAL_GAS_EQUATIONS.h:8-58), EULER_EQUATION_1D (EULER_EQUATION.h:6-62),
// ROE_SOLVER_1D (ROESOLVER.h:9-41).
struct V3 {
    double v[3];
};

inline double p1(const double* q, double g) { return (g - 1) * (q[2] - 0.5 * sqr(q[1]) / q[0]); }
inline double c1(const double* q, double g) { return std::sqrt(g * p1(q, g) / q[0]); }
inline double h1(const double* q, double g) { return (q[2] + p1(q, g)) / q[0]; }

inline V3 fu1(const double* q, double g)
{
    const double rho = q[0], u = q[1] / q[0], E = q[2], p = p1(q, g);
    return V3{{rho * u, rho * u * u + p, (E + p) * u}};
}

inline void inv1(double u, double H, double c, const double* b, double* x)
{
    double x2 = (H - u * u) * b[0] + u * b[1] - b[2];
    x2 *= 0.4 / (c * c);
    double x3 = b[1] + (c - u) * b[0] - c * x2;
    x3 /= 2 * c;
    x[0] = b[0] - x2 - x3;
    x[1] = x2;
    x[2] = x3;
}

// Face flux from six states s[0..5] = cells -3..+2 of the face (WENOZ.h:160-205 / WENO.h:129-174).
V3 face_flux_1d(const double* const* s, double alpha, double g, int scheme)
{
    double fu[6][3], RQ[6][3], RF[6][3], fp[6][3], fm[6][3];
    for (int p = 0; p < 6; ++p) {
        V3 f = fu1(s[p], g);
        for (int k = 0; k < 3; ++k) fu[p][k] = f.v[k];
    }
    const double* l = s[2];
    const double* r = s[3];
    const double rho_l = l[0], rho_r = r[0];
    const double u_l = l[1] / l[0], u_r = r[1] / r[0];
    const double H_l = h1(l, g), H_r = h1(r, g);
    const double den = std::sqrt(rho_l) + std::sqrt(rho_r);
    double u = std::sqrt(rho_l) * u_l + std::sqrt(rho_r) * u_r;
    u /= den;
    double H = std::sqrt(rho_l) * H_l + std::sqrt(rho_r) * H_r;
    H /= den;
    const double c = std::sqrt((g - 1) * (H - 0.5 * u * u));
    const double r1[3] = {1, u - c, H - u * c}, r2[3] = {1, u, 0.5 * (u * u)}, r3[3] = {1, u + c, H + u * c};
    for (int p = 0; p < 6; ++p) {
        inv1(u, H, c, s[p], RQ[p]);
        inv1(u, H, c, fu[p], RF[p]);
    }
    for (int p = 0; p < 6; ++p)
        for (int k = 0; k < 3; ++k) {
            fp[p][k] = 0.5 * (RF[p][k] + alpha * RQ[p][k]);
            fm[p][k] = 0.5 * (RF[p][k] - alpha * RQ[p][k]);
        }
    double S[3];
    for (int k = 0; k < 3; ++k) {
        const double lr = recon_left(fp[4][k], fp[3][k], fp[2][k], fp[1][k], fp[0][k], scheme);
        const double rl = recon_left(fm[1][k], fm[2][k], fm[3][k], fm[4][k], fm[5][k], scheme);
        S[k] = lr + rl;
    }
    V3 out;
    for (int k = 0; k < 3; ++k) out.v[k] = S[0] * r1[k] + S[1] * r2[k] + S[2] * r3[k];
    return out;
}

// =============================================================================================
// 1D AWCM state.
struct O1D {
    int L = 0, maxl = 0, nxc = 0, nx = 0, w = 0;
    double gamma = 1.4, x_min = 0, dx = 0;
    int scheme = 0;
    std::vector<double> q[3], qc[3], qt[3];
    std::vector<uint8_t> m;   // mask bits per ghosted point
    std::vector<int> lv[4];  // levels, interior points
    // the enum-driven BOUNDARY_MANAGER_1D<T> (BOUNDARY_MANAGER_1D.h:17-76) when set: the condition
    // of every ghosted point (FIELD_UNIFORM_1D<BOUNDARY_CONDITION> layout)
    std::vector<int> bcf;
    int D(int lev) const { return 1 << (maxl - lev); }
    bool get(int i, int b) const { return (m[i + G] >> b) & 1; }
    void set(int i, int b)
    {
        if (i < -G || i >= nx + G) return;  // off the ghosted line: dropped (reference UB)
        m[i + G] |= (uint8_t)(1u << b);
    }
    void clr(int i, int b) { m[i + G] &= (uint8_t)~(1u << b); }
    double& Q(int p, int i) { return q[p][i + G]; }
};

void copy_bit(std::vector<uint8_t>& m, int from, int to)
{
    for (auto& x : m) x = (uint8_t)((x & ~(1u << to)) | (((x >> from) & 1u) << to));
}

// ForwardWaveletTransformEuler (Wavelet/WAVELET_1D.h:282-335): density only, thresholds mask0.
void fwt1d(O1D& s, double tol)
{
    const int N1 = s.nx - 1;
    for (int lev = s.maxl - 1; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2;
        for (int i = h; i <= N1 - h; i += D) {
            if (!s.get(i, 0)) continue;
            int is = i - D - h, k = 1;
            if (is < 0) is = 0, k = 0;
            else if (i + D + h > N1) is = N1 - 3 * D, k = 2;
            for (int cnt = 0; cnt < 4; ++cnt) s.Q(0, i) -= W(cnt, k) * s.Q(0, is + cnt * D);
            s.Q(0, i) *= 0.5;
            if (absd(s.Q(0, i)) < tol) s.clr(i, 0);
        }
        for (int i = D; i <= N1 - D; i += D) {
            if (!s.get(i, 0)) continue;
            int is = i - D - h, k = 1;
            if (is < 0) is = h, k = 0;
            else if (i + D + h > N1) is = N1 - 3 * D - h, k = 2;
            for (int cnt = 0; cnt < 4; ++cnt) s.Q(0, i) += W(cnt, k) * s.Q(0, is + cnt * D);
        }
    }
}

// InverseWaveletTransformEuler (Wavelet/WAVELET_1D.h:337-391).
void iwt1d(O1D& s, int b)
{
    const int N1 = s.nx - 1;
    for (int lev = 0; lev < s.maxl; ++lev) {
        const int D = s.D(lev), h = D / 2;
        for (int i = D; i <= N1 - D; i += D) {
            if (!s.get(i, b)) { s.Q(0, i) = 0; continue; }
            int is = i - D - h, k = 1;
            if (is < 0) is = h, k = 0;
            else if (i + D + h > N1) is = N1 - 3 * D - h, k = 2;
            for (int cnt = 0; cnt < 4; ++cnt) s.Q(0, i) -= W(cnt, k) * s.Q(0, is + cnt * D);
        }
        for (int i = h; i <= N1 - h; i += D) {
            if (!s.get(i, b)) { s.Q(0, i) = 0; continue; }
            int is = i - D - h, k = 1;
            if (is < 0) is = 0, k = 0;
            else if (i + D + h > N1) is = N1 - 3 * D, k = 2;
            s.Q(0, i) *= 2;
            for (int cnt = 0; cnt < 4; ++cnt) s.Q(0, i) += W(cnt, k) * s.Q(0, is + cnt * D);
        }
    }
}

// AWCM_MANAGER_1D::CheckReconstruction (Wavelet/AWCM_MANAGER_1D.h:45-71), in place, fine to coarse.
void cr1d(O1D& s, int b)
{
    const int N1 = s.nx - 1;
    for (int lev = s.maxl - 1; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2;
        for (int i = h; i <= N1 - h; i += D) {
            if (!s.get(i, b)) continue;
            int is = i - D - h;
            if (is < 0) is = 0;
            else if (i + D + h > N1) is = N1 - 3 * D;
            for (int cnt = 0; cnt < 4; ++cnt) s.set(is + cnt * D, b);
        }
    }
}

// AWCM_MANAGER_1D::AddAdjacentZone (Wavelet/AWCM_MANAGER_1D.h:14-43), reading a copy of the mask.
void aaz1d(O1D& s, int b)
{
    const int N1 = s.nx - 1;
    copy_bit(s.m, b, 6);
    {
        const int D = s.D(s.maxl - 1), h = D / 2;
        for (int i = h; i <= N1 - h; i += D)
            if (s.get(i, 6)) { s.set(i - 1, b); s.set(i + 1, b); }
    }
    for (int lev = s.maxl - 2; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2, q4 = D / 4;
        for (int i = h; i <= N1 - h; i += D)
            if (s.get(i, 6)) { s.set(i - q4, b); s.set(i + q4, b); }
    }
}

// AWCM_MANAGER_1D::AddPointForDifferentiation (Wavelet/AWCM_MANAGER_1D.h:73-107).
void apd1d(O1D& s, int b, int l)
{
    const int N1 = s.nx - 1;
    copy_bit(s.m, b, 6);
    for (int i = 0; i <= N1; ++i) {
        if (!s.get(i, 6)) continue;
        const int lev = s.lv[l][i];
        const int D = s.D(lev);
        const int is = i - 2 * D, ie = i + 2 * D;
        if (lev == s.maxl) {
            for (int cnt = -3; cnt < 4; ++cnt) s.set(i + cnt, b);
        } else if (is <= 0) {
            for (int cnt = 0; cnt < 6; ++cnt) s.set(cnt * D, b);
        } else if (ie >= N1) {
            for (int cnt = 0; cnt < 6; ++cnt) s.set(N1 - cnt * D, b);
        } else {
            for (int cnt = 0; cnt < 5; ++cnt) s.set(is + cnt * D, b);
        }
    }
}

// Mask read for the level search; the ghost ring of every mask is always set (the masks start
// all true, ghosts included, and no pass clears a ghost), and indices beyond it read as set.
inline bool mask_at_1d(const O1D& s, int i, int b)
{
    if (i < -G || i >= s.nx + G) return true;
    return s.get(i, b);
}

// AWCM_MANAGER_1D::ComputeLevel (Wavelet/AWCM_MANAGER_1D.h:109-133); level left as it was when no
// neighbour is found; the two end points are forced to the finest level.
void cl1d(O1D& s, int l, int b)
{
    const int N1 = s.nx - 1;
    for (int i = 1; i <= N1 - 1; ++i) {
        if (!s.get(i, b)) { s.lv[l][i] = 0; continue; }
        int dx = 1;
        for (int lev = s.maxl; lev >= 0; --lev) {
            if (mask_at_1d(s, i - dx, b) || mask_at_1d(s, i + dx, b)) { s.lv[l][i] = lev; break; }
            dx *= 2;
        }
    }
    s.lv[l][0] = s.maxl;
    s.lv[l][N1] = s.maxl;
}

// AWCM_1D::BadingBoundary (Wavelet/AWCM_1D.h:73-80): three points at each end.
void band1d(O1D& s, int b)
{
    const int N1 = s.nx - 1;
    for (int i = 0; i <= N1; ++i)
        if (!(3 <= i && i <= N1 - 3)) s.set(i, b);
}

// WAVELET_1D::InterpolateEuler(q, mra, from, to) (Wavelet/WAVELET_1D.h:393-431): momentum and
// energy at points of `to` that were not in `from`, coarse to fine.
void interp1d(O1D& s, int from, int to)
{
    const int N1 = s.nx - 1;
    copy_bit(s.m, to, 5);
    for (int i = 0; i <= N1; ++i)
        if (s.get(i, from)) s.clr(i, 5);
    cr1d(s, 5);
    for (int lev = 0; lev < s.maxl; ++lev) {
        const int D = s.D(lev), h = D / 2;
        for (int i = h; i <= N1 - h; i += D) {
            if (!s.get(i, 5) || s.get(i, from)) continue;
            int is = i - D - h, k = 1;
            if (is < 0) is = 0, k = 0;
            else if (i + D + h > N1) is = N1 - 3 * D, k = 2;
            for (int p = 1; p < 3; ++p) {
                s.Q(p, i) = 0;
                for (int cnt = 0; cnt < 4; ++cnt) s.Q(p, i) += W(cnt, k) * s.Q(p, is + cnt * D);
            }
        }
    }
}

void remove_residue_1d(O1D& s, int b)
{
    for (int i = 0; i < s.nx; ++i)
        if (!s.get(i, b)) s.Q(0, i) = s.Q(1, i) = s.Q(2, i) = 0;
}

// AWCM_1D::PrepareEuler (Wavelet/AWCM_1D.h:86-120).
void prepare1d(O1D& s, double tol)
{
    copy_bit(s.m, 0, 4);
    fwt1d(s, tol);
    band1d(s, 0);
    aaz1d(s, 0);
    cr1d(s, 0);
    for (int k = 1; k <= 3; ++k) {
        copy_bit(s.m, k - 1, k);
        cl1d(s, k - 1, k - 1);
        aaz1d(s, k);
        apd1d(s, k, k - 1);
        cr1d(s, k);
    }
    cl1d(s, 3, 3);
    iwt1d(s, 3);
    interp1d(s, 4, 3);
}

// BOUNDARY_MANAGER::SetBoundaryCondition (Problems/1D/PROBLEM_SHOCKTUBE.h:86-107): copy the end points.
// BOUNDARY_CONDITION values (BOUNDARY_MANAGER_2D.h:7-13).
constexpr int kPeriodic = -3, kExtrapolation = -2;

void bc1d(O1D& s)
{
    if (!s.bcf.empty()) {
        // BOUNDARY_MANAGER_1D<T>::SetLeft/RightBoundaryCondition (BOUNDARY_MANAGER_1D.h:47-69)
        const int N1 = s.nx - 1;
        for (int p = 0; p < 3; ++p)
            for (int c = 0; c < G; ++c) {
                const int kl = s.bcf[G - 1 - c], kr = s.bcf[N1 + G + 1 + c];
                if (kl == kExtrapolation) s.Q(p, -1 - c) = s.Q(p, 0);
                if (kl == kPeriodic) s.Q(p, -1 - c) = s.Q(p, N1 - c);
                if (kr == kExtrapolation) s.Q(p, N1 + 1 + c) = s.Q(p, N1);
                if (kr == kPeriodic) s.Q(p, N1 + 1 + c) = s.Q(p, c);
            }
        return;
    }
    for (int p = 0; p < 3; ++p)
        for (int g = 1; g <= G; ++g) {
            s.Q(p, -g) = s.Q(p, 0);
            s.Q(p, s.nx - 1 + g) = s.Q(p, s.nx - 1);
        }
}

// Coarse-level flux derivative, AWCM_1D::DifferentiateEuler* (Wavelet/AWCM_1D.h:142-189) with the
// branch selection of the driver (main_1d_euler.cpp:111-133).  The right-boundary forms are the
// left formulas on the mirrored stencil, as in the reference.
V3 coarse_dF_1d(O1D& s, int i, int d, std::vector<double>* qt)
{
    const double g = 1.4;  // EULER_EQUATION_1D euler_eqn(1.4) inside the reference's helpers
    auto F = [&](int ii) {
        const double q[3] = {qt[0][ii + G], qt[1][ii + G], qt[2][ii + G]};
        return fu1(q, g);
    };
    const double d1 = 2.0 / 3.0, d2 = -1.0 / 12.0;
    const double d01 = -1.0 / 3.0, d11 = -1.0 / 2.0, d21 = 1.0, d31 = -1.0 / 6.0;
    const double d02 = 1.0 / 12.0, d12 = -2.0 / 3.0, d22 = 0, d32 = 2.0 / 3.0;
    const int iend = s.nx - 1;
    V3 r;
    if (i - 2 * d > 0 && i + 2 * d < iend) {
        V3 fll = F(i - 2 * d), fl = F(i - d), fr = F(i + d), frr = F(i + 2 * d);
        for (int p = 0; p < 3; ++p) r.v[p] = d1 * (fr.v[p] - fl.v[p]) + d2 * (frr.v[p] - fll.v[p]);
    } else if (i - 2 * d < 0) {
        V3 a = F(i - d), b = F(i), c = F(i + d), e = F(i + 2 * d);
        for (int p = 0; p < 3; ++p) r.v[p] = d01 * a.v[p] + d11 * b.v[p] + d21 * c.v[p] + d31 * e.v[p];
    } else if (i == 2 * d) {
        V3 a = F(i - 2 * d), b = F(i - d), c = F(i), e = F(i + d), f = F(i + 2 * d);
        for (int p = 0; p < 3; ++p)
            r.v[p] = d02 * a.v[p] + d12 * b.v[p] + d22 * c.v[p] + d32 * e.v[p] + d2 * f.v[p];
    } else if (i > iend - 2 * d) {
        V3 a = F(i + d), b = F(i), c = F(i - d), e = F(i - 2 * d);
        for (int p = 0; p < 3; ++p) r.v[p] = d01 * a.v[p] + d11 * b.v[p] + d21 * c.v[p] + d31 * e.v[p];
    } else {
        V3 a = F(i + 2 * d), b = F(i + d), c = F(i), e = F(i - d), f = F(i - 2 * d);
        for (int p = 0; p < 3; ++p)
            r.v[p] = d02 * a.v[p] + d12 * b.v[p] + d22 * c.v[p] + d32 * e.v[p] + d2 * f.v[p];
    }
    return r;
}

double alpha1d(O1D& s, int b, int l)
{
    double a = 0;
    for (int i = 0; i < s.nx; ++i) {
        if (!s.get(i, b) || s.lv[l][i] != s.maxl) continue;
        const double q[3] = {s.Q(0, i), s.Q(1, i), s.Q(2, i)};
        const double u = q[1] / q[0];
        const double c = c1(q, s.gamma);
        a = maxd(a, absd(u) + c);
    }
    return a;
}

// RK3 stage over mask bit b with level set l (main_1d_euler.cpp:97-245).
void stage1d(O1D& s, int b, int l, double alpha, double dt, int kind)
{
    for (int p = 0; p < 3; ++p) s.qt[p] = s.q[p];
    for (int i = 0; i < s.nx; ++i) {
        if (!s.get(i, b)) continue;
        const int lev = s.lv[l][i];
        const int d = s.D(lev);
        V3 dF;
        if (lev == s.maxl) {
            const double* st[7];
            double buf[7][3];
            for (int o = 0; o < 7; ++o) {
                for (int p = 0; p < 3; ++p) buf[o][p] = s.qt[p][i - 3 + o + G];
                st[o] = buf[o];
            }
            V3 Fl = face_flux_1d(st, alpha, s.gamma, s.scheme);
            V3 Fr = face_flux_1d(st + 1, alpha, s.gamma, s.scheme);
            for (int p = 0; p < 3; ++p) dF.v[p] = Fr.v[p] - Fl.v[p];
        } else {
            dF = coarse_dF_1d(s, i, d, s.qt);
        }
        const double sc = dt / (s.dx * d);
        for (int p = 0; p < 3; ++p) {
            double& Q = s.Q(p, i);
            if (kind == 1) Q = Q - sc * dF.v[p];
            else if (kind == 2) Q = 0.75 * s.qc[p][i + G] + 0.25 * (Q - sc * dF.v[p]);
            else Q = (s.qc[p][i + G] + 2.0 * (Q - sc * dF.v[p])) / 3.0;
        }
    }
}

void step1d(O1D& s, double tol, double cfl, double t, double t_next, double* out)
{
    prepare1d(s, tol);
    double mv = 0;
    for (int i = 0; i < s.nx; ++i) {
        if (!s.get(i, 3)) continue;
        const double q[3] = {s.Q(0, i), s.Q(1, i), s.Q(2, i)};
        const double c = c1(q, s.gamma);
        const double u = q[1] / q[0];
        mv = maxd(mv, absd(u) + c);
    }
    double dt = cfl * s.dx / mv;
    int do_print = 0;
    if (t + dt > t_next) { dt = t_next - t; do_print = 1; }
    long cnt[4] = {0, 0, 0, 0};
    for (int i = 0; i < s.nx; ++i)
        for (int k = 0; k < 4; ++k) cnt[k] += s.get(i, k);
    bc1d(s);
    const double a1 = alpha1d(s, 3, 3);
    for (int p = 0; p < 3; ++p) s.qc[p] = s.q[p];
    stage1d(s, 2, 2, a1, dt, 1);
    bc1d(s);
    const double a2 = alpha1d(s, 2, 2);
    stage1d(s, 1, 1, a2, dt, 2);
    bc1d(s);
    const double a3 = alpha1d(s, 1, 1);
    stage1d(s, 0, 0, a3, dt, 3);
    remove_residue_1d(s, 0);
    out[0] = dt;
    out[1] = do_print;
    for (int k = 0; k < 4; ++k) out[2 + k] = (double)cnt[k];
    out[6] = a1;
    out[7] = a2;
    out[8] = a3;
    out[9] = mv;
}

// ---------------------------------------------------------------------------------------------
// 1D scalar AWCM, the path of Wavelet/main_1d_advect.cpp:48-224 (scheme 2): the field in plane 0
// of q, the stage outputs q_2, q_1, q_0 in the three planes of qc.

// AWCM_1D::Prepare (Wavelet/AWCM_1D.h:45-72): the scalar transforms (WAVELET_1D.h:90-196) are the
// Euler ones on plane 0; no mask_temp, no adjacent zones on mask1..mask3, no interpolation.
void prepare1d_scalar(O1D& s, double tol)
{
    fwt1d(s, tol);
    band1d(s, 0);
    aaz1d(s, 0);
    cr1d(s, 0);
    for (int k = 1; k <= 3; ++k) {
        copy_bit(s.m, k - 1, k);
        cl1d(s, k - 1, k - 1);
        apd1d(s, k, k - 1);
        cr1d(s, k);
    }
    cl1d(s, 3, 3);
    iwt1d(s, 3);
}

// Coarse-level derivative with the driver's branches (main_1d_advect.cpp:62-83):
// AWCM_1D::Differentiate, the 4-point DifferentiateAtLeftBoundary (Wavelet/AWCM_1D.h:127-135)
// and, at the right edge, the same on the mirrored stencil.  The driver's 6-argument
// DifferentiateAtLeftBoundary calls (i == 2 dx_, i + 2 dx_ == i_end) have no scalar overload in
// AWCM_1D; they evaluate the 5-point form of DifferentiateEulerAtLeftBoundary (AWCM_1D.h:174-185)
// with the identity flux.
double coarse_d_scalar_1d(const O1D& s, const std::vector<double>& in, int i, int d)
{
    auto Q = [&](int ii) { return in[ii + G]; };
    const double d1 = 2.0 / 3.0, d2 = -1.0 / 12.0;
    const double d02 = 1.0 / 12.0, d12 = -2.0 / 3.0, d22 = 0, d32 = 2.0 / 3.0;
    const int iend = s.nx - 1;
    if (i - 2 * d > 0 && i + 2 * d < iend) return d1 * (Q(i + d) - Q(i - d)) + d2 * (Q(i + 2 * d) - Q(i - 2 * d));
    if (i - 2 * d < 0) return d1 * (Q(i + d) - Q(i - d)) + d2 * (Q(i + 2 * d) - Q(i - d));
    if (i == 2 * d) return d02 * Q(i - 2 * d) + d12 * Q(i - d) + d22 * Q(i) + d32 * Q(i + d) + d2 * Q(i + 2 * d);
    if (i + 2 * d > iend) return d1 * (Q(i - d) - Q(i + d)) + d2 * (Q(i - 2 * d) - Q(i + d));
    return d02 * Q(i + 2 * d) + d12 * Q(i + d) + d22 * Q(i) + d32 * Q(i - d) + d2 * Q(i - 2 * d);
}

// One stage: out = in (ghosts included), then on the points of mask b with level set l
// out(i) -= dt (F_r - F_l) / (dx dx_) on the finest level (F = WENO5::ReconstructRight, WENO.h:
// 101-104) or out(i) -= dt / (dx dx_) dF below it, then the ghost copies of the end points.
// Stencils that would leave the ghosted line (only reachable from inconsistent user-set
// masks/levels) are skipped.
void scalar_stage1d(O1D& s, const std::vector<double>& in, std::vector<double>& out, int b, int l, double dt)
{
    out = in;
    auto right = [&](int c) {  // ReconstructRight(in(c-2..c+2)) = ReconstructLeft(in(c+2..c-2))
        return recon_left(in[c + 2 + G], in[c + 1 + G], in[c + G], in[c - 1 + G], in[c - 2 + G], 1);
    };
    for (int i = 0; i < s.nx; ++i) {
        if (!s.get(i, b)) continue;
        const int lev = s.lv[l][i];
        if (lev < 0 || lev > s.maxl) continue;
        const int d = s.D(lev);
        if (lev != s.maxl && (i - 2 * d < -G || i + 2 * d > s.nx - 1 + G)) continue;
        double& o = out[i + G];
        if (lev == s.maxl) {
            const double F_l = right(i - 1), F_r = right(i);
            o = o - dt * (F_r - F_l) / (s.dx * d);
        } else {
            o = o - dt / (s.dx * d) * coarse_d_scalar_1d(s, in, i, d);
        }
    }
    for (int g = 1; g <= G; ++g) {
        out[G - g] = out[G];
        out[s.nx - 1 + g + G] = out[s.nx - 1 + G];
    }
}

// One pass of the driver loop: Prepare, the stages at the fixed dt with the combinations
// q_1 = 3/4 q + 1/4 q_1 on mask1 (after q_1's ghost copies) and q = 1/3 q + 2/3 q_0 on mask0,
// then PostProcess (RemoveResidue on mask0).  q's own ghosts are never rewritten.
void scalar_step1d(O1D& s, double tol, double dt, double* out)
{
    prepare1d_scalar(s, tol);
    long cnt[4] = {0, 0, 0, 0};
    for (int i = 0; i < s.nx; ++i)
        for (int k = 0; k < 4; ++k) cnt[k] += s.get(i, k);
    std::vector<double>& q = s.q[0];
    std::vector<double>& q2 = s.qc[0];
    std::vector<double>& q1 = s.qc[1];
    std::vector<double>& q0 = s.qc[2];
    scalar_stage1d(s, q, q2, 2, 2, dt);
    scalar_stage1d(s, q2, q1, 1, 1, dt);
    for (int i = 0; i < s.nx; ++i)
        if (s.get(i, 1)) q1[i + G] = 0.75 * q[i + G] + 0.25 * q1[i + G];
    scalar_stage1d(s, q1, q0, 0, 0, dt);
    for (int i = 0; i < s.nx; ++i)
        if (s.get(i, 0)) q[i + G] = 1.0 / 3.0 * q[i + G] + 2.0 / 3.0 * q0[i + G];
    for (int i = 0; i < s.nx; ++i)
        if (!s.get(i, 0)) q[i + G] = 0;
    out[0] = dt;
    for (int k = 0; k < 4; ++k) out[1 + k] = (double)cnt[k];
}

// =============================================================================================
// 2D physics: IDEAL_GAS_2D (IDEAL_GAS_EQUATIONS.h:60-111), EULER_EQUATION_2D (EULER_EQUATION.h:64-156),
// ROE_SOLVER_2D (ROESOLVER.h:43-110).
struct V4 {
    double v[4];
};

inline double p2(const double* q, double g) { return (g - 1) * (q[3] - 0.5 * (sqr(q[1]) + sqr(q[2])) / q[0]); }
inline double c2(const double* q, double g) { return std::sqrt(g * p2(q, g) / q[0]); }
inline double h2(const double* q, double g) { return (q[3] + p2(q, g)) / q[0]; }

inline V4 fu2(const double* q, double g)
{
    const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3], p = p2(q, g);
    return V4{{rho * u, rho * u * u + p, rho * v * u, (E + p) * u}};
}

inline V4 gu2(const double* q, double g)
{
    const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3], p = p2(q, g);
    return V4{{rho * v, rho * u * v, rho * v * v + p, (E + p) * v}};
}

inline double srx(const double* q, double g) { return absd(q[1] / q[0]) + c2(q, g); }
inline double sry(const double* q, double g) { return absd(q[2] / q[0]) + c2(q, g); }

// Characteristic projection x = R^-1 b, x-direction (ROESOLVER.h:73-83) and y-direction (:86-96).
inline void invx(double u, double v, double H, double c, const double* b, double* x)
{
    double x3 = (H - u * u - v * v) * b[0] + u * b[1] + v * b[2] - b[3];
    x3 *= 0.4 / c / c;
    const double x2 = b[2] - v * b[0];
    double x4 = b[1] + (c - u) * b[0] - c * x3;
    x4 /= 2 * c;
    x[0] = b[0] - x3 - x4;
    x[1] = x2;
    x[2] = x3;
    x[3] = x4;
}

inline void invy(double u, double v, double H, double c, const double* b, double* x)
{
    double x3 = (H - u * u - v * v) * b[0] + v * b[2] + u * b[1] - b[3];
    x3 *= 0.4 / c / c;
    const double x2 = b[1] - u * b[0];
    double x4 = b[2] + (c - v) * b[0] - c * x3;
    x4 /= 2 * c;
    x[0] = b[0] - x3 - x4;
    x[1] = x2;
    x[2] = x3;
    x[3] = x4;
}

// WENOZ_EULER_SOLVER_2D::ComputeFluxX / ComputeFluxY (WENOZ.h:236-320); s[0..5] = cells -3..+2.
V4 face_flux_2d(const double* const* s, double alpha, double g, int dir, double wz_eps, double wz_delta)
{
    double f[6][4], RQ[6][4], RF[6][4], fp[6][4], fm[6][4];
    for (int p = 0; p < 6; ++p) {
        V4 t = dir == 0 ? fu2(s[p], g) : gu2(s[p], g);
        for (int k = 0; k < 4; ++k) f[p][k] = t.v[k];
    }
    const double* l = s[2];
    const double* r = s[3];
    const double rho_l = l[0], rho_r = r[0];
    const double H_l = h2(l, g), H_r = h2(r, g);
    const double u_l = l[1] / l[0], u_r = r[1] / r[0];
    const double v_l = l[2] / l[0], v_r = r[2] / r[0];
    const double den = std::sqrt(rho_l) + std::sqrt(rho_r);
    double u = std::sqrt(rho_l) * u_l + std::sqrt(rho_r) * u_r;
    u /= den;
    double v = std::sqrt(rho_l) * v_l + std::sqrt(rho_r) * v_r;
    v /= den;
    double H = std::sqrt(rho_l) * H_l + std::sqrt(rho_r) * H_r;
    H /= den;
    const double c = std::sqrt(0.4 * (H - 0.5 * (u * u + v * v)));
    double r1[4], r2[4], r3[4], r4[4];
    if (dir == 0) {
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
    for (int p = 0; p < 6; ++p) {
        if (dir == 0) {
            invx(u, v, H, c, s[p], RQ[p]);
            invx(u, v, H, c, f[p], RF[p]);
        } else {
            invy(u, v, H, c, s[p], RQ[p]);
            invy(u, v, H, c, f[p], RF[p]);
        }
    }
    for (int p = 0; p < 6; ++p)
        for (int k = 0; k < 4; ++k) {
            fp[p][k] = 0.5 * (RF[p][k] + alpha * RQ[p][k]);
            fm[p][k] = 0.5 * (RF[p][k] - alpha * RQ[p][k]);
        }
    double S[4];
    for (int k = 0; k < 4; ++k) {
        const double lr = recon_left(fp[4][k], fp[3][k], fp[2][k], fp[1][k], fp[0][k], 0, wz_eps, wz_delta);
        const double rl = recon_left(fm[1][k], fm[2][k], fm[3][k], fm[4][k], fm[5][k], 0, wz_eps, wz_delta);
        S[k] = lr + rl;
    }
    V4 out;
    for (int k = 0; k < 4; ++k) out.v[k] = S[0] * r1[k] + S[1] * r2[k] + S[2] * r3[k] + S[3] * r4[k];
    return out;
}

// =============================================================================================
// 2D AWCM state.
enum { BC_QUAD = 0, BC_DMACH = 1, BC_PERIODIC = 2, BC_SHOCK_VORTEX = 3, BC_WIND_TUNNEL = 5 };

struct O2D {
    int L = 0, maxl = 0, nx = 0, ny = 0, w = 0;
    size_t plane = 0;
    double gamma = 1.4, x_min = 0, y_min = 0, dx = 0, dy = 0;
    int bc_kind = BC_QUAD;
    int freeze = 0;
    double wz_eps = 1e-40;  // WENOZ5::eps (WENOZ.h:13-18), a public member of the reference solver
    double wz_delta = 0.0;  // > 0: smoothed tau = sqrt((b0-b2)^2 + delta^2) (no reference counterpart)
    std::vector<double> q[4], q2[4], q1[4], q0[4];
    std::vector<uint8_t> m;
    std::vector<int> lv[4];
    bool scalar = false;  // scalar AWCM (main_2d_advect.cpp): q[0] carries the field
    // the enum-driven BOUNDARY_MANAGER_2D<TT> (BOUNDARY_MANAGER_2D.h:23-159) when set: the condition
    // of every ghosted point (FIELD_UNIFORM_2D<BOUNDARY_CONDITION> layout)
    std::vector<int> bcf;
    // wind tunnel (BOUNDARY_MANAGER_WT, Problems/2D/PROBLEM_WINDTUNNEL.h:52-222): the step's corner
    // i_bdry = int(0.6/dx), j_bdry = int(0.2/dy) (:75-76) and the x-sweep copy of a stage input
    int wt_i = 0, wt_j = 0;
    std::vector<double> qx[4];
    int D(int lev) const { return 1 << (maxl - lev); }
    size_t at(int i, int j) const { return (size_t)(j + G) * w + (i + G); }
    bool get(int i, int j, int b) const { return (m[at(i, j)] >> b) & 1; }
    void set(int i, int j, int b)
    {
        if (i < -G || i >= nx + G || j < -G || j >= ny + G) return;  // dropped (reference UB)
        m[at(i, j)] |= (uint8_t)(1u << b);
    }
    void clr(int i, int j, int b) { m[at(i, j)] &= (uint8_t)~(1u << b); }
    int& LV(int l, int i, int j) { return lv[l][(size_t)j * nx + i]; }
};

inline void clamp_predict(int& s, int& k, int c, int D, int N1)
{
    // predict stencil of a detail point: nodes c-3D/2 .. c+3D/2, one-sided at the ends
    const int h = D / 2;
    s = c - D - h;
    k = 1;
    if (s < 0) s = 0, k = 0;
    else if (c + D + h > N1) s = N1 - 3 * D, k = 2;
}

inline void clamp_update(int& s, int& k, int c, int D, int N1)
{
    // update stencil of an even point: the four nearest detail points, one-sided at the ends
    const int h = D / 2;
    s = c - D - h;
    k = 1;
    if (s < 0) s = h, k = 0;
    else if (c + D + h > N1) s = N1 - 3 * D - h, k = 2;
}

// ForwardWaveletTransformationEuler (Wavelet/WAVELET_2D.h:478-624): per level d3, d1, d2, c.
void fwt2d(O2D& s, double tol)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    std::vector<double>& q = s.q[0];
    auto Q = [&](int i, int j) -> double& { return q[s.at(i, j)]; };
    for (int lev = s.maxl - 1; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2;
#pragma omp parallel for schedule(static)
        for (int j = h; j <= NY - h; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, 0)) continue;
                int is, k1, js, k2;
                clamp_predict(is, k1, i, D, NX);
                clamp_predict(js, k2, j, D, NY);
                double& v = Q(i, j);
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v -= Q(mm, j) * W(c, k1);
                for (int c = 0, n = js; c < 4; ++c, n += D) v -= Q(i, n) * W(c, k2);
                for (int c2 = 0, n = js; c2 < 4; ++c2, n += D)
                    for (int c1 = 0, mm = is; c1 < 4; ++c1, mm += D) v += Q(mm, n) * W(c1, k1) * W(c2, k2);
                v *= 0.25;
                if (absd(v) < tol) s.clr(i, j, 0);
            }
#pragma omp parallel for schedule(static)
        for (int j = D; j <= NY - D; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, 0)) continue;
                int is, k;
                clamp_predict(is, k, i, D, NX);
                double& v = Q(i, j);
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v -= Q(mm, j) * W(c, k);
                v *= 0.5;
                if (absd(v) < tol) s.clr(i, j, 0);
            }
#pragma omp parallel for schedule(static)
        for (int j = h; j <= NY - h; j += D)
            for (int i = D; i <= NX - D; i += D) {
                if (!s.get(i, j, 0)) continue;
                int js, k;
                clamp_predict(js, k, j, D, NY);
                double& v = Q(i, j);
                for (int c = 0, n = js; c < 4; ++c, n += D) v -= Q(i, n) * W(c, k);
                v *= 0.5;
                if (absd(v) < tol) s.clr(i, j, 0);
            }
#pragma omp parallel for schedule(static)
        for (int j = D; j <= NY - D; j += D)
            for (int i = D; i <= NX - D; i += D) {
                if (!s.get(i, j, 0)) continue;
                int is, k1, js, k2;
                clamp_update(is, k1, i, D, NX);
                clamp_update(js, k2, j, D, NY);
                double& v = Q(i, j);
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v += Q(mm, j) * W(c, k1);
                for (int c = 0, n = js; c < 4; ++c, n += D) v += Q(i, n) * W(c, k2);
                for (int c2 = 0, n = js; c2 < 4; ++c2, n += D)
                    for (int c1 = 0, mm = is; c1 < 4; ++c1, mm += D) v += Q(mm, n) * W(c1, k1) * W(c2, k2);
            }
    }
}

// InverseWaveletTransformationEuler (Wavelet/WAVELET_2D.h:626-782): per level c, d2, d1, d3.
void iwt2d(O2D& s, int b)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    std::vector<double>& q = s.q[0];
    auto Q = [&](int i, int j) -> double& { return q[s.at(i, j)]; };
    for (int lev = 0; lev < s.maxl; ++lev) {
        const int D = s.D(lev), h = D / 2;
#pragma omp parallel for schedule(static)
        for (int j = D; j <= NY - D; j += D)
            for (int i = D; i <= NX - D; i += D) {
                if (!s.get(i, j, b)) { Q(i, j) = 0; continue; }
                int is, k1, js, k2;
                clamp_update(is, k1, i, D, NX);
                clamp_update(js, k2, j, D, NY);
                double& v = Q(i, j);
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v -= Q(mm, j) * W(c, k1);
                for (int c = 0, n = js; c < 4; ++c, n += D) v -= Q(i, n) * W(c, k2);
                for (int c2 = 0, n = js; c2 < 4; ++c2, n += D)
                    for (int c1 = 0, mm = is; c1 < 4; ++c1, mm += D) v -= Q(mm, n) * W(c1, k1) * W(c2, k2);
            }
#pragma omp parallel for schedule(static)
        for (int j = h; j <= NY - h; j += D)
            for (int i = D; i <= NX - D; i += D) {
                if (!s.get(i, j, b)) { Q(i, j) = 0; continue; }
                int js, k;
                clamp_predict(js, k, j, D, NY);
                double& v = Q(i, j);
                v *= 2.0;
                for (int c = 0, n = js; c < 4; ++c, n += D) v += Q(i, n) * W(c, k);
            }
#pragma omp parallel for schedule(static)
        for (int j = D; j <= NY - D; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, b)) { Q(i, j) = 0; continue; }
                int is, k;
                clamp_predict(is, k, i, D, NX);
                double& v = Q(i, j);
                v *= 2.0;
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v += Q(mm, j) * W(c, k);
            }
#pragma omp parallel for schedule(static)
        for (int j = h; j <= NY - h; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, b)) { Q(i, j) = 0; continue; }
                int is, k1, js, k2;
                clamp_predict(is, k1, i, D, NX);
                clamp_predict(js, k2, j, D, NY);
                double& v = Q(i, j);
                v *= 4.0;
                for (int c = 0, mm = is; c < 4; ++c, mm += D) v += Q(mm, j) * W(c, k1);
                for (int c = 0, n = js; c < 4; ++c, n += D) v += Q(i, n) * W(c, k2);
                for (int c2 = 0, n = js; c2 < 4; ++c2, n += D)
                    for (int c1 = 0, mm = is; c1 < 4; ++c1, mm += D) v -= Q(mm, n) * W(c1, k1) * W(c2, k2);
            }
    }
}

// AWCM_MANAGER_2D::CheckReconstruction (Wavelet/AWCM_MANAGER_2D.h:63-158): per level d3, d1, d2.
void cr2d(O2D& s, int b)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    for (int lev = s.maxl - 1; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2;
        int k;
        for (int j = h; j <= NY - h; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, b)) continue;
                int is, js;
                clamp_predict(is, k, i, D, NX);
                clamp_predict(js, k, j, D, NY);
                for (int c = 0; c < 4; ++c) s.set(is + c * D, j, b);
                for (int c = 0; c < 4; ++c) s.set(i, js + c * D, b);
                for (int c2 = 0; c2 < 4; ++c2)
                    for (int c1 = 0; c1 < 4; ++c1) s.set(is + c1 * D, js + c2 * D, b);
            }
        for (int j = D; j <= NY - D; j += D)
            for (int i = h; i <= NX - h; i += D) {
                if (!s.get(i, j, b)) continue;
                int is;
                clamp_predict(is, k, i, D, NX);
                for (int c = 0; c < 4; ++c) s.set(is + c * D, j, b);
            }
        for (int j = h; j <= NY - h; j += D)
            for (int i = D; i <= NX - D; i += D) {
                if (!s.get(i, j, b)) continue;
                int js;
                clamp_predict(js, k, j, D, NY);
                for (int c = 0; c < 4; ++c) s.set(i, js + c * D, b);
            }
    }
}

// Visits the three detail sub-bands of one level: (half, coarse), (coarse, half), (half, half),
// with the sub-grid extents of MRA_GRID_INT_2D::Initialize (Wavelet/MRA_GRID_UNIFORM_2D.h:114-131).
template <class Fn>
void for_subbands(const O2D& s, int lev, Fn fn)
{
    const int NX = s.nx - 1, NY = s.ny - 1, D = s.D(lev), h = D / 2;
    for (int j = D; j <= NY - D; j += D)
        for (int i = h; i <= NX - h; i += D) fn(i, j);
    for (int j = h; j <= NY - h; j += D)
        for (int i = D; i <= NX - D; i += D) fn(i, j);
    for (int j = h; j <= NY - h; j += D)
        for (int i = h; i <= NX - h; i += D) fn(i, j);
}

// AWCM_MANAGER_2D::AddAdjacentZone (Wavelet/AWCM_MANAGER_2D.h:14-61), reading a copy of the mask.
void aaz2d(O2D& s, int b)
{
    copy_bit(s.m, b, 6);
    for_subbands(s, s.maxl - 1, [&](int i, int j) {
        if (!s.get(i, j, 6)) return;
        s.set(i - 1, j, b);
        s.set(i + 1, j, b);
        s.set(i, j - 1, b);
        s.set(i, j + 1, b);
    });
    for (int lev = s.maxl - 2; lev >= 0; --lev) {
        const int D = s.D(lev), h = D / 2, q4 = D / 4;
        for_subbands(s, lev, [&](int i, int j) {
            if (!s.get(i, j, 6)) return;
            s.set(i - q4, j, b);
            s.set(i + q4, j, b);
            s.set(i, j - q4, b);
            s.set(i, j + q4, b);
            s.set(i - h, j, b);
            s.set(i + h, j, b);
            s.set(i, j - h, b);
            s.set(i, j + h, b);
        });
    }
}

// AWCM_MANAGER_2D::AddPointForDifferentiation (Wavelet/AWCM_MANAGER_2D.h:160-213).
void apd2d(O2D& s, int b, int l)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    copy_bit(s.m, b, 6);
    for (int j = 1; j <= NY - 1; ++j)
        for (int i = 1; i <= NX - 1; ++i) {
            if (!s.get(i, j, 6)) continue;
            const int lev = s.LV(l, i, j);
            const int D = s.D(lev);
            if (lev == s.maxl) {
                for (int c = -3; c <= 3; ++c) {
                    s.set(i + c, j, b);
                    s.set(i, j + c, b);
                }
                continue;
            }
            int lo = -2, hi = 2;
            if (i - 2 * D < 0) lo = -1, hi = 2;
            else if (i + 2 * D > NX) lo = -2, hi = 1;
            for (int c = lo; c <= hi; ++c) s.set(i + D * c, j, b);
            lo = -2, hi = 2;
            if (j - 2 * D < 0) lo = -1, hi = 2;
            else if (j + 2 * D > NY) lo = -2, hi = 1;
            for (int c = lo; c <= hi; ++c) s.set(i, j + D * c, b);
        }
}

inline bool mask_at_2d(const O2D& s, int i, int j, int b)
{
    // see mask_at_1d
    if (i < -G || i >= s.nx + G || j < -G || j >= s.ny + G) return true;
    return s.get(i, j, b);
}

// AWCM_MANAGER_2D::ComputeLevel (Wavelet/AWCM_MANAGER_2D.h:215-241).
void cl2d(O2D& s, int l, int b)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i) {
            if (!s.get(i, j, b)) { s.LV(l, i, j) = 0; continue; }
            int dx = 1;
            for (int lev = s.maxl; lev >= 0; --lev) {
                if (mask_at_2d(s, i - dx, j, b) || mask_at_2d(s, i + dx, j, b) || mask_at_2d(s, i, j - dx, b) ||
                    mask_at_2d(s, i, j + dx, b)) {
                    s.LV(l, i, j) = lev;
                    break;
                }
                dx *= 2;
            }
        }
}

// BandingMask (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:205-213): two points at each edge.
void band2d(O2D& s, int b)
{
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i)
            if (!(2 <= i && i <= s.nx - 3 && j >= 2 && j <= s.ny - 3)) s.set(i, j, b);
    if (s.bc_kind != BC_WIND_TUNNEL) return;
    // BOUNDARY_MANAGER_WT::BandingMask (PROBLEM_WINDTUNNEL.h:202-220): also the band around the
    // step's top (|j - j_bdry| <= 2, i >= i_bdry - 2) and front (|i - i_bdry| <= 2, j <= j_bdry + 2).
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i) {
            if (std::abs(j - s.wt_j) <= 2 && i >= s.wt_i - 2) s.set(i, j, b);
            if (std::abs(i - s.wt_i) <= 2 && j <= s.wt_j + 2) s.set(i, j, b);
        }
}

// WAVELET_2D::InterpolateEuler (Wavelet/WAVELET_2D.h:784-907): components 1..3 at new points.
// to < 0: every grid point (InterpolateAllGridEuler, WAVELET_2D.h:912-1044, mask_temp all true
// minus mask_from); p0: first interpolated component (1 for InterpolateEuler, 0 for the dense
// field).
void interp2d(O2D& s, int from, int to, int p0 = 1)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    if (to >= 0) copy_bit(s.m, to, 5);
    else
        for (auto& b : s.m) b |= (uint8_t)(1u << 5);
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i <= NX; ++i)
            if (s.get(i, j, from)) s.clr(i, j, 5);
    cr2d(s, 5);
    auto need = [&](int i, int j) { return s.get(i, j, 5) && !s.get(i, j, from); };
    for (int lev = 0; lev < s.maxl; ++lev) {
        const int D = s.D(lev), h = D / 2;
        for (int p = p0; p < 4; ++p) {
            std::vector<double>& q = s.q[p];
            auto Q = [&](int i, int j) -> double& { return q[s.at(i, j)]; };
            for (int j = D; j <= NY - D; j += D)
                for (int i = h; i <= NX - h; i += D) {
                    if (!need(i, j)) continue;
                    int is, k;
                    clamp_predict(is, k, i, D, NX);
                    double v = 0.0;
                    for (int c = 0, mm = is; c < 4; ++c, mm += D) v += Q(mm, j) * W(c, k);
                    Q(i, j) = v;
                }
            for (int j = h; j <= NY - h; j += D)
                for (int i = D; i <= NX - D; i += D) {
                    if (!need(i, j)) continue;
                    int js, k;
                    clamp_predict(js, k, j, D, NY);
                    double v = 0.0;
                    for (int c = 0, n = js; c < 4; ++c, n += D) v += Q(i, n) * W(c, k);
                    Q(i, j) = v;
                }
        }
        for (int p = p0; p < 4; ++p) {
            std::vector<double>& q = s.q[p];
            auto Q = [&](int i, int j) -> double& { return q[s.at(i, j)]; };
            for (int j = h; j <= NY - h; j += D)
                for (int i = h; i <= NX - h; i += D) {
                    if (!need(i, j)) continue;
                    int is, k1, js, k2;
                    clamp_predict(is, k1, i, D, NX);
                    clamp_predict(js, k2, j, D, NY);
                    double v = 0.0;
                    for (int c = 0, mm = is; c < 4; ++c, mm += D) v += Q(mm, j) * W(c, k1);
                    for (int c = 0, n = js; c < 4; ++c, n += D) v += Q(i, n) * W(c, k2);
                    for (int c2 = 0, n = js; c2 < 4; ++c2, n += D)
                        for (int c1 = 0, mm = is; c1 < 4; ++c1, mm += D) v -= Q(mm, n) * W(c1, k1) * W(c2, k2);
                    Q(i, j) = v;
                }
        }
    }
}

// AWCM_MANAGER_2D::RemoveResidueEuler (Wavelet/AWCM_MANAGER_2D.h:267-280): interior points only.
void remove_residue_2d(O2D& s, int b)
{
    for (int j = 1; j <= s.ny - 2; ++j)
        for (int i = 1; i <= s.nx - 2; ++i)
            if (!s.get(i, j, b))
                for (int p = 0; p < 4; ++p) s.q[p][s.at(i, j)] = 0.0;
}

// AWCM_2D::PrepareEuler (Wavelet/AWCM_2D.h:114-147).
void prepare2d(O2D& s, double tol)
{
    if (!s.scalar) copy_bit(s.m, 0, 4);  // the scalar Prepare keeps no previous mask0
    fwt2d(s, tol);
    band2d(s, 0);
    aaz2d(s, 0);
    cr2d(s, 0);
    for (int k = 1; k <= 3; ++k) {
        copy_bit(s.m, k - 1, k);
        cl2d(s, k - 1, k - 1);
        apd2d(s, k, k - 1);
        cr2d(s, k);
    }
    iwt2d(s, 3);
    // AWCM_2D::Prepare, the scalar form (Wavelet/AWCM_2D.h:52-79), stops after the inverse transform
    if (!s.scalar) interp2d(s, 4, 3);
}

double euler_E(double g, double rho, double u, double v, double p) { return p / (g - 1) + 0.5 * rho * (u * u + v * v); }

// Boundary managers: transmissive BOUNDARY_MANAGER_QUAD (Problems/2D/PROBLEM_QUADRANTS.h:123-203),
// BOUNDARY_MANAGER_DMACH(t) (Problems/2D/PROBLEM_DOUBLEMACH.h:106-245), periodic
// BOUNDARY_MANAGER_ISENVORTEX (Problems/2D/PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h:107-171).
// Only edge ghosts are filled; corner ghosts are never read by the axis-aligned stencils.
// BOUNDARY_MANAGER_2D<TT>::SetBoundaryCondition(field) (BOUNDARY_MANAGER_2D.h:61-158): left, right,
// bottom, top strips (extrapolation or periodic image per ghost cell), then the corner blocks
// (extrapolation only).
void bc2d_generic(O2D& s, std::vector<double>* f)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    auto F = [&](int p, int i, int j) -> double& { return f[p][s.at(i, j)]; };
    auto K = [&](int i, int j) { return s.bcf[s.at(i, j)]; };
    auto copy = [&](int i, int j, int si, int sj) {
        for (int p = 0; p < 4; ++p) F(p, i, j) = F(p, si, sj);
    };
    for (int j = 0; j <= NY; ++j)
        for (int c = 0; c < G; ++c) {
            if (K(-1 - c, j) == kExtrapolation) copy(-1 - c, j, 0, j);
            if (K(-1 - c, j) == kPeriodic) copy(-1 - c, j, NX - c, j);
        }
    for (int j = 0; j <= NY; ++j)
        for (int c = 0; c < G; ++c) {
            if (K(NX + 1 + c, j) == kExtrapolation) copy(NX + 1 + c, j, NX, j);
            if (K(NX + 1 + c, j) == kPeriodic) copy(NX + 1 + c, j, c, j);
        }
    for (int i = 0; i <= NX; ++i)
        for (int c = 0; c < G; ++c) {
            if (K(i, -1 - c) == kExtrapolation) copy(i, -1 - c, i, 0);
            if (K(i, -1 - c) == kPeriodic) copy(i, -1 - c, i, NY - c);
        }
    for (int i = 0; i <= NX; ++i)
        for (int c = 0; c < G; ++c) {
            if (K(i, NY + 1 + c) == kExtrapolation) copy(i, NY + 1 + c, i, NY);
            if (K(i, NY + 1 + c) == kPeriodic) copy(i, NY + 1 + c, i, c);
        }
    for (int a = 0; a < G; ++a)
        for (int b = 0; b < G; ++b) {
            if (K(-1 - a, -1 - b) == kExtrapolation) copy(-1 - a, -1 - b, 0, 0);
            if (K(-1 - a, NY + 1 + b) == kExtrapolation) copy(-1 - a, NY + 1 + b, 0, NY);
            if (K(NX + 1 + a, -1 - b) == kExtrapolation) copy(NX + 1 + a, -1 - b, NX, 0);
            if (K(NX + 1 + a, NY + 1 + b) == kExtrapolation) copy(NX + 1 + a, NY + 1 + b, NX, NY);
        }
}

void bc2d(O2D& s, std::vector<double>* f, double t)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    auto F = [&](int p, int i, int j) -> double& { return f[p][s.at(i, j)]; };
    const double g = 1.4;
    if (!s.bcf.empty()) {
        bc2d_generic(s, f);
        return;
    }
    if (s.bc_kind == BC_WIND_TUNNEL) {
        // BOUNDARY_MANAGER_WT::SetBoundaryCondition (PROBLEM_WINDTUNNEL.h:94-199): Mach 3 inflow on the
        // left, zero-order extrapolation on the right (interior rows), reflected v on the top
        // (interior columns); the bottom is filled per sweep direction (wt_fill_x / wt_fill_y).
        const double in[4] = {1.4, 1.4 * 3, 1.4 * 0, euler_E(1.4, 1.4, 3, 0, 1)};
        for (int j = 0; j <= NY; ++j)
            for (int c = 0; c < G; ++c)
                for (int p = 0; p < 4; ++p) F(p, -1 - c, j) = in[p];
        for (int j = 0; j <= NY; ++j)
            for (int c = 0; c < G; ++c)
                for (int p = 0; p < 4; ++p) F(p, NX + 1 + c, j) = F(p, NX, j);
        for (int i = 0; i <= NX; ++i)
            for (int c = 0; c < G; ++c)
                for (int p = 0; p < 4; ++p) F(p, i, NY + 1 + c) = p == 2 ? -F(p, i, NY) : F(p, i, NY);
        return;
    }
    if (s.bc_kind == BC_PERIODIC) {
        for (int j = 0; j <= NY; ++j)
            for (int c = 0; c < G; ++c)
                for (int p = 0; p < 4; ++p) {
                    F(p, -1 - c, j) = F(p, NX - c, j);
                    F(p, NX + 1 + c, j) = F(p, c, j);
                }
        for (int i = 0; i <= NX; ++i)
            for (int c = 0; c < G; ++c)
                for (int p = 0; p < 4; ++p) {
                    F(p, i, -1 - c) = F(p, i, NY - c);
                    F(p, i, NY + 1 + c) = F(p, i, c);
                }
        return;
    }
    if (s.bc_kind == BC_DMACH) {
        const double rho = 8, u = 8.25 * std::sqrt(3.0) * 0.5, v = -8.25 * 0.5, p = 116.5;
        const double inflow[4] = {rho, rho * u, rho * v, euler_E(s.gamma, rho, u, v, p)};
        for (int j = 0; j <= NY; ++j)
            for (int i = -1; i >= -G; --i)
                for (int k = 0; k < 4; ++k) F(k, i, j) = inflow[k];
    } else {
        for (int j = 0; j <= NY; ++j)
            for (int i = -1; i >= -G; --i)
                for (int k = 0; k < 4; ++k) F(k, i, j) = F(k, 0, j);
    }
    for (int j = 0; j <= NY; ++j)
        for (int i = NX + 1; i <= NX + G; ++i)
            for (int k = 0; k < 4; ++k) F(k, i, j) = F(k, NX, j);
    if (s.bc_kind == BC_DMACH) {
        const double sqrt3 = std::sqrt(3.0);
        const double post[4] = {8, 8 * 8.25 * sqrt3 * 0.5, -8 * 8.25 * 0.5,
                                euler_E(g, 8, 8.25 * sqrt3 * 0.5, -8.25 * 0.5, 116.5)};
        const double pre[4] = {1.4, 1.4 * 0, 1.4 * 0, euler_E(g, 1.4, 0, 0, 1)};
        for (int i = 0; i <= NX; ++i) {
            const double x = s.x_min + i * s.dx;
            for (int j = -1; j >= -G; --j) {
                if (x > 1.0 / 6.0) {
                    F(0, i, j) = F(0, i, 0);
                    F(1, i, j) = F(1, i, 0);
                    F(2, i, j) = -F(2, i, 0);
                    F(3, i, j) = F(3, i, 0);
                } else {
                    for (int k = 0; k < 4; ++k) F(k, i, j) = post[k];
                }
            }
            const double xs = 1.0 / 6.0 + (1 + 20 * t) / sqrt3;
            for (int j = NY + 1; j <= NY + G; ++j)
                for (int k = 0; k < 4; ++k) F(k, i, j) = x < xs ? post[k] : pre[k];
        }
    } else if (s.bc_kind == BC_SHOCK_VORTEX) {
        // BOUNDARY_MANAGER_SHOCK_VORTEX::SetBottom/TopBoundaryCondition
        // (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:145-175): walls, rho v reflected.
        for (int i = 0; i <= NX; ++i)
            for (int c = 1; c <= G; ++c)
                for (int k = 0; k < 4; ++k) {
                    const double sg = k == 2 ? -1.0 : 1.0;
                    F(k, i, -c) = sg * F(k, i, 0);
                    F(k, i, NY + c) = sg * F(k, i, NY);
                }
    } else {
        for (int i = 0; i <= NX; ++i)
            for (int c = 1; c <= G; ++c)
                for (int k = 0; k < 4; ++k) {
                    F(k, i, -c) = F(k, i, 0);
                    F(k, i, NY + c) = F(k, i, NY);
                }
    }
}

// BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition (PROBLEM_WINDTUNNEL.h:124-168).  x direction: the
// three columns i_bdry.. i_bdry+2 up to row j_bdry (ghost rows included) mirror column i_bdry-1 with
// rho u reflected; y direction: the bottom ghost rows mirror row 0 (columns -3 .. Nx+1) and the rows
// j_bdry-2 .. j_bdry right of i_bdry mirror row j_bdry+1, rho v reflected.
void wt_fill_x(O2D& s, std::vector<double>* f)
{
    auto F = [&](int p, int i, int j) -> double& { return f[p][s.at(i, j)]; };
    for (int j = -G; j <= s.wt_j; ++j)
        for (int c = 0; c < 3; ++c)
            for (int p = 0; p < 4; ++p) F(p, s.wt_i + c, j) = p == 1 ? -F(p, s.wt_i - 1, j) : F(p, s.wt_i - 1, j);
}
void wt_fill_y(O2D& s, std::vector<double>* f)
{
    auto F = [&](int p, int i, int j) -> double& { return f[p][s.at(i, j)]; };
    const int NX = s.nx - 1;
    for (int i = -G; i < NX + G; ++i)
        for (int c = 0; c < 3; ++c)
            for (int p = 0; p < 4; ++p) F(p, i, -1 - c) = p == 2 ? -F(p, i, 0) : F(p, i, 0);
    for (int i = s.wt_i; i <= NX + G; ++i)
        for (int c = 0; c < 3; ++c)
            for (int p = 0; p < 4; ++p) F(p, i, s.wt_j - c) = p == 2 ? -F(p, i, s.wt_j + 1) : F(p, i, s.wt_j + 1);
}
// The wind tunnel's stage input: the x-sweep copy gets the x-direction bottom fill; the field
// itself the x- and then the y-direction fill.
void wt_stage_input(O2D& s, std::vector<double>* f)
{
    for (int p = 0; p < 4; ++p) s.qx[p] = f[p];
    wt_fill_x(s, s.qx);
    wt_fill_x(s, f);
    wt_fill_y(s, f);
}

void alpha2d(O2D& s, std::vector<double>* f, int b, std::vector<double>& ax, std::vector<double>& ay)
{
    ax.assign(s.ny, 0.0);
    ay.assign(s.nx, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i) {
            if (!s.get(i, j, b)) continue;
            const size_t a = s.at(i, j);
            const double q[4] = {f[0][a], f[1][a], f[2][a], f[3][a]};
            ax[j] = maxd(ax[j], srx(q, s.gamma));
        }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s.nx; ++i)
        for (int j = 0; j < s.ny; ++j) {
            if (!s.get(i, j, b)) continue;
            const size_t a = s.at(i, j);
            const double q[4] = {f[0][a], f[1][a], f[2][a], f[3][a]};
            ay[i] = maxd(ay[i], sry(q, s.gamma));
        }
}

// One RK3 stage (main_2d_euler(quad).cpp:108-163, 188-243, 267-322) over mask bit b, level set l.
// inx: the field the x-direction fluxes read (the wind tunnel's x-sweep copy), else in.
void stage2d(O2D& s, std::vector<double>* in, std::vector<double>* out, int b, int l, const std::vector<double>& ax,
             const std::vector<double>& ay, double dt, int kind, std::vector<double>* inx = nullptr)
{
    if (!inx) inx = in;
    const int NX = s.nx - 1, NY = s.ny - 1;
    const double g = s.gamma;
    const double d1 = 2.0 / 3.0, d2 = -1.0 / 12.0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i <= NX; ++i) {
            if (!s.get(i, j, b)) continue;
            const int lev = s.LV(l, i, j);
            const int d = s.D(lev);
            double dF[4], dG[4];
            auto st = [&](int ii, int jj, double* o) {
                const size_t a = s.at(ii, jj);
                for (int p = 0; p < 4; ++p) o[p] = in[p][a];
            };
            auto stx = [&](int ii, int jj, double* o) {
                const size_t a = s.at(ii, jj);
                for (int p = 0; p < 4; ++p) o[p] = inx[p][a];
            };
            if (lev == s.maxl) {
                double bx[7][4], by[7][4];
                const double *px[7], *py[7];
                for (int o = 0; o < 7; ++o) {
                    stx(i - 3 + o, j, bx[o]);
                    st(i, j - 3 + o, by[o]);
                    px[o] = bx[o];
                    py[o] = by[o];
                }
                V4 a = face_flux_2d(px, ax[j], g, 0, s.wz_eps, s.wz_delta);
                V4 bb = face_flux_2d(px + 1, ax[j], g, 0, s.wz_eps, s.wz_delta);
                for (int p = 0; p < 4; ++p) dF[p] = bb.v[p] - a.v[p];
                a = face_flux_2d(py, ay[i], g, 1, s.wz_eps, s.wz_delta);
                bb = face_flux_2d(py + 1, ay[i], g, 1, s.wz_eps, s.wz_delta);
                for (int p = 0; p < 4; ++p) dG[p] = bb.v[p] - a.v[p];
            } else {
                double b5[5][4];
                V4 f[5];
                for (int o = 0; o < 5; ++o) {
                    const int ii = i + (o - 2) * d;
                    if ((o == 0 && i <= d) || (o == 4 && i >= NX - d && !(i <= d))) continue;
                    stx(ii, j, b5[o]);
                    f[o] = fu2(b5[o], g);
                }
                for (int p = 0; p < 4; ++p) {
                    if (i <= d) dF[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[4].v[p] - f[1].v[p]);
                    else if (i >= NX - d) dF[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[3].v[p] - f[0].v[p]);
                    else dF[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[4].v[p] - f[0].v[p]);
                }
                for (int o = 0; o < 5; ++o) {
                    const int jj = j + (o - 2) * d;
                    if ((o == 0 && j <= d) || (o == 4 && j >= NY - d && !(j <= d))) continue;
                    st(i, jj, b5[o]);
                    f[o] = gu2(b5[o], g);
                }
                for (int p = 0; p < 4; ++p) {
                    if (j <= d) dG[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[4].v[p] - f[1].v[p]);
                    else if (j >= NY - d) dG[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[3].v[p] - f[0].v[p]);
                    else dG[p] = d1 * (f[3].v[p] - f[1].v[p]) + d2 * (f[4].v[p] - f[0].v[p]);
                }
            }
            const double sc = dt / (s.dx * d);
            const size_t a = s.at(i, j);
            for (int p = 0; p < 4; ++p) {
                const double r = in[p][a] - sc * (dF[p] + dG[p]);
                out[p][a] = kind == 2 ? 0.75 * s.q[p][a] + 0.25 * (in[p][a] - sc * (dF[p] + dG[p])) : r;
            }
        }
}

void step2d(O2D& s, double tol, double cfl, double t, double t_next, double dt_fixed, double* alpha_io, double* out)
{
    if (!s.freeze) prepare2d(s, tol);
    const bool wt = s.bc_kind == BC_WIND_TUNNEL && s.bcf.empty();
    std::vector<double>* qx = wt ? s.qx : nullptr;
    // Wind tunnel: the bottom fills write solid cells of mask3 (left non-physical by PrepareEuler),
    // so its first stage input is filled before the CFL scan; the other managers write ghost cells
    // only and keep the driver's order (main_2d_euler(quad).cpp:61-85).
    if (wt) {
        bc2d(s, s.q, t);
        wt_stage_input(s, s.q);
    }
    double mv = 0;
    {
        std::vector<double> part(omp_get_max_threads(), 0.0);
#pragma omp parallel
        {
            double loc = 0;
#pragma omp for schedule(static)
            for (int j = 0; j < s.ny; ++j)
                for (int i = 0; i < s.nx; ++i) {
                    if (!s.get(i, j, 3)) continue;
                    const size_t a = s.at(i, j);
                    const double q[4] = {s.q[0][a], s.q[1][a], s.q[2][a], s.q[3][a]};
                    loc = maxd(loc, srx(q, s.gamma) + sry(q, s.gamma));
                }
            part[omp_get_thread_num()] = loc;
        }
        for (double v : part) mv = maxd(mv, v);
    }
    double dt = cfl * s.dx / mv;
    if (dt_fixed > 0) dt = dt_fixed;
    int do_print = 0;
    if (t + dt > t_next) { dt = t_next - t; do_print = 1; }

    std::vector<double> ax, ay;
    // freeze 2: replay the recorded LF speeds from alpha_io; 1 (or normal mode): compute them and
    // record them into alpha_io when it is given.
    const bool frozen = s.freeze == 2 && alpha_io;
    auto load_alpha = [&](int stage, std::vector<double>* f, int b) {
        double* base = alpha_io ? alpha_io + (size_t)stage * (s.nx + s.ny) : nullptr;
        if (frozen) {
            ax.assign(base, base + s.ny);
            ay.assign(base + s.ny, base + s.ny + s.nx);
        } else {
            alpha2d(s, f, b, ax, ay);
            if (base) {
                std::memcpy(base, ax.data(), sizeof(double) * s.ny);
                std::memcpy(base + s.ny, ay.data(), sizeof(double) * s.nx);
            }
        }
    };
    if (!wt) bc2d(s, s.q, t);
    load_alpha(0, s.q, 3);
    stage2d(s, s.q, s.q2, 2, 2, ax, ay, dt, 1, qx);
    bc2d(s, s.q2, t);
    if (wt) wt_stage_input(s, s.q2);
    load_alpha(1, s.q2, 2);
    stage2d(s, s.q2, s.q1, 1, 1, ax, ay, dt, 2, qx);
    bc2d(s, s.q1, t);
    if (wt) wt_stage_input(s, s.q1);
    load_alpha(2, s.q1, 1);
    stage2d(s, s.q1, s.q0, 0, 0, ax, ay, dt, 3, qx);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i) {
            if (!s.get(i, j, 0)) continue;
            const size_t a = s.at(i, j);
            for (int p = 0; p < 4; ++p) s.q[p][a] = (s.q[p][a] + 2.0 * s.q0[p][a]) / 3.0;
        }
    // Frozen-mask mode (the gradient configuration) keeps the points outside mask0: without the
    // per-step PrepareEuler nothing would refill the stencil points of mask3 \ mask0.
    if (!s.freeze) remove_residue_2d(s, 0);
    long cnt[4] = {0, 0, 0, 0};
    for (int j = 0; j < s.ny; ++j)
        for (int i = 0; i < s.nx; ++i)
            for (int k = 0; k < 4; ++k) cnt[k] += s.get(i, j, k);
    out[0] = dt;
    out[1] = do_print;
    for (int k = 0; k < 4; ++k) out[2 + k] = (double)cnt[k];
    out[6] = mv;
}

int bit_of(int mask_id) { return mask_id >= 0 && mask_id <= 3 ? mask_id : 4; }

}  // namespace

// =============================================================================================
extern "C" {

void* or1d_create(int num_levels, int nx_coarse, double x_min, double x_max, double gamma, int scheme)
{
    O1D* s = new O1D();
    s->L = num_levels;
    s->maxl = num_levels - 1;
    s->nxc = nx_coarse;
    s->nx = (nx_coarse - 1) * (1 << (num_levels - 1)) + 1;
    s->w = s->nx + 2 * G;
    s->gamma = gamma;
    s->scheme = scheme;
    s->x_min = x_min;
    s->dx = (x_max - x_min) / (s->nx - 1);
    for (int p = 0; p < 3; ++p) {
        s->q[p].assign(s->w, 0.0);
        s->qc[p].assign(s->w, 0.0);
        s->qt[p].assign(s->w, 0.0);
    }
    s->m.assign(s->w, 1u);  // mask0 true everywhere, ghosts included (AWCM_1D.h:34)
    for (int l = 0; l < 4; ++l) s->lv[l].assign(s->nx, 0);
    return s;
}

void or1d_destroy(void* h) { delete static_cast<O1D*>(h); }
int or1d_nx(void* h) { return static_cast<O1D*>(h)->nx; }

void or1d_set_q(void* h, const double* q)
{
    O1D* s = static_cast<O1D*>(h);
    for (int a = 0; a < s->w; ++a)
        for (int p = 0; p < 3; ++p) s->q[p][a] = q[a * 3 + p];
}

void or1d_get_q(void* h, double* q)
{
    O1D* s = static_cast<O1D*>(h);
    for (int a = 0; a < s->w; ++a)
        for (int p = 0; p < 3; ++p) q[a * 3 + p] = s->q[p][a];
}

void or1d_init_riemann(void* h, double x_interface, double rho_l, double u_l, double p_l, double rho_r, double u_r,
                       double p_r)
{
    O1D* s = static_cast<O1D*>(h);
    for (int i = -G; i < s->nx + G; ++i) {
        const double x = s->x_min + s->dx * i;
        const bool left = x <= x_interface;
        const double rho = left ? rho_l : rho_r, u = left ? u_l : u_r, p = left ? p_l : p_r;
        s->Q(0, i) = rho;
        s->Q(1, i) = rho * u;
        s->Q(2, i) = p / (s->gamma - 1) + 0.5 * rho * sqr(u);
    }
}

void or1d_get_masks(void* h, uint8_t* m)
{
    O1D* s = static_cast<O1D*>(h);
    const int bits[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r)
        for (int a = 0; a < s->w; ++a) m[r * s->w + a] = (s->m[a] >> bits[r]) & 1;
}

void or1d_set_masks(void* h, const uint8_t* m)
{
    O1D* s = static_cast<O1D*>(h);
    const int bits[5] = {4, 0, 1, 2, 3};
    for (int a = 0; a < s->w; ++a) {
        uint8_t v = 0;
        for (int r = 0; r < 5; ++r) v |= (uint8_t)((m[r * s->w + a] != 0) << bits[r]);
        s->m[a] = v;
    }
}

void or1d_get_levels(void* h, int* lv)
{
    O1D* s = static_cast<O1D*>(h);
    for (int r = 0; r < 4; ++r) std::memcpy(lv + r * s->nx, s->lv[r].data(), sizeof(int) * s->nx);
}

void or1d_set_levels(void* h, const int* lv)
{
    O1D* s = static_cast<O1D*>(h);
    for (int r = 0; r < 4; ++r) std::memcpy(s->lv[r].data(), lv + r * s->nx, sizeof(int) * s->nx);
}

void or1d_prepare(void* h, double tol)
{
    O1D& s = *static_cast<O1D*>(h);
    if (s.scheme == 2) prepare1d_scalar(s, tol);
    else prepare1d(s, tol);
}
void or1d_fwt(void* h, double tol) { fwt1d(*static_cast<O1D*>(h), tol); }
void or1d_iwt(void* h, int mask_id) { iwt1d(*static_cast<O1D*>(h), bit_of(mask_id)); }

void or1d_manager(void* h, int op, int mask_id, int level_id)
{
    O1D& s = *static_cast<O1D*>(h);
    const int b = bit_of(mask_id);
    switch (op) {
        case 0: aaz1d(s, b); break;
        case 1: cr1d(s, b); break;
        case 2: apd1d(s, b, level_id); break;
        case 3: cl1d(s, level_id, b); break;
        case 4: remove_residue_1d(s, b); break;
        case 5: band1d(s, b); break;
        default: break;
    }
}

// WAVELET_1D::InterpolateEuler(Q, mra, from, to) (Wavelet/WAVELET_1D.h:393-431) and the
// transmissive BOUNDARY_MANAGER::SetBoundaryCondition (Problems/1D/PROBLEM_SHOCKTUBE.h:86-107).
void or1d_interpolate(void* h, int from_id, int to_id)
{
    interp1d(*static_cast<O1D*>(h), bit_of(from_id), bit_of(to_id));
}
void or1d_apply_bc(void* h) { bc1d(*static_cast<O1D*>(h)); }
// bc: Nx+6 BOUNDARY_CONDITION values; attaches the generic manager.
void or1d_set_bc_field(void* h, const int* bc)
{
    O1D& s = *static_cast<O1D*>(h);
    s.bcf.assign(bc, bc + s.nx + 2 * G);
}
// bc: (Ny+6) x (Nx+6) BOUNDARY_CONDITION values; attaches the generic manager.
void or2d_set_bc_field(void* h, const int* bc)
{
    O2D& s = *static_cast<O2D*>(h);
    s.bcf.assign((size_t)(s.nx + 2 * G) * (s.ny + 2 * G), 0);
    for (int j = -G; j < s.ny + G; ++j)
        for (int i = -G; i < s.nx + G; ++i) s.bcf[s.at(i, j)] = bc[(size_t)(j + G) * (s.nx + 2 * G) + (i + G)];
}

// EULER_EQUATION_1D::ComputeFu / Spectral_Radius (EULER_EQUATION.h:16-26, 42-47) and
// EULER_EQUATION_2D::ComputeFu / ComputeGu / Spectral_RadiusX / Spectral_RadiusY (:74-99, :118-142)
// over n states (3 or 4 doubles each).
void or_euler1d_flux(const double* q, double* f, int n, double g)
{
    for (int t = 0; t < n; ++t) {
        const V3 v = fu1(q + 3 * t, g);
        for (int k = 0; k < 3; ++k) f[3 * t + k] = v.v[k];
    }
}
void or_euler1d_sr(const double* q, double* out, int n, double g)
{
    for (int t = 0; t < n; ++t) out[t] = absd(q[3 * t + 1] / q[3 * t]) + c1(q + 3 * t, g);
}
void or_euler2d_flux(const double* q, double* f, int n, int dir, double g)
{
    for (int t = 0; t < n; ++t) {
        const V4 v = dir == 0 ? fu2(q + 4 * t, g) : gu2(q + 4 * t, g);
        for (int k = 0; k < 4; ++k) f[4 * t + k] = v.v[k];
    }
}
void or_euler2d_sr(const double* q, double* out, int n, int dir, double g)
{
    for (int t = 0; t < n; ++t) out[t] = dir == 0 ? srx(q + 4 * t, g) : sry(q + 4 * t, g);
}

void or1d_step(void* h, double tol, double cfl, double t, double t_next, double* out)
{
    step1d(*static_cast<O1D*>(h), tol, cfl, t, t_next, out);
}

void or1d_scalar_step(void* h, double tol, double dt, double* out)
{
    scalar_step1d(*static_cast<O1D*>(h), tol, dt, out);
}

int or1d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out)
{
    double t = 0, upd = 0, o[10];
    int n = 0;
    while (n < max_steps) {
        or1d_step(h, tol, cfl, t, t_end, o);
        t += o[0];
        upd += o[2];
        ++n;
        if (t >= t_end) break;
    }
    out[0] = t;
    out[1] = upd;
    return n;
}

void* or2d_create(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                  double y_max, int bc_kind)
{
    O2D* s = new O2D();
    s->L = num_levels;
    s->maxl = num_levels - 1;
    s->nx = (nx_coarse - 1) * (1 << (num_levels - 1)) + 1;
    s->ny = (ny_coarse - 1) * (1 << (num_levels - 1)) + 1;
    s->w = s->nx + 2 * G;
    s->plane = (size_t)s->w * (s->ny + 2 * G);
    s->x_min = x_min;
    s->y_min = y_min;
    s->dx = (x_max - x_min) / (s->nx - 1);
    s->dy = (y_max - y_min) / (s->ny - 1);
    s->bc_kind = bc_kind;
    s->wt_i = int(0.6 / s->dx);
    s->wt_j = int(0.2 / s->dy);
    for (int p = 0; p < 4; ++p) {
        s->q[p].assign(s->plane, 0.0);
        s->q2[p].assign(s->plane, 0.0);
        s->q1[p].assign(s->plane, 0.0);
        s->q0[p].assign(s->plane, 0.0);
    }
    s->m.assign(s->plane, 1u);  // mask0 true everywhere (AWCM_2D.h:37)
    for (int l = 0; l < 4; ++l) s->lv[l].assign((size_t)s->nx * s->ny, s->maxl);  // AWCM_2D.h:38-41
    return s;
}

void or2d_destroy(void* h) { delete static_cast<O2D*>(h); }

void or2d_dims(void* h, int* nx, int* ny)
{
    O2D* s = static_cast<O2D*>(h);
    *nx = s->nx;
    *ny = s->ny;
}

void or2d_set_q(void* h, const double* q)
{
    O2D* s = static_cast<O2D*>(h);
    for (size_t a = 0; a < s->plane; ++a)
        for (int p = 0; p < 4; ++p) s->q[p][a] = q[a * 4 + p];
}

void or2d_get_q(void* h, double* q)
{
    O2D* s = static_cast<O2D*>(h);
    for (size_t a = 0; a < s->plane; ++a)
        for (int p = 0; p < 4; ++p) q[a * 4 + p] = s->q[p][a];
}

// Initial states of QUADRANTS (Problems/2D/PROBLEM_QUADRANTS.h:34-80), DOUBLEMACH
// (Problems/2D/PROBLEM_DOUBLEMACH.h:34-62) and ISENTROPIC_VORTEX_ADVECTION
// (Problems/2D/PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h:38-64), ghosts included; see the harness for
// the meaning of a and b.
void or2d_init_problem(void* h, int kind, double a, double b)
{
    O2D* s = static_cast<O2D*>(h);
    const double g = s->gamma;
    const double PI = 4. * std::atan(1.);
    for (int j = -G; j < s->ny + G; ++j)
        for (int i = -G; i < s->nx + G; ++i) {
            const double x = s->x_min + (i - 0) * s->dx, y = s->y_min + (j - 0) * s->dy;
            double rho, u, v, p, Q[4];
            if (kind == 0) {
                if (x >= a && y >= b) { rho = 1.5; u = 0; v = 0; p = 1.5; }
                else if (x < a && y >= b) { rho = 0.532258064516129; u = 1.206045378311055; v = 0; p = 0.3; }
                else if (x < a && y < b) {
                    rho = 0.137992831541219; u = 1.206045378311055; v = 1.206045378311055; p = 0.029032258064516;
                } else { rho = 0.532258064516129; u = 0; v = 1.206045378311055; p = 0.3; }
                Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = euler_E(g, rho, u, v, p);
            } else if (kind == 1) {
                if (y > std::sqrt(3.0) * (x - 1.0 / 6.0)) { rho = 8; u = 8.25 * std::sqrt(3.0) * 0.5; v = -8.25 * 0.5; p = 116.5; }
                else { rho = a; u = 0; v = 0; p = 1; }
                Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = euler_E(g, rho, u, v, p);
            } else if (kind == 2) {
                const double rr = sqr(x - a) + sqr(y - b);
                const double beta = 5;
                rho = 1 - (g - 1) * sqr(beta) / (8 * g * PI * PI) * std::exp(1 - rr);
                rho = std::pow(rho, 1.0 / (g - 1.0));
                double rhou = 0 - beta / (2 * PI) * std::exp((1 - rr) * 0.5) * (y - b);
                rhou *= rho;
                double rhov = 1 + beta / (2 * PI) * std::exp((1 - rr) * 0.5) * (x - a);
                rhov *= rho;
                p = std::pow(rho, g);
                Q[0] = rho, Q[1] = rhou, Q[2] = rhov, Q[3] = euler_E(g, rho, rhou / rho, rhov / rho, p);
            }
            if (kind == 4) {
                // WINDTUNNEL::Initialize (Problems/2D/PROBLEM_WINDTUNNEL.h:14-47): Mach 3 uniform flow
                rho = 1.4, u = 3, v = 0, p = 1;
                Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = euler_E(g, rho, u, v, p);
            }
            if (kind == 3) {
                // SHOCK_VORTEX::Initialize (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:32-66)
                const double Mv = 0.5;
                const double r = std::sqrt(sqr(x - a) + sqr(y - b));
                if (x <= 0) {
                    rho = 1.394708041144614, u = -0.860403729339060, v = 0, p = 1.121834000000000;
                } else {
                    rho = 1 - (g - 1) / 2 * sqr(Mv) * std::exp(1 - r * r);
                    rho = std::pow(rho, 1 / (g - 1));
                    p = 1 - (g - 1) / 2 * sqr(Mv) * std::exp(1 - r * r);
                    p = std::pow(p, g / (g - 1));
                    p = 1 / g * p;
                    u = Mv * std::exp(0.5 * (1 - r * r)) * (-y) - 1.200011999940001;
                    v = Mv * std::exp(0.5 * (1 - r * r)) * (x - a);
                }
                Q[0] = rho, Q[1] = rho * u, Q[2] = rho * v, Q[3] = euler_E(g, rho, u, v, p);
            }
            for (int k = 0; k < 4; ++k) s->q[k][s->at(i, j)] = Q[k];
        }
}

void or2d_get_masks(void* h, uint8_t* m)
{
    O2D* s = static_cast<O2D*>(h);
    const int bits[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r)
        for (size_t a = 0; a < s->plane; ++a) m[r * s->plane + a] = (s->m[a] >> bits[r]) & 1;
}

void or2d_set_masks(void* h, const uint8_t* m)
{
    O2D* s = static_cast<O2D*>(h);
    const int bits[5] = {4, 0, 1, 2, 3};
    for (size_t a = 0; a < s->plane; ++a) {
        uint8_t v = 0;
        for (int r = 0; r < 5; ++r) v |= (uint8_t)((m[r * s->plane + a] != 0) << bits[r]);
        s->m[a] = v;
    }
}

void or2d_get_levels(void* h, int* lv)
{
    O2D* s = static_cast<O2D*>(h);
    const size_t n = (size_t)s->nx * s->ny;
    for (int r = 0; r < 4; ++r) std::memcpy(lv + r * n, s->lv[r].data(), sizeof(int) * n);
}

void or2d_set_levels(void* h, const int* lv)
{
    O2D* s = static_cast<O2D*>(h);
    const size_t n = (size_t)s->nx * s->ny;
    for (int r = 0; r < 4; ++r) std::memcpy(s->lv[r].data(), lv + r * n, sizeof(int) * n);
}

void or2d_prepare(void* h, double tol) { prepare2d(*static_cast<O2D*>(h), tol); }
void or2d_fwt(void* h, double tol) { fwt2d(*static_cast<O2D*>(h), tol); }
void or2d_iwt(void* h, int mask_id) { iwt2d(*static_cast<O2D*>(h), bit_of(mask_id)); }
void or2d_interpolate(void* h, int from_id, int to_id)
{
    interp2d(*static_cast<O2D*>(h), bit_of(from_id), bit_of(to_id));
}

// Scalar AWCM driver loop (Wavelet/main_2d_advect.cpp:48-190): Prepare, the periodic
// BOUNDARY_MANAGER of Problems/2D/PROBLEM_BOX_ADVECTION.h (edge ghosts), three SSP-RK3 stages of
// linear advection with unit velocity (finest level: WENO5::ReconstructRight upwind faces, WENO.h:101-104,
// both faces per point as the driver computes them; coarser levels: AWCM_2D::Differentiate*,
// Wavelet/AWCM_2D.h:95-109), q = 1/3 q + 2/3 q0 on mask0, PostProcess (RemoveResidue on mask0).
void scalar_bc2d(O2D& s, std::vector<double>& f)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    for (int j = 0; j <= NY; ++j)
        for (int c = 0; c < G; ++c) {
            f[s.at(-1 - c, j)] = f[s.at(NX - c, j)];
            f[s.at(NX + 1 + c, j)] = f[s.at(c, j)];
        }
    for (int i = 0; i <= NX; ++i)
        for (int c = 0; c < G; ++c) {
            f[s.at(i, -1 - c)] = f[s.at(i, NY - c)];
            f[s.at(i, NY + 1 + c)] = f[s.at(i, c)];
        }
}

void scalar_stage2d(O2D& s, const std::vector<double>& in, std::vector<double>& out, int bit, int l, double dt,
                    int kind)
{
    const int NX = s.nx - 1, NY = s.ny - 1;
    const double d1 = 2.0 / 3.0, d2 = -1.0 / 12.0;
    const std::vector<double>& qn = s.q[0];
    auto Q = [&](int i, int j) { return in[s.at(i, j)]; };
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i <= NX; ++i) {
            if (!s.get(i, j, bit)) continue;
            const int lev = s.LV(l, i, j);
            const int d = s.D(lev);
            const double dxl = s.dx * d;
            double dF, dG;
            if (lev == s.maxl) {
                double a = recon_left(Q(i + 1, j), Q(i, j), Q(i - 1, j), Q(i - 2, j), Q(i - 3, j), 1);
                double b = recon_left(Q(i + 2, j), Q(i + 1, j), Q(i, j), Q(i - 1, j), Q(i - 2, j), 1);
                dF = b - a;
                a = recon_left(Q(i, j + 1), Q(i, j), Q(i, j - 1), Q(i, j - 2), Q(i, j - 3), 1);
                b = recon_left(Q(i, j + 2), Q(i, j + 1), Q(i, j), Q(i, j - 1), Q(i, j - 2), 1);
                dG = b - a;
            } else {
                if (i <= d) dF = d1 * (Q(i + d, j) - Q(i - d, j)) + d2 * (Q(i + 2 * d, j) - Q(i - d, j));
                else if (i >= NX - d) dF = d1 * (Q(i + d, j) - Q(i - d, j)) + d2 * (Q(i + d, j) - Q(i - 2 * d, j));
                else dF = d1 * (Q(i + d, j) - Q(i - d, j)) + d2 * (Q(i + 2 * d, j) - Q(i - 2 * d, j));
                if (j <= d) dG = d1 * (Q(i, j + d) - Q(i, j - d)) + d2 * (Q(i, j + 2 * d) - Q(i, j - d));
                else if (j >= NY - d) dG = d1 * (Q(i, j + d) - Q(i, j - d)) + d2 * (Q(i, j + d) - Q(i, j - 2 * d));
                else dG = d1 * (Q(i, j + d) - Q(i, j - d)) + d2 * (Q(i, j + 2 * d) - Q(i, j - 2 * d));
            }
            const size_t a = s.at(i, j);
            if (kind == 2) out[a] = 0.75 * qn[a] + 0.25 * (in[a] - dt / dxl * (dF + dG));
            else out[a] = in[a] - dt / dxl * (dF + dG);
        }
}

void scalar_step2d(O2D& s, double tol, double dt, double* out)
{
    prepare2d(s, tol);
    scalar_bc2d(s, s.q[0]);
    scalar_stage2d(s, s.q[0], s.q2[0], 2, 2, dt, 1);
    scalar_bc2d(s, s.q2[0]);
    scalar_stage2d(s, s.q2[0], s.q1[0], 1, 1, dt, 2);
    scalar_bc2d(s, s.q1[0]);
    scalar_stage2d(s, s.q1[0], s.q0[0], 0, 0, dt, 3);
    const int NX = s.nx - 1, NY = s.ny - 1;
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i <= NX; ++i)
            if (s.get(i, j, 0)) {
                const size_t a = s.at(i, j);
                s.q[0][a] = 1.0 / 3.0 * s.q[0][a] + 2.0 / 3.0 * s.q0[0][a];
            }
    for (int j = 1; j <= NY - 1; ++j)
        for (int i = 1; i <= NX - 1; ++i)
            if (!s.get(i, j, 0)) s.q[0][s.at(i, j)] = 0.0;
    if (out)
        for (int k = 0; k < 4; ++k) {
            long c = 0;
            for (int j = 0; j <= NY; ++j)
                for (int i = 0; i <= NX; ++i) c += s.get(i, j, k);
            out[k] = (double)c;
        }
}

void or2d_set_scalar(void* h, int on) { static_cast<O2D*>(h)->scalar = on != 0; }
void or2d_scalar_set_q(void* h, const double* q)
{
    O2D* s = static_cast<O2D*>(h);
    for (size_t a = 0; a < s->plane; ++a) s->q[0][a] = q[a];
}
void or2d_scalar_get_q(void* h, double* q)
{
    O2D* s = static_cast<O2D*>(h);
    for (size_t a = 0; a < s->plane; ++a) q[a] = s->q[0][a];
}
void or2d_scalar_step(void* h, double tol, double dt, double* out) { scalar_step2d(*static_cast<O2D*>(h), tol, dt, out); }

void or2d_interpolate_all(void* h, int from_id)
{
    interp2d(*static_cast<O2D*>(h), bit_of(from_id), -1, 0);
}

void or2d_manager(void* h, int op, int mask_id, int level_id)
{
    O2D& s = *static_cast<O2D*>(h);
    const int b = bit_of(mask_id);
    switch (op) {
        case 0: aaz2d(s, b); break;
        case 1: cr2d(s, b); break;
        case 2: apd2d(s, b, level_id); break;
        case 3: cl2d(s, level_id, b); break;
        case 4: remove_residue_2d(s, b); break;
        case 5: band2d(s, b); break;
        default: break;
    }
}

// The wind tunnel manager's own calls (see ref2d_wt_call): 0 = bottom fill for the x direction,
// 1 = for the y direction, 2 = BandingMask(mask_id).
void or2d_wt_call(void* h, int which, int mask_id)
{
    O2D& s = *static_cast<O2D*>(h);
    if (which == 0) wt_fill_x(s, s.q);
    else if (which == 1) wt_fill_y(s, s.q);
    else band2d(s, bit_of(mask_id));
}

void or2d_apply_bc(void* h, double t)
{
    O2D* s = static_cast<O2D*>(h);
    bc2d(*s, s->q, t);
}

void or2d_step(void* h, double tol, double cfl, double t, double t_next, double dt_fixed, double* alpha_io,
               double* out)
{
    step2d(*static_cast<O2D*>(h), tol, cfl, t, t_next, dt_fixed, alpha_io, out);
}

void or2d_set_freeze(void* h, int freeze) { static_cast<O2D*>(h)->freeze = freeze; }
void or2d_set_wenoz(void* h, double eps, double tau_delta)
{
    static_cast<O2D*>(h)->wz_eps = eps;
    static_cast<O2D*>(h)->wz_delta = tau_delta;
}

int or2d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out)
{
    double t = 0, upd = 0, o[8];
    int n = 0;
    while (n < max_steps) {
        or2d_step(h, tol, cfl, t, t_end, 0.0, nullptr, o);
        t += o[0];
        upd += o[2];
        ++n;
        if (t >= t_end) break;
    }
    out[0] = t;
    out[1] = upd;
    return n;
}

int or2d_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

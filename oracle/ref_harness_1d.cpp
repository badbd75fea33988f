// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// C-ABI harness over the reference's own 1D AWCM Euler code (doseongju/C_pp-library).
// The reference headers are compiled in place from the reference tree by oracle/Makefile;
// nothing of them is copied here.  The reference has no library entry point for the time
// step: its RK3 loop lives inside main() of Wavelet/main_1d_euler.cpp:61-260.  ref1d_step()
// below restates that loop body as a function (same calls, same order, same arithmetic)
// so the checker can drive it step by step.  Two numerics are selectable:
//   scheme 0: WENO-Z face fluxes, WENOZ_EULER_SOLVER_1D::ComputeFlux (WENOZ.h:160-205),
//             applied to the two faces of a point the way WENO_EULER_SOLVER_1D::ComputedF
//             (WENO.h:176-184) does it -- the 1D Sod configuration of the benchmark;
//   scheme 1: the shipped driver's classic WENO5 ComputedF (WENO.h:176-184);
//   scheme 2: the scalar path of Wavelet/main_1d_advect.cpp:48-224 (AWCM_1D::Prepare and
//             PostProcess, WENO5::ReconstructRight, AWCM_1D::Differentiate*), ref1d_scalar_step.
#include "FIELD_UNIFORM_1D.h"

// The reference's ARRAY_1D has no AssignAllValue(), which FIELD_UNIFORM_1D<T>::AssignAllValues
// (FIELD_UNIFORM_1D.h:65-68) calls and AWCM_1D's constructor instantiates for bool
// (Wavelet/AWCM_1D.h:34).  This explicit specialisation supplies the missing behaviour
// (assign every element, ghosts included) without touching the reference sources.
template <>
void FIELD_UNIFORM_1D<bool>::AssignAllValues(const bool& v)
{
    for (int w = 0; w < arr.i_res; ++w) arr.val[w] = v;
}

#include "WENO.h"
#include "WENOZ.h"
#include "ARRAY.h"
#include "ARRAY_1D.h"
#include "Problems/1D/PROBLEM_SHOCKTUBE.h"
#include "Wavelet/AWCM_1D.h"
#include "BOUNDARY_MANAGER_1D.h"

#include <cstdint>
#include <cstring>

namespace {

struct Ref1D {
    MRA_GRID_INT_1D mra;
    AWCM_1D* awcm = nullptr;
    GRID_UNIFORM_1D grid;
    FIELD_UNIFORM_1D<VECTOR_3D<double>> Q, Q_temp, Q_copy;
    BOUNDARY_MANAGER* bc = nullptr;
    // The enum-driven BOUNDARY_MANAGER_1D<VECTOR_3D<double>> (BOUNDARY_MANAGER_1D.h:17-76) and its
    // condition field, used in place of bc once set (ref1d_set_bc_field).
    FIELD_UNIFORM_1D<BOUNDARY_CONDITION> bcf;
    BOUNDARY_MANAGER_1D<VECTOR_3D<double>>* generic = nullptr;
    WENO_EULER_SOLVER_1D* weno = nullptr;
    WENOZ_EULER_SOLVER_1D* wenoz = nullptr;
    FIELD_UNIFORM_1D<double> sq, sq_0, sq_1, sq_2;  // scheme 2: q and the stage fields q_0, q_1, q_2
    WENO5 weno5;
    double gamma = 1.4;
    int scheme = 0;
    int nx = 0;
};

void apply_bc(Ref1D* s)
{
    if (s->generic) s->generic->SetBoundaryCondition(s->Q);
    else s->bc->SetBoundaryCondition();
}

FIELD_UNIFORM_1D<bool>& mask_ref(Ref1D* s, int id)
{
    switch (id) {
        case 0: return s->awcm->mask0;
        case 1: return s->awcm->mask1;
        case 2: return s->awcm->mask2;
        case 3: return s->awcm->mask3;
        default: return s->awcm->mask_temp;
    }
}

FIELD_UNIFORM_1D<int>& level_ref(Ref1D* s, int id)
{
    switch (id) {
        case 0: return s->awcm->level0;
        case 1: return s->awcm->level1;
        case 2: return s->awcm->level2;
        default: return s->awcm->level3;
    }
}

// One RK3 stage of Wavelet/main_1d_euler.cpp (stage bodies :97-136, :153-191, :208-245).
// kind 1: Q = Q - s dF; kind 2: Q = 0.75 Qc + 0.25 (Q - s dF); kind 3: Q = (Qc + 2 (Q - s dF)) / 3.
void stage1d(Ref1D* s, const FIELD_UNIFORM_1D<bool>& mask, const FIELD_UNIFORM_1D<int>& level,
             double alpha_x, double dt, int kind)
{
    const int max_level = s->mra.num_levels - 1;
    const double dx = s->grid.dx;
    FIELD_UNIFORM_1D<VECTOR_3D<double>>& Q = s->Q;
    FIELD_UNIFORM_1D<VECTOR_3D<double>>& Q_temp = s->Q_temp;
    FIELD_UNIFORM_1D<VECTOR_3D<double>>& Q_copy = s->Q_copy;
    AWCM_1D& awcm = *s->awcm;
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (mask(i) == false) continue;
        const int lev = level(i);
        const int dx_ = s->mra.dx[lev];
        VECTOR_3D<double> dF;
        if (lev == max_level) {
            if (s->scheme == 1) {
                s->weno->ComputedF(Q_temp(i - 3), Q_temp(i - 2), Q_temp(i - 1), Q_temp(i), Q_temp(i + 1),
                                   Q_temp(i + 2), Q_temp(i + 3), alpha_x, dF);
            } else {
                VECTOR_3D<double> F_l, F_r;
                s->wenoz->ComputeFlux(Q_temp(i - 3), Q_temp(i - 2), Q_temp(i - 1), Q_temp(i), Q_temp(i + 1),
                                      Q_temp(i + 2), alpha_x, F_l);
                s->wenoz->ComputeFlux(Q_temp(i - 2), Q_temp(i - 1), Q_temp(i), Q_temp(i + 1), Q_temp(i + 2),
                                      Q_temp(i + 3), alpha_x, F_r);
                dF = (F_r - F_l);
            }
        } else {
            const int i_end = s->grid.i_end;
            if (i - 2 * dx_ > 0 && i + 2 * dx_ < i_end)
                awcm.DifferentiateEuler(Q_temp(i - 2 * dx_), Q_temp(i - dx_), Q_temp(i), Q_temp(i + dx_),
                                        Q_temp(i + 2 * dx_), dF);
            else if (i - 2 * dx_ < 0)
                awcm.DifferentiateEulerAtLeftBoundary(Q_temp(i - dx_), Q_temp(i), Q_temp(i + dx_),
                                                      Q_temp(i + 2 * dx_), dF);
            else if (i == 2 * dx_)
                awcm.DifferentiateEulerAtLeftBoundary(Q_temp(i - 2 * dx_), Q_temp(i - dx_), Q_temp(i),
                                                      Q_temp(i + dx_), Q_temp(i + 2 * dx_), dF);
            else if (i > i_end - 2 * dx_)
                awcm.DifferentiateEulerAtRightBoundary(Q_temp(i - 2 * dx_), Q_temp(i - dx_), Q_temp(i),
                                                       Q_temp(i + dx_), dF);
            else
                awcm.DifferentiateEulerAtRightBoundary(Q_temp(i - 2 * dx_), Q_temp(i - dx_), Q_temp(i),
                                                       Q_temp(i + dx_), Q_temp(i + 2 * dx_), dF);
        }
        if (kind == 1)
            Q(i) = Q(i) - dt / (dx * dx_) * dF;
        else if (kind == 2)
            Q(i) = 0.75 * Q_copy(i) + 0.25 * (Q(i) - dt / (dx * dx_) * dF);
        else
            Q(i) = (Q_copy(i) + 2.0 * (Q(i) - dt / (dx * dx_) * dF)) / 3.0;
    }
}

// The 5-point form of AWCM_1D::DifferentiateEulerAtLeftBoundary (Wavelet/AWCM_1D.h:174-185) on
// scalars, with AWCM_1D's own coefficients: main_1d_advect.cpp calls a 6-argument scalar
// DifferentiateAtLeftBoundary (:74, :82 and the same lines of the later stages) that AWCM_1D does
// not declare, so the driver does not compile as shipped; the flux of unit-speed advection is
// the field itself, which makes this the vector form's meaning for a scalar.
double left5(const AWCM_1D& a, double ll, double l, double c, double r, double rr)
{
    return a.d02 * ll + a.d12 * l + a.d22 * c + a.d32 * r + a.d2 * rr;
}

// One stage of Wavelet/main_1d_advect.cpp (:50-99, :100-155, :164-212): out = q, the update of
// the points of the mask, the ghost copies of the end points.
void scalar_stage1d(Ref1D* s, const FIELD_UNIFORM_1D<double>& q, FIELD_UNIFORM_1D<double>& out,
                    const FIELD_UNIFORM_1D<bool>& mask, const FIELD_UNIFORM_1D<int>& level, double dt)
{
    AWCM_1D& awcm = *s->awcm;
    const MRA_GRID_INT_1D& mra = s->mra;
    const int max_lev = mra.num_levels - 1;
    const double dx = s->grid.dx;
    const int i_res = s->nx;
    out = q;
    double dF = 0;
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (mask(i) == false) continue;
        const int lev = level(i);
        const int dx_ = mra.grid[lev].dx;
        if (lev == max_lev) {
            double F_r, F_l;
            s->weno5.ReconstructRight(q(i - 3), q(i - 2), q(i - 1), q(i), q(i + 1), F_l);
            s->weno5.ReconstructRight(q(i - 2), q(i - 1), q(i), q(i + 1), q(i + 2), F_r);
            out(i) = out(i) - dt * (F_r - F_l) / (dx * dx_);
        } else {
            if (i - 2 * dx_ > 0 && i + 2 * dx_ < s->grid.i_end)
                awcm.Differentiate(q(i - 2 * dx_), q(i - dx_), q(i), q(i + dx_), q(i + 2 * dx_), dF);
            else if (i - 2 * dx_ < 0)
                awcm.DifferentiateAtLeftBoundary(q(i - dx_), q(i), q(i + dx_), q(i + 2 * dx_), dF);
            else if (i == 2 * dx_)
                dF = left5(awcm, q(i - 2 * dx_), q(i - dx_), q(i), q(i + dx_), q(i + 2 * dx_));
            else if (i + 2 * dx_ > s->grid.i_end)
                awcm.DifferentiateAtLeftBoundary(q(i + dx_), q(i), q(i - dx_), q(i - 2 * dx_), dF);
            else
                dF = left5(awcm, q(i + 2 * dx_), q(i + dx_), q(i), q(i - dx_), q(i - 2 * dx_));
            out(i) = out(i) - dt / (dx * dx_) * dF;
        }
    }
    out(-1) = out(0);
    out(-2) = out(0);
    out(-3) = out(0);
    out(i_res) = out(i_res - 1);
    out(i_res + 1) = out(i_res - 1);
    out(i_res + 2) = out(i_res - 1);
}

// LF-splitting speed over the finest-level points of a mask (main_1d_euler.cpp:86-95).
double alpha1d(Ref1D* s, const FIELD_UNIFORM_1D<bool>& mask, const FIELD_UNIFORM_1D<int>& level)
{
    const IDEAL_GAS_1D EOS(s->gamma);
    const int max_level = s->mra.num_levels - 1;
    double alpha_x = 0;
    FIELD_UNIFORM_1D<VECTOR_3D<double>>& Q = s->Q;
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (mask(i) == false || level(i) != max_level) continue;
        double u, c;
        u = Q(i)[1] / Q(i)[0];
        c = EOS.c(Q(i));
        alpha_x = MAX(alpha_x, ABS(u) + c);
    }
    return alpha_x;
}

}  // namespace

extern "C" {

void* ref1d_create(int num_levels, int nx_coarse, double x_min, double x_max, double gamma, int scheme)
{
    Ref1D* s = new Ref1D();
    s->mra.Initialize(num_levels, nx_coarse);
    s->awcm = new AWCM_1D(s->mra);
    s->nx = s->mra.Nx;
    s->grid.Initialize(0, s->nx, x_min, x_max);
    s->Q.Initialize(s->grid, 3);
    s->bc = new BOUNDARY_MANAGER(s->Q);
    s->gamma = gamma;
    s->scheme = scheme;
    s->weno = new WENO_EULER_SOLVER_1D(gamma);
    s->wenoz = new WENOZ_EULER_SOLVER_1D(gamma);
    if (scheme == 2) s->sq.Initialize(s->grid, 3);
    return s;
}

void ref1d_destroy(void* h)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    delete s->bc;
    delete s->generic;
    delete s->weno;
    delete s->wenoz;
    delete s->awcm;
    delete s;
}

int ref1d_nx(void* h) { return static_cast<Ref1D*>(h)->nx; }

// q: (Nx+6) x 3 doubles, point i (ghosts -3..Nx+2) at row i+3.
// Scheme 2: the field is component 0 (components 1 and 2 are ignored, and read back as 0).
void ref1d_set_q(void* h, const double* q)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    for (int i = -3; i < s->nx + 3; ++i) {
        if (s->scheme == 2) s->sq(i) = q[(i + 3) * 3];
        else
            for (int p = 0; p < 3; ++p) s->Q(i)[p] = q[(i + 3) * 3 + p];
    }
}

void ref1d_get_q(void* h, double* q)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    for (int i = -3; i < s->nx + 3; ++i)
        for (int p = 0; p < 3; ++p) q[(i + 3) * 3 + p] = s->scheme == 2 ? (p == 0 ? s->sq(i) : 0.0) : s->Q(i)[p];
}

// Sod-type initial state on the cell-centred grid, as SHOCKTUBE::Initialize builds it
// (Problems/1D/PROBLEM_SHOCKTUBE.h:14-54) but with the interface and states as arguments.
void ref1d_init_riemann(void* h, double x_interface, double rho_l, double u_l, double p_l, double rho_r,
                        double u_r, double p_r)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    const IDEAL_GAS_1D EOS(s->gamma);
    ITERATION_GRID_1D(s->grid, 3)
    {
        const double x = s->grid(i);
        double rho, u, p;
        if (x <= x_interface) { rho = rho_l; u = u_l; p = p_l; }
        else { rho = rho_r; u = u_r; p = p_r; }
        s->Q(i)[0] = rho;
        s->Q(i)[1] = rho * u;
        s->Q(i)[2] = EOS.E(rho, u, p);
    }
}

// masks: 5 rows of (Nx+6) bytes: mask_temp, mask0, mask1, mask2, mask3 (ghosts included).
void ref1d_get_masks(void* h, uint8_t* m)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    const int w = s->nx + 6;
    const int ids[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r) {
        FIELD_UNIFORM_1D<bool>& mk = mask_ref(s, ids[r]);
        for (int i = -3; i < s->nx + 3; ++i) m[r * w + i + 3] = mk(i) ? 1 : 0;
    }
}

void ref1d_set_masks(void* h, const uint8_t* m)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    const int w = s->nx + 6;
    const int ids[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r) {
        FIELD_UNIFORM_1D<bool>& mk = mask_ref(s, ids[r]);
        for (int i = -3; i < s->nx + 3; ++i) mk(i) = m[r * w + i + 3] != 0;
    }
}

// levels: 4 rows of Nx ints (level0..level3).
void ref1d_get_levels(void* h, int* lv)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    for (int r = 0; r < 4; ++r) {
        FIELD_UNIFORM_1D<int>& l = level_ref(s, r);
        for (int i = 0; i < s->nx; ++i) lv[r * s->nx + i] = l(i);
    }
}

void ref1d_set_levels(void* h, const int* lv)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    for (int r = 0; r < 4; ++r) {
        FIELD_UNIFORM_1D<int>& l = level_ref(s, r);
        for (int i = 0; i < s->nx; ++i) l(i) = lv[r * s->nx + i];
    }
}

// AWCM_1D::PrepareEuler (Wavelet/AWCM_1D.h:86-120); scheme 2: AWCM_1D::Prepare (:45-72).
void ref1d_prepare(void* h, double tol)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    if (s->scheme == 2) s->awcm->Prepare(s->sq, tol);
    else s->awcm->PrepareEuler(s->Q, tol);
}

void ref1d_fwt(void* h, double tol)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    if (s->scheme == 2) s->awcm->wavelet.ForwardWaveletTransform(s->sq, s->mra, s->awcm->mask0, tol);
    else s->awcm->wavelet.ForwardWaveletTransformEuler(s->Q, s->mra, s->awcm->mask0, tol);
}

void ref1d_iwt(void* h, int mask_id)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    if (s->scheme == 2) s->awcm->wavelet.InverseWaveletTransform(s->sq, s->mra, mask_ref(s, mask_id));
    else s->awcm->wavelet.InverseWaveletTransformEuler(s->Q, s->mra, mask_ref(s, mask_id));
}

// One pass of the loop body of Wavelet/main_1d_advect.cpp:48-224 (it lives inside the driver's
// main()) at the fixed dt.  out[0] = dt, out[1..4] = |mask0..mask3| after Prepare.
void ref1d_scalar_step(void* h, double tol, double dt, double* out)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    AWCM_1D& awcm = *s->awcm;
    FIELD_UNIFORM_1D<double>& q = s->sq;
    awcm.Prepare(q, tol);
    long cnt[4] = {0, 0, 0, 0};
    ITERATION_GRID_1D(s->grid, 0)
    {
        cnt[0] += awcm.mask0(i);
        cnt[1] += awcm.mask1(i);
        cnt[2] += awcm.mask2(i);
        cnt[3] += awcm.mask3(i);
    }
    scalar_stage1d(s, q, s->sq_2, awcm.mask2, awcm.level2, dt);
    scalar_stage1d(s, s->sq_2, s->sq_1, awcm.mask1, awcm.level1, dt);
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (awcm.mask1(i) == false) continue;
        s->sq_1(i) = 0.75 * q(i) + 0.25 * s->sq_1(i);
    }
    scalar_stage1d(s, s->sq_1, s->sq_0, awcm.mask0, awcm.level0, dt);
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (awcm.mask0(i) == false) continue;
        q(i) = 1.0 / 3.0 * q(i) + 2.0 / 3.0 * s->sq_0(i);
    }
    awcm.PostProcess(q);
    out[0] = dt;
    for (int k = 0; k < 4; ++k) out[1 + k] = (double)cnt[k];
}

void ref1d_interpolate(void* h, int from_id, int to_id)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    s->awcm->wavelet.InterpolateEuler(s->Q, s->mra, mask_ref(s, from_id), mask_ref(s, to_id));
}

void ref1d_apply_bc(void* h) { apply_bc(static_cast<Ref1D*>(h)); }

// bc: Nx+6 BOUNDARY_CONDITION values; the generic manager takes over the ghost fills.
void ref1d_set_bc_field(void* h, const int* bc)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    s->bcf.Initialize(s->grid, 3);
    for (int i = -3; i < s->nx + 3; ++i) s->bcf(i) = (BOUNDARY_CONDITION)bc[i + 3];
    delete s->generic;
    s->generic = new BOUNDARY_MANAGER_1D<VECTOR_3D<double>>(s->bcf);
}

// The reference's EULER_EQUATION_1D itself over n states of 3 doubles.
void ref_euler1d_flux(const double* q, double* f, int n, double gamma)
{
    const EULER_EQUATION_1D eq(gamma);
    for (int t = 0; t < n; ++t) {
        VECTOR_3D<double> Q(q[3 * t], q[3 * t + 1], q[3 * t + 2]), fu;
        eq.ComputeFu(Q, fu);
        for (int k = 0; k < 3; ++k) f[3 * t + k] = fu[k];
    }
}
void ref_euler1d_sr(const double* q, double* out, int n, double gamma)
{
    const EULER_EQUATION_1D eq(gamma);
    for (int t = 0; t < n; ++t) out[t] = eq.Spectral_Radius(VECTOR_3D<double>(q[3 * t], q[3 * t + 1], q[3 * t + 2]));
}

// AWCM_MANAGER_1D passes on one of the facade's masks.
// op 0 AddAdjacentZone, 1 CheckReconstruction, 2 AddPointForDifferentiation(level_id),
// 3 ComputeLevel(level_id <- mask), 4 RemoveResidue(Q, mask), 5 BadingBoundary.
void ref1d_manager(void* h, int op, int mask_id, int level_id)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    FIELD_UNIFORM_1D<bool>& m = mask_ref(s, mask_id);
    switch (op) {
        case 0: AWCM_MANAGER_1D::AddAdjacentZone(m, s->mra); break;
        case 1: AWCM_MANAGER_1D::CheckReconstruction(m, s->mra); break;
        case 2: AWCM_MANAGER_1D::AddPointForDifferentiation(m, s->mra, level_ref(s, level_id)); break;
        case 3: AWCM_MANAGER_1D::ComputeLevel(level_ref(s, level_id), m, s->mra); break;
        case 4: AWCM_MANAGER_1D::RemoveResidue(s->Q, m, s->mra); break;
        case 5: s->awcm->BadingBoundary(m); break;
        default: break;
    }
}

// One pass of the driver loop, Wavelet/main_1d_euler.cpp:61-259, with the output time
// t_next standing in for arr_printing_times[cnt].
// out[0] = dt, out[1] = do_print, out[2..5] = |mask0..mask3| after PrepareEuler,
// out[6..8] = alpha_x of the three stages, out[9] = max_velocity.
void ref1d_step(void* h, double tol, double cfl, double t, double t_next, double* out)
{
    Ref1D* s = static_cast<Ref1D*>(h);
    AWCM_1D& awcm = *s->awcm;
    FIELD_UNIFORM_1D<VECTOR_3D<double>>& Q = s->Q;
    const IDEAL_GAS_1D EOS(s->gamma);
    const double dx = s->grid.dx;

    awcm.PrepareEuler(Q, tol);

    double max_velocity = 0;
    ITERATION_GRID_1D(s->grid, 0)
    {
        if (awcm.mask3(i) == false) continue;
        const double c = EOS.c(Q(i));
        const double u = Q(i)[1] / Q(i)[0];
        max_velocity = MAX(max_velocity, (ABS(u) + c));
    }
    double dt = cfl * dx / max_velocity;
    int do_print = 0;
    if (t + dt > t_next) {
        dt = t_next - t;
        do_print = 1;
    }
    long cnt[4] = {0, 0, 0, 0};
    for (int i = 0; i < s->nx; ++i) {
        cnt[0] += awcm.mask0(i);
        cnt[1] += awcm.mask1(i);
        cnt[2] += awcm.mask2(i);
        cnt[3] += awcm.mask3(i);
    }

    apply_bc(s);
    double a1 = alpha1d(s, awcm.mask3, awcm.level3);
    s->Q_copy = Q;
    s->Q_temp = Q;
    stage1d(s, awcm.mask2, awcm.level2, a1, dt, 1);

    apply_bc(s);
    double a2 = alpha1d(s, awcm.mask2, awcm.level2);
    s->Q_temp = Q;
    stage1d(s, awcm.mask1, awcm.level1, a2, dt, 2);

    apply_bc(s);
    double a3 = alpha1d(s, awcm.mask1, awcm.level1);
    s->Q_temp = Q;
    stage1d(s, awcm.mask0, awcm.level0, a3, dt, 3);

    awcm.PostProcessEuler(Q);

    out[0] = dt;
    out[1] = do_print;
    for (int k = 0; k < 4; ++k) out[2 + k] = (double)cnt[k];
    out[6] = a1;
    out[7] = a2;
    out[8] = a3;
    out[9] = max_velocity;
}

// Runs steps until t >= t_end (the driver's loop with a single output time), or max_steps.
// Returns the number of steps; out[0] = final t, out[1] = sum over steps of |mask0|.
int ref1d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out)
{
    double t = 0, upd = 0, o[10];
    int n = 0;
    while (n < max_steps) {
        ref1d_step(h, tol, cfl, t, t_end, o);
        t += o[0];
        upd += o[2];
        ++n;
        if (t >= t_end) break;
    }
    out[0] = t;
    out[1] = upd;
    return n;
}

}  // extern "C"

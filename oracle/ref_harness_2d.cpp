// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// C-ABI harness over the reference's own 2D AWCM Euler code (doseongju/C_pp-library),
// compiled in place from the reference tree by oracle/Makefile (no reference source is
// copied here).  The reference's step loop is main() of Wavelet/main_2d_euler(quad).cpp:56-350
// (and the double-Mach variant Wavelet/main_2d_euler(dmach).cpp, which differs only in the
// problem and in passing t to the boundary manager); ref2d_step() restates one pass of it as a
// function with the same calls, order and arithmetic, OpenMP included.
#include "OMP_MANAGER.h"
#include "Problems/2D/PROBLEM_QUADRANTS.h"
#include "Problems/2D/PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h"
#include "Problems/2D/PROBLEM_BOX_ADVECTION.h"
#include "AWCM_2D.h"
#include "WENO.h"
#include "WENOZ.h"
#include "EULER_EQUATION.h"
#include "BOUNDARY_MANAGER_2D.h"

#include <cstdint>
#include <omp.h>
#include <vector>

namespace {

enum { BC_QUAD = 0, BC_DMACH = 1, BC_PERIODIC = 2, BC_SHOCK_VORTEX = 3, BC_WIND_TUNNEL = 5 };

// One boundary manager per field, of the kind the problem uses, or the enum-driven
// BOUNDARY_MANAGER_2D<VECTOR_4D<double>> (BOUNDARY_MANAGER_2D.h:23-159) once a condition field is set.
struct BC2D {
    int kind;
    BOUNDARY_MANAGER_QUAD* quad = nullptr;
    BOUNDARY_MANAGER_DMACH* dmach = nullptr;
    BOUNDARY_MANAGER_ISENVORTEX* periodic = nullptr;
    BOUNDARY_MANAGER_SHOCK_VORTEX* shock_vortex = nullptr;
    BOUNDARY_MANAGER_2D<VECTOR_4D<double>>* generic = nullptr;
    BOUNDARY_MANAGER_WT* wt = nullptr;
    FIELD_UNIFORM_2D<VECTOR_4D<double>>* field;
    BC2D(int k, FIELD_UNIFORM_2D<VECTOR_4D<double>>& Q) : kind(k), field(&Q)
    {
        if (k == BC_WIND_TUNNEL) wt = new BOUNDARY_MANAGER_WT(Q);
        else if (k == BC_DMACH) dmach = new BOUNDARY_MANAGER_DMACH(Q);
        else if (k == BC_PERIODIC) periodic = new BOUNDARY_MANAGER_ISENVORTEX(Q);
        else if (k == BC_SHOCK_VORTEX) shock_vortex = new BOUNDARY_MANAGER_SHOCK_VORTEX(Q);
        else quad = new BOUNDARY_MANAGER_QUAD(Q);
    }
    ~BC2D()
    {
        delete quad;
        delete dmach;
        delete periodic;
        delete shock_vortex;
        delete generic;
        delete wt;
    }
    // The wind tunnel's SetBoundaryCondition fills left, right and top ("Except bottom boundary!!",
    // PROBLEM_WINDTUNNEL.h:193-199); its bottom fills are per sweep direction (stage_input_wt).
    void apply(double t)
    {
        if (generic) generic->SetBoundaryCondition(*field);
        else if (wt) wt->SetBoundaryCondition();
        else if (dmach) dmach->SetBoundaryCondition(t);
        else if (periodic) periodic->SetBoundaryCondition();
        else if (shock_vortex) shock_vortex->SetBoundaryCondition();
        else quad->SetBoundaryCondition();
    }
};

struct Ref2D {
    MRA_GRID_INT_2D mra;
    AWCM_2D* awcm = nullptr;
    GRID_UNIFORM_2D grid;
    FIELD_UNIFORM_2D<VECTOR_4D<double>> Q, Q_0, Q_1, Q_2;
    BC2D *bc = nullptr, *bc0 = nullptr, *bc1 = nullptr, *bc2 = nullptr;
    double gamma = 1.4;
    int nx = 0, ny = 0;
    int bc_kind = BC_QUAD;
    // When set, ref2d_step skips PrepareEuler and PostProcessEuler (masks/levels stay as stored)
    // and, given an alpha buffer, takes the three LF speeds from it instead of recomputing them.
    int freeze_mask = 0;
    // Value given to the public member WENOZ5::eps (WENOZ.h:13-18) of every WENOZ_EULER_SOLVER_2D
    // the stages construct; the solver's own default is 1e-40.
    double wenoz_eps = 1e-40;
    // Scalar AWCM (Wavelet/main_2d_advect.cpp): the field and its stage copies, each with the
    // periodic BOUNDARY_MANAGER of Problems/2D/PROBLEM_BOX_ADVECTION.h; created by ref2d_set_scalar.
    FIELD_UNIFORM_2D<double> S, S_0, S_1, S_2;
    BOUNDARY_MANAGER *bs = nullptr, *bs1 = nullptr, *bs2 = nullptr;
    // The condition field of the enum-driven manager (ref2d_set_bc_field).
    FIELD_UNIFORM_2D<BOUNDARY_CONDITION> bcf;
    // Wind tunnel: the x-sweep copy of a stage input (its bottom filled for the x direction).
    FIELD_UNIFORM_2D<VECTOR_4D<double>> Qx;
};

// The stage input of the wind tunnel (BOUNDARY_MANAGER_WT, Problems/2D/PROBLEM_WINDTUNNEL.h:52-222):
// after SetBoundaryCondition (left, right, top), the x-direction fluxes read a copy with
// SetBottomBoundaryCondition(true, false) applied (the step's front face), while the field itself
// takes the x- and then the y-direction bottom fill (bottom wall, step top) and feeds the
// y-direction fluxes, the LF speeds and the point updates.
void stage_input_wt(Ref2D* s, FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qs)
{
    for (int j = Qs.j_start_g; j <= Qs.j_end_g; ++j)
        for (int i = Qs.i_start_g; i <= Qs.i_end_g; ++i) s->Qx(i, j) = Qs(i, j);
    BOUNDARY_MANAGER_WT(s->Qx).SetBottomBoundaryCondition(true, false);
    BOUNDARY_MANAGER_WT bm(Qs);
    bm.SetBottomBoundaryCondition(true, false);
    bm.SetBottomBoundaryCondition(false, true);
}

// AWCM_2D::PrepareEuler (Wavelet/AWCM_2D.h:114-147) with the wind tunnel's BandingMask in place
// of the shock-vortex one: the alternative the reference leaves commented out at AWCM_2D.h:121.
void prepare_euler_wt(Ref2D* s, double tol)
{
    AWCM_2D& a = *s->awcm;
    FIELD_UNIFORM_2D<VECTOR_4D<double>>& q = s->Q;
    a.mask_temp = a.mask0;
    a.wavelet.ForwardWaveletTransformationEuler(q, a.mra_grid, a.mask0, tol);
    BOUNDARY_MANAGER_WT boundary_manager(q);
    boundary_manager.BandingMask(a.mask0);
    AWCM_MANAGER_2D::AddAdjacentZone(a.mask0, a.mra_grid);
    AWCM_MANAGER_2D::CheckReconstruction(a.mask0, a.mra_grid);
    a.mask1 = a.mask0;
    AWCM_MANAGER_2D::ComputeLevel(a.level0, a.mask0, a.mra_grid);
    AWCM_MANAGER_2D::AddPointForDifferentiation(a.mask1, a.mra_grid, a.level0);
    AWCM_MANAGER_2D::CheckReconstruction(a.mask1, a.mra_grid);
    a.mask2 = a.mask1;
    AWCM_MANAGER_2D::ComputeLevel(a.level1, a.mask1, a.mra_grid);
    AWCM_MANAGER_2D::AddPointForDifferentiation(a.mask2, a.mra_grid, a.level1);
    AWCM_MANAGER_2D::CheckReconstruction(a.mask2, a.mra_grid);
    a.mask3 = a.mask2;
    AWCM_MANAGER_2D::ComputeLevel(a.level2, a.mask2, a.mra_grid);
    AWCM_MANAGER_2D::AddPointForDifferentiation(a.mask3, a.mra_grid, a.level2);
    AWCM_MANAGER_2D::CheckReconstruction(a.mask3, a.mra_grid);
    a.wavelet.InverseWaveletTransformationEuler(q, a.mra_grid, a.mask3);
    a.wavelet.InterpolateEuler(q, a.mra_grid, a.mask_temp, a.mask3);
}

FIELD_UNIFORM_2D<bool>& mask_ref(Ref2D* s, int id)
{
    switch (id) {
        case 0: return s->awcm->mask0;
        case 1: return s->awcm->mask1;
        case 2: return s->awcm->mask2;
        case 3: return s->awcm->mask3;
        default: return s->awcm->mask_temp;
    }
}

FIELD_UNIFORM_2D<int>& level_ref(Ref2D* s, int id)
{
    switch (id) {
        case 0: return s->awcm->level0;
        case 1: return s->awcm->level1;
        case 2: return s->awcm->level2;
        default: return s->awcm->level3;
    }
}

// Per-row and per-column LF speeds over a mask (main_2d_euler(quad).cpp:86-104).
void alpha2d(Ref2D* s, const FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qs, const FIELD_UNIFORM_2D<bool>& mask,
             std::vector<double>& alpha_x, std::vector<double>& alpha_y)
{
    EULER_EQUATION_2D euler_eqn(s->gamma);
    const GRID_UNIFORM_2D& grid = s->grid;
    for (auto& a : alpha_x) a = 0;
    for (auto& a : alpha_y) a = 0;
#pragma omp parallel
    {
#pragma omp for
        ITERATION_GRID_2D(grid, 0)
        {
            if (mask(i, j) == 0) continue;
            alpha_x[j] = MAX(alpha_x[j], euler_eqn.Spectral_RadiusX(Qs(i, j)));
        }
#pragma omp for
        ITERATION_GRID_2D_IJ(grid, 0)
        {
            if (mask(i, j) == 0) continue;
            alpha_y[i] = MAX(alpha_y[i], euler_eqn.Spectral_RadiusY(Qs(i, j)));
        }
    }
}

// One RK3 stage body (main_2d_euler(quad).cpp:108-163, :188-243, :267-322).
// out = Qin - dt/dx (dF + dG)                      (kind 1, 3)
// out = 0.75 Qn + 0.25 (Qin - dt/dx (dF + dG))     (kind 2)
// Qx: the field the x-direction fluxes read (the wind tunnel's x-sweep copy), else Qin.
void stage2d(Ref2D* s, const FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qin, FIELD_UNIFORM_2D<VECTOR_4D<double>>& out,
             const FIELD_UNIFORM_2D<bool>& mask, const FIELD_UNIFORM_2D<int>& level,
             const std::vector<double>& alpha_x, const std::vector<double>& alpha_y, double dt, int kind,
             const FIELD_UNIFORM_2D<VECTOR_4D<double>>* Qx_ = nullptr)
{
    const FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qx = Qx_ ? *Qx_ : Qin;
    const int max_lev = s->mra.num_levels - 1;
    const GRID_UNIFORM_2D& grid = s->grid;
    const FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qn = s->Q;
    AWCM_2D& awcm = *s->awcm;
    EULER_EQUATION_2D euler_eqn(s->gamma);
#pragma omp parallel
    {
        WENOZ_EULER_SOLVER_2D wenoz_solver;
        wenoz_solver.wenoz.eps = s->wenoz_eps;
#pragma omp for
        ITERATION_GRID_2D(grid, 0)
        {
            VECTOR_4D<double> dF, dG;
            VECTOR_4D<double> F_ll, F_l, F_c, F_r, F_rr;
            VECTOR_4D<double> G_bb, G_b, G_c, G_t, G_tt;
            if (mask(i, j) == false) continue;
            const int lev = level(i, j);
            const int d = s->mra.grid[lev].dx;
            const double dx = grid.dx * d;
            if (lev == max_lev) {
                VECTOR_4D<double> a, b;
                wenoz_solver.ComputeFluxX(Qx(i - 3, j), Qx(i - 2, j), Qx(i - 1, j), Qx(i, j), Qx(i + 1, j),
                                          Qx(i + 2, j), alpha_x[j], a);
                wenoz_solver.ComputeFluxX(Qx(i - 2, j), Qx(i - 1, j), Qx(i, j), Qx(i + 1, j), Qx(i + 2, j),
                                          Qx(i + 3, j), alpha_x[j], b);
                dF = b - a;
                wenoz_solver.ComputeFluxY(Qin(i, j - 3), Qin(i, j - 2), Qin(i, j - 1), Qin(i, j), Qin(i, j + 1),
                                          Qin(i, j + 2), alpha_y[i], a);
                wenoz_solver.ComputeFluxY(Qin(i, j - 2), Qin(i, j - 1), Qin(i, j), Qin(i, j + 1), Qin(i, j + 2),
                                          Qin(i, j + 3), alpha_y[i], b);
                dG = b - a;
            } else {
                // The reference evaluates F (G) at all five points; the ones its branch does not use
                // (i-2d when i <= d, i+2d when i >= i_end-d) can lie outside the field, so they are skipped.
                if (i > d) euler_eqn.ComputeFu(Qx(i - 2 * d, j), F_ll);
                euler_eqn.ComputeFu(Qx(i - d, j), F_l), euler_eqn.ComputeFu(Qx(i, j), F_c);
                euler_eqn.ComputeFu(Qx(i + d, j), F_r);
                if (i <= d || i < grid.i_end - d) euler_eqn.ComputeFu(Qx(i + 2 * d, j), F_rr);
                if (i <= d)
                    awcm.DifferentiateAtLeftBoundary(F_l, F_c, F_r, F_rr, dF);
                else if (i >= grid.i_end - d)
                    awcm.DifferentiateAtRightBoundary(F_ll, F_l, F_c, F_r, dF);
                else
                    awcm.Differentiate(F_ll, F_l, F_c, F_r, F_rr, dF);

                if (j > d) euler_eqn.ComputeGu(Qin(i, j - 2 * d), G_bb);
                euler_eqn.ComputeGu(Qin(i, j - d), G_b), euler_eqn.ComputeGu(Qin(i, j), G_c);
                euler_eqn.ComputeGu(Qin(i, j + d), G_t);
                if (j <= d || j < grid.j_end - d) euler_eqn.ComputeGu(Qin(i, j + 2 * d), G_tt);
                if (j <= d)
                    awcm.DifferentiateAtLeftBoundary(G_b, G_c, G_t, G_tt, dG);
                else if (j >= grid.j_end - d)
                    awcm.DifferentiateAtRightBoundary(G_bb, G_b, G_c, G_t, dG);
                else
                    awcm.Differentiate(G_bb, G_b, G_c, G_t, G_tt, dG);
            }
            if (kind == 2)
                out(i, j) = 0.75 * Qn(i, j) + 0.25 * (Qin(i, j) - dt / dx * (dF + dG));
            else
                out(i, j) = Qin(i, j) - dt / dx * (dF + dG);
        }
    }
}

}  // namespace

extern "C" {

// bc_kind: 0 transmissive (BOUNDARY_MANAGER_QUAD), 1 double Mach (BOUNDARY_MANAGER_DMACH),
// 2 periodic (BOUNDARY_MANAGER_ISENVORTEX).
void* ref2d_create(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                   double y_max, int bc_kind)
{
    Ref2D* s = new Ref2D();
    s->mra.Initialize(num_levels, nx_coarse, ny_coarse);
    s->awcm = new AWCM_2D(s->mra);
    s->nx = s->mra.Nx;
    s->ny = s->mra.Ny;
    s->bc_kind = bc_kind;
    s->grid.Initialize(0, 0, s->nx, s->ny, x_min, y_min, x_max, y_max);
    s->Q.Initialize(s->grid, 3);
    s->Q_0.Initialize(s->grid, 3);
    s->Q_1.Initialize(s->grid, 3);
    s->Q_2.Initialize(s->grid, 3);
    s->Qx.Initialize(s->grid, 3);
    s->bc = new BC2D(bc_kind, s->Q);
    s->bc0 = new BC2D(bc_kind, s->Q_0);
    s->bc1 = new BC2D(bc_kind, s->Q_1);
    s->bc2 = new BC2D(bc_kind, s->Q_2);
    return s;
}

void ref2d_destroy(void* h)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    delete s->bc;
    delete s->bc0;
    delete s->bc1;
    delete s->bc2;
    delete s->bs;
    delete s->bs1;
    delete s->bs2;
    delete s->awcm;
    delete s;
}

void ref2d_dims(void* h, int* nx, int* ny)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    *nx = s->nx;
    *ny = s->ny;
}

// q: (Ny+6) rows of (Nx+6) points x 4 doubles, point (i,j) at ((j+3)*(Nx+6) + i+3)*4.
void ref2d_set_q(void* h, const double* q)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    for (int j = -3; j < s->ny + 3; ++j)
        for (int i = -3; i < s->nx + 3; ++i)
            for (int p = 0; p < 4; ++p) s->Q(i, j)[p] = q[((size_t)(j + 3) * w + (i + 3)) * 4 + p];
}

void ref2d_get_q(void* h, double* q)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    for (int j = -3; j < s->ny + 3; ++j)
        for (int i = -3; i < s->nx + 3; ++i)
            for (int p = 0; p < 4; ++p) q[((size_t)(j + 3) * w + (i + 3)) * 4 + p] = s->Q(i, j)[p];
}

// Initial states built by the reference's problem classes, with the geometry of the harness grid.
// kind 0: four-quadrant Riemann problem, QUADRANTS::Initialize states (PROBLEM_QUADRANTS.h:42-78)
//         with the split at (a, b);
// kind 1: double Mach reflection, DOUBLEMACH::Initialize (PROBLEM_DOUBLEMACH.h:34-62) with the
//         pre-shock density a;
// kind 2: isentropic vortex, ISENTROPIC_VORTEX_ADVECTION::Initialize (:38-64) centred at (a, b).
void ref2d_init_problem(void* h, int kind, double a, double b)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const double gamma = s->gamma;
    IDEAL_GAS_2D EOS(gamma);
    const GRID_UNIFORM_2D& grid = s->grid;
    FIELD_UNIFORM_2D<VECTOR_4D<double>>& Q = s->Q;
    ITERATION_GRID_2D(grid, 3)
    {
        const double x = grid(i, j).x;
        const double y = grid(i, j).y;
        double rho, u, v, p;
        if (kind == 0) {
            if (x >= a && y >= b) { rho = 1.5; u = 0; v = 0; p = 1.5; }
            else if (x < a && y >= b) { rho = 0.532258064516129; u = 1.206045378311055; v = 0; p = 0.3; }
            else if (x < a && y < b) {
                rho = 0.137992831541219; u = 1.206045378311055; v = 1.206045378311055; p = 0.029032258064516;
            } else { rho = 0.532258064516129; u = 0; v = 1.206045378311055; p = 0.3; }
            Q(i, j)[0] = rho;
            Q(i, j)[1] = rho * u;
            Q(i, j)[2] = rho * v;
            Q(i, j)[3] = EOS.E(rho, u, v, p);
        } else if (kind == 1) {
            if (y > sqrt(3.0) * (x - 1.0 / 6.0)) { rho = 8; u = 8.25 * sqrt(3.0) * 0.5; v = -8.25 * 0.5; p = 116.5; }
            else { rho = a; u = 0; v = 0; p = 1; }
            Q(i, j)[0] = rho;
            Q(i, j)[1] = rho * u;
            Q(i, j)[2] = rho * v;
            Q(i, j)[3] = EOS.E(rho, u, v, p);
        } else if (kind == 4) {
            // WINDTUNNEL::Initialize (Problems/2D/PROBLEM_WINDTUNNEL.h:14-47): Mach 3 uniform flow
            rho = 1.4; u = 3; v = 0; p = 1;
            Q(i, j)[0] = rho;
            Q(i, j)[1] = rho * u;
            Q(i, j)[2] = rho * v;
            Q(i, j)[3] = EOS.E(rho, u, v, p);
        } else if (kind == 3) {
            // SHOCK_VORTEX::Initialize (Problems/2D/PROBLEM_SHOCK_VORTEX_INTERACTION.h:32-66), vortex at (a, b)
            const double M_v = 0.5;
            const double r = sqrt(SQR(x - a) + SQR(y - b));
            if (x <= 0) { rho = 1.394708041144614; u = -0.860403729339060; v = 0; p = 1.121834000000000; }
            else {
                rho = 1 - (gamma - 1) / 2 * SQR(M_v) * exp(1 - r * r);
                rho = pow(rho, 1 / (gamma - 1));
                p = 1 - (gamma - 1) / 2 * SQR(M_v) * exp(1 - r * r);
                p = pow(p, gamma / (gamma - 1));
                p = 1 / gamma * p;
                u = M_v * exp(0.5 * (1 - r * r)) * (-y) - 1.200011999940001;
                v = M_v * exp(0.5 * (1 - r * r)) * (x - a);
            }
            Q(i, j)[0] = rho;
            Q(i, j)[1] = rho * u;
            Q(i, j)[2] = rho * v;
            Q(i, j)[3] = EOS.E(rho, u, v, p);
        } else {
            const double rr = SQR(x - a) + SQR(y - b);
            const double beta = 5;
            double rhou, rhov;
            rho = 1 - (gamma - 1) * SQR(beta) / (8 * gamma * PI * PI) * exp(1 - rr);
            rho = pow(rho, 1.0 / (gamma - 1.0));
            rhou = 0 - beta / (2 * PI) * exp((1 - rr) * 0.5) * (y - b);
            rhou *= rho;
            rhov = 1 + beta / (2 * PI) * exp((1 - rr) * 0.5) * (x - a);
            rhov *= rho;
            p = pow(rho, gamma);
            Q(i, j)[0] = rho;
            Q(i, j)[1] = rhou;
            Q(i, j)[2] = rhov;
            Q(i, j)[3] = EOS.E(rho, rhou / rho, rhov / rho, p);
        }
    }
}

// masks: 5 planes of (Ny+6) x (Nx+6) bytes: mask_temp, mask0..mask3 (ghosts included).
void ref2d_get_masks(void* h, uint8_t* m)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    const size_t plane = (size_t)w * (s->ny + 6);
    const int ids[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r) {
        FIELD_UNIFORM_2D<bool>& mk = mask_ref(s, ids[r]);
        for (int j = -3; j < s->ny + 3; ++j)
            for (int i = -3; i < s->nx + 3; ++i) m[r * plane + (size_t)(j + 3) * w + i + 3] = mk(i, j) ? 1 : 0;
    }
}

void ref2d_set_masks(void* h, const uint8_t* m)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    const size_t plane = (size_t)w * (s->ny + 6);
    const int ids[5] = {4, 0, 1, 2, 3};
    for (int r = 0; r < 5; ++r) {
        FIELD_UNIFORM_2D<bool>& mk = mask_ref(s, ids[r]);
        for (int j = -3; j < s->ny + 3; ++j)
            for (int i = -3; i < s->nx + 3; ++i) mk(i, j) = m[r * plane + (size_t)(j + 3) * w + i + 3] != 0;
    }
}

// levels: 4 planes of Ny x Nx ints.
void ref2d_get_levels(void* h, int* lv)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const size_t plane = (size_t)s->nx * s->ny;
    for (int r = 0; r < 4; ++r) {
        FIELD_UNIFORM_2D<int>& l = level_ref(s, r);
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) lv[r * plane + (size_t)j * s->nx + i] = l(i, j);
    }
}

void ref2d_set_levels(void* h, const int* lv)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const size_t plane = (size_t)s->nx * s->ny;
    for (int r = 0; r < 4; ++r) {
        FIELD_UNIFORM_2D<int>& l = level_ref(s, r);
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) l(i, j) = lv[r * plane + (size_t)j * s->nx + i];
    }
}

// AWCM_2D::PrepareEuler (Wavelet/AWCM_2D.h:114-147).
void ref2d_prepare(void* h, double tol)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->awcm->PrepareEuler(s->Q, tol);
}

void ref2d_fwt(void* h, double tol)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->awcm->wavelet.ForwardWaveletTransformationEuler(s->Q, s->mra, s->awcm->mask0, tol);
}

void ref2d_iwt(void* h, int mask_id)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->awcm->wavelet.InverseWaveletTransformationEuler(s->Q, s->mra, mask_ref(s, mask_id));
}

void ref2d_interpolate(void* h, int from_id, int to_id)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->awcm->wavelet.InterpolateEuler(s->Q, s->mra, mask_ref(s, from_id), mask_ref(s, to_id));
}

void ref2d_interpolate_all(void* h, int from_id)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->awcm->wavelet.InterpolateAllGridEuler(s->Q, s->mra, mask_ref(s, from_id));
}

// Scalar AWCM: one pass of the loop of Wavelet/main_2d_advect.cpp:48-190 (AWCM_2D::Prepare, the box
// manager's periodic fill, three SSP-RK3 stages of unit-velocity advection with WENO5 upwind faces on
// the finest level and AWCM_2D::Differentiate* below, 1/3 Q + 2/3 Q_0 on mask0, PostProcess),
// restated as a function with the same calls, order and arithmetic.  out[4] = |mask0..mask3|.
void ref2d_set_scalar(void* h, int on)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    if (!on || s->bs) return;
    for (FIELD_UNIFORM_2D<double>* f : {&s->S, &s->S_0, &s->S_1, &s->S_2}) {
        f->Initialize(s->grid, 3);
        f->AssignAllValues(0.0);
    }
    s->bs = new BOUNDARY_MANAGER(s->S);
    s->bs1 = new BOUNDARY_MANAGER(s->S_1);
    s->bs2 = new BOUNDARY_MANAGER(s->S_2);
}

void ref2d_scalar_set_q(void* h, const double* q)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    for (int j = -3; j < s->ny + 3; ++j)
        for (int i = -3; i < s->nx + 3; ++i) s->S(i, j) = q[(size_t)(j + 3) * w + (i + 3)];
}

void ref2d_scalar_get_q(void* h, double* q)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    const int w = s->nx + 6;
    for (int j = -3; j < s->ny + 3; ++j)
        for (int i = -3; i < s->nx + 3; ++i) q[(size_t)(j + 3) * w + (i + 3)] = s->S(i, j);
}

void ref2d_scalar_step(void* h, double tol, double dt, double* out)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    AWCM_2D& awcm = *s->awcm;
    const GRID_UNIFORM_2D& grid = s->grid;
    MRA_GRID_INT_2D& mra_grid = s->mra;
    const int max_lev = mra_grid.num_levels - 1;
    FIELD_UNIFORM_2D<double>& Q = s->S;
    WENO5 weno;
    auto stage = [&](FIELD_UNIFORM_2D<double>& in, FIELD_UNIFORM_2D<double>& res, FIELD_UNIFORM_2D<bool>& mask,
                     FIELD_UNIFORM_2D<int>& level, int kind) {
        ITERATION_GRID_2D(grid, 0)
        {
            double dF = 0, dG = 0;
            if (mask(i, j) == false) continue;
            const int lev = level(i, j);
            const int d = mra_grid.grid[lev].dx;
            const double dx = grid.dx * d;
            if (lev == max_lev) {
                double a, b;
                weno.ReconstructRight(in(i - 3, j), in(i - 2, j), in(i - 1, j), in(i, j), in(i + 1, j), a);
                weno.ReconstructRight(in(i - 2, j), in(i - 1, j), in(i, j), in(i + 1, j), in(i + 2, j), b);
                dF = b - a;
                weno.ReconstructRight(in(i, j - 3), in(i, j - 2), in(i, j - 1), in(i, j), in(i, j + 1), a);
                weno.ReconstructRight(in(i, j - 2), in(i, j - 1), in(i, j), in(i, j + 1), in(i, j + 2), b);
                dG = b - a;
            } else {
                if (i <= d) awcm.DifferentiateAtLeftBoundary(in(i - d, j), in(i, j), in(i + d, j), in(i + 2 * d, j), dF);
                else if (i >= grid.i_end - d)
                    awcm.DifferentiateAtRightBoundary(in(i - 2 * d, j), in(i - d, j), in(i, j), in(i + d, j), dF);
                else awcm.Differentiate(in(i - 2 * d, j), in(i - d, j), in(i, j), in(i + d, j), in(i + 2 * d, j), dF);
                if (j <= d) awcm.DifferentiateAtLeftBoundary(in(i, j - d), in(i, j), in(i, j + d), in(i, j + 2 * d), dG);
                else if (j >= grid.j_end - d)
                    awcm.DifferentiateAtRightBoundary(in(i, j - 2 * d), in(i, j - d), in(i, j), in(i, j + d), dG);
                else awcm.Differentiate(in(i, j - 2 * d), in(i, j - d), in(i, j), in(i, j + d), in(i, j + 2 * d), dG);
            }
            if (kind == 2) res(i, j) = 0.75 * Q(i, j) + 0.25 * (in(i, j) - dt / dx * (dF + dG));
            else res(i, j) = in(i, j) - dt / dx * (dF + dG);
        }
    };
    awcm.Prepare(Q, tol);
    s->bs->SetBoundaryCondition();
    stage(Q, s->S_2, awcm.mask2, awcm.level2, 1);
    s->bs2->SetBoundaryCondition();
    stage(s->S_2, s->S_1, awcm.mask1, awcm.level1, 2);
    s->bs1->SetBoundaryCondition();
    stage(s->S_1, s->S_0, awcm.mask0, awcm.level0, 3);
    ITERATION_GRID_2D(grid, 0)
    {
        if (awcm.mask0(i, j) == true) Q(i, j) = (1.0 / 3.0 * Q(i, j) + 2.0 / 3.0 * s->S_0(i, j));
    }
    awcm.PostProcess(Q);
    if (out) {
        long cnt[4] = {0, 0, 0, 0};
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                cnt[0] += awcm.mask0(i, j);
                cnt[1] += awcm.mask1(i, j);
                cnt[2] += awcm.mask2(i, j);
                cnt[3] += awcm.mask3(i, j);
            }
        for (int k = 0; k < 4; ++k) out[k] = (double)cnt[k];
    }
}

// AWCM_MANAGER_2D passes on one of the facade's masks.
// op 0 AddAdjacentZone, 1 CheckReconstruction, 2 AddPointForDifferentiation(level_id),
// 3 ComputeLevel(level_id <- mask), 4 RemoveResidueEuler(Q, mask), 5 BandingMask.
void ref2d_manager(void* h, int op, int mask_id, int level_id)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    FIELD_UNIFORM_2D<bool>& m = mask_ref(s, mask_id);
    switch (op) {
        case 0: AWCM_MANAGER_2D::AddAdjacentZone(m, s->mra); break;
        case 1: AWCM_MANAGER_2D::CheckReconstruction(m, s->mra); break;
        case 2: AWCM_MANAGER_2D::AddPointForDifferentiation(m, s->mra, level_ref(s, level_id)); break;
        case 3: AWCM_MANAGER_2D::ComputeLevel(level_ref(s, level_id), m, s->mra); break;
        case 4: AWCM_MANAGER_2D::RemoveResidueEuler(s->Q, m, s->mra); break;
        case 5: {
            BOUNDARY_MANAGER_SHOCK_VORTEX bm(s->Q);
            bm.BandingMask(m);
            break;
        }
        default: break;
    }
}

// bc: (Ny+6) x (Nx+6) BOUNDARY_CONDITION values; every field's manager becomes the reference's
// BOUNDARY_MANAGER_2D<VECTOR_4D<double>> over that condition field.
void ref2d_set_bc_field(void* h, const int* bc)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->bcf.Initialize(s->grid, 3);
    const int w = s->nx + 6;
    for (int j = -3; j < s->ny + 3; ++j)
        for (int i = -3; i < s->nx + 3; ++i) s->bcf(i, j) = (BOUNDARY_CONDITION)bc[(size_t)(j + 3) * w + (i + 3)];
    for (BC2D* b : {s->bc, s->bc0, s->bc1, s->bc2}) {
        delete b->generic;
        b->generic = new BOUNDARY_MANAGER_2D<VECTOR_4D<double>>(s->bcf);
    }
}

// The wind tunnel manager's own calls on the conserved field (PROBLEM_WINDTUNNEL.h:124-216):
// which 0 = SetBottomBoundaryCondition(true, false), 1 = (false, true), 2 = BandingMask(mask_id).
void ref2d_wt_call(void* h, int which, int mask_id)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    BOUNDARY_MANAGER_WT bm(s->Q);
    if (which == 0) bm.SetBottomBoundaryCondition(true, false);
    else if (which == 1) bm.SetBottomBoundaryCondition(false, true);
    else bm.BandingMask(mask_ref(s, mask_id));
}

void ref2d_apply_bc(void* h, double t)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    s->bc->apply(t);
}

// One pass of the driver loop (main_2d_euler(quad).cpp:58-334), output time t_next standing in
// for arr_printing_times[cnt].  alpha_io: if freeze_mask is set, the six LF-speed arrays
// (stage 1..3: alpha_x[Ny], alpha_y[Nx]) are read from it; otherwise, when non-null, the
// computed ones are written to it.
// out[0] = dt, out[1] = do_print, out[2..5] = |mask0..mask3| (interior), out[6] = max_velocity.
void ref2d_step(void* h, double tol, double cfl, double t, double t_next, double dt_fixed, double* alpha_io,
                double* out)
{
    Ref2D* s = static_cast<Ref2D*>(h);
    AWCM_2D& awcm = *s->awcm;
    FIELD_UNIFORM_2D<VECTOR_4D<double>>& Q = s->Q;
    EULER_EQUATION_2D euler_eqn(s->gamma);
    const GRID_UNIFORM_2D& grid = s->grid;
    const double dx = grid.dx;
    const int nth = omp_get_max_threads();
    OMP_MANAGER omp_manager(nth);

    const bool wt = s->bc_kind == BC_WIND_TUNNEL;
    if (!s->freeze_mask) {
        if (wt) prepare_euler_wt(s, tol);
        else awcm.PrepareEuler(Q, tol);
    }

    // The wind tunnel's bottom fills write interior (solid) cells of mask3, which PrepareEuler leaves
    // in non-physical states (negative pressure behind the step face): for it the first stage input
    // is filled before the CFL scan, so that the scan reads the states the stage reads.  The other
    // managers write ghost cells only, outside the scan, and keep the driver's order (scan, then
    // SetBoundaryCondition: main_2d_euler(quad).cpp:61-85).
    if (wt) {
        s->bc->apply(t);
        stage_input_wt(s, Q);
    }
    double max_velocity = 0;
#pragma omp parallel
    {
        double max_velocity = 0;
#pragma omp for
        ITERATION_GRID_2D(grid, 0)
        {
            if (awcm.mask3(i, j) == false) continue;
            max_velocity = MAX(max_velocity, euler_eqn.Spectral_RadiusX(Q(i, j)) + euler_eqn.Spectral_RadiusY(Q(i, j)));
        }
        omp_manager.Input(max_velocity);
    }
    max_velocity = omp_manager.Max_double();
    double dt = cfl * dx / max_velocity;
    if (dt_fixed > 0) dt = dt_fixed;
    int do_print = 0;
    if (t + dt > t_next) {
        dt = t_next - t;
        do_print = 1;
    }

    std::vector<double> ax(s->ny), ay(s->nx);
    // freeze_mask 2: replay the recorded LF speeds from alpha_io; 1 (or normal mode): compute them
    // and record them into alpha_io when it is given.
    const int frozen = s->freeze_mask == 2 && alpha_io;
    auto load_alpha = [&](int stage, const FIELD_UNIFORM_2D<VECTOR_4D<double>>& Qs, const FIELD_UNIFORM_2D<bool>& m) {
        double* base = alpha_io ? alpha_io + (size_t)stage * (s->nx + s->ny) : nullptr;
        if (frozen) {
            for (int j = 0; j < s->ny; ++j) ax[j] = base[j];
            for (int i = 0; i < s->nx; ++i) ay[i] = base[s->ny + i];
        } else {
            alpha2d(s, Qs, m, ax, ay);
            if (base) {
                for (int j = 0; j < s->ny; ++j) base[j] = ax[j];
                for (int i = 0; i < s->nx; ++i) base[s->ny + i] = ay[i];
            }
        }
    };

    const FIELD_UNIFORM_2D<VECTOR_4D<double>>* qx = wt ? &s->Qx : nullptr;
    if (!wt) s->bc->apply(t);
    load_alpha(0, Q, awcm.mask3);
    stage2d(s, Q, s->Q_2, awcm.mask2, awcm.level2, ax, ay, dt, 1, qx);

    s->bc2->apply(t);
    if (wt) stage_input_wt(s, s->Q_2);
    load_alpha(1, s->Q_2, awcm.mask2);
    stage2d(s, s->Q_2, s->Q_1, awcm.mask1, awcm.level1, ax, ay, dt, 2, qx);

    s->bc1->apply(t);
    if (wt) stage_input_wt(s, s->Q_1);
    load_alpha(2, s->Q_1, awcm.mask1);
    stage2d(s, s->Q_1, s->Q_0, awcm.mask0, awcm.level0, ax, ay, dt, 3, qx);

#pragma omp parallel for
    ITERATION_GRID_2D(grid, 0)
    {
        if (awcm.mask0(i, j) == true) Q(i, j) = (Q(i, j) + 2.0 * s->Q_0(i, j)) / 3.0;
    }
    // Frozen-mask mode (gradient configuration): no PrepareEuler and no residue removal, so the
    // stencil points outside mask0 keep their values; fixed dt and recorded LF speeds.
    if (!s->freeze_mask) awcm.PostProcessEuler(Q);

    // Mask sizes for the caller (the metric's active-point count).  Not part of the reference's
    // step; counted with all threads so it adds little to the timed step.
    long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    const int ny = s->ny, nx = s->nx;
#pragma omp parallel for reduction(+ : c0, c1, c2, c3)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            c0 += awcm.mask0(i, j);
            c1 += awcm.mask1(i, j);
            c2 += awcm.mask2(i, j);
            c3 += awcm.mask3(i, j);
        }
    const long cnt[4] = {c0, c1, c2, c3};
    out[0] = dt;
    out[1] = do_print;
    for (int k = 0; k < 4; ++k) out[2 + k] = (double)cnt[k];
    out[6] = max_velocity;
}

void ref2d_set_freeze(void* h, int freeze) { static_cast<Ref2D*>(h)->freeze_mask = freeze; }
void ref2d_set_wenoz_eps(void* h, double eps) { static_cast<Ref2D*>(h)->wenoz_eps = eps; }

// Steps until t >= t_end or max_steps; returns the step count, out[0] = t, out[1] = sum |mask0|.
int ref2d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out)
{
    double t = 0, upd = 0, o[8];
    int n = 0;
    while (n < max_steps) {
        ref2d_step(h, tol, cfl, t, t_end, 0.0, nullptr, o);
        t += o[0];
        upd += o[2];
        ++n;
        if (t >= t_end) break;
    }
    out[0] = t;
    out[1] = upd;
    return n;
}

int ref2d_threads(void) { return omp_get_max_threads(); }

// The reference's EULER_EQUATION_2D itself over n states of 4 doubles: ComputeFu / ComputeGu
// (dir 0 / 1) and Spectral_RadiusX / Spectral_RadiusY.
void ref_euler2d_flux(const double* q, double* f, int n, int dir, double gamma)
{
    const EULER_EQUATION_2D eq(gamma);
    for (int t = 0; t < n; ++t) {
        VECTOR_4D<double> Q(q[4 * t], q[4 * t + 1], q[4 * t + 2], q[4 * t + 3]), o;
        if (dir == 0) eq.ComputeFu(Q, o);
        else eq.ComputeGu(Q, o);
        for (int k = 0; k < 4; ++k) f[4 * t + k] = o[k];
    }
}
void ref_euler2d_sr(const double* q, double* out, int n, int dir, double gamma)
{
    const EULER_EQUATION_2D eq(gamma);
    for (int t = 0; t < n; ++t) {
        const VECTOR_4D<double> Q(q[4 * t], q[4 * t + 1], q[4 * t + 2], q[4 * t + 3]);
        out[t] = dir == 0 ? eq.Spectral_RadiusX(Q) : eq.Spectral_RadiusY(Q);
    }
}

}  // extern "C"

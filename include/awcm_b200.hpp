// awcm_b200.hpp -- C++ mirror of the reference's AWCM call surface over the C-ABI of awcm_b200.h.
//
// The reference (doseongju/C_pp-library) drives its path through header-only classes:
// AWCM_1D/AWCM_2D (Wavelet/AWCM_1D.h, Wavelet/AWCM_2D.h), the static passes of AWCM_MANAGER_1D/2D
// (Wavelet/AWCM_MANAGER_1D.h, Wavelet/AWCM_MANAGER_2D.h), EULER_EQUATION_1D/2D (EULER_EQUATION.h)
// and the BOUNDARY_MANAGER* classes of Problems/.  The classes below keep those names and method
// names so a driver written against the reference changes its includes and its field hand-over,
// not its loop: the state lives on the GPU, and the host field (the reference's FIELD_UNIFORM_*
// storage layout) is copied in and out explicitly.  Every method throws awcm_b200::Error on a
// non-zero status.  Header-only; link with -lawcm_b200.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "awcm_b200.h"

namespace awcm_b200 {

struct Error : std::runtime_error {
    int status;
    Error(const char* what, int s) : std::runtime_error(std::string(what) + ": " + awcm_last_error()), status(s) {}
};

inline void check(int rc, const char* what)
{
    if (rc != AWCM_OK) throw Error(what, rc);
}

// ------------------------------------------------------------------------------------------ 2D
// AWCM_2D (Wavelet/AWCM_2D.h:10-188) together with the field it serves and its stage copies.
class AWCM_2D {
public:
    AWCM_2D(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min, double y_max,
            int bc_kind = AWCM_BC_TRANSMISSIVE)
    {
        check(awcm2d_create(num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, bc_kind, &h_), "awcm2d_create");
        check(awcm2d_dims(h_, &nx_, &ny_), "awcm2d_dims");
    }
    ~AWCM_2D() { awcm2d_destroy(h_); }
    AWCM_2D(const AWCM_2D&) = delete;
    AWCM_2D& operator=(const AWCM_2D&) = delete;

    int Nx() const { return nx_; }
    int Ny() const { return ny_; }
    awcm2d_t handle() const { return h_; }

    // Field hand-over in the reference layout: FIELD_UNIFORM_2D<VECTOR_4D<double>> storage with a
    // ghost ring of 3, (Ny+6) x (Nx+6) x 4 doubles.
    void SetField(const double* q) { check(awcm2d_set_q(h_, q), "awcm2d_set_q"); }
    void GetField(double* q) const { check(awcm2d_get_q(h_, q), "awcm2d_get_q"); }
    std::vector<double> GetField() const
    {
        std::vector<double> q((size_t)(nx_ + 6) * (ny_ + 6) * 4);
        GetField(q.data());
        return q;
    }
    void Initialize(int problem, double a, double b) { check(awcm2d_init_problem(h_, problem, a, b), "awcm2d_init_problem"); }

    // AWCM_2D::PrepareEuler / PostProcessEuler (Wavelet/AWCM_2D.h:114-152).
    void PrepareEuler(double tol) { check(awcm2d_prepare(h_, tol), "awcm2d_prepare"); }
    void PostProcessEuler() { check(awcm2d_manager(h_, AWCM_OP_REMOVE_RESIDUE, 0, 0), "awcm2d_manager"); }

    // One pass of the driver loop (main_2d_euler(quad).cpp:58-334); returns dt, sets do_print.
    double Step(double tol, double cfl, double t, double t_next, bool* do_print = nullptr, double dt_fixed = 0)
    {
        double out[8];
        check(awcm2d_step(h_, tol, cfl, t, t_next, dt_fixed, out), "awcm2d_step");
        if (do_print) *do_print = out[1] != 0;
        last_mask_sizes_[0] = (long)out[2], last_mask_sizes_[1] = (long)out[3];
        last_mask_sizes_[2] = (long)out[4], last_mask_sizes_[3] = (long)out[5];
        return out[0];
    }
    long MaskSize(int k) const { return last_mask_sizes_[k]; }

    // The public masks mask0..mask3 / mask_temp and levels of the reference facade, read back on
    // demand (ghosted (Ny+6) x (Nx+6) bytes; levels Ny x Nx).
    std::vector<uint8_t> Mask(int mask_id) const
    {
        const size_t n = (size_t)(nx_ + 6) * (ny_ + 6);
        std::vector<uint8_t> all(5 * n);
        check(awcm2d_get_masks(h_, all.data()), "awcm2d_get_masks");
        const int plane = mask_id == 4 ? 0 : mask_id + 1;
        return std::vector<uint8_t>(all.begin() + plane * n, all.begin() + (plane + 1) * n);
    }
    // WAVELET_2D::InterpolateAllGridEuler(Q, mra, mask_from) (Wavelet/WAVELET_2D.h:912-1044): the dense
    // field, interpolated at every grid point outside mask `from_id` (0 = mask0).
    void InterpolateAllGridEuler(int from_id = 0) { check(awcm2d_interpolate_all(h_, from_id), "awcm2d_interpolate_all"); }

    // Binary state file (awcm2d_save_state / awcm2d_load_state): resume a run bit for bit.
    void SaveState(const char* path, double t, long long step) const
    {
        check(awcm2d_save_state(h_, path, t, step), "awcm2d_save_state");
    }
    void LoadState(const char* path, double* t = nullptr, long long* step = nullptr)
    {
        check(awcm2d_load_state(h_, path, t, step), "awcm2d_load_state");
    }

    // Frozen-mask run and discrete adjoint (no reference counterpart): n_steps steps at fixed dt
    // on the masks of the last PrepareEuler; Adjoint returns the loss and fills grad (the
    // SetField layout) with dLoss/dQ(t0).  SetWenoZ(1e-6, 1e-6) selects the differentiable mode.
    void SetWenoZ(double eps, double tau_delta = 0) { check(awcm2d_set_wenoz(h_, eps, tau_delta), "awcm2d_set_wenoz"); }
    double FrozenRun(double t0, double dt, int n_steps, bool replay = false)
    {
        double out[3];
        check(awcm2d_frozen_run(h_, t0, dt, n_steps, replay ? 2 : 1, out), "awcm2d_frozen_run");
        return out[0];
    }
    double Adjoint(double t0, double dt, int n_steps, const double* target, double* grad, int checkpoint_every = 0,
                   bool replay = false)
    {
        double out[5];
        check(awcm2d_adjoint(h_, t0, dt, n_steps, checkpoint_every, replay ? 2 : 1, target, grad, out),
              "awcm2d_adjoint");
        return out[0];
    }

    std::vector<int> Level(int level_id) const
    {
        const size_t n = (size_t)nx_ * ny_;
        std::vector<int> all(4 * n);
        check(awcm2d_get_levels(h_, all.data()), "awcm2d_get_levels");
        return std::vector<int>(all.begin() + level_id * n, all.begin() + (level_id + 1) * n);
    }

private:
    awcm2d_t h_ = nullptr;
    int nx_ = 0, ny_ = 0;
    long last_mask_sizes_[4] = {0, 0, 0, 0};
};

// The scalar AWCM path of Wavelet/main_2d_advect.cpp (AWCM_2D::Prepare/PostProcess on a
// FIELD_UNIFORM_2D<double>, unit-velocity advection, periodic box manager).
class AWCM_2D_SCALAR {
public:
    AWCM_2D_SCALAR(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min, double y_max)
    {
        check(awcm2d_create_scalar(num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, &h_),
              "awcm2d_create_scalar");
        check(awcm2d_dims(h_, &nx_, &ny_), "awcm2d_dims");
    }
    ~AWCM_2D_SCALAR() { awcm2d_destroy(h_); }
    AWCM_2D_SCALAR(const AWCM_2D_SCALAR&) = delete;
    AWCM_2D_SCALAR& operator=(const AWCM_2D_SCALAR&) = delete;
    int Nx() const { return nx_; }
    int Ny() const { return ny_; }
    // (Ny+6) x (Nx+6) doubles, the FIELD_UNIFORM_2D<double> storage with its ghost ring of 3.
    void SetField(const double* q) { check(awcm2d_scalar_set_q(h_, q), "awcm2d_scalar_set_q"); }
    void GetField(double* q) const { check(awcm2d_scalar_get_q(h_, q), "awcm2d_scalar_get_q"); }
    // n passes of the driver loop at the fixed dt; returns the new time.
    double Advance(double tol, double dt, double t, int n)
    {
        double out[3];
        check(awcm2d_scalar_advance(h_, tol, dt, t, n, out), "awcm2d_scalar_advance");
        return out[0];
    }

private:
    awcm2d_t h_ = nullptr;
    int nx_ = 0, ny_ = 0;
};

// AWCM_MANAGER_2D (Wavelet/AWCM_MANAGER_2D.h): static passes on one of the facade's masks.
struct AWCM_MANAGER_2D {
    static void AddAdjacentZone(AWCM_2D& a, int mask_id)
    {
        check(awcm2d_manager(a.handle(), AWCM_OP_ADD_ADJACENT_ZONE, mask_id, 0), "AddAdjacentZone");
    }
    static void CheckReconstruction(AWCM_2D& a, int mask_id)
    {
        check(awcm2d_manager(a.handle(), AWCM_OP_CHECK_RECONSTRUCTION, mask_id, 0), "CheckReconstruction");
    }
    static void AddPointForDifferentiation(AWCM_2D& a, int mask_id, int level_id)
    {
        check(awcm2d_manager(a.handle(), AWCM_OP_ADD_POINT_FOR_DIFFERENTIATION, mask_id, level_id),
              "AddPointForDifferentiation");
    }
    static void ComputeLevel(AWCM_2D& a, int level_id, int mask_id)
    {
        check(awcm2d_manager(a.handle(), AWCM_OP_COMPUTE_LEVEL, mask_id, level_id), "ComputeLevel");
    }
    static void RemoveResidueEuler(AWCM_2D& a, int mask_id)
    {
        check(awcm2d_manager(a.handle(), AWCM_OP_REMOVE_RESIDUE, mask_id, 0), "RemoveResidueEuler");
    }
};

// BOUNDARY_MANAGER_QUAD / _DMACH / _ISENVORTEX / _SHOCK_VORTEX: the instance's boundary kind is
// fixed at creation; SetBoundaryCondition fills the ghost ring of its conserved field.
struct BOUNDARY_MANAGER_OF_INSTANCE_2D {
    explicit BOUNDARY_MANAGER_OF_INSTANCE_2D(AWCM_2D& a) : a_(a) {}
    void SetBoundaryCondition(double t = 0) { check(awcm2d_apply_bc(a_.handle(), t), "SetBoundaryCondition"); }

private:
    AWCM_2D& a_;
};
using BOUNDARY_MANAGER_QUAD = BOUNDARY_MANAGER_OF_INSTANCE_2D;
using BOUNDARY_MANAGER_DMACH = BOUNDARY_MANAGER_OF_INSTANCE_2D;
using BOUNDARY_MANAGER_ISENVORTEX = BOUNDARY_MANAGER_OF_INSTANCE_2D;
using BOUNDARY_MANAGER_SHOCK_VORTEX = BOUNDARY_MANAGER_OF_INSTANCE_2D;

// BOUNDARY_CONDITION of the generic managers (BOUNDARY_MANAGER_2D.h:7-13).
enum BOUNDARY_CONDITION {
    SOLID_WALL = AWCM_SOLID_WALL,
    PERIODIC = AWCM_PERIODIC,
    EXTRAPOLATION_ZERO_ORDER = AWCM_EXTRAPOLATION_ZERO_ORDER,
    SPECIFIED = AWCM_SPECIFIED,
    FLUID = AWCM_FLUID
};

// The enum-driven BOUNDARY_MANAGER_2D<TT> (BOUNDARY_MANAGER_2D.h:23-159): built over a condition
// field ((Ny+6) x (Nx+6) values in the FIELD_UNIFORM_2D layout); SetBoundaryCondition(awcm)
// attaches it to the instance (whose later stage fills then use it too) and fills the ghost ring
// of the instance's conserved field.  TT is the reference's field element type, kept for the name.
template <class TT = void>
class BOUNDARY_MANAGER_2D {
public:
    explicit BOUNDARY_MANAGER_2D(const std::vector<int>& bc) : bc_(bc) {}
    void SetBoundaryCondition(AWCM_2D& a) const
    {
        check(awcm2d_set_bc_field(a.handle(), bc_.data()), "awcm2d_set_bc_field");
        check(awcm2d_apply_bc(a.handle(), 0.0), "SetBoundaryCondition");
    }

private:
    std::vector<int> bc_;
};

// EULER_EQUATION_2D (EULER_EQUATION.h:64-156) over batches of device-resident states (n x 4).
struct EULER_EQUATION_2D {
    double gamma;
    explicit EULER_EQUATION_2D(double g = 1.4) : gamma(g) {}
    void ComputeFu(const double* q_dev, double* f_dev, int n, void* stream = nullptr) const
    {
        check(euler2d_flux(q_dev, f_dev, n, 0, gamma, stream), "ComputeFu");
    }
    void ComputeGu(const double* q_dev, double* g_dev, int n, void* stream = nullptr) const
    {
        check(euler2d_flux(q_dev, g_dev, n, 1, gamma, stream), "ComputeGu");
    }
    void Spectral_RadiusX(const double* q_dev, double* s_dev, int n, void* stream = nullptr) const
    {
        check(euler2d_spectral_radius(q_dev, s_dev, n, 0, gamma, stream), "Spectral_RadiusX");
    }
    void Spectral_RadiusY(const double* q_dev, double* s_dev, int n, void* stream = nullptr) const
    {
        check(euler2d_spectral_radius(q_dev, s_dev, n, 1, gamma, stream), "Spectral_RadiusY");
    }
};

// ------------------------------------------------------------------------------------------ 1D
// AWCM_1D (Wavelet/AWCM_1D.h:7-189) together with the field it serves: one instance on the GPU (a
// batch of one).  The field hand-over uses the FIELD_UNIFORM_1D<VECTOR_3D<double>> storage with a
// ghost ring of 3, (Nx+6) x 3 doubles.
class AWCM_1D {
public:
    AWCM_1D(int num_levels, int nx_coarse, double x_min, double x_max, double gamma = 1.4, int scheme = 0)
    {
        check(awcm1d_batch_create(1, &num_levels, &nx_coarse, &x_min, &x_max, gamma, scheme, &h_),
              "awcm1d_batch_create");
        check(awcm1d_batch_nx(h_, 0, &nx_), "awcm1d_batch_nx");
    }
    ~AWCM_1D() { awcm1d_batch_destroy(h_); }
    AWCM_1D(const AWCM_1D&) = delete;
    AWCM_1D& operator=(const AWCM_1D&) = delete;

    int Nx() const { return nx_; }
    awcm1d_batch_t handle() const { return h_; }

    void SetField(const double* q) { check(awcm1d_batch_set_q(h_, 0, q), "awcm1d_batch_set_q"); }
    void GetField(double* q) const { check(awcm1d_batch_get_q(h_, 0, q), "awcm1d_batch_get_q"); }
    std::vector<double> GetField() const
    {
        std::vector<double> q((size_t)(nx_ + 6) * 3);
        GetField(q.data());
        return q;
    }
    // SHOCKTUBE::Initialize (Problems/1D/PROBLEM_SHOCKTUBE.h:14-54): (rho, u, p) left and right.
    void InitializeRiemann(double x_interface, const double* left3, const double* right3)
    {
        check(awcm1d_batch_init_riemann(h_, 0, x_interface, left3, right3), "awcm1d_batch_init_riemann");
    }

    // AWCM_1D::PrepareEuler / PostProcessEuler / BadingBoundary (Wavelet/AWCM_1D.h:73-125).
    void PrepareEuler(double tol) { check(awcm1d_batch_prepare(h_, 0, tol), "PrepareEuler"); }
    void PostProcessEuler() { check(awcm1d_batch_manager(h_, 0, AWCM_OP_REMOVE_RESIDUE, 0, 0), "PostProcessEuler"); }
    void BadingBoundary(int mask_id) { check(awcm1d_batch_manager(h_, 0, AWCM_OP_BANDING, mask_id, 0), "BadingBoundary"); }
    // The facade's WAVELET_1D member (Wavelet/WAVELET_1D.h:282-431) on the instance's field.
    void ForwardWaveletTransformEuler(double tol) { check(awcm1d_batch_fwt(h_, 0, tol), "ForwardWaveletTransformEuler"); }
    void InverseWaveletTransformEuler(int mask_id)
    {
        check(awcm1d_batch_iwt(h_, 0, mask_id), "InverseWaveletTransformEuler");
    }
    void InterpolateEuler(int from_id, int to_id)
    {
        check(awcm1d_batch_interpolate(h_, 0, from_id, to_id), "InterpolateEuler");
    }

    // One pass of the driver loop (Wavelet/main_1d_euler.cpp:61-260); returns dt, sets do_print.
    double Step(double tol, double cfl, double t, double t_next, bool* do_print = nullptr)
    {
        check(awcm1d_batch_set_run(h_, &tol, &cfl, &t, &t_next, 0.0), "awcm1d_batch_set_run");
        check(awcm1d_batch_steps(h_, 1), "awcm1d_batch_steps");
        double s[16];
        check(awcm1d_batch_status(h_, 0, s), "awcm1d_batch_status");
        if (do_print) *do_print = s[2] != 0;
        for (int k = 0; k < 4; ++k) last_mask_sizes_[k] = (long)s[5 + k];
        return s[1];
    }
    long MaskSize(int k) const { return last_mask_sizes_[k]; }

    // The public masks (mask_id 0..3 = mask0..mask3, 4 = mask_temp; Nx+6 bytes with ghosts) and
    // levels (Nx ints) of the reference facade, read back on demand.
    std::vector<uint8_t> Mask(int mask_id) const
    {
        const size_t n = (size_t)nx_ + 6;
        std::vector<uint8_t> all(5 * n);
        check(awcm1d_batch_get_masks(h_, 0, all.data()), "awcm1d_batch_get_masks");
        const int plane = mask_id == 4 ? 0 : mask_id + 1;
        return std::vector<uint8_t>(all.begin() + plane * n, all.begin() + (plane + 1) * n);
    }
    std::vector<int> Level(int level_id) const
    {
        const size_t n = (size_t)nx_;
        std::vector<int> all(4 * n);
        check(awcm1d_batch_get_levels(h_, 0, all.data()), "awcm1d_batch_get_levels");
        return std::vector<int>(all.begin() + level_id * n, all.begin() + (level_id + 1) * n);
    }

private:
    awcm1d_batch_t h_ = nullptr;
    int nx_ = 0;
    long last_mask_sizes_[4] = {0, 0, 0, 0};
};

// AWCM_MANAGER_1D (Wavelet/AWCM_MANAGER_1D.h:7-187): static passes on one of the facade's masks.
struct AWCM_MANAGER_1D {
    static void AddAdjacentZone(AWCM_1D& a, int mask_id)
    {
        check(awcm1d_batch_manager(a.handle(), 0, AWCM_OP_ADD_ADJACENT_ZONE, mask_id, 0), "AddAdjacentZone");
    }
    static void CheckReconstruction(AWCM_1D& a, int mask_id)
    {
        check(awcm1d_batch_manager(a.handle(), 0, AWCM_OP_CHECK_RECONSTRUCTION, mask_id, 0), "CheckReconstruction");
    }
    static void AddPointForDifferentiation(AWCM_1D& a, int mask_id, int level_id)
    {
        check(awcm1d_batch_manager(a.handle(), 0, AWCM_OP_ADD_POINT_FOR_DIFFERENTIATION, mask_id, level_id),
              "AddPointForDifferentiation");
    }
    static void ComputeLevel(AWCM_1D& a, int level_id, int mask_id)
    {
        check(awcm1d_batch_manager(a.handle(), 0, AWCM_OP_COMPUTE_LEVEL, mask_id, level_id), "ComputeLevel");
    }
    static void RemoveResidue(AWCM_1D& a, int mask_id)
    {
        check(awcm1d_batch_manager(a.handle(), 0, AWCM_OP_REMOVE_RESIDUE, mask_id, 0), "RemoveResidue");
    }
};

// BOUNDARY_MANAGER (Problems/1D/PROBLEM_SHOCKTUBE.h:57-107): transmissive ghost fill.
struct BOUNDARY_MANAGER {
    explicit BOUNDARY_MANAGER(AWCM_1D& a) : a_(a) {}
    void SetBoundaryCondition() { check(awcm1d_batch_apply_bc(a_.handle(), 0), "SetBoundaryCondition"); }

private:
    AWCM_1D& a_;
};

// The enum-driven BOUNDARY_MANAGER_1D<T> (BOUNDARY_MANAGER_1D.h:17-76) over a condition field of
// Nx+6 values; SetBoundaryCondition(awcm) attaches it to the instance and fills its ghost cells.
template <class T = void>
class BOUNDARY_MANAGER_1D {
public:
    explicit BOUNDARY_MANAGER_1D(const std::vector<int>& bc) : bc_(bc) {}
    void SetBoundaryCondition(AWCM_1D& a) const
    {
        check(awcm1d_batch_set_bc_field(a.handle(), 0, bc_.data()), "awcm1d_batch_set_bc_field");
        check(awcm1d_batch_apply_bc(a.handle(), 0), "SetBoundaryCondition");
    }

private:
    std::vector<int> bc_;
};

// EULER_EQUATION_1D (EULER_EQUATION.h:6-62) over batches of device-resident states (n x 3).
struct EULER_EQUATION_1D {
    double gamma;
    explicit EULER_EQUATION_1D(double g = 1.4) : gamma(g) {}
    void ComputeFu(const double* q_dev, double* f_dev, int n, void* stream = nullptr) const
    {
        check(euler1d_flux(q_dev, f_dev, n, gamma, stream), "ComputeFu");
    }
    void Spectral_Radius(const double* q_dev, double* s_dev, int n, void* stream = nullptr) const
    {
        check(euler1d_spectral_radius(q_dev, s_dev, n, gamma, stream), "Spectral_Radius");
    }
};

// A batch of independent AWCM_1D instances advanced together (no reference counterpart: the
// reference runs one instance per process).
// scheme AWCM_SCALAR_ADVECTION gives the scalar path of Wavelet/main_1d_advect.cpp (the field in
// component 0 of SetField/GetField, dt = SetRun's dt_fixed).
class AWCM_1D_BATCH {
public:
    AWCM_1D_BATCH(const std::vector<int>& num_levels, const std::vector<int>& nx_coarse, const std::vector<double>& x_min,
                  const std::vector<double>& x_max, double gamma = 1.4, int scheme = 0)
    {
        check(awcm1d_batch_create((int)num_levels.size(), num_levels.data(), nx_coarse.data(), x_min.data(),
                                  x_max.data(), gamma, scheme, &h_),
              "awcm1d_batch_create");
    }
    ~AWCM_1D_BATCH() { awcm1d_batch_destroy(h_); }
    AWCM_1D_BATCH(const AWCM_1D_BATCH&) = delete;
    AWCM_1D_BATCH& operator=(const AWCM_1D_BATCH&) = delete;
    awcm1d_batch_t handle() const { return h_; }

    void SetField(int k, const double* q) { check(awcm1d_batch_set_q(h_, k, q), "awcm1d_batch_set_q"); }
    void GetField(int k, double* q) const { check(awcm1d_batch_get_q(h_, k, q), "awcm1d_batch_get_q"); }
    void InitializeRiemann(int k, double x_interface, const double* left3, const double* right3)
    {
        check(awcm1d_batch_init_riemann(h_, k, x_interface, left3, right3), "awcm1d_batch_init_riemann");
    }
    void SetRun(const std::vector<double>& tol, const std::vector<double>& cfl, const std::vector<double>& t,
                const std::vector<double>& t_end, double dt_fixed = 0)
    {
        check(awcm1d_batch_set_run(h_, tol.data(), cfl.data(), t.data(), t_end.data(), dt_fixed), "set_run");
    }
    void Steps(int n) { check(awcm1d_batch_steps(h_, n), "awcm1d_batch_steps"); }
    // Every instance to its end time in one launch (at most max_steps steps each).
    void RunToEnd(int max_steps = 0x7fffffff) { check(awcm1d_batch_run(h_, max_steps), "awcm1d_batch_run"); }
    void Sync() { check(awcm1d_batch_sync(h_), "awcm1d_batch_sync"); }
    std::vector<double> Status(int k) const
    {
        std::vector<double> s(16);
        check(awcm1d_batch_status(h_, k, s.data()), "awcm1d_batch_status");
        return s;
    }

private:
    awcm1d_batch_t h_ = nullptr;
};

}  // namespace awcm_b200

// TEST INFRASTRUCTURE ONLY -- the CPU restatement of the reference's AWCM compressible-Euler
// path (doseongju/C_pp-library), used as the checker for the CUDA product and as its CPU
// "port" baseline.  It never ships inside the product library.
//
// The entry points mirror, name for name, the reference-harness ones (ref1d_*/ref2d_*) so the
// tests can run either against the same inputs.  Layouts (all host, row-major, ghosts of 3):
//   1D state  q[(i+3)*3 + p],               i in [-3, Nx+2], p in 0..2
//   2D state  q[((j+3)*(Nx+6) + i+3)*4 + p]
//   masks     5 planes (mask_temp, mask0..mask3) of one byte per ghosted point
//   levels    4 planes (level0..level3) of one int per interior point
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void* or1d_create(int num_levels, int nx_coarse, double x_min, double x_max, double gamma, int scheme);
void or1d_destroy(void* h);
int or1d_nx(void* h);
void or1d_set_q(void* h, const double* q);
void or1d_get_q(void* h, double* q);
void or1d_init_riemann(void* h, double x_interface, double rho_l, double u_l, double p_l, double rho_r,
                       double u_r, double p_r);
void or1d_get_masks(void* h, uint8_t* m);
void or1d_set_masks(void* h, const uint8_t* m);
void or1d_get_levels(void* h, int* lv);
void or1d_set_levels(void* h, const int* lv);
void or1d_prepare(void* h, double tol);
void or1d_fwt(void* h, double tol);
void or1d_iwt(void* h, int mask_id);
void or1d_manager(void* h, int op, int mask_id, int level_id);
void or1d_step(void* h, double tol, double cfl, double t, double t_next, double* out);
/* scheme 2 (scalar path of Wavelet/main_1d_advect.cpp): one driver pass at the fixed dt;
 * out[0] = dt, out[1..4] = |mask0..mask3|.  The field is component 0 of set_q/get_q. */
void or1d_scalar_step(void* h, double tol, double dt, double* out);
int or1d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out);

void* or2d_create(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                  double y_max, int bc_kind);
void or2d_destroy(void* h);
void or2d_dims(void* h, int* nx, int* ny);
void or2d_set_q(void* h, const double* q);
void or2d_get_q(void* h, double* q);
void or2d_init_problem(void* h, int kind, double a, double b);
void or2d_get_masks(void* h, uint8_t* m);
void or2d_set_masks(void* h, const uint8_t* m);
void or2d_get_levels(void* h, int* lv);
void or2d_set_levels(void* h, const int* lv);
void or2d_prepare(void* h, double tol);
void or2d_fwt(void* h, double tol);
void or2d_iwt(void* h, int mask_id);
void or2d_interpolate(void* h, int from_id, int to_id);
/* Scalar AWCM (Wavelet/main_2d_advect.cpp): mode switch, field (ny+6)x(nx+6) doubles, one driver pass;
 * out[4] = |mask0..mask3|. */
void or2d_set_scalar(void* h, int on);
void or2d_scalar_set_q(void* h, const double* q);
void or2d_scalar_get_q(void* h, double* q);
void or2d_scalar_step(void* h, double tol, double dt, double* out);
/* WAVELET_2D::InterpolateAllGridEuler (Wavelet/WAVELET_2D.h:912-1044). */
void or2d_interpolate_all(void* h, int from_id);
void or2d_manager(void* h, int op, int mask_id, int level_id);
void or2d_apply_bc(void* h, double t);
void or2d_step(void* h, double tol, double cfl, double t, double t_next, double dt_fixed, double* alpha_io,
               double* out);
void or2d_set_freeze(void* h, int freeze);
/* WENO-Z epsilon of the face reconstructions (the reference solver's WENOZ5::eps, default 1e-40)
 * and the smoothing of tau = |b0 - b2| (0: none, as in the reference). */
void or2d_set_wenoz(void* h, double eps, double tau_delta);
int or2d_run(void* h, double tol, double cfl, double t_end, int max_steps, double* out);
int or2d_threads(void);

#ifdef __cplusplus
}
#endif

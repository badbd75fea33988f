/*
 * awcm_b200.h -- C-ABI of the B200-native AWCM compressible-Euler path.
 *
 * This is the drop-in boundary for the adaptive wavelet collocation (AWCM) Euler hot path of
 * doseongju/C_pp-library.  The reference exposes that path as header-only C++ classes with no ABI:
 * AWCM_1D/AWCM_2D (Wavelet/AWCM_1D.h, Wavelet/AWCM_2D.h), the static passes of AWCM_MANAGER_1D/2D
 * (Wavelet/AWCM_MANAGER_1D.h, Wavelet/AWCM_MANAGER_2D.h), EULER_EQUATION_1D/2D (EULER_EQUATION.h)
 * and the BOUNDARY_MANAGER* classes of Problems/, driven by an RK3 loop written inline in main()
 * (Wavelet/main_1d_euler.cpp:61-260, Wavelet/main_2d_euler(quad).cpp:56-350).  Each entry point
 * below names the reference interface it replaces.  The C++ mirror classes that keep the
 * reference's names are in awcm_b200.hpp.
 *
 * Conventions
 *   - Every function returns an int status: 0 ok, AWCM_ERR_* otherwise; awcm_last_error() gives text.
 *   - State lives on the GPU (one device, the current one at create time).  Host arrays use the
 *     reference's own memory layout so a caller can hand over its FIELD_UNIFORM_* storage:
 *       1D conserved state : (Nx+6) x 3 doubles, point i (ghosts -3..Nx+2) at [(i+3)*3 + p]
 *       2D conserved state : (Ny+6) x (Nx+6) x 4 doubles, point (i,j) at [((j+3)*(Nx+6) + i+3)*4 + p]
 *       masks              : 5 planes of one byte per ghosted point: mask_temp, mask0..mask3
 *       levels             : 4 planes of one int per interior point: level0..level3
 *   - Mask ids: 0..3 = mask0..mask3, 4 = mask_temp.  Level ids 0..3.
 *   - Arithmetic is IEEE double with the reference's operation order; results are bit-identical
 *     to the reference's CPU code for identical inputs.
 */
#ifndef AWCM_B200_H
#define AWCM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AWCM_OK 0
#define AWCM_ERR_ARG 1
#define AWCM_ERR_OOM 2
#define AWCM_ERR_CUDA 3
#define AWCM_ERR_TIMEOUT 4
#define AWCM_ERR_NONFINITE 5
#define AWCM_ERR_STATE 6

/* Manager pass op codes (AWCM_MANAGER_1D/2D static methods). */
#define AWCM_OP_ADD_ADJACENT_ZONE 0            /* AddAdjacentZone(mask)                  */
#define AWCM_OP_CHECK_RECONSTRUCTION 1         /* CheckReconstruction(mask)              */
#define AWCM_OP_ADD_POINT_FOR_DIFFERENTIATION 2 /* AddPointForDifferentiation(mask, level) */
#define AWCM_OP_COMPUTE_LEVEL 3                /* ComputeLevel(level, mask)              */
#define AWCM_OP_REMOVE_RESIDUE 4               /* RemoveResidue(Euler)(q, mask)          */
#define AWCM_OP_BANDING 5                      /* BadingBoundary / BandingMask(mask)     */

/* Boundary kinds (BOUNDARY_MANAGER classes of Problems/). */
#define AWCM_BC_TRANSMISSIVE 0 /* BOUNDARY_MANAGER (1D), BOUNDARY_MANAGER_QUAD (2D)   */
#define AWCM_BC_DOUBLE_MACH 1  /* BOUNDARY_MANAGER_DMACH::SetBoundaryCondition(t)      */
#define AWCM_BC_PERIODIC 2     /* BOUNDARY_MANAGER_ISENVORTEX                          */
#define AWCM_BC_SHOCK_VORTEX 3 /* BOUNDARY_MANAGER_SHOCK_VORTEX: transmissive left/right,
                                  reflecting bottom/top (PROBLEM_SHOCK_VORTEX_INTERACTION.h:78-201) */
#define AWCM_BC_GENERIC 4      /* the enum-driven BOUNDARY_MANAGER_1D<T> / BOUNDARY_MANAGER_2D<TT>
                                  (BOUNDARY_MANAGER_1D.h:17-76, BOUNDARY_MANAGER_2D.h:23-159), attached
                                  with awcm1d_batch_set_bc_field / awcm2d_set_bc_field */
#define AWCM_BC_WIND_TUNNEL 5  /* BOUNDARY_MANAGER_WT (Problems/2D/PROBLEM_WINDTUNNEL.h:52-222): Mach 3
                                  inflow left, extrapolation right, reflecting top, and the
                                  forward-facing step at (int(0.6/dx), int(0.2/dy)) filled per sweep
                                  direction; its BandingMask replaces the edge banding */

/* BOUNDARY_CONDITION values of the generic managers (BOUNDARY_MANAGER_2D.h:7-13). */
#define AWCM_SOLID_WALL (-4)
#define AWCM_PERIODIC (-3)
#define AWCM_EXTRAPOLATION_ZERO_ORDER (-2)
#define AWCM_SPECIFIED (-1)
#define AWCM_FLUID 0

/* 2D problem initial states (Problems/2D/*::Initialize). */
#define AWCM_PROBLEM_QUADRANTS 0   /* a, b = split point                      */
#define AWCM_PROBLEM_DOUBLE_MACH 1 /* a = pre-shock density                   */
#define AWCM_PROBLEM_VORTEX 2      /* a, b = vortex centre                    */
#define AWCM_PROBLEM_SHOCK_VORTEX 3 /* SHOCK_VORTEX: Mach 1.2 shock at x = 0, vortex at (a, b) */
#define AWCM_PROBLEM_WIND_TUNNEL 4  /* WINDTUNNEL: uniform Mach 3 flow (rho 1.4, u 3, v 0, p 1) */

/* Last error message of the calling thread ("" if none). */
const char* awcm_last_error(void);
/* Library version string. */
const char* awcm_version(void);
/* Dense FP64 FMA throughput of the current device in TFLOP/s (2 flops per DFMA), best of
 * `repeats` launches of `iters` FMA rounds: the denominator of the FP64 roofline. */
int awcm_measure_fp64_peak(int iters, int repeats, double* tflops);

/* ------------------------------------------------------------------------------------------- 2D
 * One 2D AWCM Euler instance: the MRA_GRID_INT_2D dyadic node grid
 * (Wavelet/MRA_GRID_UNIFORM_2D.h:87-134, Nx = (nx_coarse-1)*2^(num_levels-1)+1), the AWCM_2D
 * masks/levels (Wavelet/AWCM_2D.h:24-48) and the conserved field with its three RK stage copies. */
typedef struct awcm2d_s* awcm2d_t;

/* AWCM_2D::AWCM_2D + FIELD_UNIFORM_2D::Initialize(grid, 3) + the boundary manager of bc_kind. */
int awcm2d_create(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                  double y_max, int bc_kind, awcm2d_t* out);
int awcm2d_destroy(awcm2d_t h);
int awcm2d_dims(awcm2d_t h, int* nx, int* ny);
/* The creation arguments of the instance (and its gas constant). */
typedef struct awcm2d_geometry {
    int num_levels, nx_coarse, ny_coarse, bc_kind;
    double x_min, x_max, y_min, y_max, gamma;
} awcm2d_geometry;
int awcm2d_get_geometry(awcm2d_t h, awcm2d_geometry* out);
/* Conserved state in the reference layout (host memory), ghosts included. */
int awcm2d_set_q(awcm2d_t h, const double* q);
int awcm2d_get_q(awcm2d_t h, double* q);
int awcm2d_get_masks(awcm2d_t h, uint8_t* masks);
int awcm2d_set_masks(awcm2d_t h, const uint8_t* masks);
int awcm2d_get_levels(awcm2d_t h, int* levels);
int awcm2d_set_levels(awcm2d_t h, const int* levels);
/* QUADRANTS / DOUBLEMACH / ISENTROPIC_VORTEX_ADVECTION::Initialize (Problems/2D/). */
int awcm2d_init_problem(awcm2d_t h, int kind, double a, double b);

/* AWCM_2D::PrepareEuler(Q, tol) (Wavelet/AWCM_2D.h:114-147). */
int awcm2d_prepare(awcm2d_t h, double tol);
/* WAVELET_2D::ForwardWaveletTransformationEuler(Q, mra, mask0, tol) (Wavelet/WAVELET_2D.h:478-624). */
int awcm2d_fwt(awcm2d_t h, double tol);
/* WAVELET_2D::InverseWaveletTransformationEuler(Q, mra, mask) (Wavelet/WAVELET_2D.h:626-782). */
int awcm2d_iwt(awcm2d_t h, int mask_id);
/* WAVELET_2D::InterpolateEuler(Q, mra, mask_from, mask_to) (Wavelet/WAVELET_2D.h:784-907). */
int awcm2d_interpolate(awcm2d_t h, int from_id, int to_id);
/* WAVELET_2D::InterpolateAllGridEuler(Q, mra, mask_from) (Wavelet/WAVELET_2D.h:912-1044): every grid
 * point outside mask `from_id` gets all four components interpolated from the active points,
 * coarse to fine (the dense field behind Q.Print, main_2d_euler.cpp:334). */
int awcm2d_interpolate_all(awcm2d_t h, int from_id);
/* AWCM_MANAGER_2D passes (Wavelet/AWCM_MANAGER_2D.h:14-280) and the banding of AWCM_2D.h:122-124. */
int awcm2d_manager(awcm2d_t h, int op, int mask_id, int level_id);
/* BOUNDARY_MANAGER_{QUAD,DMACH,ISENVORTEX}::SetBoundaryCondition([t]) on the conserved field. */
int awcm2d_apply_bc(awcm2d_t h, double t);
/* Attaches the enum-driven BOUNDARY_MANAGER_2D<VECTOR_4D<double>> (BOUNDARY_MANAGER_2D.h:23-159) as
 * the instance's boundary manager (kind AWCM_BC_GENERIC from then on): bc is its
 * FIELD_UNIFORM_2D<BOUNDARY_CONDITION>, one AWCM_* condition per ghosted point ((Ny+6) x (Nx+6) ints,
 * only the ghost ring is read).  Every ghost fill (awcm2d_apply_bc and the stage fills of the step)
 * then does SetBoundaryCondition(field): zero-order extrapolation and periodic cells on the four
 * strips, extrapolated corner blocks; SOLID_WALL, SPECIFIED and FLUID cells are left as they are,
 * as in the reference, which marks the class "not used now" (:20).  The adjoint refuses such an
 * instance; state files do not carry the condition field. */
int awcm2d_set_bc_field(awcm2d_t h, const int* bc);
/* BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition(x_direction, y_direction)
 * (Problems/2D/PROBLEM_WINDTUNNEL.h:124-168) on the conserved field of a wind-tunnel instance
 * (exactly one direction).  x: the columns i_bdry .. i_bdry+2 of rows -3 .. j_bdry mirror column
 * i_bdry-1 with rho u reflected (the step's front face); y: the bottom ghost rows mirror row 0 and
 * the rows j_bdry-2 .. j_bdry right of i_bdry mirror row j_bdry+1, rho v reflected (the floor and
 * the step's top).  The reference has no AWCM driver for the wind tunnel (its AWCM_2D::PrepareEuler
 * leaves the manager commented out, Wavelet/AWCM_2D.h:121); the step of a wind-tunnel instance
 * applies, per stage, SetBoundaryCondition, then the x-direction fill to a copy that the x fluxes
 * read, then the x- and y-direction fills to the stage input that the y fluxes, the LF speeds and
 * the updates read; PrepareEuler bands with the manager's BandingMask.  The frozen-mask run and
 * the adjoint refuse a wind-tunnel instance. */
int awcm2d_wt_set_bottom(awcm2d_t h, int x_direction, int y_direction);

/* One pass of the reference driver loop (Wavelet/main_2d_euler(quad).cpp:58-334): PrepareEuler,
 * CFL dt (clipped to t_next), three SSP-RK3 stages with WENO-Z/Roe fluxes on the finest level and
 * 4th-order central differences on coarser levels, PostProcessEuler.  dt_fixed > 0 replaces the
 * CFL step.  out[8]: dt, do_print, |mask0..mask3|, max wave speed, (unused).  Synchronous.
 * A wave speed |u|+c or |v|+c that is NaN or infinite at a point of the CFL scan (mask3) or of a
 * stage's Lax-Friedrichs scan (NaN/Inf in the state, negative pressure or density) ends the step
 * with AWCM_ERR_NONFINITE (the reference has no such check and carries the NaN on); the next call
 * starts clean, so a caller can restore a state and continue.  awcm2d_advance stops at that step. */
int awcm2d_step(awcm2d_t h, double tol, double cfl, double t, double t_next, double dt_fixed, double* out);
/* Advances n_steps steps from the device-held time without host round trips (one CUDA graph per
 * step), stopping early once t >= t_end.  out[4]: final t, steps taken, sum |mask0| over the steps,
 * sum of stage points (|mask2|+|mask1|+|mask0|). */
int awcm2d_advance(awcm2d_t h, double tol, double cfl, double t_start, double t_end, int n_steps, double* out);
/* One step with the step's kernels launched eagerly and CUDA events at the phase boundaries.
 * out[19]: ms of prepare, CFL+LF speeds+dt+worklists, face kernels (stages 1..3), point-update
 * kernels (stages 1..3), boundary fills + LF speeds of stages 2-3, residue removal, total; faces
 * per stage (3), stage points (3), |mask0|, dt. */
int awcm2d_profile_step(awcm2d_t h, double tol, double cfl, double t, double t_end, double* out);
/* One step with a CUDA event after every kernel: names (32 bytes each) and device ms of up to
 * cap launches in launch order; *n = launches recorded.  Instrumentation only. */
int awcm2d_profile_kernels(awcm2d_t h, double tol, double cfl, double t, double t_end, int cap, char* names,
                           double* ms, int* n);
/* Host<->device bytes one awcm2d_step call moves (step scalars in, results out; instrumentation). */
int awcm2d_step_io_bytes(awcm2d_t h, long long* h2d, long long* d2h);
/* Kernel launches enqueued by one step (for instrumentation). */
int awcm2d_launches_per_step(awcm2d_t h, int* n);
/* PrepareEuler execution: 1 = one kernel launch per pass (default), 0 = one persistent
 * cooperative kernel with bounded-spin grid barriers.  Both give identical results. */
int awcm2d_set_prepare_mode(awcm2d_t h, int mode);
/* Test and fault-injection hook (no counterpart in the reference): the number of polls after which
 * a grid-barrier wait of the persistent PrepareEuler kernel (mode 0) gives up.  An expired wait
 * makes every CTA leave at its next barrier and the step return AWCM_ERR_TIMEOUT with the device
 * usable; the next step starts clean.  0 restores the default (2^22 polls, well over a second). */
int awcm2d_set_spin_limit(awcm2d_t h, unsigned polls);
/* CUDA stream the instance runs on (cudaStream_t), for event timing by the caller. */
int awcm2d_stream(awcm2d_t h, void** stream);

/* Binary state file (no counterpart in the reference, whose only output is the write-only text
 * dump of AWCM_MANAGER_2D::Print, Wavelet/AWCM_MANAGER_2D.h:243-255): a 128-byte header (magic
 * "AWCMST2D", version 1, the geometry, t, step, |mask0|, payload size, CRC-32 of the payload),
 * then the five mask planes bit-packed, the four level planes as bytes and the conserved state
 * of the mask0 points (between steps every other point holds zero).  Loading checks magic,
 * version, geometry, sizes and CRC (AWCM_ERR_STATE otherwise) and replaces state, masks and
 * levels; t and step are returned as stored.  The CPU checker reads and writes the same format. */
int awcm2d_save_state(awcm2d_t h, const char* path, double t, long long step);
int awcm2d_load_state(awcm2d_t h, const char* path, double* t, long long* step);

/* ------------------------------------------------------------------- 2D scalar AWCM (advection)
 * The scalar path of Wavelet/main_2d_advect.cpp:33-205: one scalar field on the same dyadic grid,
 * AWCM_2D::Prepare(FIELD_UNIFORM_2D<double>&, tol) (Wavelet/AWCM_2D.h:52-79: the Euler adaptation
 * without the interpolation of new points), linear advection with unit velocity in x and y,
 * WENO5::ReconstructRight upwind faces (WENO.h:101-104) on the finest level and
 * AWCM_2D::Differentiate* (Wavelet/AWCM_2D.h:95-109) below, SSP-RK3 at a fixed dt with the final
 * combination 1/3 q + 2/3 q0, AWCM_2D::PostProcess, and the periodic BOUNDARY_MANAGER of
 * Problems/2D/PROBLEM_BOX_ADVECTION.h.  Masks, levels and the manager passes of the 2D instance
 * apply; the Euler entry points (state, steps, adjoint) return AWCM_ERR_STATE on it. */
int awcm2d_create_scalar(int num_levels, int nx_coarse, int ny_coarse, double x_min, double x_max, double y_min,
                         double y_max, awcm2d_t* out);
/* The field in the FIELD_UNIFORM_2D<double> layout: (Ny+6) x (Nx+6) doubles, ghosts included. */
int awcm2d_scalar_set_q(awcm2d_t h, const double* q);
int awcm2d_scalar_get_q(awcm2d_t h, double* q);
/* n_steps passes of the driver loop from t at the fixed dt (one CUDA graph per step).
 * out[3]: final t, steps, sum |mask0| over the steps. */
int awcm2d_scalar_advance(awcm2d_t h, double tol, double dt, double t, int n_steps, double* out);

/* ---------------------------------------------------------------- 2D frozen-mask run and adjoint
 * No counterpart in the reference (it has no derivative code).  The frozen-mask step is the
 * driver loop of Wavelet/main_2d_euler(quad).cpp:58-334 with PrepareEuler and PostProcessEuler
 * left out: the masks and levels of the last awcm2d_prepare stay fixed, dt is fixed, and the
 * per-stage Lax-Friedrichs speeds (alpha_x per row, alpha_y per column; :86-104, :170-185,
 * :250-265) are either computed and recorded on the instance's LF-speed tape (mode 1) or replayed
 * from it (mode 2).  Tape layout per step: stage 1..3 x (alpha_x[Ny], alpha_y[Nx]) doubles, the
 * layout of the CPU checkers' frozen mode.
 *
 * awcm2d_frozen_run: n_steps frozen steps from t0.  out[3]: final t, device ms, sum |mask0|. */
int awcm2d_frozen_run(awcm2d_t h, double t0, double dt, int n_steps, int mode, double* out);
/* Loss L = 1/2 sum over the points of mask0 (the active points; the others hold no solution
 * value) of (rho(t0 + n dt) - target)^2 after n frozen steps from the current state, and the discrete adjoint dL/dQ(t0) with the LF speeds held at
 * their recorded values (the exact gradient of the mode-2 map).  target: Ny x Nx doubles (row j,
 * column i), host.  grad: host, the awcm2d_get_q layout ((Ny+6) x (Nx+6) x 4, zero on the ghost
 * ring), or NULL.  checkpoint_every: the reverse sweep restores Q from checkpoints taken every
 * that many steps and recomputes each segment's stage inputs (<= 0: ceil(sqrt(n)); >= n: all
 * stage inputs kept from the forward run, nothing recomputed).  mode 1 records the LF speeds in
 * the forward run, 2 replays the tape.  The state is left at t0 + n dt.
 * out[5]: loss, forward ms, reverse ms (recomputation included), checkpoint interval, device
 * bytes held by checkpoints, stage inputs, adjoint fields and the tape. */
int awcm2d_adjoint(awcm2d_t h, double t0, double dt, int n_steps, int checkpoint_every, int mode,
                   const double* target, double* grad, double* out);
/* WENO-Z parameters of the 2D face reconstructions (forward and adjoint): eps is the public
 * member WENOZ5::eps (WENOZ.h:13-18), 1e-40 by default as in the reference; tau_delta > 0
 * replaces tau = |b0 - b2| (WENOZ.h:84) by sqrt((b0 - b2)^2 + tau_delta^2), 0 by default (no
 * counterpart in the reference).  With the reference's values the Z weights tau/(b + eps) jump
 * between regimes wherever the smoothness indicators b are near zero (uniform far fields,
 * exponential tails) and |.| has a kink at b0 = b2, so the map is not differentiable at the scale
 * of a finite-difference check; the gradient checks run the differentiable mode
 * eps = tau_delta = 1e-6. */
int awcm2d_set_wenoz(awcm2d_t h, double eps, double tau_delta);
/* Copy the first n_steps steps of the LF-speed tape out of / into the instance. */
int awcm2d_get_alpha_tape(awcm2d_t h, int n_steps, double* tape);
int awcm2d_set_alpha_tape(awcm2d_t h, int n_steps, const double* tape);

/* ------------------------------------------------------------------------------------------- 1D
 * A batch of independent 1D AWCM Euler instances (AWCM_1D, Wavelet/AWCM_1D.h, on
 * MRA_GRID_INT_1D, Wavelet/MRA_GRID_UNIFORM_1D.h:70-98), each with its own finest level, CFL step
 * and end time.  One RK3 step of all instances is ONE persistent kernel launch (one CTA advances
 * one instance through PrepareEuler, the three stages and PostProcessEuler); a batch of one is the
 * plain single-instance form of Wavelet/main_1d_euler.cpp:61-260.  Instances are indexed 0..count-1.
 * scheme 0 = WENO-Z face fluxes (WENOZ_EULER_SOLVER_1D::ComputeFlux, WENOZ.h:160-205),
 * scheme 1 = the shipped driver's WENO5 ComputedF (WENO.h:176-184),
 * scheme 2 = the scalar AWCM path of Wavelet/main_1d_advect.cpp:48-224 (AWCM_SCALAR_ADVECTION):
 *   one field advected with unit speed, AWCM_1D::Prepare (Wavelet/AWCM_1D.h:45-72, no adjacent
 *   zones on mask1..3, no interpolation), WENO5::ReconstructRight faces (WENO.h:101-104) on the
 *   finest level and AWCM_1D::Differentiate* (AWCM_1D.h:127-140) below it, the driver's stage
 *   combinations and ghost copies, AWCM_1D::PostProcess.  The field is component 0 of set_q /
 *   get_q (components 1 and 2 are unused); every step uses dt = dt_fixed of set_run (the driver's
 *   0.5 dx is the caller's choice) with no CFL and no clipping to t_end, and an instance stops once
 *   t >= t_end.  The driver's 6-argument DifferentiateAtLeftBoundary calls (:74, :82), which name
 *   no scalar overload (the driver does not compile as shipped), take the 5-point form of
 *   DifferentiateEulerAtLeftBoundary (AWCM_1D.h:174-185) on the field. */
#define AWCM_SCALAR_ADVECTION 2
typedef struct awcm1d_batch_s* awcm1d_batch_t;

/* x_min/x_max: first and last node of each instance's cell-centred grid (GRID_UNIFORM_1D). */
int awcm1d_batch_create(int count, const int* num_levels, const int* nx_coarse, const double* x_min,
                        const double* x_max, double gamma, int scheme, awcm1d_batch_t* out);
int awcm1d_batch_destroy(awcm1d_batch_t h);
int awcm1d_batch_count(awcm1d_batch_t h, int* n);
int awcm1d_batch_nx(awcm1d_batch_t h, int k, int* nx);
int awcm1d_batch_set_q(awcm1d_batch_t h, int k, const double* q);
int awcm1d_batch_get_q(awcm1d_batch_t h, int k, double* q);
int awcm1d_batch_get_masks(awcm1d_batch_t h, int k, uint8_t* masks);
int awcm1d_batch_set_masks(awcm1d_batch_t h, int k, const uint8_t* masks);
int awcm1d_batch_get_levels(awcm1d_batch_t h, int k, int* levels);
int awcm1d_batch_set_levels(awcm1d_batch_t h, int k, const int* levels);
/* SHOCKTUBE::Initialize (Problems/1D/PROBLEM_SHOCKTUBE.h:14-54) with interface and (rho,u,p) states. */
int awcm1d_batch_init_riemann(awcm1d_batch_t h, int k, double x_interface, const double* left3,
                              const double* right3);
/* Per-instance tolerance, CFL number, current time and end (output) time; dt_fixed > 0 overrides CFL. */
int awcm1d_batch_set_run(awcm1d_batch_t h, const double* tol, const double* cfl, const double* t,
                         const double* t_end, double dt_fixed);
/* Enqueues n_steps RK3 steps of every unfinished instance (one CUDA graph replay per step). */
int awcm1d_batch_steps(awcm1d_batch_t h, int n_steps);
/* Enqueues the run of every unfinished instance to its end time (set_run), at most max_steps >= 1
 * steps each, as one launch: each CTA takes instances from the largest-first queue and runs each
 * one's steps back to back before the next, so the instances do not wait for one another at every
 * step.  The launch lasts as long as the longest instance's run: max_steps bounds it.  No
 * counterpart in the reference (its driver loop is one instance). */
int awcm1d_batch_run(awcm1d_batch_t h, int max_steps);
int awcm1d_batch_sync(awcm1d_batch_t h);
/* out[16]: t, dt, do_print, done, steps, |mask0..mask3|, max speed, alpha of stages 1..3,
 * sum over steps of |mask0|, error code, 0.  An instance whose CFL or Lax-Friedrichs scan met a
 * NaN or infinite wave speed (NaN/Inf state, negative pressure or density) stops stepping, and its
 * status call fills `out` (out[14] = AWCM_ERR_NONFINITE) and returns AWCM_ERR_NONFINITE; set_run
 * clears the flag.  The reference has no such check. */
int awcm1d_batch_status(awcm1d_batch_t h, int k, double* out);
/* out[3]: sum over instances and steps of |mask0|, total steps, finished instances. */
int awcm1d_batch_totals(awcm1d_batch_t h, double* out);
/* AWCM_MANAGER_1D pass (AWCM_OP_*) on instance k; also 10 = PrepareEuler (AWCM_1D.h:86-120),
 * 11 = ForwardWaveletTransformEuler (WAVELET_1D.h:282-335), 12 = InverseWaveletTransformEuler(mask). */
int awcm1d_batch_pass(awcm1d_batch_t h, int k, int op, int mask_id, int level_id);
/* Typed single passes on instance k (the AWCM_1D facade of Wavelet/AWCM_1D.h and the static passes
 * it calls); mask ids 0..3 = mask0..mask3, 4 = mask_temp; synchronous.
 *   AWCM_1D::PrepareEuler(Q, tol)                       Wavelet/AWCM_1D.h:86-120
 *   WAVELET_1D::ForwardWaveletTransformEuler(Q, mra, mask0, tol)   Wavelet/WAVELET_1D.h:282-335
 *   WAVELET_1D::InverseWaveletTransformEuler(Q, mra, mask)         Wavelet/WAVELET_1D.h:337-391
 *   WAVELET_1D::InterpolateEuler(Q, mra, mask_from, mask_to)       Wavelet/WAVELET_1D.h:393-431
 *   AWCM_MANAGER_1D::<op>(mask[, level]) for op = AWCM_OP_*        Wavelet/AWCM_MANAGER_1D.h:14-157,
 *     AWCM_OP_BANDING = AWCM_1D::BadingBoundary                    Wavelet/AWCM_1D.h:73-80
 *   BOUNDARY_MANAGER::SetBoundaryCondition() (transmissive)        Problems/1D/PROBLEM_SHOCKTUBE.h:86-107 */
int awcm1d_batch_prepare(awcm1d_batch_t h, int k, double tol);
int awcm1d_batch_fwt(awcm1d_batch_t h, int k, double tol);
int awcm1d_batch_iwt(awcm1d_batch_t h, int k, int mask_id);
int awcm1d_batch_interpolate(awcm1d_batch_t h, int k, int from_id, int to_id);
int awcm1d_batch_manager(awcm1d_batch_t h, int k, int op, int mask_id, int level_id);
int awcm1d_batch_apply_bc(awcm1d_batch_t h, int k);
/* Attaches the enum-driven BOUNDARY_MANAGER_1D<VECTOR_3D<double>> (BOUNDARY_MANAGER_1D.h:17-76) to
 * instance k in place of the transmissive BOUNDARY_MANAGER: bc is its FIELD_UNIFORM_1D<BOUNDARY_CONDITION>
 * (Nx+6 AWCM_* conditions; the six ghost cells are read).  Every later ghost fill of the instance
 * (awcm1d_batch_apply_bc and the stage fills of the step) applies SetBoundaryCondition(field):
 * zero-order extrapolation or the periodic image per ghost cell, other conditions untouched. */
int awcm1d_batch_set_bc_field(awcm1d_batch_t h, int k, const int* bc);
/* Launch shape of the step kernel: threads per CTA (a multiple of 32, 64..768; the default is 512
 * when no instance has more than 1100 points, else 768) and CTAs per SM (0 = occupancy limit).
 * More threads than the kernel's launch bound is AWCM_ERR_ARG.  Results do not depend on it. */
int awcm1d_batch_set_launch(awcm1d_batch_t h, int threads, int ctas_per_sm);
int awcm1d_batch_stream(awcm1d_batch_t h, void** stream);

/* Allocation-free RK3 step of ONE 1D instance.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: a host framework whose GPU memory belongs to
 * its own caching allocator (a cudaMalloc/cudaFree behind its back fragments that pool, and both
 * calls can synchronize the device and stall its pipeline), or an embedded or real-time loop that
 * gets a fixed memory budget at start-up and may not allocate afterwards.  Such a caller passes its
 * own device buffers for the instance's state and results; everything else the step needs comes
 * from a static scratch array inside this library, so the call performs no cudaMalloc, cudaFree or
 * other allocation.
 *
 *   q_dev     (in/out) conserved field, 3 component planes of Nx+6 doubles (ghost ring of 3):
 *             q_dev[p*(Nx+6) + i+3];
 *   state_dev (in/out) Nx+6 mask bytes (bits 0..3 = mask0..mask3, bit 4 = previous mask0;
 *             before the first step: 0x01 inside, 0xe1 on the ghost ring) followed by 4 planes of
 *             Nx+6 int8 levels (level0..level3; start at 0);
 *   out_dev   (out) 16 doubles in the layout of awcm1d_batch_status, for this call only: out[4]
 *             (steps) is 1 after a step and 0 when t >= t_end already, out[13] is this step's
 *             |mask0| (not a running sum), out[14] is AWCM_ERR_NONFINITE when a wave speed of the
 *             step was NaN or infinite, else 0.
 * Nx = (nx_coarse-1)*2^(num_levels-1)+1 must not exceed 8193; larger instances are rejected with
 * AWCM_ERR_ARG.  The work is enqueued on `stream` (0 = default stream) and the call returns
 * without waiting.  The first call on a device resolves the scratch array's device address (a
 * cudaGetSymbolAddress, no allocation); make that first call before any stream capture.  All
 * calls on a device share the one scratch array, which keeps the last call's contents: calls that
 * overlap on the GPU (other streams, other host threads) race, so serialize them. */
int awcm1d_step_noalloc(int num_levels, int nx_coarse, double x_min, double x_max, double gamma, int scheme,
                        double tol, double cfl, double t, double t_end, double* q_dev, uint8_t* state_dev,
                        double* out_dev, void* stream);

/* EULER_EQUATION_1D on a batch of n conserved states in device memory (n x 3 doubles):
 * ComputeFu (EULER_EQUATION.h:16-26) and Spectral_Radius |u| + c (:42-47). */
int euler1d_flux(const double* q_dev, double* f_dev, int n, double gamma, void* stream);
int euler1d_spectral_radius(const double* q_dev, double* s_dev, int n, double gamma, void* stream);
/* EULER_EQUATION_2D on a batch of n conserved states in device memory (n x 4 doubles):
 * ComputeFu/ComputeGu (EULER_EQUATION.h:74-99) and Spectral_RadiusX/Y (:118-142). */
int euler2d_flux(const double* q_dev, double* f_dev, int n, int dir, double gamma, void* stream);
int euler2d_spectral_radius(const double* q_dev, double* s_dev, int n, int dir, double gamma, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AWCM_B200_H */

/*
 * gdb200.h -- C ABI of libgdb200.so, the B200 (sm_100a) implementation of
 * GeoDynamo.jl's per-step hot path: spherical-harmonic transforms, grid-space
 * nonlinear terms and the CNAB2 banded radial solves.
 *
 * Conventions shared by every entry point:
 *   - Every function returns an int status (GD_OK = 0).  Nothing aborts or
 *     traps; gd_last_error() returns a message for the last failure on a handle.
 *   - Host arrays are borrowed for the duration of the call only.
 *   - Host spectral arrays use the reference layout: two planes (Re, Im), each
 *     nr x nlm doubles, the (l, m) index fastest in l-major order
 *     "for l in 0:lmax, m in 0:min(l,mmax)"  (src/fields.jl:6-15,
 *     src/shtnskit_transforms.jl:177-188).
 *   - Host physical arrays use the reference layout nr x nlon x nlat doubles,
 *     theta fastest (src/fields.jl:18-24).
 *   - Device ("_dev") entry points take device pointers in the native layout
 *     documented at each declaration and run asynchronously on the handle's
 *     stream.
 *   - One host thread per handle; one CUDA stream per handle.
 */
#ifndef GDB200_H
#define GDB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
  GD_OK = 0,
  GD_ERR_ARG = 1,         /* null pointer, bad id or bad size               */
  GD_ERR_CONFIG = 2,      /* unsupported grid / parameter combination       */
  GD_ERR_CUDA = 3,        /* a CUDA runtime call failed                     */
  GD_ERR_NONFINITE = 4,   /* a NaN/Inf was detected in the state            */
  GD_ERR_SINGULAR = 5,    /* zero pivot in a banded LU factorisation        */
  GD_ERR_UNSUPPORTED = 6, /* feature not available on this device           */
  GD_ERR_STATE = 7        /* call order violated                            */
};

/* Field ids (state, nonlinear terms).  GD_COMP exists when the configuration
 * has composition. */
enum { GD_U_TOR = 0, GD_U_POL = 1, GD_B_TOR = 2, GD_B_POL = 3, GD_TEMP = 4, GD_COMP = 5 };

/* Physical grids kept by the model (velocity.jl, magnetic.jl, thermal.jl). */
enum {
  GD_GRID_U_TH = 0, GD_GRID_U_PH = 1, GD_GRID_W_TH = 2, GD_GRID_W_PH = 3,
  GD_GRID_B_TH = 4, GD_GRID_B_PH = 5, GD_GRID_J_TH = 6, GD_GRID_J_PH = 7,
  GD_GRID_T = 8, GD_GRID_GTH = 9, GD_GRID_GPH = 10, GD_GRID_GR = 11,
  GD_GRID_TADV = 12, GD_GRID_VADV_TH = 13, GD_GRID_VADV_PH = 14,
  GD_GRID_IND_TH = 15, GD_GRID_IND_PH = 16,
  /* composition (compositional.jl): C, its gradient (theta, phi, r), -u.grad C + S */
  GD_GRID_C = 17, GD_GRID_CGTH = 18, GD_GRID_CGPH = 19, GD_GRID_CGR = 20, GD_GRID_CADV = 21
};

/* Boundary-condition types of a scalar field's modes (bc_type_inner /
 * bc_type_outer of the reference's scalar fields): fixed value, or fixed flux
 * dC/dr applied by the tau method (apply_flux_bc_tau!,
 * src/scalar_field_common.jl:866-935). */
enum { GD_BC_VALUE = 1, GD_BC_FLUX = 2 };

/* Precision modes. */
enum { GD_PREC_FP64 = 0, GD_PREC_MIXED = 1 };

/* Stages of the mixed-precision step that gd_set_fp64_stages can return to
 * FP64 (bit mask).  In the reference's step the theta and phi components of
 * every cross product vanish (the synthesized vectors have zero radial
 * components, src/shtnskit_field_functions.jl:264-279), so the velocity's
 * nonlinear term is its Coriolis term alone (src/velocity.jl:492-496): these
 * three stages are the whole chain the velocity, and so the kinetic energy,
 * depends on. */
enum {
  GD_STAGE_VEL_SYNTH = 1,    /* vector synthesis of u (Legendre, DMMA)                */
  GD_STAGE_VEL_PRODUCTS = 2, /* phi transforms of u and the Coriolis product          */
  GD_STAGE_VEL_ANALYSIS = 4, /* vector analysis of the velocity's terms (Legendre)    */
  GD_STAGE_VEL_ALL = 7,
  /* the vector synthesis of u on the tcgen05 tensor cores by int8 digit slices
   * (error-free products, int32 accumulation; FP64-accurate to about 2^-40
   * of row max x column max with 6 digits), writing what GD_STAGE_VEL_SYNTH
   * writes; takes precedence over GD_STAGE_VEL_SYNTH.  One shell range, lmax
   * <= 511: not with segments or a ball (GD_ERR_UNSUPPORTED). */
  GD_STAGE_VEL_SYNTH_I8 = 8
};

/* Time-stepping schemes of gd_step (the reference's ts_scheme,
 * src/simulation.jl:1054-1300): CNAB2 (build_rhs_cnab2! + solve_implicit_step!),
 * EAB2 (eab2_update! with the exponential cache of create_etd_cache) or ERK2
 * (erk2_integrate_full_step! with the cache of create_erk2_cache). */
enum { GD_SCHEME_CNAB2 = 0, GD_SCHEME_EAB2 = 1, GD_SCHEME_ERK2 = 2 };
/* geometry (src/parameters.jl:75): a spherical shell or a solid ball */
enum { GD_GEOM_SHELL = 0, GD_GEOM_BALL = 1 };

/*
 * Model configuration.  Mirrors GeoDynamoParameters (src/parameters.jl:14-76):
 * i_L/i_M/i_Th/i_Ph/i_N/i_KL, d_rratio, d_E, d_Ra, d_Pr, d_Pm, d_timestep,
 * d_implicit, i_B.  The three mode switches resolve reference quirks:
 *   ab_mode   0: CNAB2, AB1 on the first step only; 1: AB1 on every step
 *             (step_once! never advances the step counter, simulation.jl:1153).
 *   bc_mode   0: reference behaviour (temperature Dirichlet rows only,
 *             thermal.jl:262-303); 1: also zero the r=ri and r=ro rows of all
 *             five fields after each solve; 2: Dirichlet rows inside the
 *             implicit operators of all five fields (well-posed variant; the
 *             reference's operators have no boundary rows).
 *   fd_mode   0: radial difference weights from V^T w = rhs (the intent of
 *             create_derivative_matrix, linear_algebra.jl:90-132);
 *             1: the literal V c = rhs solve (ill-conditioned, kept for study).
 * composition 1 adds the compositional field C (include_composition,
 * src/simulation.jl:107-131): advected by the velocity after the magnetic phase
 * (step_once!), diffusivity Pm/Sc with schmidt = d_Sc, no-flux boundaries by
 * default (create_shtns_composition_field, src/compositional.jl:80-118).  Its
 * buoyancy is a radial force, which the vector analysis does not keep, so C
 * does not act on the velocity.  Every time scheme (the exponential ones
 * with composition as a fourth operator kind); under bc_mode 2 its boundary
 * types default to fixed values, the right-hand sides of its Dirichlet rows.
 * segments > 1 stacks that many independent shells of nr / segments levels
 * each (same grid, diffusivities, dt and modes; their own Ekman numbers through
 * gd_set_segment_ekman) along r: every per-shell kernel serves them all in one
 * launch, and the radial operators act within each segment.  The ensemble
 * groups its members this way.  CNAB2, no composition; the mode-range,
 * reverse-mode and standalone-operator entry points refuse such a handle
 * (GD_ERR_UNSUPPORTED).  Boundary values and types apply to every segment;
 * heat sources are given per shell.  0 or 1: one shell.  segment_nr (read at
 * creation only) gives segments of unequal length, each with the radial grid
 * and operators of its own level count (tau functions and flux-row factors
 * included, so flux boundaries work in every bc_mode).
 * geometry GD_GEOM_BALL is the solid sphere of GeoDynamoBall
 * (src/Ball/Ball.jl): cosine nodes on [0, r_outer] (r_outer = d_R_outer,
 * rratio unused), the angular gradient and both curl components 0 at r = 0
 * (src/scalar_field_common.jl:300-310, src/velocity.jl:417-422,
 * src/magnetic.jl:325-330), regularity (the r = 0 level 0 for l >= 1) on the
 * analysed temperature and induction terms and on the temperature after its
 * boundary rows, no inner boundary row at r = 0 (src/thermal.jl:281-312).
 * The reference's implicit operator holds 1/r and 1/r^2 at r = 0 (infinite;
 * 0 x inf at l = 0), so a ball needs bc_mode 2, whose r = 0 row is the
 * regularity condition for l >= 1 and the inner boundary value for the l = 0
 * temperature and composition (centre values); CNAB2; an outer flux row is
 * allowed, an inner flux refused (the centre row is the regularity condition).
 * Entry points whose
 * operators divide by r (reverse mode, exponential schemes, the standalone
 * timestepping operator, the distributed step) refuse a ball.
 */
typedef struct gd_config {
  int lmax, mmax, nlat, nlon, nr;
  int kl;
  double rratio;
  double ekman, rayleigh, prandtl, magnetic_prandtl;
  double dt, implicit_theta;
  int ab_mode;
  int bc_mode;
  int fd_mode;
  int precision;
  int magnetic;
  int composition;
  double schmidt;
  int segments;
  int geometry;
  double r_outer;
  const int* segment_nr;  /* segments > 1: the levels of each segment (summing to nr; null: equal) */
} gd_config;

typedef struct gd_handle gd_handle;

/* ---- lifetime ---------------------------------------------------------------
 * Replaces initialize_simulation's transform and matrix set-up:
 * create_shtnskit_config (src/shtnskit_transforms.jl:102-200),
 * create_radial_domain (src/fields.jl:108-131) and
 * create_shtns_timestepping_matrices x3 (src/timestep.jl:498-543,
 * src/simulation.jl:228-231).  Tables, difference weights and LU factors are
 * computed on the device in FP64. */
int gd_create(const gd_config* cfg, int device, gd_handle** out);
int gd_destroy(gd_handle* h);
const char* gd_last_error(const gd_handle* h);
/* nlm, bytes of device memory held by the handle. */
int gd_info(const gd_handle* h, int* nlm, size_t* device_bytes);
/* Gauss colatitudes (north to south), weights and radial nodes (host out). */
int gd_grid(gd_handle* h, double* theta, double* weights, double* r);
/* Switch precision of transforms and nonlinear terms (GD_PREC_*). */
int gd_set_precision(gd_handle* h, int mode);
/* Stages (GD_STAGE_* mask) that the mixed-precision step runs in FP64 with the
 * FP64 path's kernels; 0 (the default) runs all of them in mixed precision.
 * With GD_STAGE_VEL_ALL the velocity's nonlinear term, and so the velocity
 * field, equals the FP64 step's.  Has no effect in GD_PREC_FP64. */
int gd_set_fp64_stages(gd_handle* h, int mask);
/* Digits of 7 bits per operand of GD_STAGE_VEL_SYNTH_I8: 6 (default; 21 digit
 * products per term) or 5 (15 products, about 2^-33). */
int gd_set_int8_digits(gd_handle* h, int digits);
int gd_synchronize(gd_handle* h);

/* ---- state ------------------------------------------------------------------
 * Host <-> device copies of the spectral fields in the reference layout (the
 * five of the step, and GD_COMP with composition). */
int gd_upload_spectral(gd_handle* h, int field, const double* re, const double* im);
int gd_download_spectral(gd_handle* h, int field, double* re, double* im);
int gd_download_nonlinear(gd_handle* h, int field, double* re, double* im);
int gd_download_grid(gd_handle* h, int grid, double* out);
/* Temperature Dirichlet values [2][nlm] (inner, outer; boundary_values in
 * thermal.jl:285,297) and internal sources [nr] (add_internal_sources_local!,
 * scalar_field_common.jl:416-443).  Either pointer may be NULL. */
int gd_set_temperature_bc(gd_handle* h, const double* bvals, const double* sources);
/* Composition boundary values or fluxes [2][nlm] and internal sources [nr]
 * (boundary_values, internal_sources of SHTnsCompositionField,
 * src/compositional.jl:106-111); GD_ERR_STATE without composition. */
int gd_set_composition_bc(gd_handle* h, const double* bvals, const double* sources);
/* Boundary types (GD_BC_VALUE / GD_BC_FLUX) of every mode of a scalar field
 * (GD_TEMP or GD_COMP), inner[nlm] and outer[nlm] in the reference's l-major
 * order (bc_type_inner / bc_type_outer).  Defaults: temperature GD_BC_VALUE,
 * composition GD_BC_FLUX (zero flux).  Where a mode's type is GD_BC_FLUX its
 * boundary value is the prescribed flux dC/dr, imposed by the tau method of
 * apply_flux_bc_tau! (src/scalar_field_common.jl:866-935) on the state after
 * the field's nonlinear term: Chebyshev T_{N-1} and T_N (or the one-sided
 * combinations when one boundary has a flux) are added to the radial profile
 * with the coefficients that cancel the real profile's flux error, the same
 * correction going to the imaginary profile when it is not ~0.  Under
 * bc_mode 2 (boundary rows in the implicit operator) a flux mode's boundary
 * row is the row of D1 instead of the identity, its right-hand side the
 * prescribed flux; the tau correction is then not applied.  GD_ERR_UNSUPPORTED:
 * an inner flux type on a ball (its centre row is the regularity condition);
 * GD_ERR_SINGULAR: a zero pivot in the bc_mode 2 factors with flux rows. */
int gd_set_scalar_bc_types(gd_handle* h, int field, const int* inner, const int* outer);

/* ---- transforms on host arrays (reference layout) ---------------------------
 * shtnskit_spectral_to_physical! / batch_spectral_to_physical!
 * (src/shtnskit_field_functions.jl:11-21, 674-677): nfield scalar fields,
 * re/im are nfield consecutive nr x nlm planes, grid nfield consecutive grids. */
int gd_spectral_to_physical(gd_handle* h, int nfield, const double* re, const double* im, double* grid);
/* shtnskit_physical_to_spectral! (src/shtnskit_field_functions.jl:131-141). */
int gd_physical_to_spectral(gd_handle* h, int nfield, const double* grid, double* re, double* im);
/* shtnskit_vector_synthesis!(tor, pol, vec) (src/shtnskit_field_functions.jl:252-282):
 * poloidal coefficients act as the spheroidal potential; only theta/phi written. */
int gd_vector_synthesis(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                        const double* pol_im, double* v_theta, double* v_phi);
/* shtnskit_vector_analysis!(vec, tor, pol) (src/shtnskit_field_functions.jl:291-321). */
int gd_vector_analysis(gd_handle* h, const double* v_theta, const double* v_phi, double* tor_re,
                       double* tor_im, double* pol_re, double* pol_im);
/* ball_physical_to_spectral! / ball_vector_analysis! (src/Ball/Ball.jl:214-245):
 * the analyses above, then the first radial level set to 0 for l >= 1 (as the
 * reference does, whatever the geometry). */
int gd_ball_physical_to_spectral(gd_handle* h, int nfield, const double* grid, double* re, double* im);
int gd_ball_vector_analysis(gd_handle* h, const double* v_theta, const double* v_phi, double* tor_re,
                            double* tor_im, double* pol_re, double* pol_im);
/* enforce_ball_scalar_regularity! / enforce_ball_vector_regularity!
 * (src/Ball/Ball.jl:153-195) on a state field (GD_U_TOR .. GD_COMP): its first
 * radial level set to 0 for l >= 1. */
int gd_enforce_regularity(gd_handle* h, int field);

/* No counterpart in the reference.  Scalar synthesis (as
 * gd_spectral_to_physical, but always in FP64, whatever the handle's
 * precision mode: it runs the FP64 kernels) for callers that must not allocate
 * device memory during the call -- for example a Julia session whose GPU memory
 * is owned by CUDA.jl's pool, or a solver loop that forbids allocation after
 * set-up.  d_coef and d_grid are the caller's device buffers in the native
 * layout: d_coef holds nfield fields of two planes (Re, Im) of nr x nlm doubles
 * with the m-major mode index j = moff[m] + (l - m); d_grid receives nfield
 * grids of nr x nlat x nlon doubles, phi fastest.  The Fourier intermediate
 * uses a fixed 64 MiB array in the library's device image instead of
 * cudaMalloc: min(nfield, 4) x nr x (mmax+1) x nlat x 16 bytes must fit, else
 * GD_ERR_CONFIG.  The first call on a device looks up that array's device
 * address; make it before any stream capture.  The cached address assumes the
 * device's primary context lives as long as the process (no device reset in
 * between).  The caller's current device is restored on return.  The array is shared by every
 * call and keeps the last call's contents (each call overwrites what it
 * reads), so calls that overlap on the GPU (other streams, other threads)
 * race.  Runs asynchronously on the handle's stream; gd_synchronize() waits. */
int gd_spectral_to_physical_noalloc(gd_handle* h, int nfield, const double* d_coef, double* d_grid);

/* ---- the reference's nonlinear and time-step functions on host arrays ---------
 * The same arguments as the reference functions (spectral planes nr x nlm,
 * l-major; physical grids nr x nlon x nlat, theta fastest), for a caller that
 * keeps its fields in its own arrays.  They use the handle's model state as
 * the reference's functions use their field structs: the fields and carried
 * grids they take are copied into the handle, so a later gd_step continues
 * from them.  Computed with the FP64 kernels whatever the precision mode.
 *
 * compute_temperature_nonlinear!(temp, vel, oc) (src/thermal.jl:149-190):
 * t_re/t_im in: the temperature; out: with the Dirichlet rows applied in place
 * (thermal.jl:262-303, values of gd_set_temperature_bc).  u_theta/u_phi: the
 * velocity grids it is advected by.  t_grid (may be NULL): the temperature grid. */
int gd_compute_temperature_nonlinear(gd_handle* h, double* t_re, double* t_im, const double* u_theta,
                                     const double* u_phi, double* nl_re, double* nl_im, double* t_grid);
/* compute_composition_nonlinear!(comp, vel, oc) (src/compositional.jl:219-259) on
 * host arrays, as gd_compute_temperature_nonlinear: composition in (its
 * boundary conditions of gd_set_composition_bc / gd_set_scalar_bc_types applied
 * in place), the velocity grids it is advected by, the nonlinear term and the
 * composition grid (may be NULL) out.  Needs a handle with composition. */
int gd_compute_composition_nonlinear(gd_handle* h, double* c_re, double* c_im, const double* u_theta,
                                     const double* u_phi, double* nl_re, double* nl_im, double* c_grid);
/* compute_velocity_nonlinear!(fields, temp, comp, mag, domain) (src/velocity.jl:312-332):
 * the velocity (toroidal, poloidal), the grids j and B of the previous magnetic
 * phase (all four may be NULL only without a magnetic field) -> the nonlinear
 * terms and, when not NULL, the velocity grids u_theta, u_phi. */
int gd_compute_velocity_nonlinear(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                                  const double* pol_im, const double* j_theta, const double* j_phi,
                                  const double* b_theta, const double* b_phi, double* nl_tor_re, double* nl_tor_im,
                                  double* nl_pol_re, double* nl_pol_im, double* u_theta, double* u_phi);
/* compute_magnetic_nonlinear!(mag, vel, oc, ic, rot) (src/magnetic.jl:131-159):
 * the magnetic field (toroidal, poloidal) and the velocity grids -> the
 * nonlinear terms and, when not NULL, the grids B and j. */
int gd_compute_magnetic_nonlinear(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                                  const double* pol_im, const double* u_theta, const double* u_phi,
                                  double* nl_tor_re, double* nl_tor_im, double* nl_pol_re, double* nl_pol_im,
                                  double* b_theta, double* b_phi, double* j_theta, double* j_phi);
/* SHTnsImplicitMatrices from create_shtns_timestepping_matrices(config, domain,
 * diffusivity, dt; theta) (src/timestep.jl:489-543): per degree l the operator
 * L_l = diffusivity (d2/dr2 + (2/r) d/dr - l(l+1)/r^2) and the banded LU of
 * I/dt - theta L_l (linear_algebra.jl:23-57), on the handle's device.
 * GD_ERR_SINGULAR on a zero pivot. */
typedef struct gd_matrices gd_matrices;
int gd_create_timestepping_matrices(gd_handle* h, double diffusivity, double dt, double theta, gd_matrices** out);
int gd_destroy_timestepping_matrices(gd_matrices* m);
/* build_rhs_cnab2!(rhs, un, nl, nl_prev, dt, matrices) (src/timestep.jl:610-690):
 * rhs = un/dt + (1 - theta) L_l un + 3/2 nl - 1/2 nl_prev. */
int gd_build_rhs_cnab2(gd_handle* h, const gd_matrices* m, double dt, const double* un_re, const double* un_im,
                       const double* nl_re, const double* nl_im, const double* prev_re, const double* prev_im,
                       double* rhs_re, double* rhs_im);
/* solve_implicit_step!(sol, rhs, matrices) (src/timestep.jl:692-730): per (l, m)
 * and Re / Im plane, the banded forward and back substitution (solve_banded!,
 * linear_algebra.jl:59-88). */
int gd_solve_implicit_step(gd_handle* h, const gd_matrices* m, const double* rhs_re, const double* rhs_im,
                           double* sol_re, double* sol_im);

/* ---- model step ---------------------------------------------------------------
 * compute_temperature_nonlinear! (src/thermal.jl:149-190),
 * compute_velocity_nonlinear! (src/velocity.jl:312-332),
 * compute_magnetic_nonlinear! (src/magnetic.jl:131-159) on the device state. */
int gd_temperature_nonlinear(gd_handle* h);
int gd_velocity_nonlinear(gd_handle* h);
int gd_magnetic_nonlinear(gd_handle* h);
/* compute_composition_nonlinear! (src/compositional.jl:219-259), with the
 * velocity grids of the last velocity phase; GD_ERR_STATE without composition. */
int gd_composition_nonlinear(gd_handle* h);
/* apply_master_implicit_step! (src/simulation.jl:1151-1330) with
 * build_rhs_cnab2! + solve_implicit_step! (src/timestep.jl:610-730). */
int gd_implicit_step(gd_handle* h);
/* step_once! (scripts/bench_timestepping.jl:6-18) repeated nsteps times;
 * after the first step the sequence is replayed from a captured CUDA graph. */
int gd_step(gd_handle* h, int nsteps);
/* Like gd_step, but records nothing to host and returns immediately
 * (asynchronous on the handle's stream). */
int gd_step_async(gd_handle* h, int nsteps);
/* Rebuild the implicit matrices (and, under EAB2, the exponential cache) for a
 * new time step (src/simulation.jl:335-337). */
int gd_set_dt(gd_handle* h, double dt);
/* Select the time-stepping scheme of gd_step: ts_scheme = :cnab2, :eab2 or
 * :erk2 (src/simulation.jl:1054-1300).  The exponential schemes build, per
 * field kind and degree l, E = exp(dt A_l), phi1(dt A_l), phi2(dt A_l) and E,
 * phi1 at dt/2 (create_etd_cache / create_erk2_cache, src/timestep.jl:37-70,
 * 896-968; A_l the operator of the CNAB2 matrices) on the device.  EAB2
 * replaces the banded solve by u <- E u + dt phi1 (3/2 N - 1/2 N_prev)
 * (eab2_update!, :429-487; no AB1 start: the history starts as zeros, as
 * prev_nonlinear does); ERK2 by the staged update of erk2_integrate_full_step!
 * (stage E(dt/2) u + dt/2 phi1(dt/2) N, the nonlinear terms of the stage,
 * u <- E u + dt (phi1 N + phi2 (N_stage - N)), then the nonlinear terms of
 * the new state).  GD_ERR_UNSUPPORTED with bc_mode 2 (the reference's
 * exponential schemes have no boundary rows) or nr > 256. */
int gd_set_scheme(gd_handle* h, int scheme);
/* One matrix of the exponential cache of field kind `kind` (0 velocity,
 * 1 magnetic, 2 temperature) at degree l, nr x nr row-major: which = 0 E,
 * 1 phi1, 2 phi2, 3 E at dt/2, 4 phi1 at dt/2 (the ERK2Cache fields,
 * src/timestep.jl:830-853).  GD_ERR_ARG under GD_SCHEME_CNAB2. */
int gd_download_etd(gd_handle* h, int kind, int l, int which, double* out);
/* compute_kinetic_energy / compute_magnetic_energy (src/velocity.jl:782-825,
 * src/magnetic.jl:504-543), both as 0.5 sum (T^2+P^2)/max(l(l+1),1). */
int gd_energy(gd_handle* h, double* ekin, double* emag);
/* The same per segment of a segmented handle (segments values each; gd_energy
 * returns their sums).  Each segment's sum runs in the order of an
 * unsegmented handle of nr / segments levels. */
int gd_segment_energy(gd_handle* h, double* ekin, double* emag);
/* Scan the five fields for NaN/Inf; returns GD_ERR_NONFINITE if found. */
int gd_check_finite(gd_handle* h);
long gd_step_count(const gd_handle* h);

/* ---- reverse mode ---------------------------------------------------------------
 * Pieces of the gradient of an objective of the state with respect to the
 * initial state (the adjoint configuration: misfit of the radial magnetic
 * field at r = ro against a target, with respect to the initial poloidal
 * magnetic coefficients).  The reference has no adjoint.
 *
 * Transpose of gd_spectral_to_physical: for a cotangent of the grids (nfield x
 * nr x nlon x nlat, reference layout) the cotangents of the Re and Im
 * coefficients (nfield x nr x nlm each, l-major).  Computed as the Gauss
 * analysis of grid / w_theta scaled by nlon / 2 pi (m = 0) and nlon / pi (m > 0);
 * the m = 0 imaginary parts, which the synthesis ignores, get zero. */
int gd_spectral_to_physical_adjoint(gd_handle* h, int nfield, const double* grid, double* re, double* im);
/* Pullback of nsteps model steps (gd_step) with respect to the magnetic
 * field component `field` (GD_B_TOR or GD_B_POL) at their start: given the
 * cotangent lambda of that component after the steps (nr x nlm Re and Im
 * planes, l-major), returns M^T ... M^T lambda.  In the reference's step the
 * magnetic field evolves by its implicit operator alone -- its nonlinear term
 * u x B and its Lorentz coupling j x B are products with the zero radial
 * components of the synthesized vectors (src/shtnskit_field_functions.jl:
 * 264-279, src/magnetic.jl:375-404, src/velocity.jl:638-672), zero in value
 * and in first derivative -- so M = S^-1 R per step (with the boundary rows
 * of bc_mode 1 and 2), the same for every step and every state, and this is
 * the exact gradient of anything that depends on the field after the steps.
 * FP64 in both precision modes (the implicit solve is FP64 in both). */
int gd_magnetic_pullback(gd_handle* h, int field, int nsteps, const double* lam_re, const double* lam_im,
                         double* out_re, double* out_im);

/* ---- batched ensemble ----------------------------------------------------------
 * Independent shells of different sizes and parameters stepped together (the
 * batched uneven ensemble of 64 shell runs; the reference runs one model per
 * process and has no counterpart).  The members are ordinary handles created
 * from cfgs[0..n-1] on one device; each keeps its own stream and state and
 * takes every gd_* call between ensemble steps.  gd_ensemble_step runs all
 * members' steps as independent branches of one CUDA graph, one graph launch
 * per step for the whole ensemble; when the members' AB-bootstrap flags differ
 * or a member has per-kernel timing enabled, each member is stepped through
 * its own graph on its own stream instead. */
typedef struct gd_ensemble gd_ensemble;
int gd_ensemble_create(const gd_config* cfgs, int n, int device, gd_ensemble** out);
int gd_ensemble_destroy(gd_ensemble* e);
int gd_ensemble_size(const gd_ensemble* e);
/* Member i, owned by the ensemble (not to be passed to gd_destroy); null if out of range. */
gd_handle* gd_ensemble_member(gd_ensemble* e, int i);
/* nsteps steps of every member, then synchronises.  On failure returns the
 * status of the first failing member; gd_ensemble_failed_member names it. */
int gd_ensemble_step(gd_ensemble* e, int nsteps);
/* Like gd_ensemble_step without the final synchronisation (errors raised by the
 * kernels are reported by the next gd_ensemble_step); a member's own gd_* calls
 * must wait until the ensemble stream has been synchronised. */
int gd_ensemble_step_async(gd_ensemble* e, int nsteps);
int gd_ensemble_failed_member(const gd_ensemble* e);
/* The ensemble's own stream (cudaStream_t as void*): every graph-launched step is
 * joined to it, so events recorded on it bracket whole ensemble steps. */
int gd_ensemble_get_stream(gd_ensemble* e, void** stream);
/* Chooses the members' launch shapes (gd_set_launch_shape) by measurement:
 * candidate caps of the tensor-core grids -- one cap for every member, or caps
 * proportional to each member's share of the Legendre work -- each timed over
 * nsteps steps of a scratch ensemble built from the members' configurations,
 * precisions and schemes (the members themselves are not stepped, and the
 * scratch ensemble needs as much device memory again while it exists).  The
 * fastest is applied; *best_ms = its time per ensemble step, caps_out[i] =
 * member i's cap (either pointer may be null). */
int gd_ensemble_autotune(gd_ensemble* e, int nsteps, float* best_ms, int* caps_out);

/* ---- the step decomposed across ranks ---------------------------------------------
 * The reference distributes its step over MPI pencils (src/pencil_decomps.jl:
 * 136-284).  Here a rank owns whole m columns (native mode range [j0, j1),
 * j = moff[m] + l - m) for the radial half of the step -- the radial
 * derivatives and the CNAB2 solve, which couple every shell of a mode -- and a
 * slab of shells for the transform half -- syntheses, products, analyses, which
 * are independent per shell -- with one all-to-all of spectral blocks in each
 * direction between the halves:
 *   gd_derivatives(mode handle, j0, j1)          grad T, curl u, curl B -> work arrays
 *   (exchange: state and derivatives of its modes -> the shell-slab handles)
 *   gd_temperature_nonlinear, gd_velocity_nonlinear, gd_magnetic_nonlinear
 *     (shell-slab handle, in gd_step's order)    with gd_set_external_derivatives(1)
 *   (exchange: nonlinear terms of its shells -> the mode handles)
 *   gd_implicit_modes(mode handle, j0, j1)       temperature Dirichlet rows, CNAB2, history roll
 *
 * Radial derivatives of the state (compute_all_gradients_spectral!,
 * compute_vorticity_spectral_full!, compute_current_density_spectral!) for the
 * modes [j0, j1) only, into the handle's work arrays (0-2: grad T theta, phi,
 * r; 3-4: curl u toroidal, poloidal; 5-6: curl B; 8-10: grad C). */
int gd_derivatives(gd_handle* h, int j0, int j1);
/* The temperature Dirichlet rows and the CNAB2 solve (build_rhs_cnab2! +
 * solve_implicit_step!) for the modes [j0, j1) only, with the nonlinear terms in
 * the handle's current bank, then the step's history roll.  CNAB2 only. */
int gd_implicit_modes(gd_handle* h, int j0, int j1);
/* enable != 0: the nonlinear phases take the radial derivatives from the work
 * arrays instead of computing them, and leave the temperature Dirichlet rows to
 * the solve side (a shell-slab handle: nr = its shells, the sources of its
 * shells set with gd_set_temperature_bc). */
int gd_set_external_derivatives(gd_handle* h, int enable);
/* Copies the block [shells r0..r1) x [modes j0..j1) of one spectral array
 * between the handle and buf (device or pinned host memory), both planes:
 * buf = [Re, Im][r1 - r0][j1 - j0] doubles.  array 0: state field (GD_U_TOR ..
 * GD_TEMP, GD_COMP); 1: work array 0-10; 2: nonlinear term of the current bank.
 * to_buf != 0 copies from the handle into buf.  Synchronises the stream. */
int gd_copy_block(gd_handle* h, int array, int field, int r0, int r1, int j0, int j1, void* buf, int to_buf);

/* ---- reverse mode of the temperature step ----------------------------------------
 * No counterpart in the reference (it has no adjoint).  The temperature obeys
 *   T^(n+1) = C S^-1 D (R P T^n + a_n N_n T^n - b_n N_(n-1) T^(n-1)) + const
 * (compute_temperature_nonlinear!, build_rhs_cnab2!, solve_implicit_step!):
 * P the fixed-value boundary rows, R = I/dt + (1 - theta) L_l, S = I/dt -
 * theta L_l, C the bc_mode 1 row clamp, D the bc_mode 2 right-hand-side rows,
 * a_n = 1.5 and b_n = 0.5 (1 and 0 on an Adams-Bashforth start), and
 * N_n T = An(-(u_th Syn(G_th T) + u_ph Syn(G_ph T))) the advection by the
 * velocity grids that step n's temperature phase reads (the velocity does not
 * depend on the temperature: its buoyancy is radial and is not kept).  These
 * entry points are the pieces of the pullback; the caller keeps the velocity
 * grids of each step, recomputed from snapshots (checkpoint and recompute).
 * Spectral arguments are device arrays in the native layout [Re, Im][nr][nlm]
 * (gd_spectral_device converts), grids device arrays in the native grid
 * layout [nr][nlat][nlon] (gd_grid_device copies the handle's).
 *
 * Snapshot of the step state (fields, both banks of nonlinear terms, the
 * grids a step reads before writing them -- u, B and j -- the bank parity and
 * the step count) into or out of a device buffer of gd_snapshot_bytes bytes;
 * FP64 handles. */
int gd_snapshot_bytes(gd_handle* h, size_t* bytes);
int gd_snapshot(gd_handle* h, void* dev, int restore);
/* Host reference-layout (l-major) Re/Im planes <-> a native device array. */
int gd_spectral_device(gd_handle* h, double* re, double* im, double* dev, int to_device);
/* Copy of one of the handle's grids (FP64 handles) into a device buffer. */
int gd_grid_device(gd_handle* h, int grid, double* dev);
/* out = N^T nu for the advection by the velocity grids u_th, u_ph: the
 * transposed analysis, the products, the transposed synthesis and the
 * transposed spectral gradient (theta recurrence and i m, over r), FP64. */
int gd_temperature_nl_adjoint(gd_handle* h, const double* u_th, const double* u_ph, const double* nu, double* out);
/* mode 0: y = D S^-T C x; mode 1: y = P R^T x (scalar fields: P zeroes the
 * fixed-value boundary rows; the potentials have no P), with the field's
 * implicit operators.  Fixed-value boundaries only: GD_ERR_UNSUPPORTED when the
 * field has flux boundaries. */
int gd_cnab2_adjoint(gd_handle* h, int field, int mode, const double* x, double* y);
/* out = N^T psi for the velocity's nonlinear term, which in the literal step is
 * its Coriolis term alone (u x w and j x B vanish with zero radial components;
 * src/velocity.jl:492-496): N = VecAn Cor VecSyn with Cor antisymmetric per
 * grid point, so N^T = -D^-1 Lambda N Lambda^-1 D (Lambda = l(l+1), D the
 * real-coefficient weights of the phi sums).  psi, out: (tor, pol) consecutive
 * device arrays of gd_snapshot's spectral layout (spec_elems doubles each), FP64. */
int gd_velocity_nl_adjoint(gd_handle* h, const double* psi, double* out);
/* Vector-Jacobian product of the last nsteps CNAB2 steps the handle ran (those
 * ending at its step count; GD_ERR_STATE if it ran fewer) with respect to
 * (u_tor, u_pol) at their start: lambda (host, l-major (nr, nlm) planes) is the
 * cotangent of the velocity after the steps.  The velocity
 * of the literal step depends on nothing but itself (Q2: no buoyancy; the
 * Lorentz term vanishes), linearly, so no checkpoints are needed.  The
 * pullback of the FP64 step. */
int gd_velocity_pullback(gd_handle* h, int nsteps, const double* lam_tor_re, const double* lam_tor_im,
                         const double* lam_pol_re, const double* lam_pol_im, double* out_tor_re, double* out_tor_im,
                         double* out_pol_re, double* out_pol_im);
/* The pieces composed with checkpoint and recompute.  gd_temperature_forward
 * runs nsteps steps keeping a snapshot every checkpoint_every steps (and one
 * of the end state) in device memory owned by the handle (FP64, CNAB2).
 * gd_temperature_pullback then maps the cotangent of the temperature after
 * those steps (lam, reference layout) to its cotangent at their start (out):
 * segment by segment from the last, it restores the segment's snapshot, steps
 * through it again recording the velocity grids each step's temperature
 * phase reads, and applies psi^n = D S^-T C lambda^n,
 * lambda^n = P R^T psi^(n+1) + N_n^T (a_n psi^(n+1) - b_(n+1) psi^(n+2));
 * it leaves the handle in the end state of the forward run.  The snapshots
 * hold the state, both banks of nonlinear terms and the grids a step reads
 * before writing (u, B, j). */
int gd_temperature_forward(gd_handle* h, int nsteps, int checkpoint_every);
int gd_temperature_pullback(gd_handle* h, const double* lam_re, const double* lam_im, double* out_re, double* out_im);
/* The same, and the gradient with respect to the velocity potentials at the
 * start of the run: step n's advection reads the grids VecSyn(u^(n-1)) of the
 * previous velocity phase, so u^(n-1) receives
 * s^(n-1) = VecSyn^T(-(An^T nu_n) (G_th T^n, G_ph T^n)) (nu_n the cotangent of
 * step n's nonlinear term) and the velocity recursion of gd_velocity_pullback
 * carries the sources back; the grids carried into the run (read by its first
 * step) are constants.  The recompute also keeps each step's temperature
 * gradient grids (4 grids per step of a segment). */
int gd_temperature_pullback_full(gd_handle* h, const double* lam_re, const double* lam_im, double* out_re,
                                 double* out_im, double* out_tor_re, double* out_tor_im, double* out_pol_re,
                                 double* out_pol_im);
/* out (tor, pol) = VecSyn^T(-(An^T nu) (gth, gph)): the velocity cotangent of
 * one step's advection for the temperature gradient grids gth, gph (device
 * arrays, gd_grid_device layout) and the cotangent nu of its nonlinear term. */
int gd_temperature_u_adjoint(gd_handle* h, const double* gth, const double* gph, const double* nu, double* out);

/* ---- launch shape -------------------------------------------------------------------
 * No counterpart in the reference.  tc_ctas caps the persistent grid of the
 * tensor-core Legendre kernels (0, the default: one CTA per SM).  Each of those
 * CTAs holds about 192 KB of shared memory, so an uncapped launch occupies
 * every SM; members of an ensemble run side by side only when their grids are
 * capped.  The arithmetic of every tile is the same whatever CTA runs it: the
 * results do not depend on the cap.  gd_ensemble_autotune chooses the caps of
 * an ensemble's members by measurement. */
int gd_set_launch_shape(gd_handle* h, int tc_ctas);
/* Ekman number of each segment (segments values): the Coriolis and Lorentz
 * factor Pm/E of its shells (rossby_factor, src/velocity.jl:456). */
int gd_set_segment_ekman(gd_handle* h, const double* ekman);
/* Kernel launches of the next step: the kernel nodes of its captured CUDA
 * graph (captured here if needed, without running it). */
int gd_step_kernels(gd_handle* h, int* count);
int gd_get_launch_shape(const gd_handle* h, int* tc_ctas);

/* ---- error-path testing ----------------------------------------------------------
 * No counterpart in the reference.  Every wait of the tensor-core pipelines is
 * bounded: when one runs out the kernel records it, lets its copies in flight
 * land, frees its tensor memory and returns, and the call reports GD_ERR_CUDA
 * ("wait expired"); the flag is then cleared, so the handle's next calls run
 * normally.  To test that path without a GPU fault: wait_cycles bounds every
 * wait (clock cycles; <= 0 restores the default of about a second) and
 * omit_step >= 0 makes the next tensor-core synthesis on this handle (the
 * split-TF32 one, or the int8-slice synthesis of u when GD_STAGE_VEL_SYNTH_I8
 * is set and a velocity phase comes first) skip the bulk copies of that
 * pipeline step in its first CTA (once), so the waits on that stage run out.  GD_ERR_STATE without mixed-precision state. */
int gd_set_fault_test(gd_handle* h, long long wait_cycles, int omit_step);

/* ---- tracing ------------------------------------------------------------------
 * The handle's CUDA stream (a cudaStream_t passed as void*), so a caller can
 * time work on it with its own events. */
int gd_get_stream(gd_handle* h, void** stream);
/* Per-kernel timing: while enabled, gd_step runs the step sequence without graph
 * replay and brackets every kernel launch with CUDA events on the handle's
 * stream; timings accumulate per kernel name. */
int gd_profile_enable(gd_handle* h, int enable);
/* Copies up to max entries: names (max x 32 chars, NUL-terminated), total ms and
 * launch counts; *count receives the number of entries.  Resets the totals. */
int gd_profile_read(gd_handle* h, int max, char* names, double* ms, int* launches, int* count);

#ifdef __cplusplus
}
#endif

#endif /* GDB200_H */

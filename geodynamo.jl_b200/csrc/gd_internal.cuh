// gd_internal.cuh -- shared definitions of libgdb200.so (not part of the ABI).
//
// Device layouts (native; the host ABI converts to and from the reference's):
//   mode index j      m-major: j = moff[m] + (l - m), l = m..lmax.
//   spectral field    two planes (Re, Im), each [r][j] doubles.
//   tables P, dP, Q   [j][ith], ith = north-half colatitude index (0..nlat/2-1);
//                     Q = m Pbar_lm / sin(theta).
//   Fourier buffer    [comp][r][m][s][ith] complex.  Synthesis: s = 0 north row,
//                     s = 1 south row (ith mirrored).  Analysis: s = 0 holds
//                     w (G_north + G_south), s = 1 holds w (G_north - G_south),
//                     with G the (2 pi / nlon)-scaled phi transform.
//   grid              [comp][r][itheta][jphi] (phi fastest).
//   LU / linear bands [kind][col][band][l] (l fastest; kind 0 velocity,
//                     1 magnetic, 2 temperature).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/gdb200.h"

#define GD_MAX_KL 4
#define GD_NBW (2 * GD_MAX_KL + 1)

namespace gd {

// F_COMP is allocated with the others and used when the configuration has
// composition; NWORK derived spectral arrays: 0-2 grad T, 3-4 curl u, 5-6 curl
// B, 7 scratch, 8-10 grad C.
enum { F_UTOR = 0, F_UPOL = 1, F_BTOR = 2, F_BPOL = 3, F_TEMP = 4, F_COMP = 5, NFIELD = 6 };
enum { NGRID = 22, NWORK = 11 };

struct Dims {
  int L, M, nlat, nlon, nr, nth, nlm, kl;
  // native mode range [jlo, jhi) of the radial operators, the temperature
  // Dirichlet rows and the CNAB2 solve (0, nlm unless a caller restricts it to
  // the m columns one rank owns)
  int jlo, jhi;
  // independent segments of nrs = nr / nseg shells stacked along r: the radial
  // operators act within each segment (blockIdx.z); rfs / rfs32 the Coriolis
  // and Lorentz factor of each shell when the segments' Ekman numbers differ
  // (null: the scalar factor of the configuration)
  int nseg, nrs;
  const double* rfs;
  const float* rfs32;
  // ball geometry: the first level of each segment is r = 0
  int ball;
  // segments of unequal length (null: nseg segments of nrs levels, one set of
  // radial operators): seg_info [nseg][3] = first shell, levels, operator
  // variant; var_off [variant][2] = offset (doubles) of the variant's D1 / D2
  // bands and of its implicit operators; nrs is then the longest segment
  const int* seg_info;
  const long* var_off;
};

// The shells and radial operators of segment z.
struct SegView {
  int base, n;
  long band_off, op_off;
};
__device__ __forceinline__ SegView seg_view(const Dims& d, int z) {
  if (d.seg_info == nullptr) return SegView{z * d.nrs, d.nrs, 0, 0};
  const int v = d.seg_info[3 * z + 2];
  return SegView{d.seg_info[3 * z], d.seg_info[3 * z + 1], d.var_off[2 * v], d.var_off[2 * v + 1]};
}

// Analysis epilogue variants.
enum { EPI_SCALAR = 0, EPI_VECTOR = 1, EPI_CURL_INDUCTION = 2 };

// ---- set-up kernels (gd_setup.cu) ----
void launch_gauss(cudaStream_t s, int nlat, double* x, double* w, double* th, double* sth);
void launch_tables(cudaStream_t s, const Dims& d, const int* moff, const double* x, const double* sth,
                   double* P, double* dP, double* Q);
void launch_fd_weights(cudaStream_t s, int nr, int kl, int fd_mode, const double* r, double* d1, double* d2);
void launch_rec_tables(cudaStream_t s, const Dims& d, const int* moff, const double* x, const double* sth,
                       double* ra, double* rb, double* rc, double* r1a, double* r1b, double* pmm, double* sinv);
void launch_build_lu(cudaStream_t s, int nr, int kl, int L, const double* d1, const double* d2,
                     const double* rinv, const double* rinv2, const double* nu, double dt, double theta,
                     int bc_rows, double* lin, double* lu, int* status, int nkind = 3);

// ---- Legendre (gd_legendre.cu) ----
struct SynthArgs {
  const double* table0;  // scalar: P ; vector: dP
  const double* table1;  // vector: Q
  const double* coef[4]; // scalar: nf fields ; vector: [0] = S (poloidal), [1] = T (toroidal)
  double2* out;          // Fourier buffer, comps consecutive
  int nf;                // scalar: number of fields (comps) ; vector: 1 (outputs 2 comps)
  // vector only, may be null: also write the components as FP32 in the mixed
  // step's blocked layout (float4 north Re, north Im, south Re, south Im at
  // [comp][r][theta block of 2][m][pair in block]); out32_comp = float4 per component
  float4* out32;
  size_t out32_comp;
};
void launch_synth_fp64(cudaStream_t s, const Dims& d, const int* moff, const SynthArgs& a, bool vec);

struct AnalysisArgs {
  const double* table0;  // scalar: P ; vector: dP
  const double* table1;  // vector: Q
  const double2* in;     // folded Fourier buffer (comps consecutive)
  double* out[4];        // scalar: nf outputs ; vector: [0] tor, [1] pol
  int nf;
  int epi;
  const double* sth;
};
void launch_analysis_fp64(cudaStream_t s, const Dims& d, const int* moff, const AnalysisArgs& a);

// ---- phi transforms (gd_fft.cu) ----
struct FftPlan {
  int n;
  int nstage;
  int radix[16];
  int tb;  // theta pairs per CTA
};
FftPlan make_fft_plan(int nlon);
template <typename R>
void launch_fft_synth(cudaStream_t s, const Dims& d, const FftPlan& p, const void* twiddle, const void* F,
                      R* grid, int ncomp, size_t grid_comp_stride);
template <typename R>
void launch_fft_analysis(cudaStream_t s, const Dims& d, const FftPlan& p, const void* twiddle, const R* grid,
                         size_t grid_comp_stride, const double* w, void* G, int ncomp);
void make_twiddles(int n, std::vector<double>& tw);
// The Coriolis term of the velocity phase in FP64 from the velocity's FP64
// Fourier components F (comps u_theta, u_phi) to the folded transforms G
// (comps theta, phi) plus the FP32 folds g32; false (nothing launched) for an
// nlon without a compile-time plan.
bool launch_coriolis_fused(cudaStream_t s, const Dims& d, int nlon, const void* tw, const void* F, const double* cth,
                           const double* sth, double rf, const double* w, const float2* g32, void* G);

// ---- nonlinear terms (gd_nonlinear.cu) ----
template <typename R>
void launch_temperature_advection(cudaStream_t s, const Dims& d, const R* uth, const R* uph, const R* gth,
                                  const R* gph, const R* gr, const double* sources, R* out);
template <typename R>
void launch_velocity_nl(cudaStream_t s, const Dims& d, const double* cth, const double* sth_cor, double rf,
                        double lf, int magnetic, const R* uth, const R* uph, const R* wth, const R* wph,
                        const R* jth, const R* jph, const R* bth, const R* bph, R* ath, R* aph);
template <typename R>
void launch_coriolis(cudaStream_t s, const Dims& d, const double* cth, const double* sth_cor, double rf, const R* uth,
                     const R* uph, R* ath, R* aph);
template <typename R>
void launch_induction(cudaStream_t s, const Dims& d, const R* uth, const R* uph, const R* bth, const R* bph,
                      R* oth, R* oph);

// ---- spectral operators (gd_spectral.cu) ----
void launch_gradients(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                      const double* d1, const double* T, double* gth, double* gph, double* gr);
void launch_curl(cudaStream_t s, const Dims& d, const int* lof, const double* rinv, const double* rinv2,
                 const double* d1, const double* d2, const double* tor, const double* pol, double* otor,
                 double* opol);
// Tau functions of the flux boundary conditions (apply_flux_bc_tau!,
// src/scalar_field_common.jl:629-812) on the radial nodes.
// Tau functions of every segment, on its own N nodes, at 4 base of `tau`:
// tau1 = T_{N-1}(x(r)), tau2 = T_N(x(r)), tau_in = tau1 - alpha tau2 (zero
// analytic derivative at ro), tau_out = tau1 - beta tau2 (zero at ri); and its
// constants at 6 z of `consts`: the analytic dT_{N-1}/dr, dT_N/dr at ri and ro
// (dt1i, dt1o, dt2i, dt2o), (D1 tau_in)[ri], (D1 tau_out)[ro].
struct TauConsts {
  const double* tau;
  const double* consts;
};
// Boundary conditions of a scalar field for the modes [jlo, jhi): fixed-value
// rows, then the tau correction of the modes with a flux boundary.
// types: [inner, outer][nlm] GD_BC_* (native order); bvals [2][nlm] values or fluxes.
void launch_scalar_bc(cudaStream_t s, const Dims& d, const int* lof, const double* bvals_native, const int* types,
                      const double* d1, const TauConsts& tc, double* F, int op_rows);
// ball: r = 0 level of nf fields (stride fstride doubles) set to 0 for l >= 1
void launch_regularity(cudaStream_t s, const Dims& d, const int* lof, double* F, int nf, size_t fstride);
void launch_lmajor_to_native(cudaStream_t s, const Dims& d, const int* native_of_lmajor, const double* src,
                             double* dst, int nplanes);
void launch_native_to_lmajor(cudaStream_t s, const Dims& d, const int* native_of_lmajor, const double* src,
                             double* dst, int nplanes);
void launch_grid_to_native(cudaStream_t s, const Dims& d, const double* ref, double* nat, int ncomp);
void launch_grid_to_reference(cudaStream_t s, const Dims& d, const double* nat, double* ref, int ncomp);
template <typename R>
void launch_grid_cast(cudaStream_t s, size_t n, const R* src, double* dst);

// ---- CNAB2 (gd_cnab2.cu) ----
struct Cnab2Args {
  double* u[6];
  const double* nl[6];
  const double* prev[6];  // the previous step's nonlinear terms (read only)
  int kind[6];            // 0 velocity, 1 magnetic, 2 temperature, 3 composition
  int nfield;
  int boot;
  int clamp_rows;
  int bc_rows;                // Dirichlet rows in the operator: boundary rhs = the slot's value or 0
  const double* rowvals[6];   // per slot: boundary values [2][nlm] (native order) of its rows (null: 0)
  // per slot, may be null: boundary types [2][nlm] (native order); a GD_BC_FLUX
  // row takes the factors with the row of D1 there, lu_flux + (v - 1) lu_flux_stride
  // with v = inner flux | 2 outer flux (the layout of lu)
  const int* rowtypes[6];
  const double* lu_flux;
  size_t lu_flux_stride;
  double inv_dt, lin_weight;
  double dt;                  // EAB2: the time step applied to the phi1 term
  int stages;                 // sweeps to run: 1 rhs, 2 forward, 4 back substitution (0: all)
};
// ---- exponential Adams-Bashforth 2 (gd_expo.cu) ----
// nkind: 3 (velocity, magnetic, temperature), 4 with composition
size_t etd_table_doubles(const Dims& d, int nkind);
size_t etd_scratch_doubles(const Dims& d, int nkind);
void launch_etd_build(cudaStream_t s, const Dims& d, const double* lin, double dt, double* scratch, double* tab,
                      int* err, int nkind);
// out = M_top x_top + M_bot (bot_scale * x_bot) per (field, l, m, plane) column (gd_expo.cu)
struct ExpApply {
  const double* top[6];       // per slot: x_top (u), unused without top_block
  const double* bot_a[6];     // per slot: a
  const double* bot_b[6];     // per slot: b (bot_mode 1, 2)
  double* out[6];             // may equal top
  const double* lin[6];       // epilogue 1 operands
  const double* k1[6];
  int kind[6];
  int nfield;
  int top_block, bot_block;   // table blocks 0 E, 1 phi1, 2 phi2, 3 E(dt/2), 4 phi1(dt/2); -1: none
  int bot_mode;               // x_bot = 0: a, 1: 3/2 a - 1/2 b, 2: a - b
  double bot_scale;
  int epilogue;               // 0: out = acc, 1: out = lin + dt (k1 + acc)
  double dt;
  int clamp_rows;             // bc_mode 1: zero rows 0 and nr-1 of out
};
void launch_exp_apply(cudaStream_t s, const Dims& d, const int* moff, const double* tab, const ExpApply& a);
// ---- reverse mode (gd_adjoint.cu) ----
void launch_cnab2_pullback(cudaStream_t s, const Dims& d, const int* lof, const double* lin, const double* lu,
                           int kind, double dt, double theta, int clamp_rows, int bc_rows, int nsteps, double* lam);
void launch_divide_by_weights(cudaStream_t s, size_t n, int nlat, const double* w, double* g);
void launch_scale_by_order(cudaStream_t s, size_t nrows, int nlm, const int* mof, double f0, double f1, double* a);
void launch_scale_by_degree(cudaStream_t s, size_t nrows, int nlm, const int* lof, double f, int inverse, double* a);
// Temperature adjoint pieces (gd_adjoint.cu).
void launch_cnab2_adjoint(cudaStream_t s, const Dims& d, const int* lof, const double* lin, const double* lu,
                          const int* types, int kind, int mode, double dt, double theta, int clamp_rows, int bc_rows,
                          const double* x, double* y);
void launch_gradients_adjoint(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                              const double* gth, const double* gph, double* out);
void launch_neg_product(cudaStream_t s, size_t n, const double* u, const double* g, double* out);
void launch_axpby(cudaStream_t s, size_t n, double a, const double* x, double b, const double* y, double* out);
void launch_cnab2(cudaStream_t s, const Dims& d, const int* lof, const double* d1, const double* d2,
                  const double* rinv, const double* rinv2, const double* nu, const double* lu, const Cnab2Args& a);
// partial sums per segment of the energy reduction: partial holds 2 x this x nseg
constexpr int GD_ENERGY_BLOCKS = 296;
void launch_energy(cudaStream_t s, const Dims& d, const int* lof, const double* utor, const double* upol,
                   const double* btor, const double* bpol, double* partial, double* out);
void launch_check_finite(cudaStream_t s, size_t n, const double* a, int* flag);

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// Kernel attributes and device properties are per device, and one process may
// hold handles on several devices from several host threads.  These helpers
// act on the current device (every entry point makes the handle's device
// current first) and are thread-safe.
//
// Raises func's dynamic shared-memory limit on the current device to at
// least `bytes`; the largest value set so far is remembered per
// (kernel, device), so repeated launches make no driver call.
cudaError_t allow_dynamic_smem(const void* func, size_t bytes);
template <typename K>
inline cudaError_t allow_dynamic_smem(K* kernel, size_t bytes) {
  return allow_dynamic_smem(reinterpret_cast<const void*>(kernel), bytes);
}
// Multiprocessor count of the current device (148 if it cannot be read).
int current_sm_count();

}  // namespace gd

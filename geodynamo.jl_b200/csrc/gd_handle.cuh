// gd_handle.cuh -- the handle behind the opaque gd_handle* of the C ABI.
#pragma once

#include <string>
#include <vector>

#include "gd_internal.cuh"

namespace gd {
struct MixedState;
}

struct gd_handle {
  gd_config c{};
  gd::Dims d{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long step_count = 0;
  int precision = GD_PREC_FP64;
  int int8_digits = 6;        // digits per operand of GD_STAGE_VEL_SYNTH_I8
  int fp64_stages = 0;        // GD_STAGE_* run in FP64 inside the mixed-precision step
  // the phases take the radial derivatives (grad T, curl u, curl B) from the
  // work arrays instead of computing them, and leave the temperature
  // Dirichlet rows to the solve side (a shell-slab handle of a distributed step)
  bool ext_derivs = false;
  // persistent CTAs of the tensor-core Legendre kernels (0: one per SM); an
  // ensemble caps them so that its members share the SMs
  int tc_ctas = 0;
  size_t bytes = 0;
  std::vector<void*> allocs;

  std::vector<int> lv, mv, moff, perm, lof, mof;
  gd::FftPlan plan{};

  int *d_moff = nullptr, *d_lof = nullptr, *d_mof = nullptr, *d_perm = nullptr, *d_flag = nullptr;
  double *d_x = nullptr, *d_w = nullptr, *d_th = nullptr, *d_sth = nullptr, *d_cth = nullptr, *d_sthc = nullptr;
  double *d_r = nullptr, *d_rinv = nullptr, *d_rinv2 = nullptr, *d_nu = nullptr;
  double *d_P = nullptr, *d_dP = nullptr, *d_Q = nullptr;
  double *d_d1 = nullptr, *d_d2 = nullptr, *d_lin = nullptr, *d_lu = nullptr;
  double* d_tw = nullptr;
  float* d_twf = nullptr;
  double* d_state = nullptr;  // NFIELD fields (composition used when configured)
  // Two banks of the five nonlinear terms: a step writes bank nl_par and the
  // Adams-Bashforth history is the other bank (the previous step's terms), so
  // the history roll N_prev := N is a flip of nl_par instead of a copy.
  double* d_nl = nullptr;     // bank 0
  double* d_prev = nullptr;   // bank 1
  int nl_par = 0;             // bank the next nonlinear terms go to
  int last_nl_par = 0;        // bank holding the most recently computed terms
  double* d_work = nullptr;   // NWORK derived spectral fields
  double *d_bvals = nullptr, *d_sources = nullptr;    // temperature: [2][nlm] values or fluxes, [nr]
  double *d_cbvals = nullptr, *d_csources = nullptr;  // composition
  int* d_bctype = nullptr;    // [temperature, composition][inner, outer][nlm] GD_BC_*
  std::vector<int> bctype;    // host copy of d_bctype
  double* d_adj = nullptr;    // adjoint scratch (lazy): 3 spectral fields, 3 grids
  // per-shell Coriolis / Lorentz factors of a segmented handle (gd_set_segment_ekman)
  double* d_rfs = nullptr;
  float* d_rfs32 = nullptr;
  // segments: first shell, levels, operator variant; variants: levels, first
  // shell of a segment of that length, offsets of its bands and operators
  std::vector<int> seg_base, seg_n, seg_var, var_n, var_rep;
  std::vector<long> var_band, var_op;
  int* d_seg_info = nullptr;
  long* d_var_off = nullptr;
  // bc_mode 2: the implicit factors with D1 rows for prescribed fluxes at the
  // inner (1), outer (2) or both (3) boundaries, each block laid out as d_lu
  double* d_lu_flux = nullptr;
  size_t lu_flux_stride = 0;
  bool flux_rows_ok = false;
  // checkpointed forward run of gd_temperature_forward
  std::vector<void*> t_snaps;
  void* t_final = nullptr;
  int t_nsteps = 0, t_every = 0;
  long t_s0 = 0;
  double* d_tauc = nullptr;   // per segment: the six tau constants
  double* d_tau = nullptr;    // tau1, tau2, tau_in, tau_out on the radial nodes
  gd::TauConsts tau{};
  double* d_grid = nullptr;   // NGRID grids (FP64)
  double2* d_F = nullptr;     // Fourier buffer, 4 components
  double *d_epart = nullptr, *d_eout = nullptr;
  // host-ABI staging (lazy)
  double *d_stage_spec = nullptr, *d_stage_spec2 = nullptr, *d_stage_grid = nullptr, *d_stage_grid2 = nullptr;
  // time-stepping scheme and the EAB2 exponential cache (lazy)
  int scheme = 0;             // GD_SCHEME_*
  double* d_etd = nullptr;    // [kind][l][5][nr][nr]: transposed E, phi1, phi2, E(dt/2), phi1(dt/2)
  double* d_erk2 = nullptr;   // ERK2: linear and k1 terms of the five fields
  // mixed precision state (lazy)
  gd::MixedState* mixed = nullptr;
  // graphs (index: boot flag)
  cudaGraphExec_t gexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [nl_par][boot]
  int graph_gen = 0;  // bumped whenever captured step graphs become stale
  int graph_kernels[2][2] = {{0, 0}, {0, 0}};  // kernel nodes of each captured step graph
  // per-kernel event timing (gd_profile_enable)
  bool profiling = false;
  struct ProfRec { const char* name; cudaEvent_t a, b; };
  std::vector<ProfRec> prof_pending;
  std::vector<std::string> prof_names;
  std::vector<double> prof_ms;
  std::vector<int> prof_count;

  size_t spec_elems() const { return (size_t)2 * d.nr * d.nlm; }
  size_t grid_elems() const { return (size_t)d.nlat * d.nlon * d.nr; }
  double* field(int f) { return d_state + spec_elems() * f; }
  double* nl_bank(int b) { return b ? d_prev : d_nl; }
  double* nlf(int f) { return nl_bank(nl_par) + spec_elems() * f; }
  double* prevf(int f) { return nl_bank(nl_par ^ 1) + spec_elems() * f; }
  double* work(int k) { return d_work + spec_elems() * k; }
  double* grid(int g) { return d_grid + grid_elems() * g; }
};

namespace gd {
// Brackets the launches of its lifetime with CUDA events when profiling is on.
struct ProfScope {
  gd_handle* h;
  const char* name;
  cudaEvent_t a = nullptr;
  ProfScope(gd_handle* h_, const char* n) : h(h_), name(n) {
    if (h->profiling) {
      cudaEventCreate(&a);
      cudaEventRecord(a, h->stream);
    }
  }
  ~ProfScope() {
    if (h->profiling && a) {
      cudaEvent_t b;
      cudaEventCreate(&b);
      cudaEventRecord(b, h->stream);
      h->prof_pending.push_back({name, a, b});
    }
  }
};

inline int set_error(gd_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}
}  // namespace gd

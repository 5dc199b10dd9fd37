// gd_api.cu -- the C ABI (include/gdb200.h): handle lifetime, device-resident
// model state, the step sequence of step_once! and its CUDA-graph replay.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gd_handle.cuh"
#include "gd_internal.cuh"
#include "gd_mixed.cuh"
#include "gd_ozaki.cuh"

using namespace gd;


namespace {

// State fields of the configuration: the five of the reference's step, and
// composition when configured.
int nfields(const gd_handle* h) { return h->c.composition ? NFIELD : NFIELD - 1; }

int fail(gd_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(h, GD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int dalloc(gd_handle* h, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
  if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(q);
  h->bytes += n * sizeof(T);
  *p = static_cast<T*>(q);
  return GD_OK;
}

#define AL(ptr, n)                             \
  do {                                         \
    int s_ = dalloc(h, &(ptr), (size_t)(n));   \
    if (s_) return s_;                         \
  } while (0)

// Entry points built for one spherical shell per handle refuse a segmented
// handle, and those whose operators divide by r, a ball.
static int refuse_layout(gd_handle* h, const char* what) {
  return fail(h, GD_ERR_UNSUPPORTED, std::string(what) + " is not built for a " +
                                         (h->d.ball ? "ball" : "segmented") + " handle");
}

int check_launch(gd_handle* h, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return GD_OK;
}

int build_implicit(gd_handle* h) {
  const Dims& d = h->d;
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  // one set of operators per segment length (variant), on its own radial nodes
  for (size_t v = 0; v < h->var_n.size(); ++v)
    launch_build_lu(h->stream, h->var_n[v], d.kl, d.L, h->d_d1 + h->var_band[v], h->d_d2 + h->var_band[v],
                    h->d_rinv + h->var_rep[v], h->d_rinv2 + h->var_rep[v], h->d_nu, h->c.dt, h->c.implicit_theta,
                    h->c.bc_mode == 2, h->d_lin + h->var_op[v], h->d_lu + h->var_op[v], h->d_flag,
                    h->c.composition ? 4 : 3);
  int s = check_launch(h, "build_lu");
  if (s) return s;
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag) return fail(h, GD_ERR_SINGULAR, "zero pivot in a banded LU factorisation");
  // bc_mode 2: the factors for prescribed fluxes, per segment length at the
  // same offsets as the main factors (the linear operator is the same; a
  // scratch block takes the build's copy).  A zero pivot there only disables
  // flux rows (gd_set_scalar_bc_types refuses them)
  if (h->d_lu_flux) {
    CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
    for (int fv = 1; fv <= 3; ++fv)
      for (size_t v = 0; v < h->var_n.size(); ++v)
        launch_build_lu(h->stream, h->var_n[v], d.kl, d.L, h->d_d1 + h->var_band[v], h->d_d2 + h->var_band[v],
                        h->d_rinv + h->var_rep[v], h->d_rinv2 + h->var_rep[v], h->d_nu, h->c.dt,
                        h->c.implicit_theta, 1 | (fv << 1), h->d_lu_flux + 3 * h->lu_flux_stride + h->var_op[v],
                        h->d_lu_flux + (size_t)(fv - 1) * h->lu_flux_stride + h->var_op[v], h->d_flag,
                        h->c.composition ? 4 : 3);
    s = check_launch(h, "build_lu (flux rows)");
    if (s) return s;
    CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->flux_rows_ok = flag == 0;
    bool any_flux = false;
    for (int t : h->bctype) any_flux |= t == GD_BC_FLUX;
    if (!h->flux_rows_ok && any_flux)
      return fail(h, GD_ERR_SINGULAR, "zero pivot in the factorisation with flux boundary rows");
  }
  return GD_OK;
}

// Tau functions of the flux boundary conditions on the radial nodes
// (_get_tau_cache, compute_inner_tau_function, compute_outer_tau_function,
// evaluate_tau_derivative_*, src/scalar_field_common.jl:590-790): Chebyshev
// T_{N-1} and T_N of x = 2 (r - ri) / (ro - ri) - 1, their analytic radial
// derivatives at the boundaries (n^2 sign(x)^(n+1) dx/dr where |x| = 1), the
// single-boundary combinations and their D1 derivatives at the boundary they
// serve.  Needs the radial nodes and D1 on the device.
int build_tau(gd_handle* h) {
  // one set per segment length (variant), on its own nodes and D1, copied to
  // every segment of that length
  const int KL = h->d.kl, NB = 2 * GD_MAX_KL + 1, nseg = h->d.nseg;
  std::vector<double> all(4 * (size_t)h->d.nr, 0.0), cons(6 * (size_t)nseg, 0.0);
  for (size_t v = 0; v < h->var_n.size(); ++v) {
    const int N = h->var_n[v];
    std::vector<double> r(N), d1((size_t)NB * N);
    CK(cudaMemcpyAsync(r.data(), h->d_r + h->var_rep[v], sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(d1.data(), h->d_d1 + h->var_band[v], sizeof(double) * NB * N, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const double ri = r[0], ro = r[N - 1];
    auto cheb = [&](int n, double rr) {
      double x = 2.0 * (rr - ri) / (ro - ri) - 1.0;
      x = x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x);
      return std::cos(n * std::acos(x));
    };
    auto dcheb = [&](int n, double rr) {
      const double x = 2.0 * (rr - ri) / (ro - ri) - 1.0;
      double dx;
      if (std::fabs(std::fabs(x) - 1.0) < 1e-12) {
        dx = (double)n * n * std::pow(x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0), n + 1);
      } else {
        const double th = std::acos(x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x));
        dx = n * std::sin(n * th) / std::sin(th);
      }
      return dx * (2.0 / (ro - ri));
    };
    std::vector<double> t(4 * (size_t)N);
    double* t1 = t.data();
    double* t2 = t1 + N;
    double* tin = t2 + N;
    double* tout = tin + N;
    for (int i = 0; i < N; ++i) { t1[i] = cheb(N - 1, r[i]); t2[i] = cheb(N, r[i]); }
    const double dt1i = dcheb(N - 1, ri), dt1o = dcheb(N - 1, ro);
    const double dt2i = dcheb(N, ri), dt2o = dcheb(N, ro);
    const double alpha = std::fabs(dt2o) > 1e-12 ? dt1o / dt2o : 0.0;
    const double beta = std::fabs(dt2i) > 1e-12 ? dt1i / dt2i : 0.0;
    for (int i = 0; i < N; ++i) { tin[i] = t1[i] - alpha * t2[i]; tout[i] = t1[i] - beta * t2[i]; }
    // rows 0 and N - 1 of D1 (entry (i, col) at d1[(i - col + KL) + NB col])
    double din = 0.0, dout = 0.0;
    for (int col = 0; col <= KL && col < N; ++col) din += d1[(size_t)(0 - col + KL) + (size_t)NB * col] * tin[col];
    for (int col = std::max(0, N - 1 - KL); col < N; ++col)
      dout += d1[(size_t)(N - 1 - col + KL) + (size_t)NB * col] * tout[col];
    for (int z = 0; z < nseg; ++z) {
      if (h->seg_var[z] != (int)v) continue;
      std::copy(t.begin(), t.end(), all.begin() + 4 * (size_t)h->seg_base[z]);
      const double k[6] = {dt1i, dt1o, dt2i, dt2o, din, dout};
      std::copy(k, k + 6, cons.begin() + 6 * (size_t)z);
    }
  }
  CK(cudaMemcpyAsync(h->d_tau, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_tauc, cons.data(), sizeof(double) * cons.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->tau.tau = h->d_tau;
  h->tau.consts = h->d_tauc;
  return GD_OK;
}

}  // namespace

// Boundary conditions of temperature (F_TEMP) or composition (F_COMP) for the
// handle's mode range.
void gd::scalar_bc(gd_handle* h, int field) {
  const bool comp = field == F_COMP;
  const size_t NL = h->d.nlm;
  ProfScope p(h, comp ? "composition_bc" : "temperature_bc");
  launch_scalar_bc(h->stream, h->d, h->d_lof, comp ? h->d_cbvals : h->d_bvals, h->d_bctype + (comp ? 2 * NL : 0),
                   h->d_d1, h->tau, h->field(field), h->c.bc_mode == 2);
}

// ball_physical_to_spectral! / ball_vector_analysis! (src/Ball/Ball.jl:214-245)
// as called from compute_temperature_nonlinear! (src/thermal.jl:177-178),
// compute_composition_nonlinear! (src/compositional.jl:245-246) and
// compute_induction_term! (src/magnetic.jl:362-364): regularity on the analysed
// nonlinear terms.  The induction's spectral curl scales each (l, m, r) alone,
// so zeroing after it equals zeroing before it.
void gd::regular_nl(gd_handle* h, int field, int nf) {
  if (!h->d.ball) return;
  ProfScope p(h, "ball_regularity");
  launch_regularity(h->stream, h->d, h->d_lof, h->nlf(field), nf, h->spec_elems());
}

namespace {

int setup(gd_handle* h) {
  const gd_config& c = h->c;
  Dims& d = h->d;
  d.L = c.lmax; d.M = c.mmax; d.nlat = c.nlat; d.nlon = c.nlon; d.nr = c.nr; d.kl = c.kl;
  d.nth = c.nlat / 2;
  for (int l = 0; l <= d.L; ++l)
    for (int m = 0; m <= (l < d.M ? l : d.M); ++m) { h->lv.push_back(l); h->mv.push_back(m); }
  d.nlm = (int)h->lv.size();
  d.jlo = 0;
  d.jhi = d.nlm;
  d.nseg = c.segments > 1 ? c.segments : 1;
  // segment lengths (equal unless listed) and their operator variants
  h->seg_n.assign(d.nseg, d.nr / d.nseg);
  if (d.nseg > 1 && c.segment_nr)
    for (int z = 0; z < d.nseg; ++z) h->seg_n[z] = c.segment_nr[z];
  h->seg_base.assign(d.nseg, 0);
  h->seg_var.assign(d.nseg, 0);
  h->var_n.clear(); h->var_rep.clear(); h->var_band.clear(); h->var_op.clear();
  const long nbw_h = 2 * GD_MAX_KL + 1;
  for (int z = 0, b = 0; z < d.nseg; b += h->seg_n[z], ++z) {
    h->seg_base[z] = b;
    int v = 0;
    while (v < (int)h->var_n.size() && h->var_n[v] != h->seg_n[z]) ++v;
    if (v == (int)h->var_n.size()) {
      const long band = h->var_n.empty() ? 0 : h->var_band.back() + nbw_h * h->var_n.back();
      const long op = h->var_n.empty() ? 0 : h->var_op.back() + 4 * nbw_h * h->var_n.back() * (c.lmax + 1);
      h->var_n.push_back(h->seg_n[z]);
      h->var_rep.push_back(b);
      h->var_band.push_back(band);
      h->var_op.push_back(op);
    }
    h->seg_var[z] = v;
  }
  d.nrs = *std::max_element(h->seg_n.begin(), h->seg_n.end());
  d.seg_info = nullptr;
  d.var_off = nullptr;
  d.rfs = nullptr;
  d.rfs32 = nullptr;
  d.ball = c.geometry == GD_GEOM_BALL;
  h->moff.assign(d.M + 2, 0);
  for (int m = 0; m <= d.M; ++m) h->moff[m + 1] = h->moff[m] + (d.L - m + 1);
  h->perm.resize(d.nlm);
  h->lof.resize(d.nlm);
  h->mof.resize(d.nlm);
  for (int q = 0; q < d.nlm; ++q) {
    const int j = h->moff[h->mv[q]] + (h->lv[q] - h->mv[q]);
    h->perm[q] = j;
    h->lof[j] = h->lv[q];
    h->mof[j] = h->mv[q];
  }
  h->plan = make_fft_plan(d.nlon);
  if (h->plan.nstage < 0) return fail(h, GD_ERR_CONFIG, "nlon must factor into 2, 3 and 5");

  CK(cudaSetDevice(h->device));
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  const size_t NL = d.nlm, NT = d.nth, NR = d.nr, nbw = 2 * d.kl + 1;
  AL(h->d_moff, d.M + 2); AL(h->d_lof, NL); AL(h->d_mof, NL); AL(h->d_perm, NL); AL(h->d_flag, 4);
  AL(h->d_x, d.nlat); AL(h->d_w, d.nlat); AL(h->d_th, d.nlat); AL(h->d_sth, d.nlat);
  AL(h->d_cth, d.nlat); AL(h->d_sthc, d.nlat);
  AL(h->d_r, NR); AL(h->d_rinv, NR); AL(h->d_rinv2, NR); AL(h->d_nu, 4);
  AL(h->d_P, NL * NT); AL(h->d_dP, NL * NT); AL(h->d_Q, NL * NT);
  AL(h->d_d1, nbw * NR); AL(h->d_d2, nbw * NR);
  AL(h->d_lin, 4 * NR * nbw * (d.L + 1)); AL(h->d_lu, 4 * NR * nbw * (d.L + 1));
  if (c.bc_mode == 2) {
    // three flux-row variants of the factors (each laid out like d_lu: one
    // operator set per segment length at var_op), and a block that takes the
    // build's copy of the linear operator
    h->lu_flux_stride = h->var_op.back() + (size_t)4 * h->var_n.back() * nbw * (d.L + 1);
    AL(h->d_lu_flux, 4 * h->lu_flux_stride);
  }
  AL(h->d_tw, 2 * (size_t)d.nlon); AL(h->d_twf, 2 * (size_t)d.nlon);
  AL(h->d_state, NFIELD * h->spec_elems()); AL(h->d_nl, NFIELD * h->spec_elems());
  AL(h->d_prev, NFIELD * h->spec_elems());
  AL(h->d_work, NWORK * h->spec_elems());
  AL(h->d_bvals, 2 * NL); AL(h->d_sources, NR);
  AL(h->d_cbvals, 2 * NL); AL(h->d_csources, NR); AL(h->d_bctype, 4 * NL); AL(h->d_tau, 4 * NR);
  AL(h->d_tauc, 6 * (size_t)d.nseg);
  AL(h->d_grid, NGRID * h->grid_elems());
  AL(h->d_F, (size_t)4 * NR * (d.M + 1) * d.nlat);
  AL(h->d_epart, 2 * GD_ENERGY_BLOCKS * d.nseg); AL(h->d_eout, 2 * d.nseg);

  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(h->d_moff, h->moff.data(), sizeof(int) * (d.M + 2), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_lof, h->lof.data(), sizeof(int) * NL, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_mof, h->mof.data(), sizeof(int) * NL, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_perm, h->perm.data(), sizeof(int) * NL, cudaMemcpyHostToDevice, s));
  // Radial nodes r_n = ri + (1 + cos(pi (N - n) / (N - 1))) / 2 (src/fields.jl:108-131),
  // with the powers r^-1, r^-2 of its columns 3 and 2.
  std::vector<double> r(NR), ri(NR), ri2(NR);
  const double rin = c.rratio / (1.0 - c.rratio);
  const double kPi = 3.14159265358979323846;
  // every segment its own nodes for its level count.  Ball: the same cosine
  // nodes on [0, R] (create_ball_radial_domain, src/Ball/Ball.jl:34-71), r_1 = 0
  for (int z = 0; z < d.nseg; ++z) {
    const int NS = h->seg_n[z], b = h->seg_base[z];
    for (int n = 1; n <= NS; ++n) {
      const double x = 0.5 * (1.0 + std::cos(kPi * (double)(NS - n) / (double)(NS - 1)));
      r[b + n - 1] = d.ball ? (c.r_outer != 1.0 ? x * c.r_outer : x) : x + rin;
    }
  }
  if (h->var_n.size() > 1) {
    // several segment lengths: the kernels look each segment's shells and operators up
    std::vector<int> info(3 * (size_t)d.nseg);
    std::vector<long> voff(2 * h->var_n.size());
    for (int z = 0; z < d.nseg; ++z) {
      info[3 * z] = h->seg_base[z];
      info[3 * z + 1] = h->seg_n[z];
      info[3 * z + 2] = h->seg_var[z];
    }
    for (size_t v = 0; v < h->var_n.size(); ++v) {
      voff[2 * v] = h->var_band[v];
      voff[2 * v + 1] = h->var_op[v];
    }
    AL(h->d_seg_info, info.size());
    AL(h->d_var_off, voff.size());
    CK(cudaMemcpyAsync(h->d_seg_info, info.data(), sizeof(int) * info.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->d_var_off, voff.data(), sizeof(long) * voff.size(), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    d.seg_info = h->d_seg_info;
    d.var_off = h->d_var_off;
  }
  for (int n = 0; n < d.nr; ++n) { ri[n] = std::pow(r[n], -1.0); ri2[n] = std::pow(r[n], -2.0); }
  CK(cudaMemcpyAsync(h->d_r, r.data(), sizeof(double) * NR, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_rinv, ri.data(), sizeof(double) * NR, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_rinv2, ri2.data(), sizeof(double) * NR, cudaMemcpyHostToDevice, s));
  // Diffusivities: velocity Pm, magnetic 1, temperature Pm/Pr, composition
  // Pm/Sc (src/simulation.jl:228-235).
  const double nu[4] = {c.magnetic_prandtl, 1.0, c.magnetic_prandtl / c.prandtl,
                        c.composition ? c.magnetic_prandtl / c.schmidt : 0.0};
  CK(cudaMemcpyAsync(h->d_nu, nu, sizeof(nu), cudaMemcpyHostToDevice, s));
  std::vector<double> tw;
  make_twiddles(d.nlon, tw);
  std::vector<float> twf(tw.size());
  for (size_t i = 0; i < tw.size(); ++i) twf[i] = (float)tw[i];
  CK(cudaMemcpyAsync(h->d_tw, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->d_twf, twf.data(), sizeof(float) * twf.size(), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // host vectors above go out of scope

  launch_gauss(s, d.nlat, h->d_x, h->d_w, h->d_th, h->d_sth);
  launch_tables(s, d, h->d_moff, h->d_x, h->d_sth, h->d_P, h->d_dP, h->d_Q);
  for (size_t v = 0; v < h->var_n.size(); ++v)
    launch_fd_weights(s, h->var_n[v], d.kl, c.fd_mode, h->d_r + h->var_rep[v], h->d_d1 + h->var_band[v],
                      h->d_d2 + h->var_band[v]);
  int st = check_launch(h, "set-up kernels");
  if (st) return st;
  // Coriolis factors sin/cos of the colatitude grid (src/velocity.jl:278-282).
  {
    std::vector<double> th(d.nlat), cth(d.nlat), sth(d.nlat);
    CK(cudaMemcpyAsync(th.data(), h->d_th, sizeof(double) * d.nlat, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < d.nlat; ++i) { sth[i] = std::sin(th[i]); cth[i] = std::cos(th[i]); }
    CK(cudaMemcpyAsync(h->d_sthc, sth.data(), sizeof(double) * d.nlat, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->d_cth, cth.data(), sizeof(double) * d.nlat, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
  }
  CK(cudaMemsetAsync(h->d_state, 0, sizeof(double) * NFIELD * h->spec_elems(), s));
  CK(cudaMemsetAsync(h->d_nl, 0, sizeof(double) * NFIELD * h->spec_elems(), s));
  CK(cudaMemsetAsync(h->d_prev, 0, sizeof(double) * NFIELD * h->spec_elems(), s));
  CK(cudaMemsetAsync(h->d_work, 0, sizeof(double) * NWORK * h->spec_elems(), s));
  CK(cudaMemsetAsync(h->d_bvals, 0, sizeof(double) * 2 * NL, s));
  CK(cudaMemsetAsync(h->d_sources, 0, sizeof(double) * NR, s));
  CK(cudaMemsetAsync(h->d_cbvals, 0, sizeof(double) * 2 * NL, s));
  CK(cudaMemsetAsync(h->d_csources, 0, sizeof(double) * NR, s));
  {
    // boundary types: temperature fixed values, composition no-flux
    // (create_shtns_temperature_field / create_shtns_composition_field
    // defaults); with the boundary-row operator (bc_mode 2) composition has
    // fixed values too, those of its rows
    std::vector<int> bt(4 * NL);
    for (size_t q = 0; q < 2 * NL; ++q) bt[q] = GD_BC_VALUE;
    for (size_t q = 2 * NL; q < 4 * NL; ++q) bt[q] = c.bc_mode == 2 ? GD_BC_VALUE : GD_BC_FLUX;
    CK(cudaMemcpyAsync(h->d_bctype, bt.data(), sizeof(int) * bt.size(), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    h->bctype = bt;
  }
  {
    int st = build_tau(h);
    if (st) return st;
  }
  CK(cudaMemsetAsync(h->d_grid, 0, sizeof(double) * NGRID * h->grid_elems(), s));
  return build_implicit(h);
}

// ---- transform building blocks on device buffers (native layouts) ----
int synth_scalar(gd_handle* h, const double* const* coef, int nf, double* grid_out) {
  SynthArgs a{};
  a.table0 = h->d_P;
  for (int i = 0; i < nf; ++i) a.coef[i] = coef[i];
  a.nf = nf;
  a.out = h->d_F;
  { ProfScope p(h, "legendre_synth_scalar_fp64"); launch_synth_fp64(h->stream, h->d, h->d_moff, a, false); }
  { ProfScope p(h, "fft_synth_fp64"); launch_fft_synth<double>(h->stream, h->d, h->plan, h->d_tw, h->d_F, grid_out, nf, h->grid_elems()); }
  return check_launch(h, "scalar synthesis");
}

int synth_vector(gd_handle* h, const double* tor, const double* pol, double* grid_out /* 2 comps */) {
  SynthArgs a{};
  a.table0 = h->d_dP;
  a.table1 = h->d_Q;
  a.coef[0] = pol;
  a.coef[1] = tor;
  a.nf = 1;
  a.out = h->d_F;
  { ProfScope p(h, "legendre_synth_vector_fp64"); launch_synth_fp64(h->stream, h->d, h->d_moff, a, true); }
  { ProfScope p(h, "fft_synth_fp64"); launch_fft_synth<double>(h->stream, h->d, h->plan, h->d_tw, h->d_F, grid_out, 2, h->grid_elems()); }
  return check_launch(h, "vector synthesis");
}

int analysis_scalar(gd_handle* h, const double* grid_in, int nf, double* const* out) {
  { ProfScope p(h, "fft_analysis_fp64"); launch_fft_analysis<double>(h->stream, h->d, h->plan, h->d_tw, grid_in, h->grid_elems(), h->d_w, h->d_F, nf); }
  AnalysisArgs a{};
  a.table0 = h->d_P;
  a.in = h->d_F;
  for (int i = 0; i < nf; ++i) a.out[i] = out[i];
  a.nf = nf;
  a.epi = EPI_SCALAR;
  { ProfScope p(h, "legendre_analysis_scalar_fp64"); launch_analysis_fp64(h->stream, h->d, h->d_moff, a); }
  return check_launch(h, "scalar analysis");
}

int analysis_vector(gd_handle* h, const double* grid_in /* 2 comps */, double* out_tor, double* out_pol, int epi) {
  { ProfScope p(h, "fft_analysis_fp64"); launch_fft_analysis<double>(h->stream, h->d, h->plan, h->d_tw, grid_in, h->grid_elems(), h->d_w, h->d_F, 2); }
  AnalysisArgs a{};
  a.table0 = h->d_dP;
  a.table1 = h->d_Q;
  a.in = h->d_F;
  a.out[0] = out_tor;
  a.out[1] = out_pol;
  a.nf = 1;
  a.epi = epi;
  { ProfScope p(h, "legendre_analysis_vector_fp64"); launch_analysis_fp64(h->stream, h->d, h->d_moff, a); }
  return check_launch(h, "vector analysis");
}

// ---- the physics sequence (FP64) ----
int temperature_nl_fp64(gd_handle* h) {
  const Dims& d = h->d;
  if (!h->ext_derivs) {
    ProfScope p(h, "spectral_gradients");
    launch_gradients(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_TEMP), h->work(0), h->work(1),
                     h->work(2));
  }
  const double* coef[4] = {h->field(F_TEMP), h->work(0), h->work(1), h->work(2)};
  int s = synth_scalar(h, coef, 4, h->grid(GD_GRID_T));
  if (s) return s;
  { ProfScope pa(h, "nl_temperature_fp64");
    launch_temperature_advection<double>(h->stream, d, h->grid(GD_GRID_U_TH), h->grid(GD_GRID_U_PH),
                                         h->grid(GD_GRID_GTH), h->grid(GD_GRID_GPH), h->grid(GD_GRID_GR),
                                         h->d_sources, h->grid(GD_GRID_TADV)); }
  double* out[1] = {h->nlf(F_TEMP)};
  s = analysis_scalar(h, h->grid(GD_GRID_TADV), 1, out);
  if (s) return s;
  regular_nl(h, F_TEMP, 1);
  if (!h->ext_derivs) scalar_bc(h, F_TEMP);
  return check_launch(h, "temperature nonlinear");
}

// compute_composition_nonlinear! (src/compositional.jl:219-259): gradient of C
// (compute_all_gradients_spectral!, into work 8-10 unless received), batched
// synthesis of C and its gradient, -u.grad C + S_C(r) with this step's velocity
// grids (step_once! runs it after the velocity phase), analysis, then the
// boundary conditions (apply_composition_boundary_conditions_spectral!: fixed
// values and the tau flux correction).  The extra synthesis of C at :229 only
// rewrites the grid the batched one writes again.
int composition_nl_fp64(gd_handle* h) {
  const Dims& d = h->d;
  if (!h->ext_derivs) {
    ProfScope p(h, "spectral_gradients");
    launch_gradients(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_COMP), h->work(8), h->work(9),
                     h->work(10));
  }
  const double* coef[4] = {h->field(F_COMP), h->work(8), h->work(9), h->work(10)};
  int s = synth_scalar(h, coef, 4, h->grid(GD_GRID_C));
  if (s) return s;
  { ProfScope pa(h, "nl_composition_fp64");
    launch_temperature_advection<double>(h->stream, d, h->grid(GD_GRID_U_TH), h->grid(GD_GRID_U_PH),
                                         h->grid(GD_GRID_CGTH), h->grid(GD_GRID_CGPH), h->grid(GD_GRID_CGR),
                                         h->d_csources, h->grid(GD_GRID_CADV)); }
  double* out[1] = {h->nlf(F_COMP)};
  s = analysis_scalar(h, h->grid(GD_GRID_CADV), 1, out);
  if (s) return s;
  regular_nl(h, F_COMP, 1);
  if (!h->ext_derivs) scalar_bc(h, F_COMP);
  return check_launch(h, "composition nonlinear");
}

int velocity_nl_fp64(gd_handle* h) {
  const Dims& d = h->d;
  int s = synth_vector(h, h->field(F_UTOR), h->field(F_UPOL), h->grid(GD_GRID_U_TH));
  if (s) return s;
  if (!h->ext_derivs) {
    ProfScope p(h, "spectral_curl");
    launch_curl(h->stream, d, h->d_lof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_UTOR), h->field(F_UPOL),
                h->work(3), h->work(4));
  }
  s = synth_vector(h, h->work(3), h->work(4), h->grid(GD_GRID_W_TH));
  if (s) return s;
  const double rf = h->c.magnetic_prandtl / h->c.ekman;
  { ProfScope p(h, "nl_velocity_fp64");
  launch_velocity_nl<double>(h->stream, d, h->d_cth, h->d_sthc, rf, rf, h->c.magnetic, h->grid(GD_GRID_U_TH),
                             h->grid(GD_GRID_U_PH), h->grid(GD_GRID_W_TH), h->grid(GD_GRID_W_PH),
                             h->grid(GD_GRID_J_TH), h->grid(GD_GRID_J_PH), h->grid(GD_GRID_B_TH),
                             h->grid(GD_GRID_B_PH), h->grid(GD_GRID_VADV_TH), h->grid(GD_GRID_VADV_PH)); }
  return analysis_vector(h, h->grid(GD_GRID_VADV_TH), h->nlf(F_UTOR), h->nlf(F_UPOL), EPI_VECTOR);
}

int magnetic_nl_fp64(gd_handle* h) {
  const Dims& d = h->d;
  int s = synth_vector(h, h->field(F_BTOR), h->field(F_BPOL), h->grid(GD_GRID_B_TH));
  if (s) return s;
  if (!h->ext_derivs) {
    ProfScope p(h, "spectral_curl");
    launch_curl(h->stream, d, h->d_lof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_BTOR), h->field(F_BPOL),
                h->work(5), h->work(6));
  }
  s = synth_vector(h, h->work(5), h->work(6), h->grid(GD_GRID_J_TH));
  if (s) return s;
  { ProfScope p(h, "nl_induction_fp64");
    launch_induction<double>(h->stream, d, h->grid(GD_GRID_U_TH), h->grid(GD_GRID_U_PH), h->grid(GD_GRID_B_TH),
                             h->grid(GD_GRID_B_PH), h->grid(GD_GRID_IND_TH), h->grid(GD_GRID_IND_PH)); }
  s = analysis_vector(h, h->grid(GD_GRID_IND_TH), h->nlf(F_BTOR), h->nlf(F_BPOL), EPI_CURL_INDUCTION);
  if (s) return s;
  regular_nl(h, F_BTOR, 2);
  return check_launch(h, "magnetic nonlinear");
}

ExpApply exp_apply_args(gd_handle* h, const Cnab2Args& a) {
  ExpApply e{};
  e.nfield = a.nfield;
  for (int i = 0; i < a.nfield; ++i) e.kind[i] = a.kind[i];
  e.top_block = e.bot_block = -1;
  e.bot_scale = 1.0;
  e.dt = h->c.dt;
  return e;
}

int temperature_nl(gd_handle* h);
int velocity_nl(gd_handle* h);
int magnetic_nl(gd_handle* h);
int composition_nl(gd_handle* h);
int step_slots(const gd_handle* h, int* order, int* kinds);

// compute_all_nonlinear_terms! (src/simulation.jl:800-813): velocity, magnetic,
// temperature, composition, in that order (the carried grids make the order
// matter).
int all_nonlinear(gd_handle* h) {
  int s = velocity_nl(h);
  if (s) return s;
  if (h->c.magnetic) {
    s = magnetic_nl(h);
    if (s) return s;
  }
  s = temperature_nl(h);
  if (s || !h->c.composition) return s;
  return composition_nl(h);
}

// erk2_integrate_full_step! (src/simulation.jl:1054-1149) after the step's
// nonlinear terms N^n (bank nl_par): erk2_prepare_field! (linear = E u,
// k1 = phi1 N^n, stage = E_h u + dt/2 phi1_h N^n written over u), the
// nonlinear terms of the stage into the other bank, erk2_finalize_field!
// (u = linear + dt (k1 + phi2 (N_stage - N^n))), and the closing evaluation of
// the nonlinear terms at the new state (into bank nl_par), whose only lasting
// effect is on the physical grids the next step carries.
int erk2_launch(gd_handle* h, const Cnab2Args& a) {
  const size_t se = h->spec_elems();
  ExpApply e = exp_apply_args(h, a);
  int order[6], kinds[6];
  step_slots(h, order, kinds);
  double* lin[6];
  double* k1[6];
  for (int i = 0; i < a.nfield; ++i) {
    lin[i] = h->d_erk2 + (size_t)order[i] * se;
    k1[i] = h->d_erk2 + (size_t)(NFIELD + order[i]) * se;
  }
  {
    ProfScope p(h, "erk2_prepare");
    ExpApply x = e;  // linear = E u
    for (int i = 0; i < a.nfield; ++i) { x.top[i] = a.u[i]; x.out[i] = lin[i]; }
    x.top_block = 0;
    launch_exp_apply(h->stream, h->d, h->d_moff, h->d_etd, x);
    x = e;           // k1 = phi1 N^n
    for (int i = 0; i < a.nfield; ++i) { x.bot_a[i] = a.nl[i]; x.out[i] = k1[i]; }
    x.bot_block = 1;
    launch_exp_apply(h->stream, h->d, h->d_moff, h->d_etd, x);
    x = e;           // stage = E_h u + dt/2 phi1_h N^n, over u
    for (int i = 0; i < a.nfield; ++i) { x.top[i] = a.u[i]; x.bot_a[i] = a.nl[i]; x.out[i] = a.u[i]; }
    x.top_block = 3;
    x.bot_block = 4;
    x.bot_scale = 0.5 * h->c.dt;
    launch_exp_apply(h->stream, h->d, h->d_moff, h->d_etd, x);
  }
  int s = check_launch(h, "erk2 prepare");
  if (s) return s;
  h->nl_par ^= 1;  // the stage's terms go to the other bank
  s = all_nonlinear(h);
  h->nl_par ^= 1;
  if (s) return s;
  {
    ProfScope p(h, "erk2_finalize");
    ExpApply x = e;  // u = linear + dt (k1 + phi2 (N_stage - N^n))
    for (int i = 0; i < a.nfield; ++i) {
      x.bot_a[i] = h->nl_bank(h->nl_par ^ 1) + (size_t)order[i] * se;
      x.bot_b[i] = a.nl[i];
      x.out[i] = a.u[i];
      x.lin[i] = lin[i];
      x.k1[i] = k1[i];
    }
    x.bot_block = 2;
    x.bot_mode = 2;
    x.epilogue = 1;
    x.clamp_rows = a.clamp_rows;
    launch_exp_apply(h->stream, h->d, h->d_moff, h->d_etd, x);
  }
  s = check_launch(h, "erk2 finalize");
  if (s) return s;
  return all_nonlinear(h);
}

// The implicit slots of a step: temperature, velocity, magnetic field (when
// evolved), composition (when configured); their fields and diffusivity kinds.
int step_slots(const gd_handle* h, int* order, int* kinds) {
  int n = 0;
  const int f[6] = {F_TEMP, F_UTOR, F_UPOL, F_BTOR, F_BPOL, F_COMP};
  const int k[6] = {2, 0, 0, 1, 1, 3};
  for (int i = 0; i < 6; ++i) {
    if ((f[i] == F_BTOR || f[i] == F_BPOL) && !h->c.magnetic) continue;
    if (f[i] == F_COMP && !h->c.composition) continue;
    order[n] = f[i];
    kinds[n] = k[i];
    ++n;
  }
  return n;
}

int implicit_launch(gd_handle* h, int boot) {
  Cnab2Args a{};
  int order[6], kinds[6];
  a.nfield = step_slots(h, order, kinds);
  for (int i = 0; i < a.nfield; ++i) {
    a.u[i] = h->field(order[i]);
    a.nl[i] = h->nlf(order[i]);
    a.prev[i] = h->prevf(order[i]);
    a.kind[i] = kinds[i];
  }
  a.boot = boot;
  a.clamp_rows = h->c.bc_mode == 1;
  a.bc_rows = h->c.bc_mode == 2;
  // Dirichlet rows of bc_mode 2: the temperature's and the composition's
  // boundary values (or fluxes, by their boundary types), zero for the
  // velocity and magnetic potentials
  const size_t NLm = h->d.nlm;
  for (int i = 0; i < a.nfield; ++i) {
    a.rowvals[i] = order[i] == F_TEMP ? h->d_bvals : order[i] == F_COMP ? h->d_cbvals : nullptr;
    a.rowtypes[i] = order[i] == F_TEMP ? h->d_bctype : order[i] == F_COMP ? h->d_bctype + 2 * NLm : nullptr;
  }
  a.lu_flux = h->d_lu_flux;
  a.lu_flux_stride = h->lu_flux_stride;
  a.inv_dt = 1.0 / h->c.dt;
  a.lin_weight = 1.0 - h->c.implicit_theta;
  a.dt = h->c.dt;
  if (h->scheme == GD_SCHEME_EAB2) {
    // eab2_update! takes no AB1 start: N_prev is the other bank (zeros before
    // the first step, as prev_nonlinear is)
    ExpApply e = exp_apply_args(h, a);
    for (int i = 0; i < a.nfield; ++i) {
      e.top[i] = a.u[i];
      e.bot_a[i] = a.nl[i];
      e.bot_b[i] = a.prev[i];
      e.out[i] = a.u[i];
    }
    e.top_block = 0;
    e.bot_block = 1;
    e.bot_mode = 1;
    e.bot_scale = h->c.dt;
    e.clamp_rows = a.clamp_rows;
    { ProfScope p(h, "eab2_update"); launch_exp_apply(h->stream, h->d, h->d_moff, h->d_etd, e); }
    return check_launch(h, "eab2");
  }
  if (h->scheme == GD_SCHEME_ERK2) return erk2_launch(h, a);
  { ProfScope p(h, "cnab2_solve"); launch_cnab2(h->stream, h->d, h->d_lof, h->d_d1, h->d_d2, h->d_rinv, h->d_rinv2, h->d_nu, h->d_lu, a); }
  return check_launch(h, "cnab2");
}

// The EAB2 exponential cache for the handle's dt (create_etd_cache,
// src/timestep.jl:37-70), from the L_l bands of build_implicit.
int build_etd(gd_handle* h) {
  const Dims& d = h->d;
  const int nkind = h->c.composition ? 4 : 3;
  if (!h->d_etd) AL(h->d_etd, etd_table_doubles(d, nkind));
  double* scratch = nullptr;
  CK(cudaMalloc(&scratch, etd_scratch_doubles(d, nkind) * sizeof(double)));
  cudaError_t e = cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) {
    launch_etd_build(h->stream, d, h->d_lin, h->c.dt, scratch, h->d_etd, h->d_flag, nkind);
    e = cudaGetLastError();
  }
  int flag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(scratch);
  if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string("exponential cache: ") + cudaGetErrorString(e));
  if (flag) return fail(h, GD_ERR_NONFINITE, "exponential cache: non-finite operator");
  return GD_OK;
}

int temperature_nl(gd_handle* h) {
  return h->precision == GD_PREC_MIXED ? mixed_temperature_nl(h) : temperature_nl_fp64(h);
}
int velocity_nl(gd_handle* h) {
  return h->precision == GD_PREC_MIXED ? mixed_velocity_nl(h) : velocity_nl_fp64(h);
}
int magnetic_nl(gd_handle* h) {
  return h->precision == GD_PREC_MIXED ? mixed_magnetic_nl(h) : magnetic_nl_fp64(h);
}
int composition_nl(gd_handle* h) {
  return h->precision == GD_PREC_MIXED ? mixed_composition_nl(h) : composition_nl_fp64(h);
}

// step_once! (scripts/bench_timestepping.jl:6-18): temperature, velocity,
// magnetic field, composition, then the implicit step.
int step_sequence(gd_handle* h, int boot) {
  int s = temperature_nl(h);
  if (s) return s;
  s = velocity_nl(h);
  if (s) return s;
  if (h->c.magnetic) {
    s = magnetic_nl(h);
    if (s) return s;
  }
  if (h->c.composition) {
    s = composition_nl(h);
    if (s) return s;
  }
  return implicit_launch(h, boot);
}

void drop_graphs(gd_handle* h) {
  h->graph_gen++;
  for (int p = 0; p < 2; ++p)
    for (int i = 0; i < 2; ++i)
      if (h->gexec[p][i]) { cudaGraphExecDestroy(h->gexec[p][i]); h->gexec[p][i] = nullptr; }
}

// After a step's implicit solve: its nonlinear terms become the history of
// the next step (the reference's roll N_prev := N, src/simulation.jl:1312-1329).
void end_step(gd_handle* h) {
  h->last_nl_par = h->nl_par;
  h->nl_par ^= 1;
  h->step_count++;
}

// The step graph for the current nonlinear bank and bootstrap flag.
int ensure_graph(gd_handle* h, int boot) {
  cudaGraphExec_t& ge = h->gexec[h->nl_par][boot];
  if (ge) return GD_OK;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int s = step_sequence(h, boot);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (s) { if (g) cudaGraphDestroy(g); return s; }
  if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  {
    // kernel launches per step (gd_step_kernels): the graph's kernel nodes
    size_t n = 0;
    int k = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess && n > 0) {
      std::vector<cudaGraphNode_t> nodes(n);
      if (cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
        for (size_t i = 0; i < n; ++i) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
        }
    }
    h->graph_kernels[h->nl_par][boot] = k;
  }
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return GD_OK;
}

int stage_alloc(gd_handle* h) {
  if (h->d_stage_spec) return GD_OK;
  AL(h->d_stage_spec, 4 * h->spec_elems());
  AL(h->d_stage_spec2, 4 * h->spec_elems());
  AL(h->d_stage_grid, 4 * h->grid_elems());
  AL(h->d_stage_grid2, 4 * h->grid_elems());
  return GD_OK;
}

bool valid_config(const gd_config* c, std::string& why) {
  if (c->lmax < 1 || c->mmax < 0 || c->mmax > c->lmax) { why = "need 1 <= lmax, 0 <= mmax <= lmax"; return false; }
  if (c->nlat < 2 || (c->nlat & 1)) { why = "nlat must be even"; return false; }
  if (c->nlat <= c->lmax) { why = "nlat must exceed lmax (Gauss quadrature exactness)"; return false; }
  if (2 * c->mmax >= c->nlon) { why = "nlon must exceed 2 mmax"; return false; }
  if (c->nr < 3) { why = "nr must be at least 3"; return false; }
  if (c->kl != GD_MAX_KL) { why = "kl must be 4 (i_KL)"; return false; }
  if (!(c->dt > 0.0)) { why = "dt must be positive"; return false; }
  if (c->ekman == 0.0) { why = "Ekman number must be nonzero (src/velocity.jl:450-452)"; return false; }
  if (c->geometry != GD_GEOM_BALL && (c->rratio <= 0.0 || c->rratio >= 1.0)) {
    why = "rratio must lie in (0, 1)";
    return false;
  }
  if (c->bc_mode < 0 || c->bc_mode > 2) { why = "bc_mode must be 0, 1 or 2"; return false; }
  if (c->ab_mode < 0 || c->ab_mode > 1) { why = "ab_mode must be 0 or 1"; return false; }
  if (c->fd_mode < 0 || c->fd_mode > 1) { why = "fd_mode must be 0 or 1"; return false; }
  if (c->precision != GD_PREC_FP64 && c->precision != GD_PREC_MIXED) { why = "unknown precision"; return false; }
  if (c->composition != 0 && c->composition != 1) { why = "composition must be 0 or 1"; return false; }
  if (c->composition && !(c->schmidt > 0.0)) { why = "composition needs a positive Schmidt number"; return false; }
  if (c->segments < 0) { why = "segments must be >= 0"; return false; }
  if (c->segments > 1 && c->segment_nr) {
    long sum = 0;
    for (int z = 0; z < c->segments; ++z) {
      if (c->segment_nr[z] < 3) { why = "each segment needs at least 3 levels"; return false; }
      sum += c->segment_nr[z];
    }
    if (sum != c->nr) { why = "segment_nr must sum to nr"; return false; }
  } else {
    if (c->segments > 1 && c->nr % c->segments) { why = "segments must divide nr"; return false; }
    if (c->segments > 1 && c->nr / c->segments < 3) { why = "each segment needs at least 3 levels"; return false; }
  }
  if (c->segments > 1 && c->composition) { why = "segments carry no composition"; return false; }
  if (c->geometry != GD_GEOM_SHELL && c->geometry != GD_GEOM_BALL) { why = "geometry must be GD_GEOM_SHELL or GD_GEOM_BALL"; return false; }
  if (c->geometry == GD_GEOM_BALL) {
    if (!(c->r_outer > 0.0)) { why = "r_outer must be > 0 for ball geometry"; return false; }
    if (c->bc_mode != 2) {
      why = "ball geometry needs bc_mode 2: the literal operator holds 1/r and 1/r^2 at r = 0";
      return false;
    }
  }
  return true;
}

}  // namespace

// ============================================================================
extern "C" {

int gd_create(const gd_config* cfg, int device, gd_handle** out) {
  if (!cfg || !out) return GD_ERR_ARG;
  *out = nullptr;
  std::string why;
  if (!valid_config(cfg, why)) {
    fprintf(stderr, "gd_create: %s\n", why.c_str());
    return GD_ERR_CONFIG;
  }
  gd_handle* h = new gd_handle();
  h->c = *cfg;
  h->device = device;
  int s = setup(h);
  h->c.segment_nr = nullptr;  // read by the set-up only; the lengths live in seg_n
  if (s == GD_OK && cfg->precision == GD_PREC_MIXED) s = gd_set_precision(h, GD_PREC_MIXED);
  if (s != GD_OK) {
    fprintf(stderr, "gd_create: %s\n", h->err.c_str());
    gd_destroy(h);
    return s;
  }
  *out = h;
  return GD_OK;
}

int gd_destroy(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graphs(h);
  if (h->mixed) mixed_destroy(h);
  for (void* p : h->t_snaps) cudaFree(p);
  if (h->t_final) cudaFree(h->t_final);
  for (void* p : h->allocs) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return GD_OK;
}

const char* gd_last_error(const gd_handle* h) { return h ? h->err.c_str() : "null handle"; }

int gd_info(const gd_handle* h, int* nlm, size_t* device_bytes) {
  if (!h) return GD_ERR_ARG;
  if (nlm) *nlm = h->d.nlm;
  if (device_bytes) *device_bytes = h->bytes + (h->mixed ? mixed_bytes(h) : 0);
  return GD_OK;
}

int gd_grid(gd_handle* h, double* theta, double* weights, double* r) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  if (theta) CK(cudaMemcpyAsync(theta, h->d_th, sizeof(double) * h->d.nlat, cudaMemcpyDeviceToHost, h->stream));
  if (weights) CK(cudaMemcpyAsync(weights, h->d_w, sizeof(double) * h->d.nlat, cudaMemcpyDeviceToHost, h->stream));
  if (r) CK(cudaMemcpyAsync(r, h->d_r, sizeof(double) * h->d.nr, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_set_precision(gd_handle* h, int mode) {
  if (!h) return GD_ERR_ARG;
  if (mode != GD_PREC_FP64 && mode != GD_PREC_MIXED) return fail(h, GD_ERR_ARG, "unknown precision mode");
  CK(cudaSetDevice(h->device));
  if (mode == GD_PREC_MIXED && !h->mixed) {
    int s = mixed_create(h);
    if (s) return s;
  }
  if (mode != h->precision) drop_graphs(h);
  h->precision = mode;
  return GD_OK;
}

int gd_set_fp64_stages(gd_handle* h, int mask) {
  if (!h) return GD_ERR_ARG;
  if (mask < 0 || (mask & ~(GD_STAGE_VEL_ALL | GD_STAGE_VEL_SYNTH_I8)))
    return fail(h, GD_ERR_ARG, "unknown stage in the FP64 stage mask");
  if ((mask & GD_STAGE_VEL_SYNTH_I8) && !oz_supported(h->d))
    return fail(h, GD_ERR_UNSUPPORTED, "the int8-slice synthesis takes one shell range (no segments, no ball) and lmax <= 511");
  CK(cudaSetDevice(h->device));
  // the slice images first: the mask changes only once they exist
  if ((mask & GD_STAGE_VEL_SYNTH_I8) && h->mixed) {
    const int s = mixed_prepare_int8(h);
    if (s) return s;
  }
  if (mask != h->fp64_stages) drop_graphs(h);
  h->fp64_stages = mask;
  return GD_OK;
}

int gd_set_int8_digits(gd_handle* h, int digits) {
  if (!h) return GD_ERR_ARG;
  if (digits != 5 && digits != 6) return fail(h, GD_ERR_ARG, "int8 digits must be 5 or 6");
  CK(cudaSetDevice(h->device));
  if (digits != h->int8_digits) drop_graphs(h);
  h->int8_digits = digits;
  if ((h->fp64_stages & GD_STAGE_VEL_SYNTH_I8) && h->mixed) return mixed_prepare_int8(h);
  return GD_OK;
}

int gd_set_external_derivatives(gd_handle* h, int enable) {
  if (!h) return GD_ERR_ARG;
  if (enable && (h->d.nseg > 1 || h->d.ball)) return refuse_layout(h, "the distributed step");
  CK(cudaSetDevice(h->device));
  if ((enable != 0) != h->ext_derivs) drop_graphs(h);
  h->ext_derivs = enable != 0;
  return GD_OK;
}

int gd_step_kernels(gd_handle* h, int* count) {
  if (!h || !count) return GD_ERR_ARG;
  const int boot = (h->c.ab_mode == 1 || h->step_count == 0) ? 1 : 0;
  CK(cudaSetDevice(h->device));
  int s = ensure_graph(h, boot);
  if (s) return s;
  *count = h->graph_kernels[h->nl_par][boot];
  return GD_OK;
}

// Checkpointed forward run and the temperature pullback that recomputes the
// velocity grids from its snapshots (the orchestration of the pieces above).
static void free_tckpt(gd_handle* h) {
  for (void* p : h->t_snaps) cudaFree(p);
  h->t_snaps.clear();
  if (h->t_final) cudaFree(h->t_final);
  h->t_final = nullptr;
  h->t_nsteps = 0;
}

int gd_temperature_forward(gd_handle* h, int nsteps, int checkpoint_every) {
  if (!h || nsteps < 1 || checkpoint_every < 1) return h ? fail(h, GD_ERR_ARG, "need nsteps, checkpoint_every >= 1") : GD_ERR_ARG;
  if (h->precision != GD_PREC_FP64 || h->scheme != GD_SCHEME_CNAB2)
    return fail(h, GD_ERR_UNSUPPORTED, "the temperature pullback is of the FP64 CNAB2 step");
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the temperature pullback");
  CK(cudaSetDevice(h->device));
  free_tckpt(h);
  size_t nb = 0;
  gd_snapshot_bytes(h, &nb);
  const int nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
  h->t_s0 = h->step_count;
  for (int k = 0; k < nseg; ++k) {
    void* p = nullptr;
    if (cudaMalloc(&p, nb) != cudaSuccess) { free_tckpt(h); return fail(h, GD_ERR_CUDA, "out of device memory for snapshots"); }
    h->t_snaps.push_back(p);
    int s = gd_snapshot(h, p, 0);
    if (s == GD_OK) s = gd_step(h, std::min(checkpoint_every, nsteps - k * checkpoint_every));
    if (s) { free_tckpt(h); return s; }
  }
  if (cudaMalloc(&h->t_final, nb) != cudaSuccess) { free_tckpt(h); return fail(h, GD_ERR_CUDA, "out of device memory"); }
  int s = gd_snapshot(h, h->t_final, 0);
  if (s) { free_tckpt(h); return s; }
  h->t_nsteps = nsteps;
  h->t_every = checkpoint_every;
  return GD_OK;
}

// The reverse pass of gd_temperature_forward's run.  Temperature:
//   lambda_T^n = P R^T psi^(n+1) + N_n^T nu_n,  nu_n = a_n psi^(n+1) - b_(n+1) psi^(n+2),
//   psi^n = D S^-T C lambda_T^n.
// With uv (the velocity outputs), also the gradient with respect to the
// velocity at the start: step n's advection reads the velocity grids
// VecSyn(u^(n-1)) of the previous velocity phase (the grids carried into the
// window at n = 0, constant), so u^(n-1) receives
//   s^(n-1) = VecSyn^T(-(An^T nu_n) (G_th T^n, G_ph T^n))   (gd_temperature_u_adjoint)
// and the velocity recursion of gd_velocity_pullback carries it back:
//   lambda_u^n = R^T psi_u^(n+1) + N_u^T(a_n psi_u^(n+1) - b_(n+1) psi_u^(n+2)) + s^n.
static int temperature_pullback_impl(gd_handle* h, const double* lam_re, const double* lam_im, double* out_re,
                                     double* out_im, double* const* uv) {
  if (!h || !lam_re || !lam_im || !out_re || !out_im) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (h->t_nsteps < 1) return fail(h, GD_ERR_STATE, "no checkpointed forward run (gd_temperature_forward)");
  CK(cudaSetDevice(h->device));
  const size_t se = h->spec_elems(), G = h->grid_elems();
  const int K = h->t_nsteps, C = h->t_every, nseg = (K + C - 1) / C;
  const bool ab1 = h->c.ab_mode == 1;
  const bool vel = uv != nullptr;
  const int ng = vel ? 4 : 2;  // grids kept per step: u_th, u_ph (and G_th T, G_ph T)
  auto boot = [&](int n) { return ab1 || h->t_s0 + n == 0; };
  // temperature: lam, psi1, psi2, tmp, nlt; velocity: lam, psi1, psi2, tmp, nlt, src (2 se each)
  double *lam = nullptr, *ust = nullptr;
  if (cudaMalloc(&lam, (5 + (vel ? 12 : 0)) * se * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&ust, (size_t)C * ng * G * sizeof(double)) != cudaSuccess) {
    if (lam) cudaFree(lam);
    return fail(h, GD_ERR_CUDA, "out of device memory for the pullback");
  }
  double *psi1 = lam + se, *psi2 = psi1 + se, *tmp = psi2 + se, *nlt = tmp + se;
  double* ul = nlt + se;  // velocity block
  double *upsi1 = ul + 2 * se, *upsi2 = upsi1 + 2 * se, *utmp = upsi2 + 2 * se, *unlt = utmp + 2 * se,
         *usrc = unlt + 2 * se;
  auto done = [&](int st) {
    cudaFree(lam);
    cudaFree(ust);
    return st;
  };
  auto usolve = [&](const double* x, double* y) {  // D S^-T C per potential
    int st = gd_cnab2_adjoint(h, GD_U_TOR, 0, x, y);
    return st ? st : gd_cnab2_adjoint(h, GD_U_POL, 0, x + se, y + se);
  };
  int s = gd_spectral_device(h, const_cast<double*>(lam_re), const_cast<double*>(lam_im), lam, 1);
  if (s) return done(s);
  s = gd_cnab2_adjoint(h, GD_TEMP, 0, lam, psi1);
  if (s) return done(s);
  CK(cudaMemsetAsync(psi2, 0, se * sizeof(double), h->stream));
  if (vel) {
    // the velocity after the run carries no cotangent of its own here
    CK(cudaMemsetAsync(ul, 0, 12 * se * sizeof(double), h->stream));
  }
  for (int k = nseg - 1; k >= 0 && s == GD_OK; --k) {
    const int c0 = k * C, c1 = std::min(K, c0 + C);
    s = gd_snapshot(h, h->t_snaps[k], 1);
    for (int n = c0; n < c1 && s == GD_OK; ++n) {
      double* u = ust + (size_t)(n - c0) * ng * G;
      s = gd_grid_device(h, GD_GRID_U_TH, u);
      if (s == GD_OK) s = gd_grid_device(h, GD_GRID_U_PH, u + G);
      if (s == GD_OK && (vel || n < c1 - 1)) s = gd_step(h, 1);
      // the temperature gradient grids of step n's temperature phase
      if (s == GD_OK && vel) s = gd_grid_device(h, GD_GRID_GTH, u + 2 * G);
      if (s == GD_OK && vel) s = gd_grid_device(h, GD_GRID_GPH, u + 3 * G);
    }
    for (int n = c1 - 1; n >= c0 && s == GD_OK; --n) {
      const double a_n = boot(n) ? 1.0 : 1.5;
      const double b_n1 = (n + 1 >= K || boot(n + 1)) ? 0.0 : 0.5;
      launch_axpby(h->stream, se, a_n, psi1, -b_n1, psi2, tmp);  // nu_n
      const double* u = ust + (size_t)(n - c0) * ng * G;
      s = gd_temperature_nl_adjoint(h, u, u + G, tmp, nlt);
      if (s == GD_OK) s = gd_cnab2_adjoint(h, GD_TEMP, 1, psi1, lam);
      if (s == GD_OK) launch_axpby(h->stream, se, 1.0, lam, 1.0, nlt, lam);
      if (s == GD_OK && vel) {
        // lambda_u^n with the source s^n of step n + 1 (usrc), then the source of step n
        launch_axpby(h->stream, 2 * se, a_n, upsi1, -b_n1, upsi2, utmp);
        s = gd_velocity_nl_adjoint(h, utmp, unlt);
        if (s == GD_OK) s = gd_cnab2_adjoint(h, GD_U_TOR, 1, upsi1, ul);
        if (s == GD_OK) s = gd_cnab2_adjoint(h, GD_U_POL, 1, upsi1 + se, ul + se);
        if (s == GD_OK) launch_axpby(h->stream, 2 * se, 1.0, ul, 1.0, unlt, ul);
        if (s == GD_OK) launch_axpby(h->stream, 2 * se, 1.0, ul, 1.0, usrc, ul);
        if (s == GD_OK && n >= 1) s = gd_temperature_u_adjoint(h, u + 2 * G, u + 3 * G, tmp, usrc);
        if (s == GD_OK && n == 0) CK(cudaMemsetAsync(usrc, 0, 2 * se * sizeof(double), h->stream));
      }
      if (s == GD_OK && n > 0) {
        std::swap(psi1, psi2);
        s = gd_cnab2_adjoint(h, GD_TEMP, 0, lam, psi1);
        if (s == GD_OK && vel) {
          std::swap(upsi1, upsi2);
          s = usolve(ul, upsi1);
        }
      }
    }
  }
  if (s == GD_OK) s = gd_snapshot(h, h->t_final, 1);
  if (s == GD_OK) s = gd_spectral_device(h, out_re, out_im, lam, 0);
  if (s == GD_OK && vel) s = gd_spectral_device(h, uv[0], uv[1], ul, 0);
  if (s == GD_OK && vel) s = gd_spectral_device(h, uv[2], uv[3], ul + se, 0);
  return done(s);
}

int gd_temperature_pullback(gd_handle* h, const double* lam_re, const double* lam_im, double* out_re, double* out_im) {
  return temperature_pullback_impl(h, lam_re, lam_im, out_re, out_im, nullptr);
}

int gd_temperature_pullback_full(gd_handle* h, const double* lam_re, const double* lam_im, double* out_re,
                                 double* out_im, double* out_tor_re, double* out_tor_im, double* out_pol_re,
                                 double* out_pol_im) {
  if (!out_tor_re || !out_tor_im || !out_pol_re || !out_pol_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  double* uv[4] = {out_tor_re, out_tor_im, out_pol_re, out_pol_im};
  return temperature_pullback_impl(h, lam_re, lam_im, out_re, out_im, uv);
}

// s = VecSyn^T(-(An^T nu) (gth, gph)) with An^T = W Syn D and VecSyn^T =
// D^-1 Lambda VecAn W^-1 (the Gauss weights cancel): the cotangent of the
// velocity potentials whose synthesized grids advect the temperature.
int gd_temperature_u_adjoint(gd_handle* h, const double* gth, const double* gph, const double* nu, double* out) {
  if (!h || !gth || !gph || !nu || !out) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the temperature-velocity adjoint");
  CK(cudaSetDevice(h->device));
  const size_t se = h->spec_elems(), G = h->grid_elems();
  if (!h->d_adj) AL(h->d_adj, 3 * se + 4 * G);
  const Dims& d = h->d;
  double* nup = h->d_adj;            // D nu
  double* g = h->d_adj + 3 * se;     // Syn(D nu)
  double* hq = g + G;                // -g gth, -g gph (consecutive for the vector analysis)
  const double tp = 2.0 * 3.14159265358979323846 / d.nlon;
  CK(cudaMemcpyAsync(nup, nu, se * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  launch_scale_by_order(h->stream, 2 * (size_t)d.nr, d.nlm, h->d_mof, tp, 0.5 * tp, nup);
  const double* coef[1] = {nup};
  int s = synth_scalar(h, coef, 1, g);
  if (s) return s;
  launch_neg_product(h->stream, G, gth, g, hq);
  launch_neg_product(h->stream, G, gph, g, hq + G);
  s = analysis_vector(h, hq, out, out + se, EPI_VECTOR);
  if (s) return s;
  launch_scale_by_degree(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_lof, 1.0, 0, out);
  launch_scale_by_order(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_mof, 1.0 / tp, 2.0 / tp, out);
  s = check_launch(h, "temperature-velocity adjoint");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_set_launch_shape(gd_handle* h, int tc_ctas) {
  if (!h || tc_ctas < 0) return h ? fail(h, GD_ERR_ARG, "tc_ctas must be >= 0") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (tc_ctas != h->tc_ctas) drop_graphs(h);
  h->tc_ctas = tc_ctas;
  return GD_OK;
}

int gd_get_launch_shape(const gd_handle* h, int* tc_ctas) {
  if (!h || !tc_ctas) return GD_ERR_ARG;
  *tc_ctas = h->tc_ctas;
  return GD_OK;
}

int gd_set_segment_ekman(gd_handle* h, const double* ekman) {
  if (!h || !ekman) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  const int nseg = h->d.nseg;
  for (int g = 0; g < nseg; ++g)
    if (!(ekman[g] > 0.0) || !std::isfinite(ekman[g])) return fail(h, GD_ERR_ARG, "Ekman numbers must be positive");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  // rossby_factor (src/velocity.jl:456): Pm / E of each shell's segment, in
  // FP64 for the FP64 kernels and rounded once to FP32 for the fused kernel
  std::vector<double> rf(h->d.nr);
  std::vector<float> rf32(h->d.nr);
  for (int k = 0; k < h->d.nr; ++k) {
    rf[k] = h->c.magnetic_prandtl / ekman[std::upper_bound(h->seg_base.begin(), h->seg_base.end(), k) -
                                          h->seg_base.begin() - 1];
    rf32[k] = (float)rf[k];
  }
  if (!h->d_rfs) {
    AL(h->d_rfs, h->d.nr);
    AL(h->d_rfs32, h->d.nr);
  }
  CK(cudaMemcpyAsync(h->d_rfs, rf.data(), sizeof(double) * h->d.nr, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_rfs32, rf32.data(), sizeof(float) * h->d.nr, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  drop_graphs(h);
  h->d.rfs = h->d_rfs;
  h->d.rfs32 = h->d_rfs32;
  return GD_OK;
}

static bool mode_range_ok(const gd_handle* h, int j0, int j1) { return 0 <= j0 && j0 <= j1 && j1 <= h->d.nlm; }


int gd_set_composition_bc(gd_handle* h, const double* bvals, const double* sources) {
  if (!h) return GD_ERR_ARG;
  if (!h->c.composition) return fail(h, GD_ERR_STATE, "the configuration has no composition");
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  if (bvals) {
    CK(cudaMemcpyAsync(h->d_stage_spec, bvals, 2 * (size_t)h->d.nlm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    Dims d1 = h->d;
    d1.nr = 1;
    launch_lmajor_to_native(h->stream, d1, h->d_perm, h->d_stage_spec, h->d_cbvals, 2);
  }
  if (sources) CK(cudaMemcpyAsync(h->d_csources, sources, h->d.nr * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "set composition bc");
}

int gd_set_scalar_bc_types(gd_handle* h, int field, const int* inner, const int* outer) {
  if (!h || !inner || !outer) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (field != GD_TEMP && field != GD_COMP) return fail(h, GD_ERR_ARG, "boundary types are for GD_TEMP or GD_COMP");
  if (field == GD_COMP && !h->c.composition) return fail(h, GD_ERR_STATE, "the configuration has no composition");
  const size_t NL = h->d.nlm;
  std::vector<int> t(2 * NL);
  bool flux = false;
  for (size_t q = 0; q < NL; ++q) {
    const int a = inner[q], b = outer[q];
    if ((a != GD_BC_VALUE && a != GD_BC_FLUX) || (b != GD_BC_VALUE && b != GD_BC_FLUX))
      return fail(h, GD_ERR_ARG, "boundary types must be GD_BC_VALUE or GD_BC_FLUX");
    flux |= a == GD_BC_FLUX || b == GD_BC_FLUX;
    t[h->perm[q]] = a;  // l-major q -> native
    t[NL + h->perm[q]] = b;
  }
  bool inner_flux = false;
  for (size_t q = 0; q < NL; ++q) inner_flux |= inner[q] == GD_BC_FLUX;
  if (inner_flux && h->d.ball)
    return fail(h, GD_ERR_UNSUPPORTED, "a ball has no inner boundary: its centre row is the regularity condition");
  if (flux && h->c.bc_mode == 2 && !h->flux_rows_ok)
    return fail(h, GD_ERR_SINGULAR, "the implicit factorisation with flux boundary rows has a zero pivot");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpyAsync(h->d_bctype + (field == GD_COMP ? 2 * NL : 0), t.data(), sizeof(int) * 2 * NL,
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  std::copy(t.begin(), t.end(), h->bctype.begin() + (field == GD_COMP ? 2 * NL : 0));
  return GD_OK;
}

// ---- reverse mode of the temperature step -------------------------------------
// Grids a step reads before writing them: the velocity grids (temperature
// phase), the magnetic field and current grids (the velocity phase's Lorentz
// term).  A snapshot holds these and the spectral state.
static const int kCarried[6] = {GD_GRID_U_TH, GD_GRID_U_PH, GD_GRID_B_TH, GD_GRID_B_PH, GD_GRID_J_TH, GD_GRID_J_PH};

int gd_snapshot_bytes(gd_handle* h, size_t* bytes) {
  if (!h || !bytes) return GD_ERR_ARG;
  *bytes = 64 + sizeof(double) * (3 * NFIELD * h->spec_elems() + 6 * h->grid_elems());
  return GD_OK;
}

int gd_snapshot(gd_handle* h, void* dev, int restore) {
  if (!h || !dev) return h ? fail(h, GD_ERR_ARG, "null buffer") : GD_ERR_ARG;
  if (h->precision != GD_PREC_FP64)
    return fail(h, GD_ERR_UNSUPPORTED, "snapshots hold the FP64 path's state (the mixed step keeps Fourier buffers)");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  const size_t se = NFIELD * h->spec_elems() * sizeof(double), gb = h->grid_elems() * sizeof(double);
  char* b = static_cast<char*>(dev);
  long long hdr[3] = {h->nl_par, h->last_nl_par, h->step_count};
  const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
  if (!restore) {
    CK(cudaMemcpyAsync(b, hdr, sizeof(hdr), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(b + 64, h->d_state, se, dd, h->stream));
    CK(cudaMemcpyAsync(b + 64 + se, h->d_nl, se, dd, h->stream));
    CK(cudaMemcpyAsync(b + 64 + 2 * se, h->d_prev, se, dd, h->stream));
    for (int g = 0; g < 6; ++g) CK(cudaMemcpyAsync(b + 64 + 3 * se + g * gb, h->grid(kCarried[g]), gb, dd, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  } else {
    CK(cudaMemcpyAsync(hdr, b, sizeof(hdr), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->d_state, b + 64, se, dd, h->stream));
    CK(cudaMemcpyAsync(h->d_nl, b + 64 + se, se, dd, h->stream));
    CK(cudaMemcpyAsync(h->d_prev, b + 64 + 2 * se, se, dd, h->stream));
    for (int g = 0; g < 6; ++g) CK(cudaMemcpyAsync(h->grid(kCarried[g]), b + 64 + 3 * se + g * gb, gb, dd, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->nl_par = (int)hdr[0];
    h->last_nl_par = (int)hdr[1];
    h->step_count = hdr[2];
  }
  return GD_OK;
}

int gd_spectral_device(gd_handle* h, double* re, double* im, double* dev, int to_device) {
  if (!h || !re || !im || !dev) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm;
  if (to_device) {
    CK(cudaMemcpyAsync(h->d_stage_spec, re, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_stage_spec + plane, im, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, dev, 2);
  } else {
    launch_native_to_lmajor(h->stream, h->d, h->d_perm, dev, h->d_stage_spec, 2);
    CK(cudaMemcpyAsync(re, h->d_stage_spec, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(im, h->d_stage_spec + plane, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "spectral device copy");
}

int gd_grid_device(gd_handle* h, int grid, double* dev) {
  if (!h || !dev || grid < 0 || grid >= NGRID) return h ? fail(h, GD_ERR_ARG, "bad grid or pointer") : GD_ERR_ARG;
  if (h->precision != GD_PREC_FP64) return fail(h, GD_ERR_UNSUPPORTED, "device grids are the FP64 path's");
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(dev, h->grid(grid), h->grid_elems() * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_temperature_nl_adjoint(gd_handle* h, const double* u_th, const double* u_ph, const double* nu, double* out) {
  if (!h || !u_th || !u_ph || !nu || !out) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the nonlinear-term adjoint");
  CK(cudaSetDevice(h->device));
  const size_t se = h->spec_elems(), G = h->grid_elems();
  if (!h->d_adj) AL(h->d_adj, 3 * se + 4 * G);
  double* nup = h->d_adj;        // D nu
  double* ath = nup + se;        // An(-u_th g), then D' scaled
  double* aph = ath + se;
  double* g = h->d_adj + 3 * se; // Syn(D nu)
  double* hth = g + G;           // -u_th g, -u_ph g (consecutive for the two-field analysis)
  const double tp = 2.0 * 3.14159265358979323846 / h->d.nlon;
  // An^T = W Syn D with D = 2 pi / nlon (m = 0), pi / nlon (m > 0); Syn^T = D' An W^-1
  // with D' = D^-1: the Gauss weights cancel between them
  CK(cudaMemcpyAsync(nup, nu, se * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  launch_scale_by_order(h->stream, 2 * (size_t)h->d.nr, h->d.nlm, h->d_mof, tp, 0.5 * tp, nup);
  const double* coef[1] = {nup};
  int s = synth_scalar(h, coef, 1, g);
  if (s) return s;
  launch_neg_product(h->stream, G, u_th, g, hth);
  launch_neg_product(h->stream, G, u_ph, g, hth + G);
  double* outs[2] = {ath, aph};
  s = analysis_scalar(h, hth, 2, outs);
  if (s) return s;
  launch_scale_by_order(h->stream, 4 * (size_t)h->d.nr, h->d.nlm, h->d_mof, 1.0 / tp, 2.0 / tp, ath);
  launch_gradients_adjoint(h->stream, h->d, h->d_lof, h->d_mof, h->d_rinv, ath, aph, out);
  s = check_launch(h, "temperature nonlinear adjoint");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_cnab2_adjoint(gd_handle* h, int field, int mode, const double* x, double* y) {
  if (!h || !x || !y || (mode != 0 && mode != 1) || field < 0 || field >= nfields(h))
    return h ? fail(h, GD_ERR_ARG, "bad field, mode or pointer") : GD_ERR_ARG;
  if (h->scheme != GD_SCHEME_CNAB2) return fail(h, GD_ERR_UNSUPPORTED, "the adjoint is of the CNAB2 step");
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the CNAB2 adjoint");
  const size_t NL = h->d.nlm;
  const bool scalar = field == GD_TEMP || field == GD_COMP;
  const int kind = field == GD_TEMP ? 2 : field == GD_COMP ? 3 : (field == GD_U_TOR || field == GD_U_POL) ? 0 : 1;
  const int* types = nullptr;
  if (scalar) {
    const size_t o = field == GD_COMP ? 2 * NL : 0;
    for (size_t q = 0; q < 2 * NL; ++q)
      if (h->bctype[o + q] == GD_BC_FLUX)
        return fail(h, GD_ERR_UNSUPPORTED, "the adjoint covers fixed-value boundaries (no tau flux rows)");
    types = h->d_bctype + o;
  }
  CK(cudaSetDevice(h->device));
  launch_cnab2_adjoint(h->stream, h->d, h->d_lof, h->d_lin, h->d_lu, types, kind, mode, h->c.dt, h->c.implicit_theta,
                       h->c.bc_mode == 1, h->c.bc_mode == 2, x, y);
  int s = check_launch(h, "cnab2 adjoint");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_derivatives(gd_handle* h, int j0, int j1) {
  if (!h) return GD_ERR_ARG;
  if (h->d.nseg > 1) return refuse_layout(h, "the mode-range derivatives");
  if (!mode_range_ok(h, j0, j1)) return fail(h, GD_ERR_ARG, "mode range outside [0, nlm]");
  CK(cudaSetDevice(h->device));
  if (j1 == j0) return GD_OK;
  Dims d = h->d;
  d.jlo = j0;
  d.jhi = j1;
  { ProfScope p(h, "spectral_gradients");
    launch_gradients(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_TEMP), h->work(0), h->work(1),
                     h->work(2)); }
  { ProfScope p(h, "spectral_curl");
    launch_curl(h->stream, d, h->d_lof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_UTOR), h->field(F_UPOL),
                h->work(3), h->work(4));
    if (h->c.magnetic)
      launch_curl(h->stream, d, h->d_lof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_BTOR),
                  h->field(F_BPOL), h->work(5), h->work(6)); }
  if (h->c.composition) {
    ProfScope p(h, "spectral_gradients");
    launch_gradients(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_COMP), h->work(8), h->work(9),
                     h->work(10));
  }
  int s = check_launch(h, "derivatives");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_implicit_modes(gd_handle* h, int j0, int j1) {
  if (!h) return GD_ERR_ARG;
  if (h->d.nseg > 1) return refuse_layout(h, "the mode-range solve");
  if (!mode_range_ok(h, j0, j1)) return fail(h, GD_ERR_ARG, "mode range outside [0, nlm]");
  if (h->scheme != GD_SCHEME_CNAB2) return fail(h, GD_ERR_UNSUPPORTED, "the mode-range solve supports CNAB2 only");
  CK(cudaSetDevice(h->device));
  const int boot = (h->c.ab_mode == 1 || h->step_count == 0) ? 1 : 0;
  int s = GD_OK;
  if (j1 > j0) {
    const Dims full = h->d;
    h->d.jlo = j0;
    h->d.jhi = j1;
    scalar_bc(h, F_TEMP);
    if (h->c.composition) scalar_bc(h, F_COMP);
    s = implicit_launch(h, boot);
    h->d = full;
  }
  if (s) return s;
  s = check_launch(h, "mode-range implicit step");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  end_step(h);
  return GD_OK;
}

int gd_copy_block(gd_handle* h, int array, int field, int r0, int r1, int j0, int j1, void* buf, int to_buf) {
  if (!h || !buf) return h ? fail(h, GD_ERR_ARG, "null buffer") : GD_ERR_ARG;
  const int nf = array == 1 ? NWORK : nfields(h);
  if (array < 0 || array > 2 || field < 0 || field >= nf) return fail(h, GD_ERR_ARG, "bad array or field");
  if (!(0 <= r0 && r0 <= r1 && r1 <= h->d.nr) || !mode_range_ok(h, j0, j1))
    return fail(h, GD_ERR_ARG, "block outside the handle's shells or modes");
  CK(cudaSetDevice(h->device));
  double* base = array == 0 ? h->field(field) : array == 1 ? h->work(field) : h->nlf(field);
  const size_t NM = h->d.nlm, plane = (size_t)h->d.nr * NM;
  const size_t w = (size_t)(j1 - j0) * sizeof(double), rows = (size_t)(r1 - r0);
  if (w == 0 || rows == 0) return GD_OK;
  for (int c = 0; c < 2; ++c) {
    double* a = base + c * plane + (size_t)r0 * NM + j0;
    double* b = static_cast<double*>(buf) + (size_t)c * rows * (j1 - j0);
    if (to_buf)
      CK(cudaMemcpy2DAsync(b, w, a, NM * sizeof(double), w, rows, cudaMemcpyDefault, h->stream));
    else
      CK(cudaMemcpy2DAsync(a, NM * sizeof(double), b, w, w, rows, cudaMemcpyDefault, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_set_fault_test(gd_handle* h, long long wait_cycles, int omit_step) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  drop_graphs(h);  // captured steps hold the previous settings
  return mixed_set_fault_test(h, wait_cycles, omit_step);
}

int gd_synchronize(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (h->precision == GD_PREC_MIXED) return mixed_check_error(h);
  return GD_OK;
}

int gd_upload_spectral(gd_handle* h, int field, const double* re, const double* im) {
  if (!h || !re || !im || field < 0 || field >= nfields(h)) return h ? fail(h, GD_ERR_ARG, "bad field or pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm;
  CK(cudaMemcpyAsync(h->d_stage_spec, re, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_stage_spec + plane, im, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, h->field(field), 2);
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "upload");
}

static int download_spec(gd_handle* h, const double* src, double* re, double* im) {
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm;
  launch_native_to_lmajor(h->stream, h->d, h->d_perm, src, h->d_stage_spec, 2);
  CK(cudaMemcpyAsync(re, h->d_stage_spec, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(im, h->d_stage_spec + plane, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "download");
}

int gd_download_spectral(gd_handle* h, int field, double* re, double* im) {
  if (!h || !re || !im || field < 0 || field >= nfields(h)) return h ? fail(h, GD_ERR_ARG, "bad field or pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  return download_spec(h, h->field(field), re, im);
}

int gd_download_nonlinear(gd_handle* h, int field, double* re, double* im) {
  if (!h || !re || !im || field < 0 || field >= nfields(h)) return h ? fail(h, GD_ERR_ARG, "bad field or pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  return download_spec(h, h->nl_bank(h->last_nl_par) + h->spec_elems() * field, re, im);
}

int gd_download_grid(gd_handle* h, int grid, double* out) {
  if (!h || !out || grid < 0 || grid >= NGRID) return h ? fail(h, GD_ERR_ARG, "bad grid id or pointer") : GD_ERR_ARG;
  if (grid >= GD_GRID_C && !h->c.composition) return fail(h, GD_ERR_STATE, "the configuration has no composition");
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const double* src = h->grid(grid);
  if (h->precision == GD_PREC_MIXED) {
    s = mixed_grid_to_double(h, grid, h->d_stage_grid2);
    if (s) return s;
    src = h->d_stage_grid2;
  }
  launch_grid_to_reference(h->stream, h->d, src, h->d_stage_grid, 1);
  CK(cudaMemcpyAsync(out, h->d_stage_grid, h->grid_elems() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "download grid");
}

int gd_set_temperature_bc(gd_handle* h, const double* bvals, const double* sources) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  if (bvals) {
    CK(cudaMemcpyAsync(h->d_stage_spec, bvals, 2 * (size_t)h->d.nlm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    // two rows of nlm, permuted like one two-row plane
    Dims d1 = h->d;
    d1.nr = 1;
    launch_lmajor_to_native(h->stream, d1, h->d_perm, h->d_stage_spec, h->d_bvals, 2);
  }
  if (sources) CK(cudaMemcpyAsync(h->d_sources, sources, h->d.nr * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "set temperature bc");
}

int gd_spectral_to_physical(gd_handle* h, int nfield, const double* re, const double* im, double* grid) {
  if (!h || !re || !im || !grid || nfield < 1) return h ? fail(h, GD_ERR_ARG, "bad arguments") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm, G = h->grid_elems();
  for (int f0 = 0; f0 < nfield; f0 += 4) {
    const int nf = nfield - f0 < 4 ? nfield - f0 : 4;
    const double* coef[4];
    for (int i = 0; i < nf; ++i) {
      CK(cudaMemcpyAsync(h->d_stage_spec + 2 * plane * i, re + plane * (f0 + i), plane * sizeof(double),
                         cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(h->d_stage_spec + 2 * plane * i + plane, im + plane * (f0 + i), plane * sizeof(double),
                         cudaMemcpyHostToDevice, h->stream));
    }
    launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, h->d_stage_spec2, 2 * nf);
    for (int i = 0; i < nf; ++i) coef[i] = h->d_stage_spec2 + 2 * plane * i;
    if (h->precision == GD_PREC_MIXED) s = mixed_api_synth_scalar(h, coef, nf, h->d_stage_grid2);
    else s = synth_scalar(h, coef, nf, h->d_stage_grid2);
    if (s) return s;
    launch_grid_to_reference(h->stream, h->d, h->d_stage_grid2, h->d_stage_grid, nf);
    CK(cudaMemcpyAsync(grid + G * f0, h->d_stage_grid, G * nf * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return check_launch(h, "spectral_to_physical");
}

// The r = 0 level (the first of each segment) of nf spectral fields, stride
// fstride, set to 0 for l >= 1 whatever the geometry, as the reference's
// enforce_ball_*_regularity! do (src/Ball/Ball.jl:153-195).
static void zero_first_level(gd_handle* h, double* F, int nf, size_t fstride) {
  Dims dz = h->d;
  dz.ball = 1;
  launch_regularity(h->stream, dz, h->d_lof, F, nf, fstride);
}

static int physical_to_spectral(gd_handle* h, int nfield, const double* grid, double* re, double* im, bool regular) {
  if (!h || !re || !im || !grid || nfield < 1) return h ? fail(h, GD_ERR_ARG, "bad arguments") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm, G = h->grid_elems();
  for (int f0 = 0; f0 < nfield; f0 += 4) {
    const int nf = nfield - f0 < 4 ? nfield - f0 : 4;
    CK(cudaMemcpyAsync(h->d_stage_grid, grid + G * f0, G * nf * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    launch_grid_to_native(h->stream, h->d, h->d_stage_grid, h->d_stage_grid2, nf);
    double* out[4];
    for (int i = 0; i < nf; ++i) out[i] = h->d_stage_spec2 + 2 * plane * i;
    if (h->precision == GD_PREC_MIXED) s = mixed_api_analysis_scalar(h, h->d_stage_grid2, nf, out);
    else s = analysis_scalar(h, h->d_stage_grid2, nf, out);
    if (s) return s;
    if (regular) zero_first_level(h, h->d_stage_spec2, nf, 2 * plane);
    launch_native_to_lmajor(h->stream, h->d, h->d_perm, h->d_stage_spec2, h->d_stage_spec, 2 * nf);
    for (int i = 0; i < nf; ++i) {
      CK(cudaMemcpyAsync(re + plane * (f0 + i), h->d_stage_spec + 2 * plane * i, plane * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
      CK(cudaMemcpyAsync(im + plane * (f0 + i), h->d_stage_spec + 2 * plane * i + plane, plane * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
  }
  return check_launch(h, "physical_to_spectral");
}

int gd_physical_to_spectral(gd_handle* h, int nfield, const double* grid, double* re, double* im) {
  return physical_to_spectral(h, nfield, grid, re, im, false);
}

int gd_ball_physical_to_spectral(gd_handle* h, int nfield, const double* grid, double* re, double* im) {
  return physical_to_spectral(h, nfield, grid, re, im, true);
}

int gd_enforce_regularity(gd_handle* h, int field) {
  if (!h || field < 0 || field >= nfields(h)) return h ? fail(h, GD_ERR_ARG, "bad field") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  zero_first_level(h, h->field(field), 1, 0);
  int s = check_launch(h, "enforce regularity");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

int gd_spectral_to_physical_adjoint(gd_handle* h, int nfield, const double* grid, double* re, double* im) {
  if (!h || !re || !im || !grid || nfield < 1) return h ? fail(h, GD_ERR_ARG, "bad arguments") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm, G = h->grid_elems();
  const double f0 = (double)h->d.nlon / (2.0 * 3.14159265358979323846), f1 = 2.0 * f0;
  for (int f0i = 0; f0i < nfield; f0i += 4) {
    const int nf = nfield - f0i < 4 ? nfield - f0i : 4;
    CK(cudaMemcpyAsync(h->d_stage_grid, grid + G * f0i, G * nf * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    launch_divide_by_weights(h->stream, G * nf, h->d.nlat, h->d_w, h->d_stage_grid);
    launch_grid_to_native(h->stream, h->d, h->d_stage_grid, h->d_stage_grid2, nf);
    double* out[4];
    for (int i = 0; i < nf; ++i) out[i] = h->d_stage_spec2 + 2 * plane * i;
    if (h->precision == GD_PREC_MIXED) s = mixed_api_analysis_scalar(h, h->d_stage_grid2, nf, out);
    else s = analysis_scalar(h, h->d_stage_grid2, nf, out);
    if (s) return s;
    launch_scale_by_order(h->stream, 2 * (size_t)h->d.nr * nf, h->d.nlm, h->d_mof, f0, f1, h->d_stage_spec2);
    launch_native_to_lmajor(h->stream, h->d, h->d_perm, h->d_stage_spec2, h->d_stage_spec, 2 * nf);
    for (int i = 0; i < nf; ++i) {
      CK(cudaMemcpyAsync(re + plane * (f0i + i), h->d_stage_spec + 2 * plane * i, plane * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
      CK(cudaMemcpyAsync(im + plane * (f0i + i), h->d_stage_spec + 2 * plane * i + plane, plane * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
  }
  return check_launch(h, "spectral_to_physical_adjoint");
}

// The velocity's nonlinear term of the literal step is its Coriolis term alone
// (u x w and j x B vanish with zero radial components), linear in u:
//   N = VecAn Cor VecSyn,  Cor = pointwise [[0, -c], [c, 0]], c = Pm/E cos(theta(min(j, nlat - 1))),
// with VecAn = Lambda^-1 VecSyn^T W D^-1 (Lambda = l(l+1), W the Gauss weights
// and D = 2 pi / nlon (m = 0), pi / nlon (m > 0) the real-coefficient
// weighting of the phi sums), so VecSyn^T = D^-1 Lambda VecAn W^-1 and
// VecAn^T = W VecSyn Lambda^-1 D; Cor is antisymmetric, hence
//   N^T = -D^-1 Lambda N Lambda^-1 D,
// evaluated with the FP64 forward kernels.  psi, out: (tor, pol) consecutive,
// spec_elems each, native layout on the device.
int gd_velocity_nl_adjoint(gd_handle* h, const double* psi, double* out) {
  if (!h || !psi || !out) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the velocity nonlinear-term adjoint");
  CK(cudaSetDevice(h->device));
  const size_t se = h->spec_elems(), G = h->grid_elems();
  if (!h->d_adj) AL(h->d_adj, 3 * se + 4 * G);
  const Dims& d = h->d;
  double* x = h->d_adj;               // Lambda^-1 D psi, tor then pol
  double* g = h->d_adj + 3 * se;      // VecSyn x: theta, phi
  double* z = g + 2 * G;              // Cor VecSyn x: theta, phi
  const double tp = 2.0 * 3.14159265358979323846 / d.nlon;
  CK(cudaMemcpyAsync(x, psi, 2 * se * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  launch_scale_by_order(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_mof, tp, 0.5 * tp, x);
  launch_scale_by_degree(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_lof, 1.0, 1, x);
  int s = synth_vector(h, x, x + se, g);
  if (s) return s;
  const double rf = h->c.magnetic_prandtl / h->c.ekman;
  launch_coriolis<double>(h->stream, d, h->d_cth, h->d_sthc, rf, g, g + G, z, z + G);
  s = analysis_vector(h, z, out, out + se, EPI_VECTOR);
  if (s) return s;
  launch_scale_by_degree(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_lof, -1.0, 0, out);
  launch_scale_by_order(h->stream, 4 * (size_t)d.nr, d.nlm, h->d_mof, 1.0 / tp, 2.0 / tp, out);
  s = check_launch(h, "velocity nonlinear adjoint");
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  return GD_OK;
}

// Reverse mode of the last nsteps CNAB2 steps of the velocity (those that end
// at the handle's step count; the bootstrap pattern follows from it):
// u^(n+1) = C S^-1 D (R u^n + a_n N u^n - b_n N u^(n-1)) (AB2 weights
// a = 3/2, b = 1/2; a = 1, b = 0 on a bootstrap step), so with
// psi^(n+1) = D S^-T C lambda^(n+1):
//   lambda^n = R^T psi^(n+1) + N^T (a_n psi^(n+1) - b_(n+1) psi^(n+2)).
// Linear and independent of the state (N is the Coriolis term), so no
// checkpoints; lambda^0 is the gradient with respect to (u_tor, u_pol) at the
// start.  The pullback of the FP64 step, whatever the handle's precision.
int gd_velocity_pullback(gd_handle* h, int nsteps, const double* lam_tor_re, const double* lam_tor_im,
                         const double* lam_pol_re, const double* lam_pol_im, double* out_tor_re, double* out_tor_im,
                         double* out_pol_re, double* out_pol_im) {
  if (!h || nsteps < 0 || !lam_tor_re || !lam_tor_im || !lam_pol_re || !lam_pol_im || !out_tor_re || !out_tor_im ||
      !out_pol_re || !out_pol_im)
    return h ? fail(h, GD_ERR_ARG, "bad arguments") : GD_ERR_ARG;
  if (h->scheme != GD_SCHEME_CNAB2) return fail(h, GD_ERR_UNSUPPORTED, "the pullback is of the CNAB2 step");
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the velocity pullback");
  if (h->step_count < nsteps) return fail(h, GD_ERR_STATE, "the handle has not run the steps to pull back");
  CK(cudaSetDevice(h->device));
  const size_t se = h->spec_elems();
  const long s0 = h->step_count - nsteps;
  const bool ab1 = h->c.ab_mode == 1;
  auto boot = [&](int n) { return ab1 || s0 + n == 0; };
  double* lam = nullptr;  // lam, psi1, psi2, tmp, nlt: (tor, pol) each
  if (cudaMalloc(&lam, 10 * se * sizeof(double)) != cudaSuccess)
    return fail(h, GD_ERR_CUDA, "out of device memory for the pullback");
  double *psi1 = lam + 2 * se, *psi2 = psi1 + 2 * se, *tmp = psi2 + 2 * se, *nlt = tmp + 2 * se;
  auto done = [&](int st) {
    cudaFree(lam);
    return st;
  };
  auto solveT = [&](const double* x, double* y) {  // D S^-T C per potential
    int st = gd_cnab2_adjoint(h, GD_U_TOR, 0, x, y);
    return st ? st : gd_cnab2_adjoint(h, GD_U_POL, 0, x + se, y + se);
  };
  int s = gd_spectral_device(h, const_cast<double*>(lam_tor_re), const_cast<double*>(lam_tor_im), lam, 1);
  if (!s) s = gd_spectral_device(h, const_cast<double*>(lam_pol_re), const_cast<double*>(lam_pol_im), lam + se, 1);
  if (s) return done(s);
  if (nsteps > 0) {
    s = solveT(lam, psi1);
    CK(cudaMemsetAsync(psi2, 0, 2 * se * sizeof(double), h->stream));
  }
  for (int n = nsteps - 1; n >= 0 && s == GD_OK; --n) {
    const double a_n = boot(n) ? 1.0 : 1.5;
    const double b_n1 = (n + 1 >= nsteps || boot(n + 1)) ? 0.0 : 0.5;
    launch_axpby(h->stream, 2 * se, a_n, psi1, -b_n1, psi2, tmp);
    s = gd_velocity_nl_adjoint(h, tmp, nlt);
    if (s == GD_OK) s = gd_cnab2_adjoint(h, GD_U_TOR, 1, psi1, lam);
    if (s == GD_OK) s = gd_cnab2_adjoint(h, GD_U_POL, 1, psi1 + se, lam + se);
    if (s == GD_OK) launch_axpby(h->stream, 2 * se, 1.0, lam, 1.0, nlt, lam);
    if (s == GD_OK && n > 0) {
      std::swap(psi1, psi2);
      s = solveT(lam, psi1);
    }
  }
  if (s == GD_OK) s = gd_spectral_device(h, out_tor_re, out_tor_im, lam, 0);
  if (s == GD_OK) s = gd_spectral_device(h, out_pol_re, out_pol_im, lam + se, 0);
  if (s == GD_OK) s = check_launch(h, "velocity pullback");
  return done(s);
}

int gd_magnetic_pullback(gd_handle* h, int field, int nsteps, const double* lam_re, const double* lam_im,
                         double* out_re, double* out_im) {
  if (!h || !lam_re || !lam_im || !out_re || !out_im || nsteps < 0 || (field != GD_B_TOR && field != GD_B_POL))
    return h ? fail(h, GD_ERR_ARG, "bad arguments (field must be GD_B_TOR or GD_B_POL)") : GD_ERR_ARG;
  if (h->scheme != GD_SCHEME_CNAB2) return fail(h, GD_ERR_UNSUPPORTED, "the pullback is of the CNAB2 propagator");
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "the magnetic pullback");
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm;
  CK(cudaMemcpyAsync(h->d_stage_spec, lam_re, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_stage_spec + plane, lam_im, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, h->d_stage_spec2, 2);
  // without the magnetic field the step leaves it untouched: the pullback is the identity
  if (h->c.magnetic && nsteps > 0)
    launch_cnab2_pullback(h->stream, h->d, h->d_lof, h->d_lin, h->d_lu, 1, h->c.dt, h->c.implicit_theta,
                          h->c.bc_mode == 1, h->c.bc_mode == 2, nsteps, h->d_stage_spec2);
  launch_native_to_lmajor(h->stream, h->d, h->d_perm, h->d_stage_spec2, h->d_stage_spec, 2);
  CK(cudaMemcpyAsync(out_re, h->d_stage_spec, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(out_im, h->d_stage_spec + plane, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "magnetic_pullback");
}

int gd_vector_synthesis(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                        const double* pol_im, double* v_theta, double* v_phi) {
  if (!h || !tor_re || !tor_im || !pol_re || !pol_im || !v_theta || !v_phi)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm, G = h->grid_elems();
  const double* src[4] = {tor_re, tor_im, pol_re, pol_im};
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(h->d_stage_spec + plane * i, src[i], plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, h->d_stage_spec2, 4);
  const double* tor = h->d_stage_spec2;
  const double* pol = h->d_stage_spec2 + 2 * plane;
  if (h->precision == GD_PREC_MIXED) s = mixed_api_synth_vector(h, tor, pol, h->d_stage_grid2);
  else s = synth_vector(h, tor, pol, h->d_stage_grid2);
  if (s) return s;
  launch_grid_to_reference(h->stream, h->d, h->d_stage_grid2, h->d_stage_grid, 2);
  CK(cudaMemcpyAsync(v_theta, h->d_stage_grid, G * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(v_phi, h->d_stage_grid + G, G * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "vector synthesis");
}

static int vector_analysis(gd_handle* h, const double* v_theta, const double* v_phi, double* tor_re, double* tor_im,
                           double* pol_re, double* pol_im, bool regular) {
  if (!h || !tor_re || !tor_im || !pol_re || !pol_im || !v_theta || !v_phi)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = stage_alloc(h);
  if (s) return s;
  const size_t plane = (size_t)h->d.nr * h->d.nlm, G = h->grid_elems();
  CK(cudaMemcpyAsync(h->d_stage_grid, v_theta, G * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_stage_grid + G, v_phi, G * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_grid_to_native(h->stream, h->d, h->d_stage_grid, h->d_stage_grid2, 2);
  double* tor = h->d_stage_spec2;
  double* pol = h->d_stage_spec2 + 2 * plane;
  if (h->precision == GD_PREC_MIXED) s = mixed_api_analysis_vector(h, h->d_stage_grid2, tor, pol);
  else s = analysis_vector(h, h->d_stage_grid2, tor, pol, EPI_VECTOR);
  if (s) return s;
  if (regular) zero_first_level(h, tor, 2, 2 * plane);
  launch_native_to_lmajor(h->stream, h->d, h->d_perm, h->d_stage_spec2, h->d_stage_spec, 4);
  double* dst[4] = {tor_re, tor_im, pol_re, pol_im};
  for (int i = 0; i < 4; ++i)
    CK(cudaMemcpyAsync(dst[i], h->d_stage_spec + plane * i, plane * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "vector analysis");
}

int gd_vector_analysis(gd_handle* h, const double* v_theta, const double* v_phi, double* tor_re, double* tor_im,
                       double* pol_re, double* pol_im) {
  return vector_analysis(h, v_theta, v_phi, tor_re, tor_im, pol_re, pol_im, false);
}

int gd_ball_vector_analysis(gd_handle* h, const double* v_theta, const double* v_phi, double* tor_re, double* tor_im,
                            double* pol_re, double* pol_im) {
  return vector_analysis(h, v_theta, v_phi, tor_re, tor_im, pol_re, pol_im, true);
}

// ---- the reference's argument lists on host arrays ----
namespace {
// host spectral planes (l-major) -> native layout at dst (through the l-major staging buffer)
int put_spec(gd_handle* h, const double* re, const double* im, double* dst) {
  const size_t plane = (size_t)h->d.nr * h->d.nlm;
  CK(cudaMemcpyAsync(h->d_stage_spec, re, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_stage_spec + plane, im, plane * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_lmajor_to_native(h->stream, h->d, h->d_perm, h->d_stage_spec, dst, 2);
  return check_launch(h, "upload");
}
// host grid (reference layout) -> native grid at dst
int put_grid(gd_handle* h, const double* g, double* dst) {
  CK(cudaMemcpyAsync(h->d_stage_grid, g, h->grid_elems() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_grid_to_native(h->stream, h->d, h->d_stage_grid, dst, 1);
  return check_launch(h, "grid upload");
}
int get_grid(gd_handle* h, const double* src, double* g) {
  launch_grid_to_reference(h->stream, h->d, src, h->d_stage_grid, 1);
  CK(cudaMemcpyAsync(g, h->d_stage_grid, h->grid_elems() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return check_launch(h, "grid download");
}
int nl_prepare(gd_handle* h) {
  CK(cudaSetDevice(h->device));
  return stage_alloc(h);
}
}  // namespace

struct gd_matrices {
  gd_handle* h = nullptr;
  double diffusivity = 0.0, dt = 0.0, theta = 0.0;
  double* d_nu = nullptr;   // the diffusivity
  double* d_lin = nullptr;  // L_l bands [col][band][l]
  double* d_lu = nullptr;   // LU factors of I/dt - theta L_l, same layout
};

int gd_create_timestepping_matrices(gd_handle* h, double diffusivity, double dt, double theta, gd_matrices** out) {
  if (!h || !out) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (!(dt > 0.0) || !std::isfinite(diffusivity) || !std::isfinite(theta))
    return fail(h, GD_ERR_ARG, "need dt > 0 and finite diffusivity and theta");
  if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "a standalone timestepping operator");
  CK(cudaSetDevice(h->device));
  const Dims& d = h->d;
  const size_t n = (size_t)d.nr * (2 * d.kl + 1) * (d.L + 1);
  gd_matrices* m = new gd_matrices();
  m->h = h;
  m->diffusivity = diffusivity;
  m->dt = dt;
  m->theta = theta;
  cudaError_t e = cudaMalloc(&m->d_nu, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&m->d_lin, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&m->d_lu, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_nu, &diffusivity, sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream);
  if (e == cudaSuccess) {
    launch_build_lu(h->stream, d.nr, d.kl, d.L, h->d_d1, h->d_d2, h->d_rinv, h->d_rinv2, m->d_nu, dt, theta, 0,
                    m->d_lin, m->d_lu, h->d_flag, 1);
    e = cudaGetLastError();
  }
  int flag = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess || flag) {
    gd_destroy_timestepping_matrices(m);
    if (e != cudaSuccess) return fail(h, GD_ERR_CUDA, std::string("timestepping matrices: ") + cudaGetErrorString(e));
    return fail(h, GD_ERR_SINGULAR, "zero pivot in a banded LU factorisation");
  }
  *out = m;
  return GD_OK;
}

int gd_destroy_timestepping_matrices(gd_matrices* m) {
  if (!m) return GD_ERR_ARG;
  cudaSetDevice(m->h->device);
  cudaFree(m->d_nu);
  cudaFree(m->d_lin);
  cudaFree(m->d_lu);
  delete m;
  return GD_OK;
}

// The CNAB2 column kernel on one field of host arrays: sweeps `stages` over
// the staged field in slot 0 of the second spectral staging buffer.
static int cnab2_host(gd_handle* h, const gd_matrices* m, double dt, int stages) {
  Cnab2Args a{};
  const size_t se = h->spec_elems();
  a.u[0] = h->d_stage_spec2;
  a.nl[0] = h->d_stage_spec2 + se;
  a.prev[0] = h->d_stage_spec2 + 2 * se;
  a.kind[0] = 0;
  a.nfield = 1;
  a.rowvals[0] = nullptr;  // no boundary rows of a given value
  a.inv_dt = 1.0 / dt;
  a.lin_weight = 1.0 - m->theta;
  a.dt = dt;
  a.stages = stages;
  { ProfScope p(h, "cnab2_solve"); launch_cnab2(h->stream, h->d, h->d_lof, h->d_d1, h->d_d2, h->d_rinv, h->d_rinv2, m->d_nu, m->d_lu, a); }
  return check_launch(h, "cnab2");
}

int gd_build_rhs_cnab2(gd_handle* h, const gd_matrices* m, double dt, const double* un_re, const double* un_im,
                       const double* nl_re, const double* nl_im, const double* prev_re, const double* prev_im,
                       double* rhs_re, double* rhs_im) {
  if (!h || !m || !un_re || !un_im || !nl_re || !nl_im || !prev_re || !prev_im || !rhs_re || !rhs_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (m->h != h) return fail(h, GD_ERR_ARG, "matrices belong to another handle");
  if (!(dt > 0.0)) return fail(h, GD_ERR_ARG, "need dt > 0");
  int s = nl_prepare(h);
  const size_t se = h->spec_elems();
  if (!s) s = put_spec(h, un_re, un_im, h->d_stage_spec2);
  if (!s) s = put_spec(h, nl_re, nl_im, h->d_stage_spec2 + se);
  if (!s) s = put_spec(h, prev_re, prev_im, h->d_stage_spec2 + 2 * se);
  if (!s) s = cnab2_host(h, m, dt, 1);
  return s ? s : download_spec(h, h->d_stage_spec2, rhs_re, rhs_im);
}

int gd_solve_implicit_step(gd_handle* h, const gd_matrices* m, const double* rhs_re, const double* rhs_im,
                           double* sol_re, double* sol_im) {
  if (!h || !m || !rhs_re || !rhs_im || !sol_re || !sol_im) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (m->h != h) return fail(h, GD_ERR_ARG, "matrices belong to another handle");
  int s = nl_prepare(h);
  if (!s) s = put_spec(h, rhs_re, rhs_im, h->d_stage_spec2);
  if (!s) s = cnab2_host(h, m, m->dt, 6);
  return s ? s : download_spec(h, h->d_stage_spec2, sol_re, sol_im);
}

int gd_compute_temperature_nonlinear(gd_handle* h, double* t_re, double* t_im, const double* u_theta,
                                     const double* u_phi, double* nl_re, double* nl_im, double* t_grid) {
  if (!h || !t_re || !t_im || !u_theta || !u_phi || !nl_re || !nl_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  int s = nl_prepare(h);
  if (!s) s = put_spec(h, t_re, t_im, h->field(F_TEMP));
  if (!s) s = put_grid(h, u_theta, h->grid(GD_GRID_U_TH));
  if (!s) s = put_grid(h, u_phi, h->grid(GD_GRID_U_PH));
  if (!s) s = temperature_nl_fp64(h);
  if (!s) s = download_spec(h, h->nlf(F_TEMP), nl_re, nl_im);
  if (!s) s = download_spec(h, h->field(F_TEMP), t_re, t_im);
  if (!s && t_grid) s = get_grid(h, h->grid(GD_GRID_T), t_grid);
  return s;
}

int gd_compute_composition_nonlinear(gd_handle* h, double* c_re, double* c_im, const double* u_theta,
                                     const double* u_phi, double* nl_re, double* nl_im, double* c_grid) {
  if (!h || !c_re || !c_im || !u_theta || !u_phi || !nl_re || !nl_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  if (!h->c.composition) return fail(h, GD_ERR_STATE, "the configuration has no composition");
  int s = nl_prepare(h);
  if (!s) s = put_spec(h, c_re, c_im, h->field(F_COMP));
  if (!s) s = put_grid(h, u_theta, h->grid(GD_GRID_U_TH));
  if (!s) s = put_grid(h, u_phi, h->grid(GD_GRID_U_PH));
  if (!s) s = composition_nl_fp64(h);
  if (!s) s = download_spec(h, h->nlf(F_COMP), nl_re, nl_im);
  if (!s) s = download_spec(h, h->field(F_COMP), c_re, c_im);
  if (!s && c_grid) s = get_grid(h, h->grid(GD_GRID_C), c_grid);
  return s;
}

int gd_compute_velocity_nonlinear(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                                  const double* pol_im, const double* j_theta, const double* j_phi,
                                  const double* b_theta, const double* b_phi, double* nl_tor_re, double* nl_tor_im,
                                  double* nl_pol_re, double* nl_pol_im, double* u_theta, double* u_phi) {
  if (!h || !tor_re || !tor_im || !pol_re || !pol_im || !nl_tor_re || !nl_tor_im || !nl_pol_re || !nl_pol_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  const bool grids = j_theta && j_phi && b_theta && b_phi;
  if (h->c.magnetic && !grids) return fail(h, GD_ERR_ARG, "the Lorentz term needs the j and B grids");
  int s = nl_prepare(h);
  if (!s) s = put_spec(h, tor_re, tor_im, h->field(F_UTOR));
  if (!s) s = put_spec(h, pol_re, pol_im, h->field(F_UPOL));
  if (!s && grids) s = put_grid(h, j_theta, h->grid(GD_GRID_J_TH));
  if (!s && grids) s = put_grid(h, j_phi, h->grid(GD_GRID_J_PH));
  if (!s && grids) s = put_grid(h, b_theta, h->grid(GD_GRID_B_TH));
  if (!s && grids) s = put_grid(h, b_phi, h->grid(GD_GRID_B_PH));
  if (!s) s = velocity_nl_fp64(h);
  if (!s) s = download_spec(h, h->nlf(F_UTOR), nl_tor_re, nl_tor_im);
  if (!s) s = download_spec(h, h->nlf(F_UPOL), nl_pol_re, nl_pol_im);
  if (!s && u_theta) s = get_grid(h, h->grid(GD_GRID_U_TH), u_theta);
  if (!s && u_phi) s = get_grid(h, h->grid(GD_GRID_U_PH), u_phi);
  return s;
}

int gd_compute_magnetic_nonlinear(gd_handle* h, const double* tor_re, const double* tor_im, const double* pol_re,
                                  const double* pol_im, const double* u_theta, const double* u_phi,
                                  double* nl_tor_re, double* nl_tor_im, double* nl_pol_re, double* nl_pol_im,
                                  double* b_theta, double* b_phi, double* j_theta, double* j_phi) {
  if (!h || !tor_re || !tor_im || !pol_re || !pol_im || !u_theta || !u_phi || !nl_tor_re || !nl_tor_im ||
      !nl_pol_re || !nl_pol_im)
    return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  int s = nl_prepare(h);
  if (!s) s = put_spec(h, tor_re, tor_im, h->field(F_BTOR));
  if (!s) s = put_spec(h, pol_re, pol_im, h->field(F_BPOL));
  if (!s) s = put_grid(h, u_theta, h->grid(GD_GRID_U_TH));
  if (!s) s = put_grid(h, u_phi, h->grid(GD_GRID_U_PH));
  if (!s) s = magnetic_nl_fp64(h);
  if (!s) s = download_spec(h, h->nlf(F_BTOR), nl_tor_re, nl_tor_im);
  if (!s) s = download_spec(h, h->nlf(F_BPOL), nl_pol_re, nl_pol_im);
  if (!s && b_theta) s = get_grid(h, h->grid(GD_GRID_B_TH), b_theta);
  if (!s && b_phi) s = get_grid(h, h->grid(GD_GRID_B_PH), b_phi);
  if (!s && j_theta) s = get_grid(h, h->grid(GD_GRID_J_TH), j_theta);
  if (!s && j_phi) s = get_grid(h, h->grid(GD_GRID_J_PH), j_phi);
  return s;
}

int gd_temperature_nonlinear(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = temperature_nl(h);
  if (s) return s;
  h->last_nl_par = h->nl_par;
  CK(cudaStreamSynchronize(h->stream));
  return h->precision == GD_PREC_MIXED ? mixed_check_error(h) : GD_OK;
}
int gd_velocity_nonlinear(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = velocity_nl(h);
  if (s) return s;
  h->last_nl_par = h->nl_par;
  CK(cudaStreamSynchronize(h->stream));
  return h->precision == GD_PREC_MIXED ? mixed_check_error(h) : GD_OK;
}
int gd_magnetic_nonlinear(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int s = magnetic_nl(h);
  if (s) return s;
  h->last_nl_par = h->nl_par;
  CK(cudaStreamSynchronize(h->stream));
  return h->precision == GD_PREC_MIXED ? mixed_check_error(h) : GD_OK;
}
int gd_composition_nonlinear(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  if (!h->c.composition) return fail(h, GD_ERR_STATE, "the configuration has no composition");
  CK(cudaSetDevice(h->device));
  int s = composition_nl(h);
  if (s) return s;
  h->last_nl_par = h->nl_par;
  CK(cudaStreamSynchronize(h->stream));
  return h->precision == GD_PREC_MIXED ? mixed_check_error(h) : GD_OK;
}
int gd_implicit_step(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  const int boot = (h->c.ab_mode == 1 || h->step_count == 0) ? 1 : 0;
  int s = implicit_launch(h, boot);
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  end_step(h);
  return GD_OK;
}

int gd_step_async(gd_handle* h, int nsteps) {
  if (!h || nsteps < 0) return h ? fail(h, GD_ERR_ARG, "nsteps must be >= 0") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  for (int i = 0; i < nsteps; ++i) {
    const int boot = (h->c.ab_mode == 1 || h->step_count == 0) ? 1 : 0;
    if (h->profiling) {
      int s = step_sequence(h, boot);
      if (s) return s;
    } else {
      int s = ensure_graph(h, boot);
      if (s) return s;
      CK(cudaGraphLaunch(h->gexec[h->nl_par][boot], h->stream));
    }
    end_step(h);
  }
  return GD_OK;
}

int gd_step(gd_handle* h, int nsteps) {
  int s = gd_step_async(h, nsteps);
  if (s) return s;
  CK(cudaStreamSynchronize(h->stream));
  if (h->precision == GD_PREC_MIXED) return mixed_check_error(h);
  return GD_OK;
}

int gd_set_dt(gd_handle* h, double dt) {
  if (!h || !(dt > 0.0)) return h ? fail(h, GD_ERR_ARG, "dt must be positive") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  h->c.dt = dt;
  drop_graphs(h);
  int s = build_implicit(h);
  if (s == GD_OK && h->scheme != GD_SCHEME_CNAB2) s = build_etd(h);
  return s;
}

int gd_set_scheme(gd_handle* h, int scheme) {
  if (!h || (scheme != GD_SCHEME_CNAB2 && scheme != GD_SCHEME_EAB2 && scheme != GD_SCHEME_ERK2))
    return h ? fail(h, GD_ERR_ARG, "scheme must be GD_SCHEME_CNAB2, GD_SCHEME_EAB2 or GD_SCHEME_ERK2") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (scheme != GD_SCHEME_CNAB2) {
    if (h->d.nseg > 1 || h->d.ball) return refuse_layout(h, "an exponential scheme");
    if (h->c.bc_mode == 2)
      return fail(h, GD_ERR_UNSUPPORTED,
                  "the exponential schemes have no boundary rows (bc_mode 2 is a CNAB2 operator option)");
    if (h->d.nr > 256) return fail(h, GD_ERR_UNSUPPORTED, "the exponential schemes support nr <= 256");
    if (scheme == GD_SCHEME_ERK2 && !h->d_erk2) AL(h->d_erk2, 2 * NFIELD * h->spec_elems());
    int s = build_etd(h);
    if (s) return s;
  }
  if (scheme != h->scheme) drop_graphs(h);
  h->scheme = scheme;
  return GD_OK;
}

int gd_download_etd(gd_handle* h, int kind, int l, int which, double* out) {
  if (!h || !out || kind < 0 || kind > (h && h->c.composition ? 3 : 2) || l < 0 || l > h->d.L || which < 0 ||
      which > 4)
    return h ? fail(h, GD_ERR_ARG, "bad kind, degree, matrix or pointer") : GD_ERR_ARG;
  if (h->scheme == GD_SCHEME_CNAB2 || !h->d_etd) return fail(h, GD_ERR_ARG, "no exponential scheme is selected");
  CK(cudaSetDevice(h->device));
  const size_t n = h->d.nr, n2 = n * n;
  std::vector<double> t(n2);
  CK(cudaMemcpyAsync(t.data(), h->d_etd + ((size_t)(kind * (h->d.L + 1) + l) * 5 + which) * n2, n2 * sizeof(double),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < n; ++i)
    for (size_t k = 0; k < n; ++k) out[i * n + k] = t[k * n + i];
  return GD_OK;
}

int gd_energy(gd_handle* h, double* ekin, double* emag) {
  if (!h || !ekin || !emag) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  launch_energy(h->stream, h->d, h->d_lof, h->field(F_UTOR), h->field(F_UPOL), h->c.magnetic ? h->field(F_BTOR) : nullptr,
                h->field(F_BPOL), h->d_epart, h->d_eout);
  std::vector<double> e(2 * (size_t)h->d.nseg);
  CK(cudaMemcpyAsync(e.data(), h->d_eout, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // a segmented handle: the sum over its segments
  *ekin = e[0];
  *emag = e[1];
  for (int g = 1; g < h->d.nseg; ++g) {
    *ekin += e[2 * g];
    *emag += e[2 * g + 1];
  }
  return check_launch(h, "energy");
}

int gd_segment_energy(gd_handle* h, double* ekin, double* emag) {
  if (!h || !ekin || !emag) return h ? fail(h, GD_ERR_ARG, "null pointer") : GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  launch_energy(h->stream, h->d, h->d_lof, h->field(F_UTOR), h->field(F_UPOL), h->c.magnetic ? h->field(F_BTOR) : nullptr,
                h->field(F_BPOL), h->d_epart, h->d_eout);
  std::vector<double> e(2 * (size_t)h->d.nseg);
  CK(cudaMemcpyAsync(e.data(), h->d_eout, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int g = 0; g < h->d.nseg; ++g) {
    ekin[g] = e[2 * g];
    emag[g] = e[2 * g + 1];
  }
  return check_launch(h, "segment energy");
}

int gd_check_finite(gd_handle* h) {
  if (!h) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  launch_check_finite(h->stream, nfields(h) * h->spec_elems(), h->d_state, h->d_flag);
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag) return fail(h, GD_ERR_NONFINITE, "non-finite value in the spectral state");
  return check_launch(h, "check_finite");
}

long gd_step_count(const gd_handle* h) { return h ? h->step_count : -1; }

int gd_get_stream(gd_handle* h, void** stream) {
  if (!h || !stream) return GD_ERR_ARG;
  *stream = (void*)h->stream;
  return GD_OK;
}

int gd_profile_enable(gd_handle* h, int enable) {
  if (!h) return GD_ERR_ARG;
  h->profiling = enable != 0;
  return GD_OK;
}

int gd_profile_read(gd_handle* h, int max, char* names, double* ms, int* launches, int* count) {
  if (!h || !count || max < 0) return GD_ERR_ARG;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  for (auto& p : h->prof_pending) {
    float t = 0.f;
    cudaEventElapsedTime(&t, p.a, p.b);
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
    size_t k = 0;
    while (k < h->prof_names.size() && h->prof_names[k] != p.name) ++k;
    if (k == h->prof_names.size()) { h->prof_names.push_back(p.name); h->prof_ms.push_back(0.0); h->prof_count.push_back(0); }
    h->prof_ms[k] += t;
    h->prof_count[k] += 1;
  }
  h->prof_pending.clear();
  const int n = (int)h->prof_names.size();
  *count = n;
  for (int k = 0; k < n && k < max; ++k) {
    if (names) { std::strncpy(names + 32 * k, h->prof_names[k].c_str(), 31); names[32 * k + 31] = 0; }
    if (ms) ms[k] = h->prof_ms[k];
    if (launches) launches[k] = h->prof_count[k];
  }
  h->prof_names.clear(); h->prof_ms.clear(); h->prof_count.clear();
  return GD_OK;
}

// ---- batched ensemble ----------------------------------------------------------
struct gd_ensemble {
  std::vector<gd_handle*> members;
  int device = 0;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t gexec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [nl_par][boot]
  std::vector<int> gens;  // members' graph generations the ensemble graphs were captured at
  int failed = -1;
};

int gd_ensemble_destroy(gd_ensemble* e) {
  if (!e) return GD_ERR_ARG;
  cudaSetDevice(e->device);
  if (e->master) cudaStreamSynchronize(e->master);
  for (int p = 0; p < 2; ++p)
    for (int i = 0; i < 2; ++i)
      if (e->gexec[p][i]) cudaGraphExecDestroy(e->gexec[p][i]);
  for (gd_handle* h : e->members) gd_destroy(h);
  for (cudaEvent_t ev : e->joins) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->master) cudaStreamDestroy(e->master);
  delete e;
  return GD_OK;
}

int gd_ensemble_create(const gd_config* cfgs, int n, int device, gd_ensemble** out) {
  if (!cfgs || !out || n <= 0) return GD_ERR_ARG;
  *out = nullptr;
  gd_ensemble* e = new gd_ensemble();
  e->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&e->master, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
    gd_ensemble_destroy(e);
    return GD_ERR_CUDA;
  }
  for (int i = 0; i < n; ++i) {
    gd_handle* h = nullptr;
    const int s = gd_create(&cfgs[i], device, &h);
    if (s != GD_OK) {
      fprintf(stderr, "gd_ensemble_create: member %d: status %d\n", i, s);
      gd_ensemble_destroy(e);
      return s;
    }
    e->members.push_back(h);
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      gd_ensemble_destroy(e);
      return GD_ERR_CUDA;
    }
    e->joins.push_back(ev);
  }
  *out = e;
  return GD_OK;
}

int gd_ensemble_size(const gd_ensemble* e) { return e ? (int)e->members.size() : -1; }

gd_handle* gd_ensemble_member(gd_ensemble* e, int i) {
  return (e && i >= 0 && i < (int)e->members.size()) ? e->members[i] : nullptr;
}

int gd_ensemble_failed_member(const gd_ensemble* e) { return e ? e->failed : -1; }

int gd_ensemble_get_stream(gd_ensemble* e, void** stream) {
  if (!e || !stream) return GD_ERR_ARG;
  *stream = (void*)e->master;
  return GD_OK;
}

// One graph: fork from the master stream to every member's stream, each
// member's step sequence, join back.
static int ensemble_graph(gd_ensemble* e, int par, int boot) {
  bool stale = e->gens.size() != e->members.size();
  for (size_t i = 0; i < e->members.size() && !stale; ++i) stale = e->gens[i] != e->members[i]->graph_gen;
  if (stale) {  // a member's parameters, precision or dt changed since the capture
    for (int p = 0; p < 2; ++p)
      for (int b = 0; b < 2; ++b)
        if (e->gexec[p][b]) { cudaGraphExecDestroy(e->gexec[p][b]); e->gexec[p][b] = nullptr; }
    e->gens.clear();
    for (gd_handle* h : e->members) e->gens.push_back(h->graph_gen);
  }
  if (e->gexec[par][boot]) return GD_OK;
  if (cudaStreamBeginCapture(e->master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return GD_ERR_CUDA;
  int st = GD_OK;
  cudaError_t ce = cudaEventRecord(e->fork, e->master);
  for (size_t i = 0; i < e->members.size() && st == GD_OK && ce == cudaSuccess; ++i) {
    gd_handle* h = e->members[i];
    ce = cudaStreamWaitEvent(h->stream, e->fork, 0);
    if (ce != cudaSuccess) break;
    st = step_sequence(h, boot);
    if (st != GD_OK) { e->failed = (int)i; break; }
    ce = cudaEventRecord(e->joins[i], h->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->master, e->joins[i], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(e->master, &g);
  if (st != GD_OK || ce != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return st != GD_OK ? st : GD_ERR_CUDA;
  }
  const cudaError_t ie = cudaGraphInstantiate(&e->gexec[par][boot], g, 0);
  cudaGraphDestroy(g);
  return ie == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

int gd_ensemble_step_async(gd_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return GD_ERR_ARG;
  if (cudaSetDevice(e->device) != cudaSuccess) return GD_ERR_CUDA;
  e->failed = -1;
  for (int k = 0; k < nsteps; ++k) {
    int boot = -1, par = -1;
    bool together = true;
    for (gd_handle* h : e->members) {
      const int b = (h->c.ab_mode == 1 || h->step_count == 0) ? 1 : 0;
      if (boot < 0) { boot = b; par = h->nl_par; }
      if (b != boot || h->nl_par != par || h->profiling) together = false;
    }
    if (together) {
      // the members' streams may still run work queued outside the ensemble
      for (gd_handle* h : e->members) {
        cudaEvent_t ev = e->joins[0];
        if (cudaEventRecord(ev, h->stream) != cudaSuccess || cudaStreamWaitEvent(e->master, ev, 0) != cudaSuccess)
          return GD_ERR_CUDA;
      }
      const int s = ensemble_graph(e, par, boot);
      if (s != GD_OK) return s;
      if (cudaGraphLaunch(e->gexec[par][boot], e->master) != cudaSuccess) return GD_ERR_CUDA;
      for (gd_handle* h : e->members) end_step(h);
    } else {
      // each member's stream first waits for the ensemble's earlier graph launches
      if (cudaEventRecord(e->fork, e->master) != cudaSuccess) return GD_ERR_CUDA;
      for (gd_handle* h : e->members)
        if (cudaStreamWaitEvent(h->stream, e->fork, 0) != cudaSuccess) return GD_ERR_CUDA;
      for (size_t i = 0; i < e->members.size(); ++i) {
        const int s = gd_step_async(e->members[i], 1);
        if (s != GD_OK) { e->failed = (int)i; return s; }
        // later graph launches on the master stream wait for this member
        if (cudaEventRecord(e->joins[i], e->members[i]->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->master, e->joins[i], 0) != cudaSuccess)
          return GD_ERR_CUDA;
      }
    }
  }
  return GD_OK;
}

// Launch-shape search for an ensemble: candidate caps of the members'
// tensor-core grids, each timed over nsteps graph-launched ensemble steps of a
// scratch ensemble with the same configurations, precisions and schemes (the
// caller's members are never stepped); the fastest is applied to the members.
// Candidates: one cap for every member (one CTA per SM, 74, 37, 18, 8, 4), and
// caps proportional to each member's share of the Legendre work
// (lmax + 1)^3 nr, scaled by 2, 4, 8 and 16 SMs' worth.
int gd_ensemble_autotune(gd_ensemble* e, int nsteps, float* best_ms, int* caps_out) {
  if (!e || nsteps < 1) return GD_ERR_ARG;
  if (cudaSetDevice(e->device) != cudaSuccess) return GD_ERR_CUDA;
  const int n = (int)e->members.size();
  std::vector<gd_config> cfgs(n);
  for (int i = 0; i < n; ++i) {
    cfgs[i] = e->members[i]->c;
    // the member's segment lengths (the caller's array was read at creation only)
    if (e->members[i]->d.nseg > 1) cfgs[i].segment_nr = e->members[i]->seg_n.data();
    cfgs[i].precision = GD_PREC_FP64;  // set below, with the member's stages
  }
  gd_ensemble* t = nullptr;
  int st = gd_ensemble_create(cfgs.data(), n, e->device, &t);
  if (st != GD_OK) return st;
  for (int i = 0; i < n && st == GD_OK; ++i) {
    gd_handle* src = e->members[i];
    gd_handle* h = t->members[i];
    if (src->precision != GD_PREC_FP64) st = gd_set_precision(h, src->precision);
    if (st == GD_OK) st = gd_set_int8_digits(h, src->int8_digits);
    if (st == GD_OK) st = gd_set_fp64_stages(h, src->fp64_stages);
    if (st == GD_OK && src->scheme != h->scheme) st = gd_set_scheme(h, src->scheme);
  }
  const int sms = current_sm_count();
  std::vector<double> w(n);
  double wsum = 0.0;
  for (int i = 0; i < n; ++i) {
    const double l1 = e->members[i]->d.L + 1.0;
    w[i] = l1 * l1 * l1 * e->members[i]->d.nr;
    wsum += w[i];
  }
  std::vector<std::vector<int>> cands;
  for (int cap : {0, 74, 37, 18, 8, 4}) cands.push_back(std::vector<int>(n, cap < sms ? cap : 0));
  for (int c : {2, 4, 8, 16}) {
    std::vector<int> v(n);
    for (int i = 0; i < n; ++i) v[i] = std::max(1, std::min(sms, (int)std::lround(sms * c * w[i] / wsum)));
    cands.push_back(v);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (st == GD_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) st = GD_ERR_CUDA;
  float best = -1.f;
  size_t besti = 0;
  for (size_t c = 0; c < cands.size() && st == GD_OK; ++c) {
    for (int i = 0; i < n && st == GD_OK; ++i) st = gd_set_launch_shape(t->members[i], cands[c][i]);
    if (st == GD_OK) st = gd_ensemble_step(t, 2);  // captures the graphs of this shape
    if (st != GD_OK) break;
    float ms = 0.f;
    if (cudaEventRecord(e0, t->master) != cudaSuccess) { st = GD_ERR_CUDA; break; }
    st = gd_ensemble_step_async(t, nsteps);
    if (st != GD_OK) break;
    if (cudaEventRecord(e1, t->master) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { st = GD_ERR_CUDA; break; }
    st = gd_ensemble_step(t, 0);  // error flags of the timed steps
    if (st == GD_OK && (best < 0.f || ms < best)) { best = ms; besti = c; }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  gd_ensemble_destroy(t);
  if (st != GD_OK) return st;
  for (int i = 0; i < n && st == GD_OK; ++i) st = gd_set_launch_shape(e->members[i], cands[besti][i]);
  if (st != GD_OK) return st;
  if (best_ms) *best_ms = best / nsteps;
  if (caps_out)
    for (int i = 0; i < n; ++i) caps_out[i] = cands[besti][i];
  return GD_OK;
}

int gd_ensemble_step(gd_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return GD_ERR_ARG;
  int st = gd_ensemble_step_async(e, nsteps);
  if (st != GD_OK) return st;
  if (cudaStreamSynchronize(e->master) != cudaSuccess) return GD_ERR_CUDA;
  for (size_t i = 0; i < e->members.size(); ++i) {
    gd_handle* h = e->members[i];
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) { e->failed = (int)i; return GD_ERR_CUDA; }
    if (h->precision == GD_PREC_MIXED) {
      const int s = mixed_check_error(h);
      if (s != GD_OK) { e->failed = (int)i; return s; }
    }
  }
  return GD_OK;
}

}  // extern "C"

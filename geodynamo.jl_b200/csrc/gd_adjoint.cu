// gd_adjoint.cu -- reverse-mode pieces of the step: the pullback of the
// implicit CNAB2 propagator of a field whose nonlinear term is identically
// zero, and the scalings that turn the Gauss analysis into the transpose of
// the scalar synthesis.
//
// In the reference's step the vector syntheses write only the theta and phi
// components (src/shtnskit_field_functions.jl:264-279), so u x B
// (src/magnetic.jl:375-404) and j x B (src/velocity.jl:638-672) are products
// with a zero radial factor in every term: the magnetic nonlinear term is zero
// and neither product depends on B or u to first order.  A magnetic field
// component therefore evolves by its implicit operator alone,
//   B^(n+1) = M B^n,  M = S^-1 R  (bc_mode 0),  P_c S^-1 R  (bc_mode 1: rows
//   0 and nr-1 zeroed after the solve),  S_D^-1 D R  (bc_mode 2: Dirichlet rows
//   in S, boundary rows of the right-hand side zeroed),
// with S = I/dt - theta L_l (banded LU, src/timestep.jl:498-543,
// src/linear_algebra.jl:23-88) and R = I/dt + (1 - theta) L_l
// (build_rhs_cnab2!, src/timestep.jl:610-690), the same matrix for every step
// (the Adams-Bashforth terms vanish with the nonlinear term), independent of
// the rest of the state.  Its pullback is lambda <- M^T lambda per step.
#include "gd_internal.cuh"

namespace gd {

constexpr int PB_THREADS = 64;  // columns per block; each keeps its column in shared memory

// One thread per (l, m) column and Re/Im plane: nsteps applications of M^T to
// lambda (native layout [plane][r][j], updated in place).  Band entries (row i,
// column c) of the factors and of L_l sit at [(c nbw + kl + i - c)(L + 1) + l]
// (k_build_lu); the LU is S = L_f U_f with unit L_f.
template <int KL>
__global__ void __launch_bounds__(PB_THREADS) k_cnab2_pullback(Dims d, const int* __restrict__ lof,
                                                              const double* __restrict__ lin,
                                                              const double* __restrict__ lu, int kind, double inv_dt,
                                                              double lin_weight, int clamp_rows, int bc_rows,
                                                              int nsteps, double* __restrict__ lam) {
  constexpr int NB = 2 * KL + 1;
  extern __shared__ double col_s[];  // [nr][PB_THREADS]
  const int N = d.nr;
  const int tid = threadIdx.x;
  const int j = blockIdx.x * PB_THREADS + tid;
  const int plane = blockIdx.y;
  if (j >= d.nlm) return;
  const size_t NM = d.nlm, Lp1 = (size_t)d.L + 1;
  const int l = lof[j];
  const double* F = lu + (size_t)kind * N * NB * Lp1 + l;
  const double* Lb = lin + (size_t)kind * N * NB * Lp1 + l;
  auto band = [&](const double* B, int i, int c) { return B[((size_t)c * NB + (KL + i - c)) * Lp1]; };
  double* g = lam + (size_t)plane * N * NM + j;
  double* x = col_s + tid;  // x[i * PB_THREADS]
  for (int i = 0; i < N; ++i) x[i * PB_THREADS] = g[(size_t)i * NM];

  for (int s = 0; s < nsteps; ++s) {
    if (clamp_rows) {
      x[0] = 0.0;
      x[(N - 1) * PB_THREADS] = 0.0;
    }
    // U_f^T w = x (forward): w_i = (x_i - sum_{k<i} U_f[k][i] w_k) / U_f[i][i]
    for (int i = 0; i < N; ++i) {
      double acc = x[i * PB_THREADS];
#pragma unroll
      for (int t = KL; t >= 1; --t) {
        const int k = i - t;
        if (k >= 0) acc -= band(F, k, i) * x[k * PB_THREADS];
      }
      x[i * PB_THREADS] = acc / band(F, i, i);
    }
    // L_f^T z = w (backward, unit diagonal): z_i = w_i - sum_{k>i} L_f[k][i] z_k
    for (int i = N - 1; i >= 0; --i) {
      double acc = x[i * PB_THREADS];
#pragma unroll
      for (int t = KL; t >= 1; --t) {
        const int k = i + t;
        if (k < N) acc -= band(F, k, i) * x[k * PB_THREADS];
      }
      x[i * PB_THREADS] = acc;
    }
    if (bc_rows) {
      x[0] = 0.0;
      x[(N - 1) * PB_THREADS] = 0.0;
    }
    // lambda = R^T z: lambda_i = z_i / dt + (1 - theta) sum_k L_l[k][i] z_k, in
    // place with a window of the z values still needed
    double win[NB];  // win[t] = z_(i - KL + t)
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int k = t - KL;
      win[t] = (k >= 0 && k < N) ? x[k * PB_THREADS] : 0.0;
    }
    for (int i = 0; i < N; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int k = i - KL + t;
        if (k >= 0 && k < N) acc += band(Lb, k, i) * win[t];
      }
      x[i * PB_THREADS] = inv_dt * win[KL] + lin_weight * acc;
#pragma unroll
      for (int t = 0; t < NB - 1; ++t) win[t] = win[t + 1];
      const int nxt = i + KL + 1;
      win[NB - 1] = nxt < N ? x[nxt * PB_THREADS] : 0.0;
    }
  }
  for (int i = 0; i < N; ++i) g[(size_t)i * NM] = x[i * PB_THREADS];
}

void launch_cnab2_pullback(cudaStream_t s, const Dims& d, const int* lof, const double* lin, const double* lu,
                           int kind, double dt, double theta, int clamp_rows, int bc_rows, int nsteps, double* lam) {
  const size_t smem = (size_t)d.nr * PB_THREADS * sizeof(double);
  allow_dynamic_smem(k_cnab2_pullback<GD_MAX_KL>, smem);
  dim3 grid(ceil_div(d.nlm, PB_THREADS), 2);
  k_cnab2_pullback<GD_MAX_KL><<<grid, PB_THREADS, smem, s>>>(d, lof, lin, lu, kind, 1.0 / dt, 1.0 - theta, clamp_rows,
                                                             bc_rows, nsteps, lam);
}

// Transpose of the scalar synthesis through the Gauss analysis A:
//   S^T g = c_m (nlon / 2 pi) A(g / w_theta),  c_0 = 1, c_m = 2 (m > 0):
// the analysis weights each colatitude by w_theta and the phi transform by
// 2 pi / nlon, while the real-field synthesis counts each m > 0 twice.
// Grid in the reference layout (theta fastest).
__global__ void k_divide_by_weights(size_t n, int nlat, const double* __restrict__ w, double* __restrict__ g) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    g[e] = g[e] / w[e % nlat];
}
// Spectral rows in the native layout (mode j fastest), mof[j] = m.
__global__ void k_scale_by_order(size_t nrows, int nlm, const int* __restrict__ mof, double f0, double f1,
                                 double* __restrict__ a) {
  const size_t n = nrows * (size_t)nlm;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    a[e] *= mof[e % nlm] == 0 ? f0 : f1;
}

void launch_divide_by_weights(cudaStream_t s, size_t n, int nlat, const double* w, double* g) {
  k_divide_by_weights<<<592, 256, 0, s>>>(n, nlat, w, g);
}
void launch_scale_by_order(cudaStream_t s, size_t nrows, int nlm, const int* mof, double f0, double f1, double* a) {
  k_scale_by_order<<<592, 256, 0, s>>>(nrows, nlm, mof, f0, f1, a);
}

// a *= f l(l+1) (inverse 0) or f / (l(l+1)) with 0 at l = 0 (inverse 1), per
// native mode j of every row
__global__ void k_scale_by_degree(size_t nrows, int nlm, const int* __restrict__ lof, double f, int inverse,
                                  double* __restrict__ a) {
  const size_t n = nrows * (size_t)nlm;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int l = lof[e % nlm];
    const double lf = (double)l * (l + 1.0);
    a[e] *= inverse ? (l > 0 ? f / lf : 0.0) : f * lf;
  }
}

void launch_scale_by_degree(cudaStream_t s, size_t nrows, int nlm, const int* lof, double f, int inverse, double* a) {
  k_scale_by_degree<<<592, 256, 0, s>>>(nrows, nlm, lof, f, inverse, a);
}

// ---------------------------------------------------------------------------
// Adjoint of the temperature step (reverse mode of step_once! with respect to
// the temperature).  In the reference's step the temperature obeys
//   T^(n+1) = C S^-1 D (R P T^n + a_n N_n T^n - b_n N_(n-1) T^(n-1)) + const
// (compute_temperature_nonlinear!, src/thermal.jl:149-190; build_rhs_cnab2! +
// solve_implicit_step!, src/timestep.jl:610-730), where P sets the fixed-value
// boundary rows (a constant: their rows of the Jacobian vanish), R = I/dt +
// (1 - theta) L_l, S = I/dt - theta L_l, C zeroes rows 0 and nr - 1 after the
// solve (bc_mode 1), D replaces the right-hand side's boundary rows by
// constants (bc_mode 2), a_n = 1.5 (1 on the Adams-Bashforth start),
// b_n = 0.5 (0 on the start), and N_n T = An(-(u_th Syn(G_th T) +
// u_ph Syn(G_ph T))) is the advection by the velocity grids of step n, linear in
// T (u_r = 0: the radial term vanishes; the sources are constant).
// ---------------------------------------------------------------------------

// One thread per (l, m) column and plane (blockIdx.y):
//   mode 0: y = D S^-T C x   (transposed banded solve with the LU factors);
//   mode 1: y = P R^T x      (types[j] / types[nlm + j]: inner / outer boundary
//                             type of the mode; GD_BC_VALUE rows are zeroed).
template <int KL>
__global__ void __launch_bounds__(128) k_cnab2_adjoint(Dims d, const int* __restrict__ lof, const double* __restrict__ lin,
                                                      const double* __restrict__ lu, const int* __restrict__ types,
                                                      int kind, int mode, double inv_dt, double lin_weight,
                                                      int clamp_rows, int bc_rows, const double* __restrict__ x,
                                                      double* __restrict__ y) {
  constexpr int NB = 2 * KL + 1;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.nlm) return;
  const int N = d.nr;
  const size_t NM = d.nlm, Lp1 = (size_t)d.L + 1, off = (size_t)blockIdx.y * N * NM + j;
  const int l = lof[j];
  const double* F = lu + (size_t)kind * N * NB * Lp1 + l;
  const double* Lb = lin + (size_t)kind * N * NB * Lp1 + l;
  auto band = [&](const double* B, int i, int c) { return B[((size_t)c * NB + (KL + i - c)) * Lp1]; };
  const double* xc = x + off;
  double* yc = y + off;
  if (mode == 0) {
    // C x, then U_f^T w = C x (forward), L_f^T z = w (backward, unit diagonal), then D
    for (int i = 0; i < N; ++i) {
      double acc = (clamp_rows && (i == 0 || i == N - 1)) ? 0.0 : xc[(size_t)i * NM];
#pragma unroll
      for (int t = KL; t >= 1; --t) {
        const int k = i - t;
        if (k >= 0) acc -= band(F, k, i) * yc[(size_t)k * NM];
      }
      yc[(size_t)i * NM] = acc / band(F, i, i);
    }
    for (int i = N - 1; i >= 0; --i) {
      double acc = yc[(size_t)i * NM];
#pragma unroll
      for (int t = KL; t >= 1; --t) {
        const int k = i + t;
        if (k < N) acc -= band(F, k, i) * yc[(size_t)k * NM];
      }
      yc[(size_t)i * NM] = acc;
    }
    if (bc_rows) {
      yc[0] = 0.0;
      yc[(size_t)(N - 1) * NM] = 0.0;
    }
  } else {
    // R^T x: y_i = x_i / dt + (1 - theta) sum_k L_l[k][i] x_k, then P
    for (int i = 0; i < N; ++i) {
      double acc = 0.0;
      for (int k = i - KL < 0 ? 0 : i - KL; k <= i + KL && k < N; ++k) acc += band(Lb, k, i) * xc[(size_t)k * NM];
      double v = inv_dt * xc[(size_t)i * NM] + lin_weight * acc;
      // P: the scalar fields' fixed-value rows (no projection for the potentials, types null)
      if (types && ((i == 0 && types[j] == GD_BC_VALUE) || (i == N - 1 && types[NM + j] == GD_BC_VALUE))) v = 0.0;
      yc[(size_t)i * NM] = v;
    }
  }
}

void launch_cnab2_adjoint(cudaStream_t s, const Dims& d, const int* lof, const double* lin, const double* lu,
                          const int* types, int kind, int mode, double dt, double theta, int clamp_rows, int bc_rows,
                          const double* x, double* y) {
  dim3 grid(ceil_div(d.nlm, 128), 2);
  k_cnab2_adjoint<GD_MAX_KL><<<grid, 128, 0, s>>>(d, lof, lin, lu, types, kind, mode, 1.0 / dt, 1.0 - theta,
                                                   clamp_rows, bc_rows, x, y);
}

// out = G_th^T gth + G_ph^T gph for every shell (native layout [plane][r][j]):
// the transpose of the theta recurrence (couples (l -+ 1, m), the neighbouring
// native indices of the same order) and of the phi derivative (i m), both
// divided by r as in k_gradients.
__global__ void k_gradients_adjoint(Dims d, const int* __restrict__ lof, const int* __restrict__ mof,
                                    const double* __restrict__ rinv, const double* __restrict__ gth,
                                    const double* __restrict__ gph, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (j >= d.nlm || k >= d.nr) return;
  const int l = lof[j], m = mof[j];
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM, at = (size_t)k * NM + j;
  // forward: gth_j = (Ap(l) T_(l+1) + Am(l) T_(l-1)) / r with
  //   Ap(l) = sqrt((l+1)^2 - m^2) sqrt((l+1+m)(l+1-m)) / (2l+1)  (l + 1 <= L)
  //   Am(l) = -sqrt(l^2 - m^2) sqrt((l+m)(l-m)) / (2l-1)         (l - 1 >= m)
  // so T_j receives Ap(l-1) gth_(j-1) (from l - 1 >= m) and Am(l+1) gth_(j+1) (l + 1 <= L)
  double a_lo = 0.0, a_hi = 0.0;
  if (l - 1 >= m) {
    const double lp = l - 1.0;
    a_lo = sqrt((lp + 1) * (lp + 1) - (double)m * m) * sqrt((lp + 1 + m) * (lp + 1 - m)) / (2.0 * lp + 1.0);
  }
  if (l + 1 <= d.L) {
    const double ln = l + 1.0;
    a_hi = -sqrt(ln * ln - (double)m * m) * sqrt((ln + m) * (ln - m)) / (2.0 * ln - 1.0);
  }
  const double ri = rinv[k];
  for (int c = 0; c < 2; ++c) {
    const double* g = gth + c * plane;
    double v = 0.0;
    if (l - 1 >= m) v += a_lo * g[at - 1];
    if (l + 1 <= d.L) v += a_hi * g[at + 1];
    out[c * plane + at] = v * ri;
  }
  // forward: gph_re = -m T_im / r, gph_im = m T_re / r
  out[at] += (double)m * gph[plane + at] * ri;
  out[plane + at] -= (double)m * gph[at] * ri;
}

void launch_gradients_adjoint(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                              const double* gth, const double* gph, double* out) {
  dim3 grid(ceil_div(d.nlm, 128), d.nr);
  k_gradients_adjoint<<<grid, 128, 0, s>>>(d, lof, mof, rinv, gth, gph, out);
}

// out = -u g on grids of the same layout: the advection's velocity factor.
__global__ void k_neg_product(size_t n, const double* __restrict__ u, const double* __restrict__ g,
                              double* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = -(u[e] * g[e]);
}

void launch_neg_product(cudaStream_t s, size_t n, const double* u, const double* g, double* out) {
  k_neg_product<<<592, 256, 0, s>>>(n, u, g, out);
}

// out = a x + b y (out may alias x or y)
__global__ void k_axpby(size_t n, double a, const double* x, double b, const double* y, double* out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = a * x[e] + b * y[e];
}

void launch_axpby(cudaStream_t s, size_t n, double a, const double* x, double b, const double* y, double* out) {
  k_axpby<<<592, 256, 0, s>>>(n, a, x, b, y, out);
}

}  // namespace gd

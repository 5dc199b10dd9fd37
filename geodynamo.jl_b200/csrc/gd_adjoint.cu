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

}  // namespace gd

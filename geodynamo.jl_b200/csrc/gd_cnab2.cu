// gd_cnab2.cu -- the CNAB2 implicit step for every (field, l, m) radial system
// in one launch, energy diagnostics and a finite-value scan.
//
// build_rhs_cnab2! (src/timestep.jl:610-690):
//   rhs = u/dt + 1.5 N - 0.5 N_prev + (1 - theta) L_l u
// solve_implicit_step! + solve_banded! (src/timestep.jl:692-730,
// src/linear_algebra.jl:59-88): forward substitution with the unit lower
// factor, back substitution with the upper factor.  One thread owns one (l, m)
// column of one field and walks r with register windows; Re and Im share the
// factors.  The AB bootstrap (src/simulation.jl:1153-1170) and the history roll
// (:1312-1329) are folded into the same pass.
#include "gd_internal.cuh"

namespace gd {

template <int KL>
__global__ void __launch_bounds__(128) k_cnab2(Dims d, const int* __restrict__ lof, const double* __restrict__ lin,
                                               const double* __restrict__ lu, Cnab2Args a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int fs = blockIdx.y;
  if (j >= d.nlm || fs >= a.nfield) return;
  const int N = d.nr;
  const int l = lof[j];
  const int kind = a.kind[fs];
  const size_t NM = d.nlm, plane = (size_t)N * NM;
  const size_t Lp1 = (size_t)d.L + 1;
  constexpr int NB = 2 * KL + 1;
  double* ure = a.u[fs];
  double* uim = ure + plane;
  const double* nre = a.nl[fs];
  const double* nim = nre + plane;
  double* pre = a.prev[fs];
  double* pim = pre + plane;
  const double* LIN = lin + (size_t)kind * N * NB * Lp1 + l;
  const double* LU = lu + (size_t)kind * N * NB * Lp1 + l;

  // window wr[t] = u[i - KL + t]
  double wr[NB], wi[NB];
#pragma unroll
  for (int t = 0; t < NB; ++t) {
    const int idx = t - KL;
    wr[t] = (idx >= 0 && idx < N) ? ure[(size_t)idx * NM + j] : 0.0;
    wi[t] = (idx >= 0 && idx < N) ? uim[(size_t)idx * NM + j] : 0.0;
  }
  double yr[KL], yi[KL];  // y[i - KL + t]
#pragma unroll
  for (int t = 0; t < KL; ++t) yr[t] = yi[t] = 0.0;

  for (int i = 0; i < N; ++i) {
    const size_t at = (size_t)i * NM + j;
    // (1 - theta) L u, summed over columns in ascending order
    double Lr = 0.0, Li = 0.0;
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int col = i - KL + t;
      if (col >= 0 && col < N) {
        const double cf = LIN[((size_t)col * NB + (KL + i - col)) * Lp1];
        Lr += cf * wr[t];
        Li += cf * wi[t];
      }
    }
    const double n_r = nre[at], n_i = nim[at];
    double p_r, p_i;
    if (a.boot) { p_r = n_r; p_i = n_i; } else { p_r = pre[at]; p_i = pim[at]; }
    double vr = a.inv_dt * wr[KL] + 1.5 * n_r - 0.5 * p_r;
    double vi = a.inv_dt * wi[KL] + 1.5 * n_i - 0.5 * p_i;
    vr += a.lin_weight * Lr;
    vi += a.lin_weight * Li;
    if (a.bc_rows && (i == 0 || i == N - 1)) {
      vr = (fs == a.temp_slot) ? a.bvals[(i == 0 ? 0 : NM) + j] : 0.0;
      vi = 0.0;
    }
    // history roll: prev := nl
    pre[at] = n_r;
    pim[at] = n_i;
    // forward substitution (unit lower factor)
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int t = 0; t < KL; ++t) {
      const int col = i - KL + t;
      if (col >= 0) {
        const double cf = LU[((size_t)col * NB + (KL + i - col)) * Lp1];
        sr += cf * yr[t];
        si += cf * yi[t];
      }
    }
    const double y_r = vr - sr, y_i = vi - si;
    ure[at] = y_r;
    uim[at] = y_i;
#pragma unroll
    for (int t = 0; t < KL - 1; ++t) { yr[t] = yr[t + 1]; yi[t] = yi[t + 1]; }
    yr[KL - 1] = y_r;
    yi[KL - 1] = y_i;
#pragma unroll
    for (int t = 0; t < NB - 1; ++t) { wr[t] = wr[t + 1]; wi[t] = wi[t + 1]; }
    const int nxt = i + KL + 1;
    wr[NB - 1] = (nxt < N) ? ure[(size_t)nxt * NM + j] : 0.0;
    wi[NB - 1] = (nxt < N) ? uim[(size_t)nxt * NM + j] : 0.0;
  }
  // back substitution; xr[t] = x[i + 1 + t]
  double xr[KL], xi[KL];
#pragma unroll
  for (int t = 0; t < KL; ++t) xr[t] = xi[t] = 0.0;
  for (int i = N - 1; i >= 0; --i) {
    const size_t at = (size_t)i * NM + j;
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int t = 0; t < KL; ++t) {
      const int col = i + 1 + t;
      if (col < N) {
        const double cf = LU[((size_t)col * NB + (KL + i - col)) * Lp1];
        sr += cf * xr[t];
        si += cf * xi[t];
      }
    }
    const double dg = LU[((size_t)i * NB + KL) * Lp1];
    double x_r = (ure[at] - sr) / dg;
    double x_i = (uim[at] - si) / dg;
    if (a.clamp_rows && (i == 0 || i == N - 1)) { x_r = 0.0; x_i = 0.0; }
    ure[at] = x_r;
    uim[at] = x_i;
#pragma unroll
    for (int t = KL - 1; t > 0; --t) { xr[t] = xr[t - 1]; xi[t] = xi[t - 1]; }
    xr[0] = x_r;
    xi[0] = x_i;
  }
}

void launch_cnab2(cudaStream_t s, const Dims& d, const int* lof, const double* lin, const double* lu,
                  const Cnab2Args& a) {
  dim3 grid(ceil_div(d.nlm, 128), a.nfield);
  k_cnab2<GD_MAX_KL><<<grid, 128, 0, s>>>(d, lof, lin, lu, a);
}

// 0.5 sum over (r, l, m) of (T^2 + P^2) / max(l(l+1), 1) for velocity and
// magnetic fields (src/magnetic.jl:519-542).  Deterministic two-level sum.
__global__ void k_energy_partial(Dims d, const int* __restrict__ lof, const double* __restrict__ ut,
                                 const double* __restrict__ up, const double* __restrict__ bt,
                                 const double* __restrict__ bp, double* __restrict__ partial) {
  __shared__ double sk[256], sm[256];
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  double ek = 0.0, em = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
    const int l = lof[i % NM];
    const double lfv = (double)l * (l + 1.0);
    const double w = 1.0 / (lfv > 1.0 ? lfv : 1.0);
    ek += w * (ut[i] * ut[i] + ut[plane + i] * ut[plane + i] + up[i] * up[i] + up[plane + i] * up[plane + i]);
    if (bt) em += w * (bt[i] * bt[i] + bt[plane + i] * bt[plane + i] + bp[i] * bp[i] + bp[plane + i] * bp[plane + i]);
  }
  sk[threadIdx.x] = ek;
  sm[threadIdx.x] = em;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sk[threadIdx.x] += sk[threadIdx.x + s]; sm[threadIdx.x] += sm[threadIdx.x + s]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = sk[0]; partial[2 * blockIdx.x + 1] = sm[0]; }
}

__global__ void k_energy_final(int nblk, const double* __restrict__ partial, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double ek = 0.0, em = 0.0;
  for (int b = 0; b < nblk; ++b) { ek += partial[2 * b]; em += partial[2 * b + 1]; }
  out[0] = 0.5 * ek;
  out[1] = 0.5 * em;
}

void launch_energy(cudaStream_t s, const Dims& d, const int* lof, const double* utor, const double* upol,
                   const double* btor, const double* bpol, double* partial, double* out) {
  const int nblk = 296;
  k_energy_partial<<<nblk, 256, 0, s>>>(d, lof, utor, upol, btor, bpol, partial);
  k_energy_final<<<1, 32, 0, s>>>(nblk, partial, out);
}

__global__ void k_check_finite(size_t n, const double* __restrict__ a, int* flag) {
  int bad = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(a[i])) bad = 1;
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

void launch_check_finite(cudaStream_t s, size_t n, const double* a, int* flag) {
  k_check_finite<<<296, 256, 0, s>>>(n, a, flag);
}

}  // namespace gd

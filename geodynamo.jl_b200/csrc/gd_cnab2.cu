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

// One thread solves the (l, m) column of NF fields that share a diffusivity
// (u_tor + u_pol, B_tor + B_pol, or T), so the per-l LU factors are loaded
// once for both.  The linear operator L_l = nu lap - nu l(l+1)/r^2 is rebuilt
// from the shared Laplacian band with the same roundings as the set-up kernel.
template <int KL, int NF>
__device__ __forceinline__ void cnab2_columns(const Dims& d, int j, int l, const double* __restrict__ lu,
                                              const double* __restrict__ sband /* nu lap, smem */,
                                              const double* __restrict__ srinv2, double nu, const Cnab2Args& a,
                                              const int* slots) {
  const int N = d.nr;
  const size_t NM = d.nlm, plane = (size_t)N * NM;
  const size_t Lp1 = (size_t)d.L + 1;
  constexpr int NB = 2 * KL + 1;
  const double nulf = __dmul_rn(nu, (double)l * (l + 1));
  double* __restrict__ ure[NF];
  double* __restrict__ uim[NF];
  const double* __restrict__ nre[NF];
  const double* __restrict__ nim[NF];
  double* __restrict__ pre[NF];
  double* __restrict__ pim[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    ure[f] = a.u[slots[f]]; uim[f] = ure[f] + plane;
    nre[f] = a.nl[slots[f]]; nim[f] = nre[f] + plane;
    pre[f] = a.prev[slots[f]]; pim[f] = pre[f] + plane;
  }
  const double* LU = lu + l;  // kind offset applied by the caller
  double wr[NF][NB], wi[NF][NB];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int idx = t - KL;
      wr[f][t] = (idx >= 0 && idx < N) ? ure[f][(size_t)idx * NM + j] : 0.0;
      wi[f][t] = (idx >= 0 && idx < N) ? uim[f][(size_t)idx * NM + j] : 0.0;
    }
  double yr[NF][KL], yi[NF][KL];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < KL; ++t) yr[f][t] = yi[f][t] = 0.0;

#pragma unroll 4
  for (int i = 0; i < N; ++i) {
    const size_t at = (size_t)i * NM + j;
    double cfl[NB];
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int col = i - KL + t;
      double cf = 0.0;
      if (col >= 0 && col < N) {
        cf = sband[col * NB + (KL + i - col)];
        if (t == KL) cf = __dsub_rn(cf, __dmul_rn(nulf, srinv2[i]));
      }
      cfl[t] = cf;
    }
    double lfac[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
      const int col = i - KL + t;
      lfac[t] = (col >= 0) ? LU[((size_t)col * NB + (KL + i - col)) * Lp1] : 0.0;
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double Lr = 0.0, Li = 0.0;
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int col = i - KL + t;
        if (col >= 0 && col < N) {
          Lr += cfl[t] * wr[f][t];
          Li += cfl[t] * wi[f][t];
        }
      }
      const double n_r = nre[f][at], n_i = nim[f][at];
      double p_r, p_i;
      if (a.boot) { p_r = n_r; p_i = n_i; } else { p_r = pre[f][at]; p_i = pim[f][at]; }
      double vr = a.inv_dt * wr[f][KL] + 1.5 * n_r - 0.5 * p_r;
      double vi = a.inv_dt * wi[f][KL] + 1.5 * n_i - 0.5 * p_i;
      vr += a.lin_weight * Lr;
      vi += a.lin_weight * Li;
      if (a.bc_rows && (i == 0 || i == N - 1)) {
        vr = (slots[f] == a.temp_slot) ? a.bvals[(i == 0 ? 0 : NM) + j] : 0.0;
        vi = 0.0;
      }
      pre[f][at] = n_r;
      pim[f][at] = n_i;
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        const int col = i - KL + t;
        if (col >= 0) {
          sr += lfac[t] * yr[f][t];
          si += lfac[t] * yi[f][t];
        }
      }
      const double y_r = vr - sr, y_i = vi - si;
      ure[f][at] = y_r;
      uim[f][at] = y_i;
#pragma unroll
      for (int t = 0; t < KL - 1; ++t) { yr[f][t] = yr[f][t + 1]; yi[f][t] = yi[f][t + 1]; }
      yr[f][KL - 1] = y_r;
      yi[f][KL - 1] = y_i;
#pragma unroll
      for (int t = 0; t < NB - 1; ++t) { wr[f][t] = wr[f][t + 1]; wi[f][t] = wi[f][t + 1]; }
      const int nxt = i + KL + 1;
      wr[f][NB - 1] = (nxt < N) ? ure[f][(size_t)nxt * NM + j] : 0.0;
      wi[f][NB - 1] = (nxt < N) ? uim[f][(size_t)nxt * NM + j] : 0.0;
    }
  }
  double xr[NF][KL], xi[NF][KL];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < KL; ++t) xr[f][t] = xi[f][t] = 0.0;
#pragma unroll 4
  for (int i = N - 1; i >= 0; --i) {
    const size_t at = (size_t)i * NM + j;
    double ufac[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
      const int col = i + 1 + t;
      ufac[t] = (col < N) ? LU[((size_t)col * NB + (KL + i - col)) * Lp1] : 0.0;
    }
    const double dg = LU[((size_t)i * NB + KL) * Lp1];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        const int col = i + 1 + t;
        if (col < N) {
          sr += ufac[t] * xr[f][t];
          si += ufac[t] * xi[f][t];
        }
      }
      double x_r = (ure[f][at] - sr) / dg;
      double x_i = (uim[f][at] - si) / dg;
      if (a.clamp_rows && (i == 0 || i == N - 1)) { x_r = 0.0; x_i = 0.0; }
      ure[f][at] = x_r;
      uim[f][at] = x_i;
#pragma unroll
      for (int t = KL - 1; t > 0; --t) { xr[f][t] = xr[f][t - 1]; xi[f][t] = xi[f][t - 1]; }
      xr[f][0] = x_r;
      xi[f][0] = x_i;
    }
  }
}

// blockIdx.y = field slot; the block's Laplacian band uses that field's diffusivity.
template <int KL>
__global__ void __launch_bounds__(128) k_cnab2(Dims d, const int* __restrict__ lof, const double* __restrict__ d1,
                                               const double* __restrict__ d2, const double* __restrict__ rinv,
                                               const double* __restrict__ rinv2, const double* __restrict__ nu,
                                               const double* __restrict__ lu, Cnab2Args a) {
  constexpr int NB = 2 * KL + 1;
  extern __shared__ double sm[];
  double* sband = sm;                 // nu * lap, [col][band]
  double* srinv2 = sm + (size_t)d.nr * NB;
  const int slot = blockIdx.y;
  if (slot >= a.nfield) return;
  const int g = a.kind[slot];
  const int slots[1] = {slot};
  const double nuk = nu[g];
  const int N = d.nr;
  for (int e = threadIdx.x; e < N * NB; e += blockDim.x) {
    const int col = e / NB, b = e % NB, i = col + b - KL;
    double v = 0.0;
    if (i >= 0 && i < N) {
      const size_t q = b + (size_t)NB * col;
      // same roundings as the set-up kernel: nu * (d2 + (2 r^-1) d1)
      v = __dmul_rn(nuk, __dadd_rn(d2[q], __dmul_rn(__dmul_rn(2.0, rinv[i]), d1[q])));
    }
    sband[e] = v;
  }
  for (int i = threadIdx.x; i < N; i += blockDim.x) srinv2[i] = rinv2[i];
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.nlm) return;
  const int l = lof[j];
  const double* LUk = lu + (size_t)g * N * NB * ((size_t)d.L + 1);
  cnab2_columns<KL, 1>(d, j, l, LUk, sband, srinv2, nuk, a, slots);
}

void launch_cnab2(cudaStream_t s, const Dims& d, const int* lof, const double* d1, const double* d2,
                  const double* rinv, const double* rinv2, const double* nu, const double* lu, const Cnab2Args& a) {
  dim3 grid(ceil_div(d.nlm, 128), a.nfield);
  const size_t smem = ((size_t)d.nr * GD_NBW + d.nr) * sizeof(double);
  k_cnab2<GD_MAX_KL><<<grid, 128, smem, s>>>(d, lof, d1, d2, rinv, rinv2, nu, lu, a);
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

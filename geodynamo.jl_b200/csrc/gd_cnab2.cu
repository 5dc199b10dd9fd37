// gd_cnab2.cu -- the CNAB2 implicit step for every (field, l, m) radial system
// in one launch, energy diagnostics and a finite-value scan.
//
// build_rhs_cnab2! (src/timestep.jl:610-690):
//   rhs = u/dt + 1.5 N - 0.5 N_prev + (1 - theta) L_l u
// solve_implicit_step! + solve_banded! (src/timestep.jl:692-730,
// src/linear_algebra.jl:59-88): forward substitution with the unit lower
// factor, back substitution with the upper factor.  One thread owns one (l, m)
// column of one field and walks r with register windows; Re and Im share the
// factors.  The AB bootstrap (src/simulation.jl:1153-1170) is folded into the
// same pass; the history roll (:1312-1329) is the handle's switch of the two
// banks of nonlinear terms after the step (N_prev is read from the other bank).
#include <type_traits>

#include "gd_internal.cuh"

namespace gd {

// One thread solves the (l, m) column of one field.  Three sweeps over r, each
// with loads that do not depend on the running recurrence so the unrolled
// loops keep many loads in flight:
//   1. rhs = u/dt + 1.5 N - 0.5 N_prev + (1 - theta) L_l u  (written over u);
//   2. forward substitution with the unit lower factor (y over u);
//   3. back substitution with the upper factor (x over u).
// L_l = nu lap - nu l(l+1)/r^2 is rebuilt from the block's shared Laplacian
// band with the same roundings as the set-up kernel.
template <int KL>
__device__ __forceinline__ void cnab2_column(const Dims& d, int j, int l, const double* __restrict__ LU,
                                             const double* __restrict__ sband, const double* __restrict__ srinv2,
                                             double nu, const Cnab2Args& a, int slot, int N, int base) {
  // the segment's N levels start at shell base; the planes span all shells
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  const size_t Lp1 = (size_t)d.L + 1;
  constexpr int NB = 2 * KL + 1;
  const double nulf = __dmul_rn(nu, (double)l * (l + 1));
  const size_t s0 = (size_t)base * NM + j;
  double* __restrict__ ure = a.u[slot] + s0;
  double* __restrict__ uim = a.u[slot] + plane + s0;
  const double* __restrict__ nre = a.nl[slot] + s0;
  const double* __restrict__ nim = a.nl[slot] + plane + s0;
  const double* __restrict__ pre = a.prev[slot] + s0;
  const double* __restrict__ pim = a.prev[slot] + plane + s0;
  const double* __restrict__ F = LU + l;
  const bool boot = a.boot != 0;
  const bool rows = a.bc_rows != 0;
  const double* __restrict__ rowv = a.rowvals[slot];
  const int stages = a.stages ? a.stages : 7;

  // sweep 1: right-hand side, rows in batches of RB whose loads are issued
  // first.  With FWD the forward substitution of sweep 2 runs in the same pass
  // (both walk r upward; the window keeps the original u the band still
  // needs), so y is written over u without a second pass through memory.
  constexpr int RB = 4;
  auto rhs_sweep = [&](auto fwd_tag) {
    constexpr bool FWD = decltype(fwd_tag)::value;
    constexpr int RBF = FWD ? 3 : 4;  // the factor rows take the registers of a fourth row
    double wr[NB], wi[NB];
    double yr[KL], yi[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) yr[t] = yi[t] = 0.0;
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int idx = t - KL;
      wr[t] = (idx >= 0 && idx < N) ? ure[(size_t)idx * NM] : 0.0;
      wi[t] = (idx >= 0 && idx < N) ? uim[(size_t)idx * NM] : 0.0;
    }
    for (int i0 = 0; i0 < N; i0 += RBF) {
      double unr[RBF], uni[RBF], nr_[RBF], ni_[RBF], pr_[RBF], pi_[RBF];
      double lf[RBF][FWD ? KL : 1];
#pragma unroll
      for (int b = 0; b < RBF; ++b) {
        const int i = i0 + b, nxt = i + KL + 1;
        unr[b] = (nxt < N) ? ure[(size_t)nxt * NM] : 0.0;
        uni[b] = (nxt < N) ? uim[(size_t)nxt * NM] : 0.0;
        if (i < N) {
          nr_[b] = nre[(size_t)i * NM];
          ni_[b] = nim[(size_t)i * NM];
          pr_[b] = boot ? nr_[b] : pre[(size_t)i * NM];
          pi_[b] = boot ? ni_[b] : pim[(size_t)i * NM];
        } else {
          nr_[b] = ni_[b] = pr_[b] = pi_[b] = 0.0;
        }
        if constexpr (FWD) {
#pragma unroll
          for (int t = 0; t < KL; ++t) {
            const int col = i - KL + t;
            lf[b][t] = (i < N && col >= 0) ? F[((size_t)col * NB + (KL + i - col)) * Lp1] : 0.0;
          }
        }
      }
#pragma unroll
      for (int b = 0; b < RBF; ++b) {
        const int i = i0 + b;
        if (i >= N) break;
        const size_t at = (size_t)i * NM;
        double Lr = 0.0, Li = 0.0;
#pragma unroll
        for (int t = 0; t < NB; ++t) {
          const int col = i - KL + t;
          if (col >= 0 && col < N) {
            double cf = sband[col * NB + (KL + i - col)];
            if (t == KL) cf = __dsub_rn(cf, __dmul_rn(nulf, srinv2[i]));
            Lr += cf * wr[t];
            Li += cf * wi[t];
          }
        }
        double vr = a.inv_dt * wr[KL] + 1.5 * nr_[b] - 0.5 * pr_[b];
        double vi = a.inv_dt * wi[KL] + 1.5 * ni_[b] - 0.5 * pi_[b];
        vr += a.lin_weight * Lr;
        vi += a.lin_weight * Li;
        if (rows && (i == 0 || i == N - 1)) {
          // ball: the r = 0 row of l >= 1 is the regularity condition (value 0)
          vr = (rowv != nullptr && !(d.ball && i == 0 && l > 0)) ? rowv[(i == 0 ? 0 : NM) + j] : 0.0;
          vi = 0.0;
        }
        if constexpr (FWD) {
          double sr = 0.0, si = 0.0;
#pragma unroll
          for (int t = 0; t < KL; ++t) {
            if (i - KL + t >= 0) {
              sr += lf[b][t] * yr[t];
              si += lf[b][t] * yi[t];
            }
          }
          vr = vr - sr;
          vi = vi - si;
#pragma unroll
          for (int t = 0; t < KL - 1; ++t) { yr[t] = yr[t + 1]; yi[t] = yi[t + 1]; }
          yr[KL - 1] = vr;
          yi[KL - 1] = vi;
        }
        ure[at] = vr;
        uim[at] = vi;
#pragma unroll
        for (int t = 0; t < NB - 1; ++t) { wr[t] = wr[t + 1]; wi[t] = wi[t + 1]; }
        wr[NB - 1] = unr[b];
        wi[NB - 1] = uni[b];
      }
    }
  };
  const bool fused = (stages & 3) == 3;
  if (fused) rhs_sweep(std::true_type{});
  else if (stages & 1) rhs_sweep(std::false_type{});
  // sweep 2: forward substitution (unit lower factor), y[i - KL + t] in yr[t]
  if ((stages & 2) && !fused) {
  double yr[KL], yi[KL];
#pragma unroll
  for (int t = 0; t < KL; ++t) yr[t] = yi[t] = 0.0;
  for (int i0 = 0; i0 < N; i0 += RB) {
    double br[RB], bi[RB], lf[RB][KL];
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = i0 + b;
      br[b] = (i < N) ? ure[(size_t)i * NM] : 0.0;
      bi[b] = (i < N) ? uim[(size_t)i * NM] : 0.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        const int col = i - KL + t;
        lf[b][t] = (i < N && col >= 0) ? F[((size_t)col * NB + (KL + i - col)) * Lp1] : 0.0;
      }
    }
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = i0 + b;
      if (i >= N) break;
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        if (i - KL + t >= 0) {
          sr += lf[b][t] * yr[t];
          si += lf[b][t] * yi[t];
        }
      }
      const double y_r = br[b] - sr, y_i = bi[b] - si;
      ure[(size_t)i * NM] = y_r;
      uim[(size_t)i * NM] = y_i;
#pragma unroll
      for (int t = 0; t < KL - 1; ++t) { yr[t] = yr[t + 1]; yi[t] = yi[t + 1]; }
      yr[KL - 1] = y_r;
      yi[KL - 1] = y_i;
    }
  }
  }
  // sweep 3: back substitution, x[i + 1 + t] in xr[t]
  if (stages & 4) {
  double xr[KL], xi[KL];
#pragma unroll
  for (int t = 0; t < KL; ++t) xr[t] = xi[t] = 0.0;
  for (int i0 = N - 1; i0 >= 0; i0 -= RB) {
    double yv[RB], yw[RB], uf[RB][KL], dg[RB];
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = i0 - b;
      yv[b] = (i >= 0) ? ure[(size_t)i * NM] : 0.0;
      yw[b] = (i >= 0) ? uim[(size_t)i * NM] : 0.0;
      dg[b] = (i >= 0) ? F[((size_t)i * NB + KL) * Lp1] : 1.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        const int col = i + 1 + t;
        uf[b][t] = (i >= 0 && col < N) ? F[((size_t)col * NB + (KL + i - col)) * Lp1] : 0.0;
      }
    }
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = i0 - b;
      if (i < 0) break;
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        if (i + 1 + t < N) {
          sr += uf[b][t] * xr[t];
          si += uf[b][t] * xi[t];
        }
      }
      const double x_r = (yv[b] - sr) / dg[b];
      const double x_i = (yw[b] - si) / dg[b];
      // bc_mode 1 zeroes the boundary rows after the whole solve: the
      // substitution itself continues with the solved values
      const bool clamp = a.clamp_rows && (i == 0 || i == N - 1);
      ure[(size_t)i * NM] = clamp ? 0.0 : x_r;
      uim[(size_t)i * NM] = clamp ? 0.0 : x_i;
#pragma unroll
      for (int t = KL - 1; t > 0; --t) { xr[t] = xr[t - 1]; xi[t] = xi[t - 1]; }
      xr[0] = x_r;
      xi[0] = x_i;
    }
  }
  }
}

// blockIdx.y = field slot; the block's Laplacian band uses that field's diffusivity.
template <int KL>
// 160 registers, three 128-thread blocks per SM (more columns in flight than
// wider row batches would give)
__global__ void __launch_bounds__(128, 3) k_cnab2(Dims d, const int* __restrict__ lof, const double* __restrict__ d1,
                                               const double* __restrict__ d2, const double* __restrict__ rinv,
                                               const double* __restrict__ rinv2, const double* __restrict__ nu,
                                               const double* __restrict__ lu, Cnab2Args a) {
  constexpr int NB = 2 * KL + 1;
  extern __shared__ double sm[];
  double* sband = sm;                 // nu * lap, [col][band]
  double* srinv2 = sm + (size_t)d.nrs * NB;
  const int slot = blockIdx.y;
  if (slot >= a.nfield) return;
  const int g = a.kind[slot];
  const double nuk = nu[g];
  // the segment's radial operators (its variant's band, its shells' 1/r)
  const SegView sv = seg_view(d, blockIdx.z);
  const int N = sv.n;
  d1 += sv.band_off;
  d2 += sv.band_off;
  rinv += sv.base;
  rinv2 += sv.base;
  lu += sv.op_off;
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
  const int j = d.jlo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.jhi) return;
  const int l = lof[j];
  const double* LUk = lu + (size_t)g * N * NB * ((size_t)d.L + 1);
  const int* rt = a.rowtypes[slot];
  if (a.bc_rows && rt != nullptr && a.lu_flux != nullptr) {
    // a prescribed flux at a boundary: the factors with the row of D1 there
    const int fv = (rt[j] == GD_BC_FLUX ? 1 : 0) | (rt[d.nlm + j] == GD_BC_FLUX ? 2 : 0);
    if (fv)
      LUk = a.lu_flux + (size_t)(fv - 1) * a.lu_flux_stride + sv.op_off + (size_t)g * N * NB * ((size_t)d.L + 1);
  }
  cnab2_column<KL>(d, j, l, LUk, sband, srinv2, nuk, a, slot, N, sv.base);
}

void launch_cnab2(cudaStream_t s, const Dims& d, const int* lof, const double* d1, const double* d2,
                  const double* rinv, const double* rinv2, const double* nu, const double* lu, const Cnab2Args& a) {
  dim3 grid(ceil_div(d.jhi - d.jlo, 128), a.nfield, d.nseg);
  const size_t smem = ((size_t)d.nrs * GD_NBW + d.nrs) * sizeof(double);
  k_cnab2<GD_MAX_KL><<<grid, 128, smem, s>>>(d, lof, d1, d2, rinv, rinv2, nu, lu, a);
}

// 0.5 sum over (r, l, m) of (T^2 + P^2) / max(l(l+1), 1) for velocity and
// magnetic fields (src/magnetic.jl:519-542).  Deterministic two-level sum,
// one per segment (blockIdx.y), each in the order of an unsegmented handle.
__global__ void k_energy_partial(Dims d, const int* __restrict__ lof, const double* __restrict__ ut,
                                 const double* __restrict__ up, const double* __restrict__ bt,
                                 const double* __restrict__ bp, double* __restrict__ partial) {
  __shared__ double sk[256], sm[256];
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  const SegView sv = seg_view(d, blockIdx.y);
  const size_t seg0 = (size_t)sv.base * NM, segn = (size_t)sv.n * NM;
  ut += seg0;
  up += seg0;
  if (bt) {
    bt += seg0;
    bp += seg0;
  }
  double ek = 0.0, em = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < segn; i += (size_t)gridDim.x * blockDim.x) {
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
  if (threadIdx.x == 0) {
    const size_t q = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    partial[2 * q] = sk[0];
    partial[2 * q + 1] = sm[0];
  }
}

// out[2 g], out[2 g + 1]: kinetic and magnetic energy of segment g
__global__ void k_energy_final(int nblk, int nseg, const double* __restrict__ partial, double* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nseg) return;
  partial += (size_t)2 * nblk * g;
  double ek = 0.0, em = 0.0;
  for (int b = 0; b < nblk; ++b) { ek += partial[2 * b]; em += partial[2 * b + 1]; }
  out[2 * g] = 0.5 * ek;
  out[2 * g + 1] = 0.5 * em;
}

void launch_energy(cudaStream_t s, const Dims& d, const int* lof, const double* utor, const double* upol,
                   const double* btor, const double* bpol, double* partial, double* out) {
  const int nblk = GD_ENERGY_BLOCKS;
  k_energy_partial<<<dim3(nblk, d.nseg), 256, 0, s>>>(d, lof, utor, upol, btor, bpol, partial);
  k_energy_final<<<ceil_div(d.nseg, 32), 32, 0, s>>>(nblk, d.nseg, partial, out);
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

// gd_spectral.cu -- spectral-space operators on the native layout (two planes
// Re/Im of [r][j], j m-major), plus layout conversions used by the host ABI.
#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"

namespace gd {

// Radial operators: each thread owns one mode j and a run of consecutive
// levels, so every coefficient is read once per run (plus the 2 KL halo).
// The gradient kernel walks its run with a register window of 2 KL + 1
// levels.  The curl kernel stages a block's runs (128 modes) plus the halo of
// both planes in shared memory by asynchronous 8-byte copies, all in flight
// together, with the band columns and 1/r values those levels use, and reads
// every level's window and coefficients from there.  Band sums run over the
// same levels in the same order as the banded matrix-vector product they
// restate.
constexpr int RB_R = 16;          // most levels per block
constexpr int RAD_THREADS = 128;  // modes per block

__device__ __forceinline__ void stage8(double* s, const double* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(s)), "l"(g)
               : "memory");
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Levels per block: the nr levels split evenly over ceil(nr / RB_R) blocks.
static inline int radial_rows(int nr) { return ceil_div(nr, ceil_div(nr, RB_R)); }

// Shared-memory image of one block: win[plane][level][thread] holds levels
// k0 - KL .. k0 + RB_R + KL - 1 (zero outside 0 .. nr-1); band[b][NB (i +
// KL) + e] holds entry e of band column k0 + i of the block's matrix b; rv[q][i]
// holds 1/r^(q+1) at level k0 + i.
template <int KL, int NBAND>
struct RadialStage {
  static constexpr int NB = 2 * KL + 1, ROWS = RB_R + 2 * KL;
  double win[2][ROWS][RAD_THREADS];
  double band[NBAND][ROWS * NB];
  double rv[2][RB_R];
};

template <int KL>
__device__ __forceinline__ void stage_column(double (*win)[RB_R + 2 * KL][RAD_THREADS], const double* P, size_t plane,
                                             size_t NM, int N, int k0, int rows, int j) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int t = 0; t < RB_R + 2 * KL; ++t) {
      const int kk = k0 - KL + t;
      if (kk >= 0 && kk < N && t < rows + 2 * KL)
        stage8(&win[c][t][tid], P + c * plane + (size_t)kk * NM + j);
      else
        win[c][t][tid] = 0.0;
    }
}

// Band columns k0 - KL .. k0 + rows + KL - 1 (those inside 0 .. N-1) of a
// band matrix stored column by column, NB entries each; plain block-strided
// copies, ordered before use by the block barrier.
template <int KL>
__device__ __forceinline__ void stage_band(double* sb, const double* band, int N, int k0, int rows) {
  constexpr int NB = 2 * KL + 1;
  const int c0 = max(0, k0 - KL), c1 = min(N, k0 + rows + KL);
  const int off = (c0 - (k0 - KL)) * NB;
  for (int e = threadIdx.x; e < (c1 - c0) * NB; e += RAD_THREADS) sb[off + e] = band[(size_t)c0 * NB + e];
}

template <int KL, int NBAND>
static size_t radial_smem() {
  return sizeof(RadialStage<KL, NBAND>);
}

// compute_all_gradients_spectral! (src/scalar_field_common.jl:125-345):
// theta derivative by the reference's recurrence coefficients (:158,171), phi
// derivative i m, radial derivative by the banded D1, then x 1/r on the
// angular components (:317-321).  In m-major order (l +- 1, m) sits at j +- 1.
// IMG: the mixed path's scalar synthesis reads g_theta, g_phi, g_r as split
// TF32 image columns (field slots 1, 2, 3 of n = (field nr + r) 2 + re/im);
// they are written there instead of to the FP64 arrays.
template <int KL, bool IMG>
__global__ void k_gradients(Dims d, const int* __restrict__ lof, const int* __restrict__ mof,
                            const double* __restrict__ rinv, const double* __restrict__ d1,
                            const double* __restrict__ T, double* __restrict__ gth, double* __restrict__ gph,
                            double* __restrict__ gr, SynthImageOut img) {
  constexpr int NB = 2 * KL + 1;
  const int j = d.jlo + blockIdx.x * blockDim.x + threadIdx.x;
  const int k0 = blockIdx.y * RB_R;
  if (j >= d.jhi) return;
  const int l = lof[j], m = mof[j];
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  // segment blockIdx.z: levels base .. base + N - 1 (the whole column when nseg = 1)
  const SegView sv = seg_view(d, blockIdx.z);
  const int N = sv.n, base = sv.base;
  if (k0 >= N) return;
  d1 += sv.band_off;
  T += (size_t)base * NM;
  rinv += base;
  if (!IMG) {
    gth += (size_t)base * NM;
    gph += (size_t)base * NM;
    gr += (size_t)base * NM;
  }
  const bool up = l + 1 <= d.L, dn = l >= 1 && l - 1 >= m;
  const double Ap = up ? sqrt((double)(l + 1) * (l + 1) - (double)m * m) * sqrt((double)(l + 1 + m) * (double)(l + 1 - m)) /
                             (2.0 * l + 1.0)
                       : 0.0;
  const double Am = dn ? -sqrt((double)l * l - (double)m * m) * sqrt((double)(l + m) * (double)(l - m)) / (2.0 * l - 1.0)
                       : 0.0;
  const SynthImagePos ip = IMG ? synth_image_pos(img, d.L, m, l) : SynthImagePos{};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    const double* P = T + c * plane;
    double w[NB];
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const int kk = k0 - KL + t;
      w[t] = (kk >= 0 && kk < N) ? P[(size_t)kk * NM + j] : 0.0;
    }
    for (int b = 0; b < RB_R; ++b) {
      const int k = k0 + b;
      if (k >= N) break;
      const size_t at = (size_t)k * NM + j;
      double sr = 0.0;
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int jj = k - KL + t;
        if (jj >= 0 && jj < N) sr += d1[(KL + k - jj) + (size_t)NB * jj] * w[t];
      }
      if (IMG) {
        const int n = (3 * d.nr + base + k) * 2 + c;
        synth_image_put(img, 256, ip, n >> 8, n & 255, sr);
      } else {
        gr[c * plane + at] = sr;
      }
#pragma unroll
      for (int t = 0; t < NB - 1; ++t) w[t] = w[t + 1];
      const int nx = k + KL + 1;
      w[NB - 1] = nx < N ? P[(size_t)nx * NM + j] : 0.0;
    }
  }
  for (int b = 0; b < RB_R; ++b) {
    const int k = k0 + b;
    if (k >= N) break;
    const size_t at = (size_t)k * NM + j;
    double dr = 0.0, di = 0.0;
    if (up) {
      dr += Ap * T[at + 1];
      di += Ap * T[plane + at + 1];
    }
    if (dn) {
      dr += Am * T[at - 1];
      di += Am * T[plane + at - 1];
    }
    const double ri = rinv[k];
    double v[4] = {dr * ri, di * ri, (-(double)m * T[plane + at]) * ri, ((double)m * T[at]) * ri};
    // ball: the angular components stay 0 at r = 0 (src/scalar_field_common.jl:300-310)
    if (d.ball && k == 0) v[0] = v[1] = v[2] = v[3] = 0.0;
    if (IMG) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int n = ((1 + (q >> 1)) * d.nr + base + k) * 2 + (q & 1);
        synth_image_put(img, 256, ip, n >> 8, n & 255, v[q]);
      }
    } else {
      gth[at] = v[0];
      gth[plane + at] = v[1];
      gph[at] = v[2];
      gph[plane + at] = v[3];
    }
  }
}

void launch_gradients(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                      const double* d1, const double* T, double* gth, double* gph, double* gr) {
  dim3 grid(ceil_div(d.jhi - d.jlo, 128), ceil_div(d.nrs, RB_R), d.nseg);
  // the band half-width is validated to GD_MAX_KL at creation
  k_gradients<GD_MAX_KL, false><<<grid, 128, 0, s>>>(d, lof, mof, rinv, d1, T, gth, gph, gr, SynthImageOut{});
}

void launch_gradients_img(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                          const double* d1, const double* T, const SynthImageOut& img) {
  dim3 grid(ceil_div(d.jhi - d.jlo, 128), ceil_div(d.nrs, RB_R), d.nseg);
  k_gradients<GD_MAX_KL, true><<<grid, 128, 0, s>>>(d, lof, mof, rinv, d1, T, nullptr, nullptr, nullptr, img);
}

// compute_vorticity_spectral_full! (src/velocity.jl:340-441) and
// compute_current_density_spectral! (src/magnetic.jl:253-349):
//   curl_tor = l(l+1)/r^2 P - D2 P - (2/r) D1 P,   curl_pol = -l(l+1)/r^2 T.
// IMG: the mixed path's vector synthesis of the curl reads it as split TF32
// image columns 32 shells x [S re, S im, T re, T im] (S = curl_pol, T =
// curl_tor), column tile r / 32; written there instead of to the FP64 arrays.
template <int KL, bool IMG>
__global__ void __launch_bounds__(RAD_THREADS, 4) k_curl(Dims d, const int* __restrict__ lof,
                                                         const int* __restrict__ mof, const double* __restrict__ rinv,
                                                         const double* __restrict__ rinv2,
                                                         const double* __restrict__ d1, const double* __restrict__ d2,
                                                         const double* __restrict__ tor,
                                                         const double* __restrict__ pol, double* __restrict__ otor,
                                                         double* __restrict__ opol, int rows, SynthImageOut img) {
  constexpr int NB = 2 * KL + 1;
  extern __shared__ __align__(16) unsigned char rad_smem[];
  auto& st = *reinterpret_cast<RadialStage<KL, 2>*>(rad_smem);
  const int tid = threadIdx.x;
  const int j = d.jlo + blockIdx.x * RAD_THREADS + tid;
  const int k0 = blockIdx.y * rows;
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  // segment blockIdx.z: levels base .. base + N - 1 (the whole column when nseg = 1)
  const SegView sv = seg_view(d, blockIdx.z);
  const int N = sv.n, base = sv.base;
  if (k0 >= N) return;  // the whole block: a shorter segment
  d1 += sv.band_off;
  d2 += sv.band_off;
  tor += (size_t)base * NM;
  pol += (size_t)base * NM;
  rinv += base;
  rinv2 += base;
  if (!IMG) {
    otor += (size_t)base * NM;
    opol += (size_t)base * NM;
  }
  const bool live = j < d.jhi;
  if (live) stage_column<KL>(st.win, pol, plane, NM, N, k0, rows, j);
  stage_band<KL>(st.band[0], d1, N, k0, rows);
  stage_band<KL>(st.band[1], d2, N, k0, rows);
  if (tid < rows && k0 + tid < N) {
    st.rv[0][tid] = rinv[k0 + tid];
    st.rv[1][tid] = rinv2[k0 + tid];
  }
  // the toroidal values of the block's levels: plain loads, in flight with
  // the staging copies
  double tv[2][RB_R];
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < RB_R; ++b) {
      const int k = k0 + b;
      tv[c][b] = (live && b < rows && k < N) ? tor[c * plane + (size_t)k * NM + j] : 0.0;
    }
  stage_wait();
  __syncthreads();
  if (!live) return;
  const double lf = (double)lof[j] * (lof[j] + 1.0);
  const SynthImagePos ip = IMG ? synth_image_pos(img, d.L, mof[j], lof[j]) : SynthImagePos{};
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int b = 0; b < RB_R; ++b) {
      const int k = k0 + b;
      if (b >= rows || k >= N) break;
      double a1 = 0.0, a2 = 0.0;
#pragma unroll
      for (int t = 0; t < NB; ++t) {
        const int jj = k - KL + t;
        if (jj >= 0 && jj < N) {
          const int q = (2 * KL - t) + NB * (b + t);
          const double w = st.win[c][b + t][tid];
          a1 += st.band[0][q] * w;
          a2 += st.band[1][q] * w;
        }
      }
      const size_t at = (size_t)k * NM + j;
      double vt = lf * st.rv[1][b] * st.win[c][b + KL][tid] - a2 - 2.0 * st.rv[0][b] * a1;
      double vp = -lf * st.rv[1][b] * tv[c][b];
      // ball: both components are set to 0 at r = 0 (src/velocity.jl:417-422,
      // src/magnetic.jl:325-330)
      if (d.ball && k == 0) vt = vp = 0.0;
      if (IMG) {
        const int kg = base + k;  // column tiles run over all shells
        const int col = (kg & 31) * 4 + c;
        synth_image_put(img, 128, ip, kg >> 5, col, vp);
        synth_image_put(img, 128, ip, kg >> 5, col + 2, vt);
      } else {
        otor[c * plane + at] = vt;
        opol[c * plane + at] = vp;
      }
    }
  }
}

void launch_curl(cudaStream_t s, const Dims& d, const int* lof, const double* rinv, const double* rinv2,
                 const double* d1, const double* d2, const double* tor, const double* pol, double* otor,
                 double* opol) {
  const int rows = radial_rows(d.nrs);
  dim3 grid(ceil_div(d.jhi - d.jlo, RAD_THREADS), ceil_div(d.nrs, rows), d.nseg);
  const size_t smem = radial_smem<GD_MAX_KL, 2>();
  allow_dynamic_smem(k_curl<GD_MAX_KL, false>, smem);
  k_curl<GD_MAX_KL, false><<<grid, RAD_THREADS, smem, s>>>(d, lof, nullptr, rinv, rinv2, d1, d2, tor, pol, otor,
                                                           opol, rows, SynthImageOut{});
}

void launch_curl_img(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                     const double* rinv2, const double* d1, const double* d2, const double* tor, const double* pol,
                     const SynthImageOut& img) {
  const int rows = radial_rows(d.nrs);
  dim3 grid(ceil_div(d.jhi - d.jlo, RAD_THREADS), ceil_div(d.nrs, rows), d.nseg);
  const size_t smem = radial_smem<GD_MAX_KL, 2>();
  allow_dynamic_smem(k_curl<GD_MAX_KL, true>, smem);
  k_curl<GD_MAX_KL, true><<<grid, RAD_THREADS, smem, s>>>(d, lof, mof, rinv, rinv2, d1, d2, tor, pol, nullptr,
                                                          nullptr, rows, img);
}

// apply_temperature_boundary_conditions_spectral! (src/thermal.jl:262-303):
// Dirichlet rows r = ri and r = ro of the temperature state.
// Boundary conditions of a scalar field (apply_temperature_boundary_conditions_spectral!,
// src/thermal.jl:262-303; apply_composition_boundary_conditions_spectral!,
// src/compositional.jl:318-370).  One thread per mode: fixed-value rows first
// (Re = value, Im = 0), then, for a flux boundary, the tau correction of
// apply_flux_bc_tau! (src/scalar_field_common.jl:866-935): the flux error of
// the real profile at each flux boundary (prescribed - (D1 Re)[boundary]),
// coefficients of the tau functions that cancel it, and the same correction
// added to Re and, when any |Im| exceeds 1e-12, to Im.
__global__ void k_scalar_bc(Dims d, const int* __restrict__ lof, const double* __restrict__ bv,
                            const int* __restrict__ types, const double* __restrict__ d1, TauConsts tc,
                            double* __restrict__ F, int op_rows) {
  const int j = d.jlo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.jhi) return;
  // segment blockIdx.y: its own boundary rows, radial profile and tau functions
  const SegView sv = seg_view(d, blockIdx.y);
  const int N = sv.n, KL = d.kl, NB = 2 * GD_MAX_KL + 1;
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  F += (size_t)sv.base * NM;
  d1 += sv.band_off;
  double* re = F + j;
  double* im = F + plane + j;
  // ball: no inner boundary at r = 0 (src/thermal.jl:281-282); regularity
  // after the boundary rows (src/thermal.jl:310-312, src/Ball/Ball.jl:153-170)
  const int ti = d.ball ? -1 : types[j], to = types[NM + j];
  const bool regular = d.ball && lof[j] > 0;
  if (ti == GD_BC_VALUE) { re[0] = bv[j]; im[0] = 0.0; }
  if (to == GD_BC_VALUE) { re[(size_t)(N - 1) * NM] = bv[NM + j]; im[(size_t)(N - 1) * NM] = 0.0; }
  // with the boundary-row operator (op_rows) a flux is a row of the implicit
  // solve, not a correction of the state
  const bool fi = !op_rows && ti == GD_BC_FLUX, fo = !op_rows && to == GD_BC_FLUX;
  if (!fi && !fo) {
    if (regular) re[0] = im[0] = 0.0;
    return;
  }
  // boundary fluxes of the real profile: rows 0 and N - 1 of the banded D1
  // (entry (i, col) at d1[(i - col + KL) + NB col])
  double qi = 0.0, qo = 0.0;
  for (int col = 0; col <= KL && col < N; ++col) qi += d1[(0 - col + KL) + NB * col] * re[(size_t)col * NM];
  for (int col = N - 1 - KL < 0 ? 0 : N - 1 - KL; col < N; ++col)
    qo += d1[(N - 1 - col + KL) + NB * col] * re[(size_t)col * NM];
  const double ei = fi ? bv[j] - qi : 0.0, eo = fo ? bv[NM + j] - qo : 0.0;
  double c1 = 0.0, c2 = 0.0;
  const double* tb = tc.tau + 4 * (size_t)sv.base;
  const double* kc = tc.consts + 6 * (size_t)blockIdx.y;
  const double dt1i = kc[0], dt1o = kc[1], dt2i = kc[2], dt2o = kc[3], din = kc[4], dout = kc[5];
  const double *t1 = tb, *t2 = tb + N;
  if (fi && fo) {  // compute_tau_coefficients_both
    const double det = dt1i * dt2o - dt1o * dt2i;
    if (fabs(det) > 1e-12) {
      c1 = (ei * dt2o - eo * dt2i) / det;
      c2 = (eo * dt1i - ei * dt1o) / det;
    }
  } else if (fi) {  // compute_tau_coefficients_inner
    c1 = ei / din;
    t1 = tb + 2 * N;
    t2 = nullptr;
  } else {          // compute_tau_coefficients_outer
    c1 = eo / dout;
    t1 = tb + 3 * N;
    t2 = nullptr;
  }
  bool im_live = false;
  for (int i = 0; i < N; ++i) im_live |= fabs(im[(size_t)i * NM]) > 1e-12;
  for (int i = 0; i < N; ++i) {
    // profile += c1 tau1 + c2 tau2, without contraction into fused multiply-adds
    double corr = __dmul_rn(c1, t1[i]);
    if (t2) corr = __dadd_rn(corr, __dmul_rn(c2, t2[i]));
    re[(size_t)i * NM] = __dadd_rn(re[(size_t)i * NM], corr);
    if (im_live) im[(size_t)i * NM] = __dadd_rn(im[(size_t)i * NM], corr);
  }
  if (regular) re[0] = im[0] = 0.0;
}

// enforce_ball_scalar_regularity! / enforce_ball_vector_regularity!
// (src/Ball/Ball.jl:153-195): the r = 0 level (the first of every segment) of
// each of nf fields is set to 0 for l >= 1.
__global__ void k_regularity(Dims d, const int* __restrict__ lof, double* __restrict__ F, int nf, size_t fstride) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.nlm || lof[j] < 1) return;
  const size_t NM = d.nlm, plane = (size_t)d.nr * NM;
  double* f = F + blockIdx.z * fstride + (size_t)seg_view(d, blockIdx.y).base * NM + j;
  f[0] = 0.0;
  f[plane] = 0.0;
}

void launch_regularity(cudaStream_t s, const Dims& d, const int* lof, double* F, int nf, size_t fstride) {
  if (!d.ball || nf < 1) return;
  k_regularity<<<dim3(ceil_div(d.nlm, 128), d.nseg, nf), 128, 0, s>>>(d, lof, F, nf, fstride);
}

void launch_scalar_bc(cudaStream_t s, const Dims& d, const int* lof, const double* bvals_native, const int* types,
                      const double* d1, const TauConsts& tc, double* F, int op_rows) {
  k_scalar_bc<<<dim3(ceil_div(d.jhi - d.jlo, 128), d.nseg), 128, 0, s>>>(d, lof, bvals_native, types, d1, tc, F,
                                                                        op_rows);
}

__global__ void k_perm(int nlm, size_t rows, const int* __restrict__ perm, const double* __restrict__ src,
                       double* __restrict__ dst, int to_native) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t row = blockIdx.y + (size_t)gridDim.y * blockIdx.z;
  if (q >= nlm || row >= rows) return;
  const size_t base = row * nlm;
  if (to_native) dst[base + perm[q]] = src[base + q];
  else dst[base + q] = src[base + perm[q]];
}

static void launch_perm(cudaStream_t s, const Dims& d, const int* perm, const double* src, double* dst, int nplanes,
                        int to_native) {
  const size_t rows = (size_t)nplanes * d.nr;
  const unsigned gy = (unsigned)(rows < 65535 ? rows : 65535);
  const unsigned gz = (unsigned)((rows + gy - 1) / gy);
  dim3 grid(ceil_div(d.nlm, 256), gy, gz);
  k_perm<<<grid, 256, 0, s>>>(d.nlm, rows, perm, src, dst, to_native);
}

void launch_lmajor_to_native(cudaStream_t s, const Dims& d, const int* native_of_lmajor, const double* src,
                             double* dst, int nplanes) {
  launch_perm(s, d, native_of_lmajor, src, dst, nplanes, 1);
}
void launch_native_to_lmajor(cudaStream_t s, const Dims& d, const int* native_of_lmajor, const double* src,
                             double* dst, int nplanes) {
  launch_perm(s, d, native_of_lmajor, src, dst, nplanes, 0);
}

// Per-shell transpose between the reference grid layout [r][phi][theta] and
// the native [r][theta][phi].
__global__ void k_transpose(int rows_in, int cols_in, const double* __restrict__ src, double* __restrict__ dst) {
  __shared__ double tile[32][33];
  const size_t shell = blockIdx.z;
  const double* s = src + shell * (size_t)rows_in * cols_in;
  double* o = dst + shell * (size_t)rows_in * cols_in;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows_in && c < cols_in) tile[k][threadIdx.x] = s[(size_t)r * cols_in + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows_in && c < cols_in) o[(size_t)c * rows_in + r] = tile[threadIdx.x][k];
  }
}

void launch_grid_to_native(cudaStream_t s, const Dims& d, const double* ref, double* nat, int ncomp) {
  // ref: rows = phi (nlon), cols = theta (nlat)
  dim3 grid(ceil_div(d.nlat, 32), ceil_div(d.nlon, 32), (unsigned)(d.nr * ncomp));
  k_transpose<<<grid, dim3(32, 8), 0, s>>>(d.nlon, d.nlat, ref, nat);
}
void launch_grid_to_reference(cudaStream_t s, const Dims& d, const double* nat, double* ref, int ncomp) {
  dim3 grid(ceil_div(d.nlon, 32), ceil_div(d.nlat, 32), (unsigned)(d.nr * ncomp));
  k_transpose<<<grid, dim3(32, 8), 0, s>>>(d.nlat, d.nlon, nat, ref);
}

template <typename R>
__global__ void k_cast(size_t n, const R* __restrict__ src, double* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
template <typename R>
void launch_grid_cast(cudaStream_t s, size_t n, const R* src, double* dst) {
  k_cast<R><<<148 * 8, 256, 0, s>>>(n, src, dst);
}
template void launch_grid_cast<float>(cudaStream_t, size_t, const float*, double*);
template void launch_grid_cast<double>(cudaStream_t, size_t, const double*, double*);

}  // namespace gd

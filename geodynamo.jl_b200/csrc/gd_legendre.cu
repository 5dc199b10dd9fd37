// gd_legendre.cu -- FP64 Legendre synthesis and analysis as batched per-m
// contractions on the FP64 tensor pipe (DMMA m16n8k8), with even/odd folding.
//
// For a fixed order m the l-sum is split by the parity of l - m.  Even and
// odd partial sums come from separate warp groups (warps 0-3 even, 4-7 odd)
// that share one shared-memory tile; the epilogue combines them into the
// north and south rows (synthesis) or selects the folded input (analysis).
// These are the arithmetic of SHTnsKit.synthesis / analysis /
// SHsphtor_to_spat / spat_to_SHsphtor as called per shell in
// src/shtnskit_field_functions.jl:102-123, 218-239, 252-321, batched over all
// shells and fields in one launch.
#include <stdint.h>

#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"

namespace gd {

// D (16 x 8) += A (16 x 8, row-major) B (8 x 8, column-major) on the FP64 tensor
// pipe, per thread (g = lane / 4, t = lane % 4):
//   a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4];  b = B[t][g], B[t+4][g];
//   d = C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1].
__device__ __forceinline__ void dmma16(double& d0, double& d1, double& d2, double& d3, const double* a,
                                       const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d0), "+d"(d1), "+d"(d2), "+d"(d3)
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Asynchronous global -> shared copies of the operand tiles.  Every CTA keeps
// LEG_STAGES K chunks in flight: chunk c + LEG_STAGES - 1 is loading while
// chunk c is multiplied, so the tensor pipe does not wait for global latency.
// An invalid element (past the last degree, colatitude or column) is copied
// with a source size of 0, which writes zeros and reads nothing.
constexpr int LEG_STAGES = 3;

__device__ __forceinline__ void cpa8(double* sdst, const double* gsrc, bool valid) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cpa16(double* sdst, const double* gsrc, bool valid) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Scalar synthesis: F_m(theta) = sum_l a_lm Pbar_lm(theta), all fields/shells.
// CTA tile: 64 theta (north) x 64 columns n = (field, r, re/im); K chunks of
// 32 degrees (16 per parity) in a LEG_STAGES-deep cp.async pipeline.
// ---------------------------------------------------------------------------
#define SS_TM 64
#define SS_TN 64
#define SS_KC 32
#define SS_SA 66
#define SS_SB 66
constexpr int SS_STAGE = SS_KC * SS_SA + SS_KC * SS_SB;  // doubles per pipeline stage

static size_t synth_scalar_smem() { return (size_t)LEG_STAGES * SS_STAGE * sizeof(double) + SS_TN * sizeof(void*); }

__global__ void __launch_bounds__(256, 2) k_synth_scalar(Dims d, const int* __restrict__ moff,
                                                         const double* __restrict__ P, SynthArgs a) {
  extern __shared__ double smem[];
  // column n -> pointer to its coefficients of order m at degree 0 (null past the last column)
  const double** colp = reinterpret_cast<const double**>(smem + LEG_STAGES * SS_STAGE);
  const int m = blockIdx.z;
  const int th0 = blockIdx.y * SS_TM;
  const int n0 = blockIdx.x * SS_TN;
  const int Ntot = a.nf * d.nr * 2;
  if (th0 >= d.nth || n0 >= Ntot) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int par = warp >> 2, wq = warp & 3;
  const int thw = (wq >> 1) * 32, nw = (wq & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int mb = moff[m];
  const size_t NM = (size_t)d.nlm;
  for (int n = tid; n < SS_TN; n += 256) {
    const int ng = n0 + n;
    const double* p = nullptr;
    if (ng < Ntot) {
      const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
      p = a.coef[f] + ((size_t)c * d.nr + r) * NM + mb - m;
    }
    colp[n] = p;
  }
  __syncthreads();
  const int nch = (d.L - m + SS_KC) / SS_KC;  // K chunks of this order
  const bool pairs = (d.nth & 1) == 0;
  auto load = [&](int ch) {
    double* As = smem + (ch % LEG_STAGES) * SS_STAGE;  // [q][theta]
    double* Bs = As + SS_KC * SS_SA;                    // [q][n]
    const int l0 = m + ch * SS_KC;
    if (pairs) {  // two colatitudes per 16-byte copy (rows 16-byte aligned: nth even)
      for (int e = tid; e < SS_KC * SS_TM / 2; e += 256) {
        const int q = e / (SS_TM / 2), th = 2 * (e % (SS_TM / 2));
        const int l = l0 + q, ith = th0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        cpa16(As + q * SS_SA + th, ok ? P + (size_t)(mb + l - m) * d.nth + ith : P, ok);
      }
    } else {
      for (int e = tid; e < SS_KC * SS_TM; e += 256) {
        const int q = e / SS_TM, th = e % SS_TM;
        const int l = l0 + q, ith = th0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        cpa8(As + q * SS_SA + th, ok ? P + (size_t)(mb + l - m) * d.nth + ith : P, ok);
      }
    }
    for (int e = tid; e < SS_KC * SS_TN; e += 256) {
      const int q = e % SS_KC, n = e / SS_KC;
      const int l = l0 + q;
      const double* c = colp[n];
      const bool ok = c != nullptr && l <= d.L;
      cpa8(Bs + q * SS_SB + n, ok ? c + l : P, ok);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int c = 0; c < LEG_STAGES - 1; ++c) {
    if (c < nch) load(c);
    cpa_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cpa_wait<LEG_STAGES - 2>();
    __syncthreads();  // chunk ch landed; every warp is done with chunk ch - 1's stage
    if (ch + LEG_STAGES - 1 < nch) load(ch + LEG_STAGES - 1);
    cpa_commit();
    const double* As = smem + (ch % LEG_STAGES) * SS_STAGE;
    const double* Bs = As + SS_KC * SS_SA;
    // two K steps of 8 degrees of this warp's parity: rows q0 (k = 8 ks + t) and q1 (k + 4);
    // a step whose 16 degrees all lie past L only adds zero products and is skipped
#pragma unroll
    for (int ks = 0; ks < SS_KC / 16; ++ks) {
      if (m + ch * SS_KC + 16 * ks > d.L) break;
      const int q0 = 2 * (8 * ks + t) + par, q1 = q0 + 8;
      double af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r0 = thw + 16 * i + g;
        af[i][0] = As[q0 * SS_SA + r0];
        af[i][1] = As[q0 * SS_SA + r0 + 8];
        af[i][2] = As[q1 * SS_SA + r0];
        af[i][3] = As[q1 * SS_SA + r0 + 8];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bf[j][0] = Bs[q0 * SS_SB + nw + 8 * j + g];
        bf[j][1] = Bs[q1 * SS_SB + nw + 8 * j + g];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (n0 + nw + 8 * j < Ntot)  // column blocks past the last column stay zero
            dmma16(acc[2 * i][j][0], acc[2 * i][j][1], acc[2 * i + 1][j][0], acc[2 * i + 1][j][1], af[i], bf[j]);
    }
  }
  cpa_wait<0>();
  __syncthreads();
  // combine parities through shared memory
  double* Es = smem;  // [wq][i][j][lane][2]
  if (par == 1) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = (((wq * 4 + i) * 4 + j) * 32 + lane) * 2;
        Es[o] = acc[i][j][0];
        Es[o + 1] = acc[i][j][1];
      }
  }
  __syncthreads();
  if (par == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int ith = th0 + thw + 8 * i + g;
      if (ith >= d.nth) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int ng = n0 + nw + 8 * j + 2 * t;
        if (ng >= Ntot) continue;
        const int o = (((wq * 4 + i) * 4 + j) * 32 + lane) * 2;
        const double ore = Es[o], oim = Es[o + 1];
        const double ere = acc[i][j][0], eim = acc[i][j][1];
        const int f = ng / (2 * d.nr), r = (ng % (2 * d.nr)) >> 1;
        const size_t base = (((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2) * d.nth + ith;
        a.out[base] = make_double2(ere + ore, eim + oim);
        a.out[base + d.nth] = make_double2(ere - ore, eim - oim);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Vector synthesis (spheroidal S = poloidal, toroidal T):
//   V_theta = sum dP S + i sum Q T,   V_phi = i sum Q S - sum dP T.
// CTA tile: 32 theta x 32 columns n = (r, re/im); tables {dP, Q} x fields
// {S, T}; pipelined like the scalar synthesis.
// ---------------------------------------------------------------------------
#define VS_TM 32
#define VS_TN 32
#define VS_KC 32
#define VS_SA 34
#define VS_SB 34
constexpr int VS_STAGE = 2 * VS_KC * VS_SA + 2 * VS_KC * VS_SB;

static size_t synth_vector_smem() {
  return (size_t)LEG_STAGES * VS_STAGE * sizeof(double) + 2 * VS_TN * sizeof(void*);
}

__global__ void __launch_bounds__(256, 2) k_synth_vector(Dims d, const int* __restrict__ moff,
                                                         const double* __restrict__ dP,
                                                         const double* __restrict__ Q, SynthArgs a) {
  extern __shared__ double smem[];
  const double** colp = reinterpret_cast<const double**>(smem + LEG_STAGES * VS_STAGE);  // [fld][n]
  const int m = blockIdx.z;
  const int th0 = blockIdx.y * VS_TM;
  const int n0 = blockIdx.x * VS_TN;
  const int Ntot = d.nr * 2;
  if (th0 >= d.nth || n0 >= Ntot) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int par = warp >> 2, wq = warp & 3;
  const int thw = (wq >> 1) * 16, nw = (wq & 1) * 16;
  const int g = lane >> 2, t = lane & 3;
  const int mb = moff[m];
  const size_t NM = (size_t)d.nlm;
  for (int e = tid; e < 2 * VS_TN; e += 256) {
    const int fld = e / VS_TN, ng = n0 + e % VS_TN;
    colp[e] = ng < Ntot ? a.coef[fld] + ((size_t)(ng & 1) * d.nr + (ng >> 1)) * NM + mb - m : nullptr;
  }
  __syncthreads();
  const int nch = (d.L - m + VS_KC) / VS_KC;
  const bool pairs = (d.nth & 1) == 0;
  auto load = [&](int ch) {
    double* As = smem + (ch % LEG_STAGES) * VS_STAGE;  // [tab][q][theta]
    double* Bs = As + 2 * VS_KC * VS_SA;                // [fld][q][n]
    const int l0 = m + ch * VS_KC;
    if (pairs) {  // two colatitudes per 16-byte copy (rows 16-byte aligned: nth even)
      for (int e = tid; e < VS_KC * VS_TM; e += 256) {
        const int tab = e / (VS_KC * VS_TM / 2), rem = e % (VS_KC * VS_TM / 2);
        const int q = rem / (VS_TM / 2), th = 2 * (rem % (VS_TM / 2));
        const int l = l0 + q, ith = th0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        const double* T = tab == 0 ? dP : Q;
        cpa16(As + (tab * VS_KC + q) * VS_SA + th, ok ? T + (size_t)(mb + l - m) * d.nth + ith : T, ok);
      }
    } else {
      for (int e = tid; e < 2 * VS_KC * VS_TM; e += 256) {
        const int tab = e / (VS_KC * VS_TM), rem = e % (VS_KC * VS_TM);
        const int q = rem / VS_TM, th = rem % VS_TM;
        const int l = l0 + q, ith = th0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        const double* T = tab == 0 ? dP : Q;
        cpa8(As + (tab * VS_KC + q) * VS_SA + th, ok ? T + (size_t)(mb + l - m) * d.nth + ith : T, ok);
      }
    }
    for (int e = tid; e < 2 * VS_KC * VS_TN; e += 256) {
      const int fld = e / (VS_KC * VS_TN), rem = e % (VS_KC * VS_TN);
      const int q = rem % VS_KC, n = rem / VS_KC;
      const int l = l0 + q;
      const double* c = colp[fld * VS_TN + n];
      const bool ok = c != nullptr && l <= d.L;
      cpa8(Bs + (fld * VS_KC + q) * VS_SB + n, ok ? c + l : dP, ok);
    }
  };

  double acc[2][2][2][2][2];  // [tab][fld][i][j][re/im]
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[x][y][i][j][0] = acc[x][y][i][j][1] = 0.0;

#pragma unroll
  for (int c = 0; c < LEG_STAGES - 1; ++c) {
    if (c < nch) load(c);
    cpa_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cpa_wait<LEG_STAGES - 2>();
    __syncthreads();
    if (ch + LEG_STAGES - 1 < nch) load(ch + LEG_STAGES - 1);
    cpa_commit();
    const double* As = smem + (ch % LEG_STAGES) * VS_STAGE;
    const double* Bs = As + 2 * VS_KC * VS_SA;
#pragma unroll
    for (int ks = 0; ks < VS_KC / 16; ++ks) {
      if (m + ch * VS_KC + 16 * ks > d.L) break;  // only zero products left
      const int q0 = 2 * (8 * ks + t) + par, q1 = q0 + 8;
      double af[2][4], bf[2][2][2];
#pragma unroll
      for (int x = 0; x < 2; ++x) {
        const double* A0 = As + (x * VS_KC + q0) * VS_SA + thw + g;
        const double* A1 = As + (x * VS_KC + q1) * VS_SA + thw + g;
        af[x][0] = A0[0];
        af[x][1] = A0[8];
        af[x][2] = A1[0];
        af[x][3] = A1[8];
      }
#pragma unroll
      for (int y = 0; y < 2; ++y)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          bf[y][j][0] = Bs[(y * VS_KC + q0) * VS_SB + nw + 8 * j + g];
          bf[y][j][1] = Bs[(y * VS_KC + q1) * VS_SB + nw + 8 * j + g];
        }
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            if (n0 + nw + 8 * j < Ntot)
              dmma16(acc[x][y][0][j][0], acc[x][y][0][j][1], acc[x][y][1][j][0], acc[x][y][1][j][1], af[x],
                     bf[y][j]);
    }
  }
  cpa_wait<0>();
  __syncthreads();
  double* Es = smem;  // [wq][16 tiles][lane][2]
  if (par == 1) {
    int k = 0;
#pragma unroll
    for (int x = 0; x < 2; ++x)
#pragma unroll
      for (int y = 0; y < 2; ++y)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j, ++k) {
            const int o = ((wq * 16 + k) * 32 + lane) * 2;
            Es[o] = acc[x][y][i][j][0];
            Es[o + 1] = acc[x][y][i][j][1];
          }
  }
  __syncthreads();
  if (par == 0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int ith = th0 + thw + 8 * i + g;
      if (ith >= d.nth) continue;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int ng = n0 + nw + 8 * j + 2 * t;
        if (ng >= Ntot) continue;
        const int r = ng >> 1;
        // the odd-parity partial sums of this (i, j) tile, [tab][fld][re/im]
        double odd[2][2][1][1][2];
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
          for (int y = 0; y < 2; ++y) {
            const int o = ((wq * 16 + ((x * 2 + y) * 2 + i) * 2 + j) * 32 + lane) * 2;
            odd[x][y][0][0][0] = Es[o];
            odd[x][y][0][0][1] = Es[o + 1];
          }
        double2 v32[2][2];  // [comp][s]: the values of the blocked FP32 copy
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          // tab 0 = dP (parity opposite to P), tab 1 = Q (parity of P); fld 0 = S, 1 = T
          double DS[2], DT[2], QS[2], QT[2];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const double eDS = acc[0][0][i][j][c], oDS = odd[0][0][0][0][c];
            const double eDT = acc[0][1][i][j][c], oDT = odd[0][1][0][0][c];
            const double eQS = acc[1][0][i][j][c], oQS = odd[1][0][0][0][c];
            const double eQT = acc[1][1][i][j][c], oQT = odd[1][1][0][0][c];
            if (s == 0) {
              DS[c] = eDS + oDS; DT[c] = eDT + oDT; QS[c] = eQS + oQS; QT[c] = eQT + oQT;
            } else {
              DS[c] = oDS - eDS; DT[c] = oDT - eDT; QS[c] = eQS - oQS; QT[c] = eQT - oQT;
            }
          }
          const double2 vth = make_double2(DS[0] - QT[1], DS[1] + QT[0]);
          const double2 vph = make_double2(-QS[1] - DT[0], QS[0] - DT[1]);
          const size_t b0 = (((size_t)(0 * d.nr + r) * (d.M + 1) + m) * 2 + s) * d.nth + ith;
          const size_t b1 = (((size_t)(1 * d.nr + r) * (d.M + 1) + m) * 2 + s) * d.nth + ith;
          a.out[b0] = vth;
          a.out[b1] = vph;
          v32[0][s] = vth;
          v32[1][s] = vph;
        }
        if (a.out32 != nullptr) {
          constexpr int FBK = FOURIER_BLOCK;
          const size_t run = (size_t)((d.nth + FBK - 1) / FBK) * (d.M + 1) * FBK;
          const size_t off = (size_t)r * run + ((size_t)(ith / FBK) * (d.M + 1) + m) * FBK + ith % FBK;
#pragma unroll
          for (int c = 0; c < 2; ++c)
            a.out32[c * a.out32_comp + off] = make_float4((float)v32[c][0].x, (float)v32[c][0].y,
                                                          (float)v32[c][1].x, (float)v32[c][1].y);
        }
      }
    }
  }
}

void launch_synth_fp64(cudaStream_t s, const Dims& d, const int* moff, const SynthArgs& a, bool vec) {
  if (!vec) {
    dim3 grid(ceil_div(a.nf * d.nr * 2, SS_TN), ceil_div(d.nth, SS_TM), d.M + 1);
    allow_dynamic_smem(k_synth_scalar, synth_scalar_smem());
    k_synth_scalar<<<grid, 256, synth_scalar_smem(), s>>>(d, moff, a.table0, a);
  } else {
    dim3 grid(ceil_div(d.nr * 2, VS_TN), ceil_div(d.nth, VS_TM), d.M + 1);
    allow_dynamic_smem(k_synth_vector, synth_vector_smem());
    k_synth_vector<<<grid, 256, synth_vector_smem(), s>>>(d, moff, a.table0, a.table1, a);
  }
}

// ---------------------------------------------------------------------------
// Scalar analysis: a_lm = sum_{north theta} Pbar_lm(theta) G_{s(l-m)}(theta),
// with G_+ = w (G_N + G_S), G_- = w (G_N - G_S) prepared by the phi transform.
// CTA tile: 64 consecutive l (32 per parity) x 64 columns n = (field, r,
// re/im); K = colatitude in chunks of 16, pipelined.
// ---------------------------------------------------------------------------
#define SA_TL 64
#define SA_TN 64
#define SA_KC 16
#define SA_SA 18
#define SA_SB 68
#define SA_SO 66
constexpr int SA_STAGE = SA_TL * SA_SA + 2 * SA_KC * SA_SB;

static size_t analysis_scalar_smem() {
  return (size_t)LEG_STAGES * SA_STAGE * sizeof(double) + (SA_TN / 2) * sizeof(long long);
}

__global__ void __launch_bounds__(256, 2) k_analysis_scalar(Dims d, const int* __restrict__ moff,
                                                            const double* __restrict__ P, AnalysisArgs a) {
  extern __shared__ double smem[];
  // column pair -> offset of its folded input of order m (-1 past the last column)
  long long* colin = reinterpret_cast<long long*>(smem + LEG_STAGES * SA_STAGE);
  const int m = blockIdx.z;
  const int l0 = m + blockIdx.y * SA_TL;
  const int n0 = blockIdx.x * SA_TN;
  const int Ntot = a.nf * d.nr * 2;
  if (l0 > d.L || n0 >= Ntot) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int par = warp >> 2, wq = warp & 3;
  const int lw = (wq >> 1) * 16, nw = (wq & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int mb = moff[m];
  const size_t NM = (size_t)d.nlm;
  const int npairs = Ntot / 2;
  for (int pr = tid; pr < SA_TN / 2; pr += 256) {
    const int pg = n0 / 2 + pr;
    long long ib = -1;
    if (pg < npairs) {
      const int f = pg / d.nr, r = pg % d.nr;
      ib = (long long)(((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2) * d.nth;
    }
    colin[pr] = ib;
  }
  __syncthreads();
  const double* Gin = reinterpret_cast<const double*>(a.in);
  const int nch = (d.nth + SA_KC - 1) / SA_KC;
  const bool pairs = (d.nth & 1) == 0;
  auto load = [&](int ch) {
    double* As = smem + (ch % LEG_STAGES) * SA_STAGE;  // [l][theta]
    double* Bs = As + SA_TL * SA_SA;                    // [s][theta][n]
    const int k0 = ch * SA_KC;
    if (pairs) {  // two colatitudes per 16-byte copy (rows 16-byte aligned: nth even)
      for (int e = tid; e < SA_TL * SA_KC / 2; e += 256) {
        const int lq = e / (SA_KC / 2), th = 2 * (e % (SA_KC / 2));
        const int l = l0 + lq, ith = k0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        cpa16(As + lq * SA_SA + th, ok ? P + (size_t)(mb + l - m) * d.nth + ith : P, ok);
      }
    } else {
      for (int e = tid; e < SA_TL * SA_KC; e += 256) {
        const int lq = e / SA_KC, th = e % SA_KC;
        const int l = l0 + lq, ith = k0 + th;
        const bool ok = l <= d.L && ith < d.nth;
        cpa8(As + lq * SA_SA + th, ok ? P + (size_t)(mb + l - m) * d.nth + ith : P, ok);
      }
    }
    for (int e = tid; e < 2 * SA_KC * (SA_TN / 2); e += 256) {
      const int th = e % SA_KC, rest = e / SA_KC;
      const int sp = rest & 1, pr = rest >> 1;  // pr = column pair within tile
      const int ith = k0 + th;
      const long long ib = colin[pr];
      const bool ok = ib >= 0 && ith < d.nth;
      cpa16(Bs + (sp * SA_KC + th) * SA_SB + 2 * pr, ok ? Gin + 2 * ((size_t)ib + (size_t)sp * d.nth + ith) : Gin,
            ok);
    }
  };

  double acc[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int c = 0; c < LEG_STAGES - 1; ++c) {
    if (c < nch) load(c);
    cpa_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cpa_wait<LEG_STAGES - 2>();
    __syncthreads();
    if (ch + LEG_STAGES - 1 < nch) load(ch + LEG_STAGES - 1);
    cpa_commit();
    const double* As = smem + (ch % LEG_STAGES) * SA_STAGE;
    const double* Bs = As + SA_TL * SA_SA;
    // two K steps of 8 colatitudes: th0 = 8 ks + t and th0 + 4
#pragma unroll
    for (int ks = 0; ks < SA_KC / 8; ++ks) {
      const int th0 = 8 * ks + t, th1 = th0 + 4;
      const int lq0 = 2 * (lw + g) + par, lq1 = 2 * (lw + 8 + g) + par;
      double af[4], bf[4][2];
      af[0] = As[lq0 * SA_SA + th0];
      af[1] = As[lq1 * SA_SA + th0];
      af[2] = As[lq0 * SA_SA + th1];
      af[3] = As[lq1 * SA_SA + th1];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bf[j][0] = Bs[(par * SA_KC + th0) * SA_SB + nw + 8 * j + g];
        bf[j][1] = Bs[(par * SA_KC + th1) * SA_SB + nw + 8 * j + g];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma16(acc[0][j][0], acc[0][j][1], acc[1][j][0], acc[1][j][1], af, bf[j]);
    }
  }
  cpa_wait<0>();
  __syncthreads();
  // stage [n][l] in shared memory, then write contiguous l runs of each output plane
  double* Os = smem;  // [64 n][SA_SO]
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int lq = 2 * (lw + 8 * i + g) + par;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int nl = nw + 8 * j + 2 * t;
      double re = acc[i][j][0], im = acc[i][j][1];
      if (m == 0) im = 0.0;  // store_coefficients_from_shtnskit!, :433-435
      Os[nl * SA_SO + lq] = re;
      Os[(nl + 1) * SA_SO + lq] = im;
    }
  }
  __syncthreads();
  for (int e = tid; e < SA_TN * SA_TL; e += 256) {
    const int lq = e % SA_TL, nl = e / SA_TL;
    const int ng = n0 + nl, l = l0 + lq;
    if (ng < Ntot && l <= d.L) {
      const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
      a.out[f][((size_t)c * d.nr + r) * NM + mb + (l - m)] = Os[nl * SA_SO + lq];
    }
  }
}

// ---------------------------------------------------------------------------
// Vector analysis (spat_to_SHsphtor):
//   S = [sum dP G_th - i sum Q G_ph] / l(l+1),  T = [-i sum Q G_th - sum dP G_ph] / l(l+1)
// where the dP terms use the fold of opposite parity.  Columns n = (r, re/im);
// pipelined like the scalar analysis.
// ---------------------------------------------------------------------------
#define VA_TL 64
#define VA_TN 32
#define VA_KC 16
#define VA_SA 18
#define VA_SB 36
#define VA_SO 66
constexpr int VA_STAGE = 2 * VA_TL * VA_SA + 4 * VA_KC * VA_SB;

static size_t analysis_vector_smem() { return (size_t)LEG_STAGES * VA_STAGE * sizeof(double); }

__global__ void __launch_bounds__(256, 2) k_analysis_vector(Dims d, const int* __restrict__ moff,
                                                            const double* __restrict__ dP,
                                                            const double* __restrict__ Q, AnalysisArgs a) {
  extern __shared__ double smem[];
  const int m = blockIdx.z;
  const int l0 = m + blockIdx.y * VA_TL;
  const int n0 = blockIdx.x * VA_TN;
  const int Ntot = d.nr * 2;
  if (l0 > d.L || n0 >= Ntot) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int par = warp >> 2, wq = warp & 3;
  const int lw = (wq >> 1) * 16, nw = (wq & 1) * 16;
  const int g = lane >> 2, t = lane & 3;
  const int mb = moff[m];
  const size_t NM = (size_t)d.nlm;
  const int sP = par, sD = 1 - par;
  const double* Gin = reinterpret_cast<const double*>(a.in);
  const int nch = (d.nth + VA_KC - 1) / VA_KC;
  auto load = [&](int ch) {
    double* As = smem + (ch % LEG_STAGES) * VA_STAGE;  // [tab][l][theta]
    double* Bs = As + 2 * VA_TL * VA_SA;                // [comp][s][theta][n]
    const int k0 = ch * VA_KC;
    for (int e = tid; e < 2 * VA_TL * VA_KC; e += 256) {
      const int tab = e / (VA_TL * VA_KC), rem = e % (VA_TL * VA_KC);
      const int lq = rem / VA_KC, th = rem % VA_KC;
      const int l = l0 + lq, ith = k0 + th;
      const bool ok = l <= d.L && ith < d.nth;
      const double* T = tab == 0 ? dP : Q;
      cpa8(As + (tab * VA_TL + lq) * VA_SA + th, ok ? T + (size_t)(mb + l - m) * d.nth + ith : T, ok);
    }
    for (int e = tid; e < 4 * VA_KC * (VA_TN / 2); e += 256) {
      const int th = e % VA_KC, rest = e / VA_KC;
      const int cs = rest & 3, pr = rest >> 2;  // cs = comp*2 + s
      const int comp = cs >> 1, sp = cs & 1;
      const int r = n0 / 2 + pr, ith = k0 + th;
      const bool ok = r < d.nr && ith < d.nth;
      const size_t at = (((size_t)(comp * d.nr + r) * (d.M + 1) + m) * 2 + sp) * d.nth + ith;
      cpa16(Bs + (cs * VA_KC + th) * VA_SB + 2 * pr, ok ? Gin + 2 * at : Gin, ok);
    }
  };

  // acc[prod][i][j][c], prod: 0 = dP.Gth, 1 = dP.Gph, 2 = Q.Gth, 3 = Q.Gph
  double acc[4][2][2][2];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) acc[p][i][j][0] = acc[p][i][j][1] = 0.0;

#pragma unroll
  for (int c = 0; c < LEG_STAGES - 1; ++c) {
    if (c < nch) load(c);
    cpa_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cpa_wait<LEG_STAGES - 2>();
    __syncthreads();
    if (ch + LEG_STAGES - 1 < nch) load(ch + LEG_STAGES - 1);
    cpa_commit();
    const double* As = smem + (ch % LEG_STAGES) * VA_STAGE;
    const double* Bs = As + 2 * VA_TL * VA_SA;
#pragma unroll
    for (int ks = 0; ks < VA_KC / 8; ++ks) {
      const int th0 = 8 * ks + t, th1 = th0 + 4;
      const int lq0 = 2 * (lw + g) + par, lq1 = 2 * (lw + 8 + g) + par;
      double aD[4], aQ[4], bth[2][2][2], bph[2][2][2];  // b[fold][j][k half]
      aD[0] = As[(0 * VA_TL + lq0) * VA_SA + th0];
      aD[1] = As[(0 * VA_TL + lq1) * VA_SA + th0];
      aD[2] = As[(0 * VA_TL + lq0) * VA_SA + th1];
      aD[3] = As[(0 * VA_TL + lq1) * VA_SA + th1];
      aQ[0] = As[(1 * VA_TL + lq0) * VA_SA + th0];
      aQ[1] = As[(1 * VA_TL + lq1) * VA_SA + th0];
      aQ[2] = As[(1 * VA_TL + lq0) * VA_SA + th1];
      aQ[3] = As[(1 * VA_TL + lq1) * VA_SA + th1];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n = nw + 8 * j + g;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int th = h ? th1 : th0;
          bth[0][j][h] = Bs[((0 * 2 + sD) * VA_KC + th) * VA_SB + n];
          bph[0][j][h] = Bs[((1 * 2 + sD) * VA_KC + th) * VA_SB + n];
          bth[1][j][h] = Bs[((0 * 2 + sP) * VA_KC + th) * VA_SB + n];
          bph[1][j][h] = Bs[((1 * 2 + sP) * VA_KC + th) * VA_SB + n];
        }
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        dmma16(acc[0][0][j][0], acc[0][0][j][1], acc[0][1][j][0], acc[0][1][j][1], aD, bth[0][j]);
        dmma16(acc[1][0][j][0], acc[1][0][j][1], acc[1][1][j][0], acc[1][1][j][1], aD, bph[0][j]);
        dmma16(acc[2][0][j][0], acc[2][0][j][1], acc[2][1][j][0], acc[2][1][j][1], aQ, bth[1][j]);
        dmma16(acc[3][0][j][0], acc[3][0][j][1], acc[3][1][j][0], acc[3][1][j][1], aQ, bph[1][j]);
      }
    }
  }
  cpa_wait<0>();
  __syncthreads();
  double* Os = smem;  // [out field][32 n][VA_SO]
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int lq = 2 * (lw + 8 * i + g) + par;
    const int l = l0 + lq;
    const double f = (l == 0) ? 0.0 : 1.0 / ((double)l * (l + 1.0));
    const double lf = (double)l * (l + 1.0);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double Sre = (acc[0][i][j][0] + acc[3][i][j][1]) * f;
      const double Sim = (acc[0][i][j][1] - acc[3][i][j][0]) * f;
      const double Tre = (acc[2][i][j][1] - acc[1][i][j][0]) * f;
      const double Tim = (-acc[2][i][j][0] - acc[1][i][j][1]) * f;
      double o0re, o0im, o1re, o1im;  // out[0] = toroidal slot, out[1] = poloidal slot
      if (a.epi == EPI_CURL_INDUCTION) {
        // compute_curl_of_induction! (src/magnetic.jl:407-445)
        o0re = lf * Sre; o0im = lf * ((m == 0) ? 0.0 : Sim);
        o1re = -lf * Tre; o1im = -lf * ((m == 0) ? 0.0 : Tim);
      } else {
        o0re = Tre; o0im = (m == 0) ? 0.0 : Tim;
        o1re = Sre; o1im = (m == 0) ? 0.0 : Sim;
      }
      const int nl = nw + 8 * j + 2 * t;
      Os[(0 * 32 + nl) * VA_SO + lq] = o0re;
      Os[(0 * 32 + nl + 1) * VA_SO + lq] = o0im;
      Os[(1 * 32 + nl) * VA_SO + lq] = o1re;
      Os[(1 * 32 + nl + 1) * VA_SO + lq] = o1im;
    }
  }
  __syncthreads();
  for (int e = tid; e < 2 * 32 * VA_TL; e += 256) {
    const int lq = e % VA_TL, rest = e / VA_TL;
    const int nl = rest % 32, fo = rest / 32;
    const int ng = n0 + nl, l = l0 + lq;
    if (ng < Ntot && l <= d.L) {
      const int r = ng >> 1, c = ng & 1;
      a.out[fo][((size_t)c * d.nr + r) * NM + mb + (l - m)] = Os[(fo * 32 + nl) * VA_SO + lq];
    }
  }
}

void launch_analysis_fp64(cudaStream_t s, const Dims& d, const int* moff, const AnalysisArgs& a) {
  if (a.epi == EPI_SCALAR) {
    dim3 grid(ceil_div(a.nf * d.nr * 2, SA_TN), ceil_div(d.L + 1, SA_TL), d.M + 1);
    allow_dynamic_smem(k_analysis_scalar, analysis_scalar_smem());
    k_analysis_scalar<<<grid, 256, analysis_scalar_smem(), s>>>(d, moff, a.table0, a);
  } else {
    dim3 grid(ceil_div(d.nr * 2, VA_TN), ceil_div(d.L + 1, VA_TL), d.M + 1);
    allow_dynamic_smem(k_analysis_vector, analysis_vector_smem());
    k_analysis_vector<<<grid, 256, analysis_vector_smem(), s>>>(d, moff, a.table0, a.table1, a);
  }
}

}  // namespace gd

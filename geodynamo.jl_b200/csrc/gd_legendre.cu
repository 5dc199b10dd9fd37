// gd_legendre.cu -- FP64 Legendre synthesis and analysis as batched per-m
// contractions on the FP64 tensor pipe (DMMA m8n8k4), with even/odd folding.
//
// For a fixed order m the l-sum is split by the parity of l - m.  Even and
// odd partial sums come from separate warp groups (warps 0-3 even, 4-7 odd)
// that share one shared-memory tile; the epilogue combines them into the
// north and south rows (synthesis) or selects the folded input (analysis).
// These are the arithmetic of SHTnsKit.synthesis / analysis /
// SHsphtor_to_spat / spat_to_SHsphtor as called per shell in
// src/shtnskit_field_functions.jl:102-123, 218-239, 252-321, batched over all
// shells and fields in one launch.
#include "gd_internal.cuh"

namespace gd {

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// Scalar synthesis: F_m(theta) = sum_l a_lm Pbar_lm(theta), all fields/shells.
// CTA tile: 64 theta (north) x 64 columns n = (field, r, re/im).
// ---------------------------------------------------------------------------
#define SS_TM 64
#define SS_TN 64
#define SS_KC 32
#define SS_SA 66
#define SS_SB 66

__global__ void __launch_bounds__(256) k_synth_scalar(Dims d, const int* __restrict__ moff,
                                                      const double* __restrict__ P, SynthArgs a) {
  __shared__ double smem[SS_KC * SS_SA + SS_KC * SS_SB];
  double* As = smem;                   // [q][theta]
  double* Bs = smem + SS_KC * SS_SA;   // [q][n]
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

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  for (int l0 = m; l0 <= d.L; l0 += SS_KC) {
    // table tile
    for (int e = tid; e < SS_KC * SS_TM; e += 256) {
      const int q = e / SS_TM, th = e % SS_TM;
      const int l = l0 + q, ith = th0 + th;
      double v = 0.0;
      if (l <= d.L && ith < d.nth) v = P[(size_t)(mb + l - m) * d.nth + ith];
      As[q * SS_SA + th] = v;
    }
    // coefficient tile
    for (int e = tid; e < SS_KC * SS_TN; e += 256) {
      const int q = e % SS_KC, n = e / SS_KC;
      const int l = l0 + q, ng = n0 + n;
      double v = 0.0;
      if (l <= d.L && ng < Ntot) {
        const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
        v = a.coef[f][((size_t)c * d.nr + r) * NM + mb + (l - m)];
      }
      Bs[q * SS_SB + n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < SS_KC / 8; ++kk) {
      const int q = 2 * (4 * kk + t) + par;
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = As[q * SS_SA + thw + 8 * i + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[q * SS_SB + nw + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }
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
// CTA tile: 32 theta x 32 columns n = (r, re/im); tables {dP, Q} x fields {S, T}.
// ---------------------------------------------------------------------------
#define VS_TM 32
#define VS_TN 32
#define VS_KC 32
#define VS_SA 34
#define VS_SB 34

__global__ void __launch_bounds__(256) k_synth_vector(Dims d, const int* __restrict__ moff,
                                                      const double* __restrict__ dP,
                                                      const double* __restrict__ Q, SynthArgs a) {
  __shared__ double smem[2 * VS_KC * VS_SA + 2 * VS_KC * VS_SB];
  double* As = smem;                       // [tab][q][theta]
  double* Bs = smem + 2 * VS_KC * VS_SA;   // [fld][q][n]
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

  double acc[2][2][2][2][2];  // [tab][fld][i][j][re/im]
#pragma unroll
  for (int x = 0; x < 2; ++x)
#pragma unroll
    for (int y = 0; y < 2; ++y)
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[x][y][i][j][0] = acc[x][y][i][j][1] = 0.0;

  for (int l0 = m; l0 <= d.L; l0 += VS_KC) {
    for (int e = tid; e < 2 * VS_KC * VS_TM; e += 256) {
      const int tab = e / (VS_KC * VS_TM), rem = e % (VS_KC * VS_TM);
      const int q = rem / VS_TM, th = rem % VS_TM;
      const int l = l0 + q, ith = th0 + th;
      double v = 0.0;
      if (l <= d.L && ith < d.nth) v = (tab == 0 ? dP : Q)[(size_t)(mb + l - m) * d.nth + ith];
      As[(tab * VS_KC + q) * VS_SA + th] = v;
    }
    for (int e = tid; e < 2 * VS_KC * VS_TN; e += 256) {
      const int fld = e / (VS_KC * VS_TN), rem = e % (VS_KC * VS_TN);
      const int q = rem % VS_KC, n = rem / VS_KC;
      const int l = l0 + q, ng = n0 + n;
      double v = 0.0;
      if (l <= d.L && ng < Ntot) {
        const int r = ng >> 1, c = ng & 1;
        v = a.coef[fld][((size_t)c * d.nr + r) * NM + mb + (l - m)];
      }
      Bs[(fld * VS_KC + q) * VS_SB + n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < VS_KC / 8; ++kk) {
      const int q = 2 * (4 * kk + t) + par;
      double af[2][2], bf[2][2];
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int i = 0; i < 2; ++i) af[x][i] = As[(x * VS_KC + q) * VS_SA + thw + 8 * i + g];
#pragma unroll
      for (int y = 0; y < 2; ++y)
#pragma unroll
        for (int j = 0; j < 2; ++j) bf[y][j] = Bs[(y * VS_KC + q) * VS_SB + nw + 8 * j + g];
#pragma unroll
      for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y)
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma(acc[x][y][i][j][0], acc[x][y][i][j][1], af[x][i], bf[y][j]);
    }
    __syncthreads();
  }
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
    double odd[2][2][2][2][2];
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
            odd[x][y][i][j][0] = Es[o];
            odd[x][y][i][j][1] = Es[o + 1];
          }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int ith = th0 + thw + 8 * i + g;
      if (ith >= d.nth) continue;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int ng = n0 + nw + 8 * j + 2 * t;
        if (ng >= Ntot) continue;
        const int r = ng >> 1;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          // tab 0 = dP (parity opposite to P), tab 1 = Q (parity of P); fld 0 = S, 1 = T
          double DS[2], DT[2], QS[2], QT[2];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const double eDS = acc[0][0][i][j][c], oDS = odd[0][0][i][j][c];
            const double eDT = acc[0][1][i][j][c], oDT = odd[0][1][i][j][c];
            const double eQS = acc[1][0][i][j][c], oQS = odd[1][0][i][j][c];
            const double eQT = acc[1][1][i][j][c], oQT = odd[1][1][i][j][c];
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
        }
      }
    }
  }
}

void launch_synth_fp64(cudaStream_t s, const Dims& d, const int* moff, const SynthArgs& a, bool vec) {
  if (!vec) {
    dim3 grid(ceil_div(a.nf * d.nr * 2, SS_TN), ceil_div(d.nth, SS_TM), d.M + 1);
    k_synth_scalar<<<grid, 256, 0, s>>>(d, moff, a.table0, a);
  } else {
    dim3 grid(ceil_div(d.nr * 2, VS_TN), ceil_div(d.nth, VS_TM), d.M + 1);
    k_synth_vector<<<grid, 256, 0, s>>>(d, moff, a.table0, a.table1, a);
  }
}

// ---------------------------------------------------------------------------
// Scalar analysis: a_lm = sum_{north theta} Pbar_lm(theta) G_{s(l-m)}(theta),
// with G_+ = w (G_N + G_S), G_- = w (G_N - G_S) prepared by the phi transform.
// CTA tile: 64 consecutive l (32 per parity) x 128 columns n = (field, r, re/im).
// ---------------------------------------------------------------------------
#define SA_TL 64
#define SA_TN 128
#define SA_KC 16
#define SA_SA 18
#define SA_SB 132
#define SA_SO 66

__global__ void __launch_bounds__(256) k_analysis_scalar(Dims d, const int* __restrict__ moff,
                                                         const double* __restrict__ P, AnalysisArgs a) {
  __shared__ double smem[SA_TL * SA_SA + 2 * SA_KC * SA_SB];
  double* As = smem;                   // [l][theta]
  double* Bs = smem + SA_TL * SA_SA;   // [s][theta][n]
  const int m = blockIdx.z;
  const int l0 = m + blockIdx.y * SA_TL;
  const int n0 = blockIdx.x * SA_TN;
  const int Ntot = a.nf * d.nr * 2;
  if (l0 > d.L || n0 >= Ntot) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int par = warp >> 2, wq = warp & 3;
  const int lw = (wq >> 1) * 16, nw = (wq & 1) * 64;
  const int g = lane >> 2, t = lane & 3;
  const int mb = moff[m];
  const size_t NM = (size_t)d.nlm;
  const int npairs = Ntot / 2;

  double acc[2][8][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  for (int k0 = 0; k0 < d.nth; k0 += SA_KC) {
    for (int e = tid; e < SA_TL * SA_KC; e += 256) {
      const int lq = e / SA_KC, th = e % SA_KC;
      const int l = l0 + lq, ith = k0 + th;
      double v = 0.0;
      if (l <= d.L && ith < d.nth) v = P[(size_t)(mb + l - m) * d.nth + ith];
      As[lq * SA_SA + th] = v;
    }
    for (int e = tid; e < 2 * SA_KC * (SA_TN / 2); e += 256) {
      const int th = e % SA_KC, rest = e / SA_KC;
      const int s = rest & 1, pr = rest >> 1;  // pr = column pair within tile
      const int pg = n0 / 2 + pr, ith = k0 + th;
      double2 v = make_double2(0.0, 0.0);
      if (pg < npairs && ith < d.nth) {
        const int f = pg / d.nr, r = pg % d.nr;
        v = a.in[(((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2 + s) * d.nth + ith];
      }
      Bs[(s * SA_KC + th) * SA_SB + 2 * pr] = v.x;
      Bs[(s * SA_KC + th) * SA_SB + 2 * pr + 1] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < SA_KC / 4; ++kk) {
      const int th = 4 * kk + t;
      double af[2], bf[8];
#pragma unroll
      for (int i = 0; i < 2; ++i) af[i] = As[(2 * (lw + 8 * i + g) + par) * SA_SA + th];
#pragma unroll
      for (int j = 0; j < 8; ++j) bf[j] = Bs[(par * SA_KC + 4 * kk + (t)) * SA_SB + nw + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }
  // stage [n][l] in shared memory, half of the n tile at a time, then write
  // contiguous l runs of each output plane.
  double* Os = smem;  // [64 n][SA_SO]
  for (int half = 0; half < 2; ++half) {
    if ((nw >> 6) == half) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int lq = 2 * (lw + 8 * i + g) + par;
        const int l = l0 + lq;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int nl = 8 * j + 2 * t;  // within the half
          double re = acc[i][j][0], im = acc[i][j][1];
          if (m == 0) im = 0.0;  // store_coefficients_from_shtnskit!, :433-435
          (void)l;
          Os[nl * SA_SO + lq] = re;
          Os[(nl + 1) * SA_SO + lq] = im;
        }
      }
    }
    __syncthreads();
    for (int e = tid; e < 64 * SA_TL; e += 256) {
      const int lq = e % SA_TL, nl = e / SA_TL;
      const int ng = n0 + half * 64 + nl, l = l0 + lq;
      if (ng < Ntot && l <= d.L) {
        const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
        a.out[f][((size_t)c * d.nr + r) * NM + mb + (l - m)] = Os[nl * SA_SO + lq];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Vector analysis (spat_to_SHsphtor):
//   S = [sum dP G_th - i sum Q G_ph] / l(l+1),  T = [-i sum Q G_th - sum dP G_ph] / l(l+1)
// where the dP terms use the fold of opposite parity.  Columns n = (r, re/im).
// ---------------------------------------------------------------------------
#define VA_TL 64
#define VA_TN 32
#define VA_KC 16
#define VA_SA 18
#define VA_SB 36
#define VA_SO 66

__global__ void __launch_bounds__(256) k_analysis_vector(Dims d, const int* __restrict__ moff,
                                                         const double* __restrict__ dP,
                                                         const double* __restrict__ Q, AnalysisArgs a) {
  __shared__ double smem[2 * VA_TL * VA_SA + 4 * VA_KC * VA_SB];
  double* As = smem;                        // [tab][l][theta]
  double* Bs = smem + 2 * VA_TL * VA_SA;    // [comp][s][theta][n]
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

  // acc[prod][i][j][c], prod: 0 = dP.Gth, 1 = dP.Gph, 2 = Q.Gth, 3 = Q.Gph
  double acc[4][2][2][2];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) acc[p][i][j][0] = acc[p][i][j][1] = 0.0;

  for (int k0 = 0; k0 < d.nth; k0 += VA_KC) {
    for (int e = tid; e < 2 * VA_TL * VA_KC; e += 256) {
      const int tab = e / (VA_TL * VA_KC), rem = e % (VA_TL * VA_KC);
      const int lq = rem / VA_KC, th = rem % VA_KC;
      const int l = l0 + lq, ith = k0 + th;
      double v = 0.0;
      if (l <= d.L && ith < d.nth) v = (tab == 0 ? dP : Q)[(size_t)(mb + l - m) * d.nth + ith];
      As[(tab * VA_TL + lq) * VA_SA + th] = v;
    }
    for (int e = tid; e < 4 * VA_KC * (VA_TN / 2); e += 256) {
      const int th = e % VA_KC, rest = e / VA_KC;
      const int cs = rest & 3, pr = rest >> 2;  // cs = comp*2 + s
      const int comp = cs >> 1, s = cs & 1;
      const int r = n0 / 2 + pr, ith = k0 + th;
      double2 v = make_double2(0.0, 0.0);
      if (r < d.nr && ith < d.nth)
        v = a.in[(((size_t)(comp * d.nr + r) * (d.M + 1) + m) * 2 + s) * d.nth + ith];
      Bs[(cs * VA_KC + th) * VA_SB + 2 * pr] = v.x;
      Bs[(cs * VA_KC + th) * VA_SB + 2 * pr + 1] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < VA_KC / 4; ++kk) {
      const int th = 4 * kk + t;
      double aD[2], aQ[2], bth[2][2], bph[2][2];  // b[fold][j]
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int lq = 2 * (lw + 8 * i + g) + par;
        aD[i] = As[(0 * VA_TL + lq) * VA_SA + th];
        aQ[i] = As[(1 * VA_TL + lq) * VA_SA + th];
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n = nw + 8 * j + g;
        bth[0][j] = Bs[((0 * 2 + sD) * VA_KC + th) * VA_SB + n];
        bph[0][j] = Bs[((1 * 2 + sD) * VA_KC + th) * VA_SB + n];
        bth[1][j] = Bs[((0 * 2 + sP) * VA_KC + th) * VA_SB + n];
        bph[1][j] = Bs[((1 * 2 + sP) * VA_KC + th) * VA_SB + n];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          dmma(acc[0][i][j][0], acc[0][i][j][1], aD[i], bth[0][j]);
          dmma(acc[1][i][j][0], acc[1][i][j][1], aD[i], bph[0][j]);
          dmma(acc[2][i][j][0], acc[2][i][j][1], aQ[i], bth[1][j]);
          dmma(acc[3][i][j][0], acc[3][i][j][1], aQ[i], bph[1][j]);
        }
    }
    __syncthreads();
  }
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
    k_analysis_scalar<<<grid, 256, 0, s>>>(d, moff, a.table0, a);
  } else {
    dim3 grid(ceil_div(d.nr * 2, VA_TN), ceil_div(d.L + 1, VA_TL), d.M + 1);
    k_analysis_vector<<<grid, 256, 0, s>>>(d, moff, a.table0, a.table1, a);
  }
}

}  // namespace gd

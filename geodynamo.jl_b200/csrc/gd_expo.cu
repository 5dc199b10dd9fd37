// gd_expo.cu -- the exponential time schemes of apply_master_implicit_step!
// (ts_scheme = :eab2 and :erk2, src/simulation.jl:1054-1300) with the dense
// per-l caches of create_etd_cache (src/timestep.jl:37-70) and
// create_erk2_cache (:896-968).  Per radial system (field, l, m):
//   EAB2 (eab2_update!, :429-487):
//     u^{n+1} = E u^n + dt phi1 (3/2 N^n - 1/2 N^{n-1}),
//   ERK2 (erk2_prepare_field! / erk2_finalize_field!, :1316-1557):
//     stage   = E_h u^n + (dt/2) phi1_h N^n,
//     u^{n+1} = E u^n + dt (phi1 N^n + phi2 (N(stage) - N^n)),
// E = exp(dt A_l), phi1 = phi1(dt A_l), phi2 = phi2(dt A_l), E_h and phi1_h the
// same at dt/2; A_l = nu (d2 + (2/r) d1) - nu l(l+1)/r^2, the operator the
// CNAB2 matrices are built from (the handle's L_l band, same roundings).  The
// reference applies EAB2's E and phi1 to the velocity and magnetic fields by
// Krylov approximations (eab2_update_krylov_cached!, :358-427, m = 20, tol
// 1e-8); here every field uses the dense matrices, composition (kind 3)
// included.
#include "gd_internal.cuh"

namespace gd {

// ---------------------------------------------------------------------------
// Exponential cache.  E, phi1 and phi2 of X = dt A_l by scaling and squaring
// with truncated Taylor series: Y = X / 2^s with ||Y||_1 <= 1/2 and s >= 1,
//   E(Y) = sum Y^k / k!,  P(Y) = sum Y^k / (k + 1)!,  Q(Y) = sum Y^k / (k + 2)!
// for k <= K = 18 (the first omitted term is below 2^-19 / 19! ~ 1.6e-23 of
// ||Y||^0), then s doublings (functions of one matrix commute):
//   E(2Y) = E(Y)^2,  P(2Y) = P(Y) (E(Y) + I) / 2,  Q(2Y) = (2 Q(Y) + P(Y)^2) / 4,
// the last two from e^Y = I + Y P(Y) and P(Y) = I + Y Q(Y).  The half-step
// matrices are the state before the last doubling.  This forms phi1 and phi2
// without the inverse of A_l, which create_etd_cache and compute_phi1_function
// use: A_l has no boundary rows, so the radial equation's two homogeneous
// solutions leave it numerically singular (condition ~1e16 for every l).  One
// CTA per (kind, l); its n x n matrices live in a global scratch slice and
// every product is a CTA-wide tiled GEMM.  Output per (kind, l): five n x n
// blocks, each transposed (block b, row k = column k of the matrix) --
//   0: E, 1: phi1, 2: phi2, 3: E at dt/2, 4: phi1 at dt/2 --
// so that blocks 0 and 1 together are the EAB2 operand [E | phi1] with one
// contiguous k-row per stacked input row.
// ---------------------------------------------------------------------------
constexpr int EX_THREADS = 256;
constexpr int EX_T = 64;   // GEMM output tile (EX_T x EX_T), 4 x 4 per thread
constexpr int EX_K = 16;   // GEMM K chunk
constexpr int EX_TAYLOR = 18;
constexpr int ETD_BLOCKS = 5;

// C = alpha A B, n x n row-major in global memory (C distinct from A and B).
__device__ void ex_gemm(int n, const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
                        double alpha, double* sA, double* sB) {
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  for (int i0 = 0; i0 < n; i0 += EX_T)
    for (int j0 = 0; j0 < n; j0 += EX_T) {
      double acc[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = 0.0;
      for (int k0 = 0; k0 < n; k0 += EX_K) {
        for (int e = tid; e < EX_T * EX_K; e += EX_THREADS) {
          const int r = e / EX_K, c = e % EX_K;
          sA[e] = (i0 + r < n && k0 + c < n) ? A[(size_t)(i0 + r) * n + k0 + c] : 0.0;
          const int r2 = e / EX_T, c2 = e % EX_T;
          sB[e] = (k0 + r2 < n && j0 + c2 < n) ? B[(size_t)(k0 + r2) * n + j0 + c2] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < EX_K; ++k) {
          double a[4], b[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            a[q] = sA[(ty * 4 + q) * EX_K + k];
            b[q] = sB[k * EX_T + tx * 4 + q];
          }
#pragma unroll
          for (int p = 0; p < 4; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
        }
        __syncthreads();
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int gi = i0 + ty * 4 + p, gj = j0 + tx * 4 + q;
          if (gi < n && gj < n) C[(size_t)gi * n + gj] = alpha * acc[p][q];
        }
    }
  __syncthreads();
}

// lin: the handle's L_l bands, [kind][col][band][l] with entry (row i, col c)
// at band KL + i - c (k_build_lu).  scratch: 6 n^2 doubles per CTA.
__global__ void __launch_bounds__(EX_THREADS) k_etd_build(int n, int kl, int L, const double* __restrict__ lin,
                                                          double dt, double* __restrict__ scratch,
                                                          double* __restrict__ tab, int* err) {
  __shared__ double sA[EX_T * EX_K], sB[EX_K * EX_T];
  __shared__ double red[EX_THREADS / 32];
  __shared__ int s_sh;
  const int g = blockIdx.y, l = blockIdx.x;
  const int nb = 2 * kl + 1;
  const size_t n2 = (size_t)n * n;
  double* X = scratch + (size_t)(g * (L + 1) + l) * 6 * n2;
  double* Pw = X + n2;
  double* T = Pw + n2;
  double* E = T + n2;
  double* P = E + n2;
  double* Q = P + n2;
  double* out = tab + (size_t)(g * (L + 1) + l) * ETD_BLOCKS * n2;
  const double* Lb = lin + (size_t)g * n * nb * (L + 1) + l;
  const int tid = threadIdx.x;
  // X = dt A_l (dense)
  for (size_t e = tid; e < n2; e += EX_THREADS) {
    const int i = (int)(e / n), c = (int)(e % n);
    const int b = kl + i - c;
    X[e] = (b >= 0 && b < nb) ? dt * Lb[((size_t)c * nb + b) * (L + 1)] : 0.0;
  }
  __syncthreads();
  // s from the 1-norm (largest column sum), at least 1 for the half step
  double cmax = 0.0;
  for (int c = tid; c < n; c += EX_THREADS) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += fabs(X[(size_t)i * n + c]);
    cmax = fmax(cmax, sum);
  }
  for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if ((tid & 31) == 0) red[tid >> 5] = cmax;
  __syncthreads();
  if (tid == 0) {
    double v = 0.0;
    for (int w = 0; w < EX_THREADS / 32; ++w) v = fmax(v, red[w]);
    int s = 1;
    if (!(v < 1e300)) {  // not finite: flag and leave the table unusable
      atomicExch(err, 1);
      s = -1;
    } else {
      v *= 0.5;
      while (v > 0.5 && s < 1000) {
        v *= 0.5;
        ++s;
      }
    }
    s_sh = s;
  }
  __syncthreads();
  const int s = s_sh;
  if (s < 0) return;
  const double sc = ldexp(1.0, -s);
  // Y = X / 2^s (exact); E = I + Y, P = I + Y / 2, Q = I / 2 + Y / 6, Pw = Y
  for (size_t e = tid; e < n2; e += EX_THREADS) {
    const int i = (int)(e / n), c = (int)(e % n);
    const double y = X[e] * sc, id = i == c ? 1.0 : 0.0;
    X[e] = y;
    Pw[e] = y;
    E[e] = id + y;
    P[e] = id + 0.5 * y;
    Q[e] = 0.5 * id + y / 6.0;
  }
  __syncthreads();
  for (int k = 2; k <= EX_TAYLOR; ++k) {
    ex_gemm(n, Pw, X, T, 1.0 / k, sA, sB);  // T = Y^k / k!
    const double rk1 = 1.0 / (k + 1), rk12 = 1.0 / ((double)(k + 1) * (k + 2));
    for (size_t e = tid; e < n2; e += EX_THREADS) {
      const double t = T[e];
      Pw[e] = t;
      E[e] += t;
      P[e] += t * rk1;
      Q[e] += t * rk12;
    }
    __syncthreads();
  }
  // doublings; before the last one E and P are the half-step matrices
  for (int it = 0; it < s; ++it) {
    if (it == s - 1) {
      for (size_t e = tid; e < n2; e += EX_THREADS) {
        const int i = (int)(e / n), c = (int)(e % n);
        out[3 * n2 + (size_t)c * n + i] = E[e];
        out[4 * n2 + (size_t)c * n + i] = P[e];
      }
    }
    ex_gemm(n, P, P, T, 1.0, sA, sB);   // P^2
    for (size_t e = tid; e < n2; e += EX_THREADS) {
      const int i = (int)(e / n), c = (int)(e % n);
      Q[e] = 0.25 * (2.0 * Q[e] + T[e]);   // Q(2Y) = (2 Q + P^2) / 4
      X[e] = E[e] + (i == c ? 1.0 : 0.0);  // E + I
    }
    __syncthreads();
    ex_gemm(n, P, X, T, 0.5, sA, sB);   // P(2Y) = P (E + I) / 2
    ex_gemm(n, E, E, Pw, 1.0, sA, sB);  // E(2Y) = E^2
    for (size_t e = tid; e < n2; e += EX_THREADS) {
      P[e] = T[e];
      E[e] = Pw[e];
    }
    __syncthreads();
  }
  for (size_t e = tid; e < n2; e += EX_THREADS) {
    const int i = (int)(e / n), c = (int)(e % n);
    out[(size_t)c * n + i] = E[e];
    out[n2 + (size_t)c * n + i] = P[e];
    out[2 * n2 + (size_t)c * n + i] = Q[e];
  }
}

size_t etd_table_doubles(const Dims& d, int nkind) {
  return (size_t)nkind * (d.L + 1) * ETD_BLOCKS * d.nr * d.nr;
}
size_t etd_scratch_doubles(const Dims& d, int nkind) { return (size_t)nkind * (d.L + 1) * 6 * d.nr * d.nr; }

void launch_etd_build(cudaStream_t st, const Dims& d, const double* lin, double dt, double* scratch, double* tab,
                      int* err, int nkind) {
  k_etd_build<<<dim3(d.L + 1, nkind), EX_THREADS, 0, st>>>(d.nr, d.kl, d.L, lin, dt, scratch, tab, err);
}

// ---------------------------------------------------------------------------
// Applying the cache: out = M_top x_top + M_bot (c x_bot) per (field, l, m,
// plane) column, M_top and M_bot blocks of the (kind, l) table, x_top = u and
// x_bot = a, 3/2 a - 1/2 b or a - b (ExpApply); epilogue out = acc or
// out = lin + dt (k1 + acc).  CTA = (column chunk, l, field slot): the columns
// of order l are (m, plane) for m = 0 .. min(l, M), 64 per CTA; every thread
// owns an 8-row x 4-column tile of the output and the K loop runs over the
// stacked operand in chunks of 16 rows, double-buffered: asynchronous 8-byte
// copies of the next chunk's matrix rows and gathered input columns are in
// flight while the current chunk is multiplied (bottom inputs are combined
// once they land).  The columns are read in full before the tile is written,
// so out may be x_top.  16 x ceil(nr / 8) threads: nr <= 256.
// ---------------------------------------------------------------------------
constexpr int EU_COLS = 64;
constexpr int EU_RT = 8;   // rows per thread
constexpr int EU_CT = 4;   // columns per thread
constexpr int EU_KC = 16;  // K rows per chunk

__device__ __forceinline__ void eu_copy8(double* s, const double* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(s)), "l"(g)
               : "memory");
}

// MAXT = the thread bound the build is compiled for: 288 (nr <= 144, two CTAs
// per SM) or 512 (nr <= 256, one).
template <int MAXT>
__global__ void __launch_bounds__(MAXT, 576 / MAXT) k_exp_apply(Dims d, const int* __restrict__ moff,
                                                               const double* __restrict__ tab, ExpApply a) {
  extern __shared__ __align__(16) double eu_smem[];
  const int n = d.nr;
  const int npad = ((n + EU_RT - 1) / EU_RT) * EU_RT;
  double* sM = eu_smem;                       // [2][EU_KC][npad]: k-rows of the stacked matrix
  double* sA = sM + 2 * EU_KC * npad;         // [2][EU_KC][EU_COLS]: input rows (x_top, or a then x_bot)
  double* sB = sA + 2 * EU_KC * EU_COLS;      // [2][EU_KC][EU_COLS]: b rows
  __shared__ int colj[EU_COLS];               // column -> mode index j (-1 past the last column)
  __shared__ unsigned char colp[EU_COLS];
  const int slot = blockIdx.z;
  if (slot >= a.nfield) return;
  const int l = d.L - (int)blockIdx.y;
  const int mcount = min(l, d.M) + 1;
  const int c0 = blockIdx.x * EU_COLS;
  if (c0 >= 2 * mcount) return;
  const int g = a.kind[slot];
  const size_t NM = d.nlm, plane = (size_t)n * NM, n2 = (size_t)n * n;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int tx = tid % (EU_COLS / EU_CT), ty = tid / (EU_COLS / EU_CT);
  for (int c = tid; c < EU_COLS; c += nt) {
    const int cc = c0 + c;
    if (cc < 2 * mcount) {
      const int m = cc >> 1;
      colj[c] = moff[m] + l - m;
      colp[c] = (unsigned char)(cc & 1);
    } else {
      colj[c] = -1;
      colp[c] = 0;
    }
  }
  __syncthreads();
  const double* tl = tab + (size_t)(g * (d.L + 1) + l) * ETD_BLOCKS * n2;
  const double* Mt = a.top_block >= 0 ? tl + a.top_block * n2 : nullptr;
  const double* Mb = a.bot_block >= 0 ? tl + a.bot_block * n2 : nullptr;
  const double* __restrict__ xt = a.top[slot];
  const double* __restrict__ xa = a.bot_a[slot];
  const double* __restrict__ xb = a.bot_b[slot];
  const int ktop = Mt ? n : 0;
  const int K = ktop + (Mb ? n : 0);
  const bool two = a.bot_mode != 0;
  const int nch = (K + EU_KC - 1) / EU_KC;
  auto issue = [&](int ch, int buf) {
    const int k0 = ch * EU_KC;
    double* m_ = sM + buf * EU_KC * npad;
    double* a_ = sA + buf * EU_KC * EU_COLS;
    double* b_ = sB + buf * EU_KC * EU_COLS;
    for (int e = tid; e < EU_KC * npad; e += nt) {
      const int r = e / npad, i = e % npad, k = k0 + r;
      if (k < K && i < n)
        eu_copy8(m_ + e, (k < ktop ? Mt + (size_t)k * n : Mb + (size_t)(k - ktop) * n) + i);
      else
        m_[e] = 0.0;
    }
    for (int e = tid; e < EU_KC * EU_COLS; e += nt) {
      const int r = e / EU_COLS, c = e % EU_COLS, k = k0 + r;
      const int j = colj[c];
      if (j >= 0 && k < K) {
        const size_t at = (size_t)colp[c] * plane + (size_t)(k < ktop ? k : k - ktop) * NM + j;
        if (k < ktop) {
          eu_copy8(a_ + e, xt + at);
        } else {
          eu_copy8(a_ + e, xa + at);
          if (two) eu_copy8(b_ + e, xb + at);
        }
      } else {
        a_[e] = 0.0;
        b_[e] = 0.0;
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[EU_RT][EU_CT];
#pragma unroll
  for (int p = 0; p < EU_RT; ++p)
#pragma unroll
    for (int q = 0; q < EU_CT; ++q) acc[p][q] = 0.0;
  issue(0, 0);
  for (int ch = 0; ch < nch; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nch) {
      issue(ch + 1, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const int k0 = ch * EU_KC;
    double* a_ = sA + buf * EU_KC * EU_COLS;
    if (k0 + EU_KC > ktop) {
      // bottom rows: c a, c (3/2 a - 1/2 b) or c (a - b)
      const double* b_ = sB + buf * EU_KC * EU_COLS;
      for (int e = tid; e < EU_KC * EU_COLS; e += nt) {
        const int k = k0 + e / EU_COLS;
        if (k >= ktop && k < K) {
          const double v = a.bot_mode == 1 ? 1.5 * a_[e] - 0.5 * b_[e] : a.bot_mode == 2 ? a_[e] - b_[e] : a_[e];
          a_[e] = a.bot_scale * v;
        }
      }
      __syncthreads();
    }
    const double* m_ = sM + buf * EU_KC * npad;
#pragma unroll 4
    for (int r = 0; r < EU_KC; ++r) {
      double mv[EU_RT], xv[EU_CT];
      const double2* mr = reinterpret_cast<const double2*>(m_ + r * npad + ty * EU_RT);
      const double2* xr = reinterpret_cast<const double2*>(a_ + r * EU_COLS + tx * EU_CT);
#pragma unroll
      for (int p = 0; p < EU_RT / 2; ++p) {
        const double2 t = mr[p];
        mv[2 * p] = t.x;
        mv[2 * p + 1] = t.y;
      }
#pragma unroll
      for (int q = 0; q < EU_CT / 2; ++q) {
        const double2 t = xr[q];
        xv[2 * q] = t.x;
        xv[2 * q + 1] = t.y;
      }
#pragma unroll
      for (int p = 0; p < EU_RT; ++p)
#pragma unroll
        for (int q = 0; q < EU_CT; ++q) acc[p][q] = fma(mv[p], xv[q], acc[p][q]);
    }
    __syncthreads();
  }
  double* __restrict__ uo = a.out[slot];
  const double* __restrict__ lin = a.lin[slot];
  const double* __restrict__ k1 = a.k1[slot];
#pragma unroll
  for (int q = 0; q < EU_CT; ++q) {
    const int c = tx * EU_CT + q;
    const int j = colj[c];
    if (j < 0) continue;
    const size_t base = (size_t)colp[c] * plane + j;
#pragma unroll
    for (int p = 0; p < EU_RT; ++p) {
      const int i = ty * EU_RT + p;
      if (i >= n) continue;
      const size_t at = base + (size_t)i * NM;
      double v = acc[p][q];
      if (a.epilogue == 1) v = lin[at] + a.dt * (k1[at] + v);
      // bc_mode 1 zeroes the boundary rows after the update
      const bool clamp = a.clamp_rows && (i == 0 || i == n - 1);
      uo[at] = clamp ? 0.0 : v;
    }
  }
}

// The same contraction on the FP64 tensor cores (mma.sync m8n8k4, nr <= 144):
// 8 warps; warp (h, cp) owns row tiles h * TC_RTH .. + TC_RTH - 1 (8 rows each)
// and column tiles 2 cp, 2 cp + 1 (8 columns each) of the CTA's npad x 64
// output.  Fragments (lane = 4 g + t): A[g][t] = matrix row k = 4 s + t, column
// i = 8 tile + g; B[t][g] = input row k, column 8 tile + g; the accumulators
// hold C[g][2 t], C[g][2 t + 1].  Shared rows are strided by 4 mod 16 doubles,
// so the fragment loads are free of bank conflicts.
constexpr int TC_RTH = 9;              // row tiles per warp half: npad <= 144
constexpr int TC_THREADS = 256;
__host__ __device__ constexpr int tc_stride(int w) { return w + ((4 - w) % 16 + 16) % 16; }
constexpr int TC_SX = tc_stride(EU_COLS);  // 68

__device__ __forceinline__ void exp_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(TC_THREADS, 2) k_exp_apply_tc(Dims d, const int* __restrict__ moff,
                                                                const double* __restrict__ tab, ExpApply a) {
  extern __shared__ __align__(16) double eu_smem[];
  const int n = d.nr;
  const int npad = ((n + EU_RT - 1) / EU_RT) * EU_RT;
  const int SM = tc_stride(npad);
  double* sM = eu_smem;                       // [2][EU_KC][SM]
  double* sA = sM + 2 * EU_KC * SM;           // [2][EU_KC][TC_SX]
  double* sB = sA + 2 * EU_KC * TC_SX;        // [2][EU_KC][TC_SX]
  __shared__ int colj[EU_COLS];
  __shared__ unsigned char colp[EU_COLS];
  const int slot = blockIdx.z;
  if (slot >= a.nfield) return;
  const int l = d.L - (int)blockIdx.y;
  const int mcount = min(l, d.M) + 1;
  const int c0 = blockIdx.x * EU_COLS;
  if (c0 >= 2 * mcount) return;
  const int g = a.kind[slot];
  const size_t NM = d.nlm, plane = (size_t)n * NM, n2 = (size_t)n * n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int fg = lane >> 2, ft = lane & 3;
  const int wh = warp >> 2, wc = warp & 3;   // row half, column pair
  for (int c = tid; c < EU_COLS; c += TC_THREADS) {
    const int cc = c0 + c;
    if (cc < 2 * mcount) {
      const int m = cc >> 1;
      colj[c] = moff[m] + l - m;
      colp[c] = (unsigned char)(cc & 1);
    } else {
      colj[c] = -1;
      colp[c] = 0;
    }
  }
  __syncthreads();
  const double* tl = tab + (size_t)(g * (d.L + 1) + l) * ETD_BLOCKS * n2;
  const double* Mt = a.top_block >= 0 ? tl + a.top_block * n2 : nullptr;
  const double* Mb = a.bot_block >= 0 ? tl + a.bot_block * n2 : nullptr;
  const double* __restrict__ xt = a.top[slot];
  const double* __restrict__ xa = a.bot_a[slot];
  const double* __restrict__ xb = a.bot_b[slot];
  const int ktop = Mt ? n : 0;
  const int K = ktop + (Mb ? n : 0);
  const bool two = a.bot_mode != 0;
  const int nch = (K + EU_KC - 1) / EU_KC;
  auto issue = [&](int ch, int buf) {
    const int k0 = ch * EU_KC;
    double* m_ = sM + buf * EU_KC * SM;
    double* a_ = sA + buf * EU_KC * TC_SX;
    double* b_ = sB + buf * EU_KC * TC_SX;
    if (tid < npad) {  // thread tid copies matrix column tid of the chunk's rows
      for (int r = 0; r < EU_KC; ++r) {
        const int k = k0 + r;
        double* dst = m_ + r * SM + tid;
        if (k < K && tid < n)
          eu_copy8(dst, (k < ktop ? Mt + (size_t)k * n : Mb + (size_t)(k - ktop) * n) + tid);
        else
          *dst = 0.0;
      }
    }
    for (int e = tid; e < EU_KC * EU_COLS; e += TC_THREADS) {
      const int r = e >> 6, c = e & (EU_COLS - 1), k = k0 + r;
      const int j = colj[c];
      double* da = a_ + r * TC_SX + c;
      double* db = b_ + r * TC_SX + c;
      if (j >= 0 && k < K) {
        const size_t at = (size_t)colp[c] * plane + (size_t)(k < ktop ? k : k - ktop) * NM + j;
        if (k < ktop) {
          eu_copy8(da, xt + at);
        } else {
          eu_copy8(da, xa + at);
          if (two) eu_copy8(db, xb + at);
        }
      } else {
        *da = 0.0;
        *db = 0.0;
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  double acc[TC_RTH][2][2];
#pragma unroll
  for (int i = 0; i < TC_RTH; ++i)
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) acc[i][jj][0] = acc[i][jj][1] = 0.0;
  const int rt0 = wh * TC_RTH;          // first row tile of this warp
  const int nrt = npad / 8;             // row tiles of the CTA
  issue(0, 0);
  for (int ch = 0; ch < nch; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nch) {
      issue(ch + 1, buf ^ 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const int k0 = ch * EU_KC;
    double* a_ = sA + buf * EU_KC * TC_SX;
    if (k0 + EU_KC > ktop) {
      const double* b_ = sB + buf * EU_KC * TC_SX;
      for (int e = tid; e < EU_KC * EU_COLS; e += TC_THREADS) {
        const int r = e >> 6, c = e & (EU_COLS - 1), k = k0 + r;
        if (k >= ktop && k < K) {
          const int o = r * TC_SX + c;
          const double v = a.bot_mode == 1 ? 1.5 * a_[o] - 0.5 * b_[o] : a.bot_mode == 2 ? a_[o] - b_[o] : a_[o];
          a_[o] = a.bot_scale * v;
        }
      }
      __syncthreads();
    }
    const double* m_ = sM + buf * EU_KC * SM;
#pragma unroll
    for (int ks = 0; ks < EU_KC / 4; ++ks) {
      const int r = 4 * ks + ft;
      double bf[2];
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) bf[jj] = a_[r * TC_SX + (2 * wc + jj) * 8 + fg];
#pragma unroll
      for (int i = 0; i < TC_RTH; ++i) {
        if (rt0 + i < nrt) {
          const double af = m_[r * SM + (rt0 + i) * 8 + fg];
          exp_dmma(acc[i][0][0], acc[i][0][1], af, bf[0]);
          exp_dmma(acc[i][1][0], acc[i][1][1], af, bf[1]);
        }
      }
    }
    __syncthreads();
  }
  double* __restrict__ uo = a.out[slot];
  const double* __restrict__ lin = a.lin[slot];
  const double* __restrict__ k1 = a.k1[slot];
#pragma unroll
  for (int jj = 0; jj < 2; ++jj)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = (2 * wc + jj) * 8 + 2 * ft + h;
      const int j = colj[c];
      if (j < 0) continue;
      const size_t base = (size_t)colp[c] * plane + j;
#pragma unroll
      for (int i = 0; i < TC_RTH; ++i) {
        const int row = (rt0 + i) * 8 + fg;
        if (rt0 + i >= nrt || row >= n) continue;
        const size_t at = base + (size_t)row * NM;
        double v = acc[i][jj][h];
        if (a.epilogue == 1) v = lin[at] + a.dt * (k1[at] + v);
        // bc_mode 1 zeroes the boundary rows after the update
        const bool clamp = a.clamp_rows && (row == 0 || row == n - 1);
        uo[at] = clamp ? 0.0 : v;
      }
    }
}

int exp_apply_threads(const Dims& d) { return (EU_COLS / EU_CT) * ((d.nr + EU_RT - 1) / EU_RT); }

void launch_exp_apply(cudaStream_t st, const Dims& d, const int* moff, const double* tab, const ExpApply& a) {
  const int npad = ((d.nr + EU_RT - 1) / EU_RT) * EU_RT;
  const size_t smem = (size_t)2 * EU_KC * (npad + 2 * EU_COLS) * sizeof(double);
  allow_dynamic_smem(k_exp_apply<288>, smem);
  allow_dynamic_smem(k_exp_apply<512>, smem);
  const int ncc = ceil_div(2 * (d.M + 1), EU_COLS);
  const dim3 grid(ncc, d.L + 1, a.nfield);
  if (npad <= 2 * TC_RTH * 8) {
    const size_t tsmem = (size_t)2 * EU_KC * (tc_stride(npad) + 2 * TC_SX) * sizeof(double);
    allow_dynamic_smem(k_exp_apply_tc, tsmem);
    k_exp_apply_tc<<<grid, TC_THREADS, tsmem, st>>>(d, moff, tab, a);
    return;
  }
  const int nt = exp_apply_threads(d);
  if (nt <= 288)
    k_exp_apply<288><<<grid, nt, smem, st>>>(d, moff, tab, a);
  else
    k_exp_apply<512><<<grid, nt, smem, st>>>(d, moff, tab, a);
}

}  // namespace gd

// gd_ozaki.cu -- FP64-accurate vector synthesis on the 5th-generation tensor
// cores by integer digit slices (tcgen05.mma kind::i8, int32 accumulation in
// tensor memory).
//
// Splitting.  Every operand value x is scaled by a power of two (one exponent
// e per table row, one per coefficient column, both over the degrees of both
// parities, with |x| < 2^e) and rounded to the integer X = rint(x 2^(7G-1-e)),
// which is written as G signed digits in balanced base 128,
//   X = sum_{i<G} d_i 128^(G-1-i),  d_0 in [-64, 64], d_i in [-64, 63],
// so x = 2^e sum_i d_i 2^(-6-7i) + r with |r| <= 2^(e-7G) (round to nearest:
// unbiased).  A digit product d_i d'_j is exact in int32, and so is every sum
// of them the tensor core forms (|sum| <= G K 64^2 << 2^31).  Products of one
// group g = i + j share the weight 2^(-12-7g) and accumulate in one TMEM
// accumulator; groups g >= G are not formed.  The epilogue forms
// sum_g acc_g 128^(G-1-g) exactly in int64 (|sum| < 2^58), combines the even
// and odd parities exactly, converts once to FP64 and multiplies by the row
// and column scales 2^(e_row - 12 - 7(G-1)) and 2^(e_col).  This is the
// error-free transformation of Ozaki, Ogita, Oishi and Rump (Numer.
// Algorithms 59, 2012) on int8 digits
// with the product triangle cut at G groups; the error of one term is about
// 2^(-7G) of (row max)(column max), against 2^-53 of |x y| in FP64.
//
// Operation: the vector synthesis of SHsphtor_to_spat (per shell in
// src/shtnskit_field_functions.jl:252-321),
//   V_theta = sum dP S + i sum Q T,   V_phi = i sum Q S - sum dP T,
// with Q = m Pbar / sin(theta), for all shells of one field pair in one launch,
// writing the FP64 Fourier layout of the DMMA synthesis (and its FP32 blocked
// copy).  Parity: for each order m the sum over l splits by the parity of
// l - m; north = even + odd, south = even - odd (dP has the opposite
// symmetry).
//
// Tile = (m, 64 colatitudes, N coefficient columns).  The MMA's M = 128 rows
// are the 64 dP rows and the 64 Q rows of those colatitudes, so the two
// tables share one B operand; the accumulators are [parity][group] x N.  One
// pipeline step is one 32-degree K step of one parity: the G table slices
// and the G coefficient slices of that step (K-major, SWIZZLE_32B: 32-byte
// rows, so a step copies exactly its degrees), and G MMAs: table digit i
// against coefficient digits 0 .. G-1-i as one B operand of (G - i) N
// columns.  The even-parity accumulators are drained while the odd-parity MMAs run and are
// free again for the next tile's even MMAs.  The dP and Q rows of one
// colatitude sit in different TMEM lane quarters: their partial results meet
// in shared memory.
#include <algorithm>

#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"
#include "gd_ozaki.cuh"
#include "gd_tc.cuh"

namespace gd {

using namespace tc;

namespace {

constexpr int OZ_TH = 64;                 // colatitudes per tile
constexpr int OZ_M = 2 * OZ_TH;           // MMA rows: dP then Q
constexpr int OZ_KS = 32;                 // degrees per K step (one int8 MMA)
constexpr int OZ_A_SLICE = OZ_M * OZ_KS;  // one table slice of one K step (4 KB)
constexpr int OZ_THREADS = 320;           // producer, MMA issuer, 8 epilogue warps
constexpr int OZ_EPI = OZ_THREADS - 64;
constexpr int OZ_PB = 256;                // TMEM columns per parity
constexpr int OZ_SMEM_MAX = 232448;       // 227 KB of dynamic shared memory per CTA
constexpr int OZ_COEF_SMEM = 200 * 1024;  // the coefficient columns of one image tile (lmax <= 511)
constexpr int OZ_CT = 512;                // threads of a coefficient-image CTA

__host__ __device__ __forceinline__ int oz_kpar(int L, int m, int p) {
  return p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2;
}
// K steps of parity p of order m, and their maximum over m (order 0, even)
__host__ __device__ __forceinline__ int oz_nks(int L, int m, int p) { return (oz_kpar(L, m, p) + OZ_KS - 1) / OZ_KS; }
__host__ __device__ __forceinline__ int oz_nksmax(int L) { return oz_nks(L, 0, 0); }

// Byte offset of (row, k) in a K-major SWIZZLE_32B tile of 32-byte rows: 8-row
// atoms of 256 bytes, the 16-byte half index XOR-ed with bit 2 of the row.
__host__ __device__ __forceinline__ uint32_t sw32_byte(uint32_t row, uint32_t k) {
  return (row >> 3) * 256u + (row & 7u) * 32u + ((((k >> 4) ^ (row >> 2)) & 1u) << 4) + (k & 15u);
}

// Shared-memory matrix descriptor of a K-major SWIZZLE_32B tile: start >> 4,
// LBO 16 B (unused: one atom spans the MMA's K), SBO 256 B between 8-row
// groups, version 1, layout SWIZZLE_32B (6) in [61,64).
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(256u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)6u << 61);
}

// Smallest e with |x| < 2^e for every x of a row or column of maximum amax.
__device__ __forceinline__ int oz_exp(double amax) { return amax > 0.0 ? ilogb(amax) + 1 : 0; }

// The G balanced base-128 digits of X = rint(x * sc) (sc = 2^(7G-1-e), so
// |x sc| < 2^(7G-1)); digit 0 most significant.
template <int G>
__device__ __forceinline__ void oz_digits(double x, double sc, signed char* dg) {
  long long X = __double2ll_rn(x * sc);
#pragma unroll
  for (int i = G - 1; i > 0; --i) {
    const int d = (int)(((X + 64) & 127) - 64);
    dg[i] = (signed char)d;
    X = (X - d) >> 7;
  }
  dg[0] = (signed char)X;
}

// Instruction descriptor, kind::i8: D S32 (bits 4-5 = 2), A and B signed 8-bit
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ __forceinline__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// 32 lanes x 8 columns of int32 accumulators.
__device__ __forceinline__ void tmem_ld8i(uint32_t taddr, int* v) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = (int)r[i];
}

// Tiles of the synthesis: (m, colatitude tile, column tile), column tile fastest
// so that consecutive tiles reuse one table image from L2.
struct OzTile {
  int m, th, ct;
};
__device__ __forceinline__ OzTile oz_tile(int tt, int ntt, int ncb) {
  OzTile t;
  t.ct = tt % ncb;
  t.th = (tt / ncb) % ntt;
  t.m = tt / (ncb * ntt);
  return t;
}

// Shared memory of one CTA: stages, the dP/Q exchange, barriers.
template <int G, int N>
struct OzSmem {
  static constexpr int B_SLICE = N * OZ_KS;
  static constexpr int STEP = G * OZ_A_SLICE + G * B_SLICE;        // bytes of one step
  static constexpr int ST = (STEP + 1023) / 1024 * 1024;            // stage stride
  static constexpr int XCH = 2 * OZ_TH * (N / 4) * 8 * 8;          // exchange bytes (two buffers)
  static constexpr int CSC = 2 * N * 8;                             // column scales (two buffers)
  static constexpr int FIXED = 1024 + XCH + CSC + 512;              // alignment slack, exchange, scales, barriers
  static constexpr int S = (OZ_SMEM_MAX - FIXED) / ST;              // stages
  static constexpr int BYTES = FIXED + S * ST;
};

}  // namespace

// ---------------------------------------------------------------------------
// Table images (set-up): step (m, th, p, ks) = G slices of 128 rows x 32 bytes,
// rows 0-63 dP and 64-127 Q of colatitudes 64 th + row % 64, byte k ->
// l = m + p + 2 (32 ks + k); row scale 2^(e - 12 - 7(G-1)) per (m, th, row),
// e over the degrees of both parities.
// ---------------------------------------------------------------------------
template <int G>
__global__ void __launch_bounds__(OZ_M) k_oz_table_image(Dims d, const int* __restrict__ moff,
                                                         const double* __restrict__ dP,
                                                         const double* __restrict__ Q, signed char* __restrict__ img,
                                                         double* __restrict__ rsc) {
  const int th = blockIdx.x, m = blockIdx.y, p = blockIdx.z;
  const int row = threadIdx.x;
  const int ntt = (d.nth + OZ_TH - 1) / OZ_TH, nks = oz_nksmax(d.L);
  const int K = oz_kpar(d.L, m, p);
  const int ith = th * OZ_TH + (row & (OZ_TH - 1));
  const double* T = row < OZ_TH ? dP : Q;
  const bool ok = ith < d.nth;
  const size_t base = (size_t)moff[m] + p;  // table row of degree m + p
  // one exponent for both parities, so that the epilogue combines the even
  // and odd sums in integers
  double amax = 0.0;
  if (ok)
    for (int l = m; l <= d.L; ++l) amax = fmax(amax, fabs(T[((size_t)moff[m] + l - m) * d.nth + ith]));
  const int e = oz_exp(amax);
  const size_t tix = ((size_t)m * ntt + th) * 2 + p;
  if (p == 0) rsc[((size_t)m * ntt + th) * OZ_M + row] = ldexp(1.0, e - 12 - 7 * (G - 1));
  const double sc = ldexp(1.0, 7 * G - 1 - e);
  for (int ks = 0; ks < nks; ++ks) {
    signed char* out = img + (tix * nks + ks) * (size_t)G * OZ_A_SLICE;
    for (int k = 0; k < OZ_KS; ++k) {
      const int kk = ks * OZ_KS + k;
      const double x = (ok && kk < K) ? T[(base + 2 * (size_t)kk) * d.nth + ith] : 0.0;
      signed char dg[G];
      oz_digits<G>(x, sc, dg);
      const uint32_t o = sw32_byte(row, k);
#pragma unroll
      for (int i = 0; i < G; ++i) out[(size_t)i * OZ_A_SLICE + o] = dg[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Coefficient images (every call): step (m, p, ct, ks) = G slices of N rows x
// 32 bytes, row c = column (shell ct N/4 + c/4, [S re, S im, T re, T im][c % 4]),
// byte k -> l = m + p + 2 (32 ks + k); column scale 2^e per (m, ct, c), e over
// the degrees of both parities.
// Only the K steps of the order's degrees are written (the MMAs read no
// others).
// ---------------------------------------------------------------------------
template <int G, int N>
__global__ void __launch_bounds__(OZ_CT) k_oz_coef_image(Dims d, const int* __restrict__ moff,
                                                       const double* __restrict__ S, const double* __restrict__ T,
                                                       signed char* __restrict__ img, double* __restrict__ csc,
                                                       int ncb) {
  constexpr int BSL = N * OZ_KS;
  extern __shared__ double cv[];  // [N][L - m + 1]: the tile's columns, degree fastest
  __shared__ double sc[1][N];
  const int ct = blockIdx.x, m = blockIdx.y;
  const int nks = oz_nksmax(d.L);
  const int nl = d.L - m + 1;
  const size_t NM = d.nlm;
  const int mb = moff[m];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NW = OZ_CT / 32;
  // one coalesced read of every coefficient of the tile, eight loads in flight
  // per lane, and the column maximum over the degrees of both parities
  for (int c = warp; c < N; c += NW) {
    const int r = ct * (N / 4) + (c >> 2), fld = (c >> 1) & 1, ci = c & 1;
    const double* src = r < d.nr ? (fld == 0 ? S : T) + ((size_t)ci * d.nr + r) * NM + mb : nullptr;
    double amax = 0.0;
    for (int j0 = 0; j0 < nl; j0 += 256) {
      double x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = j0 + 32 * u + lane;
        x[u] = (src != nullptr && j < nl) ? __ldg(src + j) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = j0 + 32 * u + lane;
        if (j < nl) cv[c * nl + j] = x[u];
        amax = fmax(amax, fabs(x[u]));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (lane == 0) {
      const int e = oz_exp(amax);
      sc[0][c] = ldexp(1.0, 7 * G - 1 - e);
      csc[((size_t)m * ncb + ct) * N + c] = ldexp(1.0, e);
    }
  }
  __syncthreads();
  // digits: each thread four consecutive degrees of one column, one 32-bit
  // word per slice (the four bytes stay together under the 32-byte swizzle)
  for (int p = 0; p < 2; ++p) {
    const int nk = oz_nks(d.L, m, p);
    for (int ks = 0; ks < nk; ++ks) {
      signed char* out = img + ((((size_t)m * 2 + p) * ncb + ct) * nks + ks) * (size_t)G * BSL;
      for (int e = tid; e < N * (OZ_KS / 4); e += blockDim.x) {
        const int c = e / (OZ_KS / 4), k0 = 4 * (e % (OZ_KS / 4));
        uint32_t w[G];
#pragma unroll
        for (int i = 0; i < G; ++i) w[i] = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int j = p + 2 * (ks * OZ_KS + k0 + u);  // degree m + j
          const double x = j < nl ? cv[c * nl + j] : 0.0;
          signed char dg[G];
          oz_digits<G>(x, sc[0][c], dg);
#pragma unroll
          for (int i = 0; i < G; ++i) w[i] |= (uint32_t)(uint8_t)dg[i] << (8 * u);
        }
        const uint32_t o = sw32_byte(c, k0);
#pragma unroll
        for (int i = 0; i < G; ++i) *reinterpret_cast<uint32_t*>(out + (size_t)i * BSL + o) = w[i];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The synthesis.  Persistent CTAs over tiles, 320 threads: warp 0 feeds the
// stages with bulk copies (step (p, ks): the G table slices and the G
// coefficient slices), warp 1 issues the MMAs (digit i of the table against
// digits 0 .. G-1-i of the coefficients in one MMA, products (i, j) into
// group i + j) and commits them to the stage's `empty` barrier and, after a
// parity's last step, to tfull[p]; warps 2-9 (two per TMEM lane quarter, half
// the columns each) drain parity p into FP64 on tfull[p], release it on
// tempty[p], combine north and south, meet their partner rows in shared
// memory and write the outputs.
// ---------------------------------------------------------------------------
template <int G, int N>
__global__ void __launch_bounds__(OZ_THREADS, 1) k_oz_synth_vector(Dims d, const signed char* __restrict__ imgA,
                                                                   const double* __restrict__ rsc,
                                                                   const signed char* __restrict__ imgB,
                                                                   const double* __restrict__ csc, int ncb,
                                                                   OzSynthArgs a) {
  using SM = OzSmem<G, N>;
  constexpr int S = SM::S;
  constexpr int BSL = SM::B_SLICE;
  constexpr int SH = N / 4;   // shells per tile
  constexpr int HC = N / 2;   // columns per epilogue half
  constexpr int HS = SH / 2;  // shells per epilogue half
  static_assert(G * N <= OZ_PB, "accumulators of one parity exceed their TMEM half");
  static_assert(N % 16 == 0 && HC % 8 == 0 && HS % 2 == 0, "tile width");
  static_assert(S >= 2, "pipeline stages");
  constexpr uint32_t NCOL = 512;
  extern __shared__ unsigned char smem_raw[];
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  unsigned char* stg = reinterpret_cast<unsigned char*>(base);
  double* xch = reinterpret_cast<double*>(base + (size_t)S * SM::ST);  // [2][SH][8][64 colatitudes]
  double* colsc = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(xch) + SM::XCH);  // [2][N]
  uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(colsc) + SM::CSC);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;  // [2]
  uint64_t* tempty = tfull + 2; // [2]
  uint64_t* drain = tempty + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
  int* sfail = reinterpret_cast<int*>(tslot + 1);

  const int L = d.L;
  const int ntt = (d.nth + OZ_TH - 1) / OZ_TH, nksm = oz_nksmax(L);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int p = 0; p < 2; ++p) {
      mbar_init(&tfull[p], 1);
      mbar_init(&tempty[p], OZ_EPI);
    }
    mbar_init(drain, 1);
    *sfail = 0;
  }
  if (warp == 0) tmem_alloc(tslot, NCOL);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const int ntiles = (d.M + 1) * ntt * ncb;
  bool ok = true;
  int issued = -1;   // producer: last pipeline step whose bulk copies were issued
  int omitted = -1;  // producer: the step an error-path test left out

  if (warp == 0) {
    int gs = 0;
    for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x) {
      const OzTile t = oz_tile(tt, ntt, ncb);
      for (int p = 0; p < 2 && ok; ++p) {
        const int nk = oz_nks(L, t.m, p);
        for (int ks = 0; ks < nk; ++ks) {
          const int Gs = gs++, s = Gs % S, u = Gs / S;
          if (u >= 1 && !mbar_wait(&empty[s], (u - 1) & 1, a.err, a.wait_limit)) {
            ok = false;
            break;
          }
          // error-path tests: CTA 0 may omit one step's copies, so the MMA
          // warp's bounded wait on that stage runs out
          const bool omit = a.omit_plus1 == Gs + 1 && blockIdx.x == 0;
          if (lane == 0 && !omit) {
            unsigned char* A = stg + (size_t)s * SM::ST;
            const size_t ta = (((size_t)t.m * ntt + t.th) * 2 + p) * nksm + ks;
            const size_t tb = (((size_t)t.m * 2 + p) * ncb + t.ct) * nksm + ks;
            mbar_arrive_expect_tx(&full[s], G * OZ_A_SLICE + G * BSL);
            bulk_g2s(A, imgA + ta * (G * OZ_A_SLICE), G * OZ_A_SLICE, &full[s]);
            bulk_g2s(A + G * OZ_A_SLICE, imgB + tb * (G * BSL), G * BSL, &full[s]);
          }
          if (!omit) issued = Gs;
          else omitted = Gs;
          __syncwarp();
        }
      }
    }
  } else if (warp == 1) {
    int gs = 0, q = 0;
    for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x, ++q) {
      const OzTile t = oz_tile(tt, ntt, ncb);
      for (int p = 0; p < 2 && ok; ++p) {
        if (q >= 1 && !mbar_wait(&tempty[p], (q - 1) & 1, a.err, a.wait_limit)) {
          ok = false;
          break;
        }
        const int nk = oz_nks(L, t.m, p);
        for (int ks = 0; ks < nk; ++ks) {
          const int Gs = gs++, s = Gs % S;
          if (!mbar_wait(&full[s], (Gs / S) & 1, a.err, a.wait_limit)) {
            ok = false;
            break;
          }
          fence_after_sync();
          if (lane == 0) {
            const uint32_t sa = smem_addr(stg + (size_t)s * SM::ST);
            const uint32_t sb = sa + G * OZ_A_SLICE;
            // one MMA per table digit i: the coefficient slices 0 .. G-1-i are
            // consecutive row blocks of one K-major tile, so they form one B
            // operand of (G - i) N columns, and their products land in the
            // accumulators of groups i .. G-1 (columns from i N)
#pragma unroll
            for (int i = 0; i < G; ++i)
              mma_i8(tmem + p * OZ_PB + i * N, sw32_desc(sa + i * OZ_A_SLICE), sw32_desc(sb), idesc_i8(OZ_M, (G - i) * N),
                     (ks == 0 && i == 0) ? 0u : 1u);
            mma_commit(smem_addr(&empty[s]));
            if (ks == nk - 1) mma_commit(smem_addr(&tfull[p]));
          }
          __syncwarp();
        }
        if (ok && nk == 0) {
          if (lane == 0) mma_commit(smem_addr(&tfull[p]));
          __syncwarp();
        }
      }
    }
  } else {
    const int qw = warp & 3, half = (warp - 2) >> 2, etid = tid - 64;
    const int row = qw * 32 + lane, tab = row >= OZ_TH ? 1 : 0, thl = row & (OZ_TH - 1);
    const uint32_t trow = tmem + ((uint32_t)(qw * 32) << 16);
    // dP rows write the outputs of the first HS/2 shells of their half, Q rows the rest
    const int own0 = tab == 0 ? 0 : HS / 2;
    const size_t FBK = FOURIER_BLOCK;
    const size_t run32 = (size_t)((d.nth + FBK - 1) / FBK) * (d.M + 1) * FBK;
    int q = 0;
    for (int tt = blockIdx.x; tt < ntiles; tt += gridDim.x, ++q) {
      const OzTile t = oz_tile(tt, ntt, ncb);
      const int ith = t.th * OZ_TH + thl;
      const int buf = q & 1;
      double* xb = xch + (size_t)buf * OZ_TH * SH * 8;
      double* cs = colsc + buf * N;
      // this tile's column scales into shared memory (read after the exchange barrier)
      if (etid < N) cs[etid] = csc[((size_t)t.m * ncb + t.ct) * N + etid];
      const double rs = rsc[((size_t)t.m * ntt + t.th) * OZ_M + row];
      long long S2[2][HC];  // per parity: sum_g acc_g 128^(G-1-g), exact
      bool good = true;
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const bool w = mbar_wait(&tfull[p], q & 1, a.err, a.wait_limit);
        good = good && w;
        fence_after_sync();
        const bool any = w && oz_kpar(L, t.m, p) > 0;
#pragma unroll
        for (int c0 = 0; c0 < HC; c0 += 8) {
          int acc[G][8];
          if (any) {
#pragma unroll
            for (int g = 0; g < G; ++g) tmem_ld8i(trow + p * OZ_PB + g * N + half * HC + c0, acc[g]);
            tmem_ld_wait();
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            long long x = 0;
            if (any) {
              x = acc[0][j];
#pragma unroll
              for (int g = 1; g < G; ++g) x = x * 128 + acc[g][j];
            }
            S2[p][c0 + j] = x;
          }
        }
        fence_before_sync();
        mbar_arrive(&tempty[p]);  // tensor memory back to the MMA warp
      }
      if (!good) atomicExch(sfail, 1);
      // per shell of this half: [S north re, im, T north re, im, S south re, im,
      // T south re, im] scaled by the row; north and south exact in int64;
      // shells k < HS/2 go out through the dP rows, the rest through the Q rows
      double own[HS / 2][8];
#pragma unroll
      for (int k2 = 0; k2 < HS / 2; ++k2) {
        double xa[8], xo[8];  // shells k2 and HS/2 + k2
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const long long Ea = S2[0][4 * k2 + c], Oa = S2[1][4 * k2 + c];
          const long long Eb = S2[0][4 * (HS / 2 + k2) + c], Ob = S2[1][4 * (HS / 2 + k2) + c];
          xa[c] = (double)(Ea + Oa) * rs;
          xo[c] = (double)(Eb + Ob) * rs;
          xa[4 + c] = (double)(tab == 0 ? Oa - Ea : Ea - Oa) * rs;
          xo[4 + c] = (double)(tab == 0 ? Ob - Eb : Eb - Ob) * rs;
        }
        const int kout = tab == 0 ? HS / 2 + k2 : k2;  // the shell this row hands over
        // [shell][value][colatitude]: the lanes of a warp (consecutive
        // colatitudes) touch consecutive words
        double* dst = xb + (size_t)(half * HS + kout) * 8 * OZ_TH + thl;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          own[k2][c] = tab == 0 ? xa[c] : xo[c];
          dst[c * OZ_TH] = tab == 0 ? xo[c] : xa[c];
        }
      }
      // one barrier per tile: the exchange and the column scales are double
      // buffered, so tile q + 2 writes them only after every thread has passed
      // this barrier of tile q + 1, that is, after its reads of tile q
      named_bar_sync(1, OZ_EPI);
      if (*sfail) {
        ok = false;
        break;
      }
#pragma unroll
      for (int k = 0; k < HS / 2; ++k) {
        const int sh = half * HS + own0 + k;
        const int r = t.ct * SH + sh;
        const double* pr = xb + (size_t)sh * 8 * OZ_TH + thl;
        double D[8], Qv[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const double sc = cs[4 * sh + (c & 3)];
          const double pv = pr[c * OZ_TH];
          D[c] = (tab == 0 ? own[k][c] : pv) * sc;
          Qv[c] = (tab == 0 ? pv : own[k][c]) * sc;
        }
        if (ith < d.nth && r < d.nr) {
          double2 vth[2], vph[2];
#pragma unroll
          for (int s = 0; s < 2; ++s) {
            const double* Ds = D + 4 * s;
            const double* Qs = Qv + 4 * s;
            // [0] S re, [1] S im, [2] T re, [3] T im
            vth[s] = make_double2(Ds[0] - Qs[3], Ds[1] + Qs[2]);
            vph[s] = make_double2(-Qs[1] - Ds[2], Qs[0] - Ds[3]);
            const size_t b0 = (((size_t)(0 * d.nr + r) * (d.M + 1) + t.m) * 2 + s) * d.nth + ith;
            const size_t b1 = (((size_t)(1 * d.nr + r) * (d.M + 1) + t.m) * 2 + s) * d.nth + ith;
            a.out[b0] = vth[s];
            a.out[b1] = vph[s];
          }
          if (a.out32 != nullptr) {
            const size_t off = (size_t)r * run32 + ((size_t)(ith / FBK) * (d.M + 1) + t.m) * FBK + ith % FBK;
            a.out32[off] = make_float4((float)vth[0].x, (float)vth[0].y, (float)vth[1].x, (float)vth[1].y);
            a.out32[a.out32_comp + off] =
                make_float4((float)vph[0].x, (float)vph[0].y, (float)vph[1].x, (float)vph[1].y);
          }
        }
      }
    }
  }
  ok = __syncthreads_and(ok);
  // after an expired wait anywhere in the CTA: the producer lets its last bulk
  // copies land and the MMA warp waits for the MMAs it has issued, before
  // tensor memory is freed and the CTA exits
  if (!ok && warp == 0)
    for (int g = max(0, issued - S + 1); g <= issued; ++g)  // every stage's last issued copies
      if (g != omitted) mbar_wait(&full[g % S], (g / S) & 1, a.err, a.wait_limit);
  if (!ok && warp == 1) {
    if (lane == 0) mma_commit(smem_addr(drain));
    __syncwarp();
    mbar_wait(drain, 0, a.err, a.wait_limit);
  }
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, NCOL);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
OzLayout oz_layout(const Dims& d, int digits) {
  OzLayout o{};
  o.digits = digits;
  o.ncols = digits == 5 ? 48 : 32;
  const int ntt = ceil_div(d.nth, OZ_TH), nks = oz_nksmax(d.L);
  o.ncb = ceil_div(4 * d.nr, o.ncols);
  o.a_bytes = (size_t)(d.M + 1) * ntt * 2 * nks * digits * OZ_A_SLICE;
  o.rs_elems = (size_t)(d.M + 1) * ntt * OZ_M;
  o.b_bytes = (size_t)(d.M + 1) * 2 * o.ncb * nks * digits * (size_t)o.ncols * OZ_KS;
  o.cs_elems = (size_t)(d.M + 1) * o.ncb * o.ncols;
  return o;
}

bool oz_supported(const Dims& d) {
  return d.nseg <= 1 && !d.ball && d.nth >= 1 && (size_t)sizeof(double) * 48 * (d.L + 1) <= (size_t)OZ_COEF_SMEM;
}

void launch_oz_tables(cudaStream_t s, const Dims& d, const int* moff, const double* dP, const double* Q,
                      const OzLayout& o, signed char* imgA, double* rsc) {
  const dim3 grid(ceil_div(d.nth, OZ_TH), d.M + 1, 2);
  if (o.digits == 5)
    k_oz_table_image<5><<<grid, OZ_M, 0, s>>>(d, moff, dP, Q, imgA, rsc);
  else
    k_oz_table_image<6><<<grid, OZ_M, 0, s>>>(d, moff, dP, Q, imgA, rsc);
}

template <int G, int N>
static void run_synth(cudaStream_t s, const Dims& d, const int* moff, const OzLayout& o, const double* S,
                      const double* T, const signed char* imgA, const double* rsc, signed char* imgB, double* csc,
                      const OzSynthArgs& a) {
  const size_t cbytes = sizeof(double) * N * (d.L + 1);
  // cached per device (and thread-safe) inside allow_dynamic_smem
  allow_dynamic_smem(k_oz_synth_vector<G, N>, OzSmem<G, N>::BYTES);
  allow_dynamic_smem(k_oz_coef_image<G, N>, OZ_COEF_SMEM);
  k_oz_coef_image<G, N><<<dim3(o.ncb, d.M + 1), OZ_CT, cbytes, s>>>(d, moff, S, T, imgB, csc, o.ncb);
  const int ntiles = (d.M + 1) * ceil_div(d.nth, OZ_TH) * o.ncb;
  const int ctas = std::min(ntiles, a.max_ctas > 0 ? std::min(a.max_ctas, current_sm_count()) : current_sm_count());
  k_oz_synth_vector<G, N><<<ctas, OZ_THREADS, OzSmem<G, N>::BYTES, s>>>(d, imgA, rsc, imgB, csc, o.ncb, a);
}

void launch_oz_synth_vector(cudaStream_t s, const Dims& d, const int* moff, const OzLayout& o, const double* S,
                            const double* T, const signed char* imgA, const double* rsc, signed char* imgB,
                            double* csc, const OzSynthArgs& a) {
  if (o.digits == 5)
    run_synth<5, 48>(s, d, moff, o, S, T, imgA, rsc, imgB, csc, a);
  else
    run_synth<6, 32>(s, d, moff, o, S, T, imgA, rsc, imgB, csc, a);
}

}  // namespace gd

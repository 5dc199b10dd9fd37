// gd_legendre_tc.cu -- mixed-precision Legendre synthesis and analysis on the
// 5th-generation tensor cores (tcgen05.mma kind::tf32, M = 128, N <= 256),
// FP32 accumulation in tensor memory.
//
// Each FP32/FP64 operand x is split into TF32 hi = rn(x) and lo = rn(x - hi);
// every tile product is hi*hi + hi*lo + lo*hi, which carries about 22 bits.
// The associated Legendre tables (Pbar, dPbar/dtheta, m Pbar / sin) are stored
// once as pre-split, pre-swizzled shared-memory images (K-major SWIZZLE_128B
// tiles of 128 rows x 32 TF32); the runtime operand (spectral coefficients for
// synthesis, folded phi transforms for analysis) is split by the loader
// threads while it is written to shared memory.
//
// Parity: for each order m the sum over l splits by the parity of l - m.
// Synthesis keeps the even and odd partial sums in separate tensor-memory
// column ranges and forms north = even + odd, south = even - odd (the
// theta-derivative table has the opposite symmetry).  Analysis multiplies the
// even rows by the fold w (G_N + G_S) and the odd rows by w (G_N - G_S).
//
// Arithmetic of SHTnsKit.synthesis / analysis / SHsphtor_to_spat /
// spat_to_SHsphtor as called per shell in src/shtnskit_field_functions.jl
// (:102-123, :218-239, :252-321); all shells and fields in one launch.
#include <algorithm>

#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"
#include "gd_tc.cuh"

namespace gd {

using namespace tc;

namespace {

constexpr int TC_M = 128;
constexpr int TC_N2 = 128;    // synthesis and scalar analysis column tile
constexpr int TC_K = 32;                       // TF32 elements per 128-byte row
constexpr int TILE_A_FLOATS = TC_M * TC_K;      // 4096 floats = 16 KB
constexpr int CHUNK_FLOATS = 2 * TILE_A_FLOATS; // hi image then lo image (32 KB)
// Pipelined kernels: every stage holds one (chunk, parity) step; stages sit
// back to back after a 1024-byte aligned base, then one mbarrier per stage
// and the TMEM address slot (192 KB + alignment slack per CTA).

__device__ __forceinline__ int kpar(int L, int m, int p) { return p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2; }
__device__ __host__ __forceinline__ int nck_h(int L, int m, int p) {
  const int k = p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2;
  return (k + TC_K - 1) / TC_K;
}

// Degree tiles of the analysis: 128 rows of one parity each, enough for the
// even parity of m = 0 (lmax <= 255 takes one).
__device__ __host__ __forceinline__ int nlt_of(int L) { return ((L + 2) / 2 + TC_M - 1) / TC_M; }
// Rows of parity p of order m that fall in degree tile lt.
__device__ __forceinline__ int krows(int L, int m, int p, int lt) {
  return max(0, min(TC_M, kpar(L, m, p) - TC_M * lt));
}

// chunk index of the synthesis image for (m, theta tile, parity, k chunk)
__device__ __forceinline__ long synth_chunk(const long* cofs, int L, int m, int tile, int p, int kc) {
  const int n0 = nck_h(L, m, 0), n1 = nck_h(L, m, 1);
  return cofs[m] + (long)tile * (n0 + n1) + (p == 0 ? kc : n0 + kc);
}

__device__ __forceinline__ void put_split_f(float* hi, float* lo, int row, int k, float x) {
  const float h = tf32_rn(x);
  const float l = tf32_rn(x - h);
  const uint32_t o = sw128_offset(row, k) >> 2;
  hi[o] = h;
  lo[o] = l;
}

// 3 TF32 products of one 32-deep chunk into tmem column offset dcol.
__device__ __forceinline__ void issue_chunk(uint32_t tmem, uint32_t dcol, const float* Ahi, const float* Alo,
                                            const float* Bhi, const float* Blo, bool first, uint32_t idesc) {
  const uint32_t ah = smem_addr(Ahi), al = smem_addr(Alo), bh = smem_addr(Bhi), bl = smem_addr(Blo);
#pragma unroll
  for (int ks = 0; ks < TC_K / 8; ++ks) {
    const uint32_t off = ks * 32;  // 8 TF32 = 32 bytes along K
    const uint64_t adh = sw128_desc(ah + off), adl = sw128_desc(al + off);
    const uint64_t bdh = sw128_desc(bh + off), bdl = sw128_desc(bl + off);
    mma_tf32(tmem + dcol, adh, bdh, idesc, (first && ks == 0) ? 0u : 1u);
    mma_tf32(tmem + dcol, adh, bdl, idesc, 1u);
    mma_tf32(tmem + dcol, adl, bdh, idesc, 1u);
  }
}


}  // namespace

// ---------------------------------------------------------------------------
// Table images.
// Synthesis chunk (m, tile, p, kc): row r -> ith = 128 tile + r,
//   k -> l = m + p + 2 (32 kc + k).
// Analysis chunk (m, p, lt, c): row i -> l = m + p + 2 (128 lt + i), k -> ith = 32 c + k.
// ---------------------------------------------------------------------------
__global__ void k_build_synth_image(Dims d, const int* __restrict__ moff, const long* __restrict__ cofs,
                                    const double* __restrict__ T, float* __restrict__ img) {
  const int m = blockIdx.z;
  const int n0 = nck_h(d.L, m, 0), n1 = nck_h(d.L, m, 1);
  const int ntile = (d.nth + TC_M - 1) / TC_M;
  const int local = blockIdx.y;  // (tile, p, kc) flattened
  if (local >= ntile * (n0 + n1)) return;
  const int tile = local / (n0 + n1), rem = local % (n0 + n1);
  const int p = rem < n0 ? 0 : 1, kc = rem < n0 ? rem : rem - n0;
  float* hi = img + (cofs[m] + local) * (long)CHUNK_FLOATS;
  float* lo = hi + TILE_A_FLOATS;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TC_M * TC_K; e += gridDim.x * blockDim.x) {
    const int row = e / TC_K, k = e % TC_K;
    const int ith = tile * TC_M + row;
    const int l = m + p + 2 * (TC_K * kc + k);
    double v = 0.0;
    if (ith < d.nth && l <= d.L) v = T[(size_t)(moff[m] + l - m) * d.nth + ith];
    const float h = tf32_rn((float)v);
    const float lw = tf32_rn((float)(v - (double)h));
    const uint32_t o = sw128_offset(row, k) >> 2;
    hi[o] = h;
    lo[o] = lw;
  }
}

__global__ void k_build_analysis_image(Dims d, const int* __restrict__ moff, const double* __restrict__ T,
                                       float* __restrict__ img) {
  const int m = blockIdx.z;
  const int nthc = (d.nth + TC_K - 1) / TC_K, nlt = nlt_of(d.L);
  const int p = blockIdx.y / (nlt * nthc), lt = (blockIdx.y / nthc) % nlt, c = blockIdx.y % nthc;
  float* hi = img + (((long)(m * 2 + p) * nlt + lt) * nthc + c) * CHUNK_FLOATS;
  float* lo = hi + TILE_A_FLOATS;
  const int kp = krows(d.L, m, p, lt);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TC_M * TC_K; e += gridDim.x * blockDim.x) {
    const int row = e / TC_K, k = e % TC_K;
    const int ith = TC_K * c + k;
    const int l = m + p + 2 * (TC_M * lt + row);
    double v = 0.0;
    if (row < kp && ith < d.nth && l <= d.L) v = T[(size_t)(moff[m] + l - m) * d.nth + ith];
    const float h = tf32_rn((float)v);
    const float lw = tf32_rn((float)(v - (double)h));
    const uint32_t o = sw128_offset(row, k) >> 2;
    hi[o] = h;
    lo[o] = lw;
  }
}

long tc_synth_chunks(const Dims& d, std::vector<long>& cofs) {
  const int ntile = (d.nth + TC_M - 1) / TC_M;
  cofs.assign(d.M + 2, 0);
  for (int m = 0; m <= d.M; ++m) cofs[m + 1] = cofs[m] + (long)ntile * (nck_h(d.L, m, 0) + nck_h(d.L, m, 1));
  return cofs[d.M + 1];
}
long tc_analysis_chunks(const Dims& d) {
  return (long)(d.M + 1) * 2 * nlt_of(d.L) * ((d.nth + TC_K - 1) / TC_K);
}
size_t tc_chunk_bytes() { return (size_t)CHUNK_FLOATS * 4; }

void launch_build_tc_images(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const double* T,
                            float* synth_img, float* anal_img) {
  if (synth_img) {
    const int ntile = (d.nth + TC_M - 1) / TC_M;
    const int maxloc = ntile * (nck_h(d.L, 0, 0) + nck_h(d.L, 0, 1));
    k_build_synth_image<<<dim3(8, maxloc, d.M + 1), 256, 0, s>>>(d, moff, cofs, T, synth_img);
  }
  if (anal_img) {
    const int nthc = (d.nth + TC_K - 1) / TC_K;
    k_build_analysis_image<<<dim3(8, 2 * nlt_of(d.L) * nthc, d.M + 1), 256, 0, s>>>(d, moff, T, anal_img);
  }
}

// ---------------------------------------------------------------------------
// Synthesis, two kernels.
//
// 1. k_synth_coef_image: the runtime coefficients of one call as split,
//    swizzled TF32 B-operand chunks: chunk (column tile ct, m, step it) =
//    hi then lo image of NCS columns x 32 K (scalar NCS = 256 columns
//    n = (field, r, re/im); vector NCS = 128: 32 shells x [S re, S im, T re,
//    T im]; the valid columns of a tile are a prefix),
//    K -> l = m + p + 2 (32 kc + k).  One CTA per (kc, m, ct) covers both
//    parities, so each warp reads l-contiguous runs of every coefficient row.
// 2. k_tc_synth4: persistent CTAs over tiles (m, 128-row theta tile, column
//    tile), 320 threads: warp 0 feeds the two pipeline stages with bulk copies
//    only (table chunk(s) and the coefficient chunk, transaction bytes on the
//    stage's `full` barrier), warp 1 issues the split-TF32 MMAs (3 products
//    per 8-deep K slice) and commits them to the stage's `empty` barrier and,
//    after a tile's last step, to `tfull`; warps 2-9 (two per TMEM lane
//    quarter, alternate 8-column chunks) wait on `tfull`, read the
//    accumulators, release them on `tempty` and write the blocked Fourier
//    layout while the next tile's stages are already loading.  Scalar: accumulators [even | odd] x 256.
//    Vector: [P even | P odd | dP even | dP odd] x 128; the m/sin(theta) of
//    the Q = m Pbar / sin(theta) terms is applied to the Pbar sums.  Rows past
//    the last colatitude and columns past the last shell are neither copied
//    nor (columns) multiplied: the MMA width follows the tile's valid columns.
// ---------------------------------------------------------------------------
constexpr int SY_THREADS = 320;  // producer, MMA issuer, 8 epilogue warps (two per TMEM lane quarter)
constexpr int SY_EPI = SY_THREADS - 64;

// step it -> (parity p, K chunk kc): odd-parity chunks interleave with the
// even ones while both exist
__device__ __forceinline__ void synth_step_pk(int it, int nc1, int& p, int& kc) {
  kc = it < 2 * nc1 ? (it >> 1) : nc1 + (it - 2 * nc1);
  p = it < 2 * nc1 ? (it & 1) : 0;
}
__device__ __forceinline__ int synth_step_of(int p, int kc, int nc1) { return kc < nc1 ? 2 * kc + p : nc1 + kc; }

template <bool VEC>
__global__ void __launch_bounds__(256) k_synth_coef_image(Dims d, const int* __restrict__ moff,
                                                          const long* __restrict__ cofs, int ntt, TcSynthArgs a) {
  constexpr int NCS = VEC ? TC_N2 : 2 * TC_N2;
  constexpr int BT = NCS * TC_K;
  __shared__ const double* colp[NCS];
  __shared__ unsigned char mine[NCS];  // column belongs to a field of prep_mask
  const int kc = blockIdx.x, m = blockIdx.y, ct = blockIdx.z;
  const int L = d.L;
  const int nc0 = nck_h(L, m, 0), nc1 = nck_h(L, m, 1);
  if (kc >= nc0) return;
  const size_t NM = d.nlm;
  const int mb = moff[m];
  const int Ntot = a.nf * d.nr * 2;
  for (int c = threadIdx.x; c < NCS; c += blockDim.x) {
    const double* src = nullptr;
    bool own = true;
    if (VEC) {
      const int fld = (c >> 1) & 1, r = ct * 32 + (c >> 2), ci = c & 1;
      own = (a.prep_mask >> fld) & 1;
      if (r < d.nr) src = a.coef[fld] + ((size_t)ci * d.nr + r) * NM + mb - m;
    } else {
      const int ng = ct * NCS + c;
      if (ng < Ntot) {
        const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, ci = rem & 1;
        own = (a.prep_mask >> f) & 1;
        src = a.coef[f] + ((size_t)ci * d.nr + r) * NM + mb - m;
      }
    }
    colp[c] = own ? src : nullptr;
    mine[c] = own ? 1 : 0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long base = (long)ct * a.ttot + cofs[m] / ntt;
  float* h0 = a.bimg + (base + synth_step_of(0, kc, nc1)) * (2L * BT);
  float* h1 = kc < nc1 ? a.bimg + (base + synth_step_of(1, kc, nc1)) * (2L * BT) : nullptr;
  const int l0 = m + 2 * (TC_K * kc + lane);
  // rows in batches of four per warp, every load of a batch issued before its stores
  constexpr int RB = 4;
  for (int row0 = warp; row0 < NCS; row0 += 8 * RB) {
    double v0[RB], v1[RB];
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int row = row0 + 8 * u;
      const double* src = row < NCS ? colp[row] : nullptr;
      v0[u] = (src != nullptr && l0 <= L) ? src[l0] : 0.0;
      v1[u] = (src != nullptr && l0 + 1 <= L) ? src[l0 + 1] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int row = row0 + 8 * u;
      // rows of other fields are written by their producer kernels
      if (row < NCS && mine[row]) {
        const uint32_t o = sw128_offset(row, lane) >> 2;
        const float f0 = __double2float_rn(v0[u]), g0 = tf32_rn(f0);
        h0[o] = g0;
        h0[BT + o] = tf32_rn(f0 - g0);
        if (h1 != nullptr) {
          const float f1 = __double2float_rn(v1[u]), g1 = tf32_rn(f1);
          h1[o] = g1;
          h1[BT + o] = tf32_rn(f1 - g1);
        }
      }
    }
  }
}

template <bool VEC>
__global__ void __launch_bounds__(SY_THREADS, 1) k_tc_synth4(Dims d, const int* __restrict__ moff,
                                                             const long* __restrict__ cofs,
                                                             const float* __restrict__ imgP,
                                                             const float* __restrict__ imgD,
                                                             const double* __restrict__ sinv, TcSynthArgs a, int ntt,
                                                             int ncol) {
  constexpr int S = 2;
  constexpr int NCS = VEC ? TC_N2 : 2 * TC_N2;   // columns per tile: vector 128, scalar 256
  constexpr int A_FL = (VEC ? 2 : 1) * CHUNK_FLOATS;
  constexpr int BT = NCS * TC_K;                  // one B image (hi or lo)
  constexpr int ST_FL = A_FL + 2 * BT;
  constexpr uint32_t NCOL = 512;
  extern __shared__ unsigned char smem_raw[];
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  float* stg = reinterpret_cast<float*>(base);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)S * ST_FL * 4);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;
  uint64_t* tempty = tfull + 1;
  uint64_t* drain = tempty + 1;  // after a failed wait: completion of the MMAs already issued
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);

  const int L = d.L;
  const int Ntot = a.nf * d.nr * 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, SY_EPI);
    mbar_init(drain, 1);
  }
  if (warp == 0) tmem_alloc(tslot, NCOL);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const int ntiles = (d.M + 1) * ntt * ncol;
  bool ok = true;
  int issued = -1;  // producer: last pipeline step whose bulk copies were issued

  if (warp == 0) {
    // producer: bulk copies only.  Step (tile tt, it): table chunk(s) and the
    // coefficient chunk; table rows past the last colatitude and coefficient
    // columns past the last valid one only reach accumulator rows / columns
    // the epilogue never reads, so whole 8-row swizzle atoms of the rest are
    // copied.
    auto step_src = [&](int tt, int it, const float*& s0, const float*& s1, const float*& sb, uint32_t& pa,
                        uint32_t& pb) {
      const int m = tt / (ntt * ncol), tile = (tt / ncol) % ntt, ct = tt % ncol;
      const int nc1 = nck_h(L, m, 1);
      int p, kc;
      synth_step_pk(it, nc1, p, kc);
      const long ch = synth_chunk(cofs, L, m, tile, p, kc);
      const long bch = (long)ct * a.ttot + cofs[m] / ntt + it;
      pa = (uint32_t)min(TC_M, (d.nth - tile * TC_M + 7) & ~7) * 128u;
      const int nvalid = VEC ? 4 * min(32, d.nr - ct * 32) : min(NCS, Ntot - ct * NCS);
      pb = (uint32_t)((nvalid + 7) & ~7) * 128u;
      s0 = imgP + ch * CHUNK_FLOATS;
      s1 = imgD + ch * CHUNK_FLOATS;
      sb = a.bimg + bch * (2L * BT);
    };
    int gs = 0;
    for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x) {
      const int m = tt / (ntt * ncol);
      const int nc1 = nck_h(L, m, 1), T = nck_h(L, m, 0) + nc1;
      for (int it = 0; it < T; ++it) {
        const int G = gs + it, s = G & 1, u = G >> 1;
        if (u >= 1 && !mbar_wait(&empty[s], (u - 1) & 1, a.err, a.wait_limit)) {
          ok = false;
          break;
        }
        // error-path tests: CTA 0 may omit one step's copies, so the MMA
        // warp's bounded wait on that stage runs out
        const bool omit = a.omit_plus1 == G + 1 && blockIdx.x == 0;
        if (lane == 0 && !omit) {
          float* A = stg + s * ST_FL;
          const float *s0, *s1, *sb;
          uint32_t pa, pb;
          step_src(tt, it, s0, s1, sb, pa, pb);
          mbar_arrive_expect_tx(&full[s], (VEC ? 4u : 2u) * pa + 2u * pb);
          bulk_g2s(A, s0, pa, &full[s]);
          bulk_g2s(A + TILE_A_FLOATS, s0 + TILE_A_FLOATS, pa, &full[s]);
          if (VEC) {
            bulk_g2s(A + CHUNK_FLOATS, s1, pa, &full[s]);
            bulk_g2s(A + CHUNK_FLOATS + TILE_A_FLOATS, s1 + TILE_A_FLOATS, pa, &full[s]);
          }
          bulk_g2s(A + A_FL, sb, pb, &full[s]);
          bulk_g2s(A + A_FL + BT, sb + BT, pb, &full[s]);
        }
        if (!omit) issued = G;
        __syncwarp();
      }
      gs += T;
    }
  } else if (warp == 1) {
    // MMA issuer
    int gs = 0, q = 0;
    for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x, ++q) {
      const int m = tt / (ntt * ncol), ct = tt % ncol;
      const int nc1 = nck_h(L, m, 1), T = nck_h(L, m, 0) + nc1;
      const int nvalid = VEC ? 4 * min(32, d.nr - ct * 32) : min(NCS, Ntot - ct * NCS);
      const uint32_t ids = idesc_tf32(TC_M, (nvalid + 15) & ~15);
      if (q >= 1 && !mbar_wait(tempty, (q - 1) & 1, a.err, a.wait_limit)) {
        ok = false;
        break;
      }
      for (int it = 0; it < T; ++it) {
        const int G = gs + it, s = G & 1;
        if (!mbar_wait(&full[s], (G >> 1) & 1, a.err, a.wait_limit)) {
          ok = false;
          break;
        }
        fence_after_sync();
        if (lane == 0) {
          int p, kc;
          synth_step_pk(it, nc1, p, kc);
          const float* A = stg + s * ST_FL;
          const float* B = A + A_FL;
#pragma unroll
          for (int t = 0; t < (VEC ? 2 : 1); ++t)
            issue_chunk(tmem, (t * 2 + p) * NCS, A + t * CHUNK_FLOATS, A + t * CHUNK_FLOATS + TILE_A_FLOATS, B,
                        B + BT, kc == 0, ids);
          mma_commit(smem_addr(&empty[s]));
          if (it == T - 1) mma_commit(smem_addr(tfull));
        }
        __syncwarp();
      }
      gs += T;
    }
  } else {
    // epilogue warps 2-9: TMEM lane quarter warp & 3; the two warps of a
    // quarter take alternate 8-column chunks
    const int qw = warp & 3, half = (warp - 2) >> 2;
    // scalar columns n = (f nr + r) 2 + re/im: the pair n / 2 = f nr + r indexes the (comp, r) run
    const size_t run = (size_t)a.nblk * (d.M + 1) * FOURIER_BLOCK;
    const uint32_t trow = tmem + ((uint32_t)(qw * 32) << 16);
    int q = 0;
    for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x, ++q) {
      const int m = tt / (ntt * ncol), tile = (tt / ncol) % ntt, ct = tt % ncol;
      const int nc1 = nck_h(L, m, 1);
      if (!mbar_wait(tfull, q & 1, a.err, a.wait_limit)) {
        ok = false;
        break;
      }
      fence_after_sync();
      const int ith = tile * TC_M + qw * 32 + lane;
      // offset of (theta block, m, pair) within one (comp, r) run of the blocked layout
      const size_t ioff = ((size_t)(ith / FOURIER_BLOCK) * (d.M + 1) + m) * FOURIER_BLOCK + ith % FOURIER_BLOCK;
      const int nvalid = VEC ? 4 * min(32, d.nr - ct * 32) : min(NCS, Ntot - ct * NCS);
      const int cend = (nvalid + 7) & ~7;  // accumulator columns holding valid results
      // this warp's last chunk: after its loads the warp releases the accumulators
      const int nch = cend / 8, mine = nch > half ? (nch - 1 - half) / 2 + 1 : 0;
      const int clast = mine > 0 ? 8 * (half + 2 * (mine - 1)) : -1;
      if (clast < 0) {
        fence_before_sync();
        mbar_arrive(tempty);
      }
      if (!VEC) {
        for (int c0 = 8 * half; c0 < cend; c0 += 16) {
          float e[8], o[8];
          tmem_ld8(trow + c0, e);
          if (nc1 > 0) tmem_ld8(trow + NCS + c0, o);
          tmem_ld_wait();
          if (nc1 == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) o[j] = 0.f;
          }
          if (c0 == clast) {
            fence_before_sync();
            mbar_arrive(tempty);  // accumulators read: the next tile's MMAs may start
          }
          if (ith < d.nth) {
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
              const int ng = ct * NCS + c0 + j;
              if (ng >= Ntot) continue;
              a.out[(size_t)(ng >> 1) * run + ioff] =
                  make_float4(e[j] + o[j], e[j + 1] + o[j + 1], e[j] - o[j], e[j + 1] - o[j + 1]);
            }
          }
        }
      } else {
        // columns (shell, component, re/im): 8 columns = 2 shells x [S re, S im, T re, T im]
        const int r0 = ct * 32;
        const float ms = (ith < d.nth) ? (float)((double)m * sinv[ith]) : 0.f;
        for (int c0 = 8 * half; c0 < cend; c0 += 16) {
          float pe[8], po[8], de[8], dq[8];
          tmem_ld8(trow + 0 * TC_N2 + c0, pe);
          tmem_ld8(trow + 2 * TC_N2 + c0, de);
          if (nc1 > 0) {
            tmem_ld8(trow + 1 * TC_N2 + c0, po);
            tmem_ld8(trow + 3 * TC_N2 + c0, dq);
          }
          tmem_ld_wait();
          if (nc1 == 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) po[j] = dq[j] = 0.f;
          }
          if (c0 == clast) {
            fence_before_sync();
            mbar_arrive(tempty);
          }
          if (ith < d.nth) {
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
              const int r = r0 + c0 / 4 + s2;
              if (r >= d.nr) continue;
              const int b = 4 * s2;
              float vt[4], vp[4];  // (north Re, north Im, south Re, south Im)
#pragma unroll
              for (int sN = 0; sN < 2; ++sN) {
                float PS[2], PT[2], DS[2], DT[2];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                  if (sN == 0) {
                    PS[c] = pe[b + c] + po[b + c]; PT[c] = pe[b + 2 + c] + po[b + 2 + c];
                    DS[c] = de[b + c] + dq[b + c]; DT[c] = de[b + 2 + c] + dq[b + 2 + c];
                  } else {  // dPbar has the opposite north/south symmetry
                    PS[c] = pe[b + c] - po[b + c]; PT[c] = pe[b + 2 + c] - po[b + 2 + c];
                    DS[c] = dq[b + c] - de[b + c]; DT[c] = dq[b + 2 + c] - de[b + 2 + c];
                  }
                }
                const float QS0 = ms * PS[0], QS1 = ms * PS[1], QT0 = ms * PT[0], QT1 = ms * PT[1];
                vt[2 * sN] = DS[0] - QT1; vt[2 * sN + 1] = DS[1] + QT0;
                vp[2 * sN] = -QS1 - DT[0]; vp[2 * sN + 1] = QS0 - DT[1];
              }
              a.out[(size_t)(0 * d.nr + r) * run + ioff] = make_float4(vt[0], vt[1], vt[2], vt[3]);
              a.out[(size_t)(1 * d.nr + r) * run + ioff] = make_float4(vp[0], vp[1], vp[2], vp[3]);
            }
          }
        }
      }
    }
  }
  ok = __syncthreads_and(ok);
  // after an expired wait anywhere in the CTA: the producer lets its last bulk
  // copies land (a step the MMA warp consumed has completed its phase
  // already, so this returns at once), and the MMA warp waits for the MMAs it
  // has issued, before tensor memory is freed and the CTA exits
  if (!ok && warp == 0 && issued >= 0) mbar_wait(&full[issued & 1], (issued >> 1) & 1, a.err, a.wait_limit);
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
// Analysis.  CTA = (m, degree tile, column tile); K = colatitude in chunks of 32; two
// loader groups of 4 warps (group g fills stage g: bulk copies of the table
// chunks, FP32 inputs split to TF32 hi/lo while written) and one MMA warp.
// Scalar: 128 columns n = (field, r, re/im), one step per (theta chunk,
// parity), stages of 64 KB, accumulators [even | odd] x 128.
// Vector: 128 columns, 32 shells x [G_theta re, im, G_phi re, im]; one step
// per (theta chunk, fold f): the B tile holds fold f once and meets both the
// dPbar chunk of parity 1 - f and the Q chunk of parity f, so every input
// element is loaded once per tile; stages of 96 KB, accumulators
// [dP even | dP odd | Q even | Q odd] x 128.  Columns past the last shell or
// field are not loaded and the MMA width follows the tile's valid columns.
// ---------------------------------------------------------------------------
constexpr int WS_THREADS = 288;  // 2 loader groups x 4 warps + 1 MMA warp

// MMA width of a tile with `nval` valid columns (M = 128 takes N % 16 == 0)
__device__ __forceinline__ int tile_width(int nval) { return (nval + 15) & ~15; }

template <bool VEC>
__global__ void __launch_bounds__(WS_THREADS, 1) k_tc_analysis3(Dims d, const int* __restrict__ moff,
                                                         const float* __restrict__ img0,
                                                         const float* __restrict__ img1, TcAnalysisArgs a,
                                                         int ncol, int csz) {
  constexpr int S = 2;
  constexpr int NC = TC_N2;                      // columns
  constexpr int A_FL = (VEC ? 2 : 1) * CHUNK_FLOATS;
  constexpr int BT = NC * TC_K;                  // one B image (hi or lo)
  constexpr int B_FL = 2 * BT;
  constexpr int ST_FL = A_FL + B_FL;
  constexpr uint32_t NCOL = VEC ? 512 : 256;
  extern __shared__ unsigned char smem_raw[];
  const uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  float* stg = reinterpret_cast<float*>(base);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)S * ST_FL * 4);
  uint64_t* empty = full + S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(empty + S);
  uint64_t* drain = empty + S + 1;  // after a failed wait: completion of the MMAs already issued
  // scalar: column pair -> folded-input base (-1 past the last column);
  // column -> output row (null past the last column)
  long long* colin = reinterpret_cast<long long*>(empty + S + 2);
  double** colout = reinterpret_cast<double**>(colin + NC / 2);

  const int L = d.L;
  const size_t NM = d.nlm;
  const int Ntot = a.nf * d.nr * 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 128);
      mbar_init(&empty[s], 1);
    }
    mbar_init(drain, 1);
  }
  if (warp == 0) tmem_alloc(tslot, NCOL);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const int nthc = (d.nth + TC_K - 1) / TC_K;

  bool ok = true;
  int issued = -1;  // loader thread 0 of a group: last use of its stage with bulk copies issued
  int gs = 0;       // pipeline steps of the earlier tiles
  const int nlt = nlt_of(L);
  const int ntiles = (d.M + 1) * nlt * ncol;
  // persistent CTA: tiles (m, degree tile, column tile), m-major; a degree
  // tile past both parities' last degree of its order has no work
  for (int tt = blockIdx.x; tt < ntiles && ok; tt += gridDim.x) {
  const int m = tt / (nlt * ncol), lt = (tt / ncol) % nlt, ct = tt % ncol;
  if (krows(L, m, 0, lt) == 0) continue;
  const int mb = moff[m];
  // balanced column tiles: vector csz shells, scalar csz column pairs
  const int n0 = ct * 2 * csz;
  const int nval = VEC ? 4 * min(csz, d.nr - ct * csz) : min(2 * csz, Ntot - n0);
  const int r0 = ct * csz;
  const int nw = tile_width(nval);
  const uint32_t idesc = idesc_tf32(TC_M, nw);
  __syncthreads();  // the previous tile's epilogue is done with TMEM and the column tables
  if (!VEC) {
    for (int c = tid; c < NC; c += blockDim.x) {
      const int ng = n0 + c;
      double* dst = nullptr;
      if (c < nval) {
        const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, ci = rem & 1;
        dst = a.out[f] + ((size_t)ci * d.nr + r) * NM + mb - m;
      }
      colout[c] = dst;
      if ((c & 1) == 0) {
        const int pg = ng >> 1;
        long long ib = -1;
        if (c < nval) {
          const int f = pg / d.nr, r = pg % d.nr;
          ib = (long long)((((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2) * d.nth);
        }
        colin[c >> 1] = ib;
      }
    }
    __syncthreads();
  }

  const int k1 = krows(L, m, 1, lt);
  const int np = k1 > 0 ? 2 : 1;
  // scalar: steps (chunk, parity); vector: steps (chunk, fold), both folds
  // always (with k1 = 0 no odd-parity rows are copied or read)
  const int ns = VEC ? 2 : np;
  const int T = nthc * ns;

  if (warp < 8) {
    const int g = warp >> 2, gw = warp & 3, gt = tid & 127;
    float* A = stg + g * ST_FL;
    float* B = A + A_FL;
    // one float2 (re, im column pair) per item; NC / 2 pairs over 4 warps.
    // The inputs of a group's next step are loaded into registers while the
    // MMA still reads the stage.
    constexpr int NV = NC / 8;
    float2 v[NV];
    auto load_step = [&](int it) {
      const int cc = it / ns, p = it % ns;  // vector: p is the fold
      const int ith = TC_K * cc + lane;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const int pr = gw + 4 * i;
        v[i] = make_float2(0.f, 0.f);
        if (2 * pr >= nw || ith >= d.nth) continue;
        if (!VEC) {
          const long long ib = colin[pr];
          if (ib >= 0) v[i] = __ldg(&a.in[(size_t)ib + (size_t)p * d.nth + ith]);
        } else {
          const int r = r0 + (pr >> 1), comp = pr & 1;
          if (r < r0 + csz && r < d.nr)
            v[i] = __ldg(&a.in[(((size_t)(comp * d.nr + r) * (d.M + 1) + m) * 2 + p) * d.nth + ith]);
        }
      }
    };
    int it = (g - gs) & 1;
    if (it < T) load_step(it);
    for (; it < T; it += 2) {
      const int u = (gs + it) >> 1;
      if (u >= 1 && !mbar_wait(&empty[g], (u - 1) & 1, a.err, a.wait_limit)) {
        ok = false;
        break;
      }
      const int cc = it / ns, p = it % ns;
      if (gt == 0) {
        // table rows past the parity's last degree only reach accumulator
        // rows the epilogue never reads: copy whole 8-row swizzle atoms of
        // the valid ones (hi and lo images separately)
        const int pa0 = VEC ? 1 - p : p, pa1 = p;  // parity of the first / second table chunk
        const uint32_t ra0 = (uint32_t)((krows(L, m, pa0, lt) + 7) & ~7) * 128u;
        const uint32_t ra1 = VEC ? (uint32_t)((krows(L, m, pa1, lt) + 7) & ~7) * 128u : 0u;
        mbar_expect_tx(&full[g], 2u * (ra0 + ra1));
        const float* s0 = img0 + (((long)(m * 2 + pa0) * nlt + lt) * nthc + cc) * CHUNK_FLOATS;
        if (ra0 > 0) {
          bulk_g2s(A, s0, ra0, &full[g]);
          bulk_g2s(A + TILE_A_FLOATS, s0 + TILE_A_FLOATS, ra0, &full[g]);
        }
        if (VEC && ra1 > 0) {
          const float* s1 = img1 + (((long)(m * 2 + pa1) * nlt + lt) * nthc + cc) * CHUNK_FLOATS;
          bulk_g2s(A + CHUNK_FLOATS, s1, ra1, &full[g]);
          bulk_g2s(A + CHUNK_FLOATS + TILE_A_FLOATS, s1 + TILE_A_FLOATS, ra1, &full[g]);
        }
        issued = u;
      }
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        const int pr = gw + 4 * i;
        if (2 * pr >= nw) continue;
        put_split_f(B, B + BT, 2 * pr, lane, v[i].x);
        put_split_f(B, B + BT, 2 * pr + 1, lane, v[i].y);
      }
      fence_proxy_async();
      mbar_arrive(&full[g]);
      if (it + 2 < T) load_step(it + 2);
    }
  } else {
    for (int it = 0; it < T; ++it) {
      const int s = (gs + it) & 1;
      if (!mbar_wait(&full[s], ((gs + it) >> 1) & 1, a.err, a.wait_limit)) {
        ok = false;
        break;
      }
      fence_after_sync();
      if (lane == 0) {
        const int cc = it / ns, p = it % ns;
        const float* A = stg + s * ST_FL;
        const float* B = A + A_FL;
        if (!VEC) {
          issue_chunk(tmem, p * NC, A, A + TILE_A_FLOATS, B, B + BT, cc == 0, idesc);
        } else {  // fold p: dPbar rows of parity 1 - p, Q rows of parity p
          issue_chunk(tmem, (0 * 2 + 1 - p) * NC, A, A + TILE_A_FLOATS, B, B + BT, cc == 0, idesc);
          issue_chunk(tmem, (1 * 2 + p) * NC, A + CHUNK_FLOATS, A + CHUNK_FLOATS + TILE_A_FLOATS, B, B + BT,
                      cc == 0, idesc);
        }
        mma_commit(smem_addr(&empty[s]));
      }
      __syncwarp();
    }
  }
  // drain: the last MMA batch of each stage in this tile
  if (ok) {
#pragma unroll
    for (int q = 1; q <= S; ++q)
      if (T - q >= 0) ok = mbar_wait(&empty[(gs + T - q) & 1], ((gs + T - q) >> 1) & 1, a.err, a.wait_limit) && ok;
  }
  ok = __syncthreads_and(ok);
  fence_after_sync();
  if (ok && warp < 8) {
    const int q = warp & 3, half = warp >> 2;
    const int i = q * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
    for (int p = 0; p < np; ++p) {
      const int kp = krows(L, m, p, lt);
      const int l = m + p + 2 * (TC_M * lt + i);
      if (!VEC) {
        for (int c0 = (NC / 2) * half; c0 < (NC / 2) * half + NC / 2 && c0 < nw; c0 += 8) {
          float v[8];
          tmem_ld8(trow + p * NC + c0, v);
          tmem_ld_wait();
          if (i < kp) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              double* dst = colout[c0 + j];
              if (dst == nullptr) continue;
              // columns alternate (Re, Im); Im of m = 0 is stored as 0
              const double val = (((c0 + j) & 1) == 1 && m == 0) ? 0.0 : (double)v[j];
              dst[l] = val;
            }
          }
        }
      } else {
        const double fl = (l == 0) ? 0.0 : 1.0 / ((double)l * (l + 1.0));
        const double lf = (double)l * (l + 1.0);
        // 8 columns = 2 shells x [G_theta re, im, G_phi re, im]
        for (int c0 = (NC / 2) * half; c0 < (NC / 2) * half + NC / 2 && c0 < nw; c0 += 8) {
          float dp[8], q[8];
          tmem_ld8(trow + (0 * 2 + p) * NC + c0, dp);
          tmem_ld8(trow + (1 * 2 + p) * NC + c0, q);
          tmem_ld_wait();
          if (i >= kp) continue;
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            const int r = r0 + c0 / 4 + s2;
            if (4 * (r - r0) >= nval) continue;
            const int b = 4 * s2;
            const double Sre = ((double)dp[b] + (double)q[b + 3]) * fl;
            const double Sim = ((double)dp[b + 1] - (double)q[b + 2]) * fl;
            const double Tre = ((double)q[b + 1] - (double)dp[b + 2]) * fl;
            const double Tim = (-(double)q[b] - (double)dp[b + 3]) * fl;
            double o0re, o0im, o1re, o1im;
            if (a.epi == EPI_CURL_INDUCTION) {
              o0re = lf * Sre; o0im = lf * ((m == 0) ? 0.0 : Sim);
              o1re = -lf * Tre; o1im = -lf * ((m == 0) ? 0.0 : Tim);
            } else {
              o0re = Tre; o0im = (m == 0) ? 0.0 : Tim;
              o1re = Sre; o1im = (m == 0) ? 0.0 : Sim;
            }
            const size_t at = (size_t)r * NM + mb + (l - m);
            const size_t plane = (size_t)d.nr * NM;
            a.out[0][at] = o0re; a.out[0][plane + at] = o0im;
            a.out[1][at] = o1re; a.out[1][plane + at] = o1im;
          }
        }
      }
    }
  }
  fence_before_sync();
  gs += T;
  }  // tiles
  if (!ok && issued >= 0) mbar_wait(&full[(threadIdx.x >> 7) & 1], issued & 1, a.err, a.wait_limit);
  if (!ok && warp == 8) {
    // the MMAs issued before the failure finish before tensor memory is freed
    if (lane == 0) mma_commit(smem_addr(drain));
    __syncwarp();
    mbar_wait(drain, 0, a.err, a.wait_limit);
  }
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, NCOL);
}

// ---------------------------------------------------------------------------
// Synthesis: stages + full/empty per stage, tfull, tempty, drain and the TMEM
// address slot.  Analysis: stages + full/empty per stage, drain, the TMEM
// address slot and the scalar kernels' per-column tables (one pointer per
// column, one offset per pair).
static size_t synth_smem(bool vec) {
  const int S = 2, NCS = vec ? TC_N2 : 2 * TC_N2, A = (vec ? 2 : 1) * CHUNK_FLOATS, B = 2 * NCS * TC_K;
  return 1024 + (size_t)S * (A + B) * 4 + 8 * (2 * S + 4);
}
static size_t analysis_smem(bool vec) {
  const int S = 2, NC = TC_N2, A = (vec ? 2 : 1) * CHUNK_FLOATS;
  const int B = 2 * NC * TC_K;
  return 1024 + (size_t)S * (A + B) * 4 + 8 * (2 * S + 2) + (size_t)NC * 8 + (size_t)(NC / 2) * 8;
}
static void set_attrs() {
  allow_dynamic_smem(k_tc_synth4<false>, synth_smem(false));
  allow_dynamic_smem(k_tc_synth4<true>, synth_smem(true));
  allow_dynamic_smem(k_tc_analysis3<false>, analysis_smem(false));
  allow_dynamic_smem(k_tc_analysis3<true>, analysis_smem(true));
}

// One persistent CTA per SM (at most one tile each when there are fewer
// tiles), or fewer when the caller caps the grid: members of an ensemble then
// share the SMs instead of each filling them in turn.
static int sm_count() { return current_sm_count(); }
static int cta_cap(int max_ctas) { return max_ctas > 0 ? std::min(max_ctas, sm_count()) : sm_count(); }

void launch_tc_synth(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const float* imgP,
                     const float* imgD, const double* sinv, const TcSynthArgs& a, bool vec) {
  set_attrs();
  const int ntt = (d.nth + TC_M - 1) / TC_M;
  const int kcmax = nck_h(d.L, 0, 0);
  if (!vec) {
    const int ncol = ceil_div(a.nf * d.nr * 2, 2 * TC_N2);
    const int ntiles = (d.M + 1) * ntt * ncol;
    if (a.prep_mask) k_synth_coef_image<false><<<dim3(kcmax, d.M + 1, ncol), 256, 0, s>>>(d, moff, cofs, ntt, a);
    k_tc_synth4<false><<<std::min(ntiles, cta_cap(a.max_ctas)), SY_THREADS, synth_smem(false), s>>>(d, moff, cofs, imgP,
                                                                                          imgD, sinv, a, ntt, ncol);
  } else {
    const int ncol = ceil_div(d.nr, 32);
    const int ntiles = (d.M + 1) * ntt * ncol;
    if (a.prep_mask) k_synth_coef_image<true><<<dim3(kcmax, d.M + 1, ncol), 256, 0, s>>>(d, moff, cofs, ntt, a);
    k_tc_synth4<true><<<std::min(ntiles, cta_cap(a.max_ctas)), SY_THREADS, synth_smem(true), s>>>(d, moff, cofs, imgP, imgD,
                                                                                        sinv, a, ntt, ncol);
  }
}

size_t tc_synth_bimage_floats(const Dims& d, long ttot) {
  const long ncol_s = ceil_div(4L * d.nr * 2, 2 * TC_N2), ncol_v = ceil_div(d.nr, 32);
  const long s = ncol_s * ttot * 2L * (2 * TC_N2) * TC_K, v = ncol_v * ttot * 2L * TC_N2 * TC_K;
  return (size_t)(s > v ? s : v);
}

void launch_tc_analysis(cudaStream_t s, const Dims& d, const int* moff, const float* img0, const float* img1,
                        const TcAnalysisArgs& a) {
  set_attrs();
  if (a.epi == EPI_SCALAR) {
    const int npair = a.nf * d.nr, ncol = ceil_div(2 * npair, TC_N2), csz = ceil_div(npair, ncol);
    const int ntiles = (d.M + 1) * nlt_of(d.L) * ncol;
    k_tc_analysis3<false><<<std::min(ntiles, cta_cap(a.max_ctas)), WS_THREADS, analysis_smem(false), s>>>(d, moff, img0,
                                                                                                img1, a, ncol, csz);
  } else {
    const int ncol = ceil_div(d.nr, 32), csz = ceil_div(d.nr, ncol);
    const int ntiles = (d.M + 1) * nlt_of(d.L) * ncol;
    k_tc_analysis3<true><<<std::min(ntiles, cta_cap(a.max_ctas)), WS_THREADS, analysis_smem(true), s>>>(d, moff, img0, img1,
                                                                                              a, ncol, csz);
  }
}

}  // namespace gd

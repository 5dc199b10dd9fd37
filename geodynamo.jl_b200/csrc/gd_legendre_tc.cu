// gd_legendre_tc.cu -- mixed-precision Legendre synthesis and analysis on the
// 5th-generation tensor cores (tcgen05.mma kind::tf32, M = 128, N = 64),
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
#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"
#include "gd_tc.cuh"

namespace gd {

using namespace tc;

namespace {

constexpr int TC_M = 128;
constexpr int TC_N = 64;
constexpr int TC_K = 32;                       // TF32 elements per 128-byte row
constexpr int TILE_A_FLOATS = TC_M * TC_K;      // 4096 floats = 16 KB
constexpr int TILE_B_FLOATS = TC_N * TC_K;      // 2048 floats = 8 KB
constexpr int CHUNK_FLOATS = 2 * TILE_A_FLOATS; // hi image then lo image (32 KB)
constexpr uint32_t IDESC = idesc_tf32(TC_M, TC_N);
// A: [parity][hi,lo] x 16 KB ; B: [2 slots][hi,lo] x 8 KB ; barrier + TMEM slot.
// 97 KB per CTA: two CTAs per SM, each holding at most 256 TMEM columns.
constexpr int SMEM_A = 2 * CHUNK_FLOATS * 4;    // 64 KB
constexpr int SMEM_B = 2 * 2 * TILE_B_FLOATS * 4;  // 32 KB
constexpr size_t SMEM_BYTES = 1024 + SMEM_A + SMEM_B + 64;

__device__ __forceinline__ int kpar(int L, int m, int p) { return p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2; }
__device__ __host__ __forceinline__ int nck_h(int L, int m, int p) {
  const int k = p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2;
  return (k + TC_K - 1) / TC_K;
}

// chunk index of the synthesis image for (m, theta tile, parity, k chunk)
__device__ __forceinline__ long synth_chunk(const long* cofs, int L, int m, int tile, int p, int kc) {
  const int n0 = nck_h(L, m, 0), n1 = nck_h(L, m, 1);
  return cofs[m] + (long)tile * (n0 + n1) + (p == 0 ? kc : n0 + kc);
}

struct Smem {
  float* A;        // [p][hi|lo] chunks (CHUNK_FLOATS each)
  float* B;        // [slot][hi|lo] (TILE_B_FLOATS each)
  uint64_t* bar;
  uint32_t* tslot;
};

__device__ __forceinline__ Smem carve(unsigned char* raw) {
  const uintptr_t p = (reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023);
  Smem s;
  s.A = reinterpret_cast<float*>(p);
  s.B = reinterpret_cast<float*>(p + SMEM_A);
  s.bar = reinterpret_cast<uint64_t*>(p + SMEM_A + SMEM_B);
  s.tslot = reinterpret_cast<uint32_t*>(p + SMEM_A + SMEM_B + 16);
  return s;
}

__device__ __forceinline__ float* Bslot(const Smem& s, int slot, int hl) {
  return s.B + (slot * 2 + hl) * TILE_B_FLOATS;
}

// Copy one pre-swizzled 32 KB chunk (hi + lo) into A[p].
__device__ __forceinline__ void load_chunk(const Smem& s, int p, const float* __restrict__ img, long chunk) {
  const uint4* src = reinterpret_cast<const uint4*>(img + chunk * CHUNK_FLOATS);
  uint4* dst = reinterpret_cast<uint4*>(s.A + p * CHUNK_FLOATS);
  for (int i = threadIdx.x; i < CHUNK_FLOATS / 4; i += 128) dst[i] = __ldg(&src[i]);
}


__device__ __forceinline__ void put_split(float* hi, float* lo, int row, int k, double x) {
  const float h = tf32_rn((float)x);
  const float l = tf32_rn((float)(x - (double)h));
  const uint32_t o = sw128_offset(row, k) >> 2;
  hi[o] = h;
  lo[o] = l;
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
                                            const float* Bhi, const float* Blo, bool first) {
  const uint32_t ah = smem_addr(Ahi), al = smem_addr(Alo), bh = smem_addr(Bhi), bl = smem_addr(Blo);
#pragma unroll
  for (int ks = 0; ks < TC_K / 8; ++ks) {
    const uint32_t off = ks * 32;  // 8 TF32 = 32 bytes along K
    const uint64_t adh = sw128_desc(ah + off), adl = sw128_desc(al + off);
    const uint64_t bdh = sw128_desc(bh + off), bdl = sw128_desc(bl + off);
    mma_tf32(tmem + dcol, adh, bdh, IDESC, (first && ks == 0) ? 0u : 1u);
    mma_tf32(tmem + dcol, adh, bdl, IDESC, 1u);
    mma_tf32(tmem + dcol, adl, bdh, IDESC, 1u);
  }
}

// Commit the MMAs issued so far by thread 0 and wait for them (all threads).
__device__ __forceinline__ bool commit_wait(const Smem& s, uint32_t& phase, int* err) {
  if (threadIdx.x == 0) mma_commit(smem_addr(s.bar));
  const bool ok = mbar_wait(s.bar, phase, err);
  phase ^= 1u;
  fence_after_sync();
  return ok;
}

__device__ __forceinline__ void tc_prologue(const Smem& s, uint32_t ncols) {
  if (threadIdx.x == 0) mbar_init(s.bar, 1);
  if ((threadIdx.x >> 5) == 0) tmem_alloc(s.tslot, ncols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
}

__device__ __forceinline__ void tc_epilogue_free(const Smem& s, uint32_t tmem, uint32_t ncols) {
  fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace

// ---------------------------------------------------------------------------
// Table images.
// Synthesis chunk (m, tile, p, kc): row r -> ith = 128 tile + r,
//   k -> l = m + p + 2 (32 kc + k).
// Analysis chunk (m, p, c): row i -> l = m + p + 2 i, k -> ith = 32 c + k.
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
  const int nthc = (d.nth + TC_K - 1) / TC_K;
  const int p = blockIdx.y / nthc, c = blockIdx.y % nthc;
  float* hi = img + ((long)(m * 2 + p) * nthc + c) * CHUNK_FLOATS;
  float* lo = hi + TILE_A_FLOATS;
  const int kp = (p == 0) ? (d.L - m + 2) / 2 : (d.L - m + 1) / 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < TC_M * TC_K; e += gridDim.x * blockDim.x) {
    const int row = e / TC_K, k = e % TC_K;
    const int ith = TC_K * c + k;
    const int l = m + p + 2 * row;
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
long tc_analysis_chunks(const Dims& d) { return (long)(d.M + 1) * 2 * ((d.nth + TC_K - 1) / TC_K); }
size_t tc_chunk_bytes() { return (size_t)CHUNK_FLOATS * 4; }

void launch_build_tc_images(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const double* T,
                            float* synth_img, float* anal_img) {
  const int ntile = (d.nth + TC_M - 1) / TC_M;
  const int maxloc = ntile * (nck_h(d.L, 0, 0) + nck_h(d.L, 0, 1));
  k_build_synth_image<<<dim3(8, maxloc, d.M + 1), 256, 0, s>>>(d, moff, cofs, T, synth_img);
  const int nthc = (d.nth + TC_K - 1) / TC_K;
  k_build_analysis_image<<<dim3(8, 2 * nthc, d.M + 1), 256, 0, s>>>(d, moff, T, anal_img);
}

// ---------------------------------------------------------------------------
// Scalar synthesis: columns n = (field, r, re/im) flattened, 64 per CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 2) k_tc_synth_scalar(Dims d, const int* __restrict__ moff,
                                                            const long* __restrict__ cofs,
                                                            const float* __restrict__ img, TcSynthArgs a) {
  extern __shared__ unsigned char smem_raw[];
  const Smem s = carve(smem_raw);
  const int m = blockIdx.z, tile = blockIdx.y, n0 = blockIdx.x * TC_N;
  const int Ntot = a.nf * d.nr * 2;
  if (tile * TC_M >= d.nth || n0 >= Ntot) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = d.L, mb = moff[m];
  const size_t NM = d.nlm;
  const int nc0 = nck_h(L, m, 0), nc1 = nck_h(L, m, 1);
  tc_prologue(s, 128);
  const uint32_t tmem = *s.tslot;
  uint32_t phase = 0;
  bool ok = true;
  for (int kc = 0; kc < nc0 && ok; ++kc) {
    load_chunk(s, 0, img, synth_chunk(cofs, L, m, tile, 0, kc));
    if (kc < nc1) load_chunk(s, 1, img, synth_chunk(cofs, L, m, tile, 1, kc));
    for (int row = warp; row < TC_N; row += 4) {
      const int ng = n0 + row;
      double v0 = 0.0, v1 = 0.0;
      const int l = m + 2 * (TC_K * kc + lane);
      if (ng < Ntot) {
        const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
        const double* src = a.coef[f] + ((size_t)c * d.nr + r) * NM + mb - m;
        if (l <= L) v0 = src[l];
        if (l + 1 <= L) v1 = src[l + 1];
      }
      put_split(Bslot(s, 0, 0), Bslot(s, 0, 1), row, lane, v0);
      put_split(Bslot(s, 1, 0), Bslot(s, 1, 1), row, lane, v1);
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after_sync();
      issue_chunk(tmem, 0, s.A, s.A + TILE_A_FLOATS, Bslot(s, 0, 0), Bslot(s, 0, 1), kc == 0);
      if (kc < nc1)
        issue_chunk(tmem, TC_N, s.A + CHUNK_FLOATS, s.A + CHUNK_FLOATS + TILE_A_FLOATS, Bslot(s, 1, 0),
                    Bslot(s, 1, 1), kc == 0);
    }
    ok = commit_wait(s, phase, a.err);
  }
  if (ok) {
    const int ith = tile * TC_M + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < TC_N; c0 += 8) {
      float e[8], o[8];
      tmem_ld8(trow + c0, e);
      if (nc1 > 0) tmem_ld8(trow + TC_N + c0, o);
      tmem_ld_wait();
      if (nc1 == 0) {
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = 0.f;
      }
      if (ith < d.nth) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const int ng = n0 + c0 + j;
          if (ng >= Ntot) continue;
          const int f = ng / (2 * d.nr), r = (ng % (2 * d.nr)) >> 1;
          const size_t base = (((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2) * d.nth + ith;
          a.out[base] = make_float2(e[j] + o[j], e[j + 1] + o[j + 1]);
          a.out[base + d.nth] = make_float2(e[j] - o[j], e[j + 1] - o[j + 1]);
        }
      }
    }
  }
  tc_epilogue_free(s, tmem, 128);
}

// ---------------------------------------------------------------------------
// Vector synthesis: 16 shells per CTA, columns [S: 16 r x re/im][T: 16 r x re/im].
// Accumulators: [dP even | dP odd | Q even | Q odd] x 64 columns.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 2) k_tc_synth_vector(Dims d, const int* __restrict__ moff,
                                                            const long* __restrict__ cofs,
                                                            const float* __restrict__ img_dp,
                                                            const float* __restrict__ img_q, TcSynthArgs a) {
  extern __shared__ unsigned char smem_raw[];
  const Smem s = carve(smem_raw);
  const int m = blockIdx.z, tile = blockIdx.y, r0 = blockIdx.x * 16;
  if (tile * TC_M >= d.nth || r0 >= d.nr) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = d.L, mb = moff[m];
  const size_t NM = d.nlm;
  const int nc0 = nck_h(L, m, 0), nc1 = nck_h(L, m, 1);
  tc_prologue(s, 256);
  const uint32_t tmem = *s.tslot;
  uint32_t phase = 0;
  bool ok = true;
  for (int kc = 0; kc < nc0 && ok; ++kc) {
    for (int row = warp; row < TC_N; row += 4) {
      const int fld = row >> 5, r = r0 + ((row & 31) >> 1), c = row & 1;
      double v0 = 0.0, v1 = 0.0;
      const int l = m + 2 * (TC_K * kc + lane);
      if (r < d.nr) {
        const double* src = a.coef[fld] + ((size_t)c * d.nr + r) * NM + mb - m;
        if (l <= L) v0 = src[l];
        if (l + 1 <= L) v1 = src[l + 1];
      }
      put_split(Bslot(s, 0, 0), Bslot(s, 0, 1), row, lane, v0);
      put_split(Bslot(s, 1, 0), Bslot(s, 1, 1), row, lane, v1);
    }
    for (int t = 0; t < 2 && ok; ++t) {
      const float* img = t == 0 ? img_dp : img_q;
      load_chunk(s, 0, img, synth_chunk(cofs, L, m, tile, 0, kc));
      if (kc < nc1) load_chunk(s, 1, img, synth_chunk(cofs, L, m, tile, 1, kc));
      fence_proxy_async();
      __syncthreads();
      if (threadIdx.x == 0) {
        fence_after_sync();
        issue_chunk(tmem, (t * 2 + 0) * TC_N, s.A, s.A + TILE_A_FLOATS, Bslot(s, 0, 0), Bslot(s, 0, 1), kc == 0);
        if (kc < nc1)
          issue_chunk(tmem, (t * 2 + 1) * TC_N, s.A + CHUNK_FLOATS, s.A + CHUNK_FLOATS + TILE_A_FLOATS,
                      Bslot(s, 1, 0), Bslot(s, 1, 1), kc == 0);
      }
      ok = commit_wait(s, phase, a.err);
    }
  }
  if (ok) {
    const int ith = tile * TC_M + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int jj = 0; jj < 32; jj += 8) {
      float dse[8], dso[8], dte[8], dto[8], qse[8], qso[8], qte[8], qto[8];
      tmem_ld8(trow + 0 * TC_N + jj, dse);
      tmem_ld8(trow + 0 * TC_N + 32 + jj, dte);
      tmem_ld8(trow + 2 * TC_N + jj, qse);
      tmem_ld8(trow + 2 * TC_N + 32 + jj, qte);
      if (nc1 > 0) {
        tmem_ld8(trow + 1 * TC_N + jj, dso);
        tmem_ld8(trow + 1 * TC_N + 32 + jj, dto);
        tmem_ld8(trow + 3 * TC_N + jj, qso);
        tmem_ld8(trow + 3 * TC_N + 32 + jj, qto);
      }
      tmem_ld_wait();
      if (nc1 == 0) {
#pragma unroll
        for (int j = 0; j < 8; ++j) dso[j] = dto[j] = qso[j] = qto[j] = 0.f;
      }
      if (ith < d.nth) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const int r = r0 + (jj + j) / 2;
          if (r >= d.nr) continue;
#pragma unroll
          for (int sN = 0; sN < 2; ++sN) {
            float DS[2], DT[2], QS[2], QT[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              if (sN == 0) {
                DS[c] = dse[j + c] + dso[j + c]; DT[c] = dte[j + c] + dto[j + c];
                QS[c] = qse[j + c] + qso[j + c]; QT[c] = qte[j + c] + qto[j + c];
              } else {  // dP has the opposite north/south symmetry
                DS[c] = dso[j + c] - dse[j + c]; DT[c] = dto[j + c] - dte[j + c];
                QS[c] = qse[j + c] - qso[j + c]; QT[c] = qte[j + c] - qto[j + c];
              }
            }
            const size_t b0 = (((size_t)(0 * d.nr + r) * (d.M + 1) + m) * 2 + sN) * d.nth + ith;
            const size_t b1 = (((size_t)(1 * d.nr + r) * (d.M + 1) + m) * 2 + sN) * d.nth + ith;
            a.out[b0] = make_float2(DS[0] - QT[1], DS[1] + QT[0]);
            a.out[b1] = make_float2(-QS[1] - DT[0], QS[0] - DT[1]);
          }
        }
      }
    }
  }
  tc_epilogue_free(s, tmem, 256);
}

// ---------------------------------------------------------------------------
// Scalar analysis: CTA per (m, 64 columns n = (field, r, re/im)); K = theta.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 2) k_tc_analysis_scalar(Dims d, const int* __restrict__ moff,
                                                               const float* __restrict__ img, TcAnalysisArgs a) {
  extern __shared__ unsigned char smem_raw[];
  const Smem s = carve(smem_raw);
  const int m = blockIdx.z, n0 = blockIdx.x * TC_N;
  const int Ntot = a.nf * d.nr * 2;
  if (n0 >= Ntot) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = d.L, mb = moff[m];
  const size_t NM = d.nlm;
  const int k1 = kpar(L, m, 1);
  const int nthc = (d.nth + TC_K - 1) / TC_K;
  tc_prologue(s, 128);
  const uint32_t tmem = *s.tslot;
  uint32_t phase = 0;
  bool ok = true;
  for (int cc = 0; cc < nthc && ok; ++cc) {
    load_chunk(s, 0, img, ((long)(m * 2 + 0) * nthc + cc));
    if (k1 > 0) load_chunk(s, 1, img, ((long)(m * 2 + 1) * nthc + cc));
    // B: fold s -> slot s ; rows (f, r, re) and (f, r, im)
    for (int pr = warp; pr < TC_N / 2; pr += 4) {
      const int pg = n0 / 2 + pr;
      const int ith = TC_K * cc + lane;
#pragma unroll
      for (int sf = 0; sf < 2; ++sf) {
        float2 v = make_float2(0.f, 0.f);
        if (pg < Ntot / 2 && ith < d.nth) {
          const int f = pg / d.nr, r = pg % d.nr;
          v = a.in[(((size_t)(f * d.nr + r) * (d.M + 1) + m) * 2 + sf) * d.nth + ith];
        }
        put_split_f(Bslot(s, sf, 0), Bslot(s, sf, 1), 2 * pr, lane, v.x);
        put_split_f(Bslot(s, sf, 0), Bslot(s, sf, 1), 2 * pr + 1, lane, v.y);
      }
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      fence_after_sync();
      issue_chunk(tmem, 0, s.A, s.A + TILE_A_FLOATS, Bslot(s, 0, 0), Bslot(s, 0, 1), cc == 0);
      if (k1 > 0)
        issue_chunk(tmem, TC_N, s.A + CHUNK_FLOATS, s.A + CHUNK_FLOATS + TILE_A_FLOATS, Bslot(s, 1, 0),
                    Bslot(s, 1, 1), cc == 0);
    }
    ok = commit_wait(s, phase, a.err);
  }
  if (ok) {
    const int i = warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int p = 0; p < 2; ++p) {
      if (p == 1 && k1 == 0) break;
      const int kp = kpar(L, m, p);
      const int l = m + p + 2 * i;
      for (int c0 = 0; c0 < TC_N; c0 += 8) {
        float v[8];
        tmem_ld8(trow + p * TC_N + c0, v);
        tmem_ld_wait();
        if (i < kp) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int ng = n0 + c0 + j;
            if (ng >= Ntot) continue;
            const int f = ng / (2 * d.nr), rem = ng % (2 * d.nr), r = rem >> 1, c = rem & 1;
            const double val = (c == 1 && m == 0) ? 0.0 : (double)v[j];
            a.out[f][((size_t)c * d.nr + r) * NM + mb + (l - m)] = val;
          }
        }
      }
    }
  }
  tc_epilogue_free(s, tmem, 128);
}

// ---------------------------------------------------------------------------
// Vector analysis: CTA per (m, 16 shells); columns [G_theta: 16 r x re/im][G_phi].
// Accumulators [dP even | dP odd | Q even | Q odd]; the dP rows of parity p take
// the fold 1 - p, the Q rows the fold p.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 2) k_tc_analysis_vector(Dims d, const int* __restrict__ moff,
                                                               const float* __restrict__ img_dp,
                                                               const float* __restrict__ img_q, TcAnalysisArgs a) {
  extern __shared__ unsigned char smem_raw[];
  const Smem s = carve(smem_raw);
  const int m = blockIdx.z, r0 = blockIdx.x * 16;
  if (r0 >= d.nr) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int L = d.L, mb = moff[m];
  const size_t NM = d.nlm;
  const int k1 = kpar(L, m, 1);
  const int nthc = (d.nth + TC_K - 1) / TC_K;
  tc_prologue(s, 256);
  const uint32_t tmem = *s.tslot;
  uint32_t phase = 0;
  bool ok = true;
  for (int cc = 0; cc < nthc && ok; ++cc) {
    for (int pr = warp; pr < TC_N / 2; pr += 4) {
      const int comp = pr >> 4, r = r0 + (pr & 15);
      const int ith = TC_K * cc + lane;
#pragma unroll
      for (int sf = 0; sf < 2; ++sf) {
        float2 v = make_float2(0.f, 0.f);
        if (r < d.nr && ith < d.nth) v = a.in[(((size_t)(comp * d.nr + r) * (d.M + 1) + m) * 2 + sf) * d.nth + ith];
        put_split_f(Bslot(s, sf, 0), Bslot(s, sf, 1), 2 * pr, lane, v.x);
        put_split_f(Bslot(s, sf, 0), Bslot(s, sf, 1), 2 * pr + 1, lane, v.y);
      }
    }
    for (int t = 0; t < 2 && ok; ++t) {
      const float* img = t == 0 ? img_dp : img_q;
      load_chunk(s, 0, img, ((long)(m * 2 + 0) * nthc + cc));
      if (k1 > 0) load_chunk(s, 1, img, ((long)(m * 2 + 1) * nthc + cc));
      fence_proxy_async();
      __syncthreads();
      if (threadIdx.x == 0) {
        fence_after_sync();
        // parity 0 rows: dP takes fold 1, Q fold 0; parity 1 rows: dP fold 0, Q fold 1
        const int f0 = (t == 0) ? 1 : 0, f1 = 1 - f0;
        issue_chunk(tmem, (t * 2 + 0) * TC_N, s.A, s.A + TILE_A_FLOATS, Bslot(s, f0, 0), Bslot(s, f0, 1), cc == 0);
        if (k1 > 0)
          issue_chunk(tmem, (t * 2 + 1) * TC_N, s.A + CHUNK_FLOATS, s.A + CHUNK_FLOATS + TILE_A_FLOATS,
                      Bslot(s, f1, 0), Bslot(s, f1, 1), cc == 0);
      }
      ok = commit_wait(s, phase, a.err);
    }
  }
  if (ok) {
    const int i = warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int p = 0; p < 2; ++p) {
      if (p == 1 && k1 == 0) break;
      const int kp = kpar(L, m, p);
      const int l = m + p + 2 * i;
      const double fl = (l == 0) ? 0.0 : 1.0 / ((double)l * (l + 1.0));
      const double lf = (double)l * (l + 1.0);
      for (int jj = 0; jj < 32; jj += 8) {
        float dth[8], dph[8], qth[8], qph[8];
        tmem_ld8(trow + (0 * 2 + p) * TC_N + jj, dth);
        tmem_ld8(trow + (0 * 2 + p) * TC_N + 32 + jj, dph);
        tmem_ld8(trow + (1 * 2 + p) * TC_N + jj, qth);
        tmem_ld8(trow + (1 * 2 + p) * TC_N + 32 + jj, qph);
        tmem_ld_wait();
        if (i >= kp) continue;
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const int r = r0 + (jj + j) / 2;
          if (r >= d.nr) continue;
          const double Sre = ((double)dth[j] + (double)qph[j + 1]) * fl;
          const double Sim = ((double)dth[j + 1] - (double)qph[j]) * fl;
          const double Tre = ((double)qth[j + 1] - (double)dph[j]) * fl;
          const double Tim = (-(double)qth[j] - (double)dph[j + 1]) * fl;
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
  tc_epilogue_free(s, tmem, 256);
}

// ---------------------------------------------------------------------------
static bool g_attr_done = false;
static void set_attrs() {
  if (g_attr_done) return;
  cudaFuncSetAttribute(k_tc_synth_scalar, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  cudaFuncSetAttribute(k_tc_synth_vector, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  cudaFuncSetAttribute(k_tc_analysis_scalar, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  cudaFuncSetAttribute(k_tc_analysis_vector, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  g_attr_done = true;
}

void launch_tc_synth(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const float* img0,
                     const float* img1, const TcSynthArgs& a, bool vec) {
  set_attrs();
  const int ntile = (d.nth + TC_M - 1) / TC_M;
  if (!vec) {
    dim3 grid(ceil_div(a.nf * d.nr * 2, TC_N), ntile, d.M + 1);
    k_tc_synth_scalar<<<grid, 128, SMEM_BYTES, s>>>(d, moff, cofs, img0, a);
  } else {
    dim3 grid(ceil_div(d.nr, 16), ntile, d.M + 1);
    k_tc_synth_vector<<<grid, 128, SMEM_BYTES, s>>>(d, moff, cofs, img0, img1, a);
  }
}

void launch_tc_analysis(cudaStream_t s, const Dims& d, const int* moff, const float* img0, const float* img1,
                        const TcAnalysisArgs& a) {
  set_attrs();
  if (a.epi == EPI_SCALAR) {
    dim3 grid(ceil_div(a.nf * d.nr * 2, TC_N), 1, d.M + 1);
    k_tc_analysis_scalar<<<grid, 128, SMEM_BYTES, s>>>(d, moff, img0, a);
  } else {
    dim3 grid(ceil_div(d.nr, 16), 1, d.M + 1);
    k_tc_analysis_vector<<<grid, 128, SMEM_BYTES, s>>>(d, moff, img0, img1, a);
  }
}

}  // namespace gd

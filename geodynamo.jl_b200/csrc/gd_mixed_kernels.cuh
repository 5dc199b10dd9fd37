// gd_mixed_kernels.cuh -- launch interface of the tensor-core Legendre kernels.
#pragma once

#include <vector>

#include "gd_internal.cuh"
#include "gd_tc.cuh"

namespace gd {

// 32-deep K chunks of parity p (l - m even / odd) for order m.
__host__ __device__ __forceinline__ int tc_nck(int L, int m, int p) {
  const int k = p == 0 ? (L - m + 2) / 2 : (L - m + 1) / 2;
  return (k + 31) / 32;
}
// Synthesis pipeline step of (parity p, K chunk kc): odd-parity chunks
// interleave with the even ones while both exist.
__host__ __device__ __forceinline__ int tc_step_of(int p, int kc, int nc1) { return kc < nc1 ? 2 * kc + p : nc1 + kc; }

// Destination of runtime coefficients written straight into a synthesis
// B image (split TF32 hi / lo, 128-byte swizzled): chunk (column tile ct, m,
// step) at ct * ttot + bofs[m] + step, NCS columns x 32 K each.
struct SynthImageOut {
  float* img;         // null: write FP64 outputs instead
  const long* bofs;   // first step of order m within a column tile
  long ttot;          // steps per column tile
};

// Where mode (l, m) lands in every chunk of a synthesis image: the step
// within the column tile and the K index; fixed for a thread that owns one
// mode and walks r.
struct SynthImagePos {
  long step;  // bofs[m] + step of (parity, K chunk)
  int k;      // K index in the chunk
};
__device__ __forceinline__ SynthImagePos synth_image_pos(const SynthImageOut& o, int L, int m, int l) {
  const int q = l - m, p = q & 1, idx = q >> 1;
  return SynthImagePos{o.bofs[m] + tc_step_of(p, idx >> 5, tc_nck(L, m, 1)), idx & 31};
}
// Split v = hi + lo into column col of column tile ct.
__device__ __forceinline__ void synth_image_put(const SynthImageOut& o, int ncs, const SynthImagePos& at, int ct,
                                                int col, double v) {
  float* hi = o.img + ((long)ct * o.ttot + at.step) * (2L * ncs * 32);
  const uint32_t off = tc::sw128_offset((uint32_t)col, (uint32_t)at.k) >> 2;
  const float f = __double2float_rn(v), h = tc::tf32_rn(f);
  hi[off] = h;
  hi[(size_t)ncs * 32 + off] = tc::tf32_rn(f - h);
}

// Colatitude pairs per block of the blocked Fourier layout written by the
// synthesis and read by the fused phase kernels: float4 (north Re, north Im,
// south Re, south Im) at [comp][r][theta block][m][pair in block].
constexpr int FOURIER_BLOCK = 2;

struct TcSynthArgs {
  const double* coef[4];  // scalar: nf fields ; vector: [0] = S (poloidal), [1] = T (toroidal)
  float4* out;            // blocked FP32 Fourier buffer, comps consecutive
  int nblk;               // theta blocks (ceil(nth / FOURIER_BLOCK))
  int nf;
  int* err;               // set to 1 if a bounded wait expires
  long long wait_limit;   // clock cycles of each bounded wait (0: the default)
  int omit_plus1;         // > 0: CTA 0 omits the bulk copies of pipeline step omit_plus1 - 1 (error-path tests)
  float* bimg;            // split coefficient images (tc_synth_bimage_floats floats)
  long ttot;              // pipeline steps summed over m (one column tile)
  int prep_mask;          // fields the pre-pass writes into bimg (the others are written by their producer)
  int max_ctas;           // persistent CTAs of the launch (0: one per SM)
};

// Floats of coefficient-image scratch the synthesis needs (the scalar case, 4 fields, bounds both).
size_t tc_synth_bimage_floats(const Dims& d, long ttot);

// Recurrence data for on-the-fly table rows (see k_rec_tables).
struct TcRec {
  const double *ra, *rb, *rc;  // per m-major mode
  const double *r1a, *r1b;     // m = 1 column, per l
  const double* pmm;           // [m][ith]
  const double *x, *sth, *sinv;
};

struct TcAnalysisArgs {
  const float2* in;       // folded FP32 Fourier buffer
  double* out[4];         // scalar: nf outputs ; vector: [0] toroidal slot, [1] poloidal slot
  int nf;
  int epi;
  int* err;
  long long wait_limit;   // clock cycles of each bounded wait (0: the default)
  int max_ctas;           // persistent CTAs of the launch (0: one per SM)
};

long tc_synth_chunks(const Dims& d, std::vector<long>& cofs);
long tc_analysis_chunks(const Dims& d);
size_t tc_chunk_bytes();
// Builds the synthesis and/or analysis image of one FP64 table (either pointer may be null).
void launch_build_tc_images(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const double* T,
                            float* synth_img, float* anal_img);
void launch_tc_synth(cudaStream_t s, const Dims& d, const int* moff, const long* cofs, const float* imgP,
                     const float* imgD, const double* sinv, const TcSynthArgs& a, bool vec);
void launch_tc_analysis(cudaStream_t s, const Dims& d, const int* moff, const float* img0, const float* img1,
                        const TcAnalysisArgs& a);
void launch_cast_d2f(cudaStream_t s, size_t n, const double* src, float* dst);
// Radial operators of gd_spectral.cu writing a synthesis B image instead of FP64 arrays.
void launch_gradients_img(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                          const double* d1, const double* T, const SynthImageOut& img);
void launch_curl_img(cudaStream_t s, const Dims& d, const int* lof, const int* mof, const double* rinv,
                     const double* rinv2, const double* d1, const double* d2, const double* tor, const double* pol,
                     const SynthImageOut& img);

}  // namespace gd

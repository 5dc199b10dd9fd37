// gd_mixed_kernels.cuh -- launch interface of the tensor-core Legendre kernels.
#pragma once

#include <vector>

#include "gd_internal.cuh"

namespace gd {

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
  float* bimg;            // scratch for the split coefficient images (tc_synth_bimage_floats)
  long ttot;              // pipeline steps summed over m (one column tile)
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

}  // namespace gd

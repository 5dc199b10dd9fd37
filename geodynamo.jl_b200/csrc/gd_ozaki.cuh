// gd_ozaki.cuh -- FP64-accurate vector synthesis on the tcgen05 tensor cores by
// int8 digit slices (gd_ozaki.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace gd {

struct Dims;

// Sizes of the slice images for a handle's dimensions and digit count (5 or 6
// digits of 7 bits per operand; 48 or 32 coefficient columns per tile).
struct OzLayout {
  int digits;
  int ncols;      // coefficient columns per tile
  int ncb;        // column tiles (4 nr columns: [S re, S im, T re, T im] per shell)
  size_t a_bytes;  // table images
  size_t rs_elems; // table row scales (double)
  size_t b_bytes;  // coefficient images
  size_t cs_elems; // coefficient column scales (double)
};

struct OzSynthArgs {
  double2* out;       // FP64 Fourier layout of the DMMA synthesis: [comp][r][m][north, south][theta]
  float4* out32;      // may be null: the FP32 blocked copy (as SynthArgs::out32)
  size_t out32_comp;  // float4 per component of out32
  int* err;           // set to 1 if a bounded wait expires
  long long wait_limit;
  int omit_plus1;     // > 0: CTA 0 omits the bulk copies of pipeline step omit_plus1 - 1 (error-path tests)
  int max_ctas;       // persistent CTAs (0: one per SM)
};

OzLayout oz_layout(const Dims& d, int digits);
// One shell range without segments or a ball centre (the tile decomposition
// assumes one radial grid).
bool oz_supported(const Dims& d);
// Table images and row exponents of dP and Q (set-up, once per handle).
void launch_oz_tables(cudaStream_t s, const Dims& d, const int* moff, const double* dP, const double* Q,
                      const OzLayout& o, signed char* imgA, double* rsc);
// Coefficient images of S (poloidal) and T (toroidal), then the synthesis.
void launch_oz_synth_vector(cudaStream_t s, const Dims& d, const int* moff, const OzLayout& o, const double* S,
                            const double* T, const signed char* imgA, const double* rsc, signed char* imgB,
                            double* csc, const OzSynthArgs& a);

}  // namespace gd

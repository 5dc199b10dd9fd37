// gd_fused.cuh -- launch interface of the fused per-phase grid kernels
// (gd_fused.cu) of the mixed-precision step.
#pragma once

#include "gd_internal.cuh"

namespace gd {

enum { FUSED_GRID = 0, FUSED_TEMPERATURE = 1, FUSED_VELOCITY = 2, FUSED_INDUCTION = 3 };

struct FusedArgs {
  const float4* fin[8];  // blocked Fourier coefficients, one pointer per input component
  int nin;
  float* gout[8];        // grid phase: one grid per input
  float2* G;             // folded transforms of the products [comp][r][m][s][ith]
  const double* w;       // Gauss weights (north half)
  const double* cth;     // Coriolis cos/sin tables, indexed by min(phi index, nlat - 1)
  const double* sthc;
  const double* sources; // internal heat sources per shell
  float rf, lf;          // Pm/E for the advection and Lorentz factors
  float cf;              // Pm/E for the Coriolis term (0: the term is formed elsewhere)
};

// Theta blocks of the blocked Fourier layout and float4 elements per component.
int fourier_blocks(const Dims& d);
size_t fourier_comp_elems(const Dims& d);
size_t fused_smem_bytes(int phase, int nlon);
void launch_fused(cudaStream_t s, const Dims& d, const FftPlan& p, const void* twf, int phase, const FusedArgs& a);

}  // namespace gd

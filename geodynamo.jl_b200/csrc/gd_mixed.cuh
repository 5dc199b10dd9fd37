// gd_mixed.cuh -- mixed-precision path: FP32 phi transforms and nonlinear
// products (fused per phase, grids in shared memory); Legendre contractions
// on the tcgen05 tensor cores in split TF32 (hi*hi + hi*lo + lo*hi, FP32
// accumulation in tensor memory); spectral state, radial operators and CNAB2
// stay FP64.
#pragma once

struct gd_handle;

namespace gd {
int mixed_create(gd_handle* h);
// Slice images and scratch of the int8-slice velocity synthesis
// (GD_STAGE_VEL_SYNTH_I8) for h->int8_digits; nothing if they exist already.
int mixed_prepare_int8(gd_handle* h);
// GD_ERR_CUDA if a tensor-core wait expired since creation (synchronises the stream).
int mixed_check_error(gd_handle* h);
// Error-path tests: the bound of every tensor-core wait (clock cycles, <= 0:
// the default) and a one-shot omission of the copies of one pipeline step in
// CTA 0 of the next synthesis (omit_step < 0: none).
int mixed_set_fault_test(gd_handle* h, long long wait_cycles, int omit_step);
void mixed_destroy(gd_handle* h);
size_t mixed_bytes(const gd_handle* h);
int mixed_temperature_nl(gd_handle* h);
int mixed_composition_nl(gd_handle* h);
// Boundary conditions (fixed values, tau flux correction) of F_TEMP or F_COMP
// over the handle's mode range (gd_api.cu).
void scalar_bc(gd_handle* h, int field);
// ball: the r = 0 level of nf consecutive nonlinear terms from field set to 0 for l >= 1
void regular_nl(gd_handle* h, int field, int nf);
int mixed_velocity_nl(gd_handle* h);
int mixed_magnetic_nl(gd_handle* h);
// GD_ERR_UNSUPPORTED for the product grids, which the mixed step does not store.
int mixed_grid_to_double(gd_handle* h, int grid, double* out);
int mixed_api_synth_scalar(gd_handle* h, const double* const* coef, int nf, double* grid_out);
int mixed_api_synth_vector(gd_handle* h, const double* tor, const double* pol, double* grid_out);
int mixed_api_analysis_scalar(gd_handle* h, const double* grid_in, int nf, double* const* out);
int mixed_api_analysis_vector(gd_handle* h, const double* grid_in, double* tor, double* pol);
}  // namespace gd

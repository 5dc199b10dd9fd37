// gd_mixed.cu -- mixed-precision path (placeholder until the tensor-core kernels land).
#include "gd_handle.cuh"
#include "gd_mixed.cuh"

namespace gd {
int mixed_create(gd_handle* h) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed precision not built"); }
void mixed_destroy(gd_handle*) {}
size_t mixed_bytes(const gd_handle*) { return 0; }
int mixed_temperature_nl(gd_handle* h) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed precision not built"); }
int mixed_velocity_nl(gd_handle* h) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed precision not built"); }
int mixed_magnetic_nl(gd_handle* h) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed precision not built"); }
void mixed_grid_to_double(gd_handle*, int, double*) {}
int mixed_api_synth_scalar(gd_handle* h, const double* const*, int, double*) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed"); }
int mixed_api_synth_vector(gd_handle* h, const double*, const double*, double*) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed"); }
int mixed_api_analysis_scalar(gd_handle* h, const double*, int, double* const*) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed"); }
int mixed_api_analysis_vector(gd_handle* h, const double*, double*, double*) { return set_error(h, GD_ERR_UNSUPPORTED, "mixed"); }
}  // namespace gd

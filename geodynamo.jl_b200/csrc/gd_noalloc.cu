// gd_noalloc.cu -- scalar synthesis that allocates no device memory.
//
// gd_spectral_to_physical() stages host arrays through buffers the handle
// allocates on first use.  Some callers cannot allow any allocation at call
// time: a Julia session whose GPU memory belongs to CUDA.jl's pool (a direct
// cudaMalloc from a ccall'd library bypasses that pool and can fail once the
// pool holds the free memory), or a solver loop in a framework that forbids
// allocation between its own set-up and tear-down.  This entry point serves
// them: inputs and outputs are the caller's device buffers, and the Fourier
// intermediate lives in a fixed-size array in the library's device image
// instead of a cudaMalloc'd buffer.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "gd_handle.cuh"
#include "gd_internal.cuh"

// Scratch for the Fourier coefficients of one call: min(nfield, 4) x nr x
// (mmax+1) x nlat complex doubles.  Every GPU that loads the library holds
// these 64 MiB until the process exits.
static const size_t kScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_fourier_scratch[size_t(64) << 20];

// Device address of g_fourier_scratch, looked up once per device with that
// device current (host code cannot use the symbol's name as a device
// address).  The cached address belongs to the device's primary context, which
// lives as long as the process unless the caller resets the device; the mutex
// makes the first lookup safe when several host threads call at once.
static std::mutex g_scratch_mu;
static void* g_scratch_addr[64] = {};

static cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fourier_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

// Makes the handle's device current for the call and restores the caller's
// current device afterwards.
namespace {
struct DeviceScope {
  int prev = -1;
  cudaError_t enter(int device) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    return cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" int gd_spectral_to_physical_noalloc(gd_handle* h, int nfield, const double* d_coef, double* d_grid) {
  if (!h) return GD_ERR_ARG;
  if (!d_coef || !d_grid || nfield < 1) return gd::set_error(h, GD_ERR_ARG, "null device pointer or nfield < 1");
  const gd::Dims& d = h->d;
  const size_t per_field = (size_t)d.nr * (d.M + 1) * d.nlat * sizeof(double2);
  const int group = nfield < 4 ? nfield : 4;
  if (per_field * group > kScratchBytes)
    return gd::set_error(h, GD_ERR_CONFIG,
                         "gd_spectral_to_physical_noalloc needs " + std::to_string(per_field * group) +
                             " bytes of Fourier scratch (min(nfield,4) x nr x (mmax+1) x nlat x 16); the fixed "
                             "maximum is " + std::to_string(kScratchBytes) + " bytes");
  if (h->device < 0 || h->device >= 64) return gd::set_error(h, GD_ERR_ARG, "device index out of range");
  DeviceScope scope;
  cudaError_t e = scope.enter(h->device);
  if (e != cudaSuccess) return gd::set_error(h, GD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  void* scratch = nullptr;
  e = scratch_address(h->device, &scratch);
  if (e != cudaSuccess)
    return gd::set_error(h, GD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  double2* F = static_cast<double2*>(scratch);
  const size_t plane = (size_t)2 * d.nr * d.nlm;  // one field: Re and Im planes
  const size_t G = (size_t)d.nlat * d.nlon * d.nr;
  for (int f0 = 0; f0 < nfield; f0 += 4) {
    const int nf = nfield - f0 < 4 ? nfield - f0 : 4;
    gd::SynthArgs a{};
    a.table0 = h->d_P;
    for (int i = 0; i < nf; ++i) a.coef[i] = d_coef + plane * (f0 + i);
    a.nf = nf;
    a.out = F;
    gd::launch_synth_fp64(h->stream, d, h->d_moff, a, false);
    gd::launch_fft_synth<double>(h->stream, d, h->plan, h->d_tw, F, d_grid + G * f0, nf, G);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return gd::set_error(h, GD_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return GD_OK;
}

// gd_mixed.cu -- the mixed-precision step: FP32 grids, phi transforms and
// grid products; split-TF32 tensor-core Legendre contractions
// (gd_legendre_tc.cu); FP64 spectral operators, CNAB2 solves and energies
// (shared with the FP64 path).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "gd_handle.cuh"
#include "gd_internal.cuh"
#include "gd_mixed.cuh"
#include "gd_fused.cuh"
#include "gd_mixed_kernels.cuh"
#include "gd_ozaki.cuh"

namespace gd {

// Blocked FP32 Fourier buffers of the synthesized components (the fused
// phase kernels transform them in shared memory; the physical grids are not
// kept in HBM and are formed on request).
enum {
  FC_T = 0, FC_GTH = 1, FC_GPH = 2, FC_GR = 3,  // temperature phase (scalar synthesis order)
  FC_U = 4, FC_W = 6, FC_B = 8, FC_J = 10,      // theta, phi pairs
  FC_C = 12,                                    // composition phase: C, d_theta C, d_phi C, d_r C
  FC_COUNT = 16
};
// components allocated: the composition's only with composition
static int fc_count(const gd_handle* h) { return h->c.composition ? FC_COUNT : FC_C; }

struct MixedState {
  double *ra = nullptr, *rb = nullptr, *rc = nullptr, *r1a = nullptr, *r1b = nullptr, *pmm = nullptr,
         *sinv = nullptr;
  long* d_cofs = nullptr;
  float* img_synth[2] = {nullptr, nullptr};          // Pbar, dPbar/dtheta (synthesis orientation)
  float* img_anal[3] = {nullptr, nullptr, nullptr};  // Pbar, dPbar/dtheta, Q (analysis orientation)
  float4* d_Fall = nullptr;    // FC_COUNT blocked components
  size_t fcomp = 0;            // float4 per component
  float2* d_G = nullptr;       // folded transforms for the analysis, 2 components
  // split coefficient images of the synthesis (zeroed once; every writer
  // keeps its layout's padding at zero): scalar (T by the pre-pass, its
  // gradient by k_gradients), vector state fields (pre-pass), vector curls (k_curl)
  float* d_bimg_s = nullptr;
  float* d_bimg_vp = nullptr;
  float* d_bimg_vc = nullptr;
  long* d_bofs = nullptr;      // first step of order m within a column tile
  long ttot = 0;               // synthesis pipeline steps over all m (one column tile)
  float* d_stage = nullptr;    // 4 FP32 grids for the host-array entry points and grid downloads
  int* d_err = nullptr;
  long long wait_limit = 0;    // clock cycles of each bounded wait (0: the kernels' default)
  int omit_plus1 = 0;          // error-path tests: the next synthesis omits a step's copies in CTA 0
  // int8-slice velocity synthesis (GD_STAGE_VEL_SYNTH_I8): table images and
  // row exponents (built once per digit count), coefficient images and
  // column exponents (rewritten every step)
  int oz_digits = 0;
  OzLayout oz{};
  signed char* oz_imgA = nullptr;
  signed char* oz_imgB = nullptr;
  double* oz_rs = nullptr;
  double* oz_cs = nullptr;
  size_t bytes = 0;
  std::vector<void*> allocs;
  float4* F(int c) const { return d_Fall + fcomp * c; }
};

namespace {

int mcheck(gd_handle* h, cudaError_t e, const char* what) {
  if (e != cudaSuccess) return set_error(h, GD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return GD_OK;
}

template <typename T>
int malloc_m(gd_handle* h, T** p, size_t n) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
  if (e != cudaSuccess) return set_error(h, GD_ERR_CUDA, std::string("cudaMalloc (mixed): ") + cudaGetErrorString(e));
  h->mixed->allocs.push_back(q);
  h->mixed->bytes += n * sizeof(T);
  *p = static_cast<T*>(q);
  return GD_OK;
}

#define MAL(ptr, n)                             \
  do {                                          \
    int s_ = malloc_m(h, &(ptr), (size_t)(n));  \
    if (s_) return s_;                          \
  } while (0)

int launched(gd_handle* h, const char* what) { return mcheck(h, cudaGetLastError(), what); }


int nblocks(const gd_handle* h) { return fourier_blocks(h->d); }

SynthImageOut image_out(gd_handle* h, float* img) {
  SynthImageOut o{};
  o.img = img;
  o.bofs = h->mixed->d_bofs;
  o.ttot = h->mixed->ttot;
  return o;
}

// Legendre synthesis of nf scalar fields into consecutive blocked components
// from `out`; the fields of prep_mask are split by the pre-pass, the others
// are already in the scalar image.
int tc_synth_scalar(gd_handle* h, const double* const* coef, int nf, float4* out, int prep_mask) {
  MixedState* x = h->mixed;
  TcSynthArgs a{};
  for (int i = 0; i < nf; ++i) a.coef[i] = coef[i];
  a.nf = nf;
  a.out = out;
  a.nblk = nblocks(h);
  a.err = x->d_err;
  a.bimg = x->d_bimg_s;
  a.ttot = x->ttot;
  a.prep_mask = prep_mask;
  a.wait_limit = x->wait_limit;
  a.omit_plus1 = x->omit_plus1;
  a.max_ctas = h->tc_ctas;
  x->omit_plus1 = 0;  // one-shot
  { ProfScope p(h, "legendre_synth_scalar_tc"); launch_tc_synth(h->stream, h->d, h->d_moff, x->d_cofs, x->img_synth[0], nullptr, x->sinv, a, false); }
  return launched(h, "mixed scalar synthesis");
}

// Vector synthesis (tor, pol) -> (theta, phi) blocked components at out,
// out + 1.  tor/pol null: the coefficients are already in the curl image.
int tc_synth_vector(gd_handle* h, const double* tor, const double* pol, float4* out) {
  MixedState* x = h->mixed;
  TcSynthArgs a{};
  a.coef[0] = pol;
  a.coef[1] = tor;
  a.nf = 1;
  a.out = out;
  a.nblk = nblocks(h);
  a.err = x->d_err;
  const bool pre = tor != nullptr;
  a.bimg = pre ? x->d_bimg_vp : x->d_bimg_vc;
  a.ttot = x->ttot;
  a.prep_mask = pre ? 3 : 0;
  a.wait_limit = x->wait_limit;
  a.omit_plus1 = x->omit_plus1;
  a.max_ctas = h->tc_ctas;
  x->omit_plus1 = 0;
  { ProfScope p(h, "legendre_synth_vector_tc"); launch_tc_synth(h->stream, h->d, h->d_moff, x->d_cofs, x->img_synth[0], x->img_synth[1], x->sinv, a, true); }
  return launched(h, "mixed vector synthesis");
}

// Physical grids of ncomp blocked components (grid-only fused kernel).
int fourier_to_grid(gd_handle* h, const float4* const* fin, int ncomp, float* grid_out) {
  FusedArgs f{};
  for (int i = 0; i < ncomp; ++i) {
    f.fin[i] = fin[i];
    f.gout[i] = grid_out + h->grid_elems() * i;
  }
  f.nin = ncomp;
  { ProfScope p(h, "fft_synth_fp32"); launch_fused(h->stream, h->d, h->plan, h->d_twf, FUSED_GRID, f); }
  return launched(h, "fourier to grid");
}

int tc_analysis_scalar_G(gd_handle* h, int nf, double* const* out) {
  MixedState* x = h->mixed;
  TcAnalysisArgs a{};
  a.in = x->d_G;
  for (int i = 0; i < nf; ++i) a.out[i] = out[i];
  a.nf = nf;
  a.epi = EPI_SCALAR;
  a.err = x->d_err;
  a.wait_limit = x->wait_limit;
  a.max_ctas = h->tc_ctas;
  { ProfScope p(h, "legendre_analysis_scalar_tc"); launch_tc_analysis(h->stream, h->d, h->d_moff, x->img_anal[0], nullptr, a); }
  return launched(h, "mixed scalar analysis");
}

int tc_analysis_vector_G(gd_handle* h, double* out_tor, double* out_pol, int epi) {
  MixedState* x = h->mixed;
  TcAnalysisArgs a{};
  a.in = x->d_G;
  a.out[0] = out_tor;
  a.out[1] = out_pol;
  a.nf = 1;
  a.epi = epi;
  a.err = x->d_err;
  a.wait_limit = x->wait_limit;
  a.max_ctas = h->tc_ctas;
  { ProfScope p(h, "legendre_analysis_vector_tc"); launch_tc_analysis(h->stream, h->d, h->d_moff, x->img_anal[1], x->img_anal[2], a); }
  return launched(h, "mixed vector analysis");
}

// Analysis of FP32 grids (host-array entry points): phi transform into d_G, then Legendre
// (nf <= 2: the components d_G holds).
int tc_analysis_scalar(gd_handle* h, const float* grid_in, int nf, double* const* out) {
  if (nf > 2) return set_error(h, GD_ERR_ARG, "scalar analysis of more than two fields per pass");
  MixedState* x = h->mixed;
  { ProfScope p(h, "fft_analysis_fp32"); launch_fft_analysis<float>(h->stream, h->d, h->plan, h->d_twf, grid_in, h->grid_elems(), h->d_w, x->d_G, nf); }
  return tc_analysis_scalar_G(h, nf, out);
}

int tc_analysis_vector(gd_handle* h, const float* grid_in, double* out_tor, double* out_pol, int epi) {
  MixedState* x = h->mixed;
  { ProfScope p(h, "fft_analysis_fp32"); launch_fft_analysis<float>(h->stream, h->d, h->plan, h->d_twf, grid_in, h->grid_elems(), h->d_w, x->d_G, 2); }
  return tc_analysis_vector_G(h, out_tor, out_pol, epi);
}

FusedArgs phase_args(gd_handle* h) {
  FusedArgs f{};
  f.G = h->mixed->d_G;
  f.w = h->d_w;
  f.cth = h->d_cth;
  f.sthc = h->d_sthc;
  f.sources = h->d_sources;
  f.rf = (float)(h->c.magnetic_prandtl / h->c.ekman);
  f.lf = f.rf;
  f.cf = f.rf;
  return f;
}

// ---- the velocity chain in FP64 (GD_STAGE_*) ----
// FP64 Fourier components: [comp][r][m][s][ith] double2, nr x (mmax+1) x nlat
// per component (the FP64 path's layout).  The velocity components use
// components 0 and 1 of the handle's FP64 Fourier buffer, the folded
// transforms of the velocity products components 2 and 3.
size_t fourier64_comp(const Dims& d) { return (size_t)d.nr * (d.M + 1) * d.nlat; }

constexpr int CV_MT = 8;   // orders per CTA
constexpr int CV_CH = 64;  // colatitude pairs per pass

// Blocked FP32 Fourier components (float4 north Re, north Im, south Re, south
// Im at [comp][r][theta block][m][pair in block]) widened to the FP64
// synthesis layout (s = north / south row), for the FP64 Coriolis stage after
// a split-TF32 synthesis.  One CTA per (component, shell) and CV_MT orders;
// both sides are read and written in contiguous runs through shared memory.
__global__ void __launch_bounds__(256) k_widen_fourier(Dims d, double2* __restrict__ f64,
                                                      const float4* __restrict__ blk, size_t fcomp) {
  __shared__ double2 buf[CV_MT][2][CV_CH];
  const int m0 = blockIdx.x * CV_MT, cr = blockIdx.y;  // cr = comp nr + r
  const int nblk = (d.nth + FOURIER_BLOCK - 1) / FOURIER_BLOCK;
  const size_t run = (size_t)nblk * (d.M + 1) * FOURIER_BLOCK;
  const int comp = cr / d.nr, r = cr % d.nr;
  double2* dst64 = f64 + (size_t)cr * (d.M + 1) * 2 * d.nth;
  const float4* src = blk + comp * fcomp + (size_t)r * run;
  for (int i0 = 0; i0 < d.nth; i0 += CV_CH) {
    // blocked side: for each theta block, CV_MT orders x FOURIER_BLOCK pairs are contiguous
    for (int e = threadIdx.x; e < CV_CH * CV_MT; e += blockDim.x) {
      const int p = e % FOURIER_BLOCK, mm = (e / FOURIER_BLOCK) % CV_MT, bl = e / (FOURIER_BLOCK * CV_MT);
      const int i = bl * FOURIER_BLOCK + p, ith = i0 + i, m = m0 + mm;
      if (m > d.M || ith >= d.nth) continue;
      const float4 v = src[((size_t)(ith / FOURIER_BLOCK) * (d.M + 1) + m) * FOURIER_BLOCK + ith % FOURIER_BLOCK];
      buf[mm][0][i] = make_double2(v.x, v.y);
      buf[mm][1][i] = make_double2(v.z, v.w);
    }
    __syncthreads();
    // FP64 side: rows (m, s) of CV_CH consecutive colatitudes
    for (int e = threadIdx.x; e < CV_MT * 2 * CV_CH; e += blockDim.x) {
      const int mm = e / (2 * CV_CH), sr = (e / CV_CH) & 1, i = e % CV_CH;
      const int m = m0 + mm, ith = i0 + i;
      if (m <= d.M && ith < d.nth) dst64[((size_t)m * 2 + sr) * d.nth + ith] = buf[mm][sr][i];
    }
    __syncthreads();
  }
}

void launch_widen_fourier(cudaStream_t s, const Dims& d, double2* f64, const float4* blk, size_t fcomp, int ncomp) {
  const dim3 grid(ceil_div(d.M + 1, CV_MT), ncomp * d.nr);
  k_widen_fourier<<<grid, 256, 0, s>>>(d, f64, blk, fcomp);
}

// Folded transforms (same layout, float2 / double2): g64 = [g64 +] g32 or g32 = g64.
__global__ void k_fold_widen(size_t n, const float2* __restrict__ g32, double2* __restrict__ g64, int add) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 v = g32[i];
    double2 o = make_double2((double)v.x, (double)v.y);
    if (add) {
      const double2 a = g64[i];
      o = make_double2(a.x + o.x, a.y + o.y);
    }
    g64[i] = o;
  }
}
__global__ void k_fold_narrow(size_t n, const double2* __restrict__ g64, float2* __restrict__ g32) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = g64[i];
    g32[i] = make_float2((float)v.x, (float)v.y);
  }
}

}  // namespace

int mixed_create(gd_handle* h) {
  if (h->mixed) return GD_OK;
  int major = 0, minor = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, h->device);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, h->device);
  if (major != 10 || minor != 0)
    return set_error(h, GD_ERR_UNSUPPORTED, "the mixed path needs an sm_100 (B200) device for tcgen05");
  h->mixed = new MixedState();
  MixedState* x = h->mixed;
  const Dims& d = h->d;
  std::vector<long> cofs;
  const long nsyn = tc_synth_chunks(d, cofs);
  const long nana = tc_analysis_chunks(d);
  const size_t cb = tc_chunk_bytes() / sizeof(float);
  MAL(x->d_cofs, cofs.size());
  for (int t = 0; t < 2; ++t) MAL(x->img_synth[t], (size_t)nsyn * cb);
  const int ntt = (d.nth + 127) / 128;
  x->ttot = nsyn / ntt;
  const size_t nimg = tc_synth_bimage_floats(d, x->ttot);
  MAL(x->d_bimg_s, nimg);
  MAL(x->d_bimg_vp, nimg);
  MAL(x->d_bimg_vc, nimg);
  MAL(x->d_bofs, d.M + 2);
  std::vector<long> bofs(d.M + 2);
  for (int m = 0; m <= d.M + 1; ++m) bofs[m] = cofs[m] / ntt;
  for (int t = 0; t < 3; ++t) MAL(x->img_anal[t], (size_t)nana * cb);
  MAL(x->ra, d.nlm); MAL(x->rb, d.nlm); MAL(x->rc, d.nlm);
  MAL(x->r1a, d.L + 1); MAL(x->r1b, d.L + 1);
  MAL(x->pmm, (size_t)(d.M + 1) * d.nth); MAL(x->sinv, d.nth);
  x->fcomp = fourier_comp_elems(d);
  MAL(x->d_Fall, (size_t)fc_count(h) * x->fcomp);
  MAL(x->d_G, (size_t)2 * d.nr * (d.M + 1) * 2 * d.nth);
  MAL(x->d_stage, (size_t)4 * h->grid_elems());
  MAL(x->d_err, 4);
  int s = mcheck(h, cudaMemcpyAsync(x->d_cofs, cofs.data(), sizeof(long) * cofs.size(), cudaMemcpyHostToDevice,
                                    h->stream), "cofs upload");
  if (s) return s;
  s = mcheck(h, cudaMemcpyAsync(x->d_bofs, bofs.data(), sizeof(long) * bofs.size(), cudaMemcpyHostToDevice,
                                h->stream), "bofs upload");
  if (s) return s;
  for (float* img : {x->d_bimg_s, x->d_bimg_vp, x->d_bimg_vc}) {
    s = mcheck(h, cudaMemsetAsync(img, 0, sizeof(float) * nimg, h->stream), "memset");
    if (s) return s;
  }
  s = mcheck(h, cudaMemsetAsync(x->r1a, 0, sizeof(double) * (d.L + 1), h->stream), "memset");
  if (s) return s;
  s = mcheck(h, cudaMemsetAsync(x->r1b, 0, sizeof(double) * (d.L + 1), h->stream), "memset");
  if (s) return s;
  launch_rec_tables(h->stream, d, h->d_moff, h->d_x, h->d_sth, x->ra, x->rb, x->rc, x->r1a, x->r1b, x->pmm, x->sinv);
  const double* tabs[3] = {h->d_P, h->d_dP, h->d_Q};
  for (int t = 0; t < 3; ++t)
    launch_build_tc_images(h->stream, d, h->d_moff, x->d_cofs, tabs[t], t < 2 ? x->img_synth[t] : nullptr,
                           x->img_anal[t]);
  s = mcheck(h, cudaStreamSynchronize(h->stream), "cofs lifetime");
  s = launched(h, "table images");
  if (s) return s;
  // the carried components start as zero grids (the reference's physical
  // fields are zero-filled at allocation, src/fields.jl:82)
  s = mcheck(h, cudaMemsetAsync(x->d_Fall, 0, sizeof(float4) * fc_count(h) * x->fcomp, h->stream), "memset");
  if (s) return s;
  s = mcheck(h, cudaMemsetAsync(x->d_err, 0, sizeof(int), h->stream), "memset");
  if (s) return s;
  s = mcheck(h, cudaStreamSynchronize(h->stream), "mixed set-up");
  if (s) return s;
  return (h->fp64_stages & GD_STAGE_VEL_SYNTH_I8) ? mixed_prepare_int8(h) : GD_OK;
}

int mixed_prepare_int8(gd_handle* h) {
  MixedState* x = h->mixed;
  if (!x) return GD_OK;
  if (x->oz_digits == h->int8_digits) return GD_OK;
  const Dims& d = h->d;
  // the images of another digit count go first (and their pointers with them,
  // so that a failed allocation below leaves nothing to free twice)
  void** old[4] = {(void**)&x->oz_imgA, (void**)&x->oz_imgB, (void**)&x->oz_rs, (void**)&x->oz_cs};
  const size_t old_bytes[4] = {x->oz.a_bytes, x->oz.b_bytes, sizeof(double) * x->oz.rs_elems,
                               sizeof(double) * x->oz.cs_elems};
  for (int i = 0; i < 4; ++i) {
    void* p = *old[i];
    if (!p) continue;
    cudaFree(p);
    x->allocs.erase(std::find(x->allocs.begin(), x->allocs.end(), p));
    x->bytes -= old_bytes[i];
    *old[i] = nullptr;
  }
  x->oz_digits = 0;
  x->oz = oz_layout(d, h->int8_digits);
  auto al = [&](size_t bytes, void** p) -> int {
    int s = mcheck(h, cudaMalloc(p, bytes), "int8 slice images");
    if (s) return s;
    x->allocs.push_back(*p);
    x->bytes += bytes;
    return GD_OK;
  };
  int s = al(x->oz.a_bytes, (void**)&x->oz_imgA);
  if (!s) s = al(x->oz.b_bytes, (void**)&x->oz_imgB);
  if (!s) s = al(sizeof(double) * x->oz.rs_elems, (void**)&x->oz_rs);
  if (!s) s = al(sizeof(double) * x->oz.cs_elems, (void**)&x->oz_cs);
  if (s) return s;
  launch_oz_tables(h->stream, d, h->d_moff, h->d_dP, h->d_Q, x->oz, x->oz_imgA, x->oz_rs);
  s = launched(h, "int8 table images");
  if (s) return s;
  s = mcheck(h, cudaStreamSynchronize(h->stream), "int8 table images");
  if (s) return s;
  x->oz_digits = h->int8_digits;
  return GD_OK;
}

void mixed_destroy(gd_handle* h) {
  if (!h->mixed) return;
  for (void* p : h->mixed->allocs) cudaFree(p);
  delete h->mixed;
  h->mixed = nullptr;
}

size_t mixed_bytes(const gd_handle* h) { return h->mixed ? h->mixed->bytes : 0; }

int mixed_check_error(gd_handle* h) {
  if (!h->mixed) return GD_OK;
  int flag = 0;
  int s = mcheck(h, cudaMemcpyAsync(&flag, h->mixed->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "err");
  if (s) return s;
  s = mcheck(h, cudaStreamSynchronize(h->stream), "err sync");
  if (s) return s;
  if (flag) {
    // reported once: the flag is cleared so the handle's next calls run normally
    s = mcheck(h, cudaMemsetAsync(h->mixed->d_err, 0, sizeof(int), h->stream), "err reset");
    if (s) return s;
    return set_error(h, GD_ERR_CUDA, "a tensor-core pipeline wait expired (results of that call are invalid)");
  }
  return GD_OK;
}

int mixed_set_fault_test(gd_handle* h, long long wait_cycles, int omit_step) {
  if (!h->mixed) return set_error(h, GD_ERR_STATE, "the handle has no mixed-precision state");
  h->mixed->wait_limit = wait_cycles > 0 ? wait_cycles : 0;
  h->mixed->omit_plus1 = omit_step >= 0 ? omit_step + 1 : 0;
  return GD_OK;
}

int mixed_temperature_nl(gd_handle* h) {
  MixedState* x = h->mixed;
  const Dims& d = h->d;
  int s;
  if (h->ext_derivs) {
    // the gradient was computed elsewhere into the work arrays: the pre-pass
    // splits all four fields
    const double* coef[4] = {h->field(F_TEMP), h->work(0), h->work(1), h->work(2)};
    s = tc_synth_scalar(h, coef, 4, x->F(FC_T), 0xF);
  } else {
    // the gradient goes straight into the scalar synthesis image (field slots 1-3)
    { ProfScope p(h, "spectral_gradients");
      launch_gradients_img(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_TEMP), image_out(h, x->d_bimg_s)); }
    const double* coef[4] = {h->field(F_TEMP), nullptr, nullptr, nullptr};
    s = tc_synth_scalar(h, coef, 4, x->F(FC_T), 1);
  }
  if (s) return s;
  // the velocity grid is the previous velocity phase's (carried in F(FC_U));
  // the temperature grid itself is not a factor of the products: like every
  // synthesized grid of the mixed step it is formed on request from its
  // Fourier buffer F(FC_T) (mixed_grid_to_double)
  FusedArgs f = phase_args(h);
  const float4* fin[5] = {x->F(FC_GR), x->F(FC_U), x->F(FC_GTH), x->F(FC_U + 1), x->F(FC_GPH)};
  for (int i = 0; i < 5; ++i) f.fin[i] = fin[i];
  f.nin = 5;
  { ProfScope p(h, "fused_temperature_fp32"); launch_fused(h->stream, d, h->plan, h->d_twf, FUSED_TEMPERATURE, f); }
  s = launched(h, "fused temperature phase");
  if (s) return s;
  double* out[1] = {h->nlf(F_TEMP)};
  s = tc_analysis_scalar_G(h, 1, out);
  if (s) return s;
  regular_nl(h, F_TEMP, 1);
  if (!h->ext_derivs) scalar_bc(h, F_TEMP);
  return launched(h, "mixed temperature nonlinear");
}

// The composition phase (compute_composition_nonlinear!, src/compositional.jl:
// 219-259): gradient (FP64, into work 8-10, unless received), split-TF32
// synthesis of C and its gradient, the fused advection -u.grad C + S_C(r) with
// the velocity components of this step's velocity phase (step_once! computes
// composition after velocity), the analysis, then the boundary conditions.
int mixed_composition_nl(gd_handle* h) {
  MixedState* x = h->mixed;
  const Dims& d = h->d;
  if (!h->ext_derivs) {
    ProfScope p(h, "spectral_gradients");
    launch_gradients(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_d1, h->field(F_COMP), h->work(8), h->work(9),
                     h->work(10));
  }
  const double* coef[4] = {h->field(F_COMP), h->work(8), h->work(9), h->work(10)};
  int s = tc_synth_scalar(h, coef, 4, x->F(FC_C), 0xF);
  if (s) return s;
  FusedArgs f = phase_args(h);
  f.sources = h->d_csources;
  const float4* fin[5] = {x->F(FC_C + 3), x->F(FC_U), x->F(FC_C + 1), x->F(FC_U + 1), x->F(FC_C + 2)};
  for (int i = 0; i < 5; ++i) f.fin[i] = fin[i];
  f.nin = 5;
  { ProfScope p(h, "fused_composition_fp32"); launch_fused(h->stream, d, h->plan, h->d_twf, FUSED_TEMPERATURE, f); }
  s = launched(h, "fused composition phase");
  if (s) return s;
  double* out[1] = {h->nlf(F_COMP)};
  s = tc_analysis_scalar_G(h, 1, out);
  if (s) return s;
  regular_nl(h, F_COMP, 1);
  if (!h->ext_derivs) scalar_bc(h, F_COMP);
  return launched(h, "mixed composition nonlinear");
}

// The velocity phase.  The stages of h->fp64_stages run in FP64 with the FP64
// path's kernels: GD_STAGE_VEL_SYNTH the vector synthesis of u (DMMA
// Legendre; its FP32 copy for the fused kernels is converted from the FP64
// result), GD_STAGE_VEL_PRODUCTS the phi transforms of u and the Coriolis
// product (the FP32 fused kernel then forms the cross products only, whose
// theta and phi components are exact zeros with zero radial components, and
// its folded transforms are added to the FP64 ones), GD_STAGE_VEL_ANALYSIS
// the vector analysis (DMMA Legendre).  With all three the velocity nonlinear
// term is the FP64 step's, so u and the kinetic energy follow the FP64 run.
int mixed_velocity_nl(gd_handle* h) {
  MixedState* x = h->mixed;
  const Dims& d = h->d;
  const int st = h->fp64_stages;
  const size_t fc64 = fourier64_comp(d);
  double2* U64 = h->d_F;             // u_theta, u_phi Fourier (FP64 synthesis layout)
  double2* G64 = h->d_F + 2 * fc64;  // folded transforms of the velocity products (FP64)
  const size_t nfold = 2 * fc64;     // double2 of the two folded components
  int s;
  if (st & GD_STAGE_VEL_SYNTH_I8) {
    if (x->oz_digits != h->int8_digits || !x->oz_imgA)
      return set_error(h, GD_ERR_STATE, "the int8 slice images are not built (set-up failed)");
    OzSynthArgs a{};
    a.out = U64;
    a.out32 = x->F(FC_U);  // the FP32 copy the fused phase kernels read
    a.out32_comp = x->fcomp;
    a.err = x->d_err;
    a.wait_limit = x->wait_limit;
    a.omit_plus1 = x->omit_plus1;
    a.max_ctas = h->tc_ctas;
    x->omit_plus1 = 0;  // one-shot
    { ProfScope p(h, "legendre_synth_vector_i8");
      launch_oz_synth_vector(h->stream, d, h->d_moff, x->oz, h->field(F_UPOL), h->field(F_UTOR), x->oz_imgA, x->oz_rs,
                             x->oz_imgB, x->oz_cs, a); }
    s = launched(h, "int8-slice velocity synthesis");
  } else if (st & GD_STAGE_VEL_SYNTH) {
    SynthArgs a{};
    a.table0 = h->d_dP;
    a.table1 = h->d_Q;
    a.coef[0] = h->field(F_UPOL);
    a.coef[1] = h->field(F_UTOR);
    a.nf = 1;
    a.out = U64;
    a.out32 = x->F(FC_U);  // the FP32 copy the fused phase kernels read
    a.out32_comp = x->fcomp;
    { ProfScope p(h, "legendre_synth_vector_fp64"); launch_synth_fp64(h->stream, d, h->d_moff, a, true); }
    s = launched(h, "FP64 velocity synthesis");
  } else {
    s = tc_synth_vector(h, h->field(F_UTOR), h->field(F_UPOL), x->F(FC_U));
    if (!s && (st & GD_STAGE_VEL_PRODUCTS)) {
      { ProfScope p(h, "fourier_convert"); launch_widen_fourier(h->stream, d, U64, x->F(FC_U), x->fcomp, 2); }
      s = launched(h, "velocity Fourier widening");
    }
  }
  if (s) return s;
  if (h->ext_derivs) {
    s = tc_synth_vector(h, h->work(3), h->work(4), x->F(FC_W));
  } else {
    { ProfScope p(h, "spectral_curl");
      launch_curl_img(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_UTOR),
                      h->field(F_UPOL), image_out(h, x->d_bimg_vc)); }
    s = tc_synth_vector(h, nullptr, nullptr, x->F(FC_W));
  }
  if (s) return s;
  // current density and magnetic field of the previous magnetic phase (F(FC_J), F(FC_B))
  FusedArgs f = phase_args(h);
  if (st & GD_STAGE_VEL_PRODUCTS) f.cf = 0.f;
  const float4* fin[8] = {x->F(FC_U), x->F(FC_U + 1), x->F(FC_W), x->F(FC_W + 1),
                          x->F(FC_J), x->F(FC_J + 1), x->F(FC_B), x->F(FC_B + 1)};
  for (int i = 0; i < 8; ++i) f.fin[i] = fin[i];
  f.nin = h->c.magnetic ? 8 : 4;
  { ProfScope p(h, "fused_velocity_fp32"); launch_fused(h->stream, d, h->plan, h->d_twf, FUSED_VELOCITY, f); }
  s = launched(h, "fused velocity phase");
  if (s) return s;
  bool fused = false;
  if (st & GD_STAGE_VEL_PRODUCTS) {
    const double rf = h->c.magnetic_prandtl / h->c.ekman;
    ProfScope p(h, "coriolis_fused_fp64");
    fused = launch_coriolis_fused(h->stream, d, d.nlon, h->d_tw, U64, h->d_cth, h->d_sthc, rf, h->d_w, x->d_G, G64);
  }
  if ((st & GD_STAGE_VEL_PRODUCTS) && !fused) {
    const double rf = h->c.magnetic_prandtl / h->c.ekman;
    { ProfScope p(h, "fft_synth_fp64");
      launch_fft_synth<double>(h->stream, d, h->plan, h->d_tw, U64, h->grid(GD_GRID_U_TH), 2, h->grid_elems()); }
    { ProfScope p(h, "nl_coriolis_fp64");
      launch_coriolis<double>(h->stream, d, h->d_cth, h->d_sthc, rf, h->grid(GD_GRID_U_TH), h->grid(GD_GRID_U_PH),
                              h->grid(GD_GRID_VADV_TH), h->grid(GD_GRID_VADV_PH)); }
    { ProfScope p(h, "fft_analysis_fp64");
      launch_fft_analysis<double>(h->stream, d, h->plan, h->d_tw, h->grid(GD_GRID_VADV_TH), h->grid_elems(), h->d_w,
                                  G64, 2); }
  }
  if ((st & (GD_STAGE_VEL_PRODUCTS | GD_STAGE_VEL_ANALYSIS)) && !fused) {
    // FP32 folded transforms of the fused kernel: added to the FP64 Coriolis
    // transforms, or widened for the FP64 analysis
    ProfScope p(h, "fold_convert");
    const int add = (st & GD_STAGE_VEL_PRODUCTS) ? 1 : 0;
    k_fold_widen<<<148 * 4, 256, 0, h->stream>>>(nfold, x->d_G, G64, add);
  }
  s = launched(h, "FP64 velocity products");
  if (s) return s;
  if (st & GD_STAGE_VEL_ANALYSIS) {
    AnalysisArgs a{};
    a.table0 = h->d_dP;
    a.table1 = h->d_Q;
    a.in = G64;
    a.out[0] = h->nlf(F_UTOR);
    a.out[1] = h->nlf(F_UPOL);
    a.nf = 1;
    a.epi = EPI_VECTOR;
    { ProfScope p(h, "legendre_analysis_vector_fp64"); launch_analysis_fp64(h->stream, d, h->d_moff, a); }
    return launched(h, "FP64 velocity analysis");
  }
  if (st & GD_STAGE_VEL_PRODUCTS) {
    ProfScope p(h, "fold_convert");
    k_fold_narrow<<<148 * 4, 256, 0, h->stream>>>(nfold, G64, x->d_G);
  }
  return tc_analysis_vector_G(h, h->nlf(F_UTOR), h->nlf(F_UPOL), EPI_VECTOR);
}

int mixed_magnetic_nl(gd_handle* h) {
  MixedState* x = h->mixed;
  const Dims& d = h->d;
  int s = tc_synth_vector(h, h->field(F_BTOR), h->field(F_BPOL), x->F(FC_B));
  if (s) return s;
  if (h->ext_derivs) {
    s = tc_synth_vector(h, h->work(5), h->work(6), x->F(FC_J));
  } else {
    { ProfScope p(h, "spectral_curl");
      launch_curl_img(h->stream, d, h->d_lof, h->d_mof, h->d_rinv, h->d_rinv2, h->d_d1, h->d_d2, h->field(F_BTOR),
                      h->field(F_BPOL), image_out(h, x->d_bimg_vc)); }
    s = tc_synth_vector(h, nullptr, nullptr, x->F(FC_J));
  }
  if (s) return s;
  FusedArgs f = phase_args(h);
  const float4* fin[4] = {x->F(FC_U), x->F(FC_U + 1), x->F(FC_B), x->F(FC_B + 1)};
  for (int i = 0; i < 4; ++i) f.fin[i] = fin[i];
  f.nin = 4;
  { ProfScope p(h, "fused_induction_fp32"); launch_fused(h->stream, d, h->plan, h->d_twf, FUSED_INDUCTION, f); }
  s = launched(h, "fused induction phase");
  if (s) return s;
  s = tc_analysis_vector_G(h, h->nlf(F_BTOR), h->nlf(F_BPOL), EPI_CURL_INDUCTION);
  if (s) return s;
  regular_nl(h, F_BTOR, 2);
  return launched(h, "ball regularity");
}

// Grid download in the mixed path: synthesized components are transformed
// from their Fourier buffers on request; the products' grids exist only
// inside the fused kernels.
int mixed_grid_to_double(gd_handle* h, int grid, double* out) {
  MixedState* x = h->mixed;
  const float* src = nullptr;
  int fc = -1;
  switch (grid) {
    case GD_GRID_U_TH: fc = FC_U; break;
    case GD_GRID_U_PH: fc = FC_U + 1; break;
    case GD_GRID_W_TH: fc = FC_W; break;
    case GD_GRID_W_PH: fc = FC_W + 1; break;
    case GD_GRID_B_TH: fc = FC_B; break;
    case GD_GRID_B_PH: fc = FC_B + 1; break;
    case GD_GRID_J_TH: fc = FC_J; break;
    case GD_GRID_J_PH: fc = FC_J + 1; break;
    case GD_GRID_GTH: fc = FC_GTH; break;
    case GD_GRID_GPH: fc = FC_GPH; break;
    case GD_GRID_GR: fc = FC_GR; break;
    case GD_GRID_T: fc = FC_T; break;
    case GD_GRID_C: fc = FC_C; break;
    case GD_GRID_CGTH: fc = FC_C + 1; break;
    case GD_GRID_CGPH: fc = FC_C + 2; break;
    case GD_GRID_CGR: fc = FC_C + 3; break;
    default:
      return set_error(h, GD_ERR_UNSUPPORTED,
                       "the mixed-precision step forms the nonlinear products in shared memory only; download "
                       "product grids with precision fp64");
  }
  if (fc >= 0) {
    const float4* fin[1] = {x->F(fc)};
    int s = fourier_to_grid(h, fin, 1, x->d_stage);
    if (s) return s;
    src = x->d_stage;
  }
  launch_grid_cast<float>(h->stream, h->grid_elems(), src, out);
  return launched(h, "grid cast");
}

int mixed_api_synth_scalar(gd_handle* h, const double* const* coef, int nf, double* grid_out) {
  MixedState* x = h->mixed;
  int s = tc_synth_scalar(h, coef, nf, x->F(FC_T), (1 << nf) - 1);
  if (s) return s;
  const float4* fin[4] = {x->F(FC_T), x->F(FC_T + 1), x->F(FC_T + 2), x->F(FC_T + 3)};
  s = fourier_to_grid(h, fin, nf, x->d_stage);
  if (s) return s;
  launch_grid_cast<float>(h->stream, (size_t)nf * h->grid_elems(), x->d_stage, grid_out);
  s = launched(h, "cast");
  return s ? s : mixed_check_error(h);
}

// Uses the vorticity buffers, which no later phase reads.
int mixed_api_synth_vector(gd_handle* h, const double* tor, const double* pol, double* grid_out) {
  MixedState* x = h->mixed;
  int s = tc_synth_vector(h, tor, pol, x->F(FC_W));
  if (s) return s;
  const float4* fin[2] = {x->F(FC_W), x->F(FC_W + 1)};
  s = fourier_to_grid(h, fin, 2, x->d_stage);
  if (s) return s;
  launch_grid_cast<float>(h->stream, 2 * h->grid_elems(), x->d_stage, grid_out);
  s = launched(h, "cast");
  return s ? s : mixed_check_error(h);
}

int mixed_api_analysis_scalar(gd_handle* h, const double* grid_in, int nf, double* const* out) {
  // the folded-transform buffer d_G holds two components: at most two fields per pass
  for (int f0 = 0; f0 < nf; f0 += 2) {
    const int nc = nf - f0 < 2 ? nf - f0 : 2;
    launch_cast_d2f(h->stream, (size_t)nc * h->grid_elems(), grid_in + (size_t)f0 * h->grid_elems(),
                    h->mixed->d_stage);
    int s = tc_analysis_scalar(h, h->mixed->d_stage, nc, out + f0);
    if (s) return s;
  }
  return mixed_check_error(h);
}

int mixed_api_analysis_vector(gd_handle* h, const double* grid_in, double* tor, double* pol) {
  launch_cast_d2f(h->stream, 2 * h->grid_elems(), grid_in, h->mixed->d_stage);
  int s = tc_analysis_vector(h, h->mixed->d_stage, tor, pol, EPI_VECTOR);
  return s ? s : mixed_check_error(h);
}

__global__ void k_cast_d2f(size_t n, const double* __restrict__ src, float* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}
void launch_cast_d2f(cudaStream_t s, size_t n, const double* src, float* dst) {
  k_cast_d2f<<<148 * 8, 256, 0, s>>>(n, src, dst);
}

}  // namespace gd

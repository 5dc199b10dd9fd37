// gd_nonlinear.cu -- grid-space nonlinear products of the FP64 step, streamed
// over the native grid layout [r][theta][phi] (the mixed-precision step forms
// the same products inside its fused phase kernels, gd_fused.cu).  Each kernel
// is the fused loop of the cited
// reference function; the radial vector components are identically zero on
// this path because the reference's vector synthesis writes only theta/phi
// (src/shtnskit_field_functions.jl:264-279), and the expressions keep those
// zero factors so the arithmetic is the reference's.
#include "gd_internal.cuh"

namespace gd {

// compute_scalar_advection_local! + add_internal_sources_local!
// (src/scalar_field_common.jl:390-443): -(u . grad T) + S(r).
// Grid: blockIdx.y = shell, grid-stride over the shell's theta-phi plane.
template <typename R>
__global__ void k_temperature_advection(Dims d, const R* __restrict__ uth, const R* __restrict__ uph,
                                        const R* __restrict__ gth, const R* __restrict__ gph,
                                        const R* __restrict__ gr, const double* __restrict__ src, R* __restrict__ out) {
  const int plane = d.nlat * d.nlon;
  const size_t base = (size_t)blockIdx.y * plane;
  const double s = src[blockIdx.y];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += gridDim.x * blockDim.x) {
    const size_t i = base + q;
    const R ur = 0;
    R v = -(ur * gr[i] + uth[i] * gth[i] + uph[i] * gph[i]);
    if (s != 0.0) v += (R)s;
    out[i] = v;
  }
}

// compute_all_nonlinear_terms! + add_lorentz_force! (src/velocity.jl:447-548,
// 638-672), theta and phi components (the radial one is discarded by the
// vector analysis).  Coriolis uses the latitude of index min(phi index, nlat)
// exactly as the reference loop does (src/velocity.jl:492-496).
template <typename R>
__global__ void k_velocity_nl(Dims d, const double* __restrict__ cth, const double* __restrict__ sth, double rf,
                              double lf, int magnetic, const R* __restrict__ uth, const R* __restrict__ uph,
                              const R* __restrict__ wth, const R* __restrict__ wph, const R* __restrict__ jth,
                              const R* __restrict__ jph, const R* __restrict__ bth, const R* __restrict__ bph,
                              R* __restrict__ ath, R* __restrict__ aph) {
  const int plane = d.nlat * d.nlon;
  const size_t base = (size_t)blockIdx.y * plane;
  // per-shell factors when the handle's segments have their own Ekman numbers
  if (d.rfs) rf = lf = d.rfs[blockIdx.y];
  const R adv = (R)(-rf), mrf = (R)(-rf), lfr = (R)lf;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += gridDim.x * blockDim.x) {
    const size_t i = base + q;
    const int jphi = q % d.nlon;
    const int tidx = jphi < d.nlat - 1 ? jphi : d.nlat - 1;
    const R ct = (R)cth[tidx], st = (R)sth[tidx];
    const R ur = 0, wr = 0;
    const R u_t = uth[i], u_p = uph[i], w_t = wth[i], w_p = wph[i];
    R at = adv * (u_p * wr - ur * w_p);
    R ap = adv * (ur * w_t - u_t * wr);
    const R zt = -ct * u_p, zp = ct * u_t + st * ur;
    at += mrf * zt;
    ap += mrf * zp;
    if (magnetic) {
      const R jr = 0, br = 0;
      at += lfr * (jph[i] * br - jr * bph[i]);
      ap += lfr * (jr * bth[i] - jth[i] * br);
    }
    ath[i] = at;
    aph[i] = ap;
  }
}

// The Coriolis part of k_velocity_nl alone, with the same expressions: the
// mixed-precision step forms the cross products in FP32 in its fused kernel
// and, when its velocity stages run in FP64, this term here (with u_r = 0 the
// cross products contribute exact zeros to theta and phi, so the sum of the
// two equals k_velocity_nl's result).
template <typename R>
__global__ void k_coriolis(Dims d, const double* __restrict__ cth, const double* __restrict__ sth, double rf,
                           const R* __restrict__ uth, const R* __restrict__ uph, R* __restrict__ ath,
                           R* __restrict__ aph) {
  const int plane = d.nlat * d.nlon;
  const size_t base = (size_t)blockIdx.y * plane;
  if (d.rfs) rf = d.rfs[blockIdx.y];
  const R mrf = (R)(-rf);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += gridDim.x * blockDim.x) {
    const size_t i = base + q;
    const int jphi = q % d.nlon;
    const int tidx = jphi < d.nlat - 1 ? jphi : d.nlat - 1;
    const R ct = (R)cth[tidx], st = (R)sth[tidx];
    const R ur = 0;
    const R u_t = uth[i], u_p = uph[i];
    const R zt = -ct * u_p, zp = ct * u_t + st * ur;
    ath[i] = mrf * zt;
    aph[i] = mrf * zp;
  }
}

// compute_velocity_cross_magnetic! (src/magnetic.jl:375-404), theta/phi.
template <typename R>
__global__ void k_induction(Dims d, const R* __restrict__ uth, const R* __restrict__ uph, const R* __restrict__ bth,
                            const R* __restrict__ bph, R* __restrict__ oth, R* __restrict__ oph) {
  const int plane = d.nlat * d.nlon;
  const size_t base = (size_t)blockIdx.y * plane;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += gridDim.x * blockDim.x) {
    const size_t i = base + q;
    const R ur = 0, br = 0;
    oth[i] = uph[i] * br - ur * bph[i];
    oph[i] = ur * bth[i] - uth[i] * br;
  }
}

// blocks per shell: enough to cover ~4 elements per thread
static dim3 grid_blocks(const Dims& d) {
  const int plane = d.nlat * d.nlon;
  int bx = (plane + 1023) / 1024;
  if (bx < 1) bx = 1;
  return dim3(bx, d.nr);
}

template <typename R>
void launch_temperature_advection(cudaStream_t s, const Dims& d, const R* uth, const R* uph, const R* gth,
                                  const R* gph, const R* gr, const double* sources, R* out) {
  k_temperature_advection<R><<<grid_blocks(d), 256, 0, s>>>(d, uth, uph, gth, gph, gr, sources, out);
}
template <typename R>
void launch_velocity_nl(cudaStream_t s, const Dims& d, const double* cth, const double* sth_cor, double rf,
                        double lf, int magnetic, const R* uth, const R* uph, const R* wth, const R* wph,
                        const R* jth, const R* jph, const R* bth, const R* bph, R* ath, R* aph) {
  k_velocity_nl<R><<<grid_blocks(d), 256, 0, s>>>(d, cth, sth_cor, rf, lf, magnetic, uth, uph, wth, wph, jth, jph,
                                                   bth, bph, ath, aph);
}
template <typename R>
void launch_coriolis(cudaStream_t s, const Dims& d, const double* cth, const double* sth_cor, double rf, const R* uth,
                     const R* uph, R* ath, R* aph) {
  k_coriolis<R><<<grid_blocks(d), 256, 0, s>>>(d, cth, sth_cor, rf, uth, uph, ath, aph);
}
template <typename R>
void launch_induction(cudaStream_t s, const Dims& d, const R* uth, const R* uph, const R* bth, const R* bph,
                      R* oth, R* oph) {
  k_induction<R><<<grid_blocks(d), 256, 0, s>>>(d, uth, uph, bth, bph, oth, oph);
}

template void launch_temperature_advection<double>(cudaStream_t, const Dims&, const double*, const double*,
                                                   const double*, const double*, const double*, const double*,
                                                   double*);
template void launch_velocity_nl<double>(cudaStream_t, const Dims&, const double*, const double*, double, double, int,
                                         const double*, const double*, const double*, const double*, const double*,
                                         const double*, const double*, const double*, double*, double*);
template void launch_coriolis<double>(cudaStream_t, const Dims&, const double*, const double*, double, const double*,
                                      const double*, double*, double*);
template void launch_induction<double>(cudaStream_t, const Dims&, const double*, const double*, const double*,
                                       const double*, double*, double*);

}  // namespace gd

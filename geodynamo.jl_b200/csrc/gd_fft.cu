// gd_fft.cu -- phi-direction transforms (the FFTW part of SHTnsKit's
// synthesis/analysis, reached from src/shtnskit_field_functions.jl:118,234).
//
// Each CTA transforms `tb` north/south row pairs of one (component, shell):
// the two real rows are packed into one complex sequence (north = real part,
// south = imaginary part) and transformed with a shared-memory Stockham
// mixed-radix FFT that ping-pongs between two buffers (radix 16 passes for
// the power-of-two part, then 8/4/2, 3 and 5; nlon = 768 takes 16 x 16 x 3).
//
// Synthesis consumes the Legendre output F[comp][r][m][s][ith] and writes
// grid rows [comp][r][theta][phi].  Analysis writes the Gauss-weighted folds
// G_+ = w (G_N + G_S), G_- = w (G_N - G_S) with G = (2 pi / nlon) sum_j f e^{-i m phi_j}.
#include <cmath>

#include "gd_fft_core.cuh"
#include "gd_internal.cuh"

namespace gd {

template <typename RT>
__global__ void __launch_bounds__(256) k_fft_synth(Dims d, FftPlan p, const typename C2<RT>::T* __restrict__ tw,
                                                   const typename C2<RT>::T* __restrict__ F, RT* __restrict__ grid,
                                                   size_t grid_comp_stride) {
  typedef typename C2<RT>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = p.n, tb = p.tb, M = d.M;
  const int rs = prow(n);
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)tb * rs;
  const int i0 = blockIdx.x * tb;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(tb, d.nth - i0);
  // zero the band of unused frequencies M < k < n - M (and whole unused rows)
  const int band = n - 2 * M - 1;
  for (int e = threadIdx.x; e < tb * band; e += kThreads) {
    const int ii = e / band, k = M + 1 + (e - ii * band);
    bufA[(size_t)ii * rs + pidx(k)].x = 0; bufA[(size_t)ii * rs + pidx(k)].y = 0;
  }
  const size_t fbase = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * tb; e += kThreads) {
    const int m = e / tb, ii = e - m * tb;
    C* row = bufA + (size_t)ii * rs;
    C fn, fs;
    if (ii < rows) {
      fn = F[fbase + ((size_t)m * 2 + 0) * d.nth + i0 + ii];
      fs = F[fbase + ((size_t)m * 2 + 1) * d.nth + i0 + ii];
    } else {
      fn.x = fn.y = fs.x = fs.y = 0;
    }
    // Z_m = F_N + i F_S, Z_{n-m} = conj(F_N) + i conj(F_S); stored conjugated
    // (the inverse transform is conj(FFT(conj(Z)))).
    if (m == 0) {
      C z; z.x = fn.x; z.y = -fs.x;
      row[0] = z;
    } else {
      C z; z.x = fn.x - fs.y; z.y = -(fn.y + fs.x);
      row[pidx(m)] = z;
      C zc; zc.x = fn.x + fs.y; zc.y = fn.y - fs.x;
      row[pidx(n - m)] = zc;
    }
  }
  __syncthreads();
  const C* res = fft_forward<RT>(bufA, bufB, tb, p, tw);
  RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * n;
  for (int e = threadIdx.x; e < rows * n; e += kThreads) {
    const int ii = e / n, j = e - ii * n;
    const C z = res[(size_t)ii * rs + pidx(j)];
    const int ith = i0 + ii;
    gbase[(size_t)ith * n + j] = z.x;
    gbase[(size_t)(d.nlat - 1 - ith) * n + j] = -z.y;
  }
}

template <typename RT>
__global__ void __launch_bounds__(256) k_fft_analysis(Dims d, FftPlan p, const typename C2<RT>::T* __restrict__ tw,
                                                      const RT* __restrict__ grid, size_t grid_comp_stride,
                                                      const double* __restrict__ w, typename C2<RT>::T* __restrict__ G) {
  typedef typename C2<RT>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = p.n, tb = p.tb, M = d.M;
  const int rs = prow(n);
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)tb * rs;
  const int i0 = blockIdx.x * tb;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(tb, d.nth - i0);
  const RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * n;
  for (int e = threadIdx.x; e < tb * n; e += kThreads) {
    const int ii = e / n, j = e - ii * n;
    C z; z.x = 0; z.y = 0;
    if (ii < rows) {
      const int ith = i0 + ii;
      z.x = gbase[(size_t)ith * n + j];
      z.y = gbase[(size_t)(d.nlat - 1 - ith) * n + j];
    }
    bufA[(size_t)ii * rs + pidx(j)] = z;
  }
  __syncthreads();
  const C* res = fft_forward<RT>(bufA, bufB, tb, p, tw);
  const RT sc = (RT)(2.0 * 3.14159265358979323846 / n);
  const size_t gb = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * rows; e += kThreads) {
    const int m = e / rows, ii = e - m * rows;
    const int ith = i0 + ii;
    const C* row = res + (size_t)ii * rs;
    const C zk = row[pidx(m)];
    C zn = row[pidx((n - m) % n)];
    zn.y = -zn.y;
    C X, Y;
    X.x = (RT)0.5 * (zk.x + zn.x); X.y = (RT)0.5 * (zk.y + zn.y);
    Y.x = (RT)0.5 * (zk.y - zn.y); Y.y = (RT)-0.5 * (zk.x - zn.x);  // -i/2 (zk - zn)
    C gn, gs;
    gn.x = sc * X.x; gn.y = sc * X.y;
    gs.x = sc * Y.x; gs.y = sc * Y.y;
    const RT wi = (RT)w[ith];
    C gp, gm;
    gp.x = wi * (gn.x + gs.x); gp.y = wi * (gn.y + gs.y);
    gm.x = wi * (gn.x - gs.x); gm.y = wi * (gn.y - gs.y);
    G[gb + ((size_t)m * 2 + 0) * d.nth + ith] = gp;
    G[gb + ((size_t)m * 2 + 1) * d.nth + ith] = gm;
  }
}

template <typename RT, int N>
__global__ void __launch_bounds__(256) k_fft_synth_ct(Dims d, const typename C2<RT>::T* __restrict__ tw,
                                                      const typename C2<RT>::T* __restrict__ F, RT* __restrict__ grid,
                                                      size_t grid_comp_stride) {
  typedef typename C2<RT>::T C;
  constexpr int RS = CtGeom<RT, N>::RS, TB = CtGeom<RT, N>::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + TB * RS;
  const int M = d.M;
  const int i0 = blockIdx.x * TB;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(TB, d.nth - i0);
  for (int e = threadIdx.x; e < TB * N; e += kThreads) {
    const int ii = e / N, k = e - ii * N;
    if (k > M && k < N - M) { bufA[ii * RS + pidx(k)].x = 0; bufA[ii * RS + pidx(k)].y = 0; }
  }
  const size_t fbase = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth + i0;
  for (int e = threadIdx.x; e < (M + 1) * TB; e += kThreads) {
    const int m = e / TB, ii = e - m * TB;
    C* row = bufA + ii * RS;
    C fn, fs;
    if (ii < rows) {
      fn = F[fbase + ((size_t)m * 2 + 0) * d.nth + ii];
      fs = F[fbase + ((size_t)m * 2 + 1) * d.nth + ii];
    } else {
      fn.x = fn.y = fs.x = fs.y = 0;
    }
    if (m == 0) {
      C z; z.x = fn.x; z.y = -fs.x;
      row[0] = z;
    } else {
      C z; z.x = fn.x - fs.y; z.y = -(fn.y + fs.x);
      row[pidx(m)] = z;
      C zc; zc.x = fn.x + fs.y; zc.y = fn.y - fs.x;
      row[pidx(N - m)] = zc;
    }
  }
  __syncthreads();
  const C* res = ct_passes<N, TB, 0, 1, C>(bufA, bufB, tw);
  RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * N;
  for (int e = threadIdx.x; e < rows * N; e += kThreads) {
    const int ii = e / N, j = e - ii * N;
    const C z = res[ii * RS + pidx(j)];
    const int ith = i0 + ii;
    gbase[(size_t)ith * N + j] = z.x;
    gbase[(size_t)(d.nlat - 1 - ith) * N + j] = -z.y;
  }
}

template <typename RT, int N>
__global__ void __launch_bounds__(256) k_fft_analysis_ct(Dims d, const typename C2<RT>::T* __restrict__ tw,
                                                         const RT* __restrict__ grid, size_t grid_comp_stride,
                                                         const double* __restrict__ w,
                                                         typename C2<RT>::T* __restrict__ G) {
  typedef typename C2<RT>::T C;
  constexpr int RS = CtGeom<RT, N>::RS, TB = CtGeom<RT, N>::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + TB * RS;
  const int M = d.M;
  const int i0 = blockIdx.x * TB;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(TB, d.nth - i0);
  const RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * N;
  for (int e = threadIdx.x; e < TB * N; e += kThreads) {
    const int ii = e / N, j = e - ii * N;
    C z; z.x = 0; z.y = 0;
    if (ii < rows) {
      const int ith = i0 + ii;
      z.x = gbase[(size_t)ith * N + j];
      z.y = gbase[(size_t)(d.nlat - 1 - ith) * N + j];
    }
    bufA[ii * RS + pidx(j)] = z;
  }
  __syncthreads();
  const C* res = ct_passes<N, TB, 0, 1, C>(bufA, bufB, tw);
  const RT sc = (RT)(2.0 * 3.14159265358979323846 / N);
  const size_t gb = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * TB; e += kThreads) {
    const int m = e / TB, ii = e - m * TB;
    if (ii >= rows) continue;
    const int ith = i0 + ii;
    const C* row = res + ii * RS;
    const C zk = row[pidx(m)];
    C zn = row[pidx(m == 0 ? 0 : N - m)];
    zn.y = -zn.y;
    C X, Y;
    X.x = (RT)0.5 * (zk.x + zn.x); X.y = (RT)0.5 * (zk.y + zn.y);
    Y.x = (RT)0.5 * (zk.y - zn.y); Y.y = (RT)-0.5 * (zk.x - zn.x);
    C gn, gs;
    gn.x = sc * X.x; gn.y = sc * X.y;
    gs.x = sc * Y.x; gs.y = sc * Y.y;
    const RT wi = (RT)w[ith];
    C gp, gm;
    gp.x = wi * (gn.x + gs.x); gp.y = wi * (gn.y + gs.y);
    gm.x = wi * (gn.x - gs.x); gm.y = wi * (gn.y - gs.y);
    G[gb + ((size_t)m * 2 + 0) * d.nth + ith] = gp;
    G[gb + ((size_t)m * 2 + 1) * d.nth + ith] = gm;
  }
}

// The Coriolis term of the velocity phase in FP64, fused.  Per (shell, TB
// colatitude pairs, output component oc): the inverse phi transform of the
// velocity component the output multiplies (theta output: u_phi, phi output:
// u_theta; with u_r = 0 the Coriolis term of each component is one product),
// the product with the Coriolis factor of latitude index min(phi index,
// nlat - 1) (src/velocity.jl:492-496), the forward transform and the Gauss
// folds, plus the folds g32 of the FP32 cross products.  These are the
// operations of the unfused chain k_fft_synth_ct -> k_coriolis ->
// k_fft_analysis_ct -> widen-and-add, in the same order, so the result is the
// same to the last bit; the grids only stay in shared memory.
template <int N>
__global__ void __launch_bounds__(256) k_coriolis_fused(Dims d, const double2* __restrict__ tw,
                                                        const double2* __restrict__ F, const double* __restrict__ cth,
                                                        const double* __restrict__ sth, double rf,
                                                        const double* __restrict__ w, const float2* __restrict__ g32,
                                                        double2* __restrict__ G) {
  typedef double2 C;
  constexpr int RS = CtGeom<double, N>::RS, TB = CtGeom<double, N>::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + TB * RS;
  const int M = d.M;
  const int i0 = blockIdx.x * TB;
  const int r = blockIdx.y, oc = blockIdx.z, sc = 1 - oc;
  const int rows = min(TB, d.nth - i0);
  for (int e = threadIdx.x; e < TB * N; e += kThreads) {
    const int ii = e / N, k = e - ii * N;
    if (k > M && k < N - M) { bufA[ii * RS + pidx(k)].x = 0; bufA[ii * RS + pidx(k)].y = 0; }
  }
  const size_t fbase = ((size_t)(sc * d.nr + r) * (M + 1)) * 2 * d.nth + i0;
  for (int e = threadIdx.x; e < (M + 1) * TB; e += kThreads) {
    const int m = e / TB, ii = e - m * TB;
    C* row = bufA + ii * RS;
    C fn, fs;
    if (ii < rows) {
      fn = F[fbase + ((size_t)m * 2 + 0) * d.nth + ii];
      fs = F[fbase + ((size_t)m * 2 + 1) * d.nth + ii];
    } else {
      fn.x = fn.y = fs.x = fs.y = 0;
    }
    if (m == 0) {
      C z; z.x = fn.x; z.y = -fs.x;
      row[0] = z;
    } else {
      C z; z.x = fn.x - fs.y; z.y = -(fn.y + fs.x);
      row[pidx(m)] = z;
      C zc; zc.x = fn.x + fs.y; zc.y = fn.y - fs.x;
      row[pidx(N - m)] = zc;
    }
  }
  __syncthreads();
  C* res = ct_passes<N, TB, 0, 1, C>(bufA, bufB, tw);
  // grid rows: north z.x, south -z.y; the products packed as (north, south)
  const double mrf = -(d.rfs ? d.rfs[r] : rf);
  for (int e = threadIdx.x; e < TB * N; e += kThreads) {
    const int ii = e / N, j = e - ii * N;
    C* at = res + ii * RS + pidx(j);
    C z = *at, o;
    if (ii < rows) {
      const int tidx = j < d.nlat - 1 ? j : d.nlat - 1;
      const double ct = cth[tidx], st = sth[tidx];
      const double ur = 0;
      const double vN = z.x, vS = -z.y;
      if (oc == 0) {
        const double ztN = -ct * vN, ztS = -ct * vS;
        o.x = mrf * ztN; o.y = mrf * ztS;
      } else {
        const double zpN = ct * vN + st * ur, zpS = ct * vS + st * ur;
        o.x = mrf * zpN; o.y = mrf * zpS;
      }
    } else {
      o.x = 0; o.y = 0;
    }
    *at = o;
  }
  __syncthreads();
  C* out = ct_passes<N, TB, 0, 1, C>(res, res == bufA ? bufB : bufA, tw);
  const double scl = 2.0 * 3.14159265358979323846 / N;
  const size_t gb = ((size_t)(oc * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * TB; e += kThreads) {
    const int m = e / TB, ii = e - m * TB;
    if (ii >= rows) continue;
    const int ith = i0 + ii;
    const C* row = out + ii * RS;
    const C zk = row[pidx(m)];
    C zn = row[pidx(m == 0 ? 0 : N - m)];
    zn.y = -zn.y;
    C X, Y;
    X.x = 0.5 * (zk.x + zn.x); X.y = 0.5 * (zk.y + zn.y);
    Y.x = 0.5 * (zk.y - zn.y); Y.y = -0.5 * (zk.x - zn.x);
    C gn, gs;
    gn.x = scl * X.x; gn.y = scl * X.y;
    gs.x = scl * Y.x; gs.y = scl * Y.y;
    const double wi = w[ith];
    C gp, gm;
    gp.x = wi * (gn.x + gs.x); gp.y = wi * (gn.y + gs.y);
    gm.x = wi * (gn.x - gs.x); gm.y = wi * (gn.y - gs.y);
    const size_t ip = gb + ((size_t)m * 2 + 0) * d.nth + ith, im = gb + ((size_t)m * 2 + 1) * d.nth + ith;
    const float2 ap = g32[ip], am = g32[im];
    G[ip] = make_double2(gp.x + (double)ap.x, gp.y + (double)ap.y);
    G[im] = make_double2(gm.x + (double)am.x, gm.y + (double)am.y);
  }
}

template <int N>
static void launch_cor(cudaStream_t s, const Dims& d, const void* tw, const void* F, const double* cth,
                       const double* sth, double rf, const double* w, const float2* g32, void* G) {
  constexpr int RS = CtGeom<double, N>::RS, TB = CtGeom<double, N>::TB;
  const size_t sm = (size_t)2 * TB * RS * sizeof(double2);
  allow_dynamic_smem(k_coriolis_fused<N>, sm);
  dim3 g(ceil_div(d.nth, TB), d.nr, 2);
  k_coriolis_fused<N><<<g, kThreads, sm, s>>>(d, (const double2*)tw, (const double2*)F, cth, sth, rf, w, g32,
                                              (double2*)G);
}

bool launch_coriolis_fused(cudaStream_t s, const Dims& d, int nlon, const void* tw, const void* F, const double* cth,
                           const double* sth, double rf, const double* w, const float2* g32, void* G) {
  switch (nlon) {
    case 24: launch_cor<24>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 48: launch_cor<48>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 96: launch_cor<96>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 144: launch_cor<144>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 192: launch_cor<192>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 288: launch_cor<288>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 384: launch_cor<384>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    case 768: launch_cor<768>(s, d, tw, F, cth, sth, rf, w, g32, G); return true;
    default: return false;
  }
}

template <typename RT, int N>
static bool launch_ct(cudaStream_t s, const Dims& d, const void* tw, const void* F, RT* grid, size_t stride,
                      int ncomp, bool synth, const double* w) {
  typedef typename C2<RT>::T C;
  constexpr int RS = CtGeom<RT, N>::RS, TB = CtGeom<RT, N>::TB;
  const size_t sm = (size_t)2 * TB * RS * sizeof(C);
  allow_dynamic_smem(k_fft_synth_ct<RT, N>, 100 * 1024);
  allow_dynamic_smem(k_fft_analysis_ct<RT, N>, 100 * 1024);
  dim3 g(ceil_div(d.nth, TB), d.nr, ncomp);
  if (synth)
    k_fft_synth_ct<RT, N><<<g, kThreads, sm, s>>>(d, (const C*)tw, (const C*)F, grid, stride);
  else
    k_fft_analysis_ct<RT, N><<<g, kThreads, sm, s>>>(d, (const C*)tw, grid, stride, w, (C*)const_cast<void*>(F));
  return true;
}

// Dispatch to a compile-time length when there is one.
template <typename RT>
static bool launch_fixed(cudaStream_t s, const Dims& d, int n, const void* tw, const void* F, RT* grid,
                         size_t stride, int ncomp, bool synth, const double* w) {
  switch (n) {
    case 24: return launch_ct<RT, 24>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 40: return launch_ct<RT, 40>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 48: return launch_ct<RT, 48>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 96: return launch_ct<RT, 96>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 144: return launch_ct<RT, 144>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 192: return launch_ct<RT, 192>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 288: return launch_ct<RT, 288>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 384: return launch_ct<RT, 384>(s, d, tw, F, grid, stride, ncomp, synth, w);
    case 768: return launch_ct<RT, 768>(s, d, tw, F, grid, stride, ncomp, synth, w);
    default: return false;
  }
}

FftPlan make_fft_plan(int nlon) {
  FftPlan p{};
  p.n = nlon;
  int m = nlon, a = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  // powers of two in passes of 16, then one pass of 8, 4 or 2 (8 x 4 instead of 16 x 2)
  int rest = a;
  if (rest >= 5 && rest % 4 == 1) { p.radix[p.nstage++] = 8; p.radix[p.nstage++] = 4; rest -= 5; }
  while (rest >= 4) { p.radix[p.nstage++] = 16; rest -= 4; }
  if (rest == 3) p.radix[p.nstage++] = 8;
  if (rest == 2) p.radix[p.nstage++] = 4;
  if (rest == 1) p.radix[p.nstage++] = 2;
  while (m % 3 == 0) { p.radix[p.nstage++] = 3; m /= 3; }
  while (m % 5 == 0) { p.radix[p.nstage++] = 5; m /= 5; }
  if (m != 1) p.nstage = -1;  // unsupported prime factor
  return p;
}

void make_twiddles(int n, std::vector<double>& tw) {
  tw.resize(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * 3.14159265358979323846 * k / n;
    tw[2 * k] = std::cos(a);
    tw[2 * k + 1] = std::sin(a);
  }
}

template <typename RT>
static int pick_tb(const Dims& d, int n) {
  // two [tb][n] complex buffers within ~56 KB (four CTAs per SM)
  int tb = (int)((56 * 1024) / (2 * (size_t)prow(n) * sizeof(typename C2<RT>::T)));
  if (tb > 16) tb = 16;
  if (tb > d.nth) tb = d.nth;
  if (tb < 1) tb = 1;
  return tb;
}

template <typename RT>
void launch_fft_synth(cudaStream_t s, const Dims& d, const FftPlan& p0, const void* twiddle, const void* F,
                      RT* grid, int ncomp, size_t grid_comp_stride) {
  typedef typename C2<RT>::T C;
  if (launch_fixed<RT>(s, d, p0.n, twiddle, F, grid, grid_comp_stride, ncomp, true, nullptr)) return;
  FftPlan p = p0;
  p.tb = pick_tb<RT>(d, p.n);
  const size_t sm = (size_t)2 * p.tb * prow(p.n) * sizeof(C);
  allow_dynamic_smem(k_fft_synth<RT>, 200 * 1024);
  dim3 grid_dim(ceil_div(d.nth, p.tb), d.nr, ncomp);
  k_fft_synth<RT><<<grid_dim, kThreads, sm, s>>>(d, p, (const C*)twiddle, (const C*)F, grid, grid_comp_stride);
}

template <typename RT>
void launch_fft_analysis(cudaStream_t s, const Dims& d, const FftPlan& p0, const void* twiddle, const RT* grid,
                         size_t grid_comp_stride, const double* w, void* G, int ncomp) {
  typedef typename C2<RT>::T C;
  if (launch_fixed<RT>(s, d, p0.n, twiddle, G, const_cast<RT*>(grid), grid_comp_stride, ncomp, false, w)) return;
  FftPlan p = p0;
  p.tb = pick_tb<RT>(d, p.n);
  const size_t sm = (size_t)2 * p.tb * prow(p.n) * sizeof(C);
  allow_dynamic_smem(k_fft_analysis<RT>, 200 * 1024);
  dim3 grid_dim(ceil_div(d.nth, p.tb), d.nr, ncomp);
  k_fft_analysis<RT><<<grid_dim, kThreads, sm, s>>>(d, p, (const C*)twiddle, grid, grid_comp_stride, w, (C*)G);
}

template void launch_fft_synth<double>(cudaStream_t, const Dims&, const FftPlan&, const void*, const void*, double*,
                                       int, size_t);
template void launch_fft_analysis<double>(cudaStream_t, const Dims&, const FftPlan&, const void*, const double*,
                                          size_t, const double*, void*, int);
template void launch_fft_analysis<float>(cudaStream_t, const Dims&, const FftPlan&, const void*, const float*,
                                         size_t, const double*, void*, int);

}  // namespace gd

// gd_fft.cu -- phi-direction transforms (the FFTW part of SHTnsKit's
// synthesis/analysis, reached from src/shtnskit_field_functions.jl:118,234).
//
// Each CTA transforms `tb` north/south row pairs of one (component, shell):
// the two real rows are packed into one complex sequence (north = real part,
// south = imaginary part) and transformed with a shared-memory Stockham
// mixed-radix FFT (radices 4, 2, 3, 5).  Every stage reads its butterflies
// into registers, synchronises, and writes them back in place.
//
// Synthesis consumes the Legendre output F[comp][r][m][s][ith] and writes
// grid rows [comp][r][theta][phi].  Analysis writes the Gauss-weighted folds
// G_+ = w (G_N + G_S), G_- = w (G_N - G_S) with G = (2 pi / nlon) sum_j f e^{-i m phi_j}.
#include <cmath>

#include "gd_internal.cuh"

namespace gd {

template <typename R> struct C2;
template <> struct C2<double> { typedef double2 T; };
template <> struct C2<float> { typedef float2 T; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }

static const int kThreads = 256;
// Complex elements each thread keeps in registers during a stage.
template <typename R> struct Emax;
template <> struct Emax<double> { static const int v = 24; };
template <> struct Emax<float> { static const int v = 48; };

template <int R, typename C>
__device__ __forceinline__ void dft(C* v) {
  typedef decltype(v[0].x) S;
  if (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]);
    const C d = csub(v[1], v[3]);
    C t3; t3.x = d.y; t3.y = -d.x;  // -i * d
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  } else if (R == 3) {
    const S h = (S)0.86602540378443864676;
    const C a0 = v[0], s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    C m; m.x = a0.x - (S)0.5 * s.x; m.y = a0.y - (S)0.5 * s.y;
    v[0] = cadd(a0, s);
    v[1].x = m.x + h * d.y; v[1].y = m.y - h * d.x;
    v[2].x = m.x - h * d.y; v[2].y = m.y + h * d.x;
  } else if (R == 5) {
    const S c1 = (S)0.30901699437494742410, c2 = (S)-0.80901699437494742410;
    const S s1 = (S)0.95105651629515357212, s2 = (S)0.58778525229247312917;
    const C a0 = v[0];
    const C p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    const C p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    v[0].x = a0.x + p1.x + p2.x; v[0].y = a0.y + p1.y + p2.y;
    C r1, r2, i1, i2;
    r1.x = a0.x + c1 * p1.x + c2 * p2.x; r1.y = a0.y + c1 * p1.y + c2 * p2.y;
    r2.x = a0.x + c2 * p1.x + c1 * p2.x; r2.y = a0.y + c2 * p1.y + c1 * p2.y;
    // forward: -i (s1 m1 + s2 m2), -i (s2 m1 - s1 m2)
    i1.x = s1 * m1.y + s2 * m2.y; i1.y = -(s1 * m1.x + s2 * m2.x);
    i2.x = s2 * m1.y - s1 * m2.y; i2.y = -(s2 * m1.x - s1 * m2.x);
    v[1] = cadd(r1, i1); v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2); v[3] = csub(r2, i2);
  }
}

// One Stockham stage over all rows of `buf` ([tb][n]).
template <int R, typename RT>
__device__ void fft_stage(typename C2<RT>::T* buf, int tb, int n, int Ns, const typename C2<RT>::T* tw) {
  typedef typename C2<RT>::T C;
  constexpr int MAXB = (Emax<RT>::v + R - 1) / R;
  const int nbf = n / R;
  const int total = tb * nbf;
  const int twstep = n / (Ns * R);
  C v[MAXB][R];
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    const int b = threadIdx.x + i * kThreads;
    if (b < total) {
      const int row = b / nbf, j = b - row * nbf;
      const int k = j % Ns;
      const C* src = buf + (size_t)row * n + j;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        C x = src[r * nbf];
        if (r > 0 && k > 0) x = cmul(x, tw[(r * k * twstep) % n]);
        v[i][r] = x;
      }
      dft<R>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MAXB; ++i) {
    const int b = threadIdx.x + i * kThreads;
    if (b < total) {
      const int row = b / nbf, j = b - row * nbf;
      const int k = j % Ns;
      const int idxD = (j / Ns) * Ns * R + k;
      C* dst = buf + (size_t)row * n + idxD;
#pragma unroll
      for (int r = 0; r < R; ++r) dst[r * Ns] = v[i][r];
    }
  }
  __syncthreads();
}

template <typename RT>
__device__ void fft_forward(typename C2<RT>::T* buf, int tb, const FftPlan& p, const typename C2<RT>::T* tw) {
  int Ns = 1;
  for (int s = 0; s < p.nstage; ++s) {
    const int R = p.radix[s];
    if (R == 4) fft_stage<4, RT>(buf, tb, p.n, Ns, tw);
    else if (R == 2) fft_stage<2, RT>(buf, tb, p.n, Ns, tw);
    else if (R == 3) fft_stage<3, RT>(buf, tb, p.n, Ns, tw);
    else fft_stage<5, RT>(buf, tb, p.n, Ns, tw);
    Ns *= R;
  }
}

template <typename RT>
__global__ void __launch_bounds__(256) k_fft_synth(Dims d, FftPlan p, const typename C2<RT>::T* __restrict__ twg,
                                                   const typename C2<RT>::T* __restrict__ F, RT* __restrict__ grid,
                                                   size_t grid_comp_stride) {
  typedef typename C2<RT>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf = tw + p.n;
  const int n = p.n, tb = p.tb, M = d.M;
  const int i0 = blockIdx.x * tb;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(tb, d.nth - i0);
  for (int k = threadIdx.x; k < n; k += kThreads) tw[k] = twg[k];
  for (int e = threadIdx.x; e < tb * n; e += kThreads) { buf[e].x = 0; buf[e].y = 0; }
  __syncthreads();
  const size_t fbase = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * rows; e += kThreads) {
    const int m = e / rows, ii = e - m * rows;
    const int ith = i0 + ii;
    const C fn = F[fbase + ((size_t)m * 2 + 0) * d.nth + ith];
    const C fs = F[fbase + ((size_t)m * 2 + 1) * d.nth + ith];
    C* row = buf + (size_t)ii * n;
    // Z_m = F_N + i F_S ; stored conjugated (inverse via conj(FFT(conj)))
    if (m == 0) {
      C z; z.x = fn.x; z.y = -fs.x;
      row[0] = z;
    } else {
      C z; z.x = fn.x - fs.y; z.y = -(fn.y + fs.x);
      row[m] = z;
      C zc; zc.x = fn.x + fs.y; zc.y = -(-fn.y + fs.x);
      row[n - m] = zc;
    }
  }
  __syncthreads();
  fft_forward<RT>(buf, tb, p, tw);
  RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * n;
  for (int e = threadIdx.x; e < rows * n; e += kThreads) {
    const int ii = e / n, j = e - ii * n;
    const C z = buf[(size_t)ii * n + j];
    const int ith = i0 + ii;
    gbase[(size_t)ith * n + j] = z.x;
    gbase[(size_t)(d.nlat - 1 - ith) * n + j] = -z.y;
  }
}

template <typename RT>
__global__ void __launch_bounds__(256) k_fft_analysis(Dims d, FftPlan p, const typename C2<RT>::T* __restrict__ twg,
                                                      const RT* __restrict__ grid, size_t grid_comp_stride,
                                                      const double* __restrict__ w, typename C2<RT>::T* __restrict__ G) {
  typedef typename C2<RT>::T C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf = tw + p.n;
  const int n = p.n, tb = p.tb, M = d.M;
  const int i0 = blockIdx.x * tb;
  const int r = blockIdx.y, comp = blockIdx.z;
  const int rows = min(tb, d.nth - i0);
  for (int k = threadIdx.x; k < n; k += kThreads) tw[k] = twg[k];
  const RT* gbase = grid + grid_comp_stride * comp + (size_t)r * d.nlat * n;
  for (int e = threadIdx.x; e < tb * n; e += kThreads) {
    const int ii = e / n, j = e - ii * n;
    C z; z.x = 0; z.y = 0;
    if (ii < rows) {
      const int ith = i0 + ii;
      z.x = gbase[(size_t)ith * n + j];
      z.y = gbase[(size_t)(d.nlat - 1 - ith) * n + j];
    }
    buf[e] = z;
  }
  __syncthreads();
  fft_forward<RT>(buf, tb, p, tw);
  const RT sc = (RT)(2.0 * 3.14159265358979323846 / n);
  const size_t gb = ((size_t)(comp * d.nr + r) * (M + 1)) * 2 * d.nth;
  for (int e = threadIdx.x; e < (M + 1) * rows; e += kThreads) {
    const int m = e / rows, ii = e - m * rows;
    const int ith = i0 + ii;
    const C* row = buf + (size_t)ii * n;
    const C zk = row[m];
    C zn = row[(n - m) % n];
    zn.y = -zn.y;
    C X, Y;
    X.x = (RT)0.5 * (zk.x + zn.x); X.y = (RT)0.5 * (zk.y + zn.y);
    // Y = -i/2 (zk - zn)
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

FftPlan make_fft_plan(int nlon) {
  FftPlan p{};
  p.n = nlon;
  int m = nlon;
  for (int rr : {4, 2, 3, 5}) {
    while (m % rr == 0) { p.radix[p.nstage++] = rr; m /= rr; }
  }
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
  const int by_regs = Emax<RT>::v * kThreads / n;
  const int by_smem = (int)((96 * 1024) / (n * sizeof(typename C2<RT>::T))) - 1;
  int tb = by_regs < by_smem ? by_regs : by_smem;
  if (tb > d.nth) tb = d.nth;
  if (tb < 1) tb = 1;
  return tb;
}

template <typename RT>
void launch_fft_synth(cudaStream_t s, const Dims& d, const FftPlan& p0, const void* twiddle, const void* F,
                      RT* grid, int ncomp, size_t grid_comp_stride) {
  typedef typename C2<RT>::T C;
  FftPlan p = p0;
  p.tb = pick_tb<RT>(d, p.n);
  const size_t sm = (size_t)(p.n + p.tb * p.n) * sizeof(C);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_fft_synth<RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  dim3 grid_dim(ceil_div(d.nth, p.tb), d.nr, ncomp);
  k_fft_synth<RT><<<grid_dim, kThreads, sm, s>>>(d, p, (const C*)twiddle, (const C*)F, grid, grid_comp_stride);
}

template <typename RT>
void launch_fft_analysis(cudaStream_t s, const Dims& d, const FftPlan& p0, const void* twiddle, const RT* grid,
                         size_t grid_comp_stride, const double* w, void* G, int ncomp) {
  typedef typename C2<RT>::T C;
  FftPlan p = p0;
  p.tb = pick_tb<RT>(d, p.n);
  const size_t sm = (size_t)(p.n + p.tb * p.n) * sizeof(C);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_fft_analysis<RT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  dim3 grid_dim(ceil_div(d.nth, p.tb), d.nr, ncomp);
  k_fft_analysis<RT><<<grid_dim, kThreads, sm, s>>>(d, p, (const C*)twiddle, grid, grid_comp_stride, w, (C*)G);
}

template void launch_fft_synth<double>(cudaStream_t, const Dims&, const FftPlan&, const void*, const void*, double*,
                                       int, size_t);
template void launch_fft_synth<float>(cudaStream_t, const Dims&, const FftPlan&, const void*, const void*, float*,
                                      int, size_t);
template void launch_fft_analysis<double>(cudaStream_t, const Dims&, const FftPlan&, const void*, const double*,
                                          size_t, const double*, void*, int);
template void launch_fft_analysis<float>(cudaStream_t, const Dims&, const FftPlan&, const void*, const float*,
                                         size_t, const double*, void*, int);

}  // namespace gd

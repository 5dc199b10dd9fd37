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

// Forward DFT of R points in registers, natural order in and out.
template <typename C> __device__ __forceinline__ C mul_mi(C a) { C r; r.x = a.y; r.y = -a.x; return r; }  // -i a

template <int R, typename C> struct Dft;

template <typename C> struct Dft<2, C> {
  static __device__ __forceinline__ void run(C* v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <typename C> struct Dft<4, C> {
  static __device__ __forceinline__ void run(C* v) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]);
    const C t3 = mul_mi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};
template <typename C> struct Dft<3, C> {
  static __device__ __forceinline__ void run(C* v) {
    typedef decltype(v[0].x) S;
    const S h = (S)0.86602540378443864676;
    const C a0 = v[0], s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    C m; m.x = a0.x - (S)0.5 * s.x; m.y = a0.y - (S)0.5 * s.y;
    v[0] = cadd(a0, s);
    v[1].x = m.x + h * d.y; v[1].y = m.y - h * d.x;
    v[2].x = m.x - h * d.y; v[2].y = m.y + h * d.x;
  }
};
template <typename C> struct Dft<5, C> {
  static __device__ __forceinline__ void run(C* v) {
    typedef decltype(v[0].x) S;
    const S c1 = (S)0.30901699437494742410, c2 = (S)-0.80901699437494742410;
    const S s1 = (S)0.95105651629515357212, s2 = (S)0.58778525229247312917;
    const C a0 = v[0];
    const C p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    const C p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    v[0].x = a0.x + p1.x + p2.x; v[0].y = a0.y + p1.y + p2.y;
    C r1, r2, i1, i2;
    r1.x = a0.x + c1 * p1.x + c2 * p2.x; r1.y = a0.y + c1 * p1.y + c2 * p2.y;
    r2.x = a0.x + c2 * p1.x + c1 * p2.x; r2.y = a0.y + c2 * p1.y + c1 * p2.y;
    i1.x = s1 * m1.y + s2 * m2.y; i1.y = -(s1 * m1.x + s2 * m2.x);
    i2.x = s2 * m1.y - s1 * m2.y; i2.y = -(s2 * m1.x - s1 * m2.x);
    v[1] = cadd(r1, i1); v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2); v[3] = csub(r2, i2);
  }
};
// Radix 8 and 16 by one decimation-in-frequency split into two half-size DFTs:
//   u_n = x_n + x_{n+R/2},  v_n = (x_n - x_{n+R/2}) W_R^n,
//   X_{2k} = DFT(u)_k,  X_{2k+1} = DFT(v)_k.
template <typename C> struct Dft<8, C> {
  static __device__ __forceinline__ void run(C* x) {
    typedef decltype(x[0].x) S;
    const S c = (S)0.70710678118654752440;
    C u[4], w[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) { u[n] = cadd(x[n], x[n + 4]); w[n] = csub(x[n], x[n + 4]); }
    // W8^1 = c (1 - i), W8^2 = -i, W8^3 = -c (1 + i)
    { C t = w[1]; w[1].x = c * (t.x + t.y); w[1].y = c * (t.y - t.x); }
    w[2] = mul_mi(w[2]);
    { C t = w[3]; w[3].x = c * (t.y - t.x); w[3].y = -c * (t.x + t.y); }
    Dft<4, C>::run(u);
    Dft<4, C>::run(w);
#pragma unroll
    for (int k = 0; k < 4; ++k) { x[2 * k] = u[k]; x[2 * k + 1] = w[k]; }
  }
};
template <typename C> struct Dft<16, C> {
  static __device__ __forceinline__ void run(C* x) {
    typedef decltype(x[0].x) S;
    // W16^n = cos(pi n / 8) - i sin(pi n / 8), n = 0..7
    const S cs[8] = {(S)1.0, (S)0.92387953251128675613, (S)0.70710678118654752440, (S)0.38268343236508977173,
                     (S)0.0, (S)-0.38268343236508977173, (S)-0.70710678118654752440, (S)-0.92387953251128675613};
    const S sn[8] = {(S)0.0, (S)0.38268343236508977173, (S)0.70710678118654752440, (S)0.92387953251128675613,
                     (S)1.0, (S)0.92387953251128675613, (S)0.70710678118654752440, (S)0.38268343236508977173};
    C u[8], w[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      u[n] = cadd(x[n], x[n + 8]);
      const C d = csub(x[n], x[n + 8]);
      w[n].x = d.x * cs[n] + d.y * sn[n];
      w[n].y = d.y * cs[n] - d.x * sn[n];
    }
    Dft<8, C>::run(u);
    Dft<8, C>::run(w);
#pragma unroll
    for (int k = 0; k < 8; ++k) { x[2 * k] = u[k]; x[2 * k + 1] = w[k]; }
  }
};

// Shared-memory rows are padded by one element every 16 so the stride-16
// stores of the first radix-16 pass do not all fall into one bank.
// Rows are further padded to an odd number of elements so the transposed
// (m, row) accesses of the load and store phases spread over the banks.
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }
__host__ __device__ __forceinline__ int prow(int n) { return (n + (n >> 4)) | 1; }

// One Stockham pass from src to dst ([tb][n] each): radix R, Ns = product of
// the radices of the earlier passes.
template <int R, typename C>
__device__ __forceinline__ void fft_pass(const C* __restrict__ src, C* __restrict__ dst, int tb, int n, int Ns,
                                         const C* __restrict__ tw) {
  const int nbf = n / R;
  const int total = tb * nbf;
  const int twstep = n / (Ns * R);
  for (int b = threadIdx.x; b < total; b += kThreads) {
    const int row = b / nbf, j = b - row * nbf;
    const int k = j % Ns;
    const C* s = src + (size_t)row * prow(n);
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[pidx(j + r * nbf)];
    if (k > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(&tw[r * k * twstep]));
    }
    Dft<R, C>::run(v);
    C* o = dst + (size_t)row * prow(n);
    const int o0 = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) o[pidx(o0 + r * Ns)] = v[r];
  }
}

// Runs all passes; returns the buffer holding the result.
template <typename RT>
__device__ typename C2<RT>::T* fft_forward(typename C2<RT>::T* a, typename C2<RT>::T* b, int tb, const FftPlan& p,
                                           const typename C2<RT>::T* tw) {
  typedef typename C2<RT>::T C;
  int Ns = 1;
  C* src = a;
  C* dst = b;
  for (int s = 0; s < p.nstage; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 16: fft_pass<16, C>(src, dst, tb, p.n, Ns, tw); break;
      case 8: fft_pass<8, C>(src, dst, tb, p.n, Ns, tw); break;
      case 4: fft_pass<4, C>(src, dst, tb, p.n, Ns, tw); break;
      case 2: fft_pass<2, C>(src, dst, tb, p.n, Ns, tw); break;
      case 3: fft_pass<3, C>(src, dst, tb, p.n, Ns, tw); break;
      default: fft_pass<5, C>(src, dst, tb, p.n, Ns, tw); break;
    }
    __syncthreads();
    Ns *= R;
    C* t = src; src = dst; dst = t;
  }
  return src;
}

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

// ---------------------------------------------------------------------------
// Compile-time variants for the transform lengths in use: every index
// division below is by a constant (the runtime-plan kernels above spend most
// of their instructions in integer division).
// ---------------------------------------------------------------------------
struct CPlan {
  int n, ns;
  int r[12];
};
constexpr CPlan make_cplan(int n) {
  CPlan p{n, 0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
  int m = n, a = 0;
  while (m % 2 == 0) { m /= 2; ++a; }
  int rest = a;
  if (rest >= 5 && rest % 4 == 1) { p.r[p.ns++] = 8; p.r[p.ns++] = 4; rest -= 5; }
  while (rest >= 4) { p.r[p.ns++] = 16; rest -= 4; }
  if (rest == 3) p.r[p.ns++] = 8;
  if (rest == 2) p.r[p.ns++] = 4;
  if (rest == 1) p.r[p.ns++] = 2;
  while (m % 3 == 0) { p.r[p.ns++] = 3; m /= 3; }
  while (m % 5 == 0) { p.r[p.ns++] = 5; m /= 5; }
  return p;
}
template <int N> struct PlanOf { static constexpr CPlan p = make_cplan(N); };

template <typename RT, int N> struct CtGeom {
  typedef typename C2<RT>::T C;
  static constexpr int RS = (N + (N >> 4)) | 1;  // padded row stride (elements)
  static constexpr int TB0 = (int)((56 * 1024) / (2 * (size_t)RS * sizeof(C)));
  static constexpr int TB = TB0 > 16 ? 16 : (TB0 < 1 ? 1 : TB0);
};

template <int R, int N, int TB, int NS, typename C>
__device__ __forceinline__ void ct_pass(const C* __restrict__ src, C* __restrict__ dst, const C* __restrict__ tw) {
  constexpr int RS = (N + (N >> 4)) | 1;
  constexpr int NBF = N / R;
  constexpr int TOTAL = TB * NBF;
  constexpr int TWSTEP = N / (NS * R);
  for (int b = threadIdx.x; b < TOTAL; b += kThreads) {
    const int row = b / NBF, j = b - row * NBF;
    const int k = j % NS;
    const C* s = src + row * RS;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[pidx(j + r * NBF)];
    if (NS > 1 && k > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(&tw[r * k * TWSTEP]));
    }
    Dft<R, C>::run(v);
    C* o = dst + row * RS;
    const int o0 = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) o[pidx(o0 + r * NS)] = v[r];
  }
}

template <int N, int TB, int S, int NS, typename C>
__device__ __forceinline__ C* ct_passes(C* src, C* dst, const C* tw) {
  constexpr CPlan P = PlanOf<N>::p;
  if constexpr (S >= P.ns) {
    return src;
  } else {
    constexpr int R = P.r[S];
    ct_pass<R, N, TB, NS, C>(src, dst, tw);
    __syncthreads();
    return ct_passes<N, TB, S + 1, NS * R, C>(dst, src, tw);
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

template <typename RT, int N>
static bool launch_ct(cudaStream_t s, const Dims& d, const void* tw, const void* F, RT* grid, size_t stride,
                      int ncomp, bool synth, const double* w) {
  typedef typename C2<RT>::T C;
  constexpr int RS = CtGeom<RT, N>::RS, TB = CtGeom<RT, N>::TB;
  const size_t sm = (size_t)2 * TB * RS * sizeof(C);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_fft_synth_ct<RT, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    cudaFuncSetAttribute(k_fft_analysis_ct<RT, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr = true;
  }
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
  if (launch_fixed<RT>(s, d, p0.n, twiddle, G, const_cast<RT*>(grid), grid_comp_stride, ncomp, false, w)) return;
  FftPlan p = p0;
  p.tb = pick_tb<RT>(d, p.n);
  const size_t sm = (size_t)2 * p.tb * prow(p.n) * sizeof(C);
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

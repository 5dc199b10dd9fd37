// gd_fft_core.cuh -- device building blocks of the phi transforms: complex
// helpers, small DFTs in registers, padded shared-memory rows and Stockham
// passes (runtime plan and compile-time lengths).  Used by the stand-alone
// transform kernels (gd_fft.cu) and by the fused per-phase kernels
// (gd_fused.cu).
#pragma once

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
// Unpadded alternative: element i of a row stored at i ^ ((i >> 4) & 15), a
// permutation inside each aligned group of 16.  Stride-16 runs (radix-16
// outputs) and unit-stride runs both spread over distinct bank pairs for
// 8-byte elements, so rows need no padding (used by the fused kernels, whose
// occupancy is bounded by shared memory).
__device__ __forceinline__ int xidx(int i) { return i ^ ((i >> 4) & 15); }

// One Stockham pass from src to dst ([tb][n] each): radix R, Ns = product of
// the radices of the earlier passes.
template <int R, typename C, int NT = kThreads>
__device__ __forceinline__ void fft_pass(const C* __restrict__ src, C* __restrict__ dst, int tb, int n, int Ns,
                                         const C* __restrict__ tw) {
  const int nbf = n / R;
  const int total = tb * nbf;
  const int twstep = n / (Ns * R);
  for (int b = threadIdx.x; b < total; b += NT) {
    const int row = b / nbf, j = b - row * nbf;
    const int k = j % Ns;
    const C* s = src + (size_t)row * prow(n);
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[pidx(j + r * nbf)];
    if (k > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[r * k * twstep]);
    }
    Dft<R, C>::run(v);
    C* o = dst + (size_t)row * prow(n);
    const int o0 = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) o[pidx(o0 + r * Ns)] = v[r];
  }
}

// Runs all passes; returns the buffer holding the result.
template <typename RT, int NT = kThreads>
__device__ typename C2<RT>::T* fft_forward(typename C2<RT>::T* a, typename C2<RT>::T* b, int tb, const FftPlan& p,
                                           const typename C2<RT>::T* tw) {
  typedef typename C2<RT>::T C;
  int Ns = 1;
  C* src = a;
  C* dst = b;
  for (int s = 0; s < p.nstage; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 16: fft_pass<16, C, NT>(src, dst, tb, p.n, Ns, tw); break;
      case 8: fft_pass<8, C, NT>(src, dst, tb, p.n, Ns, tw); break;
      case 4: fft_pass<4, C, NT>(src, dst, tb, p.n, Ns, tw); break;
      case 2: fft_pass<2, C, NT>(src, dst, tb, p.n, Ns, tw); break;
      case 3: fft_pass<3, C, NT>(src, dst, tb, p.n, Ns, tw); break;
      default: fft_pass<5, C, NT>(src, dst, tb, p.n, Ns, tw); break;
    }
    __syncthreads();
    Ns *= R;
    C* t = src; src = dst; dst = t;
  }
  return src;
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

// One compile-time Stockham pass.  Padded indices pidx(j + r * stride) are
// formed as pidx(j) + r * (stride + stride / 16) when the stride is a multiple
// of 16 (and as pidx(group base) + offset when a radix group cannot cross a
// 16-element boundary), so the inner loops carry no index arithmetic.  The
// twiddle table may live in global or shared memory.
// PT: tw is this pass's own table [r - 1][k] (k < NS, consecutive k in
// consecutive entries, so a warp's twiddle reads are conflict-free in shared
// memory); otherwise tw is the full table W_N^i.
template <int R, int N, int TB, int NS, typename C, int NT = kThreads, bool PT = false, bool XS = false>
__device__ __forceinline__ void ct_pass(const C* __restrict__ src, C* __restrict__ dst, const C* __restrict__ tw) {
  constexpr int RS = XS ? N : (N + (N >> 4)) | 1;
  constexpr int NBF = N / R;
  constexpr int TOTAL = TB * NBF;
  constexpr int TWSTEP = N / (NS * R);
  for (int b = threadIdx.x; b < TOTAL; b += NT) {
    const int row = b / NBF, j = b - row * NBF;
    const int k = j % NS;
    const C* s = src + row * RS;
    C v[R];
    if constexpr (XS) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[xidx(j + r * NBF)];
    } else if constexpr (NBF % 16 == 0) {
      const C* sj = s + pidx(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = sj[r * (NBF + NBF / 16)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[pidx(j + r * NBF)];
    }
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], PT ? tw[(r - 1) * NS + k] : tw[r * k * TWSTEP]);
    }
    Dft<R, C>::run(v);
    C* o = dst + row * RS;
    const int base = (j / NS) * NS * R;
    const int o0 = base + k;
    if constexpr (XS) {
#pragma unroll
      for (int r = 0; r < R; ++r) o[xidx(o0 + r * NS)] = v[r];
    } else if constexpr (NS % 16 == 0) {
      C* oo = o + pidx(o0);
#pragma unroll
      for (int r = 0; r < R; ++r) oo[r * (NS + NS / 16)] = v[r];
    } else if constexpr (16 % (NS * R) == 0) {
      C* oo = o + o0 + (base >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) oo[r * NS] = v[r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) o[pidx(o0 + r * NS)] = v[r];
    }
  }
}

template <int N, int TB, int S, int NS, typename C, int NT = kThreads>
__device__ __forceinline__ C* ct_passes(C* src, C* dst, const C* tw) {
  constexpr CPlan P = PlanOf<N>::p;
  if constexpr (S >= P.ns) {
    return src;
  } else {
    constexpr int R = P.r[S];
    ct_pass<R, N, TB, NS, C, NT>(src, dst, tw);
    __syncthreads();
    return ct_passes<N, TB, S + 1, NS * R, C, NT>(dst, src, tw);
  }
}

// A compile-time pass that hands its outputs (row, natural index, value) to
// f instead of storing them: the last pass of a transform whose consumer is
// pointwise in the output index.
template <int R, int N, int TB, int NS, typename C, int NT, bool PT, bool XS, class F>
__device__ __forceinline__ void ct_pass_apply(const C* __restrict__ src, const C* __restrict__ tw, F& f) {
  constexpr int RS = XS ? N : (N + (N >> 4)) | 1;
  constexpr int NBF = N / R;
  constexpr int TOTAL = TB * NBF;
  constexpr int TWSTEP = N / (NS * R);
  for (int b = threadIdx.x; b < TOTAL; b += NT) {
    const int row = b / NBF, j = b - row * NBF;
    const int k = j % NS;
    const C* s = src + row * RS;
    C v[R];
    if constexpr (XS) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[xidx(j + r * NBF)];
    } else if constexpr (NBF % 16 == 0) {
      const C* sj = s + pidx(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = sj[r * (NBF + NBF / 16)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = s[pidx(j + r * NBF)];
    }
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], PT ? tw[(r - 1) * NS + k] : tw[r * k * TWSTEP]);
    }
    Dft<R, C>::run(v);
    const int o0 = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) f(row, o0 + r * NS, v[r]);
  }
}

// Per-pass twiddle tables: pass s (NS_s > 1) owns (R_s - 1) NS_s entries
// W_N^(r k N / (NS_s R_s)) at [r - 1][k], one after the other.
constexpr int ct_pass_tw_entries(int N) {
  const CPlan p = make_cplan(N);
  int ns = 1, tot = 0;
  for (int s = 0; s < p.ns; ++s) {
    if (ns > 1) tot += (p.r[s] - 1) * ns;
    ns *= p.r[s];
  }
  return tot;
}

// Fills the per-pass tables from the full table W_N^i (global memory); TS > 1:
// the table is W_(TS N)^i, read at TS-fold indices.
template <int N, int NT, int TS = 1>
__device__ __forceinline__ void ct_fill_pass_twiddles(const float2* __restrict__ tw_full, float2* __restrict__ out) {
  constexpr CPlan P = PlanOf<N>::p;
  int ns = 1, off = 0;
#pragma unroll
  for (int s = 0; s < P.ns; ++s) {
    const int R = P.r[s];
    if (ns > 1) {
      const int step = N / (ns * R);
      for (int e = threadIdx.x; e < (R - 1) * ns; e += NT) {
        const int r = e / ns + 1, k = e - (r - 1) * ns;
        out[off + e] = tw_full[TS * r * k * step];
      }
      off += (R - 1) * ns;
    }
    ns *= R;
  }
}

// ct_passes with per-pass twiddle tables (ct_fill_pass_twiddles layout);
// XS: rows in the unpadded xidx layout.
template <int N, int TB, int S, int NS, typename C, int NT, int OFF = 0, bool XS = false>
__device__ __forceinline__ C* ct_passes_pt(C* src, C* dst, const C* tw) {
  constexpr CPlan P = PlanOf<N>::p;
  if constexpr (S >= P.ns) {
    return src;
  } else {
    constexpr int R = P.r[S];
    ct_pass<R, N, TB, NS, C, NT, true, XS>(src, dst, tw + OFF);
    __syncthreads();
    return ct_passes_pt<N, TB, S + 1, NS * R, C, NT, (NS > 1 ? OFF + (R - 1) * NS : OFF), XS>(dst, src, tw);
  }
}

// ct_passes_pt whose last pass hands its outputs to f (ct_pass_apply).
template <int N, int TB, int S, int NS, typename C, int NT, int OFF, bool XS, class F>
__device__ __forceinline__ void ct_passes_pt_apply(C* src, C* dst, const C* tw, F& f) {
  constexpr CPlan P = PlanOf<N>::p;
  constexpr int R = P.r[S];
  if constexpr (S == P.ns - 1) {
    ct_pass_apply<R, N, TB, NS, C, NT, true, XS>(src, tw + OFF, f);
  } else {
    ct_pass<R, N, TB, NS, C, NT, true, XS>(src, dst, tw + OFF);
    __syncthreads();
    ct_passes_pt_apply<N, TB, S + 1, NS * R, C, NT, (NS > 1 ? OFF + (R - 1) * NS : OFF), XS>(dst, src, tw, f);
  }
}

}  // namespace gd

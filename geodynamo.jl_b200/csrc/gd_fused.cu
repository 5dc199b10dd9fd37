// gd_fused.cu -- the grid-space part of each nonlinear phase of the
// mixed-precision step in one kernel: inverse phi transforms of the phase's
// synthesized components, the pointwise products, and the forward phi
// transform with the Gauss-weighted north/south folds that the Legendre
// analysis consumes.  The physical grids of a phase live only in shared
// memory; HBM sees the Fourier coefficients in and the folded transforms out.
//
// CTA = (block of FOURIER_BLOCK north/south colatitude pairs, shell).  The
// Fourier input is the blocked layout written by the tensor-core synthesis:
// float4 (north Re, north Im, south Re, south Im) at
//   [comp][r][theta block][m][pair in block],
// so one CTA reads one contiguous run per component.  The next component's
// coefficients are fetched into registers while the current one is
// transformed.
//
// Products are the reference's, term by term (src/scalar_field_common.jl:
// 390-443, src/velocity.jl:447-548,638-672, src/magnetic.jl:375-404), with
// the radial components identically zero because the reference's vector
// synthesis writes only theta/phi (src/shtnskit_field_functions.jl:264-279);
// every product involving a radial component is still evaluated, so
// non-finite inputs propagate as in the reference.
#include "gd_fft_core.cuh"
#include "gd_fused.cuh"
#include "gd_internal.cuh"
#include "gd_mixed_kernels.cuh"

namespace gd {

namespace {

constexpr int FB = FOURIER_BLOCK;
constexpr int FNT = 128;  // threads per CTA
constexpr int PF = 4;     // prefetched float4 per thread (covers (M+1) FB <= 512)

// compile-time lengths keep rows in the unpadded xidx layout, the runtime
// plan in the padded pidx layout
template <int N>
__device__ __forceinline__ int ridx(int i) {
  if constexpr (N > 0) return xidx(i);
  else return pidx(i);
}
template <int N>
__host__ __device__ __forceinline__ int row_stride(int n) {
  if constexpr (N > 0) return N;
  else return prow(n);
}

template <int N>
__device__ __forceinline__ float2* run_fft(float2* a, float2* b, const float2* tw, const FftPlan& p) {
  if constexpr (N > 0) {
    return ct_passes_pt<N, FB, 0, 1, float2, FNT, 0, true>(a, b, tw);
  } else {
    return fft_forward<float, FNT>(a, b, FB, p, tw);
  }
}

// Z_m = F_N + i F_S and Z_{n-m} = conj(F_N) + i conj(F_S), stored conjugated
// (the inverse transform is conj(FFT(conj(Z)))): element e = m * FB + pair.
template <int N>
__device__ __forceinline__ void pack_z(float2* bufA, int rs, int n, int e, int rows, float4 v) {
  const int m = e / FB, ii = e - m * FB;
  if (ii >= rows) v = make_float4(0.f, 0.f, 0.f, 0.f);
  float2* row = bufA + ii * rs;
  if (m == 0) {
    row[0] = make_float2(v.x, -v.z);
  } else {
    row[ridx<N>(m)] = make_float2(v.x - v.w, -(v.y + v.z));
    row[ridx<N>(n - m)] = make_float2(v.x + v.w, v.y - v.z);
  }
}

// Lengths n = 3 P with P a power of two (P >= 8).  When every order m <= M
// < P, the conjugated input y is zero on P <= k <= 2P, so with phi = 3 c + a
// the inverse transform is three P-point transforms of
//   W_a[k] = W^(k a) (y_k + y_(k + 2P) W^(2 P a)),   W = exp(-2 pi i / n),
// built straight from the frequency pair (k, P - k) -- no zero band and no
// radix-3 pass -- and the forward transform's outputs X_m, X_(n - m) (m <= M)
// follow from the P-point transforms Y_a of the sub-rows x_(3 c + a):
//   X_m = sum_a W^(m a) Y_a[m],  X_(n - m) = sum_a W^(-m a) Y_a[(P - m) mod P].
// Sub-row (pair ii, a) holds P elements at (3 ii + a) P in the xidx layout.
// The last P-point pass has fewer butterflies than threads, so the split is
// used where the products are light (the induction phase, the grid output): with the heavier
// velocity and temperature products the radix-3 pass, which spreads them over
// every thread, is faster.
template <int N> struct Split3 {
  static constexpr int P = N / 3;
  static constexpr bool ok = N > 0 && N % 3 == 0 && P >= 8 && (P & (P - 1)) == 0;
};

__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

}  // namespace

template <int N, int PH, bool S3>
__global__ void __launch_bounds__(FNT, 4) k_fused(Dims d, FftPlan p, const float2* __restrict__ tw, FusedArgs a) {
  typedef float2 C;
  constexpr int P = S3 ? N / 3 : 1;
  const int n = N > 0 ? N : p.n;
  const int rs = row_stride<N>(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + FB * rs;
  C* acc0 = bufB + FB * rs;
  C* acc1 = acc0 + FB * rs;
  C* u0 = acc1;            // phase T (one product): the velocity component in use
  // the twiddle table after the phase's buffers
  const int nbuf = PH == FUSED_GRID ? 2 : 4;
  C* stw = reinterpret_cast<C*>(smem_raw + (size_t)nbuf * FB * rs * sizeof(C));

  const int tid = threadIdx.x;
  const int ib = blockIdx.x, r = blockIdx.y;
  const int M = d.M;
  const int i0 = ib * FB;
  const int rows = min(FB, d.nth - i0);
  const int tot = (M + 1) * FB;
  const size_t boff = ((size_t)r * gridDim.x + ib) * (size_t)tot;

  // S3: the P-point passes' tables, then W^k for k < 2P
  C* const stw3 = stw + (S3 ? ct_pass_tw_entries(P) : 0);
  if constexpr (S3) {
    static_assert(ct_pass_tw_entries(P) + 2 * P <= N, "twiddles exceed the table space");
    ct_fill_pass_twiddles<P, FNT, 3>(tw, stw);
    for (int k = tid; k < 2 * P; k += FNT) stw3[k] = tw[k];
    __syncthreads();  // the input packing (build) reads W^k before the first pass barrier
  } else if constexpr (N > 0) {
    static_assert(ct_pass_tw_entries(N) <= N, "per-pass twiddles exceed the table space");
    ct_fill_pass_twiddles<N, FNT>(tw, stw);
  } else {
    for (int j = tid; j < n; j += FNT) stw[j] = tw[j];
  }
  if (PH != FUSED_GRID) {
    for (int e = tid; e < FB * rs; e += FNT) {
      acc0[e] = make_float2(0.f, 0.f);
      if (PH != FUSED_TEMPERATURE) acc1[e] = make_float2(0.f, 0.f);
    }
  }

  float4 pf[PF];
  // S3 items: (pair ii, j) for j = 0..P/2, each the frequencies j and P - j
  constexpr int H = P / 2 + 1;
  auto s3_load = [&](const float4* src, int it, float4& v1, float4& v2) {
    const int ii = it / H, j = it - ii * H;
    v1 = v2 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (it >= FB * H || ii >= rows) return;
    if (j <= M) v1 = __ldg(src + j * FB + ii);
    if (P - j <= M) v2 = __ldg(src + (P - j) * FB + ii);
  };
  auto prefetch = [&](int c) {
    const float4* src = a.fin[c] + boff;
    if constexpr (S3) {
#pragma unroll
      for (int k = 0; k < PF / 2; ++k) s3_load(src, tid + k * FNT, pf[2 * k], pf[2 * k + 1]);
    } else {
#pragma unroll
      for (int k = 0; k < PF; ++k) {
        const int e = tid + k * FNT;
        pf[k] = e < tot ? __ldg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  };
  // S3: W_a[k] for the sub-rows of pair ii from y_k and y_(k + 2P)
  auto s3_put = [&](int ii, int k, C y, C y2) {
    const C cp = stw3[P];  // W^P; W^(2P) = conj(W^P), W^(4P) = W^P
    C* row = bufA + ii * N;
    const int xk = xidx(k);
    row[xk] = cadd(y, y2);
    row[P + xk] = cmul(cadd(y, cmul(y2, conjf2(cp))), stw3[k]);
    row[2 * P + xk] = cmul(cadd(y, cmul(y2, cp)), stw3[2 * k]);
  };
  auto s3_item = [&](int it, float4 v1, float4 v2) {
    const int ii = it / H, j = it - ii * H;
    // conjugated spectrum: y_0 = (N re, -S re); y_m = (N re - S im, -(N im + S re)),
    // y_(n-m) = (N re + S im, N im - S re) for m >= 1 (pack_z)
    const C yj = j == 0 ? make_float2(v1.x, -v1.z) : make_float2(v1.x - v1.w, -(v1.y + v1.z));
    const C yj2 = make_float2(v2.x + v2.w, v2.y - v2.z);  // y_(j + 2P) from m = P - j
    s3_put(ii, j, yj, yj2);
    if (j > 0 && j < P - j) {
      const C yk = make_float2(v2.x - v2.w, -(v2.y + v2.z));  // y_(P - j)
      const C yk2 = make_float2(v1.x + v1.w, v1.y - v1.z);   // y_(n - j) = y_(P - j + 2P)
      s3_put(ii, P - j, yk, yk2);
    }
  };
  const int band = n - 2 * M - 1;  // frequencies M < k < n - M are zero
  auto build = [&](int c) {
    if constexpr (S3) {
#pragma unroll
      for (int k = 0; k < PF / 2; ++k) {
        const int it = tid + k * FNT;
        if (it < FB * H) s3_item(it, pf[2 * k], pf[2 * k + 1]);
      }
      const float4* src = a.fin[c] + boff;
      for (int it = tid + (PF / 2) * FNT; it < FB * H; it += FNT) {
        float4 v1, v2;
        s3_load(src, it, v1, v2);
        s3_item(it, v1, v2);
      }
    } else {
      for (int e = tid; e < FB * band; e += FNT) {
        const int ii = e / band, k = M + 1 + (e - ii * band);
        bufA[ii * rs + ridx<N>(k)] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < PF; ++k) {
        const int e = tid + k * FNT;
        if (e < tot) pack_z<N>(bufA, rs, n, e, rows, pf[k]);
      }
      const float4* src = a.fin[c] + boff;
      for (int e = tid + PF * FNT; e < tot; e += FNT) pack_z<N>(bufA, rs, n, e, rows, __ldg(src + e));
    }
  };
  const float ur = 0.f, wr = 0.f, jr = 0.f, br = 0.f;
  // per-shell factors when the handle's segments have their own Ekman numbers
  const float rf_r = d.rfs32 ? d.rfs32[r] : a.rf;
  const float adv = -rf_r, mrf = a.cf != 0.f ? -rf_r : -a.cf, lfr = d.rfs32 ? rf_r : a.lf;

  // consumer of one transformed component: grid rows or the products
  // inputs: T phase [g_r, u_th, g_th, u_ph, g_ph]; V phase [u_th, u_ph,
  // w_th, w_ph, j_th, j_ph, b_th, b_ph]; M phase [u_th, u_ph, b_th, b_ph]
  int c = 0;
  float s_r = (PH == FUSED_TEMPERATURE) ? (float)a.sources[r] : 0.f;
  // j: longitude index; q: storage index of (ii, j) in the phase's buffers
  auto consume = [&](int ii, int j, int q, C z) {
    if (PH == FUSED_GRID) {
      if (ii < rows) {
        float* gbase = a.gout[c] + (size_t)r * d.nlat * n;
        const int ith = i0 + ii;
        gbase[(size_t)ith * n + j] = z.x;
        gbase[(size_t)(d.nlat - 1 - ith) * n + j] = -z.y;
      }
      return;
    }
    const float vN = z.x, vS = -z.y;
    if (PH == FUSED_TEMPERATURE) {
      // -(u_r g_r + u_th g_th + u_ph g_ph) + S(r); each velocity component
      // is held only until its gradient partner arrives
      if (c == 0) {
        acc0[q] = make_float2(ur * vN, ur * vS);
      } else if (c == 1 || c == 3) {
        u0[q] = make_float2(vN, vS);
      } else if (c == 2) {
        const C u = u0[q], t = acc0[q];
        acc0[q] = make_float2(t.x + u.x * vN, t.y + u.y * vS);
      } else {
        const C u = u0[q], t = acc0[q];
        float xN = -(t.x + u.x * vN), xS = -(t.y + u.y * vS);
        if (s_r != 0.f) { xN += s_r; xS += s_r; }
        acc0[q] = make_float2(xN, xS);
      }
    } else if (PH == FUSED_VELOCITY) {
      // theta: adv (u_ph w_r - u_r w_ph) + mrf (-ct u_ph) + lf (j_ph b_r - j_r b_ph)
      // phi:   adv (u_r w_th - u_th w_r) + mrf (ct u_th + st u_r) + lf (j_r b_th - j_th b_r)
      // even inputs (theta components) feed the phi product, odd ones the theta product
      C* acc = (c & 1) ? acc0 : acc1;
      C t = acc[q];
      switch (c) {
        case 0: {
          // Coriolis factors of latitude index min(phi index, nlat - 1) (L1-cached)
          const int tj = j < d.nlat - 1 ? j : d.nlat - 1;
          const float ct = (float)__ldg(a.cth + tj), st = (float)__ldg(a.sthc + tj);
          t.x += adv * (-(vN * wr)) + mrf * (ct * vN + st * ur);
          t.y += adv * (-(vS * wr)) + mrf * (ct * vS + st * ur);
          break;
        }
        case 1: {
          const float ct = (float)__ldg(a.cth + (j < d.nlat - 1 ? j : d.nlat - 1));
          t.x += adv * (vN * wr) + mrf * (-ct * vN);
          t.y += adv * (vS * wr) + mrf * (-ct * vS);
          break;
        }
        case 2: t.x += adv * (ur * vN); t.y += adv * (ur * vS); break;
        case 3: t.x += adv * (-(ur * vN)); t.y += adv * (-(ur * vS)); break;
        case 4: t.x += lfr * (-(vN * br)); t.y += lfr * (-(vS * br)); break;
        case 5: t.x += lfr * (vN * br); t.y += lfr * (vS * br); break;
        case 6: t.x += lfr * (jr * vN); t.y += lfr * (jr * vS); break;
        default: t.x += lfr * (-(jr * vN)); t.y += lfr * (-(jr * vS)); break;
      }
      acc[q] = t;
    } else {
      // induction: theta u_ph b_r - u_r b_ph, phi u_r b_th - u_th b_r
      C* acc = (c & 1) ? acc0 : acc1;
      C t = acc[q];
      switch (c) {
        case 0: t.x += -(vN * br); t.y += -(vS * br); break;
        case 1: t.x += vN * br; t.y += vS * br; break;
        case 2: t.x += ur * vN; t.y += ur * vS; break;
        default: t.x += -(ur * vN); t.y += -(ur * vS); break;
      }
      acc[q] = t;
    }
  };

  auto consume_n = [&](int ii, int j, C z) { consume(ii, j, ii * rs + ridx<N>(j), z); };
  auto consume_s3 = [&](int sr, int cc, C z) {
    const int ii = sr / 3, a3 = sr - 3 * ii;
    consume(ii, 3 * cc + a3, sr * P + xidx(cc), z);
  };

  prefetch(0);
  for (c = 0; c < a.nin; ++c) {
    build(c);
    __syncthreads();
    if (c + 1 < a.nin) prefetch(c + 1);
    if constexpr (S3) {
      ct_passes_pt_apply<P, 3 * FB, 0, 1, C, FNT, 0, true>(bufA, bufB, stw, consume_s3);
    } else if constexpr (N > 0) {
      // the last Stockham pass feeds the consumer directly
      ct_passes_pt_apply<N, FB, 0, 1, C, FNT, 0, true>(bufA, bufB, stw, consume_n);
    } else {
      const C* res = run_fft<N>(bufA, bufB, stw, p);
      for (int e = tid; e < FB * n; e += FNT) {
        const int ii = e / n, j = e - ii * n;
        consume_n(ii, j, res[ii * rs + ridx<N>(j)]);
      }
    }
    __syncthreads();
  }
  if (PH == FUSED_GRID) return;

  // forward transforms of the products and the folds w (G_N +- G_S)
  const float sc = (float)(2.0 * 3.14159265358979323846 / n);
  const int nout = (PH == FUSED_TEMPERATURE) ? 1 : 2;
  for (int o = 0; o < nout; ++o) {
    C* src = o == 0 ? acc0 : acc1;
    const C* res;
    if constexpr (S3) res = ct_passes_pt<P, 3 * FB, 0, 1, C, FNT, 0, true>(src, o == 0 ? bufA : bufB, stw);
    else res = run_fft<N>(src, o == 0 ? bufA : bufB, stw, p);
    const size_t gb = ((size_t)(o * d.nr + r) * (M + 1)) * 2 * d.nth;
    for (int e = tid; e < tot; e += FNT) {
      const int m = e / FB, ii = e - m * FB;
      if (ii >= rows) continue;
      const int ith = i0 + ii;
      C zk, zn;
      if constexpr (S3) {
        const C* y = res + ii * N;  // Y_a at y + a P
        const int xm = xidx(m), xp = xidx(m == 0 ? 0 : P - m);
        const C w1 = stw3[m], w2 = stw3[2 * m];
        zk = cadd(y[xm], cadd(cmul(w1, y[P + xm]), cmul(w2, y[2 * P + xm])));
        zn = cadd(y[xp], cadd(cmul(conjf2(w1), y[P + xp]), cmul(conjf2(w2), y[2 * P + xp])));
      } else {
        const C* row = res + ii * rs;
        zk = row[ridx<N>(m)];
        zn = row[ridx<N>(m == 0 ? 0 : n - m)];
      }
      zn.y = -zn.y;
      const float Xx = 0.5f * (zk.x + zn.x), Xy = 0.5f * (zk.y + zn.y);
      const float Yx = 0.5f * (zk.y - zn.y), Yy = -0.5f * (zk.x - zn.x);
      const float gnx = sc * Xx, gny = sc * Xy, gsx = sc * Yx, gsy = sc * Yy;
      const float wi = (float)a.w[ith];
      a.G[gb + ((size_t)m * 2 + 0) * d.nth + ith] = make_float2(wi * (gnx + gsx), wi * (gny + gsy));
      a.G[gb + ((size_t)m * 2 + 1) * d.nth + ith] = make_float2(wi * (gnx - gsx), wi * (gny - gsy));
    }
    __syncthreads();
  }
}

namespace {

size_t fused_smem(int phase, int n, bool unpadded) {
  const size_t buf = (size_t)FB * (unpadded ? n : prow(n)) * sizeof(float2);
  const size_t twb = (size_t)n * sizeof(float2);
  switch (phase) {
    case FUSED_GRID: return 2 * buf + twb;
    default: return 4 * buf + twb;
  }
}

template <int N, int PH, bool S3>
void launch_one_k(cudaStream_t s, const Dims& d, const FftPlan& p, const float2* tw, const FusedArgs& a) {
  const int n = N > 0 ? N : p.n;
  const size_t sm = fused_smem(PH, n, N > 0);
  allow_dynamic_smem(k_fused<N, PH, S3>, sm);
  dim3 g(ceil_div(d.nth, FB), d.nr);
  k_fused<N, PH, S3><<<g, FNT, sm, s>>>(d, p, tw, a);
}

// the three-way split for the induction phase and the grid output whenever
// the orders fit below n / 3 (the usual dealiased grid nlon = 3 (M + 1))
template <int N, int PH>
void launch_one(cudaStream_t s, const Dims& d, const FftPlan& p, const float2* tw, const FusedArgs& a) {
  if constexpr (Split3<N>::ok && (PH == FUSED_INDUCTION || PH == FUSED_GRID)) {
    if (d.M + 1 <= N / 3) {
      launch_one_k<N, PH, true>(s, d, p, tw, a);
      return;
    }
  }
  launch_one_k<N, PH, false>(s, d, p, tw, a);
}

template <int N>
void launch_phase(cudaStream_t s, const Dims& d, const FftPlan& p, const float2* tw, int phase, const FusedArgs& a) {
  switch (phase) {
    case FUSED_GRID: launch_one<N, FUSED_GRID>(s, d, p, tw, a); break;
    case FUSED_TEMPERATURE: launch_one<N, FUSED_TEMPERATURE>(s, d, p, tw, a); break;
    case FUSED_VELOCITY: launch_one<N, FUSED_VELOCITY>(s, d, p, tw, a); break;
    default: launch_one<N, FUSED_INDUCTION>(s, d, p, tw, a); break;
  }
}

}  // namespace

int fourier_blocks(const Dims& d) { return ceil_div(d.nth, FB); }

size_t fourier_comp_elems(const Dims& d) { return (size_t)d.nr * fourier_blocks(d) * (d.M + 1) * FB; }

size_t fused_smem_bytes(int phase, int nlon) { return fused_smem(phase, nlon, false); }

void launch_fused(cudaStream_t s, const Dims& d, const FftPlan& p, const void* twf, int phase, const FusedArgs& a) {
  const float2* tw = static_cast<const float2*>(twf);
  switch (p.n) {
    case 24: launch_phase<24>(s, d, p, tw, phase, a); break;
    case 40: launch_phase<40>(s, d, p, tw, phase, a); break;
    case 48: launch_phase<48>(s, d, p, tw, phase, a); break;
    case 96: launch_phase<96>(s, d, p, tw, phase, a); break;
    case 144: launch_phase<144>(s, d, p, tw, phase, a); break;
    case 192: launch_phase<192>(s, d, p, tw, phase, a); break;
    case 288: launch_phase<288>(s, d, p, tw, phase, a); break;
    case 384: launch_phase<384>(s, d, p, tw, phase, a); break;
    case 768: launch_phase<768>(s, d, p, tw, phase, a); break;
    default: launch_phase<0>(s, d, p, tw, phase, a); break;
  }
}

}  // namespace gd

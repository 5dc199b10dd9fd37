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

}  // namespace

template <int N, int PH>
__global__ void __launch_bounds__(FNT, 4) k_fused(Dims d, FftPlan p, const float2* __restrict__ tw, FusedArgs a) {
  typedef float2 C;
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

  if constexpr (N > 0) {
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
  auto prefetch = [&](int c) {
    const float4* src = a.fin[c] + boff;
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int e = tid + k * FNT;
      pf[k] = e < tot ? __ldg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  const int band = n - 2 * M - 1;  // frequencies M < k < n - M are zero
  auto build = [&](int c) {
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
  };
  const float ur = 0.f, wr = 0.f, jr = 0.f, br = 0.f;
  const float adv = -a.rf, mrf = -a.rf, lfr = a.lf;

  // consumer of one transformed component: grid rows or the products
  // inputs: T phase [g_r, u_th, g_th, u_ph, g_ph, T]; V phase [u_th, u_ph,
  // w_th, w_ph, j_th, j_ph, b_th, b_ph]; M phase [u_th, u_ph, b_th, b_ph]
  int c = 0;
  float s_r = (PH == FUSED_TEMPERATURE) ? (float)a.sources[r] : 0.f;
  auto consume = [&](int ii, int j, C z) {
    if (PH == FUSED_GRID || (PH == FUSED_TEMPERATURE && c == 5)) {
      if (ii < rows) {
        float* gbase = (PH == FUSED_GRID ? a.gout[c] : a.gout[0]) + (size_t)r * d.nlat * n;
        const int ith = i0 + ii;
        gbase[(size_t)ith * n + j] = z.x;
        gbase[(size_t)(d.nlat - 1 - ith) * n + j] = -z.y;
      }
      return;
    }
    const int q = ii * rs + ridx<N>(j);
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

  prefetch(0);
  for (c = 0; c < a.nin; ++c) {
    build(c);
    __syncthreads();
    if (c + 1 < a.nin) prefetch(c + 1);
    if constexpr (N > 0) {
      // the last Stockham pass feeds the consumer directly
      ct_passes_pt_apply<N, FB, 0, 1, C, FNT, 0, true>(bufA, bufB, stw, consume);
    } else {
      const C* res = run_fft<N>(bufA, bufB, stw, p);
      for (int e = tid; e < FB * n; e += FNT) {
        const int ii = e / n, j = e - ii * n;
        consume(ii, j, res[ii * rs + ridx<N>(j)]);
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
    const C* res = run_fft<N>(src, o == 0 ? bufA : bufB, stw, p);
    const size_t gb = ((size_t)(o * d.nr + r) * (M + 1)) * 2 * d.nth;
    for (int e = tid; e < tot; e += FNT) {
      const int m = e / FB, ii = e - m * FB;
      if (ii >= rows) continue;
      const int ith = i0 + ii;
      const C* row = res + ii * rs;
      const C zk = row[ridx<N>(m)];
      C zn = row[ridx<N>(m == 0 ? 0 : n - m)];
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

template <int N, int PH>
void launch_one(cudaStream_t s, const Dims& d, const FftPlan& p, const float2* tw, const FusedArgs& a) {
  const int n = N > 0 ? N : p.n;
  const size_t sm = fused_smem(PH, n, N > 0);
  static size_t attr = 0;
  if (attr < sm) {
    cudaFuncSetAttribute(k_fused<N, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = sm;
  }
  dim3 g(ceil_div(d.nth, FB), d.nr);
  k_fused<N, PH><<<g, FNT, sm, s>>>(d, p, tw, a);
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

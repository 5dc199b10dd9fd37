// gd_setup.cu -- FP64 set-up kernels: Gauss-Legendre grid, associated Legendre
// tables, radial difference weights and the banded LU factors of the CNAB2
// implicit operators.  Everything here runs once per handle (and again when dt
// changes); the radial-operator kernels use explicitly rounded operations
// (no fused multiply-add) so the factors are reproducible operation for
// operation.
#include <math.h>

#include <map>
#include <mutex>
#include <utility>

#include "gd_internal.cuh"

namespace gd {

cudaError_t allow_dynamic_smem(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{func, dev}];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

int current_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    return 148;
  return n;
}

static const double kPi = 3.14159265358979323846;

// Gauss-Legendre nodes by Newton iteration on P_n(cos theta) in theta; the
// reference takes them from SHTnsKit.create_gauss_config
// (src/shtnskit_transforms.jl:109-112, 161-175).  North to south.
__global__ void k_gauss(int n, double* x, double* w, double* th, double* sth) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (n + 1) / 2) return;
  double t = kPi * (i + 0.75) / (n + 0.5);
  for (int it = 0; it < 100; ++it) {
    const double xx = cos(t);
    double p0 = 1.0, p1 = xx;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    const double dpdx = n * (xx * p1 - p0) / (xx * xx - 1.0);
    const double dt = p1 / (-sin(t) * dpdx);
    t -= dt;
    if (fabs(dt) < 1e-16 * fmax(1.0, t)) break;
  }
  const double xx = cos(t);
  double p0 = 1.0, p1 = xx;
  for (int k = 2; k <= n; ++k) {
    const double p2 = ((2.0 * k - 1.0) * xx * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  const double s = sin(t);
  const double q = n * (p0 - xx * p1);
  const double wi = 2.0 * s * s / (q * q);
  x[i] = xx; w[i] = wi; th[i] = t; sth[i] = s;
  x[n - 1 - i] = -xx; w[n - 1 - i] = wi; th[n - 1 - i] = kPi - t; sth[n - 1 - i] = s;
}

void launch_gauss(cudaStream_t s, int nlat, double* x, double* w, double* th, double* sth) {
  const int nt = (nlat + 1) / 2;
  k_gauss<<<ceil_div(nt, 64), 64, 0, s>>>(nlat, x, w, th, sth);
}

// Orthonormal Pbar_lm (Condon-Shortley phase), dPbar_lm/dtheta and
// Q = m Pbar_lm / sin(theta) at the north-half nodes.  One thread per
// (theta, m) walks the three-term recurrence in l.
__global__ void k_tables(int L, int M, int nth, const int* moff, const double* x, const double* sth,
                         double* P, double* dP, double* Q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (i >= nth || m > M) return;
  const double xx = x[i], s = sth[i];
  double pmm = 1.0 / sqrt(4.0 * kPi);
  double pm1 = 0.0;  // Pbar_11 for the m = 0 derivative column
  for (int mm = 1; mm <= m; ++mm) pmm = -sqrt((2.0 * mm + 1.0) / (2.0 * mm)) * s * pmm;
  if (m == 0 && L >= 1) pm1 = -sqrt(3.0 / 2.0) * s * pmm;
  const int base = moff[m];
  // column m
  double pl2 = 0.0, pl1 = pmm;       // P_{l-2}, P_{l-1}
  double q2 = 0.0, q1 = pm1;         // m = 1 column (only for m == 0)
  for (int l = m; l <= L; ++l) {
    double p;
    if (l == m) {
      p = pmm;
    } else if (l == m + 1) {
      p = sqrt(2.0 * m + 3.0) * xx * pmm;
    } else {
      const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      const double b = sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
      p = a * (xx * pl1 - b * pl2);
    }
    double d, qv;
    if (m == 0) {
      // dPbar_l0/dtheta = sqrt(l(l+1)) Pbar_l1
      double p1 = 0.0;
      if (l >= 1) {
        if (l == 1) {
          p1 = pm1;
        } else if (l == 2) {
          p1 = sqrt(5.0) * xx * pm1;
        } else {
          const double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - 1.0));
          const double b = sqrt(((l - 1.0) * (l - 1.0) - 1.0) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
          p1 = a * (xx * q1 - b * q2);
        }
        q2 = q1;
        q1 = p1;
        if (l == 1) { q2 = 0.0; q1 = pm1; }
      }
      d = (l == 0) ? 0.0 : sqrt((double)l * (l + 1.0)) * p1;
      qv = 0.0;
    } else {
      const double prev = (l > m) ? pl1 : 0.0;
      const double cf = (l > m) ? sqrt((2.0 * l + 1.0) * ((double)l * l - (double)m * m) / (2.0 * l - 1.0)) : 0.0;
      d = (l * xx * p - cf * prev) / s;
      qv = (double)m * p / s;
    }
    const size_t idx = (size_t)(base + (l - m)) * nth + i;
    P[idx] = p;
    dP[idx] = d;
    Q[idx] = qv;
    if (l == m) {
      pl2 = 0.0;
      pl1 = p;
    } else {
      pl2 = pl1;
      pl1 = p;
    }
  }
}

void launch_tables(cudaStream_t s, const Dims& d, const int* moff, const double* x, const double* sth,
                   double* P, double* dP, double* Q) {
  dim3 grid(ceil_div(d.nth, 64), d.M + 1);
  k_tables<<<grid, 64, 0, s>>>(d.L, d.M, d.nth, moff, x, sth, P, dP, Q);
}

// create_derivative_matrix (src/linear_algebra.jl:90-132): Vandermonde system
// on the clipped +-kl stencil, solved by Gaussian elimination with partial
// pivoting.  fd_mode 0 solves V^T w = rhs (difference weights); fd_mode 1 the
// literal V c = rhs.  Output in the reference band layout (2kl+1) x nr,
// column-major: entry (row i, col j) at (kl + i - j) + (2kl+1) j.
__device__ void dense_solve_rn(int n, double* A, double* b) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(A[k * 9 + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = fabs(A[i * 9 + k]);
      if (v > best) { best = v; p = i; }
    }
    if (p != k) {
      for (int j = 0; j < n; ++j) { const double t = A[k * 9 + j]; A[k * 9 + j] = A[p * 9 + j]; A[p * 9 + j] = t; }
      const double t = b[k]; b[k] = b[p]; b[p] = t;
    }
    const double dd = A[k * 9 + k];
    for (int i = k + 1; i < n; ++i) {
      const double f = __ddiv_rn(A[i * 9 + k], dd);
      A[i * 9 + k] = f;
      for (int j = k + 1; j < n; ++j) A[i * 9 + j] = __dsub_rn(A[i * 9 + j], __dmul_rn(f, A[k * 9 + j]));
      b[i] = __dsub_rn(b[i], __dmul_rn(f, b[k]));
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s = __dsub_rn(s, __dmul_rn(A[i * 9 + j], b[j]));
    b[i] = __ddiv_rn(s, A[i * 9 + i]);
  }
}

__global__ void k_fd_weights(int N, int kl, int fd_mode, const double* r, double* d1, double* d2) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int order = blockIdx.y + 1;
  if (n >= N) return;
  const int nbw = 2 * kl + 1;
  const int left = max(0, n - kl), right = min(N - 1, n + kl);
  const int S = right - left + 1;
  double V[81], A[81], b[9];
  for (int i = 0; i < S; ++i) {
    V[i * 9 + 0] = 1.0;
    for (int j = 1; j < S; ++j) V[i * 9 + j] = __dmul_rn(V[i * 9 + j - 1], __dsub_rn(r[left + i], r[n]));
  }
  for (int i = 0; i < S; ++i) b[i] = 0.0;
  if (order <= S) b[order] = (order == 2) ? 2.0 : 1.0;
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j) A[i * 9 + j] = (fd_mode == 0) ? V[j * 9 + i] : V[i * 9 + j];
  dense_solve_rn(S, A, b);
  double* out = (order == 1) ? d1 : d2;
  for (int j = 0; j < N; ++j) {
    // this thread owns row n: entries (n, j) for |n - j| <= kl
    if (j < n - kl || j > n + kl) continue;
    const int br = kl + n - j;
    double v = 0.0;
    if (j >= left && j <= right) v = b[j - left];
    out[br + (size_t)nbw * j] = v;
  }
}

void launch_fd_weights(cudaStream_t s, int nr, int kl, int fd_mode, const double* r, double* d1, double* d2) {
  dim3 grid(ceil_div(nr, 64), 2);
  k_fd_weights<<<grid, 64, 0, s>>>(nr, kl, fd_mode, r, d1, d2);
}

// create_shtns_timestepping_matrices (src/timestep.jl:498-543):
//   L_l = nu (D2 + (2/r) D1) - nu l(l+1)/r^2,   S_l = I/dt - theta L_l,
// then factorize_banded (src/linear_algebra.jl:23-57, no pivoting).
// One thread per (kind, l).  Bands in [kind][col][band][l] order.
// bc_rows (the boundary-row operator, bc_mode 2): bit 0 replaces rows 0 and
// N - 1 by boundary rows, identity rows (fixed values) unless bit 1 (inner)
// or bit 2 (outer) asks for the row of D1 there (a prescribed radial flux).
__global__ void k_build_lu(int N, int kl, int L, const double* d1, const double* d2, const double* rinv,
                           const double* rinv2, const double* nu, double inv_dt, double mth, int bc_rows,
                           double* lin, double* lu, int* status) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int kind = blockIdx.y;
  if (l > L) return;
  const int nbw = 2 * kl + 1;
  const double nk = nu[kind];
  const double lf = (double)l * (l + 1);
  const size_t Lp1 = (size_t)L + 1;
  auto at = [&](double* base, int i, int j) -> double& {
    return base[(((size_t)kind * N + j) * nbw + (kl + i - j)) * Lp1 + l];
  };
  for (int j = 0; j < N; ++j) {
    for (int b = 0; b < nbw; ++b) {
      const int i = j + b - kl;
      double lv = 0.0, d1v = 0.0;
      if (i >= 0 && i < N) {
        const size_t q = b + (size_t)nbw * j;
        d1v = d1[q];
        const double lapv = __dadd_rn(d2[q], __dmul_rn(__dmul_rn(2.0, rinv[i]), d1[q]));
        lv = __dmul_rn(nk, lapv);
        if (i == j) lv = __dsub_rn(lv, __dmul_rn(__dmul_rn(nk, lf), rinv2[i]));
      }
      double sv = __dmul_rn(lv, mth);
      if (i == j) sv = __dadd_rn(sv, inv_dt);
      if (bc_rows && (i == 0 || i == N - 1)) {  // boundary rows (bc_mode 2)
        const bool flux = (i == 0) ? (bc_rows & 2) != 0 : (bc_rows & 4) != 0;
        sv = flux ? d1v : ((i == j) ? 1.0 : 0.0);
      }
      lin[(((size_t)kind * N + j) * nbw + b) * Lp1 + l] = lv;
      lu[(((size_t)kind * N + j) * nbw + b) * Lp1 + l] = sv;
    }
  }
  int bad = 0;
  for (int k = 0; k < N - 1; ++k) {
    const double piv = at(lu, k, k);
    if (piv == 0.0) bad = 1;
    const int imax = min(N - 1, k + kl);
    for (int i = k + 1; i <= imax; ++i) {
      const double Lf = __ddiv_rn(at(lu, i, k), piv);
      at(lu, i, k) = Lf;
      for (int j = k + 1; j <= imax; ++j) at(lu, i, j) = __dsub_rn(at(lu, i, j), __dmul_rn(Lf, at(lu, k, j)));
    }
  }
  if (at(lu, N - 1, N - 1) == 0.0) bad = 1;
  if (bad) atomicExch(status, 1);
}

void launch_build_lu(cudaStream_t s, int nr, int kl, int L, const double* d1, const double* d2,
                     const double* rinv, const double* rinv2, const double* nu, double dt, double theta,
                     int bc_rows, double* lin, double* lu, int* status, int nkind) {
  dim3 grid(ceil_div(L + 1, 32), nkind);
  k_build_lu<<<grid, 32, 0, s>>>(nr, kl, L, d1, d2, rinv, rinv2, nu, 1.0 / dt, -theta, bc_rows, lin, lu, status);
}

}  // namespace gd

namespace gd {

// Coefficients of the three-term recurrence, per m-major mode j = (l, m):
//   Pbar_lm = a_lm (x Pbar_{l-1,m} - b_lm Pbar_{l-2,m})   (l >= m + 1; b = 0 at l = m + 1)
// the derivative coefficient c_lm = sqrt((2l+1)(l^2-m^2)/(2l-1)) of
//   dPbar_lm/dtheta = (l x Pbar_lm - c_lm Pbar_{l-1,m}) / sin(theta),
// the m = 1 column coefficients for the m = 0 derivative, Pbar_mm at the
// north nodes and 1/sin(theta).  Used by the tensor-core synthesis, which
// regenerates the table rows on the fly.
__global__ void k_rec_tables(int L, int M, int nth, const int* moff, const double* x, const double* sth,
                             double* ra, double* rb, double* rc, double* r1a, double* r1b, double* pmm,
                             double* sinv) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (m <= M && l >= m && l <= L) {
    const int j = moff[m] + (l - m);
    double a = 0.0, b = 0.0, c = 0.0;
    if (l == m + 1) {
      a = sqrt(2.0 * m + 3.0);
    } else if (l >= m + 2) {
      a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
      b = sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
    }
    if (l > m) c = sqrt((2.0 * l + 1.0) * ((double)l * l - (double)m * m) / (2.0 * l - 1.0));
    ra[j] = a;
    rb[j] = b;
    rc[j] = c;
  }
  if (m == 0 && l <= L) {
    double a = 0.0, b = 0.0;
    if (l == 2) {
      a = sqrt(5.0);
    } else if (l >= 3) {
      a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - 1.0));
      b = sqrt(((l - 1.0) * (l - 1.0) - 1.0) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
    }
    r1a[l] = a;
    r1b[l] = b;
  }
  if (m <= M && l < nth) {
    const double s = sth[l];
    double p = 1.0 / sqrt(4.0 * kPi);
    for (int mm = 1; mm <= m; ++mm) p = -sqrt((2.0 * mm + 1.0) / (2.0 * mm)) * s * p;
    pmm[(size_t)m * nth + l] = p;
    if (m == 0) sinv[l] = 1.0 / s;
  }
}

void launch_rec_tables(cudaStream_t s, const Dims& d, const int* moff, const double* x, const double* sth,
                       double* ra, double* rb, double* rc, double* r1a, double* r1b, double* pmm, double* sinv) {
  const int n = (d.L + 1 > d.nth ? d.L + 1 : d.nth);
  dim3 grid(ceil_div(n, 128), d.M + 1);
  k_rec_tables<<<grid, 128, 0, s>>>(d.L, d.M, d.nth, moff, x, sth, ra, rb, rc, r1a, r1b, pmm, sinv);
}

}  // namespace gd

"""Generate the golden fixtures under tests/golden/.

Independent truth comes from scipy/numpy (no oracle involved) wherever a
closed form exists:
  * Gauss nodes/weights: numpy.polynomial.legendre.leggauss
  * Pbar_lm and dPbar_lm/dtheta: scipy.special.sph_harm_y (diff_n=1)
  * scalar / vector synthesis: direct sums of Y_lm and its gradients at the grid
  * radial difference weights: numpy.linalg.solve of the transposed Vandermonde
  * one CNAB2 step with N = 0: dense numpy solve of (I/dt - theta L) x = (I/dt + (1-theta) L) u
The model trajectory fixture (``step_l7.npz``) is the oracle's own output and
pins regressions of the oracle and the CUDA path against each other.

Sizes follow the reference's own round-trip test (test/shtnskit_roundtrip.jl:
lmax = mmax = 6, nlat = 12, nlon = 24, nr = 6).  The reference seeds Julia's
RNG (Random.seed!(1234)); these fixtures use numpy's default_rng(1234).

Run:  python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np
from scipy.special import sph_harm_y

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def lm_pairs(lmax, mmax):
    return [(l, m) for l in range(lmax + 1) for m in range(min(l, mmax) + 1)]


def radial_nodes(nr, rratio=0.35):
    ri = rratio / (1.0 - rratio)
    n = np.arange(1, nr + 1)
    return 0.5 * (1.0 + np.cos(np.pi * (nr - n) / (nr - 1))) + ri


def fd_band(order, r, kl=4):
    """create_derivative_matrix with difference weights (V^T w = rhs), band layout (2kl+1, N)."""
    N = len(r)
    data = np.zeros((2 * kl + 1, N))
    for n in range(N):
        left, right = max(0, n - kl), min(N - 1, n + kl)
        S = right - left + 1
        V = np.ones((S, S))
        for j in range(1, S):
            V[:, j] = V[:, j - 1] * (r[left:right + 1] - r[n])
        rhs = np.zeros(S)
        if order <= S:
            rhs[order] = math.factorial(order)
        w = np.linalg.solve(V.T, rhs)
        for i, idx in enumerate(range(left, right + 1)):
            data[kl + n - idx, idx] = w[i]
    return data


def band_dense(b, kl=4):
    N = b.shape[1]
    A = np.zeros((N, N))
    for j in range(N):
        for i in range(max(0, j - kl), min(N, j + kl + 1)):
            A[i, j] = b[kl + i - j, j]
    return A


def main():
    lmax = mmax = 6
    nlat, nlon, nr = 12, 24, 6
    pairs = lm_pairs(lmax, mmax)
    nlm = len(pairs)
    x, w = np.polynomial.legendre.leggauss(nlat)
    x, w = x[::-1].copy(), w[::-1].copy()          # north -> south
    theta = np.arccos(x)
    phi = 2 * np.pi * np.arange(nlon) / nlon
    T, PH = np.meshgrid(theta, phi)                 # (nlon, nlat): reference grid layout per shell
    P = np.zeros((nlm, nlat // 2)); dP = np.zeros((nlm, nlat // 2))
    for q, (l, m) in enumerate(pairs):
        y, dy = sph_harm_y(l, m, theta[: nlat // 2], 0.0, diff_n=1)
        P[q] = y.real
        dP[q] = dy[..., 0].real

    rng = np.random.default_rng(1234)
    re = rng.standard_normal((nr, nlm)); im = rng.standard_normal((nr, nlm))
    M = np.array([m for _, m in pairs]); Lv = np.array([l for l, _ in pairs])
    im[:, M == 0] = 0.0
    grid = np.zeros((nr, nlon, nlat))
    for q, (l, m) in enumerate(pairs):
        Y = sph_harm_y(l, m, T, PH)
        a = re[:, q] + 1j * im[:, q]
        grid += (1 if m == 0 else 2) * (a[:, None, None] * Y).real

    tre = rng.standard_normal((nr, nlm)); tim = rng.standard_normal((nr, nlm))
    pre = rng.standard_normal((nr, nlm)); pim = rng.standard_normal((nr, nlm))
    for arr in (tim, pim):
        arr[:, M == 0] = 0.0
    for arr in (tre, tim, pre, pim):
        arr[:, Lv == 0] = 0.0
    vt = np.zeros((nr, nlon, nlat)); vp = np.zeros((nr, nlon, nlat))
    for q, (l, m) in enumerate(pairs):
        Y, dY = sph_harm_y(l, m, T, PH, diff_n=1)
        dYt = dY[..., 0]
        S = pre[:, q] + 1j * pim[:, q]; Tq = tre[:, q] + 1j * tim[:, q]
        f = 1 if m == 0 else 2
        vt += f * (S[:, None, None] * dYt + Tq[:, None, None] * 1j * m * Y / np.sin(T)).real
        vp += f * (S[:, None, None] * 1j * m * Y / np.sin(T) - Tq[:, None, None] * dYt).real
    np.savez_compressed(os.path.join(HERE, "sht_l6.npz"), x=x, w=w, theta=theta, P=P, dP=dP, re=re, im=im,
                        grid=grid, tre=tre, tim=tim, pre=pre, pim=pim, vt=vt, vp=vp,
                        dims=np.array([lmax, mmax, nlat, nlon, nr]))

    # radial operators and one CNAB2 step with N = 0 (nr = 12, l = 3, nu = 4, dt = 1e-5)
    nr2, kl = 12, 4
    r = radial_nodes(nr2)
    d1 = fd_band(1, r, kl); d2 = fd_band(2, r, kl)
    D1, D2 = band_dense(d1), band_dense(d2)
    nu, dt, th, l = 4.0, 1e-5, 0.5, 3
    Lop = nu * (D2 + np.diag(2.0 / r) @ D1) - nu * l * (l + 1) * np.diag(r ** -2.0)
    u = np.sin(np.pi * (r - r[0]) / (r[-1] - r[0])) + 0.1 * r
    rhs = u / dt + (1 - th) * (Lop @ u)
    x1 = np.linalg.solve(np.eye(nr2) / dt - th * Lop, rhs)
    np.savez_compressed(os.path.join(HERE, "radial_nr12.npz"), r=r, d1=d1, d2=d2, u=u, x1=x1,
                        params=np.array([nu, dt, th, l]))

    # small model trajectory from the oracle
    from oracle.oracle import Oracle
    sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
    import workloads
    lm7, nlat7, nlon7, nr7 = 7, 12, 24, 9
    st = workloads.seeded_state(lm7, lm7, nr7, seed=0, amp=1e-3)
    o = Oracle(lmax=lm7, nlat=nlat7, nlon=nlon7, nr=nr7, dt=1e-5)
    for k, (a, b) in st.items():
        o.set_field(k, a, b)
    o.step(1)
    nl1 = {f"nl_{k}_{c}": v for k in workloads.FIELD_ORDER for c, v in zip(("re", "im"), o.get_nl(k))}
    o.step(2)
    fin = {f"u3_{k}_{c}": v for k in workloads.FIELD_ORDER for c, v in zip(("re", "im"), o.get_field(k))}
    ek, em = o.energy()
    init = {f"u0_{k}_{c}": v for k, ab in st.items() for c, v in zip(("re", "im"), ab)}
    np.savez_compressed(os.path.join(HERE, "step_l7.npz"), dims=np.array([lm7, nlat7, nlon7, nr7]),
                        energy3=np.array([ek, em]), **init, **nl1, **fin)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()

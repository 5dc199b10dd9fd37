"""The reference applies EAB2's exponential and phi1 to the velocity and
magnetic fields through Krylov actions (eab2_update_krylov_cached!,
src/timestep.jl:358-427, m = 20, tol 1e-8); this build uses the dense per-l
matrices for every field.  Here the reference's actions, restated in
oracle/oracle.py, are compared with the dense operators on the implicit
operators A_l = nu (lap - l(l+1)/r^2) of the radial grids of the
configurations (nr = 12, 33, 129):

* the exponential action agrees with expm(dt A) v within the reference's own
  tolerance;
* its phi1 route, A^-1 (exp(dt A) v - v) / dt through the non-pivoting banded
  LU, is off by O(1) and more, because A_l has no boundary rows and is
  numerically singular (condition ~1e16-1e18): the dense series phi1 this
  build uses is the function itself (the exponential schemes' test checks
  dt A phi1 = E - I on the device)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

CASES = [(12, 1e-5), (33, 2e-6), (129, 2e-6)]


def operator(nr, dt, kind, l):
    o = O.Oracle(lmax=8, nlat=12, nlon=24, nr=nr, dt=dt)
    lin, _ = o.implicit_matrices(kind, l)
    return O.band_to_dense(lin, o.kl)


def phi1_series(A, dt):
    import scipy.linalg as sla
    n = A.shape[0]
    M = np.zeros((2 * n, 2 * n))
    M[:n, :n] = dt * A
    M[:n, n:] = np.eye(n)
    return sla.expm(M)[:n, n:]


@pytest.mark.parametrize("nr,dt", CASES)
def test_krylov_exponential_matches_dense(nr, dt):
    import scipy.linalg as sla
    for kind in (0, 1, 2):
        for l in (1, 4, 8):
            A = operator(nr, dt, kind, l)
            v = np.random.default_rng(10 * kind + l).standard_normal(nr)
            y, k = O.exp_action_krylov(A, v, dt)
            ex = sla.expm(dt * A) @ v
            err = np.max(np.abs(y - ex)) / np.max(np.abs(ex))
            assert err <= 1e-8, (nr, kind, l, k, err)


@pytest.mark.parametrize("nr,dt", CASES)
def test_krylov_phi1_route_is_unusable_on_the_singular_operator(nr, dt):
    worst = 0.0
    for l in (1, 4):
        A = operator(nr, dt, 0, l)
        assert np.linalg.cond(A) > 1e15
        v = np.random.default_rng(l).standard_normal(nr)
        x = O.phi1_action_krylov(A, v, dt)
        p = phi1_series(A, dt) @ v
        worst = max(worst, float(np.max(np.abs(x - p)) / np.max(np.abs(p))))
    assert worst > 1.0, worst

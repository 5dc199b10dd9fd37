"""CPU tests: the oracle's restatements of the exponential schemes' per-system
updates (oracle/oracle.py: eab2_update, erk2_prepare, erk2_finalize) against
the reference's own known answers (test/erk2.jl:4-78): a 1 x 1 system
du/dt = -lambda u + N with lambda = 0.5, dt = 0.1, whose matrices are the
scalar functions exp(z), phi1(z) = (e^z - 1)/z, phi2(z) = (e^z - 1 - z)/z^2 of
z = -lambda dt (and z/2).  The reference holds both scenarios to 1e-4; the
constant-forcing answers are exact for these schemes and are held to 1e-14
here."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle.oracle import eab2_update, erk2_finalize, erk2_prepare  # noqa: E402

LAM, DT = 0.5, 0.1


def scalar_matrices(z):
    e = math.exp(z)
    return np.array([[e]]), np.array([[(e - 1) / z]]), np.array([[(e - 1 - z) / z ** 2]])


def erk2(u0, nl):
    E, P1, P2 = scalar_matrices(-LAM * DT)
    Eh, P1h, _ = scalar_matrices(-LAM * DT / 2)
    u = np.array([[u0]])
    lin, k1, stage = erk2_prepare(E, P1, Eh, P1h, u, nl(u), DT)
    return float(erk2_finalize(P2, lin, k1, nl(u), nl(stage), DT)[0, 0])


def test_erk2_constant_forcing():
    # scenario 1 of test/erk2.jl: N = c
    u0, c = 0.3, 0.2
    expected = math.exp(-LAM * DT) * u0 + (1 - math.exp(-LAM * DT)) * c / LAM
    got = erk2(u0, lambda u: np.full_like(u, c))
    assert abs(got - expected) < 1e-14
    assert abs(got - expected) < 1e-4   # the reference's tolerance


def test_erk2_linear_forcing():
    # scenario 2 of test/erk2.jl: N(u) = beta u, the stage's N recomputed
    u0, beta = 0.45, 0.15
    expected = math.exp((beta - LAM) * DT) * u0
    got = erk2(u0, lambda u: beta * u)
    assert abs(got - expected) < 1e-4   # second order: the reference's tolerance
    assert abs(got - expected) > 0.0    # and not exact (the stage matters)


def test_eab2_constant_forcing():
    # E u + dt phi1 (3/2 c - 1/2 c) = exact solution with constant forcing
    u0, c = 0.3, 0.2
    E, P1, _ = scalar_matrices(-LAM * DT)
    got = float(eab2_update(E, P1, np.array([[u0]]), np.array([[c]]), np.array([[c]]), DT)[0, 0])
    expected = math.exp(-LAM * DT) * u0 + (1 - math.exp(-LAM * DT)) * c / LAM
    assert abs(got - expected) < 1e-14


def taylor_doubling(X, K=18):
    """The device's construction of the exponential cache (k_etd_build,
    geodynamo.jl_b200/csrc/gd_expo.cu), restated in numpy: Y = X / 2^s with
    ||Y||_1 <= 1/2 and s >= 1, truncated Taylor series of exp, phi1, phi2, then s
    doublings E <- E^2, P <- P (E + I) / 2, Q <- (2 Q + P^2) / 4; the half-step
    matrices are the state before the last doubling."""
    n = X.shape[0]
    eye = np.eye(n)
    s, v = 1, np.max(np.sum(np.abs(X), axis=0)) / 2
    while v > 0.5:
        v /= 2
        s += 1
    Y = X / 2.0 ** s
    E, P, Q, Pw = eye + Y, eye + Y / 2, eye / 2 + Y / 6, Y.copy()
    for k in range(2, K + 1):
        Pw = Pw @ Y / k
        E, P, Q = E + Pw, P + Pw / (k + 1), Q + Pw / ((k + 1) * (k + 2))
    half = None
    for it in range(s):
        if it == s - 1:
            half = (E.copy(), P.copy())
        Q = (2 * Q + P @ P) / 4
        P = P @ (E + eye) / 2
        E = E @ E
    return E, P, Q, half[0], half[1]


def test_device_cache_algorithm_matches_expm(oracle_mod):
    # at nr = 12 (||dt A||_1 ~ 0.3) and at the headline radial grid (nr = 129,
    # dt = 2e-6, ||dt A||_1 ~ 900): the tolerances the GPU tests hold the
    # device's cache to
    for nr, dt, tol in ((12, 1e-5, 1e-12), (129, 2e-6, 1e-9)):
        o = oracle_mod.Oracle(lmax=3, nlat=6, nlon=12, nr=nr, dt=dt)
        ref = o.etd_cache(2)
        for l in (0, 3):
            E, P, Q, Eh, Ph = taylor_doubling(dt * ref["A"][l])
            for got, key in ((E, "E"), (P, "phi1"), (Q, "phi2"), (Eh, "E_half"), (Ph, "phi1_half")):
                want = ref[key][l]
                assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < tol, (nr, l, key)

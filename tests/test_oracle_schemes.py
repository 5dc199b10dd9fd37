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

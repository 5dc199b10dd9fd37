"""GPU tests of the exponential Adams-Bashforth 2 scheme (ts_scheme = :eab2;
eab2_update!, src/timestep.jl:429-487, with the cache of create_etd_cache,
:37-70) through the C ABI.

Tolerances: the device's exponential cache against scipy's expm of the same
operator, relative to each matrix's max-norm: 1e-12 for E and phi1 (phi1 as
the top-right block of exp([[dt A, I], [0, 0]])) where ||dt A||_1 is of order
one (nr = 12, 33), 1e-9 at the headline radial grid (nr = 129, dt = 2e-6,
||dt A||_1 ~ 900: eleven doublings, and scipy's own result meets the identity
below only to ~7e-11); and the defining identity dt A phi1 = E - I.  The
reference forms phi1 as A^-1 (E - I) / dt (create_etd_cache): A_l carries no
boundary rows, so the radial equation's two homogeneous solutions make it
numerically singular (condition ~1e16 for every l) and that solve is not
usable; the identity pins phi1 instead.  Steps against the oracle's
restatement: FP64 1e-11, mixed precision 1e-5 (the trajectory tolerances of
the CNAB2 tests)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")
KINDS = ("velocity", "magnetic", "temperature")


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("lmax,nr,dt,tol", [(7, 12, 1e-5, 1e-12), (7, 33, 2e-6, 1e-12), (3, 129, 2e-6, 1e-9)])
def test_etd_cache_matches_expm(gdb, oracle_mod, lmax, nr, dt, tol):
    nlat = 2 * (lmax + 1) if lmax > 3 else 6
    g = gdb.SHTnsKitConfig(lmax, nlat, 2 * nlat, nr, dt=dt)
    g.set_scheme("eab2")
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=2 * nlat, nr=nr, dt=dt)
    for kind, name in enumerate(KINDS):
        A, E, P = o.etd_cache(kind)
        for l in sorted({0, 1, lmax // 2, lmax}):
            Eg, Pg = g.etd_matrices(name, l)
            assert rel(Eg, E[l]) < tol, (name, l)
            assert rel(Pg, P[l]) < tol, (name, l)
            assert rel(dt * A[l] @ Pg, Eg - np.eye(nr)) < max(tol, 1e-13), (name, l)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_eab2_steps_match_oracle(gdb, oracle_mod, precision, tol):
    dims = dict(lmax=15, nlat=24, nlon=48, nr=12)
    g = gdb.SHTnsKitConfig(15, 24, 48, 12, precision=precision)
    g.set_scheme("eab2")
    o = oracle_mod.Oracle(**dims)
    for k, (a, b) in workloads.seeded_state(15, 15, 12, seed=9).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    caches = [o.etd_cache(kind) for kind in range(3)]
    history = {}
    # the first step reads a zero history (no AB1 start); the later ones the rolled terms
    for n in range(3):
        g.step(1)
        o.eab2_step(caches, history)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < tol and rel(a[1], b[1]) < tol, (n, k)


def test_eab2_graph_replay_and_scheme_switch(gdb):
    st = workloads.seeded_state(15, 15, 12, seed=10)
    a = gdb.SHTnsKitConfig(15, 24, 48, 12)
    b = gdb.SHTnsKitConfig(15, 24, 48, 12)
    for m in (a, b):
        m.set_scheme("eab2")
        for k, (x, y) in st.items():
            m.set_field(k, x, y)
    a.step(4)                      # graph replays
    for _ in range(4):
        b.temperature_nl(); b.velocity_nl(); b.magnetic_nl(); b.implicit_step()
    for k in NAMES:
        x, y = a.get_field(k), b.get_field(k)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), k
    a.set_scheme("cnab2")          # back to the banded solve: graphs are rebuilt
    a.step(1)
    assert a.step_count() == 5


def test_eab2_rejects_unsupported_configurations(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 12, bc_mode=2)
    with pytest.raises(gdb.GeoDynamoError):
        g.set_scheme("eab2")
    h = gdb.SHTnsKitConfig(3, 6, 12, 300)
    with pytest.raises(gdb.GeoDynamoError):
        h.set_scheme("eab2")
    with pytest.raises(gdb.GeoDynamoError):
        h.etd_matrices("velocity", 0)      # no cache under CNAB2

"""GPU tests of the exponential time schemes through the C ABI: EAB2
(ts_scheme = :eab2; eab2_update!, src/timestep.jl:429-487) and ERK2
(ts_scheme = :erk2; erk2_integrate_full_step!, src/simulation.jl:1054-1149),
with the caches of create_etd_cache / create_erk2_cache (src/timestep.jl:37-70,
896-968) built on the device.

Tolerances: the device's cache against scipy's expm of the same operator
(phi1 and phi2 as blocks of exp([[X, I, 0], [0, 0, I], [0, 0, 0]])), relative to
each matrix's max-norm: 1e-12 where ||dt A||_1 is of order one (nr = 12, 33),
1e-9 at the headline radial grid (nr = 129, dt = 2e-6, ||dt A||_1 ~ 900: eleven
doublings); and the defining identities dt A phi1 = E - I and
dt A phi2 = phi1 - I.  The reference forms phi1 and phi2 with A^-1: A_l
carries no boundary rows, so the radial equation's two homogeneous solutions
make it numerically singular (condition ~1e16 for every l) and those solves
are not usable; the identities pin the functions instead.  Steps against the
oracle's restatement: FP64 1e-11, mixed precision 1e-5 (the trajectory
tolerances of the CNAB2 tests)."""
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
def test_exponential_cache_matches_expm(gdb, oracle_mod, lmax, nr, dt, tol):
    nlat = 2 * (lmax + 1) if lmax > 3 else 6
    g = gdb.SHTnsKitConfig(lmax, nlat, 2 * nlat, nr, dt=dt)
    g.set_scheme("erk2")
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=2 * nlat, nr=nr, dt=dt)
    eye = np.eye(nr)
    for kind, name in enumerate(KINDS):
        ref = o.etd_cache(kind)
        for l in sorted({0, 1, lmax // 2, lmax}):
            got = g.etd_matrices(name, l)
            for key in ("E", "phi1", "phi2", "E_half", "phi1_half"):
                assert rel(got[key], ref[key][l]) < tol, (name, l, key)
            A = ref["A"][l]
            assert rel(dt * A @ got["phi1"], got["E"] - eye) < max(tol, 1e-13), (name, l)
            assert rel(dt * A @ got["phi2"], got["phi1"] - eye) < max(tol, 1e-13), (name, l)
            assert rel(0.5 * dt * A @ got["phi1_half"], got["E_half"] - eye) < max(tol, 1e-13), (name, l)


def model_and_oracle(gdb, oracle_mod, scheme, precision, seed):
    g = gdb.SHTnsKitConfig(15, 24, 48, 12, precision=precision)
    g.set_scheme(scheme)
    o = oracle_mod.Oracle(lmax=15, nlat=24, nlon=48, nr=12)
    for k, (a, b) in workloads.seeded_state(15, 15, 12, seed=seed).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    return g, o, [o.etd_cache(kind) for kind in range(3)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_eab2_steps_match_oracle(gdb, oracle_mod, precision, tol):
    g, o, caches = model_and_oracle(gdb, oracle_mod, "eab2", precision, seed=9)
    history = {}
    # the first step reads a zero history (no AB1 start); the later ones the rolled terms
    for n in range(3):
        g.step(1)
        o.eab2_step(caches, history)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < tol and rel(a[1], b[1]) < tol, (n, k)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_erk2_steps_match_oracle(gdb, oracle_mod, precision, tol):
    g, o, caches = model_and_oracle(gdb, oracle_mod, "erk2", precision, seed=11)
    for n in range(3):
        g.step(1)
        o.erk2_step(caches)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < tol and rel(a[1], b[1]) < tol, (n, k)
    # the closing evaluation's nonlinear terms (state.nonlinear after the step)
    for k in NAMES:
        a, b = g.get_nl(k), o.get_nl(k)
        assert rel(a[0], b[0]) < max(tol, 1e-10), k


@pytest.mark.parametrize("scheme", ["eab2", "erk2"])
def test_exponential_schemes_with_mmax_below_lmax(gdb, oracle_mod, scheme):
    # a degree l > mmax has mmax + 1 orders, not l + 1: the column blocks of
    # the apply kernel and the oracle's per-degree blocks must agree
    g = gdb.SHTnsKitConfig(12, 20, 40, 10, mmax=6)
    g.set_scheme(scheme)
    o = oracle_mod.Oracle(lmax=12, nlat=20, nlon=40, nr=10, mmax=6)
    for k, (a, b) in workloads.seeded_state(12, 6, 10, seed=13).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    caches = [o.etd_cache(kind) for kind in range(3)]
    history = {}
    for n in range(2):
        g.step(1)
        if scheme == "eab2":
            o.eab2_step(caches, history)
        else:
            o.erk2_step(caches)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < 1e-11 and rel(a[1], b[1]) < 1e-11, (n, k)


def test_eab2_cuda_core_apply_matches_oracle(gdb, oracle_mod):
    # nr = 160 > 144 takes the CUDA-core apply kernel instead of the FP64
    # tensor-core one (two steps: a zero history, then the rolled one); 1e-9 as
    # for the cache at this size (||dt A||_1 ~ 1000)
    g = gdb.SHTnsKitConfig(7, 12, 24, 160, dt=1e-6)
    g.set_scheme("eab2")
    o = oracle_mod.Oracle(lmax=7, nlat=12, nlon=24, nr=160, dt=1e-6)
    for k, (a, b) in workloads.seeded_state(7, 7, 160, seed=12).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    caches = [o.etd_cache(kind) for kind in range(3)]
    history = {}
    for n in range(2):
        g.step(1)
        o.eab2_step(caches, history)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < 1e-9 and rel(a[1], b[1]) < 1e-9, (n, k)


@pytest.mark.parametrize("scheme", ["eab2", "erk2"])
def test_exponential_graph_replay_and_scheme_switch(gdb, scheme):
    st = workloads.seeded_state(15, 15, 12, seed=10)
    a = gdb.SHTnsKitConfig(15, 24, 48, 12)
    b = gdb.SHTnsKitConfig(15, 24, 48, 12)
    for m in (a, b):
        m.set_scheme(scheme)
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


def test_exponential_schemes_reject_unsupported_configurations(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 12, bc_mode=2)
    for scheme in ("eab2", "erk2"):
        with pytest.raises(gdb.GeoDynamoError):
            g.set_scheme(scheme)
    h = gdb.SHTnsKitConfig(3, 6, 12, 300)
    with pytest.raises(gdb.GeoDynamoError):
        h.set_scheme("erk2")
    with pytest.raises(gdb.GeoDynamoError):
        h.etd_matrices("velocity", 0)      # no cache under CNAB2


@pytest.mark.parametrize("nr,dt", [(33, 2e-6), (129, 2e-6)])
def test_device_exponential_matches_reference_krylov_action(gdb, oracle_mod, nr, dt):
    # the reference's EAB2 applies E to velocity and magnetic fields by a Krylov
    # action (eab2_update_krylov_cached!, src/timestep.jl:358-427, m = 20,
    # tol 1e-8): the device's dense E gives the same vectors within that tolerance
    g = gdb.SHTnsKitConfig(7, 12, 24, nr, dt=dt)
    g.set_scheme("eab2")
    o = oracle_mod.Oracle(lmax=7, nlat=12, nlon=24, nr=nr, dt=dt)
    for k, kind in enumerate(KINDS):
        for l in (1, 5):
            E = g.etd_matrices(kind, l)["E"]
            lin, _ = o.implicit_matrices(k, l)
            A = oracle_mod.band_to_dense(lin, o.kl)
            v = np.random.default_rng(7 * k + l).standard_normal(nr)
            y, _ = oracle_mod.exp_action_krylov(A, v, dt)
            assert rel(E @ v, y) <= 1e-8, (kind, l, rel(E @ v, y))
    g.close()


@pytest.mark.parametrize("scheme", ["eab2", "erk2"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_exponential_schemes_with_composition(gdb, oracle_mod, scheme, precision, tol):
    # composition (kind 3, nu = Pm/Sc) steps with the same dense operators: the
    # reference's EAB2 applies them by Krylov (src/simulation.jl:1286-1290), its
    # ERK2 with the dense caches (:1094-1145); compute_all_nonlinear_terms!
    # ends with the composition phase
    kw = dict(composition=1, schmidt=2.5, dt=2e-6)
    g = gdb.SHTnsKitConfig(15, 24, 48, 12, precision=precision, **kw)
    g.set_scheme(scheme)
    o = oracle_mod.Oracle(lmax=15, nlat=24, nlon=48, nr=12, **kw)
    for k, (a, b) in workloads.seeded_state(15, 15, 12, seed=13).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    cst = workloads.seeded_state(15, 15, 12, seed=113)["temp"]
    g.set_field("comp", *cst)
    o.set_field("comp", *cst)
    cbv = np.random.default_rng(6).standard_normal((2, g.nlm)) * 1e-3
    g.set_composition_bc(cbv, np.linspace(-0.2, 0.2, 12))
    o.set_composition_bc(cbv, np.linspace(-0.2, 0.2, 12))
    got = g.etd_matrices("composition", 3)
    caches = [o.etd_cache(kind) for kind in range(4)]
    assert rel(got["E"], caches[3]["E"][3]) < 1e-12
    history = {}
    for n in range(3):
        g.step(1)
        if scheme == "eab2":
            o.eab2_step(caches, history)
        else:
            o.erk2_step(caches)
        for k in NAMES + ("comp",):
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < tol and rel(a[1], b[1]) < tol, (n, k)

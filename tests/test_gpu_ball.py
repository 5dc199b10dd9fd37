"""Ball geometry (GeoDynamoBall, src/Ball/Ball.jl) on the device against the
FP64 oracle: the analyses with regularity (ball_physical_to_spectral!,
ball_vector_analysis!), the r = 0 guards of the gradient and curl kernels
(test/ball_finiteness.jl), the ball step with the boundary-row operator
(bc_mode 2) in FP64 at 1e-12 and mixed precision at 5e-6, regularity of the
state and of the nonlinear terms, segmented ball handles bit for bit, and the
refused combinations."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = workloads.FIELD_ORDER


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def l_of(lmax):
    return np.array([l for l in range(lmax + 1) for m in range(l + 1)])


def regular_state(lmax, nr, seed):
    st = workloads.seeded_state(lmax, lmax, nr, seed=seed, amp=1e-1)
    lpos = l_of(lmax) > 0
    for k, (a, b) in st.items():
        a[0, lpos] = 0.0
        b[0, lpos] = 0.0
    return st


def pair(gdb, oracle_mod, lmax, nlat, nlon, nr, precision="fp64", seed=0, r_outer=1.0, **kw):
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, geometry="ball", bc_mode=2,
                           r_outer=r_outer, **kw)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, geometry="ball", bc_mode=2, r_outer=r_outer, **kw)
    for m in (g, o):
        for k, (a, b) in regular_state(lmax, nr, seed).items():
            m.set_field(k, a, b)
    rng = np.random.default_rng(seed + 7)
    bv = np.zeros((2, g.nlm))
    bv[0, 0] = 0.4                                # the l = 0 temperature at the centre
    bv[1] = rng.standard_normal(g.nlm) * 1e-2     # outer values
    src = np.linspace(0.5, 1.0, nr)
    for m in (g, o):
        m.set_temperature_bc(bv, src)
    return g, o


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_ball_analyses_match_oracle(gdb, oracle_mod, precision, tol):
    lmax, nlat, nlon, nr = 6, 12, 24, 6   # test/ball_roundtrip.jl's sizes
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, geometry="ball", bc_mode=2)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, geometry="ball", bc_mode=2)
    rng = np.random.default_rng(3)
    lpos = l_of(lmax) > 0
    grid = rng.standard_normal(g.grid_shape())
    a = g.analysis_scalar(grid, ball=True)
    b = o.analysis_scalar(grid, ball=True)
    for x, y in zip(a, b):
        assert rel(x, y) < tol
        assert np.all(x[0, lpos] == 0.0)
    # without the ball flag the first level is the plain analysis
    plain = g.analysis_scalar(grid)
    assert np.any(plain[0][0, lpos] != 0.0)
    vt, vp = rng.standard_normal(g.grid_shape()), rng.standard_normal(g.grid_shape())
    av = g.analysis_vector(vt, vp, ball=True)
    bvv = o.analysis_vector(vt, vp, ball=True)
    for x, y in zip(av, bvv):
        assert rel(x, y) < tol
        assert np.all(x[0, lpos] == 0.0)


def test_ball_centre_is_finite(gdb, oracle_mod):
    # test/ball_finiteness.jl: random potentials with no regularity enforced;
    # vorticity and current density are finite and 0 at r = 0, and so are the
    # grids synthesised from them; the angular temperature gradient too
    lmax, nlat, nlon, nr = 6, 12, 24, 6
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, geometry="ball", bc_mode=2)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, geometry="ball", bc_mode=2)
    st = workloads.seeded_state(lmax, lmax, nr, seed=4, amp=1.0)
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.temperature_nl()
        m.velocity_nl()
        m.magnetic_nl()
    for name in ("w_th", "w_ph", "j_th", "j_ph", "gth", "gph"):
        x = g.get_grid(name)
        assert np.all(np.isfinite(x)), name
        assert np.all(x[0] == 0.0), name
        assert rel(x, o.get_grid(name)) < 1e-12, name
    assert np.all(np.isfinite(g.get_grid("gr")))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_ball_step_matches_oracle(gdb, oracle_mod, precision, tol):
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    g, o = pair(gdb, oracle_mod, lmax, nlat, nlon, nr, precision=precision, dt=2e-6)
    g.step(3)
    o.step(3)
    lpos = l_of(lmax) > 0
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert np.all(np.isfinite(x)), k
            assert rel(x, y) < tol, k
            assert np.all(x[0, lpos] == 0.0), k
    for k in ("temp", "b_tor", "b_pol"):
        for x in g.get_nl(k):
            assert np.all(x[0, lpos] == 0.0), k
    assert g.get_field("temp")[0][0, 0] == 0.4
    ek, em = g.energy()
    ok, om = o.energy()
    assert abs(ek - ok) <= tol * abs(ok) and abs(em - om) <= tol * abs(om)


def test_ball_r_outer_matches_oracle(gdb, oracle_mod):
    g, o = pair(gdb, oracle_mod, 7, 12, 24, 9, r_outer=2.0, dt=1e-5)
    g.step(2)
    o.step(2)
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < 1e-12, k


def test_segmented_ball_equals_single_balls(gdb):
    cfg = dict(lmax=15, nlat=24, nlon=48, nr=12, geometry="ball", bc_mode=2, dt=2e-6)
    members = [dict(cfg, ekman=e) for e in (3e-4, 1e-3)]
    ens = gdb.Ensemble(members, group=2)
    assert len(ens.handles) == 1
    singles = []
    for i, (c, m) in enumerate(zip(members, ens.members)):
        st = regular_state(15, 12, seed=10 + i)
        kw = {k: v for k, v in c.items() if k not in ("lmax", "nlat", "nlon", "nr")}
        s = gdb.SHTnsKitConfig(15, 24, 48, 12, **kw)
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
            s.set_field(k, a, b)
        singles.append(s)
    ens.step(3)
    for s in singles:
        s.step(3)
    for m, s in zip(ens.members, singles):
        for k in NAMES:
            a, b = m.get_field(k), s.get_field(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), k
        assert m.energy() == s.energy()
    ens.close()


def test_ball_enforce_regularity(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=2)
    st = workloads.seeded_state(7, 7, 9, seed=5, amp=1.0)
    lpos = l_of(7) > 0
    for k, (a, b) in st.items():
        g.set_field(k, a, b)
        g.enforce_regularity(k)
        x = g.get_field(k)
        assert np.all(x[0][0, lpos] == 0.0) and np.all(x[1][0, lpos] == 0.0)
        assert np.array_equal(x[0][0, ~lpos], a[0, ~lpos])
        assert np.array_equal(x[0][1:], a[1:])


def test_ball_refusals(gdb):
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=0)
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=2, r_outer=0.0)
    g = gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=2)
    with pytest.raises(gdb.GeoDynamoError):
        g.set_scheme("eab2")
    with pytest.raises(gdb.GeoDynamoError):
        g.set_external_derivatives(True)
    with pytest.raises(gdb.GeoDynamoError):
        g.temperature_forward(2, 1)
    g.step(1)
    g.check_finite()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_ball_with_composition_matches_oracle(gdb, oracle_mod, precision, tol):
    # composition in the ball: regularity of its analysed term and of its state
    # (src/compositional.jl:245-246, 368-370), the centre value of its l = 0 row
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    kw = dict(geometry="ball", bc_mode=2, composition=1, schmidt=2.0, dt=2e-6)
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, **kw)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, **kw)
    st = regular_state(lmax, nr, seed=3)
    cst = regular_state(lmax, nr, seed=103)["temp"]
    cbv = np.zeros((2, g.nlm))
    cbv[0, 0] = -0.3
    cbv[1] = np.random.default_rng(5).standard_normal(g.nlm) * 1e-2
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("comp", *cst)
        m.set_composition_bc(cbv, np.linspace(0.1, 0.4, nr))
    g.step(3)
    o.step(3)
    lpos = l_of(lmax) > 0
    for k in NAMES + ("comp",):
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < tol, k
            assert np.all(x[0, lpos] == 0.0), k
    for x in g.get_nl("comp"):
        assert np.all(x[0, lpos] == 0.0)
    assert g.get_field("comp")[0][0, 0] == -0.3


def test_ball_with_outer_flux_matches_oracle(gdb, oracle_mod):
    # a full sphere with a prescribed heat flux at its surface: the outer row of
    # the implicit solve is the row of D1; the centre keeps its regularity row
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    g, o = pair(gdb, oracle_mod, lmax, nlat, nlon, nr, dt=2e-6)
    inner = np.ones(g.nlm, dtype=int)
    outer = np.full(g.nlm, 2)
    for m in (g, o):
        m.set_bc_types("temp", inner, outer)
    g.step(3)
    o.step(3)
    lpos = l_of(lmax) > 0
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < 1e-12, k
            assert np.all(x[0, lpos] == 0.0), k

"""The oracle's ball geometry (GeoDynamoBall, src/Ball/Ball.jl) on the CPU.

The reference's own ball tests are restated here with their sizes and
tolerances: test/ball_roundtrip.jl (random physical fields analysed with
regularity: the r = 0 level is 0 for l >= 1, atol 1e-12, scalar and vector)
and test/ball_finiteness.jl (vorticity and current density finite and 0 at
r = 0 for random potentials, atol 1e-12).  Beyond them: the radial domain of
create_ball_radial_domain, the angular gradient at r = 0, and a ball step with
the boundary-row operator (bc_mode 2; the reference's operator is infinite at
r = 0) that stays finite and regular."""
import numpy as np
import pytest

LMAX, NLAT, NLON, NR = 6, 12, 24, 6   # the reference ball tests' configuration


def ball(oracle_mod, **kw):
    kw.setdefault("bc_mode", 2)
    return oracle_mod.Oracle(lmax=LMAX, nlat=NLAT, nlon=NLON, nr=NR, geometry="ball", **kw)


def l_of(o):
    return np.array([l for l in range(o.lmax + 1) for m in range(min(l, o.mmax) + 1)])


def test_ball_radial_domain(oracle_mod):
    o = ball(oracle_mod)
    _, _, _, r = o.grid()
    n = np.arange(1, NR + 1)
    want = 0.5 * (1.0 + np.cos(np.pi * (NR - n) / (NR - 1)))
    assert r[0] == 0.0 and r[-1] == pytest.approx(1.0, abs=1e-15)
    assert np.allclose(r, want, atol=1e-15)
    o2 = ball(oracle_mod, r_outer=2.5)
    assert np.allclose(o2.grid()[3], 2.5 * want, atol=1e-14)


def test_ball_roundtrip_regularity(oracle_mod):
    o = ball(oracle_mod)
    rng = np.random.default_rng(0)
    lpos = l_of(o) > 0
    re, im = o.analysis_scalar(rng.standard_normal(o.grid_shape()), ball=True)
    assert np.all(np.abs(re[0, lpos]) <= 1e-12) and np.all(np.abs(im[0, lpos]) <= 1e-12)
    # the l = 0 mode and the other levels are the plain analysis
    pre, pim = o.analysis_scalar(rng.standard_normal(o.grid_shape()) * 0 + 1.0, ball=False)
    assert abs(pre[0, 0]) > 0
    vt, vp = rng.standard_normal(o.grid_shape()), rng.standard_normal(o.grid_shape())
    tr, ti, pr, pi = o.analysis_vector(vt, vp, ball=True)
    plain = o.analysis_vector(vt, vp)
    for a, b in zip((tr, ti, pr, pi), plain):
        assert np.all(np.abs(a[0, lpos]) <= 1e-12)
        assert np.array_equal(a[1:], b[1:])


def test_ball_finiteness_at_centre(oracle_mod):
    o = ball(oracle_mod)
    rng = np.random.default_rng(1)
    sh = o.spec_shape()
    tre, tim, pre, pim = (rng.standard_normal(sh) for _ in range(4))
    out = o.curl(tre, tim, pre, pim)
    for a in out:
        assert np.all(np.isfinite(a[0])) and np.all(np.abs(a[0]) <= 1e-12)
        assert np.all(np.isfinite(a))
    g = o.gradients(tre, tim)
    assert np.all(np.isfinite(g))
    assert np.all(g[:4, 0] == 0.0)          # angular components at r = 0
    assert np.any(g[4:, 0] != 0.0)          # the radial derivative is kept


def test_ball_step_stays_regular(oracle_mod):
    o = ball(oracle_mod, dt=1e-4)
    rng = np.random.default_rng(2)
    sh = o.spec_shape()
    lpos = l_of(o) > 0
    m0 = np.array([m for l in range(o.lmax + 1) for m in range(min(l, o.mmax) + 1)]) == 0
    for name in ("u_tor", "u_pol", "b_tor", "b_pol", "temp"):
        re, im = 1e-2 * rng.standard_normal(sh), 1e-2 * rng.standard_normal(sh)
        im[:, m0] = 0.0
        re[0, lpos] = 0.0
        im[0, lpos] = 0.0
        o.set_field(name, re, im)
    bv = np.zeros((2, o.nlm))
    bv[0, 0] = 0.7   # the l = 0 temperature at r = 0 (the inner boundary value)
    bv[1, 0] = 0.2
    o.set_temperature_bc(bv)
    o.step(3)
    for name in ("u_tor", "u_pol", "b_tor", "b_pol", "temp"):
        re, im = o.get_field(name)
        assert np.all(np.isfinite(re)) and np.all(np.isfinite(im)), name
        assert np.all(re[0, lpos] == 0.0) and np.all(im[0, lpos] == 0.0), name
    tre, _ = o.get_field("temp")
    assert tre[0, 0] == 0.7 and tre[-1, 0] == 0.2
    for name in ("temp", "b_tor", "b_pol"):
        nre, nim = o.get_nl(name)
        assert np.all(nre[0, lpos] == 0.0) and np.all(nim[0, lpos] == 0.0), name
    ek, em = o.energy()
    assert np.isfinite(ek) and np.isfinite(em) and ek > 0


def test_literal_operator_is_infinite_at_centre(oracle_mod):
    # create_shtns_timestepping_matrices (src/timestep.jl:498-543) on the ball
    # domain: the r = 0 row holds nu (2/r) D1 and nu l(l+1)/r^2, infinite (and
    # 0 x inf at l = 0); which is why the ball steps with bc_mode 2
    o = ball(oracle_mod, bc_mode=0)
    for l in (0, 1, 3):
        lin, _ = o.implicit_matrices(2, l)
        assert not np.all(np.isfinite(lin)), l
    b = ball(oracle_mod, bc_mode=2)
    for l in (0, 1, 3):
        _, lu = b.implicit_matrices(2, l)
        assert np.all(np.isfinite(lu)), l

"""Reverse mode of the velocity equation on the device.

In the reference's step the velocity's nonlinear term is its Coriolis term
alone (the cross products u x w and j x B have zero theta and phi components
with zero radial components, src/velocity.jl:447-548, 638-672), a linear map N
of u, and nothing else feeds the velocity (no buoyancy in the vector analysis,
Q2).  Checked here:

- gd_velocity_nl_adjoint against the forward term by the dot-product identity
  <N x, y> = <x, N^T y> in the real coefficient arrays (1e-12);
- gd_velocity_pullback against central differences of
  J(u0) = 1/2 sum |u^K|^2 + <c, u^K> after K steps (the dynamics are linear,
  so the difference quotient is exact up to rounding), under bc_mode 0, 1, 2,
  including a start from a later step count (no bootstrap in the window)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

LMAX, NLAT, NLON, NR = 15, 24, 48, 12


def rnd(rng, shape, m0):
    re, im = rng.standard_normal(shape), rng.standard_normal(shape)
    im[:, m0] = 0.0
    return re, im


def m0_mask(lmax):
    return np.array([m for l in range(lmax + 1) for m in range(l + 1)]) == 0


def test_velocity_nl_adjoint_dot_product(gdb):
    torch = pytest.importorskip("torch")
    g = gdb.SHTnsKitConfig(LMAX, NLAT, NLON, NR)
    rng = np.random.default_rng(1)
    m0 = m0_mask(LMAX)
    sh = g.spec_shape()
    xt, xp = rnd(rng, sh, m0), rnd(rng, sh, m0)
    yt, yp = rnd(rng, sh, m0), rnd(rng, sh, m0)
    for k in ("b_tor", "b_pol", "temp"):
        g.set_field(k, np.zeros(sh), np.zeros(sh))
    g.set_field("u_tor", *xt)
    g.set_field("u_pol", *xp)
    g.velocity_nl()
    nt, np_ = g.get_nl("u_tor"), g.get_nl("u_pol")
    se = 2 * NR * g.nlm
    psi = torch.zeros(2 * se, dtype=torch.float64, device="cuda")
    out = torch.zeros(2 * se, dtype=torch.float64, device="cuda")
    g.spectral_to_device(*yt, psi[:se])
    g.spectral_to_device(*yp, psi[se:])
    g.velocity_nl_adjoint(psi, out)
    at, ap = g.spectral_from_device(out[:se]), g.spectral_from_device(out[se:])
    lhs = sum(float(np.sum(a * b)) for a, b in zip(nt + np_, yt + yp))
    rhs = sum(float(np.sum(a * b)) for a, b in zip(xt + xp, at + ap))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1e-300), (lhs, rhs)
    assert abs(lhs) > 0


def run_velocity(gdb, u0, steps, pre=0, **kw):
    g = gdb.SHTnsKitConfig(LMAX, NLAT, NLON, NR, **kw)
    st = workloads.seeded_state(LMAX, LMAX, NR, seed=7)
    for k in ("b_tor", "b_pol", "temp"):
        g.set_field(k, *st[k])
    g.set_field("u_tor", *st["u_tor"])
    g.set_field("u_pol", *st["u_pol"])
    if pre:
        g.step(pre)
    g.set_field("u_tor", *u0[0])
    g.set_field("u_pol", *u0[1])
    g.step(steps)
    return g, (g.get_field("u_tor"), g.get_field("u_pol"))


@pytest.mark.parametrize("bc_mode,pre", [(0, 0), (1, 0), (2, 0), (2, 3)])
def test_velocity_pullback_matches_central_differences(gdb, bc_mode, pre):
    K = 8
    kw = dict(bc_mode=bc_mode, dt=2e-6)
    rng = np.random.default_rng(2 + bc_mode + pre)
    m0 = m0_mask(LMAX)
    sh = (NR, (LMAX + 1) * (LMAX + 2) // 2)
    u0 = (rnd(rng, sh, m0), rnd(rng, sh, m0))
    u0 = tuple(tuple(1e-2 * a for a in f) for f in u0)
    c = (rnd(rng, sh, m0), rnd(rng, sh, m0))

    def J(u):
        _, uk = run_velocity(gdb, u, K, pre=pre, **kw)
        return sum(0.5 * float(np.sum(a * a)) + float(np.sum(a * b))
                   for f, cf in zip(uk, c) for a, b in zip(f, cf))

    g, uk = run_velocity(gdb, u0, K, pre=pre, **kw)
    # the pullback of the K steps g has just run (its bootstrap pattern from
    # the step count they began at)
    lam = [tuple(a + b for a, b in zip(f, cf)) for f, cf in zip(uk, c)]
    gt, gp = g.velocity_pullback(K, lam[0], lam[1])
    for trial in range(3):
        v = (rnd(rng, sh, m0), rnd(rng, sh, m0))
        eps = 1e-3
        up = tuple(tuple(a + eps * b for a, b in zip(f, vf)) for f, vf in zip(u0, v))
        um = tuple(tuple(a - eps * b for a, b in zip(f, vf)) for f, vf in zip(u0, v))
        fd = (J(up) - J(um)) / (2 * eps)
        ad = sum(float(np.sum(a * b)) for a, b in zip(gt + gp, v[0] + v[1]))
        assert abs(fd - ad) <= 1e-7 * max(abs(fd), 1e-300), (bc_mode, pre, trial, fd, ad)


def test_velocity_pullback_refusals(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 9)
    z = np.zeros(g.spec_shape())
    with pytest.raises(gdb.GeoDynamoError):
        g.velocity_pullback(2, (z, z), (z, z))  # no steps run yet
    g.set_scheme("eab2")
    g.step(2)
    with pytest.raises(gdb.GeoDynamoError):
        g.velocity_pullback(2, (z, z), (z, z))
    b = gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=2)
    with pytest.raises(gdb.GeoDynamoError):
        b.velocity_pullback(2, (z, z), (z, z))

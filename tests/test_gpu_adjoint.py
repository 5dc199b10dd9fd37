"""GPU tests of the reverse-mode pieces (gd_spectral_to_physical_adjoint,
gd_magnetic_pullback) and of the adjoint configuration's gradient: misfit of
the radial magnetic field at r = ro after 200 steps (lmax 63, nr 65, literal
boundaries) with respect to the initial poloidal magnetic coefficients.

Tolerances: dot-product (transpose) identities to 1e-12 (synthesis) and
1e-10 (seven steps of the implicit propagator) relative in FP64; the
gradient against FP64 central finite differences of the full GPU step and
against the forward-mode derivative of the oracle's step to 1e-6 relative, the
requirement of the adjoint configuration.  The objective is quadratic in the
initial B_pol (the field evolves linearly), so central differences carry no
truncation error and the forward-mode derivative of the oracle is its step
applied to the direction."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")
CFG = workloads.CONFIGS["adjoint_l63_nr65"]


def dot(a, b):
    return float(np.sum(a[0] * b[0]) + np.sum(a[1] * b[1]))


def test_synthesis_adjoint_is_the_transpose(gdb):
    g = gdb.SHTnsKitConfig(10, 18, 36, 3)
    re, im = workloads.transform_batch(10, 10, 3, 2, seed=5)
    grid = np.random.default_rng(6).standard_normal((2,) + g.grid_shape())
    lhs = float(np.sum(g.synth_scalar(re, im) * grid))
    are, aim = g.synth_scalar_adjoint(grid)
    rhs = float(np.sum(re * are) + np.sum(im * aim))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("bc_mode", [0, 1, 2])
def test_magnetic_pullback_is_the_transposed_propagator(gdb, bc_mode):
    # <M^K u, lam> = <u, (M^T)^K lam>, with M^K u from the full step on a
    # state whose only nonzero field is B_pol
    lmax, nlat, nlon, nr, K = 15, 24, 48, 12, 7
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, dt=1e-5, bc_mode=bc_mode)
    rng = np.random.default_rng(7)
    u = workloads.adjoint_directions(lmax, lmax, nr, count=1, seed=8)[0]
    lam = (rng.standard_normal(g.spec_shape()), rng.standard_normal(g.spec_shape()))
    zero = np.zeros(g.spec_shape())
    for k in NAMES:
        g.set_field(k, zero, zero)
    g.set_field("b_pol", *u)
    g.step(K)
    lhs = dot(g.get_field("b_pol"), lam)
    rhs = dot(u, g.magnetic_pullback("b_pol", K, *lam))
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1e-300), (lhs, rhs)


def make(gdb, state, bpol=None):
    m = gdb.SHTnsKitConfig(CFG["lmax"], CFG["nlat"], CFG["nlon"], CFG["nr"], dt=CFG["dt"], bc_mode=CFG["bc_mode"])
    for k, (a, b) in state.items():
        m.set_field(k, a, b)
    if bpol is not None:
        m.set_field("b_pol", *bpol)
    return m


def target_grid(model):
    tre, tim = workloads.adjoint_target(CFG["lmax"], CFG["lmax"], seed=1)
    re = np.zeros(model.spec_shape()); im = np.zeros(model.spec_shape())
    re[-1] = tre; im[-1] = tim
    return model.synth_scalar(re, im)[-1]


def misfit(gdb, state, bpol, target):
    m = make(gdb, state, bpol)
    m.step(CFG["steps"])
    r = gdb.radial_field_outer(m, *m.get_field("b_pol")) - target
    m.close()
    return 0.5 * float(np.sum(r * r))


def test_misfit_gradient_matches_finite_differences(gdb):
    state = workloads.adjoint_state(CFG["lmax"], CFG["lmax"], CFG["nr"], seed=0)
    m = make(gdb, state)
    target = target_grid(m)
    J, gre, gim, ckpt = gdb.magnetic_misfit(m, target, CFG["steps"], CFG["checkpoint"])
    assert [c[0] for c in ckpt] == list(range(0, CFG["steps"], CFG["checkpoint"]))
    assert J == pytest.approx(misfit(gdb, state, state["b_pol"], target), rel=1e-14)
    # the misfit must depend on B_pol: a gradient that vanishes (a boundary
    # condition pinning B_pol(ro)) would pass the comparisons vacuously
    gnorm = np.sqrt(dot((gre, gim), (gre, gim)))
    assert gnorm > 0.0
    b0 = state["b_pol"]
    for v in workloads.adjoint_directions(CFG["lmax"], CFG["lmax"], CFG["nr"], count=32, seed=2)[:8]:
        eps = 1e-3 * np.sqrt(dot(b0, b0) / dot(v, v))
        jp = misfit(gdb, state, (b0[0] + eps * v[0], b0[1] + eps * v[1]), target)
        jm = misfit(gdb, state, (b0[0] - eps * v[0], b0[1] - eps * v[1]), target)
        fd = (jp - jm) / (2 * eps)
        ad = dot((gre, gim), v)
        assert abs(ad) > 1e-6 * gnorm * np.sqrt(dot(v, v)), ad
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_misfit_gradient_matches_oracle_forward_mode(gdb, oracle_mod):
    # directional derivative of the oracle's 200-step misfit: the residual of
    # the oracle run from the seeded state, against the oracle's step applied
    # to the direction (the B_pol propagator is linear and state independent)
    state = workloads.adjoint_state(CFG["lmax"], CFG["lmax"], CFG["nr"], seed=0)
    m = make(gdb, state)
    target = target_grid(m)
    J, gre, gim, _ = gdb.magnetic_misfit(m, target, CFG["steps"], CFG["checkpoint"])
    v = workloads.adjoint_directions(CFG["lmax"], CFG["lmax"], CFG["nr"], count=32, seed=2)[0]

    def oracle_run(bpol):
        o = oracle_mod.Oracle(lmax=CFG["lmax"], nlat=CFG["nlat"], nlon=CFG["nlon"], nr=CFG["nr"], dt=CFG["dt"],
                              bc_mode=CFG["bc_mode"])
        for k, (a, b) in state.items():
            o.set_field(k, a, b)
        o.set_field("b_pol", *bpol)
        o.step(CFG["steps"])
        pre, pim = o.get_field("b_pol")
        f = m.l_values * (m.l_values + 1.0) / m.r[-1] ** 2
        re = np.zeros(m.spec_shape()); im = np.zeros(m.spec_shape())
        re[-1] = f * pre[-1]; im[-1] = f * pim[-1]
        return o.synth_scalar(re, im)[-1]

    resid = oracle_run(state["b_pol"]) - target
    assert 0.5 * float(np.sum(resid * resid)) == pytest.approx(J, rel=1e-9)
    tangent = oracle_run(v)
    fwd = float(np.sum(resid * tangent))
    ad = dot((gre, gim), v)
    assert abs(ad) > 0.0 and np.max(np.abs(tangent)) > 0.0
    assert abs(fwd - ad) <= 1e-6 * abs(ad), (fwd, ad)

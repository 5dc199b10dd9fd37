"""Reverse mode of the temperature step (gd_temperature_nl_adjoint,
gd_cnab2_adjoint, gd_snapshot; temperature_misfit's checkpoint and recompute).

* The nonlinear term's adjoint satisfies <N x, y> = <x, N^T y> against the
  forward advection (gd_compute_temperature_nonlinear) to 1e-12.
* The CNAB2 pieces equal D S^-T C x and P R^T x built densely from the
  oracle's operators (bc_mode 0, 1, 2) to 1e-12.
* The gradient of J = 1/2 |T(r_mid) - target|^2 after 30 steps (checkpoints
  every 7: uneven segments) with respect to the initial temperature matches
  FP64 central finite differences on the device and the forward-mode gradient
  of the oracle (the tangent run: the temperature's response to a direction,
  with zero sources and boundary values, the velocity unchanged) to 1e-6
  relative, for every bc_mode and for the benchmark's ab_mode 1."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "geodynamo.jl_b200"))
import workloads  # noqa: E402

SHAPE = dict(lmax=15, nlat=24, nlon=48)


def dot(a, b):
    return float(np.sum(a[0] * b[0]) + np.sum(a[1] * b[1]))


def test_temperature_nl_adjoint_dot_product(gdb):
    import torch
    g = gdb.SHTnsKitConfig(15, 24, 48, 8)
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(g.spec_shape()), rng.standard_normal(g.spec_shape()))
    y = (rng.standard_normal(g.spec_shape()), rng.standard_normal(g.spec_shape()))
    ut = rng.standard_normal(g.grid_shape())
    up = rng.standard_normal(g.grid_shape())
    _, nx, _ = g.compute_temperature_nonlinear_arrays(x[0], x[1], ut, up)
    G = g.nr * g.nlat * g.nlon
    f64 = dict(dtype=torch.float64, device="cuda")
    uth, uph = torch.empty(G, **f64), torch.empty(G, **f64)
    g.grid_to_device("u_th", uth)
    g.grid_to_device("u_ph", uph)
    yd, out = torch.empty(2 * g.nr * g.nlm, **f64), torch.empty(2 * g.nr * g.nlm, **f64)
    g.spectral_to_device(y[0], y[1], yd)
    g.temperature_nl_adjoint(uth, uph, yd, out)
    nty = g.spectral_from_device(out)
    lhs, rhs = dot(nx, y), dot(x, nty)
    print(f"<N x, y> = {lhs:.15e}, <x, N^T y> = {rhs:.15e}")
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1e-300) * 10
    g.close()


def dense_band(band, kl):
    n = band.shape[1]
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - kl), min(n, i + kl + 1)):
            D[i, j] = band[kl + i - j, j]
    return D


@pytest.mark.parametrize("bc_mode", [0, 1, 2])
def test_cnab2_adjoint_pieces_match_dense(gdb, oracle_mod, bc_mode):
    import torch
    nr, dt, th = 10, 1e-4, 0.5
    g = gdb.SHTnsKitConfig(7, 12, 24, nr, dt=dt, bc_mode=bc_mode)
    o = oracle_mod.Oracle(lmax=7, nlat=12, nlon=24, nr=nr, dt=dt, bc_mode=bc_mode)
    rng = np.random.default_rng(bc_mode)
    x = (rng.standard_normal(g.spec_shape()), rng.standard_normal(g.spec_shape()))
    f64 = dict(dtype=torch.float64, device="cuda")
    xd, yd = torch.empty(2 * nr * g.nlm, **f64), torch.empty(2 * nr * g.nlm, **f64)
    g.spectral_to_device(x[0], x[1], xd)
    for mode in (0, 1):
        g.cnab2_adjoint("temp", mode, xd, yd)
        y = g.spectral_from_device(yd)
        for q in range(g.nlm):
            l = int(g.l_values[q])
            lin, _ = o.implicit_matrices(2, l)
            L = dense_band(lin, o.kl)
            I = np.eye(nr)
            S = I / dt - th * L
            if bc_mode == 2:
                S[0] = 0.0; S[0, 0] = 1.0
                S[-1] = 0.0; S[-1, -1] = 1.0
            R = I / dt + (1 - th) * L
            for c in range(2):
                v = x[c][:, q].copy()
                if mode == 0:
                    if bc_mode == 1:
                        v[0] = v[-1] = 0.0
                    e = np.linalg.solve(S.T, v)
                    if bc_mode == 2:
                        e[0] = e[-1] = 0.0
                else:
                    e = R.T @ v
                    e[0] = e[-1] = 0.0  # fixed-value temperature rows
                got = y[c][:, q]
                assert np.max(np.abs(got - e)) <= 1e-12 * np.max(np.abs(e)), (mode, l, c)
    g.close()


CASES = [(0, 0), (1, 0), (2, 0), (0, 1)]  # (bc_mode, ab_mode)


@pytest.mark.parametrize("bc_mode,ab_mode", CASES)
def test_temperature_gradient_matches_fd_and_forward_mode(gdb, oracle_mod, bc_mode, ab_mode):
    nr, K, C = 12, 30, 7
    cfg = dict(dt=1e-5, bc_mode=bc_mode, ab_mode=ab_mode)
    st = workloads.seeded_state(15, 15, nr, seed=2, amp=0.3)
    rng = np.random.default_rng(7)
    L, M = workloads.lm_arrays(15, 15)
    nlm = L.size
    bv = rng.standard_normal((2, nlm)) * 1e-3
    src = np.linspace(0.1, 0.4, nr)
    shell = nr // 2

    def model(t0):
        m = gdb.SHTnsKitConfig(15, 24, 48, nr, **cfg)
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("temp", *t0)
        m.set_temperature_bc(bv, src)
        return m

    m = model(st["temp"])
    target = np.sin(np.arange(m.nlon * m.nlat).reshape(m.nlon, m.nlat) * 0.37) * 1e-2
    J, gre, gim = gdb.temperature_misfit(m, target, K, C, shell=shell)
    tK = m.get_field("temp")
    resid = m.synth_scalar(*tK)[shell] - target
    assert abs(J - 0.5 * np.sum(resid * resid)) <= 1e-12 * J
    m.close()

    def Jof(t0):
        mm = model(t0)
        mm.step(K)
        r = mm.synth_scalar(*mm.get_field("temp"))[shell] - target
        mm.close()
        return 0.5 * float(np.sum(r * r))

    worst_fd = worst_fm = 0.0
    for d in range(3):
        dre = rng.standard_normal((nr, nlm)) * 1e-2
        dim = rng.standard_normal((nr, nlm)) * 1e-2
        dim[:, M == 0] = 0.0
        gdot = float(np.sum(gre * dre) + np.sum(gim * dim))
        eps = 1.0
        fd = (Jof((st["temp"][0] + eps * dre, st["temp"][1] + eps * dim)) -
              Jof((st["temp"][0] - eps * dre, st["temp"][1] - eps * dim))) / (2 * eps)
        worst_fd = max(worst_fd, abs(fd - gdot) / abs(fd))
        if d == 0:
            # forward mode on the oracle: the tangent of T with zero sources and
            # boundary values, the rest of the state (and so the velocity) unchanged
            o = oracle_mod.Oracle(lmax=15, nlat=24, nlon=48, nr=nr, **cfg)
            for k, (a, b) in st.items():
                o.set_field(k, a, b)
            o.set_field("temp", dre, dim)
            o.step(K)
            dT = o.get_field("temp")
            fm = float(np.sum(resid * o.synth_scalar(dT[0], dT[1])[shell]))
            worst_fm = abs(fm - gdot) / abs(fm)
    print(f"bc_mode {bc_mode} ab_mode {ab_mode}: J {J:.6e}, FD rel err {worst_fd:.2e}, forward-mode rel err {worst_fm:.2e}")
    assert worst_fd <= 1e-6 and worst_fm <= 1e-6


def composed_pullback(gdb, model, lre, lim, K, C, s0, ab1, snaps, final):
    """The reverse pass written out from the pieces (gd_snapshot,
    gd_grid_device, gd_cnab2_adjoint, gd_temperature_nl_adjoint)."""
    import torch
    G = model.nr * model.nlat * model.nlon
    size = 2 * model.nr * model.nlm
    f64 = dict(dtype=torch.float64, device="cuda")
    lam = torch.empty(size, **f64)
    model.spectral_to_device(lre, lim, lam)
    psi1, psi2 = torch.empty(size, **f64), torch.zeros(size, **f64)
    tmp, nlt = torch.empty(size, **f64), torch.empty(size, **f64)
    model.cnab2_adjoint("temp", 0, lam, psi1)
    boot = lambda n: ab1 or s0 + n == 0  # noqa: E731
    for k in reversed(range(len(snaps))):
        c0, c1 = k * C, min(K, k * C + C)
        model.restore(snaps[k])
        ust = []
        for n in range(c0, c1):
            u = torch.empty(2 * G, **f64)
            model.grid_to_device("u_th", u[:G])
            model.grid_to_device("u_ph", u[G:])
            ust.append(u)
            if n < c1 - 1:
                model.step(1)
        for n in reversed(range(c0, c1)):
            a_n = 1.0 if boot(n) else 1.5
            b_n1 = 0.0 if (n + 1 >= K or boot(n + 1)) else 0.5
            torch.mul(psi1, a_n, out=tmp)
            if b_n1:
                tmp.sub_(psi2, alpha=b_n1)
            u = ust[n - c0]
            model.temperature_nl_adjoint(u[:G], u[G:], tmp, nlt)
            model.cnab2_adjoint("temp", 1, psi1, lam)
            lam.add_(nlt)
            if n > 0:
                psi2, psi1 = psi1, psi2
                model.cnab2_adjoint("temp", 0, lam, psi1)
    model.restore(final)
    return model.spectral_from_device(lam)


def test_native_pullback_equals_composed_pieces(gdb):
    import torch
    nr, K, C = 10, 17, 5
    st = workloads.seeded_state(15, 15, nr, seed=4, amp=0.3)
    m = gdb.SHTnsKitConfig(15, 24, 48, nr, dt=1e-5)
    for k, (a, b) in st.items():
        m.set_field(k, a, b)
    rng = np.random.default_rng(5)
    lre, lim = rng.standard_normal(m.spec_shape()), rng.standard_normal(m.spec_shape())
    nb = m.snapshot_bytes()
    snaps = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range((K + C - 1) // C)]
    final = torch.empty(nb, dtype=torch.uint8, device="cuda")
    start = torch.empty(nb, dtype=torch.uint8, device="cuda")
    m.snapshot(start)
    for k in range(len(snaps)):
        m.snapshot(snaps[k])
        m.step(min(C, K - k * C))
    m.snapshot(final)
    ref = composed_pullback(gdb, m, lre, lim, K, C, 0, False, snaps, final)
    m.restore(start)
    m.temperature_forward(K, C)
    got = m.temperature_pullback(lre, lim)
    # the same kernels in the same order; a psi^(n+1) - b psi^(n+2) is one fused
    # multiply-add in the library and two roundings in torch
    for x, y in zip(got, ref):
        assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(y))
    # the handle is left at the end of the forward run
    after = m.get_field("temp")
    m.restore(final)
    for x, y in zip(after, m.get_field("temp")):
        assert np.array_equal(x, y)
    m.close()


@pytest.mark.parametrize("bc_mode,ab_mode", [(0, 0), (2, 0), (0, 1)])
def test_temperature_gradient_wrt_velocity_matches_fd(gdb, bc_mode, ab_mode):
    # J(T^K) depends on the initial velocity through the advection of every
    # step after the first (each reads the previous velocity phase's grids);
    # gd_temperature_pullback_full returns that gradient with the temperature's
    nr, K, C = 12, 20, 6
    cfg = dict(dt=1e-5, bc_mode=bc_mode, ab_mode=ab_mode)
    st = workloads.seeded_state(15, 15, nr, seed=3, amp=0.3)
    rng = np.random.default_rng(17)
    L, M = workloads.lm_arrays(15, 15)
    nlm = L.size
    bv = rng.standard_normal((2, nlm)) * 1e-3
    src = np.linspace(0.1, 0.4, nr)
    shell = nr // 2

    def model(ut, up):
        m = gdb.SHTnsKitConfig(15, 24, 48, nr, **cfg)
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("u_tor", *ut)
        m.set_field("u_pol", *up)
        m.set_temperature_bc(bv, src)
        return m

    m = model(st["u_tor"], st["u_pol"])
    target = np.cos(np.arange(m.nlon * m.nlat).reshape(m.nlon, m.nlat) * 0.21) * 1e-2
    m.temperature_forward(K, C)
    tK = m.get_field("temp")
    resid = m.synth_scalar(*tK)[shell] - target
    gbar = np.zeros(m.grid_shape())
    gbar[shell] = resid
    lre, lim = m.synth_scalar_adjoint(gbar)
    (gtr, gti), (utr, uti), (upr, upi) = m.temperature_pullback_full(lre, lim)
    ptr, pti = m.temperature_pullback(lre, lim)
    assert np.allclose(gtr, ptr, rtol=0, atol=1e-14 * np.max(np.abs(ptr)))
    assert np.allclose(gti, pti, rtol=0, atol=1e-14 * np.max(np.abs(ptr)))
    m.close()

    def Jof(ut, up):
        mm = model(ut, up)
        mm.step(K)
        r = mm.synth_scalar(*mm.get_field("temp"))[shell] - target
        mm.close()
        return 0.5 * float(np.sum(r * r))

    worst = 0.0
    for d in range(3):
        dv = [rng.standard_normal((nr, nlm)) * 1e-3 for _ in range(4)]
        for x in (dv[1], dv[3]):
            x[:, M == 0] = 0.0
        gdot = float(np.sum(utr * dv[0]) + np.sum(uti * dv[1]) + np.sum(upr * dv[2]) + np.sum(upi * dv[3]))
        eps = 1.0
        plus = Jof((st["u_tor"][0] + eps * dv[0], st["u_tor"][1] + eps * dv[1]),
                   (st["u_pol"][0] + eps * dv[2], st["u_pol"][1] + eps * dv[3]))
        minus = Jof((st["u_tor"][0] - eps * dv[0], st["u_tor"][1] - eps * dv[1]),
                    (st["u_pol"][0] - eps * dv[2], st["u_pol"][1] - eps * dv[3]))
        fd = (plus - minus) / (2 * eps)
        assert abs(fd) > 0
        worst = max(worst, abs(fd - gdot) / abs(fd))
    print(f"bc_mode {bc_mode} ab_mode {ab_mode}: velocity-gradient FD rel err {worst:.2e}")
    assert worst <= 1e-5

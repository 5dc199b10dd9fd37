"""GPU tests of the entry points that take the reference's argument lists on
host arrays: compute_{temperature,velocity,magnetic}_nonlinear!
(src/thermal.jl:149, src/velocity.jl:312, src/magnetic.jl:131) and the CNAB2
pieces create_shtns_timestepping_matrices / build_rhs_cnab2! /
solve_implicit_step! (src/timestep.jl:498, 610, 692), against the oracle at the
FP64 path's tolerance (1e-12 relative, max-norm)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

TOL = 1e-12
SHAPE = dict(lmax=31, nlat=48, nlon=96, nr=32)


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def pair(gdb, oracle_mod, **kw):
    g = gdb.SHTnsKitConfig(SHAPE["lmax"], SHAPE["nlat"], SHAPE["nlon"], SHAPE["nr"], **kw)
    o = oracle_mod.Oracle(**SHAPE, **kw)
    return g, o


def test_nonlinear_functions_on_host_arrays(gdb, oracle_mod):
    g, o = pair(gdb, oracle_mod)
    st = workloads.seeded_state(31, 31, 32, seed=9)
    for k, (a, b) in st.items():
        o.set_field(k, a, b)
    bv = np.random.default_rng(4).standard_normal((2, g.nlm)) * 1e-3
    g.set_temperature_bc(bv); o.set_temperature_bc(bv)
    o.step(1)                       # the oracle's carried grids now hold a step's values
    # temperature: the velocity grids of the previous velocity phase
    ut, up = o.get_grid("u_th"), o.get_grid("u_ph")
    t0 = o.get_field("temp")
    o.temperature_nl()
    (tr, ti), (nre, nim), tgrid = g.compute_temperature_nonlinear_arrays(t0[0], t0[1], ut, up)
    ore, oim = o.get_nl("temp")
    assert rel(nre, ore) < TOL and rel(nim, oim) < TOL
    assert rel(tr, o.get_field("temp")[0]) < TOL          # Dirichlet rows applied in place
    assert rel(tgrid, o.get_grid("t")) < TOL
    # velocity: the j and B grids of the previous magnetic phase
    jb = [o.get_grid(n) for n in ("j_th", "j_ph", "b_th", "b_ph")]
    u = [o.get_field(k) for k in ("u_tor", "u_pol")]
    o.velocity_nl()
    ntor, npol, (ut2, up2) = g.compute_velocity_nonlinear_arrays(u[0], u[1], *jb)
    for a, b in zip(ntor + npol, o.get_nl("u_tor") + o.get_nl("u_pol")):
        assert rel(a, b) < TOL
    assert rel(ut2, o.get_grid("u_th")) < TOL and rel(up2, o.get_grid("u_ph")) < TOL
    # magnetic: the current velocity grids
    bfield = [o.get_field(k) for k in ("b_tor", "b_pol")]
    o.magnetic_nl()
    ntor, npol, grids = g.compute_magnetic_nonlinear_arrays(bfield[0], bfield[1], ut2, up2)
    for a, b in zip(ntor + npol, o.get_nl("b_tor") + o.get_nl("b_pol")):
        assert np.max(np.abs(a - b)) <= TOL * max(np.max(np.abs(b)), 1.0)
    for a, n in zip(grids, ("b_th", "b_ph", "j_th", "j_ph")):
        assert rel(a, o.get_grid(n)) < TOL, n


@pytest.mark.parametrize("kind,nu", [(0, 4.0), (1, 1.0)])
def test_cnab2_pieces_match_oracle(gdb, oracle_mod, kind, nu):
    # velocity (nu = Pm = 4) and magnetic (nu = 1) operators at the config's dt and theta
    dt = 1e-5
    g, o = pair(gdb, oracle_mod, dt=dt)
    M = gdb.create_shtns_timestepping_matrices(g, nu, dt, theta=0.5)
    rng = np.random.default_rng(kind)
    un, nl, pv = [(rng.standard_normal(g.spec_shape()), rng.standard_normal(g.spec_shape())) for _ in range(3)]
    rhs = M.build_rhs_cnab2(un, nl, pv, dt)
    sol = M.solve_implicit_step(rhs)
    # expected, per (l, m) column: dense L_l from the oracle's bands, its band solve
    for q in (0, 1, 5, 17, g.nlm - 1):
        l = int(g.l_values[q])
        lin, _ = o.implicit_matrices(kind, l)
        kl = 4
        Ld = np.zeros((g.nr, g.nr))
        for j in range(g.nr):
            for b in range(2 * kl + 1):
                i = j + b - kl
                if 0 <= i < g.nr:
                    Ld[i, j] = lin[b, j]
        for c in (0, 1):
            exp_rhs = un[c][:, q] / dt + 0.5 * (Ld @ un[c][:, q]) + 1.5 * nl[c][:, q] - 0.5 * pv[c][:, q]
            assert rel(rhs[c][:, q], exp_rhs) < 1e-12, (q, c)
            assert rel(sol[c][:, q], o.band_solve(kind, l, rhs[c][:, q])) < 1e-12, (q, c)
    # the reference-named functions on field objects
    cfg = g
    f = [gdb.create_shtns_spectral_field(cfg) for _ in range(5)]
    for x, (a, b) in zip(f[:3], (un, nl, pv)):
        x.data_real[...] = a; x.data_imag[...] = b
    gdb.build_rhs_cnab2(f[3], f[0], f[1], f[2], dt, M)
    gdb.solve_implicit_step(f[4], f[3], M)
    assert np.array_equal(f[4].data_real, sol[0]) and np.array_equal(f[4].data_imag, sol[1])
    M.close()


def test_zero_pivot_is_reported(gdb):
    # a zero operator: diffusivity 0 and 1/dt = 0 (dt = inf) leave every pivot zero
    g = gdb.SHTnsKitConfig(7, 12, 24, 9)
    with pytest.raises(gdb.GeoDynamoError) as e:
        gdb.create_shtns_timestepping_matrices(g, 0.0, float("inf"), theta=0.5)
    assert e.value.status == 5   # GD_ERR_SINGULAR
    M = gdb.create_shtns_timestepping_matrices(g, 1.0, 1e-5)   # the handle stays usable
    M.close()

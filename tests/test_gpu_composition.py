"""Composition (include_composition; compute_composition_nonlinear!,
src/compositional.jl:219-259) and the tau flux boundary conditions
(apply_flux_bc_tau!, src/scalar_field_common.jl:866-935) on the device against
the FP64 oracle: the FP64 step at 1e-12 (small grid and the headline grid),
the mixed step at the mixed path's 5e-6, the composition grids, the
decomposed step bit for bit, and the refused combinations."""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = workloads.FIELD_ORDER + ("comp",)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def model_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, precision="fp64", seed=0, **kw):
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, composition=1, schmidt=2.5, **kw)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, composition=1, schmidt=2.5, **kw)
    rng = np.random.default_rng(seed)
    st = workloads.seeded_state(lmax, lmax, nr, seed=seed, amp=1e-1)
    cst = workloads.seeded_state(lmax, lmax, nr, seed=seed + 100, amp=1e-1)["temp"]
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("comp", *cst)
    nlm = g.nlm
    # temperature: fixed values, with flux boundaries on a third of the modes;
    # composition: the default no-flux boundaries, prescribed fluxes on some modes
    tt = np.array([[1, 1], [1, 2], [2, 1], [2, 2]])[rng.integers(0, 4, nlm)].T.copy()
    tbv = rng.standard_normal((2, nlm)) * 1e-3
    cbv = np.where(rng.random((2, nlm)) < 0.3, rng.standard_normal((2, nlm)) * 1e-3, 0.0)
    src = np.linspace(0.2, 1.0, nr)
    csrc = np.linspace(-0.3, 0.3, nr)
    for m in (g, o):
        m.set_bc_types("temp", tt[0], tt[1])
        m.set_temperature_bc(tbv, src)
        m.set_composition_bc(cbv, csrc)
    return g, o


@pytest.mark.parametrize("grid", [(15, 24, 48, 12), (255, 384, 768, 5)])
def test_fp64_step_with_composition_matches_oracle(gdb, oracle_mod, grid):
    lmax, nlat, nlon, nr = grid
    g, o = model_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, dt=2e-6)
    steps = 3 if lmax < 100 else 1
    g.step(steps)
    o.step(steps)
    worst = {k: max(rel(x, y) for x, y in zip(g.get_field(k), o.get_field(k))) for k in NAMES}
    print(f"composition FP64 step lmax {lmax}: " + ", ".join(f"{k} {v:.1e}" for k, v in worst.items()))
    for k, v in worst.items():
        assert v < 1e-12, (k, v)
    for name in ("c", "cgth", "cgph", "cgr", "cadv"):
        assert rel(g.get_grid(name), o.get_grid(name)) < 1e-12, name
    g.close()


def test_mixed_step_with_composition_tracks_oracle(gdb, oracle_mod):
    g, o = model_pair(gdb, oracle_mod, 31, 48, 96, 16, precision="mixed", seed=4, dt=1e-5)
    g.step(2)
    o.step(2)
    worst = {k: max(rel(x, y) for x, y in zip(g.get_field(k), o.get_field(k))) for k in NAMES}
    print("composition mixed step: " + ", ".join(f"{k} {v:.1e}" for k, v in worst.items()))
    for k, v in worst.items():
        assert v < 5e-6, (k, v)
    for name in ("c", "cgth", "cgph", "cgr"):
        assert rel(g.get_grid(name), o.get_grid(name)) < 5e-6, name
    g.close()


def test_composition_phase_alone_matches_oracle(gdb, oracle_mod):
    # gd_composition_nonlinear after a velocity phase: the nonlinear term and
    # the boundary conditions it applies to the state
    g, o = model_pair(gdb, oracle_mod, 15, 24, 48, 10, seed=7)
    for m in (g, o):
        m.velocity_nl()
        m.composition_nl()
    assert rel(g.get_nl("comp")[0], o.get_nl("comp")[0]) < 1e-12
    for x, y in zip(g.get_field("comp"), o.get_field("comp")):
        assert rel(x, y) < 1e-12


def test_composition_with_boundary_rows_matches_oracle(gdb, oracle_mod):
    # bc_mode 2: composition's Dirichlet rows take its boundary values (and its
    # boundary types default to fixed values); the flux types are refused there
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, composition=1, schmidt=2.5, bc_mode=2, dt=2e-6)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, composition=1, schmidt=2.5, bc_mode=2, dt=2e-6)
    rng = np.random.default_rng(4)
    st = workloads.seeded_state(lmax, lmax, nr, seed=4, amp=1e-1)
    cst = workloads.seeded_state(lmax, lmax, nr, seed=104, amp=1e-1)["temp"]
    tbv = rng.standard_normal((2, g.nlm)) * 1e-2
    cbv = rng.standard_normal((2, g.nlm)) * 1e-2
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("comp", *cst)
        m.set_temperature_bc(tbv, np.linspace(0.2, 1.0, nr))
        m.set_composition_bc(cbv, np.linspace(-0.3, 0.3, nr))
    g.step(3)
    o.step(3)
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < 1e-12, k
    cre, _ = g.get_field("comp")
    assert np.array_equal(cre[0], cbv[0]) and np.array_equal(cre[-1], cbv[1])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_flux_rows_of_the_boundary_row_operator(gdb, oracle_mod, precision, tol):
    # bc_mode 2 with prescribed fluxes: the boundary row of the implicit solve is
    # the row of D1 (rhs: the flux) instead of the identity; every (inner, outer)
    # pair of types on temperature and composition, against the oracle, and the
    # rows hold after the steps
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    kw = dict(composition=1, schmidt=2.5, bc_mode=2, dt=2e-6)
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, **kw)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, **kw)
    rng = np.random.default_rng(9)
    st = workloads.seeded_state(lmax, lmax, nr, seed=6, amp=1e-1)
    cst = workloads.seeded_state(lmax, lmax, nr, seed=106, amp=1e-1)["temp"]
    pairs = np.array([[1, 1], [1, 2], [2, 1], [2, 2]])
    tt = pairs[rng.integers(0, 4, g.nlm)].T.copy()
    ct = pairs[rng.integers(0, 4, g.nlm)].T.copy()
    tbv = rng.standard_normal((2, g.nlm)) * 1e-2
    cbv = rng.standard_normal((2, g.nlm)) * 1e-2
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("comp", *cst)
        m.set_bc_types("temp", tt[0], tt[1])
        m.set_bc_types("comp", ct[0], ct[1])
        m.set_temperature_bc(tbv, np.linspace(0.2, 1.0, nr))
        m.set_composition_bc(cbv, np.linspace(-0.3, 0.3, nr))
    g.step(3)
    o.step(3)
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < tol, k
    D = o.fd_matrix(1)
    kl = o.kl
    dense = np.zeros((nr, nr))
    for i in range(nr):
        for j in range(max(0, i - kl), min(nr, i + kl + 1)):
            dense[i, j] = D[kl + i - j, j]
    for name, types, bv in (("temp", tt, tbv), ("comp", ct, cbv)):
        re, _ = g.get_field(name)
        dp = dense @ re
        for side, row in ((0, 0), (1, -1)):
            got = np.where(types[side] == 2, dp[row], re[row])
            assert np.max(np.abs(got - bv[side])) <= 1e-9, (name, side)


def test_composition_refusals(gdb):
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(7, 12, 24, 9, composition=1, schmidt=0.0)
    g = gdb.SHTnsKitConfig(7, 12, 24, 9, composition=1, schmidt=1.0)
    g.set_scheme("eab2")  # the exponential schemes carry composition too
    h = gdb.SHTnsKitConfig(7, 12, 24, 9)
    with pytest.raises(gdb.GeoDynamoError):
        h.set_composition_bc(None, np.zeros(9))
    with pytest.raises(gdb.GeoDynamoError):
        h.get_field("comp")
    with pytest.raises(gdb.GeoDynamoError):
        h.get_grid("c")
    k = gdb.SHTnsKitConfig(7, 12, 24, 9, bc_mode=2, geometry="ball")
    with pytest.raises(gdb.GeoDynamoError):  # a ball has no inner boundary
        k.set_bc_types("temp", np.full(k.nlm, 2), np.full(k.nlm, 1))
    k.set_bc_types("temp", np.full(k.nlm, 1), np.full(k.nlm, 2))  # an outer flux is fine


def test_decomposed_step_with_composition_matches_one_handle():
    import torch.multiprocessing as mp
    import dist_workers
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(dist_workers.distributed_step_device,
                       args=(2, port, "fp64", 3, 1, (31, 48, 96, 12), False, True),
                       nprocs=2, start_method="spawn", join=True)


def test_composition_host_array_entry_matches_oracle(gdb, oracle_mod):
    # gd_compute_composition_nonlinear: the drop-in for compute_composition_nonlinear!
    # on the caller's arrays (velocity grids from the caller, boundary data set before)
    g, o = model_pair(gdb, oracle_mod, 15, 24, 48, 10, seed=11)
    o.velocity_nl()
    ut, up = o.get_grid("u_th"), o.get_grid("u_ph")
    c = o.get_field("comp")
    o.composition_nl()
    (cr, ci), (nr_, ni_), cg = g.compute_composition_nonlinear_arrays(c[0], c[1], ut, up)
    ore, oim = o.get_field("comp")
    assert rel(cr, ore) < 1e-12 and rel(ci, oim) < 1e-12
    onr, oni = o.get_nl("comp")
    assert rel(nr_, onr) < 1e-12 and rel(ni_, oni) < 1e-12
    assert rel(cg, o.get_grid("c")) < 1e-12

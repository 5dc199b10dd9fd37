"""CPU tests: the FP64 oracle against the golden fixtures and known answers.

These pin the oracle before anything is compared with it: the reference's
own scalar round-trip test (test/shtnskit_roundtrip.jl:21-54), scipy's
spherical harmonics, numpy's Gauss-Legendre rule, numpy dense solves for the
radial operators, and the oracle's own trajectory fixture.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def sht():
    return dict(np.load(os.path.join(GOLD, "sht_l6.npz")))


@pytest.fixture(scope="module")
def orc6(oracle_mod):
    return oracle_mod.Oracle(lmax=6, nlat=12, nlon=24, nr=6)


def test_gauss_grid_matches_leggauss(orc6, sht):
    x, w, th, r = orc6.grid()
    assert rel(x, sht["x"]) < 1e-14
    assert rel(w, sht["w"]) < 1e-13
    assert np.all(np.diff(th) > 0), "colatitudes must run north to south"


def test_legendre_tables_match_scipy(orc6, sht):
    P, dP = orc6.tables()
    assert rel(P, sht["P"]) < 1e-13
    assert rel(dP, sht["dP"]) < 1e-13


def test_scalar_synthesis_matches_direct_sum(orc6, sht):
    g = orc6.synth_scalar(sht["re"], sht["im"])
    assert rel(g, sht["grid"]) < 1e-13


def test_reference_roundtrip_criterion(orc6, sht):
    # test/shtnskit_roundtrip.jl:47-54: relative squared error < 1e-7
    g = orc6.synth_scalar(sht["re"], sht["im"])
    re2, im2 = orc6.analysis_scalar(g)
    err = np.sum((re2 - sht["re"]) ** 2) + np.sum((im2 - sht["im"]) ** 2)
    ref = np.sum(sht["re"] ** 2) + np.sum(sht["im"] ** 2)
    assert err / ref < 1e-7
    assert err / ref < 1e-26


def test_vector_synthesis_matches_direct_sum(orc6, sht):
    vt, vp = orc6.synth_vector(sht["tre"], sht["tim"], sht["pre"], sht["pim"])
    assert rel(vt, sht["vt"]) < 1e-12
    assert rel(vp, sht["vp"]) < 1e-12


def test_vector_roundtrip(orc6, sht):
    # the reference skips this (test/shtnskit_roundtrip.jl:57-106); l >= 1 here
    out = orc6.analysis_vector(sht["vt"], sht["vp"])
    for got, key in zip(out, ("tre", "tim", "pre", "pim")):
        assert rel(got, sht[key]) < 1e-12


def test_m0_imaginary_part_zeroed(orc6, sht):
    g = orc6.synth_scalar(sht["re"], sht["im"]) + 0.3
    re, im = orc6.analysis_scalar(g)
    from oracle.oracle import lm_pairs
    m0 = [q for q, (l, m) in enumerate(lm_pairs(6, 6)) if m == 0]
    assert np.all(im[:, m0] == 0.0)


def test_radial_difference_weights(oracle_mod):
    d = dict(np.load(os.path.join(GOLD, "radial_nr12.npz")))
    o = oracle_mod.Oracle(lmax=3, nlat=6, nlon=8, nr=12)
    assert rel(o.fd_matrix(1), d["d1"]) < 1e-9
    assert rel(o.fd_matrix(2), d["d2"]) < 1e-9
    _, _, _, r = o.grid()
    assert rel(r, d["r"]) < 1e-15


def test_cnab2_known_answer(oracle_mod):
    # one CNAB2 step with N = 0 equals (I/dt - theta L)^-1 (I/dt + (1-theta) L) u
    d = dict(np.load(os.path.join(GOLD, "radial_nr12.npz")))
    o = oracle_mod.Oracle(lmax=3, nlat=6, nlon=8, nr=12, dt=1e-5, magnetic_prandtl=4.0)
    from oracle.oracle import lm_pairs
    q = lm_pairs(3, 3).index((3, 1))
    re = np.zeros((12, o.nlm)); im = np.zeros((12, o.nlm))
    re[:, q] = d["u"]; im[:, q] = -2 * d["u"]
    o.set_field("u_tor", re, im)
    o.implicit_step()
    out_re, out_im = o.get_field("u_tor")
    assert rel(out_re[:, q], d["x1"]) < 1e-9
    assert rel(out_im[:, q], -2 * d["x1"]) < 1e-9


def test_literal_vandermonde_is_ill_conditioned(oracle_mod):
    # create_derivative_matrix as written (V c = rhs) does not produce difference weights
    o = oracle_mod.Oracle(lmax=3, nlat=6, nlon=8, nr=32, fd_mode=1)
    assert np.max(np.abs(o.fd_matrix(1))) > 1e8


def test_oracle_trajectory_fixture(oracle_mod):
    d = dict(np.load(os.path.join(GOLD, "step_l7.npz")))
    lm, nlat, nlon, nr = [int(v) for v in d["dims"]]
    o = oracle_mod.Oracle(lmax=lm, nlat=nlat, nlon=nlon, nr=nr, dt=1e-5)
    names = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")
    for k in names:
        o.set_field(k, d[f"u0_{k}_re"], d[f"u0_{k}_im"])
    o.step(3)
    for k in names:
        re, im = o.get_field(k)
        assert rel(re, d[f"u3_{k}_re"]) < 1e-13, k
    assert rel(np.array(o.energy()), d["energy3"]) < 1e-13


def test_energy_formula(orc6, sht):
    # compute_magnetic_energy (src/magnetic.jl:519-542)
    from oracle.oracle import lm_pairs
    L = np.array([l for l, _ in lm_pairs(6, 6)])
    w = 1.0 / np.maximum(L * (L + 1.0), 1.0)
    orc6.set_field("b_tor", sht["tre"], sht["tim"])
    orc6.set_field("b_pol", sht["pre"], sht["pim"])
    orc6.set_field("u_tor", sht["re"], sht["im"])
    orc6.set_field("u_pol", sht["re"] * 0, sht["im"] * 0)
    ek, em = orc6.energy()
    em_ref = 0.5 * np.sum(w[None, :] * (sht["tre"] ** 2 + sht["tim"] ** 2 + sht["pre"] ** 2 + sht["pim"] ** 2))
    ek_ref = 0.5 * np.sum(w[None, :] * (sht["re"] ** 2 + sht["im"] ** 2))
    assert abs(em - em_ref) / em_ref < 1e-14
    assert abs(ek - ek_ref) / ek_ref < 1e-14


def test_literal_operator_amplifies_temperature(oracle_mod):
    # The implicit operator as written has no boundary rows (timestep.jl:519-539)
    # while the temperature's boundary rows are overwritten before each solve
    # (thermal.jl:262-303): at nr = 129, dt = 2e-6 the temperature then grows by
    # a factor of several hundred per step.  With Dirichlet rows in the
    # operator (bc_mode 2) it decays.
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(GOLD), "..", "geodynamo.jl_b200"))
    import workloads
    growth = {}
    for bc in (0, 2):
        o = oracle_mod.Oracle(lmax=7, nlat=12, nlon=24, nr=129, dt=2e-6, bc_mode=bc)
        for k, (a, b) in workloads.seeded_state(7, 7, 129, seed=0).items():
            o.set_field(k, a, b)
        t0 = np.abs(o.get_field("temp")[0]).max()
        o.step(4)
        growth[bc] = np.abs(o.get_field("temp")[0]).max() / t0
    assert growth[0] > 1e6
    assert growth[2] < 1.0


def test_uniform_boundary_pattern_is_l0_only(orc6):
    # test/shell_boundaries.jl:17-37: uniform inner / outer temperature
    # patterns (100 and 250) analysed to spectral boundary values carry only
    # l = 0 (|a_l>0| <= 1e-8 max); with orthonormal Y_00 = 1 / sqrt(4 pi) the
    # l = 0 value is the pattern times sqrt(4 pi)
    nlm = orc6.nlm
    lv = np.array([l for l in range(7) for m in range(l + 1)])
    for val in (100.0, 250.0):
        re, im = orc6.analysis_scalar(np.full(orc6.grid_shape(), val))
        for k in range(orc6.nr):
            mx = np.max(np.abs(re[k]))
            assert mx > 0
            assert np.all(np.abs(re[k, lv > 0]) <= 1e-8 * max(1.0, mx))
            assert np.all(np.abs(im[k]) <= 1e-8 * max(1.0, mx))
            assert re[k, 0] == pytest.approx(val * np.sqrt(4.0 * np.pi), rel=1e-13)
    assert nlm == lv.size

"""GPU parity: libgdb200.so (through its C ABI) against the FP64 oracle and the
golden fixtures.  Tolerances: relative max-norm error (max |a - b| / max |b|)
of 1e-12 for every transform, nonlinear term and single step of the all-FP64
path, as the requirement for the FP64 GPU step states; multi-step trajectories
are held to 1e-11 because the radial operators' conditioning (~1e7 at nr = 129)
amplifies last-bit differences step over step."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

TOL = 1e-12
NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax=None, **kw):
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, **kw)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, mmax=mmax, **kw)
    return g, o


SHAPES = [
    (6, 12, 24, 6, None),      # the reference's round-trip test size
    (31, 48, 96, 32, None),    # shell_l31_nr32
    (20, 34, 40, 7, 10),       # mmax < lmax, nlon with a factor 5, odd tiles
    (47, 72, 144, 5, None),    # 9 | nlon
]


@pytest.mark.parametrize("lmax,nlat,nlon,nr,mmax", SHAPES)
def test_scalar_transforms_match_oracle(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax):
    g, o = make_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax)
    re, im = workloads.transform_batch(lmax, g.mmax, nr, 3, seed=lmax)
    grid = g.synth_scalar(re, im)
    for f in range(3):
        assert rel(grid[f], o.synth_scalar(re[f], im[f])) < TOL
    re2, im2 = g.analysis_scalar(grid)
    for f in range(3):
        ore, oim = o.analysis_scalar(grid[f])
        assert rel(re2[f], ore) < TOL
        assert rel(im2[f], oim) < TOL
        assert rel(re2[f], re[f]) < 1e-11   # round trip


@pytest.mark.parametrize("lmax,nlat,nlon,nr,mmax", SHAPES)
def test_vector_transforms_match_oracle(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax):
    g, o = make_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax)
    re, im = workloads.transform_batch(lmax, g.mmax, nr, 2, seed=7 + lmax)
    L, M = workloads.lm_arrays(lmax, g.mmax)
    re[:, :, L == 0] = 0; im[:, :, L == 0] = 0
    vt, vp = g.synth_vector(re[0], im[0], re[1], im[1])
    ovt, ovp = o.synth_vector(re[0], im[0], re[1], im[1])
    assert rel(vt, ovt) < TOL and rel(vp, ovp) < TOL
    out = g.analysis_vector(vt, vp)
    oout = o.analysis_vector(vt, vp)
    for a, b in zip(out, oout):
        assert rel(a, b) < TOL
    assert rel(out[0], re[0]) < 1e-11 and rel(out[2], re[1]) < 1e-11


def test_golden_transforms(gdb):
    d = dict(np.load(os.path.join(GOLD, "sht_l6.npz")))
    g = gdb.SHTnsKitConfig(6, 12, 24, 6)
    assert rel(g.theta_grid, np.arccos(d["x"])) < 1e-14
    assert rel(g.gauss_weights, d["w"]) < 1e-13
    assert rel(g.synth_scalar(d["re"], d["im"]), d["grid"]) < 1e-13
    vt, vp = g.synth_vector(d["tre"], d["tim"], d["pre"], d["pim"])
    assert rel(vt, d["vt"]) < 1e-12 and rel(vp, d["vp"]) < 1e-12
    # the reference's own criterion (test/shtnskit_roundtrip.jl:54)
    re2, im2 = g.analysis_scalar(d["grid"])
    err = np.sum((re2 - d["re"]) ** 2) + np.sum((im2 - d["im"]) ** 2)
    assert err / (np.sum(d["re"] ** 2) + np.sum(d["im"] ** 2)) < 1e-7


def test_reference_api_mirror(gdb):
    d = dict(np.load(os.path.join(GOLD, "sht_l6.npz")))
    cfg = gdb.create_shtnskit_config(lmax=6, nlat=12, nlon=24, nr=6)
    spec = gdb.create_shtns_spectral_field(cfg)
    spec.data_real[...] = d["re"]; spec.data_imag[...] = d["im"]
    phys = gdb.create_shtns_physical_field(cfg)
    gdb.shtnskit_spectral_to_physical(spec, phys)
    spec2 = gdb.create_shtns_spectral_field(cfg)
    gdb.shtnskit_physical_to_spectral(phys, spec2)
    assert rel(spec2.data_real, d["re"]) < 1e-12
    physs = [gdb.create_shtns_physical_field(cfg) for _ in range(5)]
    gdb.batch_spectral_to_physical([spec] * 5, physs)
    for p in physs:
        assert rel(p.data, phys.data) < 1e-15


def load_state(g, o, st):
    for k, (a, b) in st.items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)


def test_nonlinear_terms_match_oracle(gdb, oracle_mod):
    g, o = make_pair(gdb, oracle_mod, 31, 48, 96, 32)
    st = workloads.seeded_state(31, 31, 32, seed=0)
    load_state(g, o, st)
    bv = np.random.default_rng(5).standard_normal((2, g.nlm)) * 1e-3
    src = np.linspace(0.0, 1e-3, 32)
    g.set_temperature_bc(bv, src); o.set_temperature_bc(bv, src)
    # a first full step populates the grids carried between sub-steps
    g.step(1); o.step(1)
    g.temperature_nl(); o.temperature_nl()
    for grid in ("t", "gth", "gph", "gr", "tadv"):
        assert rel(g.get_grid(grid), o.get_grid(grid)) < TOL, grid
    assert rel(g.get_nl("temp")[0], o.get_nl("temp")[0]) < TOL
    assert rel(g.get_field("temp")[0], o.get_field("temp")[0]) < TOL   # Dirichlet rows
    g.velocity_nl(); o.velocity_nl()
    for grid in ("u_th", "u_ph", "w_th", "w_ph", "vadv_th", "vadv_ph"):
        assert rel(g.get_grid(grid), o.get_grid(grid)) < TOL, grid
    for k in ("u_tor", "u_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert rel(a[0], b[0]) < TOL and rel(a[1], b[1]) < TOL, k
    g.magnetic_nl(); o.magnetic_nl()
    for grid in ("b_th", "b_ph", "j_th", "j_ph"):
        assert rel(g.get_grid(grid), o.get_grid(grid)) < TOL, grid
    for k in ("b_tor", "b_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert np.max(np.abs(a[0] - b[0])) <= 1e-30 + TOL * max(np.max(np.abs(b[0])), 1.0)


def test_single_step_matches_oracle(gdb, oracle_mod):
    g, o = make_pair(gdb, oracle_mod, 31, 48, 96, 32)
    load_state(g, o, workloads.seeded_state(31, 31, 32, seed=0))
    g.step(1); o.step(1)
    for k in NAMES:
        a, b = g.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < TOL and rel(a[1], b[1]) < TOL, k


def test_trajectory_shell_l31_nr32(gdb, oracle_mod):
    # 100 CNAB2 steps at dt = 1e-5 (the oracle configuration)
    g, o = make_pair(gdb, oracle_mod, 31, 48, 96, 32, dt=1e-5)
    load_state(g, o, workloads.seeded_state(31, 31, 32, seed=0))
    for _ in range(4):
        g.step(25); o.step(25)
        for k in NAMES:
            a, b = g.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < 1e-11 and rel(a[1], b[1]) < 1e-11, k
    ek, em = g.energy(); oek, oem = o.energy()
    assert abs(ek - oek) / oek < 1e-11 and abs(em - oem) / oem < 1e-11


def test_golden_trajectory(gdb):
    d = dict(np.load(os.path.join(GOLD, "step_l7.npz")))
    lm, nlat, nlon, nr = [int(v) for v in d["dims"]]
    g = gdb.SHTnsKitConfig(lm, nlat, nlon, nr, dt=1e-5)
    for k in NAMES:
        g.set_field(k, d[f"u0_{k}_re"], d[f"u0_{k}_im"])
    g.step(1)
    for k in NAMES:
        assert rel(g.get_nl(k)[0], d[f"nl_{k}_re"]) < TOL or np.max(np.abs(d[f"nl_{k}_re"])) == 0.0, k
    g.step(2)
    for k in NAMES:
        assert rel(g.get_field(k)[0], d[f"u3_{k}_re"]) < 1e-11, k
    assert rel(np.array(g.energy()), d["energy3"]) < 1e-11


def test_graph_replay_equals_eager_substeps(gdb):
    st = workloads.seeded_state(15, 15, 12, seed=3)
    a = gdb.SHTnsKitConfig(15, 24, 48, 12)
    b = gdb.SHTnsKitConfig(15, 24, 48, 12)
    for k, (x, y) in st.items():
        a.set_field(k, x, y); b.set_field(k, x, y)
    a.step(3)
    for _ in range(3):
        b.temperature_nl(); b.velocity_nl(); b.magnetic_nl(); b.implicit_step()
    for k in NAMES:
        assert np.array_equal(a.get_field(k)[0], b.get_field(k)[0]), k


def test_ab_mode_literal_bootstrap_every_step(gdb, oracle_mod):
    g, o = make_pair(gdb, oracle_mod, 15, 24, 48, 12, ab_mode=1)
    load_state(g, o, workloads.seeded_state(15, 15, 12, seed=1))
    g.step(3); o.step(3)
    for k in NAMES:
        assert rel(g.get_field(k)[0], o.get_field(k)[0]) < 1e-11, k


@pytest.mark.parametrize("bc_mode", [1, 2])
def test_boundary_modes_match_oracle(gdb, oracle_mod, bc_mode):
    # 1: clamp the boundary rows after the solve; 2: Dirichlet rows inside the operator
    g, o = make_pair(gdb, oracle_mod, 15, 24, 48, 12, bc_mode=bc_mode)
    load_state(g, o, workloads.seeded_state(15, 15, 12, seed=2))
    bv = np.stack([np.linspace(0.1, 0.3, g.nlm), np.linspace(-0.2, 0.05, g.nlm)])
    src = np.linspace(0.0, 1e-3, 12)
    g.set_temperature_bc(bv, src); o.set_temperature_bc(bv, src)
    g.step(4); o.step(4)
    for k in NAMES:
        a, b = g.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < 1e-11 and rel(a[1], b[1]) < 1e-11, k
    if bc_mode == 2:
        re = g.get_field("u_tor")[0]
        assert np.max(np.abs(re[0])) == 0.0 and np.max(np.abs(re[-1])) == 0.0


@pytest.mark.parametrize("bc_mode", [0, 1, 2])
@pytest.mark.parametrize("lmax,nlat,nlon,nr", [(12, 20, 40, 12), (19, 30, 60, 20), (11, 18, 36, 3)])
def test_implicit_solve_edges_match_oracle(gdb, oracle_mod, lmax, nlat, nlon, nr, bc_mode):
    # the implicit solve's edges: an odd mode count (91), a partial second
    # block of 82 modes (210), fewer levels than the band (nr = 3), under
    # every boundary mode; three steps cover the AB1 start and two AB2 steps
    # that read the other bank of nonlinear terms
    g, o = make_pair(gdb, oracle_mod, lmax, nlat, nlon, nr, bc_mode=bc_mode)
    load_state(g, o, workloads.seeded_state(lmax, lmax, nr, seed=3))
    g.step(3); o.step(3)
    for k in NAMES:
        a, b = g.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < 1e-11 and rel(a[1], b[1]) < 1e-11, k


def test_literal_temperature_growth_matches_oracle(gdb, oracle_mod):
    # bc_mode 0 (the operator as written) amplifies the temperature by a factor
    # of several hundred per step at nr = 129, dt = 2e-6; the device follows it
    g, o = make_pair(gdb, oracle_mod, 7, 12, 24, 129, dt=2e-6)
    load_state(g, o, workloads.seeded_state(7, 7, 129, seed=0))
    t0 = np.max(np.abs(o.get_field("temp")[0]))
    g.step(4); o.step(4)
    a, b = g.get_field("temp"), o.get_field("temp")
    assert np.max(np.abs(b[0])) > 1e6 * t0
    assert rel(a[0], b[0]) < 1e-10 and rel(a[1], b[1]) < 1e-10
    for k in NAMES[:4]:
        assert rel(g.get_field(k)[0], o.get_field(k)[0]) < 1e-10, k


def test_errors_are_status_codes(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 9)
    with pytest.raises(gdb.GeoDynamoError) as e:
        g.lib.gd_upload_spectral(g.h, 9, None, None) and g._check(1)
    bad = np.zeros(g.spec_shape())
    bad[3, 5] = np.nan
    g.set_field("u_pol", bad, np.zeros(g.spec_shape()))
    with pytest.raises(gdb.GeoDynamoError) as e:
        g.check_finite()
    assert e.value.status == 4
    with pytest.raises(gdb.GeoDynamoError):
        g.set_dt(-1.0)


def test_step_kernel_count_is_the_graph_node_count(gdb):
    # gd_step_kernels: the kernel nodes of the captured step graph; the FP64
    # step launches gradients, 4 + 1 + 2 syntheses with their phi transforms,
    # the products, the analyses, the boundary rows and the CNAB2 solve
    g = gdb.SHTnsKitConfig(15, 24, 48, 9)
    n0 = g.step_kernels()
    g.step(2)
    n1 = g.step_kernels()
    assert n0 == n1 and 15 <= n1 <= 40, (n0, n1)
    g.close()


@pytest.mark.parametrize("precision,tol,leak", [("fp64", 1e-13, 1e-8), ("mixed", 5e-6, 5e-6)])
def test_uniform_boundary_pattern_is_l0_only(gdb, precision, tol, leak):
    # test/shell_boundaries.jl:17-37 on the device: uniform patterns analyse to
    # l = 0 only (|a_l>0| <= 1e-8 of the largest in FP64, the reference's bound;
    # the split-TF32 analysis' own error level in mixed precision),
    # a_00 = value * sqrt(4 pi)
    g = gdb.SHTnsKitConfig(6, 12, 24, 6, precision=precision)
    lv = np.array([l for l in range(7) for m in range(l + 1)])
    for val in (100.0, 250.0):
        re, im = g.analysis_scalar(np.full(g.grid_shape(), val))
        for k in range(g.nr):
            mx = float(np.max(np.abs(re[k])))
            assert np.all(np.abs(re[k, lv > 0]) <= leak * max(1.0, mx))
            assert np.all(np.abs(im[k]) <= leak * max(1.0, mx))
            assert abs(re[k, 0] - val * np.sqrt(4.0 * np.pi)) <= tol * val * np.sqrt(4.0 * np.pi)

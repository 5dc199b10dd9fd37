"""GPU tests of the mixed-precision path (split-TF32 tensor-core Legendre
contractions, FP32 phi transforms and grid products, FP64 radial solves)
against the FP64 oracle.

Tolerances (relative max-norm): 5e-6 for single transforms and nonlinear
terms -- the split keeps ~22 significant bits per product and FP32 carries the
sums -- and 1e-5 for fields after a few steps.  The measured figures are
recorded by the accuracy study in bench.py."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")
TOL_T = 5e-6


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


SHAPES = [
    (6, 12, 24, 6, None),
    (31, 48, 96, 32, None),
    (20, 34, 40, 7, 10),
    (140, 212, 288, 5, None),   # several 128-row theta tiles, K chunks of both parities
    (255, 384, 768, 3, None),   # the headline grid (lmax 255, nlon 768)
]


@pytest.mark.parametrize("lmax,nlat,nlon,nr,mmax", SHAPES)
def test_mixed_scalar_transforms(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax):
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, precision="mixed")
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, mmax=mmax)
    re, im = workloads.transform_batch(lmax, g.mmax, nr, 3, seed=lmax)
    grid = g.synth_scalar(re, im)
    for f in range(3):
        assert rel(grid[f], o.synth_scalar(re[f], im[f])) < TOL_T
    ref = np.stack([o.synth_scalar(re[f], im[f]) for f in range(3)])
    re2, im2 = g.analysis_scalar(ref)
    for f in range(3):
        ore, oim = o.analysis_scalar(ref[f])
        assert rel(re2[f], ore) < TOL_T and rel(im2[f], oim) < TOL_T


@pytest.mark.parametrize("lmax,nlat,nlon,nr,mmax", SHAPES)
def test_mixed_vector_transforms(gdb, oracle_mod, lmax, nlat, nlon, nr, mmax):
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, precision="mixed")
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, mmax=mmax)
    re, im = workloads.transform_batch(lmax, g.mmax, nr, 2, seed=3 + lmax)
    L, M = workloads.lm_arrays(lmax, g.mmax)
    re[:, :, L == 0] = 0; im[:, :, L == 0] = 0
    vt, vp = g.synth_vector(re[0], im[0], re[1], im[1])
    ovt, ovp = o.synth_vector(re[0], im[0], re[1], im[1])
    assert rel(vt, ovt) < TOL_T and rel(vp, ovp) < TOL_T
    out = g.analysis_vector(ovt, ovp)
    oout = o.analysis_vector(ovt, ovp)
    for a, b in zip(out, oout):
        assert rel(a, b) < TOL_T


def test_mixed_step_tracks_oracle(gdb, oracle_mod):
    g = gdb.SHTnsKitConfig(31, 48, 96, 32, precision="mixed")
    o = oracle_mod.Oracle(lmax=31, nlat=48, nlon=96, nr=32)
    for k, (a, b) in workloads.seeded_state(31, 31, 32, seed=0).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.step(1); o.step(1)
    for k in ("temp", "u_tor", "u_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert rel(a[0], b[0]) < TOL_T, k
    g.step(9); o.step(9)
    for k in NAMES:
        a, b = g.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < 1e-5 and rel(a[1], b[1]) < 1e-5, k
    ek, em = g.energy(); oek, oem = o.energy()
    assert abs(ek - oek) / oek < 1e-6 and abs(em - oem) / oem < 1e-6


def test_mixed_step_l255_tracks_oracle(gdb, oracle_mod):
    # every fused phase kernel on the headline grid (nlon = 768 = 3 x 256)
    g = gdb.SHTnsKitConfig(255, 384, 768, 4, dt=2e-6, precision="mixed")
    o = oracle_mod.Oracle(lmax=255, nlat=384, nlon=768, nr=4, dt=2e-6)
    for k, (a, b) in workloads.seeded_state(255, 255, 4, seed=0).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.step(1); o.step(1)
    for k in ("temp", "u_tor", "u_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert rel(a[0], b[0]) < TOL_T and rel(a[1], b[1]) < TOL_T, k
    g.step(1); o.step(1)
    for k in NAMES:
        a, b = g.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < 1e-5 and rel(a[1], b[1]) < 1e-5, k


@pytest.mark.parametrize("nr", [3, 6])
def test_mixed_phase_products_l255(gdb, oracle_mod, nr):
    # the fused phase kernels at nlon = 768 (register-resident transforms):
    # the nonlinear terms of the second step, whose temperature phase advects
    # with the first step's velocity grid
    g = gdb.SHTnsKitConfig(255, 384, 768, nr, dt=2e-6, precision="mixed")
    o = oracle_mod.Oracle(lmax=255, nlat=384, nlon=768, nr=nr, dt=2e-6)
    for k, (a, b) in workloads.seeded_state(255, 255, nr, seed=5).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.step(1); o.step(1)
    g.temperature_nl(); o.temperature_nl()
    g.velocity_nl(); o.velocity_nl()
    g.magnetic_nl(); o.magnetic_nl()
    for k in ("temp", "u_tor", "u_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert rel(a[0], b[0]) < TOL_T and rel(a[1], b[1]) < TOL_T, k
    for k in ("b_tor", "b_pol"):
        a, b = g.get_nl(k), o.get_nl(k)
        assert np.max(np.abs(a[0])) <= 1e-30 + TOL_T * max(np.max(np.abs(b[0])), 1.0)


def test_mixed_synthesized_grids_match_oracle(gdb, oracle_mod):
    # grids of the mixed step are formed on request from its Fourier buffers
    # (the temperature grid included): after a step they are the grids the
    # step's phases synthesized, as the oracle keeps them
    g = gdb.SHTnsKitConfig(31, 48, 96, 32, precision="mixed")
    o = oracle_mod.Oracle(lmax=31, nlat=48, nlon=96, nr=32)
    for k, (a, b) in workloads.seeded_state(31, 31, 32, seed=0).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    for _ in range(2):
        g.step(1); o.step(1)
        for grid in ("t", "gth", "gph", "gr", "u_th", "u_ph", "w_th", "w_ph", "b_th", "b_ph", "j_th", "j_ph"):
            assert rel(g.get_grid(grid), o.get_grid(grid)) < TOL_T, grid


def test_precision_switch_keeps_state(gdb):
    st = workloads.seeded_state(15, 15, 12, seed=4)
    a = gdb.SHTnsKitConfig(15, 24, 48, 12)
    for k, (x, y) in st.items():
        a.set_field(k, x, y)
    a.step(2)
    a.set_precision("mixed")
    a.step(2)
    a.set_precision("fp64")
    a.step(1)
    a.check_finite()
    assert a.step_count() == 5

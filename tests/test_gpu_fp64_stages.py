"""GPU tests of the mixed-precision step with stages returned to FP64
(gd_set_fp64_stages).

In the reference's step the velocity's nonlinear term is its Coriolis term
alone: the theta and phi components of u x omega and j x B carry a zero radial
factor in every term (src/shtnskit_field_functions.jl:264-279,
src/velocity.jl:447-548, 638-672).  With the whole velocity chain in FP64 (u
synthesis, the phi transforms and Coriolis product, the velocity analysis) the
mixed step's velocity must therefore equal the FP64 step's bit for bit, whatever
precision the temperature and magnetic phases use.  Single stages are held to
the mixed path's few-step tolerance against the oracle (1e-5), which also
exercises the layout conversions between the FP32 and FP64 buffers."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def load(m, st):
    for k, (a, b) in st.items():
        m.set_field(k, a, b)


@pytest.mark.parametrize("lmax,nlat,nlon,nr,bc_mode", [
    (15, 24, 48, 12, 2),
    (20, 34, 48, 7, 0),        # an odd number of colatitude pairs (partial last block)
    (255, 384, 768, 3, 2),     # the headline grid
])
def test_velocity_chain_in_fp64_equals_fp64_step(gdb, lmax, nlat, nlon, nr, bc_mode):
    st = workloads.seeded_state(lmax, lmax, nr, seed=6)
    a = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, dt=2e-6, bc_mode=bc_mode, precision="mixed_vel64")
    b = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, dt=2e-6, bc_mode=bc_mode)
    load(a, st); load(b, st)
    a.step(4); b.step(4)
    for k in ("u_tor", "u_pol"):
        x, y = a.get_field(k), b.get_field(k)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), k
        x, y = a.get_nl(k), b.get_nl(k)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), k
    ea, eb = a.energy(), b.energy()
    assert ea[0] == eb[0]
    assert abs(ea[1] - eb[1]) <= 1e-14 * abs(eb[1])
    # the temperature stays a mixed-precision result
    assert rel(a.get_field("temp")[0], b.get_field("temp")[0]) < 1e-5
    a.check_finite()


@pytest.mark.parametrize("stages", [("vel_synth",), ("vel_products",), ("vel_analysis",),
                                    ("vel_synth", "vel_products"), ("vel_products", "vel_analysis")])
def test_single_fp64_stages_match_oracle(gdb, oracle_mod, stages):
    lmax, nlat, nlon, nr = 20, 34, 48, 7
    st = workloads.seeded_state(lmax, lmax, nr, seed=8)
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed")
    g.set_fp64_stages(stages)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr)
    load(g, st); load(o, st)
    g.step(3); o.step(3)
    for k in NAMES:
        x, y = g.get_field(k), o.get_field(k)
        assert rel(x[0], y[0]) < 1e-5 and rel(x[1], y[1]) < 1e-5, (stages, k)
    g.velocity_nl(); o.velocity_nl()
    for k in ("u_tor", "u_pol"):
        x, y = g.get_nl(k), o.get_nl(k)
        assert rel(x[0], y[0]) < 5e-6 and rel(x[1], y[1]) < 5e-6, (stages, k)
    for grid in ("u_th", "u_ph"):
        assert rel(g.get_grid(grid), o.get_grid(grid)) < 5e-6, (stages, grid)


def test_stage_mask_is_validated(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 9, precision="mixed")
    for bad in (16, -1):
        with pytest.raises(gdb.GeoDynamoError):
            g.set_fp64_stages(bad)
    g.set_fp64_stages(7)
    g.set_fp64_stages(8 | 6)  # the int8-slice synthesis with the FP64 products and analysis
    g.set_fp64_stages(0)

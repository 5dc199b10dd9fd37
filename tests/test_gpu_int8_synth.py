"""The vector synthesis of u by int8 digit slices on the tcgen05 tensor cores
(GD_STAGE_VEL_SYNTH_I8, gd_ozaki.cu) against the FP64 chain it replaces.

In the reference's step the velocity's nonlinear term is its Coriolis term
alone (src/velocity.jl:492-496), the vector synthesis of u
(SHsphtor_to_spat, src/shtnskit_field_functions.jl:252-321) followed by the
phi transforms, the Coriolis product and the vector analysis.  With the
products and the analysis in FP64, the two handles differ only in the
synthesis: the int8-slice one carries about 7 digits x 7 bits per operand and
error-free digit products, so the velocity term agrees with the DMMA chain to
rounding-level relative error (6 digits) or about 2^-33 (5 digits).  The FP32
copy of u that the other phases read is checked too (through the temperature
term, which advects with it), and three steps of the whole model against the
FP64 oracle."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = workloads.FIELD_ORDER
I8 = ("vel_synth_i8", "vel_products", "vel_analysis")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def pair(gdb, grid, digits, seed=0, **kw):
    lmax, nlat, nlon, nr = grid
    ref = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed_vel64", **kw)
    i8 = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed", **kw)
    i8.set_int8_digits(digits)
    i8.set_fp64_stages(I8)
    for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=seed, amp=1e-1).items():
        ref.set_field(k, a, b)
        i8.set_field(k, a, b)
    return ref, i8


@pytest.mark.parametrize("grid", [(15, 24, 48, 12), (63, 96, 192, 17), (255, 384, 768, 9)])
@pytest.mark.parametrize("digits,tol", [(6, 3e-10), (5, 3e-8)])
def test_velocity_term_matches_fp64_chain(gdb, grid, digits, tol):
    ref, i8 = pair(gdb, grid, digits)
    ref.velocity_nl()
    i8.velocity_nl()
    worst = max(rel(x, y) for k in ("u_tor", "u_pol") for x, y in zip(i8.get_nl(k), ref.get_nl(k)))
    print(f"int8 synthesis, {digits} digits, lmax {grid[0]} nr {grid[3]}: velocity term {worst:.2e}")
    assert worst < tol
    # the FP32 copy of u (u grids of the temperature phase) is the FP32 rounding of the same values
    for name in ("u_th", "u_ph"):
        assert rel(i8.get_grid(name), ref.get_grid(name)) < 1e-6, name
    ref.close()
    i8.close()


def test_steps_match_oracle(gdb, oracle_mod):
    lmax, nlat, nlon, nr = 31, 48, 96, 16
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed_vel64i8", bc_mode=2, dt=1e-5)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, bc_mode=2, dt=1e-5)
    for m in (g, o):
        for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=3, amp=1e-1).items():
            m.set_field(k, a, b)
    g.step(3)
    o.step(3)
    for k in ("u_tor", "u_pol"):
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < 1e-11, k
    for k in NAMES:
        for x, y in zip(g.get_field(k), o.get_field(k)):
            assert rel(x, y) < 5e-6, k
    ek, _ = g.energy()
    ok, _ = o.energy()
    assert abs(ek - ok) <= 1e-11 * abs(ok)
    g.close()


def test_int8_stage_refusals(gdb):
    b = gdb.SHTnsKitConfig(7, 12, 24, 9, geometry="ball", bc_mode=2, precision="mixed")
    with pytest.raises(gdb.GeoDynamoError):
        b.set_fp64_stages(I8)
    s = gdb.SHTnsKitConfig(7, 12, 24, 18, segments=2, precision="mixed")
    with pytest.raises(gdb.GeoDynamoError):
        s.set_fp64_stages(I8)
    g = gdb.SHTnsKitConfig(7, 12, 24, 9, precision="mixed")
    with pytest.raises(gdb.GeoDynamoError):
        g.set_int8_digits(4)
    g.set_fp64_stages(I8)
    g.step(1)
    g.check_finite()


@pytest.mark.parametrize("scheme", ["eab2", "erk2"])
def test_exponential_schemes_with_int8_synthesis(gdb, scheme):
    # the exponential schemes call the same velocity phase: with the int8
    # synthesis their velocity follows the FP64 chain's run of the same scheme
    lmax, nlat, nlon, nr = 15, 24, 48, 12
    ref, i8 = pair(gdb, (lmax, nlat, nlon, nr), 6, seed=5, dt=1e-5)
    for g in (ref, i8):
        g.set_scheme(scheme)
        g.step(3)
        g.check_finite()
    for k in ("u_tor", "u_pol"):
        for x, y in zip(i8.get_field(k), ref.get_field(k)):
            assert rel(x, y) < 1e-10, (scheme, k)
    ref.close()
    i8.close()


@pytest.mark.parametrize("lmax,mmax,nlat,nlon,nr", [(31, 20, 48, 96, 10), (511, 511, 768, 1536, 5)])
def test_truncations_and_largest_lmax(gdb, lmax, mmax, nlat, nlon, nr):
    # mmax < lmax (orders past mmax absent), and lmax = 511, the largest the
    # int8 synthesis takes (eight 32-degree K steps per parity at m = 0)
    ref = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, precision="mixed_vel64")
    i8 = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, precision="mixed_vel64i8")
    for k, (a, b) in workloads.seeded_state(lmax, mmax, nr, seed=9, amp=1e-1).items():
        ref.set_field(k, a, b)
        i8.set_field(k, a, b)
    ref.velocity_nl()
    i8.velocity_nl()
    worst = max(rel(x, y) for k in ("u_tor", "u_pol") for x, y in zip(i8.get_nl(k), ref.get_nl(k)))
    print(f"int8 synthesis, lmax {lmax} mmax {mmax}: velocity term {worst:.2e}")
    assert worst < 1e-9
    ref.close()
    i8.close()

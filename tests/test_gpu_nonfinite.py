"""Non-finite inputs propagate as in the reference.  The theta/phi components of
u x B, u x omega and j x B vanish in the literal step (the synthesized vectors
have zero radial components, src/shtnskit_field_functions.jl:264-279), but every
product is still evaluated, as the reference evaluates it: a NaN in one
magnetic coefficient makes NaN * 0 in the products of its shell, so the
induction term of that shell, and (one phase later, through the carried grids)
the Lorentz term wherever B and curl B are NaN, become NaN.  The device's
NaN pattern must equal the oracle's, FP64 and mixed; gd_check_finite then
reports the state after the step."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "geodynamo.jl_b200"))
import workloads  # noqa: E402


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_in_b_propagates_like_the_reference(gdb, oracle_mod, precision):
    lmax, nlat, nlon, nr = 15, 24, 48, 8
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr)
    st = workloads.seeded_state(lmax, lmax, nr, seed=3)
    L, M = workloads.lm_arrays(lmax, lmax)
    q = int(np.flatnonzero((L == 3) & (M == 1))[0])
    bt = (st["b_tor"][0].copy(), st["b_tor"][1].copy())
    bt[0][2, q] = np.nan  # shell 2
    for m in (g, o):
        for k, (a, b) in st.items():
            m.set_field(k, a, b)
        m.set_field("b_tor", *bt)
    # the velocity phase reads the j and B grids carried from the previous
    # magnetic phase (still zero here), the magnetic phase the new B
    for m in (g, o):
        m.velocity_nl()
        m.magnetic_nl()
    for k in ("u_tor", "u_pol", "b_tor", "b_pol"):
        for x, y in zip(g.get_nl(k), o.get_nl(k)):
            assert np.array_equal(np.isnan(x), np.isnan(y)), (precision, k)
    # the induction term reads B of its own shell only (Im at m = 0 is set to 0
    # after the analysis, NaN or not)
    re_, im_ = o.get_nl("b_pol")
    assert np.isnan(re_[2]).all() and np.isnan(im_[2]).any()
    for y in (re_, im_):
        assert not np.isnan(np.delete(y, 2, axis=0)).any()
    assert not np.isnan(o.get_nl("u_tor")[0]).any()
    # the next velocity phase carries the NaN grids of B and j = curl B (whose
    # radial stencil reaches the neighbouring shells) into the Lorentz term
    for m in (g, o):
        m.velocity_nl()
    for k in ("u_tor", "u_pol"):
        for x, y in zip(g.get_nl(k), o.get_nl(k)):
            assert np.array_equal(np.isnan(x), np.isnan(y)), (precision, k)
        assert np.isnan(o.get_nl(k)[0][2]).all(), k
    g.step(1)
    with pytest.raises(gdb.GeoDynamoError):
        g.check_finite()
    g.close()

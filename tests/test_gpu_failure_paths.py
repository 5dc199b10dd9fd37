"""GPU tests of the failure paths, in forms that fault, trap or hang no GPU.

1. A bounded tensor-core wait that runs out: the next split-TF32 synthesis
   omits the bulk copies of one pipeline step in its first CTA (with a short
   wait bound, about 8 ms), so the MMA warp's wait on that stage expires; the
   kernel records it, lets its issued copies land, frees its tensor memory and
   returns.  The call must report GD_ERR_CUDA ("wait expired"), and the next
   call on the same handle must succeed and match the oracle.
2. A zero pivot in a banded LU factorisation is GD_ERR_SINGULAR
   (tests/test_gpu_reference_api.py::test_zero_pivot_is_reported).
3. A non-finite state is GD_ERR_NONFINITE
   (tests/test_gpu_parity.py::test_errors_are_status_codes)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_expired_tensor_core_wait_is_reported_and_handle_recovers(gdb, oracle_mod):
    lmax, nlat, nlon, nr = 31, 48, 96, 8
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed")
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr)
    re, im = workloads.transform_batch(lmax, lmax, nr, 2, seed=3)
    g.set_fault_test(wait_cycles=1 << 24, omit_step=0)
    with pytest.raises(gdb.GeoDynamoError) as e:
        g.synth_scalar(re, im)
    assert e.value.status == 3 and "wait expired" in str(e.value)
    # the omission was one-shot and the flag was cleared: the handle works
    grid = g.synth_scalar(re, im)
    for f in range(2):
        assert rel(grid[f], o.synth_scalar(re[f], im[f])) < 5e-6
    g.set_fault_test(0, -1)
    st = workloads.seeded_state(lmax, lmax, nr, seed=1)
    for k, (a, b) in st.items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.step(2); o.step(2)
    for k in workloads.FIELD_ORDER:
        assert rel(g.get_field(k)[0], o.get_field(k)[0]) < 1e-5, k


def test_fault_test_needs_mixed_state(gdb):
    g = gdb.SHTnsKitConfig(7, 12, 24, 9)
    with pytest.raises(gdb.GeoDynamoError) as e:
        g.set_fault_test(1 << 24, 0)
    assert e.value.status == 7


def test_expired_wait_in_int8_synthesis_is_reported_and_handle_recovers(gdb, oracle_mod):
    # the same failure in the int8-slice velocity synthesis (the first
    # tensor-core launch of the velocity phase with GD_STAGE_VEL_SYNTH_I8)
    lmax, nlat, nlon, nr = 31, 48, 96, 8
    g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision="mixed_vel64i8", bc_mode=2, dt=1e-5)
    o = oracle_mod.Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, bc_mode=2, dt=1e-5)
    st = workloads.seeded_state(lmax, lmax, nr, seed=2)
    for k, (a, b) in st.items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.set_fault_test(wait_cycles=1 << 24, omit_step=0)
    with pytest.raises(gdb.GeoDynamoError) as e:
        g.velocity_nl()
    assert e.value.status == 3 and "wait expired" in str(e.value)
    g.set_fault_test(0, -1)
    for k, (a, b) in st.items():
        g.set_field(k, a, b)
    g.step(2)
    o.step(2)
    for k in ("u_tor", "u_pol"):
        assert rel(g.get_field(k)[0], o.get_field(k)[0]) < 1e-11, k

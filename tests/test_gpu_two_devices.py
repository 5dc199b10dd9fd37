"""Handles on two devices in one process.

Kernel attributes (the dynamic shared-memory limits above 48 KB that the
tensor-core, fused and int8-slice kernels need) and the SM count are cached
per device, so a second handle on another GPU launches the same kernels: the
same model stepped on device 0 and on device 1 gives the same fields, in the
mixed precision presets and in FP64.  Skipped when fewer than two devices are
visible."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402


def visible_devices():
    try:
        import torch
        return torch.cuda.device_count()
    except Exception:
        return 0


@pytest.mark.skipif(visible_devices() < 2, reason="needs two visible CUDA devices")
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_vel64i8"])
def test_same_model_on_two_devices(gdb, precision):
    lmax, nlat, nlon, nr = 63, 96, 192, 17
    st = workloads.seeded_state(lmax, lmax, nr, seed=8, amp=1e-1)
    handles = []
    for dev in (0, 1):
        g = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, precision=precision, dt=1e-5, device=dev)
        for k, (a, b) in st.items():
            g.set_field(k, a, b)
        handles.append(g)
    for g in handles:
        g.step(3)
        g.check_finite()
    for k in workloads.FIELD_ORDER:
        a, b = handles[0].get_field(k), handles[1].get_field(k)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (precision, k)
    for g in handles:
        g.close()

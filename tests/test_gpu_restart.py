"""GPU tests of the restart files through the C ABI: a model's state written
in the reference's restart layout (src/outputs_writer.jl:1221-1371) and read
into a fresh model is bitwise the state that was written; the file's physical
temperature is the writing model's synthesis of its spectral temperature; the restarted
run is a new run from that state (AB1 start, zero carried grids), which the
oracle follows to the trajectory tolerances of the other tests (FP64 1e-11,
mixed precision 1e-5)."""
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_continues_as_a_new_run(gdb, oracle_mod, tmp_path, precision):
    dims = (15, 24, 48, 12)
    g = gdb.SHTnsKitConfig(*dims, precision=precision)
    for k, (a, b) in workloads.seeded_state(15, 15, 12, seed=6).items():
        g.set_field(k, a, b)
    g.step(3)
    fn = gdb.write_restart(g, str(tmp_path / "restart.nc"), time=3e-5)
    data, meta = gdb.read_restart(fn)
    assert meta["current_step"] == 3 and meta["current_time"] == 3e-5
    # the physical temperature is the writing model's synthesis of its spectral
    # temperature (FP64 or split-TF32): bitwise, and within 5e-6 of FP64
    t = g.get_field("temp")
    assert np.array_equal(data["temperature"], g.synth_scalar(*t))
    g64 = gdb.SHTnsKitConfig(*dims)
    assert rel(data["temperature"], g64.synth_scalar(*t)) < (1e-300 if precision == "fp64" else 5e-6)
    h = gdb.SHTnsKitConfig(*dims, precision=precision)
    gdb.load_restart(h, fn)
    assert h.step_count() == 0
    o = oracle_mod.Oracle(lmax=15, nlat=24, nlon=48, nr=12)
    for k in NAMES:
        a, b = g.get_field(k), h.get_field(k)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), k
        o.set_field(k, *a)
    h.step(2)
    o.step(2)
    tol = 1e-11 if precision == "fp64" else 1e-5
    for k in NAMES:
        a, b = h.get_field(k), o.get_field(k)
        assert rel(a[0], b[0]) < tol and rel(a[1], b[1]) < tol, k

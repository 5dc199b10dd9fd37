"""The step at lmax = 511 (nlat = 768, nlon = 1536: the scale-out grid of the
shell/mode decomposition, src/pencil_decomps.jl:136-284): the FP64 and mixed
steps against the FP64 oracle on four shells, and the distributed step on two
ranks against one handle, bit for bit.  nlon = 1536 has no compile-time FFT
kernel, so these also cover the runtime-plan transforms."""
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

GRID = dict(lmax=511, nlat=768, nlon=1536)
NAMES = workloads.FIELD_ORDER


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_lmax511_step_matches_oracle(gdb, oracle_mod, precision, tol):
    nr = 4
    g = gdb.SHTnsKitConfig(GRID["lmax"], GRID["nlat"], GRID["nlon"], nr, dt=1e-6, bc_mode=2, precision=precision)
    o = oracle_mod.Oracle(lmax=GRID["lmax"], nlat=GRID["nlat"], nlon=GRID["nlon"], nr=nr, dt=1e-6, bc_mode=2)
    for k, (a, b) in workloads.seeded_state(511, 511, nr, seed=3).items():
        g.set_field(k, a, b)
        o.set_field(k, a, b)
    g.step(1)
    o.step(1)
    worst = {k: max(rel(x, y) for x, y in zip(g.get_field(k), o.get_field(k))) for k in NAMES}
    print(f"lmax 511 {precision} step: " + ", ".join(f"{k} {v:.1e}" for k, v in worst.items()))
    for k, v in worst.items():
        assert v < tol, (k, v)
    g.close()


def test_lmax511_distributed_step_matches_one_handle():
    import torch.multiprocessing as mp
    import dist_workers
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(dist_workers.distributed_step_device,
                       args=(2, port, "fp64", 2, 1, (511, 768, 1536, 8)), nprocs=2, start_method="spawn", join=True)

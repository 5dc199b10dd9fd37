"""The shell/mode decomposition and its all-to-all exchange on CPU ranks
(gloo, world sizes 2 and 3, separate processes)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import distributed as D  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn(fn, world, *args):
    import torch.multiprocessing as mp
    mp.start_processes(fn, args=(world, free_port()) + args, nprocs=world, start_method="spawn", join=True)


def test_partition_covers_shells_and_whole_columns():
    for world in (1, 2, 3, 5, 8):
        dec = D.Decomposition(129, 255, 255, world)
        assert dec.shells[0][0] == 0 and dec.shells[-1][1] == 129
        assert all(a[1] == b[0] for a, b in zip(dec.shells, dec.shells[1:]))
        assert dec.modes[0][0] == 0 and dec.modes[-1][1] == dec.nlm
        starts = set(D.mode_offsets(255, 255))
        assert all(j0 in starts and j1 in starts for j0, j1 in dec.modes)
        # each rank is within one column (<= 256 modes) of an even share
        assert all(abs(dec.nmode(k) - dec.nlm / world) <= 256 for k in range(world))
    # more ranks than columns: the extra ranks own none
    dec = D.Decomposition(9, 3, 3, 6)
    assert sum(dec.nmode(k) for k in range(6)) == dec.nlm


def test_exchange_volume_at_the_headline_shell():
    # 10 fields out (T, grad_r T, u, omega, B, j) and 5 back (the nonlinear terms) per step
    dec = D.Decomposition(129, 255, 255, 8)
    out_b = dec.exchange_bytes(10)
    back_b = dec.exchange_bytes(5)
    assert 0.5e9 < out_b < 0.7e9 and abs(back_b - out_b / 2) < 1e6


@pytest.mark.parametrize("world", [2, 3])
def test_transpose_roundtrip(world):
    import dist_workers
    spawn(dist_workers.transpose_roundtrip, world, 10, 15, 15)


def test_distributed_phase_matches_whole_array():
    import dist_workers
    spawn(dist_workers.phase_matches_global, 2)


@pytest.mark.parametrize("world,magnetic", [(2, 1), (3, 1), (2, 0)])
def test_distributed_step_exchanges(world, magnetic):
    """The two exchanges of the distributed step (state + derivatives to the
    shell slabs, nonlinear terms back to the mode columns) over fake handles
    give the whole handle's result bit for bit."""
    import dist_workers
    spawn(dist_workers.distributed_step_fake, world, magnetic)

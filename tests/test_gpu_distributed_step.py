"""The distributed step (DistributedStep: mode-range derivatives and CNAB2,
shell-slab nonlinear phases, two all-to-all exchanges) on the device against one
whole handle.  Both ranks run on cuda:0 and exchange over gloo through pinned
host buffers: the kernels of one rank never wait on the other's, and the result
does not depend on where a block crossed.  Bit for bit in every precision
preset: every kernel computes each mode column or shell row on its own, and the
mixed phases build their tensor-core operand images from the same FP64
derivatives whether a handle computed them or received them."""
import os
import socket
import sys

import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("precision,magnetic,world", [("fp64", 1, 2), ("fp64", 0, 2), ("fp64", 1, 3),
                                                      ("mixed_vel64", 1, 2), ("mixed", 1, 2)])
def test_distributed_step_matches_one_handle(precision, magnetic, world):
    import torch.multiprocessing as mp
    import dist_workers
    mp.start_processes(dist_workers.distributed_step_device, args=(world, free_port(), precision, 5, magnetic),
                       nprocs=world, start_method="spawn", join=True)


def test_distributed_step_nccl_device_buffers():
    """The NCCL path (device exchange buffers) on one rank: the exchanges are
    copies through device memory and the step still equals one handle's."""
    import torch.multiprocessing as mp
    import dist_workers
    mp.start_processes(dist_workers.distributed_step_device,
                       args=(1, free_port(), "mixed_vel64", 3, 1, (31, 48, 96, 12), True),
                       nprocs=1, start_method="spawn", join=True)

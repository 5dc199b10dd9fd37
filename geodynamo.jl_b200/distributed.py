"""Shell / mode decomposition of the step across ranks and its exchange step.

The step has two halves with different independence structure:

* transforms and grid products are independent per radial level (shell):
  `batch_spectral_to_physical!`, `shtnskit_vector_synthesis!`, the products and
  the analyses (src/shtnskit_field_functions.jl:11-321, src/velocity.jl:447-548,
  src/magnetic.jl:375-404, src/scalar_field_common.jl:390-443);
* the CNAB2 solves and the radial derivatives are independent per (l, m) but
  couple every shell (src/timestep.jl:610-730, src/velocity.jl:340-441).

So each rank owns a block of shells for the first half ("shell layout") and a
block of whole m columns for the second ("mode layout"), and the step
exchanges spectral fields between the two with one all-to-all per direction
(the reference's pencil transposes, src/pencil_decomps.jl:136-284, restated
for two layouts).  Whole m columns keep the theta recurrence (l +- 1, m)
local.  Spectral arrays use the library's native layout: two planes (Re, Im)
of [r][j] with j m-major (j = moff[m] + l - m).

The functions take torch tensors and a process group: NCCL over NVLink for
CUDA tensors, gloo for CPU tensors (the tests run world sizes 2 and 3 on CPU).
"""
from __future__ import annotations

import numpy as np


def mode_offsets(lmax: int, mmax: int):
    """moff[m] = first native index of order m; moff[mmax + 1] = nlm."""
    moff = [0]
    for m in range(mmax + 1):
        moff.append(moff[-1] + (lmax - m + 1))
    return moff


def split_even(n: int, parts: int):
    """Contiguous ranges of n items over `parts` ranks, sizes differing by at most one."""
    base, extra = divmod(n, parts)
    out, s = [], 0
    for k in range(parts):
        e = s + base + (1 if k < extra else 0)
        out.append((s, e))
        s = e
    return out


def native_l(lmax: int, mmax: int):
    """Degree l of every native mode index j (m-major)."""
    return np.array([l for m in range(mmax + 1) for l in range(m, lmax + 1)])


def split_m_columns(lmax: int, mmax: int, parts: int):
    """Whole m columns per rank, contiguous in m, balanced by mode count.

    Returns native index ranges (j0, j1) per rank; a rank may own no column
    when parts > mmax + 1."""
    moff = mode_offsets(lmax, mmax)
    nlm = moff[-1]
    bounds = [0]
    for k in range(1, parts):
        target = nlm * k / parts
        best = bounds[-1]
        for m in range(bounds[-1], mmax + 2):
            if abs(moff[m] - target) < abs(moff[best] - target):
                best = m
        bounds.append(best)
    bounds.append(mmax + 1)
    return [(moff[bounds[k]], moff[bounds[k + 1]]) for k in range(parts)]


class Decomposition:
    """Which shells and which (l, m) modes each of `world` ranks owns."""

    def __init__(self, nr: int, lmax: int, mmax: int | None = None, world: int = 1):
        mmax = lmax if mmax is None else mmax
        self.nr, self.lmax, self.mmax, self.world = nr, lmax, mmax, world
        self.nlm = mode_offsets(lmax, mmax)[-1]
        self.shells = split_even(nr, world)
        self.modes = split_m_columns(lmax, mmax, world)

    def nshell(self, rank):
        s0, s1 = self.shells[rank]
        return s1 - s0

    def nmode(self, rank):
        j0, j1 = self.modes[rank]
        return j1 - j0

    def shell_slab(self, full, rank):
        """Rank's shell-layout block of a full (2, nr, nlm) array."""
        s0, s1 = self.shells[rank]
        return full[:, s0:s1, :]

    def mode_slab(self, full, rank):
        """Rank's mode-layout block of a full (2, nr, nlm) array."""
        j0, j1 = self.modes[rank]
        return full[:, :, j0:j1]

    def exchange_bytes(self, nfield: int, itemsize: int = 8):
        """Bytes leaving all ranks for one transpose of nfield fields (own blocks excluded)."""
        tot = 0
        for src in range(self.world):
            for dst in range(self.world):
                if src != dst:
                    tot += 2 * self.nshell(dst) * self.nmode(src) * itemsize * nfield
        return tot


def mode_to_shell(x_mode, dec: Decomposition, rank: int, group=None):
    """(nfield, 2, nr, nmode(rank)) mode layout -> (nfield, 2, nshell(rank), nlm) shell layout."""
    import torch
    import torch.distributed as dist

    nf = x_mode.shape[0]
    sends = [x_mode[:, :, s0:s1, :].contiguous().reshape(-1) for (s0, s1) in dec.shells]
    send = torch.cat(sends)
    in_splits = [t.numel() for t in sends]
    out_splits = [nf * 2 * dec.nshell(rank) * dec.nmode(s) for s in range(dec.world)]
    recv = torch.empty(sum(out_splits), dtype=x_mode.dtype, device=x_mode.device)
    dist.all_to_all_single(recv, send, out_splits, in_splits, group=group)
    out = torch.empty((nf, 2, dec.nshell(rank), dec.nlm), dtype=x_mode.dtype, device=x_mode.device)
    off = 0
    for s in range(dec.world):
        j0, j1 = dec.modes[s]
        n = out_splits[s]
        out[:, :, :, j0:j1] = recv[off:off + n].reshape(nf, 2, dec.nshell(rank), j1 - j0)
        off += n
    return out


def shell_to_mode(x_shell, dec: Decomposition, rank: int, group=None):
    """(nfield, 2, nshell(rank), nlm) shell layout -> (nfield, 2, nr, nmode(rank)) mode layout."""
    import torch
    import torch.distributed as dist

    nf = x_shell.shape[0]
    sends = [x_shell[:, :, :, j0:j1].contiguous().reshape(-1) for (j0, j1) in dec.modes]
    send = torch.cat(sends)
    in_splits = [t.numel() for t in sends]
    out_splits = [nf * 2 * dec.nshell(s) * dec.nmode(rank) for s in range(dec.world)]
    recv = torch.empty(sum(out_splits), dtype=x_shell.dtype, device=x_shell.device)
    dist.all_to_all_single(recv, send, out_splits, in_splits, group=group)
    out = torch.empty((nf, 2, dec.nr, dec.nmode(rank)), dtype=x_shell.dtype, device=x_shell.device)
    off = 0
    for s in range(dec.world):
        s0, s1 = dec.shells[s]
        n = out_splits[s]
        out[:, :, s0:s1, :] = recv[off:off + n].reshape(nf, 2, s1 - s0, dec.nmode(rank))
        off += n
    return out


def energy_partial(x_mode, dec: Decomposition, rank: int, lof: np.ndarray):
    """0.5 sum (T^2 + P^2) / max(l(l+1), 1) over this rank's modes (src/magnetic.jl:519-542);
    fields (2, 2, nr, nmode): [tor, pol]."""
    import torch

    j0, j1 = dec.modes[rank]
    l = torch.as_tensor(lof[j0:j1], dtype=x_mode.dtype, device=x_mode.device)
    w = 1.0 / torch.clamp(l * (l + 1.0), min=1.0)
    return 0.5 * float((x_mode ** 2 * w).sum())

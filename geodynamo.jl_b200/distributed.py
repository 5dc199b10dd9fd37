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


class DistributedStep:
    """The headline step of one model across the ranks of a process group.

    Rank k owns the m columns ``dec.modes[k]`` (native mode range) for the radial
    half of the step and the shells ``dec.shells[k]`` for the transform half:

    1. ``mode.derivatives``: grad T, curl u, curl B of its modes (all shells);
    2. all-to-all: the five state fields and the seven derivative arrays, its
       modes x each rank's shells, to the shell-slab handles;
    3. ``shell``: the three nonlinear phases on its shells (all modes), with
       the derivatives received instead of computed
       (``set_external_derivatives``); the grids carried from step to step
       (the reference's ordering) stay with the shells;
    4. all-to-all: the five nonlinear terms, its shells x each rank's modes,
       back to the mode handles;
    5. ``mode.implicit_modes``: temperature Dirichlet rows, CNAB2 and the
       history roll of its modes.

    Each rank keeps a full-size mode handle (only its own columns are current)
    and a shell-slab handle of its shells.  ``device_exchange``: the blocks go
    through device buffers (NCCL); otherwise through pinned host buffers (gloo).
    Every kernel computes each column or row independently, so the result equals
    the single-handle step's bit for bit (tests/test_gpu_distributed_step.py)."""

    STATE_FIELDS = (0, 1, 2, 3, 4)
    DERIVED = (0, 1, 2, 3, 4, 5, 6)

    def __init__(self, gdb, cfg: dict, rank: int, world: int, group=None, device: int = 0,
                 precision: str = "fp64", device_exchange: bool = False):
        import torch

        c = dict(cfg)
        lmax, nlat, nlon, nr = c.pop("lmax"), c.pop("nlat"), c.pop("nlon"), c.pop("nr")
        mmax = c.pop("mmax", None)
        self.rank, self.world, self.group = rank, world, group
        self.dec = Decomposition(nr, lmax, mmax, world)
        if min(self.dec.nshell(k) for k in range(world)) < 3:
            raise ValueError("every rank needs at least three shells")
        self.mode = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, device=device, **c)
        s0, s1 = self.dec.shells[rank]
        self.shell = gdb.SHTnsKitConfig(lmax, nlat, nlon, s1 - s0, mmax=mmax, precision=precision, device=device, **c)
        self.shell.set_external_derivatives(True)
        self.nr = nr
        self.magnetic = c.get("magnetic", 1)
        self.composition = c.get("composition", 0)
        self.torch = torch
        self.dev = torch.device("cuda", device) if device_exchange else torch.device("cpu")
        self.pin = not device_exchange and torch.cuda.is_available()
        self._bufs = {}

    # -- state ---------------------------------------------------------------------
    def set_field(self, name, re, im):
        self.mode.set_field(name, re, im)

    def set_temperature_bc(self, bvals=None, sources=None):
        self.mode.set_temperature_bc(bvals, None)
        if sources is not None:
            s0, s1 = self.dec.shells[self.rank]
            self.shell.set_temperature_bc(None, np.asarray(sources, dtype=np.float64)[s0:s1])

    def set_composition_bc(self, bvals=None, sources=None):
        self.mode.set_composition_bc(bvals, None)
        if sources is not None:
            s0, s1 = self.dec.shells[self.rank]
            self.shell.set_composition_bc(None, np.asarray(sources, dtype=np.float64)[s0:s1])

    def set_bc_types(self, name, inner, outer):
        self.mode.set_bc_types(name, inner, outer)  # the boundary rows act in the mode layout

    def own_modes(self, name):
        """(re, im) of this rank's m columns of a state field, shape (nr, j1 - j0) each (native order)."""
        j0, j1 = self.dec.modes[self.rank]
        buf = self._buf(2 * self.nr * (j1 - j0))
        self.mode.copy_block(0, FIELD_IDS[name], 0, self.nr, j0, j1, buf.data_ptr(), True)
        a = buf.cpu().numpy().reshape(2, self.nr, j1 - j0)
        return a[0].copy(), a[1].copy()

    def energy(self, lof_native):
        """Kinetic and magnetic energy (the reference's formula) summed over every rank's modes."""
        import torch.distributed as dist
        parts = []
        for names in (("u_tor", "u_pol"), ("b_tor", "b_pol")):
            x = np.stack([np.stack(self.own_modes(n)) for n in names])  # (2, 2, nr, nmode)
            parts.append(energy_partial(self.torch.as_tensor(x), self.dec, self.rank, lof_native))
        t = self.torch.tensor(parts, dtype=self.torch.float64, device=self.dev)
        dist.all_reduce(t, group=self.group)
        return float(t[0]), float(t[1])

    # -- the step --------------------------------------------------------------------
    def _buf(self, n, tag=None):
        """An exchange buffer of n doubles; tagged buffers are kept between steps
        (page-locking host memory costs far more than one exchange)."""
        if tag is not None and tag in self._bufs and self._bufs[tag].numel() == n:
            return self._bufs[tag]
        t = self.torch.empty(n, dtype=self.torch.float64, device=self.dev)
        t = t.pin_memory() if self.pin else t
        if tag is not None:
            self._bufs[tag] = t
        return t

    def _exchange(self, src_handle, dst_handle, items, send_block, recv_block):
        """One all-to-all of spectral blocks: items = [(array, field)], send_block(k) /
        recv_block(k) = ((r0, r1), (j0, j1)) of the block sent to / received from rank k."""
        import torch.distributed as dist
        sizes_s = [2 * (b[0][1] - b[0][0]) * (b[1][1] - b[1][0]) for b in map(send_block, range(self.world))]
        sizes_r = [2 * (b[0][1] - b[0][0]) * (b[1][1] - b[1][0]) for b in map(recv_block, range(self.world))]
        ni = len(items)
        tag = (id(src_handle), len(items))
        send = self._buf(ni * sum(sizes_s), ("send",) + tag)
        recv = self._buf(ni * sum(sizes_r), ("recv",) + tag)
        off = 0
        for k in range(self.world):
            (r0, r1), (j0, j1) = send_block(k)
            for (arr, f) in items:
                if sizes_s[k]:
                    src_handle.copy_block(arr, f, r0, r1, j0, j1, send[off:].data_ptr(), True)
                off += sizes_s[k]
        dist.all_to_all_single(recv, send, [ni * n for n in sizes_r], [ni * n for n in sizes_s], group=self.group)
        if self.dev.type == "cuda":
            # the handles' copies run on their own streams: wait for the exchange
            self.torch.cuda.current_stream(self.dev).synchronize()
        off = 0
        for k in range(self.world):
            (r0, r1), (j0, j1) = recv_block(k)
            for (arr, f) in items:
                if sizes_r[k]:
                    dst_handle.copy_block(arr, f, r0, r1, j0, j1, recv[off:].data_ptr(), False)
                off += sizes_r[k]

    def step(self, n=1):
        me = self.rank
        j0, j1 = self.dec.modes[me]
        s0, s1 = self.dec.shells[me]
        ns = s1 - s0
        fields = self.STATE_FIELDS if self.magnetic else (0, 1, 4)
        derived = self.DERIVED if self.magnetic else (0, 1, 2, 3, 4)
        if self.composition:  # the composition and its gradient (work 8-10)
            fields = fields + (5,)
            derived = derived + (8, 9, 10)
        out_items = [(0, f) for f in fields] + [(1, k) for k in derived]
        nl_items = [(2, f) for f in fields]
        for _ in range(n):
            self.mode.derivatives(j0, j1)
            # mode layout (its modes, every shell) -> shell layout (its shells, every mode)
            self._exchange(self.mode, self.shell, out_items,
                           lambda k: (self.dec.shells[k], (j0, j1)),
                           lambda k: ((0, ns), self.dec.modes[k]))
            # the whole handle's CNAB2 step order: the temperature phase reads the
            # velocity grids carried from the previous step
            self.shell.temperature_nl()
            self.shell.velocity_nl()
            if self.magnetic:
                self.shell.magnetic_nl()
            if self.composition:
                self.shell.composition_nl()
            # nonlinear terms back: shell layout -> mode layout
            self._exchange(self.shell, self.mode, nl_items,
                           lambda k: ((0, ns), self.dec.modes[k]),
                           lambda k: (self.dec.shells[k], (j0, j1)))
            self.mode.implicit_modes(j0, j1)

    def close(self):
        self.shell.close()
        self.mode.close()


FIELD_IDS = {"u_tor": 0, "u_pol": 1, "b_tor": 2, "b_pol": 3, "temp": 4, "comp": 5}

"""Rank bodies for tests/test_distributed.py (spawned as separate processes,
gloo backend on 127.0.0.1)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))


def _init(rank, world, port, backend="gloo"):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    return dist


def transpose_roundtrip(rank, world, port, nr, lmax, mmax):
    import torch
    import distributed as D
    dist = _init(rank, world, port)
    try:
        dec = D.Decomposition(nr, lmax, mmax, world)
        g = np.random.default_rng(11).standard_normal((3, 2, nr, dec.nlm))
        full = torch.from_numpy(g)
        j0, j1 = dec.modes[rank]
        s0, s1 = dec.shells[rank]
        xs = D.mode_to_shell(full[:, :, :, j0:j1].contiguous(), dec, rank)
        assert torch.equal(xs, full[:, :, s0:s1, :])
        xm = D.shell_to_mode(xs, dec, rank)
        assert torch.equal(xm, full[:, :, :, j0:j1])
    finally:
        dist.destroy_process_group()


def phase_matches_global(rank, world, port):
    """Radial derivative in mode layout, transpose, per-shell synthesis and
    analysis, transpose back: equals the same chain on the whole array."""
    import torch
    import distributed as D
    from oracle.oracle import Oracle, lm_pairs
    import workloads
    dist = _init(rank, world, port)
    try:
        lmax, nlat, nlon, nr = 11, 18, 36, 9
        dec = D.Decomposition(nr, lmax, lmax, world)
        pairs = lm_pairs(lmax, lmax)  # reference (l-major) order
        native = [(l, m) for m in range(lmax + 1) for l in range(m, lmax + 1)]
        ref_of_native = np.array([pairs.index(p) for p in native])
        st = workloads.seeded_state(lmax, lmax, nr, seed=5)
        re, im = st["temp"]
        full = np.stack([re[:, ref_of_native], im[:, ref_of_native]])  # (2, nr, nlm) native
        og = Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr)
        D1 = og.fd_matrix(1)  # dense nr x nr first-derivative matrix

        def chain_whole(x):  # x (2, nr, nlm) native
            d = np.einsum("ij,cjk->cik", D1, x)
            o = Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=x.shape[1])
            rr = np.zeros((x.shape[1], dec.nlm)); ii = np.zeros_like(rr)
            rr[:, ref_of_native] = d[0]; ii[:, ref_of_native] = d[1]
            grid = o.synth_scalar(rr, ii)
            ar, ai = o.analysis_scalar(grid)
            return np.stack([ar[:, ref_of_native], ai[:, ref_of_native]])

        expect = chain_whole(full)
        j0, j1 = dec.modes[rank]
        s0, s1 = dec.shells[rank]
        # mode layout: radial derivative on this rank's columns (all shells)
        dm = np.einsum("ij,cjk->cik", D1, full[:, :, j0:j1])
        xs = D.mode_to_shell(torch.from_numpy(dm[None].copy()), dec, rank)[0].numpy()
        # shell layout: per-shell synthesis and analysis on this rank's shells
        o = Oracle(lmax=lmax, nlat=nlat, nlon=nlon, nr=s1 - s0)
        rr = np.zeros((s1 - s0, dec.nlm)); ii = np.zeros_like(rr)
        rr[:, ref_of_native] = xs[0]; ii[:, ref_of_native] = xs[1]
        grid = o.synth_scalar(rr, ii)
        ar, ai = o.analysis_scalar(grid)
        back = D.shell_to_mode(torch.from_numpy(np.stack([ar[:, ref_of_native], ai[:, ref_of_native]])[None].copy()),
                               dec, rank)[0].numpy()
        err = np.max(np.abs(back - expect[:, :, j0:j1])) / np.max(np.abs(expect))
        assert err < 1e-13, err
        # energy of the mode slabs, reduced over ranks, equals the whole-array energy
        lof = D.native_l(lmax, lmax)
        part = D.energy_partial(torch.from_numpy(np.stack([full[:, :, j0:j1], full[:, :, j0:j1]])), dec, rank, lof)
        t = torch.tensor([part], dtype=torch.float64)
        dist.all_reduce(t)
        w = 1.0 / np.maximum(lof * (lof + 1.0), 1.0)
        whole = 0.5 * 2 * float(np.sum(full ** 2 * w[None, None, :]))
        assert abs(float(t.item()) - whole) <= 1e-12 * whole
    finally:
        dist.destroy_process_group()


class _FakeHandle:
    """A host stand-in for the device handle with the data dependences of the step:
    derivatives couple every shell of a mode; the phases couple every mode of a
    shell and carry a per-shell grid from step to step; the solve couples every
    shell of a mode.  Elementwise arithmetic only, so any split of shells or modes
    gives the same bits."""

    def __init__(self, lmax, nlat, nlon, nr, mmax=None, device=0, precision="fp64", **kw):
        import distributed as D
        self.nr, self.nlm = nr, D.mode_offsets(lmax, lmax if mmax is None else mmax)[-1]
        self.S = np.zeros((5, 2, nr, self.nlm))
        self.W = np.zeros((8, 2, nr, self.nlm))
        self.N = np.zeros((5, 2, nr, self.nlm))
        self.G = np.zeros((nr, self.nlm))
        self.src = np.zeros(nr)
        self.ext = False
        self.magnetic = kw.get("magnetic", 1)
        r = np.arange(nr)
        self.Dr = np.cos(0.3 * (r[:, None] - 2 * r[None, :])) / nr
        self.Ar = np.exp(-np.abs(r[:, None] - r[None, :]) / 3.0) / nr

    def _radial(self, M, x):  # sum_i M[r, i] x[.., i, :], one shell at a time
        out = np.zeros_like(x)
        for i in range(self.nr):
            out += M[:, i, None] * x[..., i:i + 1, :]
        return out

    def set_field(self, name, re, im):
        f = {"u_tor": 0, "u_pol": 1, "b_tor": 2, "b_pol": 3, "temp": 4}[name]
        self.S[f, 0], self.S[f, 1] = re, im

    def set_temperature_bc(self, bvals=None, sources=None):
        if sources is not None:
            self.src = np.asarray(sources, dtype=np.float64).copy()

    def set_external_derivatives(self, enable=True):
        self.ext = bool(enable)

    def derivatives(self, j0, j1):
        for k in range(7):
            self.W[k, :, :, j0:j1] = (k + 1) * self._radial(self.Dr, self.S[k % 5, :, :, j0:j1])

    def _phase(self, fields, dk):
        if not self.ext:
            self.derivatives(0, self.nlm)
        for f, k in zip(fields, dk):
            self.N[f] = np.roll(self.S[f], 1, axis=-1) * self.W[k] + self.G
        self.G = 0.5 * self.G + np.roll(self.S[fields[0], 0], -2, axis=-1) * self.W[dk[-1], 1]

    def velocity_nl(self):
        self._phase((0, 1), (3, 4))

    def magnetic_nl(self):
        self._phase((2, 3), (5, 6))

    def temperature_nl(self):
        self._phase((4,), (0,))
        self.N[4] += self.src[None, :, None] + self.W[1] * self.W[2]

    def implicit_modes(self, j0, j1):
        for f in range(5):
            self.S[f, :, :, j0:j1] += 1e-3 * self._radial(self.Ar, self.N[f, :, :, j0:j1])

    def step(self):
        self.temperature_nl()
        self.velocity_nl()
        if self.magnetic:
            self.magnetic_nl()
        self.implicit_modes(0, self.nlm)

    def copy_block(self, array, field, r0, r1, j0, j1, ptr, to_buf):
        import ctypes
        a = (self.S, self.W, self.N)[array][field]
        n = 2 * (r1 - r0) * (j1 - j0)
        buf = np.ctypeslib.as_array((ctypes.c_double * n).from_address(ptr)).reshape(2, r1 - r0, j1 - j0)
        if to_buf:
            buf[...] = a[:, r0:r1, j0:j1]
        else:
            a[:, r0:r1, j0:j1] = buf

    def close(self):
        pass


class _FakeLib:
    SHTnsKitConfig = _FakeHandle


def distributed_step_fake(rank, world, port, magnetic):
    """DistributedStep's exchanges over fake handles equal one whole handle's steps."""
    import distributed as D
    dist = _init(rank, world, port)
    try:
        cfg = dict(lmax=9, nlat=16, nlon=32, nr=11, magnetic=magnetic)
        rng = np.random.default_rng(3)
        fields = {n: (rng.standard_normal((11, 55)), rng.standard_normal((11, 55)))
                  for n in ("u_tor", "u_pol", "b_tor", "b_pol", "temp")}
        src = rng.standard_normal(11)
        whole = _FakeHandle(**cfg)
        ds = D.DistributedStep(_FakeLib, cfg, rank, world)
        for n, (re, im) in fields.items():
            whole.set_field(n, re, im)
            ds.set_field(n, re, im)
        whole.set_temperature_bc(None, src)
        ds.set_temperature_bc(None, src)
        for _ in range(3):
            whole.step()
        ds.step(3)
        j0, j1 = ds.dec.modes[rank]
        for f, n in enumerate(("u_tor", "u_pol", "b_tor", "b_pol", "temp")):
            re, im = ds.own_modes(n)
            assert np.array_equal(re, whole.S[f, 0, :, j0:j1]), n
            assert np.array_equal(im, whole.S[f, 1, :, j0:j1]), n
        assert np.abs(whole.S).max() > 0
    finally:
        dist.destroy_process_group()


def distributed_step_device(rank, world, port, precision, steps, magnetic, grid=(31, 48, 96, 12), nccl=False,
                            composition=False):
    """DistributedStep on the device (every rank on cuda:0, gloo over pinned host
    buffers; nccl: one rank, NCCL over device buffers) against one whole handle,
    bit for bit; grid = (lmax, nlat, nlon, nr)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_package
    gdb = load_package()
    import distributed as D
    import workloads
    import torch
    if nccl:
        torch.cuda.set_device(0)
    dist = _init(rank, world, port, "nccl" if nccl else "gloo")
    try:
        lmax, nlat, nlon, nr = grid
        phys = dict(workloads.SHELL_PHYSICS)
        cfg = dict(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, dt=1e-5, magnetic=magnetic, **phys)
        if composition:
            cfg.update(composition=1, schmidt=2.0)
        st = workloads.seeded_state(lmax, lmax, nr, seed=7, amp=1e-1)
        src = np.linspace(0.5, 1.5, nr)
        c = dict(cfg)
        whole = gdb.SHTnsKitConfig(c.pop("lmax"), c.pop("nlat"), c.pop("nlon"), c.pop("nr"), precision=precision, **c)
        ds = D.DistributedStep(gdb, cfg, rank, world, precision=precision, device_exchange=nccl)
        names = workloads.FIELD_ORDER if magnetic else ("u_tor", "u_pol", "temp")
        for n in names:
            whole.set_field(n, *st[n])
            ds.set_field(n, *st[n])
        whole.set_temperature_bc(None, src)
        ds.set_temperature_bc(None, src)
        if composition:
            cst = workloads.seeded_state(lmax, lmax, nr, seed=8, amp=1e-1)["temp"]
            names = tuple(names) + ("comp",)
            whole.set_field("comp", *cst)
            ds.set_field("comp", *cst)
            csrc = np.linspace(-0.5, 0.5, nr)
            whole.set_composition_bc(None, csrc)
            ds.set_composition_bc(None, csrc)
            # temperature flux boundaries on every third mode (tau method)
            t = np.where(np.arange(whole.nlm) % 3 == 0, 2, 1)
            whole.set_bc_types("temp", t, t[::-1].copy())
            ds.set_bc_types("temp", t, t[::-1].copy())
        whole.step(steps)
        ds.step(steps)
        j0, j1 = ds.dec.modes[rank]
        import torch
        buf = torch.empty(2 * nr * (j1 - j0), dtype=torch.float64).pin_memory()
        worst = 0.0
        for n in names:
            f = D.FIELD_IDS[n]
            whole.copy_block(0, f, 0, nr, j0, j1, buf.data_ptr(), True)
            ref = buf.numpy().reshape(2, nr, j1 - j0).copy()
            re, im = ds.own_modes(n)
            got = np.stack([re, im])
            err = float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300))
            worst = max(worst, err)
            assert np.array_equal(got, ref), (n, err)
        ek, em = ds.energy(D.native_l(lmax, lmax))
        wk, wm = whole.energy()
        assert abs(ek - wk) <= 1e-12 * abs(wk), (ek, wk)
        assert abs(em - wm) <= 1e-12 * max(abs(wm), 1e-300), (em, wm)
        print(f"rank {rank} {precision} magnetic={magnetic}: max rel diff to one handle {worst:.2e}")
        ds.close()
        whole.close()
    finally:
        dist.destroy_process_group()

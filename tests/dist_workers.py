"""Rank bodies for tests/test_distributed.py (spawned as separate processes,
gloo backend on 127.0.0.1)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))


def _init(rank, world, port):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
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

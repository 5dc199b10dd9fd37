"""The allocation-free scalar synthesis, through the C ABI.

gd_spectral_to_physical_noalloc serves callers that may not allocate device
memory at call time (a Julia session whose GPU memory belongs to CUDA.jl's
pool, a solver loop that forbids allocation after set-up): its Fourier
intermediate lives in a fixed array inside the library.  The test allocates
its own device buffers with torch (the caller side) and checks two calls in a
row against gd_spectral_to_physical on the same handle, plus the size limit.
This file sorts last so a stop-at-first-failure run has already run every
other test."""
import ctypes
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def native_coefficients(re, im, lmax, mmax):
    """Reference layout (nfield, nr, nlm) l-major -> native (nfield, 2, nr, nlm) m-major."""
    pairs = [(l, m) for l in range(lmax + 1) for m in range(min(l, mmax) + 1)]
    moff = np.zeros(mmax + 2, dtype=np.int64)
    for m in range(mmax + 1):
        moff[m + 1] = moff[m] + (lmax - m + 1)
    perm = np.array([moff[m] + (l - m) for l, m in pairs])
    out = np.zeros((re.shape[0], 2, re.shape[1], re.shape[2]))
    out[:, 0][..., perm] = re
    out[:, 1][..., perm] = im
    return out


def test_noalloc_synthesis_matches_host_entry_point(gdb):
    import torch
    lmax, nlat, nlon, nr, nf = 31, 48, 96, 12, 5
    cfg = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr)
    re, im = workloads.transform_batch(lmax, lmax, nr, nf, seed=11)
    ref = cfg.synth_scalar(re, im)                      # (nf, nr, nlon, nlat)
    d_coef = torch.from_numpy(native_coefficients(re, im, lmax, lmax)).to("cuda:0")
    d_grid = torch.empty((nf, nr, nlat, nlon), dtype=torch.float64, device="cuda:0")
    lib = cfg.lib
    for call in range(2):
        d_grid.fill_(float("nan"))
        torch.cuda.synchronize()
        st = lib.gd_spectral_to_physical_noalloc(cfg.h, nf, ctypes.c_void_p(d_coef.data_ptr()),
                                                 ctypes.c_void_p(d_grid.data_ptr()))
        assert st == 0, lib.gd_last_error(cfg.h)
        cfg.synchronize()
        out = d_grid.cpu().numpy().transpose(0, 1, 3, 2)
        assert np.all(np.isfinite(out)), call
        assert rel(out, ref) < TOL, call


def test_noalloc_rejects_oversize_scratch(gdb):
    import torch
    cfg = gdb.SHTnsKitConfig(127, 192, 384, 129)   # 50.7 MB of Fourier scratch per field
    d_coef = torch.zeros((2, 2, 129, cfg.nlm), dtype=torch.float64, device="cuda:0")
    d_grid = torch.zeros((2, 129, 192, 384), dtype=torch.float64, device="cuda:0")
    st = cfg.lib.gd_spectral_to_physical_noalloc(cfg.h, 2, ctypes.c_void_p(d_coef.data_ptr()),
                                                 ctypes.c_void_p(d_grid.data_ptr()))
    assert st == 2
    assert b"maximum" in cfg.lib.gd_last_error(cfg.h)

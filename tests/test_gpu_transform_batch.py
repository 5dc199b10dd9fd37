"""The transform-only configuration: forward and inverse scalar transforms at
lmax 127 (nlat 192, nlon 384) over 97 radial shells x 9 fields, seeded
complex Gaussian coefficients x (l+1)^-1.5, through the C ABI in both
precision modes, against the FP64 oracle.

Errors are relative to the field's max-norm (max |a - b| / max |b|) and, for
the RMS figure, RMS(a - b) / RMS(b).  FP64 path: 1e-12 per transform, 1e-11
for the round trip; mixed path (split-TF32 Legendre, FP32 phi transforms):
5e-6, the single-transform tolerance of the other mixed-path tests."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

CFG = workloads.CONFIGS["transform_l127_nr97x9"]


def errs(a, b):
    a = np.asarray(a); b = np.asarray(b)
    mx = float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    rms = float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))
    return mx, rms


@pytest.fixture(scope="module")
def batch(oracle_mod):
    L, nlat, nlon, nr, nf = CFG["lmax"], CFG["nlat"], CFG["nlon"], CFG["nr"], CFG["nfield"]
    re, im = workloads.transform_batch(L, L, nr, nf, seed=0)
    o = oracle_mod.Oracle(lmax=L, nlat=nlat, nlon=nlon, nr=nr)
    grids = np.stack([o.synth_scalar(re[f], im[f]) for f in range(nf)])
    ana = [o.analysis_scalar(grids[f]) for f in range(nf)]
    return re, im, grids, ana


@pytest.mark.parametrize("precision,tol,tol_rt", [("fp64", 1e-12, 1e-11), ("mixed", 5e-6, 5e-6)])
def test_transform_batch_matches_oracle(gdb, batch, precision, tol, tol_rt):
    re, im, grids, ana = batch
    g = gdb.SHTnsKitConfig(CFG["lmax"], CFG["nlat"], CFG["nlon"], CFG["nr"], precision=precision)
    out = g.synth_scalar(re, im)
    back_re, back_im = g.analysis_scalar(grids)
    rt_re, rt_im = g.analysis_scalar(out)
    for f in range(CFG["nfield"]):
        assert errs(out[f], grids[f])[0] < tol, ("synthesis", f)
        assert errs(back_re[f], ana[f][0])[0] < tol and errs(back_im[f], ana[f][1])[0] < tol, ("analysis", f)
        assert errs(rt_re[f], re[f])[0] < tol_rt and errs(rt_im[f], im[f])[0] < tol_rt, ("round trip", f)
    g.close()

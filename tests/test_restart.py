"""CPU tests of the restart files (geodynamo.jl_b200/restart.py): the
reference's restart variables and dimensions (src/outputs_writer.jl:1221-1371)
written as netCDF-3 and read back exactly, on a stand-in model that holds
numpy arrays (no device)."""
import os
import sys

import numpy as np
import pytest
from scipy.io import netcdf_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import restart  # noqa: E402
import workloads  # noqa: E402


class StandIn:
    """The parts of SHTnsKitConfig a restart file touches, on host arrays."""

    def __init__(self, lmax, nlat, nlon, nr, mmax=None, seed=0):
        mmax = lmax if mmax is None else mmax
        self.nlat, self.nlon, self.nr = nlat, nlon, nr
        L, M = workloads.lm_arrays(lmax, mmax)
        self.l_values, self.m_values = L, M
        self.nlm = len(L)
        self.r = np.linspace(0.5385, 1.5385, nr)
        self.theta_grid = np.arccos(np.polynomial.legendre.leggauss(nlat)[0][::-1])
        self.phi_grid = 2 * np.pi * np.arange(nlon) / nlon
        self.fields = {k: (np.zeros((nr, self.nlm)), np.zeros((nr, self.nlm))) for k in restart.COMPONENTS}
        self.steps = 0
        if seed is not None:
            for k, v in workloads.seeded_state(lmax, mmax, nr, seed=seed).items():
                self.fields[k] = (v[0].copy(), v[1].copy())

    def spec_shape(self):
        return (self.nr, self.nlm)

    def step_count(self):
        return self.steps

    def get_field(self, k):
        return self.fields[k][0].copy(), self.fields[k][1].copy()

    def set_field(self, k, re, im):
        self.fields[k] = (np.array(re, dtype=np.float64), np.array(im, dtype=np.float64))

    def synth_scalar(self, re, im):
        # a stand-in grid: any deterministic (nr, nlon, nlat) array
        return np.broadcast_to(re.sum(axis=1)[:, None, None], (self.nr, self.nlon, self.nlat)).copy()


def test_restart_layout_matches_reference_variables(tmp_path):
    m = StandIn(6, 12, 24, 5)
    m.steps = 17
    fn = restart.write_restart(m, str(tmp_path / "restart_rank_0000.nc"), time=0.25, output_count=3,
                               restart_count=1)
    f = netcdf_file(fn, "r", mmap=False)
    try:
        assert f.version_byte == 2
        dims = dict(f.dimensions)
        assert dims == {"time": 1, "r": 5, "theta": 12, "phi": 24, "spectral_mode": m.nlm, "scalar": 1}
        for comp in restart.COMPONENTS.values():
            for part in ("real", "imag"):
                v = f.variables["%s_%s" % (comp, part)]
                assert v.dimensions == ("r", "spectral_mode") and v.typecode() == "d"
                assert v.representation == b"spectral_space"
        assert f.variables["temperature"].dimensions == ("r", "phi", "theta")
        for name in ("time", "step", "r", "theta", "phi", "l_values", "m_values", "last_output_time",
                     "output_count", "restart_count", "grid_file_written"):
            assert name in f.variables, name
        assert f.variables["step"][0] == 17 and f.variables["time"][0] == 0.25
        assert f.Conventions == b"CF-1.8" and f.geometry == b"shell"
        assert np.array_equal(f.variables["l_values"][:], m.l_values)
    finally:
        f.close()


def test_restart_round_trip_is_exact(tmp_path):
    a = StandIn(10, 18, 36, 7, mmax=6, seed=4)
    fn = restart.write_restart(a, str(tmp_path / "r.nc"), time=1.5, step=40, last_output_time=1.25)
    data, meta = restart.read_restart(fn)
    assert meta["current_time"] == 1.5 and meta["current_step"] == 40 and meta["last_output_time"] == 1.25
    for k, comp in restart.COMPONENTS.items():
        assert np.array_equal(data[comp]["real"], a.fields[k][0]) and np.array_equal(data[comp]["imag"], a.fields[k][1])
    b = StandIn(10, 18, 36, 7, mmax=6, seed=None)
    restart.load_restart(b, fn)
    for k in restart.COMPONENTS:
        assert np.array_equal(b.fields[k][0], a.fields[k][0]) and np.array_equal(b.fields[k][1], a.fields[k][1])


def test_restart_rejects_a_different_configuration(tmp_path):
    fn = restart.write_restart(StandIn(10, 18, 36, 7, seed=1), str(tmp_path / "r.nc"))
    with pytest.raises(ValueError):
        restart.load_restart(StandIn(10, 18, 36, 7, mmax=6, seed=None), fn)   # other (l, m) modes
    with pytest.raises(ValueError):
        restart.load_restart(StandIn(10, 18, 36, 9, seed=None), fn)           # other shell count

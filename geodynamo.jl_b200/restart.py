"""Spectral restart files in the reference's NetCDF layout.

``write_restart!`` / ``read_restart!`` (src/outputs_writer.jl:1221-1371) keep
one file per rank holding the spectral state -- the real and imaginary
coefficient planes of velocity, magnetic field and temperature on
(spectral_mode, r) -- plus the physical temperature on (theta, phi, r), the
coordinates, time and step, and the output tracker's counters.  This module
writes and reads the same dimensions, variables and attributes
(setup_coordinates! :410-464, setup_field_variables! :466-540,
write_time_data! :633-642).

Format: the reference creates NETCDF4 (HDF5) files; HDF5 is not available
here, so the files are netCDF-3 with 64-bit offsets (``scipy.io.netcdf_file``,
version 2), which every netCDF library reads, NetCDF.jl's ``NetCDF.open`` in
``read_restart!`` included.  Differences, each forced by the format or kept
to describe the solver's actual grid:

- dimension order is the C order of the file, the reverse of the reference's
  Julia order: spectral variables are ("r", "spectral_mode"), the temperature
  ("r", "phi", "theta"), matching the host layout of this package;
- ``geometry`` is a global attribute (netCDF-3 has no string variables);
- ``r``, ``theta``, ``phi`` hold the solver's radial nodes, Gauss colatitudes
  and longitudes (the reference writes uniform placeholder ranges,
  :289-291), and ``l_values`` / ``m_values`` the configuration's l-major
  (l, m) pairs (the reference's list assumes mmax = lmax, :293-303).

Restart semantics follow the reference: ``read_restart!`` returns the
spectral fields and the run continues from them as a new run (its step
counter starts from zero, so the first step takes the AB1 start,
src/simulation.jl:1153, and the physical grids carried between steps start as
zeros).  ``load_restart`` does the same on a fresh model.
"""
from __future__ import annotations

import time as _time

import numpy as np
from scipy.io import netcdf_file

# field key of this package -> component name of the reference's files
COMPONENTS = {
    "u_tor": "velocity_toroidal",
    "u_pol": "velocity_poloidal",
    "b_tor": "magnetic_toroidal",
    "b_pol": "magnetic_poloidal",
    "temp": "temperature_spectral",
}


def write_restart(model, filename, time=0.0, step=None, last_output_time=0.0, output_count=0, restart_count=0,
                  grid_file_written=True, rank=0, nprocs=1, physical_temperature=True, metadata=None):
    """Writes the model's spectral state (and its physical temperature, the
    model's own synthesis of the spectral temperature) to ``filename`` in the
    restart layout of write_restart! (outputs_writer.jl:1221).

    ``step`` defaults to the model's step count; the tracker counters are
    stored as given.  Returns the filename."""
    step = model.step_count() if step is None else int(step)
    nr, nlm = model.spec_shape()
    f = netcdf_file(filename, "w", version=2)
    try:
        # global attributes (create_netcdf_file, :363-398)
        f.title = "GeoDynamo Simulation Output"
        f.source = "GeoDynamo simulation code"
        f.history = "Created on %s by rank %d" % (_time.strftime("%Y-%m-%dT%H:%M:%S"), rank)
        f.Conventions = "CF-1.8"
        f.mpi_rank = np.int32(rank)
        f.mpi_total_ranks = np.int32(nprocs)
        f.geometry = "shell"
        meta = {"current_time": float(time), "current_step": np.int32(step), "restart_time": float(time),
                "last_output_time": float(last_output_time), "output_count": np.int32(output_count),
                "restart_count": np.int32(restart_count)}
        meta.update(metadata or {})
        for k, v in meta.items():
            setattr(f, k, np.int32(v) if isinstance(v, (int, np.integer)) and not isinstance(v, bool) else v)
        # coordinates (setup_coordinates!, :410-464)
        f.createDimension("time", 1)
        tv = f.createVariable("time", "d", ("time",))
        tv.long_name = "simulation_time"
        tv.units = "dimensionless"
        sv = f.createVariable("step", "i", ("time",))
        sv.long_name = "simulation_step"
        f.createDimension("r", nr)
        rv = f.createVariable("r", "d", ("r",))
        rv.long_name = "radial_coordinate"
        rv.units = "dimensionless"
        rv.valid_range = np.array([model.r[0], model.r[-1]])
        f.createDimension("theta", model.nlat)
        th = f.createVariable("theta", "d", ("theta",))
        th.long_name = "colatitude"
        th.units = "radians"
        th.valid_range = np.array([0.0, np.pi])
        f.createDimension("phi", model.nlon)
        ph = f.createVariable("phi", "d", ("phi",))
        ph.long_name = "azimuthal_angle"
        ph.units = "radians"
        ph.valid_range = np.array([0.0, 2 * np.pi])
        f.createDimension("spectral_mode", nlm)
        lv = f.createVariable("l_values", "i", ("spectral_mode",))
        lv.long_name = "spherical_harmonic_degree"
        mv = f.createVariable("m_values", "i", ("spectral_mode",))
        mv.long_name = "spherical_harmonic_order"
        # fields (setup_field_variables!, :466-540)
        if physical_temperature:
            tp = f.createVariable("temperature", "d", ("r", "phi", "theta"))
            tp.long_name = "temperature"
            tp.units = "dimensionless"
            tp.representation = "physical_space"
        for comp in COMPONENTS.values():
            for part, word in (("real", "real"), ("imag", "imaginary")):
                v = f.createVariable("%s_%s" % (comp, part), "d", ("r", "spectral_mode"))
                v.long_name = "%s_%s_coefficients" % (comp, word)
                v.representation = "spectral_space"
        # restart variables (write_restart!, :1246-1251)
        f.createDimension("scalar", 1)
        lo = f.createVariable("last_output_time", "d", ("scalar",))
        oc = f.createVariable("output_count", "i", ("scalar",))
        rc = f.createVariable("restart_count", "i", ("scalar",))
        gw = f.createVariable("grid_file_written", "i", ("scalar",))
        # data (write_coordinates! / write_field_data! / write_time_data!)
        tv[:] = [float(time)]
        sv[:] = [step]
        rv[:] = model.r
        th[:] = model.theta_grid
        ph[:] = model.phi_grid
        lv[:] = model.l_values
        mv[:] = model.m_values
        spec = {k: model.get_field(k) for k in COMPONENTS}
        for k, comp in COMPONENTS.items():
            f.variables[comp + "_real"][:] = spec[k][0]
            f.variables[comp + "_imag"][:] = spec[k][1]
        if physical_temperature:
            tp[:] = model.synth_scalar(*spec["temp"])
        lo[:] = [float(last_output_time)]
        oc[:] = [int(output_count)]
        rc[:] = [int(restart_count)]
        gw[:] = [1 if grid_file_written else 0]
    finally:
        f.close()
    return filename


def read_restart(filename):
    """Reads a restart file: ``(restart_data, metadata)`` as read_restart!
    (outputs_writer.jl:1275-1371) returns them -- restart_data[component] =
    {"real": (nr, nlm), "imag": (nr, nlm)} for every spectral component present
    and restart_data["temperature"] the physical temperature if present;
    metadata holds current_time, current_step and the tracker counters."""
    f = netcdf_file(filename, "r", mmap=False)
    try:
        names = set(f.variables)
        meta = {"current_time": float(f.variables["time"][0]), "current_step": int(f.variables["step"][0])}
        for k in ("last_output_time", "output_count", "restart_count"):
            if k in names:
                meta[k] = f.variables[k][0].item()
        meta["grid_file_written"] = bool(f.variables["grid_file_written"][0]) if "grid_file_written" in names else True
        data = {}
        if "temperature" in names:
            data["temperature"] = np.array(f.variables["temperature"][:], dtype=np.float64)
        for comp in list(COMPONENTS.values()) + ["composition_spectral"]:
            re, im = comp + "_real", comp + "_imag"
            if re in names and im in names:
                data[comp] = {"real": np.array(f.variables[re][:], dtype=np.float64),
                              "imag": np.array(f.variables[im][:], dtype=np.float64)}
        for k in ("l_values", "m_values", "r", "theta", "phi"):
            if k in names:
                meta[k] = np.array(f.variables[k][:])
    finally:
        f.close()
    return data, meta


def load_restart(model, filename):
    """Reads ``filename`` and sets the model's five spectral fields from it.
    The restarted run continues as a new run (see the module docstring): use a
    model whose step count is zero.  Raises ValueError when the file's shape or
    (l, m) ordering does not match the model.  Returns the metadata."""
    data, meta = read_restart(filename)
    if "l_values" in meta and (len(meta["l_values"]) != model.nlm or
                               not np.array_equal(meta["l_values"], model.l_values) or
                               not np.array_equal(meta["m_values"], model.m_values)):
        raise ValueError("restart file's (l, m) modes do not match the model")
    for key, comp in COMPONENTS.items():
        if comp not in data:
            raise ValueError("restart file has no %s" % comp)
        re, im = data[comp]["real"], data[comp]["imag"]
        if re.shape != model.spec_shape():
            raise ValueError("restart file's %s has shape %s, the model %s" % (comp, re.shape, model.spec_shape()))
        model.set_field(key, re, im)
    return meta

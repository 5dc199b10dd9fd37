"""CPU tests of the host side: the C-ABI library loads and exports every
symbol include/gdb200.h declares, argument validation needs no GPU, and the
index/workload helpers match the reference's conventions."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "gdb200.h")).read()
    return sorted(set(re.findall(r"\b(gd_[a-z_0-9]+)\s*\(", text)))


def test_header_and_exports_agree(gdb):
    syms = header_symbols()
    assert syms, "no declarations parsed"
    assert sorted(gdb.EXPORTS) == syms


def test_library_loads_and_exports_every_symbol(gdb):
    lib = gdb.load_library()
    for name in header_symbols():
        assert hasattr(lib, name), name
    assert os.path.basename(gdb.library_path()) == "libgdb200.so"


def test_invalid_configs_are_rejected_before_any_device_call(gdb):
    lib = gdb.load_library()
    bad = [
        dict(nlat=13),              # odd nlat
        dict(nlat=6),               # nlat <= lmax
        dict(nlon=12),              # nlon <= 2 mmax
        dict(kl=3),                 # i_KL other than 4
        dict(ekman=0.0),            # reference raises ArgumentError
        dict(dt=-1.0),
    ]
    for override in bad:
        kw = dict(lmax=7, mmax=7, nlat=12, nlon=24, nr=9, kl=4, rratio=0.35, ekman=3e-4, rayleigh=80.0,
                  prandtl=1.0, magnetic_prandtl=4.0, dt=1e-5, implicit_theta=0.5, ab_mode=0, bc_mode=0,
                  fd_mode=0, precision=0, magnetic=1)
        kw.update(override)
        cfg = gdb.GDConfig(**kw)
        h = ctypes.c_void_p()
        st = lib.gd_create(ctypes.byref(cfg), 0, ctypes.byref(h))
        assert st == 2, (override, st)   # GD_ERR_CONFIG
        assert not h.value
    assert lib.gd_destroy(None) == 1


def test_index_to_lm_matches_reference_loop(gdb):
    # index_to_lm_shtnskit (src/shtnskit_field_functions.jl:450-462), 1-based
    for lmax, mmax in ((6, 6), (10, 4), (31, 31)):
        idx = 0
        for l in range(lmax + 1):
            for m in range(min(l, mmax) + 1):
                idx += 1
                assert gdb.index_to_lm_shtnskit(idx, lmax, mmax) == (l, m)


def test_seeded_state_is_deterministic_and_shaped(gdb):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
    import workloads
    a = workloads.seeded_state(7, 7, 9, seed=0)
    b = workloads.seeded_state(7, 7, 9, seed=0)
    L, M = workloads.lm_arrays(7, 7)
    for k in workloads.FIELD_ORDER:
        assert a[k][0].shape == (9, L.size)
        assert np.array_equal(a[k][0], b[k][0])
        assert np.all(a[k][1][:, M == 0] == 0)
    assert np.all(a["u_tor"][0][:, L == 0] == 0)
    assert np.any(a["temp"][0][:, L == 0] != 0)

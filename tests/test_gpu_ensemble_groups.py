"""GPU tests of grouped ensembles: members whose configurations differ only in
the Ekman and Rayleigh numbers and the number of radial levels share one
segmented handle (gd_config.segments, segment_nr), their shells stacked along
r, each segment with its own radial grid and operators (one set per length)
and its own Coriolis factor.

A grouped member runs the same arithmetic on the same inputs as the member
stepped on its own handle (every per-shell kernel treats the shells alike, the
radial operators act within the segment, the energy sums each segment in the
order of an unsegmented handle): fields and energies must be bitwise equal to
single handles, FP64 and mixed precision alike."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402

NAMES = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")
GRID_KEYS = ("lmax", "nlat", "nlon", "nr")


def load(model, lmax, nr, seed):
    for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=seed).items():
        model.set_field(k, a, b)


def same_shape_members(n=64, want=3):
    """Draw indices of the first (lmax, nr) class of the seeded draw with at
    least `want` members, and of a second class (for a mixed grouping)."""
    classes = {}
    for i, c in enumerate(workloads.ensemble_draw(n)):
        classes.setdefault((c["lmax"], c["nr"]), []).append((i, c))
    big = [v for v in classes.values() if len(v) >= want]
    big.sort(key=lambda v: (v[0][1]["lmax"], v[0][1]["nr"]))
    return big[0][:want], big[1][:2]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_grouped_members_equal_single_handles(gdb, precision):
    first, second = same_shape_members()
    picks = first + second
    # interleaved order: the grouping is by configuration, not by position
    order = [picks[0], picks[3], picks[1], picks[4], picks[2]]
    assert len({c["ekman"] for _, c in order}) == len(order)
    ens = gdb.Ensemble([dict(c, precision=precision) for _, c in order], group=8)
    # the two classes share lmax 31: one handle, segments of 33 and 49 levels
    assert {c["nr"] for _, c in order} == {33, 49}
    assert len(ens.handles) == 1 and ens.handles[0].segments() == 5
    singles = []
    for (i, c), m in zip(order, ens.members):
        load(m, c["lmax"], c["nr"], i)
        kw = {k: v for k, v in c.items() if k not in GRID_KEYS}
        s = gdb.SHTnsKitConfig(c["lmax"], c["nlat"], c["nlon"], c["nr"], precision=precision, **kw)
        load(s, c["lmax"], c["nr"], i)
        singles.append(s)
    ens.step(4)
    for s in singles:
        s.step(4)
    for (i, c), m, s in zip(order, ens.members, singles):
        assert m.step_count() == s.step_count() == 4
        for k in NAMES:
            a, b = m.get_field(k), s.get_field(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (i, k)
        for k in ("u_tor", "temp"):
            a, b = m.get_nl(k), s.get_nl(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (i, k)
        assert m.energy() == s.energy(), i
    # gd_energy of a segmented handle is the sum of its segments' energies
    h = ens.handles[0]
    ek, em = h.segment_energy()
    tk, tm = h.energy()
    assert tk == pytest.approx(float(np.sum(ek)), rel=1e-14)
    assert tm == pytest.approx(float(np.sum(em)), rel=1e-14)
    ens.close()


def test_grouped_member_matches_oracle(gdb, oracle_mod):
    first, _ = same_shape_members()
    ens = gdb.Ensemble([c for _, c in first], group=8)
    assert len(ens.handles) == 1
    oracles = []
    for (i, c), m in zip(first, ens.members):
        load(m, c["lmax"], c["nr"], i)
        kw = {k: v for k, v in c.items() if k not in GRID_KEYS}
        o = oracle_mod.Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], **kw)
        load(o, c["lmax"], c["nr"], i)
        oracles.append(o)
    ens.step(3)
    for o in oracles:
        o.step(3)
    for (i, c), m, o in zip(first, ens.members, oracles):
        for k in NAMES:
            a, b = m.get_field(k), o.get_field(k)
            scale = max(float(np.max(np.abs(b[0]))), 1e-300)
            assert float(np.max(np.abs(a[0] - b[0]))) / scale < 1e-11, (i, k)
            assert float(np.max(np.abs(a[1] - b[1]))) / max(float(np.max(np.abs(b[1]))), 1e-300) < 1e-11, (i, k)
    ens.close()


def test_segmented_handle_refusals(gdb):
    kw = dict(lmax=7, nlat=12, nlon=24)
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(kw["lmax"], kw["nlat"], kw["nlon"], 19, segments=2)
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(kw["lmax"], kw["nlat"], kw["nlon"], 4, segments=2)
    with pytest.raises(gdb.GeoDynamoError):
        gdb.SHTnsKitConfig(kw["lmax"], kw["nlat"], kw["nlon"], 18, segments=2, composition=1, schmidt=2.0)
    g = gdb.SHTnsKitConfig(kw["lmax"], kw["nlat"], kw["nlon"], 18, segments=2)
    assert g.segments() == 2
    with pytest.raises(ValueError):
        g.set_segment_ekman([1e-3])
    with pytest.raises(gdb.GeoDynamoError):
        g.set_segment_ekman([1e-3, -1.0])
    with pytest.raises(gdb.GeoDynamoError):
        g.set_scheme("eab2")
    with pytest.raises(gdb.GeoDynamoError):
        g.set_external_derivatives(True)
    with pytest.raises(gdb.GeoDynamoError):
        g.temperature_forward(2, 1)
    with pytest.raises(gdb.GeoDynamoError):
        g.derivatives(0, g.nlm)
    # the handle still steps after the refusals
    g.set_segment_ekman([1e-3, 3e-4])
    load_two = workloads.seeded_state(7, 7, 18, seed=5)
    for k, (a, b) in load_two.items():
        g.set_field(k, a, b)
    g.step(2)
    g.check_finite()
    ek, em = g.segment_energy()
    assert ek.shape == (2,) and np.all(np.isfinite(ek)) and np.all(ek > 0)


@pytest.mark.parametrize("bc_mode", [0, 1, 2])
def test_segments_keep_their_own_boundary_rows(gdb, bc_mode):
    # two members of one shape on one segmented handle against two single
    # handles: boundary values and flux types (bc_mode 0/1: tau rows on the
    # state; 2: Dirichlet rows in the operator), sources per shell, clamped
    # rows (bc_mode 1); every row operation must act at each segment's own ends
    lmax, nlat, nlon, nr = 15, 24, 48, 9
    members = [dict(lmax=lmax, nlat=nlat, nlon=nlon, nr=nr, ekman=e, bc_mode=bc_mode, dt=2e-6) for e in (3e-4, 7e-4)]
    ens = gdb.Ensemble(members, group=2)
    assert len(ens.handles) == 1
    h = ens.handles[0]
    rng = np.random.default_rng(11)
    nlm = h.nlm
    bv = rng.standard_normal((2, nlm)) * 1e-2
    src = rng.standard_normal(nr)
    inner = np.where(rng.random(nlm) < 0.5, 1, 2) if bc_mode != 2 else np.ones(nlm, dtype=int)
    outer = np.where(rng.random(nlm) < 0.5, 1, 2) if bc_mode != 2 else np.ones(nlm, dtype=int)
    h.set_bc_types("temp", inner, outer)
    h.set_temperature_bc(bv, np.concatenate([src, src]))
    singles = []
    for i, (c, m) in enumerate(zip(members, ens.members)):
        kw = {k: v for k, v in c.items() if k not in ("lmax", "nlat", "nlon", "nr")}
        s = gdb.SHTnsKitConfig(lmax, nlat, nlon, nr, **kw)
        s.set_bc_types("temp", inner, outer)
        s.set_temperature_bc(bv, src)
        for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=20 + i, amp=1e-1).items():
            m.set_field(k, a, b)
            s.set_field(k, a, b)
        singles.append(s)
    ens.step(3)
    for s in singles:
        s.step(3)
    for m, s in zip(ens.members, singles):
        for k in NAMES:
            a, b = m.get_field(k), s.get_field(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (bc_mode, k)
        assert m.energy() == s.energy()
    ens.close()


@pytest.mark.parametrize("bc_mode,precision", [(0, "fp64"), (1, "fp64"), (2, "fp64"), (2, "mixed")])
def test_unequal_segments_equal_single_handles(gdb, bc_mode, precision):
    # members of 9, 13 and 9 levels on one handle (two operator variants):
    # boundary values, per-shell sources, clamped rows (bc_mode 1) and
    # Dirichlet rows (bc_mode 2) at each segment's own ends, and random flux
    # boundaries: the tau correction (bc_mode 0/1) with each segment's own tau
    # functions, flux rows (bc_mode 2) with factors per segment length
    lmax, nlat, nlon = 15, 24, 48
    nrs = (9, 13, 9)
    members = [dict(lmax=lmax, nlat=nlat, nlon=nlon, nr=n, ekman=e, bc_mode=bc_mode, dt=2e-6, precision=precision)
               for n, e in zip(nrs, (3e-4, 5e-4, 8e-4))]
    ens = gdb.Ensemble(members, group=3)
    assert len(ens.handles) == 1 and ens.handles[0].segments() == 3
    h = ens.handles[0]
    rng = np.random.default_rng(12)
    bv = rng.standard_normal((2, h.nlm)) * 1e-2
    srcs = [rng.standard_normal(n) for n in nrs]
    h.set_temperature_bc(bv, np.concatenate(srcs))
    inner = np.where(rng.random(h.nlm) < 0.5, 1, 2)
    outer = np.where(rng.random(h.nlm) < 0.5, 1, 2)
    h.set_bc_types("temp", inner, outer)
    singles = []
    for i, (c, m) in enumerate(zip(members, ens.members)):
        kw = {k: v for k, v in c.items() if k not in ("lmax", "nlat", "nlon", "nr")}
        s = gdb.SHTnsKitConfig(lmax, nlat, nlon, c["nr"], **kw)
        s.set_bc_types("temp", inner, outer)
        s.set_temperature_bc(bv, srcs[i])
        for k, (a, b) in workloads.seeded_state(lmax, lmax, c["nr"], seed=30 + i, amp=1e-1).items():
            m.set_field(k, a, b)
            s.set_field(k, a, b)
        singles.append(s)
    ens.step(3)
    for s in singles:
        s.step(3)
    for m, s in zip(ens.members, singles):
        for k in NAMES:
            a, b = m.get_field(k), s.get_field(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (bc_mode, k)
        assert m.energy() == s.energy()
    ens.close()

"""GPU tests of the batched uneven ensemble (gd_ensemble_*): members of
different sizes and parameters stepped by one graph launch per step.

Each member must evolve exactly as the same model stepped on its own handle
(same kernels, same inputs: bitwise equal), and the FP64 members must track
the oracle to the trajectory tolerance of the single-model tests (1e-11)."""
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


def rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def one_per_lmax(n=64):
    """The first member of the seeded draw for each lmax, with its draw index."""
    seen, out = set(), []
    for i, c in enumerate(workloads.ensemble_draw(n)):
        if c["lmax"] not in seen:
            seen.add(c["lmax"])
            out.append((i, c))
    return out


def load(model, lmax, nr, seed):
    for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=seed).items():
        model.set_field(k, a, b)


def test_ensemble_members_match_oracle(gdb, oracle_mod):
    picks = one_per_lmax()
    assert sorted(c["lmax"] for _, c in picks) == [31, 47, 63, 95]
    ens = gdb.Ensemble([c for _, c in picks])
    oracles = []
    for (i, c), m in zip(picks, ens.members):
        load(m, c["lmax"], c["nr"], i)
        kw = {k: v for k, v in c.items() if k not in GRID_KEYS}
        o = oracle_mod.Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], **kw)
        load(o, c["lmax"], c["nr"], i)
        oracles.append(o)
    ens.step(3)
    for o in oracles:
        o.step(3)
    for (i, c), m, o in zip(picks, ens.members, oracles):
        assert m.step_count() == 3
        for k in NAMES:
            a, b = m.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < 1e-11 and rel(a[1], b[1]) < 1e-11, (i, k)
    ens.close()


def test_mixed_ensemble_members_match_oracle(gdb, oracle_mod):
    # mixed-precision members (split-TF32 Legendre, FP32 phi transforms and
    # products, FP64 solves) against the FP64 oracle at the mixed path's
    # few-step field tolerance
    picks = one_per_lmax()
    ens = gdb.Ensemble([dict(c, precision="mixed") for _, c in picks])
    oracles = []
    for (i, c), m in zip(picks, ens.members):
        load(m, c["lmax"], c["nr"], i)
        kw = {k: v for k, v in c.items() if k not in GRID_KEYS}
        o = oracle_mod.Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], **kw)
        load(o, c["lmax"], c["nr"], i)
        oracles.append(o)
    ens.step(3)
    for o in oracles:
        o.step(3)
    for (i, c), m, o in zip(picks, ens.members, oracles):
        for k in NAMES:
            a, b = m.get_field(k), o.get_field(k)
            assert rel(a[0], b[0]) < 1e-5 and rel(a[1], b[1]) < 1e-5, (i, k)
    ens.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_equals_single_handles(gdb, precision):
    picks = one_per_lmax()[:3]
    ens = gdb.Ensemble([dict(c, precision=precision) for _, c in picks])
    singles = []
    for (i, c), m in zip(picks, ens.members):
        load(m, c["lmax"], c["nr"], i)
        kw = {k: v for k, v in c.items() if k not in GRID_KEYS}
        s = gdb.SHTnsKitConfig(c["lmax"], c["nlat"], c["nlon"], c["nr"], precision=precision, **kw)
        load(s, c["lmax"], c["nr"], i)
        singles.append(s)
    # every member bootstraps in the first ensemble graph; then one member
    # stepped on its own puts the bootstrap flags out of step (it no longer
    # needs the AB1 start while a fresh member would), which the second
    # ensemble call handles through the members' own graphs
    ens.step(2)
    for s in singles:
        s.step(2)
    ens.members[0].step(1)
    singles[0].step(1)
    ens.step(2)
    for s in singles:
        s.step(2)
    for m, s in zip(ens.members, singles):
        assert m.step_count() == s.step_count()
        for k in NAMES:
            a, b = m.get_field(k), s.get_field(k)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), k
        assert m.energy() == s.energy()
    ens.close()


def test_ensemble_rejects_bad_member(gdb):
    good = one_per_lmax()[0][1]
    with pytest.raises(gdb.GeoDynamoError):
        gdb.Ensemble([good, dict(good, nr=2)])


def test_autotune_chooses_caps_without_changing_results(gdb):
    # the launch-shape search steps a scratch ensemble only; the tuned members
    # give the same bits as untuned ones (a tile's arithmetic does not depend on
    # which persistent CTA runs it)
    cfgs = [dict(lmax=l, nlat=3 * (l + 1) // 2, nlon=3 * (l + 1), nr=nr, dt=1e-5)
            for l, nr in ((15, 9), (23, 13), (31, 17), (31, 9))]
    a = gdb.Ensemble(cfgs, precision="mixed")
    b = gdb.Ensemble(cfgs, precision="mixed")
    for i, c in enumerate(cfgs):
        load(a.members[i], c["lmax"], c["nr"], seed=i)
        load(b.members[i], c["lmax"], c["nr"], seed=i)
    ms, caps = a.autotune(3)
    print(f"autotune: {ms:.3f} ms per ensemble step, caps {caps}")
    assert ms > 0 and len(caps) == len(cfgs)
    assert all(0 <= c <= 1024 for c in caps)
    assert [m.launch_shape() for m in a.members] == caps
    assert all(m.step_count() == 0 for m in a.members)
    a.step(3)
    b.step(3)
    for ma, mb in zip(a.members, b.members):
        for k in workloads.FIELD_ORDER:
            for x, y in zip(ma.get_field(k), mb.get_field(k)):
                assert np.array_equal(x, y), k
    a.close()
    b.close()

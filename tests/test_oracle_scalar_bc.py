"""The oracle's scalar boundary conditions (fixed values and the tau flux
correction of apply_scalar_flux_bc_spectral! / apply_flux_bc_tau!,
src/scalar_field_common.jl:590-935, 1166-1198) against a second restatement
written here in numpy from the same Julia lines, for every combination of
inner/outer boundary types, on temperature and composition.  The reference
ships no vectors for these functions, so two independent restatements of its
code are compared."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))
import workloads  # noqa: E402
from oracle import oracle as O  # noqa: E402

VALUE, FLUX = 1, 2


def dense_d1(o):
    band = o.fd_matrix(1)  # rows: band row b = kl + i - j, cols: j
    N, kl = o.nr, o.kl
    D = np.zeros((N, N))
    for i in range(N):
        for j in range(max(0, i - kl), min(N, i + kl + 1)):
            D[i, j] = band[kl + i - j, j]
    return D


def restated_bc(re, im, bv, types, r, D):
    """apply_*_boundary_conditions_spectral! then apply_flux_bc_tau! per mode."""
    re, im = re.copy(), im.copy()
    N = len(r)
    ri, ro = r[0], r[-1]

    def cheb(n):  # compute_chebyshev_polynomial
        x = 2.0 * (r - ri) / (ro - ri) - 1.0
        return np.cos(n * np.arccos(np.clip(x, -1.0, 1.0)))

    def dcheb(n, rr):  # evaluate_chebyshev_derivative
        x = 2.0 * (rr - ri) / (ro - ri) - 1.0
        if abs(abs(x) - 1.0) < 1e-12:
            d = n ** 2 * np.sign(x) ** (n + 1)
        else:
            t = np.arccos(np.clip(x, -1.0, 1.0))
            d = n * np.sin(n * t) / np.sin(t)
        return d * 2.0 / (ro - ri)

    t1, t2 = cheb(N - 1), cheb(N)
    for q in range(re.shape[1]):
        if types[0, q] == VALUE:
            re[0, q], im[0, q] = bv[0, q], 0.0
        if types[1, q] == VALUE:
            re[-1, q], im[-1, q] = bv[1, q], 0.0
    for q in range(re.shape[1]):
        ai, ao = types[0, q] == FLUX, types[1, q] == FLUX
        if not (ai or ao):
            continue
        fi = bv[0, q] if ai else 0.0
        fo = bv[1, q] if ao else 0.0
        dp = D @ re[:, q]
        ei, eo = fi - dp[0], fo - dp[-1]
        if ai and ao:
            d1i, d1o, d2i, d2o = dcheb(N - 1, ri), dcheb(N - 1, ro), dcheb(N, ri), dcheb(N, ro)
            det = d1i * d2o - d1o * d2i
            c1 = c2 = 0.0
            if abs(det) > 1e-12:
                c1 = (ei * d2o - eo * d2i) / det
                c2 = (eo * d1i - ei * d1o) / det
            corr = c1 * t1 + c2 * t2
        elif ai:
            d2o = dcheb(N, ro)
            a = dcheb(N - 1, ro) / d2o if abs(d2o) > 1e-12 else 0.0
            tau = t1 - a * t2
            corr = ei / (D @ tau)[0] * tau
        else:
            d2i = dcheb(N, ri)
            b = dcheb(N - 1, ri) / d2i if abs(d2i) > 1e-12 else 0.0
            tau = t1 - b * t2
            corr = eo / (D @ tau)[-1] * tau
        live = np.any(np.abs(im[:, q]) > 1e-12)
        re[:, q] = re[:, q] + corr
        if live:
            im[:, q] = im[:, q] + corr
    return re, im


def _types(nlm, rng):
    # every (inner, outer) pair of types appears
    t = np.array([[VALUE, VALUE], [VALUE, FLUX], [FLUX, VALUE], [FLUX, FLUX]])
    return t[rng.integers(0, 4, nlm)].T.copy()


def test_tau_flux_bc_matches_restatement():
    lmax, nr = 7, 11
    o = O.Oracle(lmax=lmax, nlat=12, nlon=24, nr=nr, composition=1, schmidt=3.0)
    rng = np.random.default_rng(21)
    st = workloads.seeded_state(lmax, lmax, nr, seed=2)
    for k, (a, b) in st.items():
        o.set_field(k, a, b)
    o.set_field("comp", *workloads.seeded_state(lmax, lmax, nr, seed=3)["temp"])
    D = dense_d1(o)
    r = o.grid()[3]
    nlm = o.nlm
    for name, setter, run in (("temp", o.set_temperature_bc, o.temperature_nl),
                              ("comp", o.set_composition_bc, o.composition_nl)):
        types = _types(nlm, rng)
        bv = rng.standard_normal((2, nlm)) * 1e-3
        o.set_bc_types(name, types[0], types[1])
        setter(bv, None)
        before = o.get_field(name)
        run()
        after = o.get_field(name)
        exp = restated_bc(before[0], before[1], bv, types, r, D)
        for x, y in zip(after, exp):
            assert np.max(np.abs(x - y)) <= 1e-13 * max(np.max(np.abs(y)), 1e-300), name
        # a one-sided flux boundary is met exactly by its D1-normalised tau function
        re = after[0]
        dp = D @ re
        for q in range(nlm):
            if types[0, q] == FLUX and types[1, q] == VALUE:
                assert abs(dp[0, q] - bv[0, q]) <= 1e-9 * (1 + abs(bv[0, q]))
            if types[1, q] == FLUX and types[0, q] == VALUE:
                assert abs(dp[-1, q] - bv[1, q]) <= 1e-9 * (1 + abs(bv[1, q]))


def test_composition_defaults_to_no_flux_and_steps():
    # create_shtns_composition_field: flux boundaries of value 0 everywhere
    lmax, nr = 7, 9
    o = O.Oracle(lmax=lmax, nlat=12, nlon=24, nr=nr, composition=1, schmidt=2.0)
    c = workloads.seeded_state(lmax, lmax, nr, seed=8)["temp"]
    o.set_field("comp", *c)
    D = dense_d1(o)
    r = o.grid()[3]
    before = o.get_field("comp")
    o.composition_nl()
    after = o.get_field("comp")
    types = np.full((2, o.nlm), FLUX)
    exp = restated_bc(before[0], before[1], np.zeros((2, o.nlm)), types, r, D)
    for x, y in zip(after, exp):
        assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(y))
    o.step(3)
    assert np.all(np.isfinite(o.get_field("comp")[0]))


def test_flux_rows_of_the_boundary_row_operator():
    # bc_mode 2 (the boundary-row operator, an added option): a prescribed flux
    # is the boundary row D1 u = flux of the implicit solve, a fixed value the
    # identity row; after each step both hold exactly (to rounding), for every
    # (inner, outer) pair of types, temperature and composition alike
    lmax, nr = 7, 11
    o = O.Oracle(lmax=lmax, nlat=12, nlon=24, nr=nr, composition=1, schmidt=3.0, bc_mode=2, dt=1e-5)
    rng = np.random.default_rng(31)
    for k, (a, b) in workloads.seeded_state(lmax, lmax, nr, seed=4).items():
        o.set_field(k, a, b)
    o.set_field("comp", *workloads.seeded_state(lmax, lmax, nr, seed=5)["temp"])
    D = dense_d1(o)
    nlm = o.nlm
    bvs = {}
    for name, setter in (("temp", o.set_temperature_bc), ("comp", o.set_composition_bc)):
        types = _types(nlm, rng)
        bv = rng.standard_normal((2, nlm)) * 1e-2
        o.set_bc_types(name, types[0], types[1])
        setter(bv, None)
        bvs[name] = (types, bv)
    o.step(3)
    for name, (types, bv) in bvs.items():
        re, im = o.get_field(name)
        dp = D @ re
        for side, row in ((0, 0), (1, -1)):
            flux = types[side] == FLUX
            got = np.where(flux, dp[row], re[row])
            assert np.max(np.abs(got - bv[side])) <= 1e-10 * (1 + np.max(np.abs(bv[side]))), (name, side)
            assert np.max(np.abs(np.where(flux, (D @ im)[row], im[row]))) <= 1e-10, (name, side)

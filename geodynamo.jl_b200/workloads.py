"""Seeded synthetic workloads (no dataset is involved anywhere on this path).

Shell physics shared by every configuration: ri/ro = 0.35, E = 3e-4, Ra = 80,
Pr = 1, Pm = 4, theta = 0.5, i_KL = 4; fields u_tor, u_pol, B_tor, B_pol, T.

Initial state: ``numpy.random.default_rng(seed)`` draws standard normals in the
order field (u_tor, u_pol, b_tor, b_pol, temp) -> r -> l-major (l, m) -> (Re, Im);
coefficient = g * amp * (l + 1)^-power * sin(pi (r - ri) / (ro - ri)); Im = 0 at
m = 0; l = 0 of the toroidal/poloidal fields is zero (as randomize_vector_field!,
src/InitialConditions.jl:81).
"""
from __future__ import annotations

import numpy as np

FIELD_ORDER = ("u_tor", "u_pol", "b_tor", "b_pol", "temp")

SHELL_PHYSICS = dict(rratio=0.35, ekman=3e-4, rayleigh=80.0, prandtl=1.0, magnetic_prandtl=4.0,
                     implicit_theta=0.5, kl=4)

# Named workloads (sizes of the reference's documented configurations).
CONFIGS = {
    "shell_l31_nr32": dict(lmax=31, nlat=48, nlon=96, nr=32, dt=1e-5, steps=100),
    "transform_l127_nr97x9": dict(lmax=127, nlat=192, nlon=384, nr=97, nfield=9),
    "shell_l255_nr129": dict(lmax=255, nlat=384, nlon=768, nr=129, dt=2e-6, steps=1000),
    # the scale-out grid of the shell/mode decomposition (lmax 511 on the
    # headline radial grid)
    "shell_l511_nr129": dict(lmax=511, nlat=768, nlon=1536, nr=129, dt=1e-6, steps=100),
    # the same shell with 33 radial levels: per-shell kernel work of the headline
    # workload at a quarter of its memory (profiling captures)
    "shell_l255_nr33": dict(lmax=255, nlat=384, nlon=768, nr=33, dt=2e-6, steps=100),
    "shell_l127_nr65": dict(lmax=127, nlat=192, nlon=384, nr=65, dt=5e-6, steps=100),
    # the headline's radial grid at lmax 127: the radial kernels' launch shape
    # of the headline workload at a quarter of its memory (profiling captures)
    "shell_l127_nr129": dict(lmax=127, nlat=192, nlon=384, nr=129, dt=2e-6, steps=100),
    # adjoint configuration: the reference's literal boundaries (bc_mode 0; any
    # Dirichlet row on B would pin B_pol(ro) and the misfit to constants),
    # started from adjoint_state (temperature zero)
    "adjoint_l63_nr65": dict(lmax=63, nlat=96, nlon=192, nr=65, dt=1e-5, steps=200, bc_mode=0, checkpoint=20),
}


def lm_arrays(lmax: int, mmax: int):
    L = np.array([l for l in range(lmax + 1) for m in range(min(l, mmax) + 1)])
    M = np.array([m for l in range(lmax + 1) for m in range(min(l, mmax) + 1)])
    return L, M


# Batched uneven ensemble: lmax from {31, 47, 63, 95} with the 3/2-rule grid
# nlat = 3 (lmax + 1) / 2, nlon = 2 nlat; nr from {33, 49, 65}; Ekman
# log-uniform in [1e-4, 1e-3]; Rayleigh uniform in [50, 150]; all from
# default_rng(3) in the order (lmax, nr, E, Ra) per instance; 200 steps at
# dt = 1e-5 (the oracle configuration's step, none being specified);
# instance i starts from seeded_state(seed=i).
ENSEMBLE_LMAX = (31, 47, 63, 95)
ENSEMBLE_NR = (33, 49, 65)


def ensemble_draw(n: int = 64, seed: int = 3):
    """List of n member configurations (dicts of SHTnsKitConfig keywords)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        lmax = int(ENSEMBLE_LMAX[rng.integers(len(ENSEMBLE_LMAX))])
        nr = int(ENSEMBLE_NR[rng.integers(len(ENSEMBLE_NR))])
        ekman = float(10.0 ** rng.uniform(-4.0, -3.0))
        rayleigh = float(rng.uniform(50.0, 150.0))
        nlat = 3 * (lmax + 1) // 2
        c = dict(SHELL_PHYSICS)
        c.update(lmax=lmax, nlat=nlat, nlon=2 * nlat, nr=nr, ekman=ekman, rayleigh=rayleigh, dt=1e-5)
        out.append(c)
    return out


def adjoint_target(lmax: int, mmax: int, seed: int = 1, lcut: int = 12):
    """Target radial-field coefficients of the adjoint configuration: complex
    Gaussian x (l+1)^-2 for l <= lcut, zero above, Im = 0 at m = 0; (re, im),
    each (nlm,) l-major."""
    rng = np.random.default_rng(seed)
    L, M = lm_arrays(lmax, mmax)
    g = rng.standard_normal((L.size, 2))
    c = g * ((L + 1.0) ** -2.0)[:, None] * (L <= lcut)[:, None]
    re = np.ascontiguousarray(c[:, 0])
    im = np.ascontiguousarray(c[:, 1])
    im[M == 0] = 0.0
    return re, im


def adjoint_state(lmax: int, mmax: int, nr: int, seed: int = 0):
    """Initial state of the adjoint configuration: seeded_state with the
    temperature set to zero.  Under the literal operator a nonzero temperature
    overflows within ~150 steps at lmax 63, nr 65; from zero (no sources, zero
    boundary values) it stays exactly zero.  The misfit does not depend on the
    temperature: it never feeds back into the velocity (the vector analysis
    drops the radial buoyancy force, src/shtnskit_field_functions.jl:309-313)
    nor into the magnetic field."""
    st = seeded_state(lmax, mmax, nr, seed=seed)
    re, im = st["temp"]
    st["temp"] = (np.zeros_like(re), np.zeros_like(im))
    return st


def adjoint_directions(lmax: int, mmax: int, nr: int, count: int = 32, seed: int = 2):
    """Random directions for the finite-difference checks of the gradient with
    respect to B_pol: standard normals (nr, nlm) x2 with the state's
    conventions (Im = 0 at m = 0, l = 0 zero), drawn from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    L, M = lm_arrays(lmax, mmax)
    out = []
    for _ in range(count):
        g = rng.standard_normal((nr, L.size, 2))
        re = np.ascontiguousarray(g[..., 0]); im = np.ascontiguousarray(g[..., 1])
        im[:, M == 0] = 0.0
        re[:, L == 0] = 0.0; im[:, L == 0] = 0.0
        out.append((re, im))
    return out


def radial_nodes(nr: int, rratio: float = 0.35):
    """r_n = ri + (1 + cos(pi (N - n) / (N - 1))) / 2, n = 1..N (src/fields.jl:108-131)."""
    ri = rratio / (1.0 - rratio)
    n = np.arange(1, nr + 1)
    return 0.5 * (1.0 + np.cos(np.pi * (nr - n) / (nr - 1))) + ri


def seeded_state(lmax: int, mmax: int, nr: int, seed: int = 0, amp: float = 1e-3, power: float = 2.0,
                 rratio: float = 0.35):
    """Dict field -> (re, im), each (nr, nlm) in the reference layout."""
    rng = np.random.default_rng(seed)
    L, M = lm_arrays(lmax, mmax)
    r = radial_nodes(nr, rratio)
    ri, ro = r[0], r[-1]
    prof = np.sin(np.pi * (r - ri) / (ro - ri))
    out = {}
    for name in FIELD_ORDER:
        g = rng.standard_normal((nr, L.size, 2))
        c = g * amp * ((L + 1.0) ** -power)[None, :, None] * prof[:, None, None]
        re = np.ascontiguousarray(c[..., 0])
        im = np.ascontiguousarray(c[..., 1])
        im[:, M == 0] = 0.0
        if name != "temp":
            re[:, L == 0] = 0.0
            im[:, L == 0] = 0.0
        out[name] = (re, im)
    return out


def transform_batch(lmax: int, mmax: int, nr: int, nfield: int, seed: int = 0, power: float = 1.5):
    """Complex Gaussian coefficients x (l+1)^-power for nfield fields: (nfield, nr, nlm) x2."""
    rng = np.random.default_rng(seed)
    L, M = lm_arrays(lmax, mmax)
    g = rng.standard_normal((nfield, nr, L.size, 2))
    c = g * ((L + 1.0) ** -power)[None, None, :, None]
    re = np.ascontiguousarray(c[..., 0])
    im = np.ascontiguousarray(c[..., 1])
    im[:, :, M == 0] = 0.0
    return re, im

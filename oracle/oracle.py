"""ctypes front end of the CPU FP64 oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs import this module.  It loads ``oracle/_build/libgdoracle.so``
(built by ``oracle/Makefile``), a C++ restatement of GeoDynamo.jl's per-step
hot path; see the header of ``gd_oracle.cpp`` for the conventions and the
reference lines each routine follows.

Arrays use the reference's layouts: spectral planes are ``(nr, nlm)`` with the
l-major (l, m) index fastest (``src/fields.jl:6-15``); physical grids are
``(nr, nlon, nlat)`` with theta fastest (``src/fields.jl:18-24``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgdoracle.so")

FIELD_IDS = {"u_tor": 0, "u_pol": 1, "b_tor": 2, "b_pol": 3, "temp": 4, "comp": 5}
GRID_IDS = {
    "u_th": 0, "u_ph": 1, "w_th": 2, "w_ph": 3, "b_th": 4, "b_ph": 5, "j_th": 6, "j_ph": 7,
    "t": 8, "gth": 9, "gph": 10, "gr": 11, "tadv": 12, "vadv_th": 13, "vadv_ph": 14,
    "ind_th": 15, "ind_ph": 16,
    "c": 17, "cgth": 18, "cgph": 19, "cgr": 20, "cadv": 21,
}


class OcConfig(ctypes.Structure):
    _fields_ = [
        ("lmax", ctypes.c_int), ("mmax", ctypes.c_int), ("nlat", ctypes.c_int),
        ("nlon", ctypes.c_int), ("nr", ctypes.c_int), ("kl", ctypes.c_int),
        ("rratio", ctypes.c_double), ("ekman", ctypes.c_double), ("rayleigh", ctypes.c_double),
        ("prandtl", ctypes.c_double), ("magnetic_prandtl", ctypes.c_double),
        ("dt", ctypes.c_double), ("implicit_theta", ctypes.c_double),
        ("ab_mode", ctypes.c_int), ("bc_mode", ctypes.c_int), ("fd_mode", ctypes.c_int),
        ("precision", ctypes.c_int), ("magnetic", ctypes.c_int),
        ("composition", ctypes.c_int), ("schmidt", ctypes.c_double),
        ("segments", ctypes.c_int), ("geometry", ctypes.c_int), ("r_outer", ctypes.c_double),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        lib.oc_create.restype = P
        lib.oc_create.argtypes = [ctypes.POINTER(OcConfig)]
        lib.oc_destroy.argtypes = [P]
        lib.oc_set_threads.argtypes = [P, ctypes.c_int]
        lib.oc_nlm.argtypes = [P]
        lib.oc_nlm.restype = ctypes.c_int
        lib.oc_grid.argtypes = [P, D, D, D, D]
        lib.oc_tables.argtypes = [P, D, D]
        lib.oc_fd_matrix.argtypes = [P, ctypes.c_int, D]
        lib.oc_lu.argtypes = [P, ctypes.c_int, ctypes.c_int, D, D]
        lib.oc_band_solve.argtypes = [P, ctypes.c_int, ctypes.c_int, D]
        lib.oc_synth_scalar.argtypes = [P, D, D, D]
        lib.oc_regularity.argtypes = [P, D, D]
        lib.oc_analysis_scalar.argtypes = [P, D, D, D]
        lib.oc_synth_vector.argtypes = [P, D, D, D, D, D, D]
        lib.oc_analysis_vector.argtypes = [P, D, D, D, D, D, D]
        lib.oc_gradients.argtypes = [P, D, D, D]
        lib.oc_curl.argtypes = [P, D, D, D, D, D]
        lib.oc_set_field.argtypes = [P, ctypes.c_int, D, D]
        lib.oc_get_field.argtypes = [P, ctypes.c_int, D, D]
        lib.oc_get_nl.argtypes = [P, ctypes.c_int, D, D]
        lib.oc_get_grid_field.argtypes = [P, ctypes.c_int, D]
        lib.oc_get_grid_field.restype = ctypes.c_int
        lib.oc_set_temperature_bc.argtypes = [P, D, D]
        lib.oc_set_composition_bc.argtypes = [P, D, D]
        lib.oc_set_bc_types.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        for name in ("oc_temperature_nl", "oc_velocity_nl", "oc_magnetic_nl", "oc_implicit_step", "oc_composition_nl"):
            getattr(lib, name).argtypes = [P]
        lib.oc_step.argtypes = [P, ctypes.c_int]
        lib.oc_energy.argtypes = [P, D, D]
        lib.oc_step_count.argtypes = [P]
        lib.oc_step_count.restype = ctypes.c_long
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def lm_pairs(lmax: int, mmax: int):
    """(l, m) per l-major index (``shtnskit_transforms.jl:177-188``)."""
    return [(l, m) for l in range(lmax + 1) for m in range(min(l, mmax) + 1)]


# -- the exponential schemes' per-system updates (test restatements) -------------
def eab2_update(E, phi1, u, n, n_prev, dt):
    """eab2_update! (src/timestep.jl:429-487) for one system: u (nr, k) columns,
    n and n_prev their nonlinear terms: E u + dt phi1 (3/2 N - 1/2 N_prev)."""
    return E @ u + dt * (phi1 @ (1.5 * n - 0.5 * n_prev))


def erk2_prepare(E, phi1, E_half, phi1_half, u, n, dt):
    """erk2_prepare_field! (src/timestep.jl:1316-1431) for one system:
    (linear, k1, stage) = (E u, phi1 N, E_h u + dt/2 phi1_h N)."""
    return E @ u, phi1 @ n, E_half @ u + 0.5 * dt * (phi1_half @ n)


def erk2_finalize(phi2, linear, k1, n, n_stage, dt):
    """erk2_finalize_field! (src/timestep.jl:1449-1557) for one system:
    linear + dt (k1 + phi2 (N_stage - N))."""
    return linear + dt * (k1 + phi2 @ (n_stage - n))


class Oracle:
    """One oracle instance: grid, tables, radial operators and a model state."""

    def __init__(self, lmax, nlat, nlon, nr, mmax=None, kl=4, rratio=0.35, ekman=3e-4,
                 rayleigh=80.0, prandtl=1.0, magnetic_prandtl=4.0, dt=1e-5, implicit_theta=0.5,
                 ab_mode=0, bc_mode=0, fd_mode=0, magnetic=1, threads=None, composition=0, schmidt=1.0,
                 geometry="shell", r_outer=1.0):
        self.lib = _load()
        mmax = lmax if mmax is None else mmax
        self.cfg = OcConfig(lmax, mmax, nlat, nlon, nr, kl, rratio, ekman, rayleigh, prandtl,
                            magnetic_prandtl, dt, implicit_theta, ab_mode, bc_mode, fd_mode, 0,
                            magnetic, int(composition), float(schmidt), 0,
                            {"shell": 0, "ball": 1}[geometry], float(r_outer))
        self.h = self.lib.oc_create(ctypes.byref(self.cfg))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        if threads is not None:
            self.lib.oc_set_threads(self.h, int(threads))
        self.lmax, self.mmax, self.nlat, self.nlon, self.nr = lmax, mmax, nlat, nlon, nr
        self.nlm = self.lib.oc_nlm(self.h)
        self.kl = kl

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.oc_destroy(h)
            self.h = None

    # -- geometry -----------------------------------------------------------------
    def grid(self):
        x = np.zeros(self.nlat); w = np.zeros(self.nlat); th = np.zeros(self.nlat)
        r = np.zeros(self.nr)
        self.lib.oc_grid(self.h, _ptr(x), _ptr(w), _ptr(th), _ptr(r))
        return x, w, th, r

    def tables(self):
        nth = self.nlat // 2
        P = np.zeros((self.nlm, nth)); dP = np.zeros((self.nlm, nth))
        self.lib.oc_tables(self.h, _ptr(P), _ptr(dP))
        return P, dP

    def fd_matrix(self, which):
        out = np.zeros((self.nr, 2 * self.kl + 1))  # column-major (2kl+1) x nr
        self.lib.oc_fd_matrix(self.h, which, _ptr(out))
        return out.T.copy()  # rows = band row, cols = column j

    def implicit_matrices(self, kind, l):
        lin = np.zeros((self.nr, 2 * self.kl + 1)); lu = np.zeros((self.nr, 2 * self.kl + 1))
        self.lib.oc_lu(self.h, kind, l, _ptr(lin), _ptr(lu))
        return lin.T.copy(), lu.T.copy()

    def band_solve(self, kind, l, b):
        x = _c(b).copy()
        self.lib.oc_band_solve(self.h, kind, l, _ptr(x))
        return x

    # -- transforms ---------------------------------------------------------------
    def spec_shape(self):
        return (self.nr, self.nlm)

    def grid_shape(self):
        return (self.nr, self.nlon, self.nlat)

    def synth_scalar(self, re, im):
        g = np.zeros(self.grid_shape())
        self.lib.oc_synth_scalar(self.h, _ptr(_c(re)), _ptr(_c(im)), _ptr(g))
        return g

    def analysis_scalar(self, grid, ball=False):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self.lib.oc_analysis_scalar(self.h, _ptr(_c(grid)), _ptr(re), _ptr(im))
        if ball:  # ball_physical_to_spectral! (Ball/Ball.jl:214-220)
            self.lib.oc_regularity(self.h, _ptr(re), _ptr(im))
        return re, im

    def synth_vector(self, tre, tim, pre, pim):
        vt = np.zeros(self.grid_shape()); vp = np.zeros(self.grid_shape())
        self.lib.oc_synth_vector(self.h, _ptr(_c(tre)), _ptr(_c(tim)), _ptr(_c(pre)), _ptr(_c(pim)),
                                 _ptr(vt), _ptr(vp))
        return vt, vp

    def analysis_vector(self, vt, vp, ball=False):
        out = [np.zeros(self.spec_shape()) for _ in range(4)]
        self.lib.oc_analysis_vector(self.h, _ptr(_c(vt)), _ptr(_c(vp)), *[_ptr(o) for o in out])
        if ball:  # ball_vector_analysis! (Ball/Ball.jl:236-245)
            self.lib.oc_regularity(self.h, _ptr(out[0]), _ptr(out[1]))
            self.lib.oc_regularity(self.h, _ptr(out[2]), _ptr(out[3]))
        return out  # tor re, tor im, pol re, pol im

    def gradients(self, re, im):
        out = np.zeros((6,) + self.spec_shape())
        self.lib.oc_gradients(self.h, _ptr(_c(re)), _ptr(_c(im)), _ptr(out))
        return out

    def curl(self, tre, tim, pre, pim):
        out = np.zeros((4,) + self.spec_shape())
        self.lib.oc_curl(self.h, _ptr(_c(tre)), _ptr(_c(tim)), _ptr(_c(pre)), _ptr(_c(pim)), _ptr(out))
        return out

    # -- state --------------------------------------------------------------------
    def set_field(self, name, re, im):
        self.lib.oc_set_field(self.h, FIELD_IDS[name], _ptr(_c(re)), _ptr(_c(im)))

    def get_field(self, name):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self.lib.oc_get_field(self.h, FIELD_IDS[name], _ptr(re), _ptr(im))
        return re, im

    def get_nl(self, name):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self.lib.oc_get_nl(self.h, FIELD_IDS[name], _ptr(re), _ptr(im))
        return re, im

    def get_grid(self, name):
        g = np.zeros(self.grid_shape())
        if self.lib.oc_get_grid_field(self.h, GRID_IDS[name], _ptr(g)) != 0:
            raise KeyError(name)
        return g

    def set_temperature_bc(self, bvals=None, sources=None):
        self.lib.oc_set_temperature_bc(
            self.h, _ptr(_c(bvals)) if bvals is not None else None,
            _ptr(_c(sources)) if sources is not None else None)

    def set_composition_bc(self, bvals=None, sources=None):
        self.lib.oc_set_composition_bc(
            self.h, _ptr(_c(bvals)) if bvals is not None else None,
            _ptr(_c(sources)) if sources is not None else None)

    def set_bc_types(self, name, inner, outer):
        """bc_type_inner / bc_type_outer (1 fixed value, 2 flux) of "temp" or "comp", l-major."""
        a = np.ascontiguousarray(inner, dtype=np.int32)
        b = np.ascontiguousarray(outer, dtype=np.int32)
        IP = ctypes.POINTER(ctypes.c_int)
        self.lib.oc_set_bc_types(self.h, FIELD_IDS[name], a.ctypes.data_as(IP), b.ctypes.data_as(IP))

    def composition_nl(self):
        self.lib.oc_composition_nl(self.h)

    def temperature_nl(self):
        self.lib.oc_temperature_nl(self.h)

    def velocity_nl(self):
        self.lib.oc_velocity_nl(self.h)

    def magnetic_nl(self):
        self.lib.oc_magnetic_nl(self.h)

    def implicit_step(self):
        self.lib.oc_implicit_step(self.h)

    def step(self, n=1):
        self.lib.oc_step(self.h, int(n))

    def energy(self):
        ek = ctypes.c_double(); em = ctypes.c_double()
        self.lib.oc_energy(self.h, ctypes.byref(ek), ctypes.byref(em))
        return ek.value, em.value

    def step_count(self):
        return self.lib.oc_step_count(self.h)

    # -- ts_scheme = :eab2 / :erk2 (test restatement) ----------------------------
    def etd_cache(self, kind):
        """create_etd_cache / create_erk2_cache (src/timestep.jl:37-70, 896-968)
        for a field kind (0 velocity, 1 magnetic, 2 temperature, 3 composition) at the
        configuration's dt: per degree l the dense operator A_l (the L_l band of
        the implicit matrices, src/timestep.jl:498-543) and the matrices E, phi1,
        phi2 of dt A_l and E, phi1 of dt A_l / 2.  exp is scipy.linalg.expm
        (scaling and squaring with Pade approximants, Al-Mohy and Higham 2009;
        Julia's matrix exp follows Higham 2005); phi1 and phi2 are the blocks of
        exp([[X, I, 0], [0, 0, I], [0, 0, 0]]) (the same functions the reference
        forms with A^-1, compute_phi1_function / compute_phi2_function; those
        solves are unusable here: A_l has no boundary rows and the radial
        equation's two homogeneous solutions leave it numerically singular).
        Returns {"A", "E", "phi1", "phi2", "E_half", "phi1_half"}, lists by l."""
        from scipy.linalg import expm
        n, kl, dt = self.nr, self.kl, self.cfg.dt
        out = {k: [] for k in ("A", "E", "phi1", "phi2", "E_half", "phi1_half")}
        for l in range(self.lmax + 1):
            lin, _ = self.implicit_matrices(kind, l)   # band rows kl + i - c, columns c
            a = np.zeros((n, n))
            for c in range(n):
                for b in range(2 * kl + 1):
                    i = c + b - kl
                    if 0 <= i < n:
                        a[i, c] = lin[b, c]
            out["A"].append(a)
            for h, suffix in ((dt, ""), (0.5 * dt, "_half")):
                big = np.zeros((3 * n, 3 * n))
                big[:n, :n] = h * a
                big[:n, n:2 * n] = np.eye(n)
                big[n:2 * n, 2 * n:] = np.eye(n)
                ex = expm(big)
                out["E" + suffix].append(ex[:n, :n].copy())
                out["phi1" + suffix].append(ex[:n, n:2 * n].copy())
                if not suffix:
                    out["phi2"].append(ex[:n, 2 * n:].copy())
        return out

    def _per_l(self, fn, *xs):
        """fn(l, *column blocks of xs) applied per degree l; returns the
        reassembled arrays (one, or a tuple)."""
        lv = np.array([p[0] for p in lm_pairs(self.lmax, self.mmax)])
        outs = None
        for l in range(self.lmax + 1):
            cols = lv == l
            r = fn(l, *[x[:, cols] for x in xs])
            r = r if isinstance(r, tuple) else (r,)
            if outs is None:
                outs = [np.empty((xs[0].shape[0], xs[0].shape[1])) for _ in r]
            for o, v in zip(outs, r):
                o[:, cols] = v
        return outs[0] if len(outs) == 1 else tuple(outs)

    FIELD_KINDS = (("u_tor", 0), ("u_pol", 0), ("b_tor", 1), ("b_pol", 1), ("temp", 2))

    def field_kinds(self):
        """The implicit fields and their diffusivity kinds (composition when configured)."""
        return self.FIELD_KINDS + ((("comp", 3),) if self.cfg.composition else ())

    def eab2_step(self, caches, history):
        """One step of step_once! under ts_scheme = :eab2: the three nonlinear
        phases, then for every field u <- E_l u + dt phi1_l (3/2 N - 1/2 N_prev)
        per (l, m) column (eab2_update!, src/timestep.jl:429-487) and the roll
        N_prev := N (src/simulation.jl:1311-1329).  caches[kind] = etd_cache(kind);
        history maps a field name to its (re, im) N_prev (missing: zeros, as
        prev_nonlinear starts) and is updated in place."""
        dt = self.cfg.dt
        self.temperature_nl()
        self.velocity_nl()
        self.magnetic_nl()
        if self.cfg.composition:
            self.composition_nl()
        for name, kind in self.field_kinds():
            c = caches[kind]
            re, im = self.get_field(name)
            nre, nim = self.get_nl(name)
            pre, pim = history.get(name, (np.zeros_like(re), np.zeros_like(im)))
            out = [self._per_l(lambda l, u_, n_, p_: eab2_update(c["E"][l], c["phi1"][l], u_, n_, p_, dt), u, nn, pp)
                   for u, nn, pp in ((re, nre, pre), (im, nim, pim))]
            self.set_field(name, *out)
            history[name] = (nre, nim)

    def _all_nonlinear(self):
        # compute_all_nonlinear_terms! (src/simulation.jl:800-813): velocity,
        # magnetic, temperature, composition
        self.velocity_nl()
        self.magnetic_nl()
        self.temperature_nl()
        if self.cfg.composition:
            self.composition_nl()

    def erk2_step(self, caches):
        """One step of step_once! under ts_scheme = :erk2: the three nonlinear
        phases, then erk2_integrate_full_step! (src/simulation.jl:1054-1149):
        erk2_prepare_field! (linear = E u, k1 = phi1 N, stage = E_h u + dt/2
        phi1_h N), the stage applied, compute_all_nonlinear_terms!,
        erk2_finalize_field! (u = linear + dt (k1 + phi2 (N_stage - N))) and a
        last compute_all_nonlinear_terms! at the new state
        (src/timestep.jl:1316-1557)."""
        dt = self.cfg.dt
        self.temperature_nl()
        self.velocity_nl()
        self.magnetic_nl()
        if self.cfg.composition:
            self.composition_nl()
        saved = {}
        for name, kind in self.field_kinds():
            c = caches[kind]
            u = self.get_field(name)
            nn = self.get_nl(name)
            prep = [self._per_l(lambda l, u_, n_: erk2_prepare(c["E"][l], c["phi1"][l], c["E_half"][l],
                                                               c["phi1_half"][l], u_, n_, dt), x, y)
                    for x, y in zip(u, nn)]
            saved[name] = ([p[0] for p in prep], [p[1] for p in prep], nn)
            self.set_field(name, *[p[2] for p in prep])
        self._all_nonlinear()
        for name, kind in self.field_kinds():
            c = caches[kind]
            lin, k1, nn = saved[name]
            ns = self.get_nl(name)
            out = [self._per_l(lambda l, li_, ki_, n_, s_: erk2_finalize(c["phi2"][l], li_, ki_, n_, s_, dt),
                               li, ki, n_, s_)
                   for li, ki, n_, s_ in zip(lin, k1, nn, ns)]
            self.set_field(name, *out)
        self._all_nonlinear()


# ---------------------------------------------------------------------------
# The reference's Krylov actions of the EAB2 path (eab2_update_krylov_cached!,
# src/timestep.jl:358-427), restated in numpy for the tests that compare them
# with the dense exponential operators.
# ---------------------------------------------------------------------------
def band_to_dense(band, kl):
    """(2kl+1, n) band (row kl + i - j, column j) -> dense n x n."""
    n = band.shape[1]
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - kl), min(n, i + kl + 1)):
            D[i, j] = band[kl + i - j, j]
    return D


def exp_action_krylov(A, v, dt, m=20, tol=1e-8):
    """exp_action_krylov (src/timestep.jl:108-225): Arnoldi with the residual
    stopping rule |H[j+1, j] y_j[end]| <= tol |y_j| and the condition-number
    guard; returns (y, Krylov dimension used)."""
    import scipy.linalg as sla
    n = len(v)
    beta = float(np.linalg.norm(v))
    if n == 0 or beta == 0.0:
        return np.zeros(n), 0
    V = np.zeros((n, m))
    H = np.zeros((m, m))
    V[:, 0] = v / beta
    kmax = m
    for j in range(m):
        w = A @ V[:, j]
        for i in range(j + 1):
            H[i, j] = V[:, i] @ w
            w = w - H[i, j] * V[:, i]
        if j < m - 1:
            H[j + 1, j] = np.linalg.norm(w)
            if H[j + 1, j] < np.finfo(float).eps * 100:
                kmax = j + 1
                break
            V[:, j + 1] = w / H[j + 1, j]
            Hj = dt * H[:j + 1, :j + 1]
            if j > 0 and np.linalg.cond(Hj) > 1e12:
                kmax = j + 1
                break
            e1 = np.zeros(j + 1)
            e1[0] = 1.0
            y = sla.expm(Hj) @ (beta * e1)
            if abs(H[j + 1, j]) * abs(y[-1]) <= tol * np.linalg.norm(y):
                kmax = j + 1
                break
    e1 = np.zeros(kmax)
    e1[0] = 1.0
    return V[:, :kmax] @ (sla.expm(dt * H[:kmax, :kmax]) @ (beta * e1)), kmax


def phi1_action_krylov(A, v, dt, m=20, tol=1e-8):
    """phi1_action_krylov (src/timestep.jl:227-268): A^-1 (exp(dt A) v - v) / dt
    with the non-pivoting banded LU of A (factorize_banded)."""
    ev, _ = exp_action_krylov(A, v, dt, m, tol)
    c = ev - v
    n = len(v)
    U = A.astype(float).copy()
    Lf = np.eye(n)
    for k in range(n - 1):
        for i in range(k + 1, n):
            Lf[i, k] = U[i, k] / U[k, k]
            U[i, :] -= Lf[i, k] * U[k, :]
    return np.linalg.solve(U, np.linalg.solve(Lf, c)) / dt

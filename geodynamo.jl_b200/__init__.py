"""Host-side mirror of GeoDynamo.jl's transform / nonlinear / timestep API over
libgdb200.so (the sm_100a kernels of this package, reached through the C ABI in
``include/gdb200.h``).

The functions keep the reference's names, argument meaning and in-place
behaviour (Julia's ``!`` suffix dropped):

=====================================  ==============================================
reference (src/...)                    here
=====================================  ==============================================
create_shtnskit_config (shtnskit_transforms.jl:102)   :func:`create_shtnskit_config`
shtnskit_spectral_to_physical! (shtnskit_field_functions.jl:11)  :func:`shtnskit_spectral_to_physical`
shtnskit_physical_to_spectral! (:131)  :func:`shtnskit_physical_to_spectral`
shtnskit_vector_synthesis! (:252)      :func:`shtnskit_vector_synthesis`
shtnskit_vector_analysis! (:291)       :func:`shtnskit_vector_analysis`
batch_spectral_to_physical! (:674)     :func:`batch_spectral_to_physical`
compute_temperature_nonlinear! (thermal.jl:149)  :func:`compute_temperature_nonlinear`
compute_velocity_nonlinear! (velocity.jl:312)    :func:`compute_velocity_nonlinear`
compute_magnetic_nonlinear! (magnetic.jl:131)    :func:`compute_magnetic_nonlinear`
apply_master_implicit_step! (simulation.jl:1151) :func:`apply_master_implicit_step`
step_once! (scripts/bench_timestepping.jl:6)     :func:`step_once`
compute_kinetic_energy / compute_magnetic_energy :func:`compute_kinetic_energy`, ...
=====================================  ==============================================

Errors raise :class:`GeoDynamoError` (the reference raises Julia exceptions).
There is no CPU fallback: if ``libgdb200.so`` is missing or no CUDA device is
present, every call that needs the device raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgdb200.so")
_CSRC = os.path.join(_HERE, "csrc")

GD_OK = 0
STATUS_NAMES = {0: "GD_OK", 1: "GD_ERR_ARG", 2: "GD_ERR_CONFIG", 3: "GD_ERR_CUDA", 4: "GD_ERR_NONFINITE",
                5: "GD_ERR_SINGULAR", 6: "GD_ERR_UNSUPPORTED", 7: "GD_ERR_STATE"}
FIELDS = {"u_tor": 0, "u_pol": 1, "b_tor": 2, "b_pol": 3, "temp": 4, "comp": 5}
BC_VALUE, BC_FLUX = 1, 2  # GD_BC_VALUE / GD_BC_FLUX (bc_type_inner / bc_type_outer)
GRIDS = {
    "u_th": 0, "u_ph": 1, "w_th": 2, "w_ph": 3, "b_th": 4, "b_ph": 5, "j_th": 6, "j_ph": 7,
    "t": 8, "gth": 9, "gph": 10, "gr": 11, "tadv": 12, "vadv_th": 13, "vadv_ph": 14,
    "ind_th": 15, "ind_ph": 16,
    "c": 17, "cgth": 18, "cgph": 19, "cgr": 20, "cadv": 21,
}
PRECISIONS = {"fp64": 0, "mixed": 1}
# Stages of the mixed-precision step that can run in FP64 (GD_STAGE_*): the
# chain the velocity, and so the kinetic energy, depends on.
# "vel_synth_i8": the vector synthesis of u on the tensor cores by int8 digit
# slices (FP64-accurate; replaces the DMMA synthesis of "vel_synth").
FP64_STAGES = {"vel_synth": 1, "vel_products": 2, "vel_analysis": 4, "vel_synth_i8": 8}
# Named precision settings: the mixed step with its velocity chain in FP64
# ("mixed_vel64"), or with the chain's synthesis by int8 slices ("mixed_vel64i8").
PRECISION_PRESETS = {"mixed_vel64": ("mixed", ("vel_synth", "vel_products", "vel_analysis")),
                     "mixed_vel64i8": ("mixed", ("vel_synth_i8", "vel_products", "vel_analysis"))}
SCHEMES = {"cnab2": 0, "eab2": 1, "erk2": 2}
GEOMETRIES = {"shell": 0, "ball": 1}   # geometry (src/parameters.jl:75)   # ts_scheme (src/simulation.jl:1054-1300)
ETD_MATRICES = ("E", "phi1", "phi2", "E_half", "phi1_half")   # ERK2Cache fields (src/timestep.jl:830-853)
KINDS = {"velocity": 0, "magnetic": 1, "temperature": 2, "composition": 3}

# Every symbol include/gdb200.h declares.
EXPORTS = (
    "gd_create", "gd_destroy", "gd_last_error", "gd_info", "gd_grid", "gd_set_precision", "gd_set_fp64_stages",
    "gd_set_int8_digits",
    "gd_synchronize",
    "gd_upload_spectral", "gd_download_spectral", "gd_download_nonlinear", "gd_download_grid",
    "gd_set_temperature_bc", "gd_spectral_to_physical", "gd_physical_to_spectral", "gd_vector_synthesis",
    "gd_vector_analysis", "gd_ball_physical_to_spectral", "gd_ball_vector_analysis", "gd_enforce_regularity",
    "gd_temperature_nonlinear", "gd_velocity_nonlinear", "gd_magnetic_nonlinear",
    "gd_implicit_step", "gd_step", "gd_step_async", "gd_set_dt", "gd_set_scheme", "gd_download_etd",
    "gd_energy", "gd_segment_energy", "gd_set_segment_ekman", "gd_check_finite",
    "gd_step_count", "gd_get_stream", "gd_profile_enable", "gd_profile_read",
    "gd_spectral_to_physical_noalloc",
    "gd_compute_temperature_nonlinear", "gd_compute_velocity_nonlinear", "gd_compute_magnetic_nonlinear",
    "gd_compute_composition_nonlinear",
    "gd_create_timestepping_matrices", "gd_destroy_timestepping_matrices", "gd_build_rhs_cnab2",
    "gd_solve_implicit_step", "gd_set_fault_test",
    "gd_derivatives", "gd_implicit_modes", "gd_set_external_derivatives", "gd_copy_block",
    "gd_set_launch_shape", "gd_get_launch_shape", "gd_ensemble_autotune", "gd_step_kernels",
    "gd_snapshot_bytes", "gd_snapshot", "gd_spectral_device", "gd_grid_device", "gd_temperature_nl_adjoint",
    "gd_cnab2_adjoint", "gd_temperature_forward", "gd_temperature_pullback", "gd_velocity_nl_adjoint",
    "gd_velocity_pullback", "gd_temperature_pullback_full", "gd_temperature_u_adjoint",
    "gd_set_composition_bc", "gd_set_scalar_bc_types", "gd_composition_nonlinear",
    "gd_spectral_to_physical_adjoint", "gd_magnetic_pullback",
    "gd_ensemble_create", "gd_ensemble_destroy", "gd_ensemble_size", "gd_ensemble_member",
    "gd_ensemble_step", "gd_ensemble_step_async", "gd_ensemble_failed_member", "gd_ensemble_get_stream",
)


class GeoDynamoError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GDConfig(ctypes.Structure):
    """``gd_config`` of include/gdb200.h (GeoDynamoParameters subset)."""
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
        ("segment_nr", ctypes.POINTER(ctypes.c_int)),
    ]


def build(verbose: bool = False) -> str:
    """Compile libgdb200.so for sm_100a in-tree (nvcc cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-C", _CSRC, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libgdb200 build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if verbose:
        print(out.stdout[-2000:])
    return _LIB_PATH


_lib = None


def library_path() -> str:
    return _LIB_PATH


def load_library():
    """Load libgdb200.so and declare its signatures; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise GeoDynamoError(6, f"{_LIB_PATH} is missing; run geodynamo build() first")
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.c_int
    sigs = {
        "gd_create": ([ctypes.POINTER(GDConfig), I, ctypes.POINTER(P)], I),
        "gd_destroy": ([P], I),
        "gd_last_error": ([P], ctypes.c_char_p),
        "gd_info": ([P, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_size_t)], I),
        "gd_grid": ([P, D, D, D], I),
        "gd_set_precision": ([P, I], I),
        "gd_set_fp64_stages": ([P, I], I),
        "gd_set_int8_digits": ([P, I], I),
        "gd_synchronize": ([P], I),
        "gd_upload_spectral": ([P, I, D, D], I),
        "gd_download_spectral": ([P, I, D, D], I),
        "gd_download_nonlinear": ([P, I, D, D], I),
        "gd_download_grid": ([P, I, D], I),
        "gd_set_temperature_bc": ([P, D, D], I),
        "gd_spectral_to_physical": ([P, I, D, D, D], I),
        "gd_physical_to_spectral": ([P, I, D, D, D], I),
        "gd_vector_synthesis": ([P, D, D, D, D, D, D], I),
        "gd_vector_analysis": ([P, D, D, D, D, D, D], I),
        "gd_ball_physical_to_spectral": ([P, I, D, D, D], I),
        "gd_ball_vector_analysis": ([P, D, D, D, D, D, D], I),
        "gd_enforce_regularity": ([P, I], I),
        "gd_temperature_nonlinear": ([P], I),
        "gd_velocity_nonlinear": ([P], I),
        "gd_magnetic_nonlinear": ([P], I),
        "gd_implicit_step": ([P], I),
        "gd_step": ([P, I], I),
        "gd_step_async": ([P, I], I),
        "gd_set_dt": ([P, ctypes.c_double], I),
        "gd_set_scheme": ([P, I], I),
        "gd_download_etd": ([P, I, I, I, D], I),
        "gd_energy": ([P, D, D], I),
        "gd_segment_energy": ([P, D, D], I),
        "gd_set_segment_ekman": ([P, D], I),
        "gd_check_finite": ([P], I),
        "gd_step_count": ([P], ctypes.c_long),
        "gd_get_stream": ([P, ctypes.POINTER(P)], I),
        "gd_profile_enable": ([P, I], I),
        "gd_profile_read": ([P, I, ctypes.c_char_p, D, ctypes.POINTER(I), ctypes.POINTER(I)], I),
        "gd_spectral_to_physical_noalloc": ([P, I, ctypes.c_void_p, ctypes.c_void_p], I),
        "gd_spectral_to_physical_adjoint": ([P, I, D, D, D], I),
        "gd_compute_temperature_nonlinear": ([P, D, D, D, D, D, D, D], I),
        "gd_compute_composition_nonlinear": ([P, D, D, D, D, D, D, D], I),
        "gd_compute_velocity_nonlinear": ([P] + [D] * 14, I),
        "gd_compute_magnetic_nonlinear": ([P] + [D] * 14, I),
        "gd_create_timestepping_matrices": ([P, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.POINTER(P)], I),
        "gd_destroy_timestepping_matrices": ([P], I),
        "gd_build_rhs_cnab2": ([P, P, ctypes.c_double] + [D] * 8, I),
        "gd_solve_implicit_step": ([P, P, D, D, D, D], I),
        "gd_set_fault_test": ([P, ctypes.c_longlong, I], I),
        "gd_derivatives": ([P, I, I], I),
        "gd_implicit_modes": ([P, I, I], I),
        "gd_set_external_derivatives": ([P, I], I),
        "gd_set_launch_shape": ([P, I], I),
        "gd_set_composition_bc": ([P, D, D], I),
        "gd_set_scalar_bc_types": ([P, I, ctypes.POINTER(I), ctypes.POINTER(I)], I),
        "gd_composition_nonlinear": ([P], I),
        "gd_get_launch_shape": ([P, ctypes.POINTER(I)], I),
        "gd_step_kernels": ([P, ctypes.POINTER(I)], I),
        "gd_snapshot_bytes": ([P, ctypes.POINTER(ctypes.c_size_t)], I),
        "gd_snapshot": ([P, P, I], I),
        "gd_spectral_device": ([P, D, D, P, I], I),
        "gd_grid_device": ([P, I, P], I),
        "gd_temperature_nl_adjoint": ([P, P, P, P, P], I),
        "gd_cnab2_adjoint": ([P, I, I, P, P], I),
        "gd_velocity_nl_adjoint": ([P, P, P], I),
        "gd_velocity_pullback": ([P, I] + [D] * 8, I),
        "gd_temperature_pullback_full": ([P] + [D] * 8, I),
        "gd_temperature_u_adjoint": ([P, P, P, P, P], I),
        "gd_temperature_forward": ([P, I, I], I),
        "gd_temperature_pullback": ([P, D, D, D, D], I),
        "gd_ensemble_autotune": ([P, I, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(I)], I),
        "gd_copy_block": ([P, I, I, I, I, I, I, ctypes.c_void_p, I], I),
        "gd_magnetic_pullback": ([P, I, I, D, D, D, D], I),
        "gd_ensemble_create": ([ctypes.POINTER(GDConfig), I, I, ctypes.POINTER(P)], I),
        "gd_ensemble_destroy": ([P], I),
        "gd_ensemble_size": ([P], I),
        "gd_ensemble_member": ([P, I], P),
        "gd_ensemble_step": ([P, I], I),
        "gd_ensemble_step_async": ([P, I], I),
        "gd_ensemble_failed_member": ([P], I),
        "gd_ensemble_get_stream": ([P, ctypes.POINTER(P)], I),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise GeoDynamoError(1, "arrays must be C-contiguous float64")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def lm_pairs(lmax: int, mmax: int):
    """(l, m) per l-major index (``shtnskit_transforms.jl:177-188``)."""
    return [(l, m) for l in range(lmax + 1) for m in range(min(l, mmax) + 1)]


def index_to_lm_shtnskit(idx: int, lmax: int, mmax: int):
    """1-based index -> (l, m) (``shtnskit_field_functions.jl:450-462``), in O(1)."""
    q = idx - 1
    if q < 0:
        return (0, 0)
    full = (mmax + 1) * (mmax + 2) // 2
    if q < full:
        l = int((np.sqrt(8 * q + 1) - 1) // 2)
        while (l + 1) * (l + 2) // 2 <= q:
            l += 1
        while l * (l + 1) // 2 > q:
            l -= 1
        return (l, q - l * (l + 1) // 2)
    rest = q - full
    l = mmax + 1 + rest // (mmax + 1)
    if l > lmax:
        return (0, 0)
    return (l, rest % (mmax + 1))


class SHTnsKitConfig:
    """Grid and handle of one transform / model configuration.

    Mirrors ``SHTnsKitConfig`` (``shtnskit_transforms.jl:61-93``): lmax, mmax,
    nlat, nlon, nlm, l_values, m_values, theta_grid, phi_grid, gauss_weights.
    The device handle also owns the model state used by the step functions.
    """

    def __init__(self, lmax, nlat, nlon, nr, mmax=None, kl=4, rratio=0.35, ekman=3e-4, rayleigh=80.0,
                 prandtl=1.0, magnetic_prandtl=4.0, dt=1e-5, implicit_theta=0.5, ab_mode=0, bc_mode=0,
                 fd_mode=0, precision="fp64", magnetic=1, device=0, composition=0, schmidt=1.0, segments=0,
                 geometry="shell", r_outer=1.0, segment_nr=None):
        self.lib = load_library()
        mmax = lmax if mmax is None else mmax
        base, stages = PRECISION_PRESETS.get(precision, (precision, ()))
        self.cfg = GDConfig(lmax, mmax, nlat, nlon, nr, kl, rratio, ekman, rayleigh, prandtl, magnetic_prandtl,
                            dt, implicit_theta, ab_mode, bc_mode, fd_mode, PRECISIONS[base], magnetic,
                            int(composition), float(schmidt), int(segments), GEOMETRIES[geometry], float(r_outer))
        if segment_nr is not None:
            self._segnr = (ctypes.c_int * len(segment_nr))(*[int(v) for v in segment_nr])
            self.cfg.segment_nr = ctypes.cast(self._segnr, ctypes.POINTER(ctypes.c_int))
        h = ctypes.c_void_p()
        st = self.lib.gd_create(ctypes.byref(self.cfg), int(device), ctypes.byref(h))
        if st != GD_OK:
            raise GeoDynamoError(st, "gd_create failed (see stderr)")
        self._owned = True
        self.device = int(device)
        self._attach(h, base)
        if stages:
            self.set_fp64_stages(stages)
            self.precision = precision

    @classmethod
    def _member(cls, lib, h, cfg: GDConfig):
        """A view of an ensemble member's handle (owned by the ensemble)."""
        self = cls.__new__(cls)
        self.lib = lib
        self.cfg = cfg
        self._owned = False
        self.device = 0
        self._attach(h, {v: k for k, v in PRECISIONS.items()}[cfg.precision])
        return self

    def _attach(self, h, precision):
        cfg = self.cfg
        lmax, mmax, nlat, nlon, nr = cfg.lmax, cfg.mmax, cfg.nlat, cfg.nlon, cfg.nr
        self.h = h
        self.lmax, self.mmax, self.nlat, self.nlon, self.nr = lmax, mmax, nlat, nlon, nr
        n = ctypes.c_int()
        b = ctypes.c_size_t()
        self._check(self.lib.gd_info(self.h, ctypes.byref(n), ctypes.byref(b)))
        self.nlm = n.value
        pairs = lm_pairs(lmax, mmax)
        self.l_values = np.array([p[0] for p in pairs])
        self.m_values = np.array([p[1] for p in pairs])
        th = np.zeros(nlat); w = np.zeros(nlat); r = np.zeros(nr)
        self._check(self.lib.gd_grid(self.h, _dptr(th), _dptr(w), _dptr(r)))
        self.theta_grid, self.gauss_weights, self.r = th, w, r
        self.phi_grid = 2 * np.pi * np.arange(nlon) / nlon
        self.precision = precision
        self.fp64_stages = 0
        self.scheme = "cnab2"

    # -- plumbing -------------------------------------------------------------
    def _check(self, st):
        if st != GD_OK:
            msg = self.lib.gd_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise GeoDynamoError(st, msg)

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.gd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self):
        n = ctypes.c_int(); b = ctypes.c_size_t()
        self._check(self.lib.gd_info(self.h, ctypes.byref(n), ctypes.byref(b)))
        return b.value

    def set_precision(self, precision):
        """"fp64", "mixed", or a preset of PRECISION_PRESETS ("mixed_vel64":
        the mixed step with its velocity chain in FP64)."""
        base, stages = PRECISION_PRESETS.get(precision, (precision, ()))
        self._check(self.lib.gd_set_precision(self.h, PRECISIONS[base]))
        self.set_fp64_stages(stages)
        self.precision = precision

    # -- the step decomposed across ranks (distributed.DistributedStep) ---------------
    def derivatives(self, j0, j1):
        """Radial derivatives of the state for native modes [j0, j1) into the work arrays."""
        self._check(self.lib.gd_derivatives(self.h, int(j0), int(j1)))

    def implicit_modes(self, j0, j1):
        """Temperature Dirichlet rows, CNAB2 and the history roll for native modes [j0, j1)."""
        self._check(self.lib.gd_implicit_modes(self.h, int(j0), int(j1)))

    def set_launch_shape(self, tc_ctas=0):
        """Cap of the tensor-core kernels' persistent grid (0: one CTA per SM)."""
        self._check(self.lib.gd_set_launch_shape(self.h, int(tc_ctas)))

    def segments(self):
        """Independent shells stacked along r in this handle (1: one shell)."""
        return max(1, int(self.cfg.segments))

    def set_segment_ekman(self, ekman):
        """Ekman number of each segment (the Coriolis and Lorentz factor Pm/E of its shells)."""
        e = _f64(np.asarray(ekman, dtype=np.float64).reshape(-1))
        if e.size != self.segments():
            raise ValueError(f"need {self.segments()} Ekman numbers")
        self._check(self.lib.gd_set_segment_ekman(self.h, _dptr(e)))

    def segment_energy(self):
        """(kinetic, magnetic) energy of each segment, arrays of segments values."""
        n = self.segments()
        ek = np.zeros(n); em = np.zeros(n)
        self._check(self.lib.gd_segment_energy(self.h, _dptr(ek), _dptr(em)))
        return ek, em

    def step_kernels(self):
        """Kernel launches of the next step (kernel nodes of its CUDA graph)."""
        n = ctypes.c_int()
        self._check(self.lib.gd_step_kernels(self.h, ctypes.byref(n)))
        return n.value

    def launch_shape(self):
        n = ctypes.c_int()
        self._check(self.lib.gd_get_launch_shape(self.h, ctypes.byref(n)))
        return n.value

    def set_external_derivatives(self, enable=True):
        self._check(self.lib.gd_set_external_derivatives(self.h, 1 if enable else 0))

    def copy_block(self, array, field, r0, r1, j0, j1, ptr, to_buf):
        """Block [r0, r1) x [j0, j1) of a state (0), work (1) or nonlinear (2)
        array to or from the buffer at ptr ([2][r1 - r0][j1 - j0] doubles)."""
        self._check(self.lib.gd_copy_block(self.h, int(array), int(field), int(r0), int(r1), int(j0), int(j1),
                                           ctypes.c_void_p(int(ptr)), 1 if to_buf else 0))

    def set_fault_test(self, wait_cycles=0, omit_step=-1):
        """Error-path testing (gd_set_fault_test): bound of every tensor-core
        wait in clock cycles (0: default) and a one-shot omission of the copies
        of one pipeline step in the next tensor-core synthesis."""
        self._check(self.lib.gd_set_fault_test(self.h, int(wait_cycles), int(omit_step)))

    def set_fp64_stages(self, stages):
        """Stages of the mixed step to run in FP64: names of FP64_STAGES or an int mask."""
        mask = stages if isinstance(stages, int) else sum(FP64_STAGES[n] for n in stages)
        self._check(self.lib.gd_set_fp64_stages(self.h, int(mask)))
        self.fp64_stages = mask

    def set_int8_digits(self, digits):
        """Digits of 7 bits per operand of the int8-slice synthesis (5 or 6)."""
        self._check(self.lib.gd_set_int8_digits(self.h, int(digits)))

    def spec_shape(self):
        return (self.nr, self.nlm)

    def grid_shape(self):
        return (self.nr, self.nlon, self.nlat)

    # -- raw transforms on numpy arrays in the reference layout ------------------
    def synth_scalar(self, re, im):
        re = _f64(re); im = _f64(im)
        nf = re.size // (self.nr * self.nlm)
        out = np.zeros((nf,) + self.grid_shape()) if re.ndim == 3 else np.zeros(self.grid_shape())
        self._check(self.lib.gd_spectral_to_physical(self.h, nf, _dptr(re), _dptr(im), _dptr(out)))
        return out

    def analysis_scalar(self, grid, ball=False):
        """shtnskit_physical_to_spectral!; ball=True: ball_physical_to_spectral!
        (the first radial level then 0 for l >= 1)."""
        grid = _f64(grid)
        nf = grid.size // (self.nr * self.nlat * self.nlon)
        shape = ((nf,) + self.spec_shape()) if grid.ndim == 4 else self.spec_shape()
        re = np.zeros(shape); im = np.zeros(shape)
        fn = self.lib.gd_ball_physical_to_spectral if ball else self.lib.gd_physical_to_spectral
        self._check(fn(self.h, nf, _dptr(grid), _dptr(re), _dptr(im)))
        return re, im

    def enforce_regularity(self, name):
        """enforce_ball_scalar_regularity! / enforce_ball_vector_regularity! on a state field."""
        self._check(self.lib.gd_enforce_regularity(self.h, FIELDS[name]))

    def synth_scalar_adjoint(self, grid):
        """Transpose of synth_scalar: grid cotangent -> (re, im) cotangents."""
        grid = _f64(grid)
        nf = grid.size // (self.nr * self.nlat * self.nlon)
        shape = ((nf,) + self.spec_shape()) if grid.ndim == 4 else self.spec_shape()
        re = np.zeros(shape); im = np.zeros(shape)
        self._check(self.lib.gd_spectral_to_physical_adjoint(self.h, nf, _dptr(grid), _dptr(re), _dptr(im)))
        return re, im

    # -- reverse mode of the temperature step (device tensors, native layouts) ----
    def snapshot_bytes(self):
        n = ctypes.c_size_t()
        self._check(self.lib.gd_snapshot_bytes(self.h, ctypes.byref(n)))
        return n.value

    def snapshot(self, buf):
        """Step state into a device buffer of snapshot_bytes() bytes (gd_snapshot)."""
        self._check(self.lib.gd_snapshot(self.h, ctypes.c_void_p(buf.data_ptr()), 0))

    def restore(self, buf):
        self._check(self.lib.gd_snapshot(self.h, ctypes.c_void_p(buf.data_ptr()), 1))

    def spectral_to_device(self, re, im, dev):
        """Reference-layout (re, im) -> native device array dev (2 nr nlm doubles)."""
        r, i = _f64(re).copy(), _f64(im).copy()
        self._check(self.lib.gd_spectral_device(self.h, _dptr(r), _dptr(i), ctypes.c_void_p(dev.data_ptr()), 1))

    def spectral_from_device(self, dev):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self._check(self.lib.gd_spectral_device(self.h, _dptr(re), _dptr(im), ctypes.c_void_p(dev.data_ptr()), 0))
        return re, im

    def grid_to_device(self, name, dev):
        self._check(self.lib.gd_grid_device(self.h, GRIDS[name], ctypes.c_void_p(dev.data_ptr())))

    def temperature_nl_adjoint(self, u_th, u_ph, nu, out):
        """out = N^T nu for the advection by the device grids u_th, u_ph."""
        v = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        self._check(self.lib.gd_temperature_nl_adjoint(self.h, v(u_th), v(u_ph), v(nu), v(out)))

    def cnab2_adjoint(self, name, mode, x, y):
        """mode 0: y = D S^-T C x; mode 1: y = P R^T x (gd_cnab2_adjoint)."""
        self._check(self.lib.gd_cnab2_adjoint(self.h, FIELDS[name], int(mode), ctypes.c_void_p(x.data_ptr()),
                                              ctypes.c_void_p(y.data_ptr())))

    def temperature_forward(self, nsteps, checkpoint_every=20):
        """nsteps steps with a device snapshot every checkpoint_every (gd_temperature_forward)."""
        self._check(self.lib.gd_temperature_forward(self.h, int(nsteps), int(checkpoint_every)))

    def temperature_pullback(self, lam_re, lam_im):
        """Cotangent of the temperature after the checkpointed run -> at its start."""
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self._check(self.lib.gd_temperature_pullback(self.h, _dptr(_f64(lam_re)), _dptr(_f64(lam_im)),
                                                     _dptr(re), _dptr(im)))
        return re, im

    def temperature_pullback_full(self, lam_re, lam_im):
        """Cotangent of the temperature after the checkpointed run -> (temperature
        (re, im), u_tor (re, im), u_pol (re, im)) at its start (gd_temperature_pullback_full)."""
        out = [np.zeros(self.spec_shape()) for _ in range(6)]
        self._check(self.lib.gd_temperature_pullback_full(self.h, _dptr(_f64(lam_re)), _dptr(_f64(lam_im)),
                                                          *[_dptr(o) for o in out]))
        return (out[0], out[1]), (out[2], out[3]), (out[4], out[5])

    def velocity_nl_adjoint(self, psi, out):
        """out = N^T psi for the velocity's (Coriolis) nonlinear term; psi, out:
        device tensors holding (tor, pol) in gd_snapshot's spectral layout."""
        self._check(self.lib.gd_velocity_nl_adjoint(self.h, ctypes.c_void_p(psi.data_ptr()),
                                                    ctypes.c_void_p(out.data_ptr())))

    def velocity_pullback(self, nsteps, lam_tor, lam_pol):
        """Pullback of the handle's last nsteps steps w.r.t. (u_tor, u_pol) at
        their start: the cotangents (re, im) of the velocity after them ->
        (tor (re, im), pol (re, im))."""
        out = [np.zeros(self.spec_shape()) for _ in range(4)]
        self._check(self.lib.gd_velocity_pullback(self.h, int(nsteps), _dptr(_f64(lam_tor[0])), _dptr(_f64(lam_tor[1])),
                                                  _dptr(_f64(lam_pol[0])), _dptr(_f64(lam_pol[1])),
                                                  *[_dptr(o) for o in out]))
        return (out[0], out[1]), (out[2], out[3])

    def magnetic_pullback(self, name, nsteps, lam_re, lam_im):
        """Pullback of nsteps steps w.r.t. the magnetic component ``name``
        ("b_tor" or "b_pol") at their start (gd_magnetic_pullback)."""
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self._check(self.lib.gd_magnetic_pullback(self.h, FIELDS[name], int(nsteps), _dptr(_f64(lam_re)),
                                                  _dptr(_f64(lam_im)), _dptr(re), _dptr(im)))
        return re, im

    def synth_vector(self, tre, tim, pre, pim):
        vt = np.zeros(self.grid_shape()); vp = np.zeros(self.grid_shape())
        self._check(self.lib.gd_vector_synthesis(self.h, _dptr(_f64(tre)), _dptr(_f64(tim)), _dptr(_f64(pre)),
                                                 _dptr(_f64(pim)), _dptr(vt), _dptr(vp)))
        return vt, vp

    def analysis_vector(self, vt, vp, ball=False):
        """shtnskit_vector_analysis!; ball=True: ball_vector_analysis!."""
        out = [np.zeros(self.spec_shape()) for _ in range(4)]
        fn = self.lib.gd_ball_vector_analysis if ball else self.lib.gd_vector_analysis
        self._check(fn(self.h, _dptr(_f64(vt)), _dptr(_f64(vp)), *[_dptr(o) for o in out]))
        return out

    # -- model state ------------------------------------------------------------
    # -- the reference's nonlinear functions on host arrays (FP64 kernels) ------------
    def compute_temperature_nonlinear_arrays(self, t_re, t_im, u_theta, u_phi):
        """compute_temperature_nonlinear! (src/thermal.jl:149-190): returns the
        temperature with its Dirichlet rows applied, the nonlinear term and the
        temperature grid."""
        tr, ti = _f64(t_re).copy(), _f64(t_im).copy()
        nre = np.zeros(self.spec_shape()); nim = np.zeros(self.spec_shape()); tg = np.zeros(self.grid_shape())
        self._check(self.lib.gd_compute_temperature_nonlinear(self.h, _dptr(tr), _dptr(ti), _dptr(_f64(u_theta)),
                                                              _dptr(_f64(u_phi)), _dptr(nre), _dptr(nim), _dptr(tg)))
        return (tr, ti), (nre, nim), tg

    def compute_composition_nonlinear_arrays(self, c_re, c_im, u_theta, u_phi):
        """compute_composition_nonlinear! (src/compositional.jl:219-259): returns the
        composition with its boundary conditions applied, the nonlinear term and
        the composition grid."""
        cr, ci = _f64(c_re).copy(), _f64(c_im).copy()
        nre = np.zeros(self.spec_shape()); nim = np.zeros(self.spec_shape()); cg = np.zeros(self.grid_shape())
        self._check(self.lib.gd_compute_composition_nonlinear(self.h, _dptr(cr), _dptr(ci), _dptr(_f64(u_theta)),
                                                              _dptr(_f64(u_phi)), _dptr(nre), _dptr(nim), _dptr(cg)))
        return (cr, ci), (nre, nim), cg

    def compute_velocity_nonlinear_arrays(self, tor, pol, j_theta=None, j_phi=None, b_theta=None, b_phi=None):
        """compute_velocity_nonlinear! (src/velocity.jl:312-332): nonlinear terms
        (tor, pol) and the velocity grids (u_theta, u_phi)."""
        out = [np.zeros(self.spec_shape()) for _ in range(4)]
        ut = np.zeros(self.grid_shape()); up = np.zeros(self.grid_shape())
        g = [None if x is None else _dptr(_f64(x)) for x in (j_theta, j_phi, b_theta, b_phi)]
        self._check(self.lib.gd_compute_velocity_nonlinear(
            self.h, _dptr(_f64(tor[0])), _dptr(_f64(tor[1])), _dptr(_f64(pol[0])), _dptr(_f64(pol[1])), *g,
            *[_dptr(o) for o in out], _dptr(ut), _dptr(up)))
        return (out[0], out[1]), (out[2], out[3]), (ut, up)

    def compute_magnetic_nonlinear_arrays(self, tor, pol, u_theta, u_phi):
        """compute_magnetic_nonlinear! (src/magnetic.jl:131-159): nonlinear terms
        (tor, pol) and the grids (b_theta, b_phi, j_theta, j_phi)."""
        out = [np.zeros(self.spec_shape()) for _ in range(4)]
        grids = [np.zeros(self.grid_shape()) for _ in range(4)]
        self._check(self.lib.gd_compute_magnetic_nonlinear(
            self.h, _dptr(_f64(tor[0])), _dptr(_f64(tor[1])), _dptr(_f64(pol[0])), _dptr(_f64(pol[1])),
            _dptr(_f64(u_theta)), _dptr(_f64(u_phi)), *[_dptr(o) for o in out], *[_dptr(g) for g in grids]))
        return (out[0], out[1]), (out[2], out[3]), tuple(grids)

    def set_field(self, name, re, im):
        self._check(self.lib.gd_upload_spectral(self.h, FIELDS[name], _dptr(_f64(re)), _dptr(_f64(im))))

    def field_names(self):
        """The state fields of this configuration (composition only when configured)."""
        return [k for k in FIELDS if k != "comp" or self.cfg.composition]

    def get_field(self, name):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self._check(self.lib.gd_download_spectral(self.h, FIELDS[name], _dptr(re), _dptr(im)))
        return re, im

    def get_nl(self, name):
        re = np.zeros(self.spec_shape()); im = np.zeros(self.spec_shape())
        self._check(self.lib.gd_download_nonlinear(self.h, FIELDS[name], _dptr(re), _dptr(im)))
        return re, im

    def get_grid(self, name):
        g = np.zeros(self.grid_shape())
        self._check(self.lib.gd_download_grid(self.h, GRIDS[name], _dptr(g)))
        return g

    def set_temperature_bc(self, bvals=None, sources=None):
        self._check(self.lib.gd_set_temperature_bc(
            self.h, _dptr(_f64(bvals)) if bvals is not None else None,
            _dptr(_f64(sources)) if sources is not None else None))

    def set_composition_bc(self, bvals=None, sources=None):
        """Composition boundary values or fluxes [2][nlm] and sources [nr]."""
        self._check(self.lib.gd_set_composition_bc(
            self.h, _dptr(_f64(bvals)) if bvals is not None else None,
            _dptr(_f64(sources)) if sources is not None else None))

    def set_bc_types(self, name, inner, outer):
        """bc_type_inner / bc_type_outer of "temp" or "comp": BC_VALUE or BC_FLUX per mode (l-major)."""
        a = np.ascontiguousarray(inner, dtype=np.int32)
        b = np.ascontiguousarray(outer, dtype=np.int32)
        if a.size != self.nlm or b.size != self.nlm:
            raise ValueError("one boundary type per mode")
        IP = ctypes.POINTER(ctypes.c_int)
        self._check(self.lib.gd_set_scalar_bc_types(self.h, FIELDS[name], a.ctypes.data_as(IP), b.ctypes.data_as(IP)))

    def composition_nl(self):
        self._check(self.lib.gd_composition_nonlinear(self.h))

    def temperature_nl(self):
        self._check(self.lib.gd_temperature_nonlinear(self.h))

    def velocity_nl(self):
        self._check(self.lib.gd_velocity_nonlinear(self.h))

    def magnetic_nl(self):
        self._check(self.lib.gd_magnetic_nonlinear(self.h))

    def implicit_step(self):
        self._check(self.lib.gd_implicit_step(self.h))

    def step(self, n=1):
        self._check(self.lib.gd_step(self.h, int(n)))

    def step_async(self, n=1):
        self._check(self.lib.gd_step_async(self.h, int(n)))

    def synchronize(self):
        self._check(self.lib.gd_synchronize(self.h))

    def set_scheme(self, scheme):
        """ts_scheme = :cnab2, :eab2 or :erk2 (src/simulation.jl:1054-1300); the
        exponential schemes build the cache of create_etd_cache /
        create_erk2_cache on the device."""
        self._check(self.lib.gd_set_scheme(self.h, SCHEMES[scheme]))
        self.scheme = scheme

    def etd_matrices(self, kind, l):
        """The exponential cache for a field kind ("velocity", "magnetic",
        "temperature") and degree l: {"E", "phi1", "phi2", "E_half",
        "phi1_half"} as nr x nr arrays."""
        out = {}
        for w, name in enumerate(ETD_MATRICES):
            m = np.zeros((self.nr, self.nr))
            self._check(self.lib.gd_download_etd(self.h, KINDS[kind], int(l), w, _dptr(m)))
            out[name] = m
        return out

    def set_dt(self, dt):
        self._check(self.lib.gd_set_dt(self.h, float(dt)))

    def energy(self):
        ek = ctypes.c_double(); em = ctypes.c_double()
        self._check(self.lib.gd_energy(self.h, ctypes.byref(ek), ctypes.byref(em)))
        return ek.value, em.value

    def check_finite(self):
        self._check(self.lib.gd_check_finite(self.h))

    def step_count(self):
        return self.lib.gd_step_count(self.h)

    def stream_ptr(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        p = ctypes.c_void_p()
        self._check(self.lib.gd_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def profile_enable(self, on=True):
        self._check(self.lib.gd_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        """{kernel name: (total ms, launches)} accumulated since the last read."""
        mx = 64
        names = ctypes.create_string_buffer(32 * mx)
        ms = np.zeros(mx)
        cnt = (ctypes.c_int * mx)()
        n = ctypes.c_int()
        self._check(self.lib.gd_profile_read(self.h, mx, names, _dptr(ms), cnt, ctypes.byref(n)))
        out = {}
        for k in range(min(n.value, mx)):
            nm = names.raw[32 * k: 32 * k + 32].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out


class SHTnsImplicitMatrices:
    """create_shtns_timestepping_matrices(config, domain, diffusivity, dt; theta)
    (src/timestep.jl:489-543): per degree l the diffusivity-scaled radial
    operator L_l and the banded LU of I/dt - theta L_l, on the model's device
    (gd_create_timestepping_matrices)."""

    def __init__(self, model: "SHTnsKitConfig", diffusivity, dt, theta=0.5):
        self.model, self.diffusivity, self.dt, self.theta = model, float(diffusivity), float(dt), float(theta)
        m = ctypes.c_void_p()
        model._check(model.lib.gd_create_timestepping_matrices(model.h, self.diffusivity, self.dt, self.theta,
                                                                ctypes.byref(m)))
        self.m = m

    def build_rhs_cnab2(self, un, nl, nl_prev, dt):
        """build_rhs_cnab2! (src/timestep.jl:610-690) on (re, im) plane pairs."""
        g = self.model
        rr = np.zeros(g.spec_shape()); ri = np.zeros(g.spec_shape())
        args = [_dptr(_f64(x)) for pair in (un, nl, nl_prev) for x in pair]
        g._check(g.lib.gd_build_rhs_cnab2(g.h, self.m, float(dt), *args, _dptr(rr), _dptr(ri)))
        return rr, ri

    def solve_implicit_step(self, rhs):
        """solve_implicit_step! (src/timestep.jl:692-730) on an (re, im) plane pair."""
        g = self.model
        sr = np.zeros(g.spec_shape()); si = np.zeros(g.spec_shape())
        g._check(g.lib.gd_solve_implicit_step(g.h, self.m, _dptr(_f64(rhs[0])), _dptr(_f64(rhs[1])), _dptr(sr),
                                              _dptr(si)))
        return sr, si

    def close(self):
        if getattr(self, "m", None) and getattr(self.model, "h", None):
            self.model.lib.gd_destroy_timestepping_matrices(self.m)
        self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radial_field_outer(model, pol_re, pol_im):
    """B_r on the grid at r = ro from poloidal coefficients (nr, nlm):
    l(l+1) / ro^2 P_lm(ro) synthesised (the build's radial-field formula; the
    reference never forms B_r).  Returns (nlon, nlat)."""
    ro = model.r[-1]
    f = model.l_values * (model.l_values + 1.0) / ro ** 2
    re = np.zeros(model.spec_shape()); im = np.zeros(model.spec_shape())
    re[-1] = f * pol_re[-1]; im[-1] = f * pol_im[-1]
    return model.synth_scalar(re, im)[-1]


def magnetic_misfit(model, target, nsteps, checkpoint_every=20):
    """Objective of the adjoint configuration and its gradient.

    Runs ``nsteps`` steps from the model's current state and returns
    (J, grad_re, grad_im, checkpoints) with
      J = 1/2 sum_grid (B_r(ro) - target)^2   (target: (nlon, nlat) grid),
    the gradient of J with respect to the initial poloidal magnetic
    coefficients (nr x nlm Re and Im planes, l-major), and the state
    (dict name -> (re, im)) every ``checkpoint_every`` steps.  Reverse pass:
    the residual goes through the transposed synthesis and the l(l+1)/ro^2
    factor to the cotangent of B_pol(ro), then through gd_magnetic_pullback.
    The pullback needs none of the checkpoints: the magnetic propagator of the
    reference's step does not depend on the state (gd_magnetic_pullback); they
    are kept for restarts and for objectives whose pullback would."""
    checkpoints = []
    done = 0
    while done < nsteps:
        if checkpoint_every and done % checkpoint_every == 0:
            checkpoints.append((done, {k: model.get_field(k) for k in model.field_names()}))
        k = min(checkpoint_every or nsteps, nsteps - done)
        model.step(k)
        done += k
    pre, pim = model.get_field("b_pol")
    resid = radial_field_outer(model, pre, pim) - target
    J = 0.5 * float(np.sum(resid * resid))
    gbar = np.zeros(model.grid_shape())
    gbar[-1] = resid
    cre, cim = model.synth_scalar_adjoint(gbar)
    ro = model.r[-1]
    f = model.l_values * (model.l_values + 1.0) / ro ** 2
    lre = np.zeros(model.spec_shape()); lim = np.zeros(model.spec_shape())
    lre[-1] = f * cre[-1]; lim[-1] = f * cim[-1]
    gre, gim = model.magnetic_pullback("b_pol", nsteps, lre, lim)
    return J, gre, gim, checkpoints


def temperature_misfit(model, target, nsteps, checkpoint_every=20, shell=None):
    """A temperature objective and its gradient by checkpoint and recompute.

    Runs ``nsteps`` steps from the model's current state (an FP64, CNAB2 model
    with fixed-value temperature boundaries) and returns (J, grad_re, grad_im)
    with J = 1/2 sum_grid (T(r_shell) - target)^2 at the end (target: the
    (nlon, nlat) grid of shell ``shell``, default the middle one) and the
    gradient of J with respect to the initial temperature coefficients (nr x
    nlm Re and Im planes, l-major).  The model is left in its state after the
    steps.  Forward: gd_temperature_forward (a device snapshot every
    ``checkpoint_every`` steps); reverse: the residual through the transposed
    synthesis, then gd_temperature_pullback (the velocity grids recomputed
    segment by segment from the snapshots)."""
    model.temperature_forward(nsteps, checkpoint_every)
    shell = model.nr // 2 if shell is None else int(shell)
    tre, tim = model.get_field("temp")
    grid = model.synth_scalar(tre, tim)
    resid = grid[shell] - np.asarray(target, dtype=np.float64)
    J = 0.5 * float(np.sum(resid * resid))
    gbar = np.zeros(model.grid_shape())
    gbar[shell] = resid
    lre, lim = model.synth_scalar_adjoint(gbar)
    gre, gim = model.temperature_pullback(lre, lim)
    return J, gre, gim


class Ensemble:
    """Independent shells stepped together (gd_ensemble_*): one CUDA graph
    launch per step runs every handle's step as its own branch.  ``members``
    are SHTnsKitConfig views of the member handles (upload, download, energy,
    nonlinear terms as for a single model); the ensemble owns the handles.

    ``group`` > 1 stacks up to that many members whose configurations differ
    only in the Ekman number, the number of radial levels and the Rayleigh
    number (which the step does not read: the vector analysis drops the radial
    buoyancy force) into one segmented handle (gd_config.segments,
    segment_nr), each member with its own radial grid and operators and its
    own Coriolis factor: every per-shell kernel then serves the whole group in
    one launch.  Its members are EnsembleSegment views of their levels."""

    def __init__(self, configs, precision="fp64", device=0, group=1):
        self.lib = load_library()
        configs = [dict(c) for c in configs]
        slots = []
        if group > 1:
            open_ = {}
            for i, c in enumerate(configs):
                key = tuple(sorted((k, repr(v)) for k, v in c.items() if k not in ("ekman", "rayleigh", "nr")))
                lst = open_.get(key)
                if lst is None or len(lst) >= group:
                    lst = []
                    open_[key] = lst
                    slots.append(lst)
                lst.append(i)
        else:
            slots = [[i] for i in range(len(configs))]
        n = len(slots)
        arr = (GDConfig * n)()
        self._segnr = []  # segment lengths, alive while the handles are created
        for i, slot in enumerate(slots):
            c = dict(configs[slot[0]])
            segnr = None
            if len(slot) > 1:
                lens = [int(configs[j]["nr"]) for j in slot]
                c["nr"] = sum(lens)
                c["segments"] = len(slot)
                if len(set(lens)) > 1:
                    segnr = (ctypes.c_int * len(lens))(*lens)
                    self._segnr.append(segnr)
            lmax = c.pop("lmax")
            mmax = c.pop("mmax", None)
            mmax = lmax if mmax is None else mmax
            arr[i] = GDConfig(lmax, mmax, c.pop("nlat"), c.pop("nlon"), c.pop("nr"), c.pop("kl", 4),
                              c.pop("rratio", 0.35), c.pop("ekman", 3e-4), c.pop("rayleigh", 80.0),
                              c.pop("prandtl", 1.0), c.pop("magnetic_prandtl", 4.0), c.pop("dt", 1e-5),
                              c.pop("implicit_theta", 0.5), c.pop("ab_mode", 0), c.pop("bc_mode", 0),
                              c.pop("fd_mode", 0), PRECISIONS[c.pop("precision", precision)],
                              c.pop("magnetic", 1), c.pop("composition", 0), c.pop("schmidt", 1.0),
                              c.pop("segments", 0), GEOMETRIES[c.pop("geometry", "shell")], c.pop("r_outer", 1.0))
            if segnr is not None:
                arr[i].segment_nr = ctypes.cast(segnr, ctypes.POINTER(ctypes.c_int))
        e = ctypes.c_void_p()
        st = self.lib.gd_ensemble_create(arr, n, int(device), ctypes.byref(e))
        if st != GD_OK:
            raise GeoDynamoError(st, "gd_ensemble_create failed (see stderr)")
        self.e = e
        self.handles = [SHTnsKitConfig._member(self.lib, ctypes.c_void_p(self.lib.gd_ensemble_member(e, i)), arr[i])
                        for i in range(n)]
        self.members = [None] * len(configs)
        for hv, slot in zip(self.handles, slots):
            if len(slot) == 1:
                self.members[slot[0]] = hv
                continue
            hv.set_segment_ekman([configs[i].get("ekman", 3e-4) for i in slot])
            base = 0
            for g, i in enumerate(slot):
                self.members[i] = EnsembleSegment(hv, g, configs[i]["nr"], base)
                base += int(configs[i]["nr"])

    def __len__(self):
        return len(self.members)

    def step(self, n=1):
        st = self.lib.gd_ensemble_step(self.e, int(n))
        if st != GD_OK:
            i = self.lib.gd_ensemble_failed_member(self.e)
            msg = self.lib.gd_last_error(self.members[i].h).decode() if i >= 0 else ""
            raise GeoDynamoError(st, f"member {i}: {msg}")

    def autotune(self, nsteps=5):
        """Chooses the members' tensor-core grid caps by timing candidates on a
        scratch copy of the ensemble (gd_ensemble_autotune); returns
        (ms per ensemble step, caps), one cap per handle."""
        ms = ctypes.c_float()
        caps = (ctypes.c_int * len(self.handles))()
        st = self.lib.gd_ensemble_autotune(self.e, int(nsteps), ctypes.byref(ms), caps)
        if st != GD_OK:
            raise GeoDynamoError(st, "gd_ensemble_autotune failed")
        return ms.value, list(caps)

    def step_async(self, n=1):
        st = self.lib.gd_ensemble_step_async(self.e, int(n))
        if st != GD_OK:
            raise GeoDynamoError(st, "gd_ensemble_step_async failed")

    def stream_ptr(self):
        s = ctypes.c_void_p()
        st = self.lib.gd_ensemble_get_stream(self.e, ctypes.byref(s))
        if st != GD_OK:
            raise GeoDynamoError(st, "gd_ensemble_get_stream failed")
        return s.value

    def close(self):
        if getattr(self, "e", None):
            for m in self.handles:
                m.h = None
            self.lib.gd_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EnsembleSegment:
    """One member of a grouped ensemble: levels [base, base + nr) of a
    segmented handle.  Fields, nonlinear terms and energies of the member
    alone; the step runs for the whole handle."""

    def __init__(self, handle, seg, nr, base=None):
        self.handle = handle
        self.seg = int(seg)
        self.nr = int(nr)
        base = self.seg * self.nr if base is None else int(base)
        self.lmax, self.mmax, self.nlat, self.nlon, self.nlm = (handle.lmax, handle.mmax, handle.nlat,
                                                                handle.nlon, handle.nlm)
        self.rows = slice(base, base + self.nr)

    def spec_shape(self):
        return (self.nr, self.nlm)

    def field_names(self):
        return self.handle.field_names()

    def set_field(self, name, re, im):
        fr, fi = self.handle.get_field(name)
        fr[self.rows] = np.asarray(re, dtype=np.float64).reshape(self.spec_shape())
        fi[self.rows] = np.asarray(im, dtype=np.float64).reshape(self.spec_shape())
        self.handle.set_field(name, fr, fi)

    def get_field(self, name):
        fr, fi = self.handle.get_field(name)
        return fr[self.rows].copy(), fi[self.rows].copy()

    def get_nl(self, name):
        fr, fi = self.handle.get_nl(name)
        return fr[self.rows].copy(), fi[self.rows].copy()

    def energy(self):
        ek, em = self.handle.segment_energy()
        return float(ek[self.seg]), float(em[self.seg])

    def step_count(self):
        return self.handle.step_count()

    def launch_shape(self):
        return self.handle.launch_shape()


# ---------------------------------------------------------------------------
# Reference-shaped field containers (src/fields.jl:6-32) and functions.
# ---------------------------------------------------------------------------
class SHTnsSpectralField:
    """``SHTnsSpectralField``: Re/Im planes, shape (nr, nlm), l-major index fastest."""

    def __init__(self, config: SHTnsKitConfig):
        self.config = config
        self.nlm = config.nlm
        self.data_real = np.zeros(config.spec_shape())
        self.data_imag = np.zeros(config.spec_shape())


class SHTnsPhysicalField:
    """``SHTnsPhysicalField``: shape (nr, nlon, nlat), theta fastest."""

    def __init__(self, config: SHTnsKitConfig):
        self.config = config
        self.nlat, self.nlon = config.nlat, config.nlon
        self.data = np.zeros(config.grid_shape())


class SHTnsVectorField:
    def __init__(self, config: SHTnsKitConfig):
        self.r_component = SHTnsPhysicalField(config)
        self.theta_component = SHTnsPhysicalField(config)
        self.phi_component = SHTnsPhysicalField(config)


def create_shtnskit_config(*, lmax, mmax=None, nlat=None, nlon=None, nr=64, **kw) -> SHTnsKitConfig:
    """Defaults follow ``create_shtnskit_config`` (nlat = lmax + 2, nlon = max(2 lmax + 1, 4)),
    rounded up to an even nlat and a 2/3/5-smooth nlon."""
    mmax = lmax if mmax is None else mmax
    if nlat is None:
        nlat = lmax + 2
        nlat += nlat & 1
    if nlon is None:
        nlon = max(2 * lmax + 1, 4)
        while True:
            m = nlon
            for p in (2, 3, 5):
                while m % p == 0:
                    m //= p
            if m == 1:
                break
            nlon += 1
    return SHTnsKitConfig(lmax, nlat, nlon, nr, mmax=mmax, **kw)


def create_shtns_spectral_field(config):
    return SHTnsSpectralField(config)


def create_shtns_physical_field(config):
    return SHTnsPhysicalField(config)


def create_shtns_vector_field(config):
    return SHTnsVectorField(config)


def shtnskit_spectral_to_physical(spec: SHTnsSpectralField, phys: SHTnsPhysicalField):
    phys.data[...] = spec.config.synth_scalar(spec.data_real, spec.data_imag)
    return phys


def shtnskit_physical_to_spectral(phys: SHTnsPhysicalField, spec: SHTnsSpectralField):
    re, im = spec.config.analysis_scalar(phys.data)
    spec.data_real[...] = re
    spec.data_imag[...] = im
    return spec


def batch_spectral_to_physical(specs, physs):
    """One batched launch for all fields (``shtnskit_field_functions.jl:651-677``)."""
    if len(specs) != len(physs):
        raise GeoDynamoError(1, "specs and physs differ in length")
    if not specs:
        return
    cfg = specs[0].config
    re = np.stack([s.data_real for s in specs])
    im = np.stack([s.data_imag for s in specs])
    out = cfg.synth_scalar(re, im)
    for p, g in zip(physs, out):
        p.data[...] = g


def shtnskit_vector_synthesis(tor: SHTnsSpectralField, pol: SHTnsSpectralField, vec: SHTnsVectorField):
    vt, vp = tor.config.synth_vector(tor.data_real, tor.data_imag, pol.data_real, pol.data_imag)
    vec.theta_component.data[...] = vt
    vec.phi_component.data[...] = vp
    return vec


def shtnskit_vector_analysis(vec: SHTnsVectorField, tor: SHTnsSpectralField, pol: SHTnsSpectralField):
    tre, tim, pre, pim = tor.config.analysis_vector(vec.theta_component.data, vec.phi_component.data)
    tor.data_real[...] = tre
    tor.data_imag[...] = tim
    pol.data_real[...] = pre
    pol.data_imag[...] = pim
    return tor, pol


class SimulationState:
    """Device-resident model state of one shell run (``SimulationState``,
    ``simulation.jl``), created from a config handle.  Field arrays live on
    the device; :meth:`field` / :meth:`set_field` copy them in the reference layout."""

    def __init__(self, config: SHTnsKitConfig):
        self.config = config

    def set_field(self, name, re, im):
        self.config.set_field(name, re, im)

    def field(self, name):
        return self.config.get_field(name)

    def nonlinear(self, name):
        return self.config.get_nl(name)


def compute_temperature_nonlinear(state: SimulationState):
    state.config.temperature_nl()


def compute_velocity_nonlinear(state: SimulationState):
    state.config.velocity_nl()


def compute_magnetic_nonlinear(state: SimulationState):
    state.config.magnetic_nl()


def apply_master_implicit_step(state: SimulationState, dt=None):
    if dt is not None and dt != state.config.cfg.dt:
        state.config.set_dt(dt)
        state.config.cfg.dt = dt
    state.config.implicit_step()


def step_once(state: SimulationState):
    """``step_once!`` (scripts/bench_timestepping.jl:6-18) as one graph replay."""
    state.config.step(1)


def create_shtns_timestepping_matrices(config: SHTnsKitConfig, diffusivity, dt, theta=0.5):
    """create_shtns_timestepping_matrices (src/timestep.jl:498-543)."""
    return SHTnsImplicitMatrices(config, diffusivity, dt, theta)


def build_rhs_cnab2(rhs: SHTnsSpectralField, un: SHTnsSpectralField, nl: SHTnsSpectralField,
                    nl_prev: SHTnsSpectralField, dt, matrices: SHTnsImplicitMatrices):
    """build_rhs_cnab2! (src/timestep.jl:610-690): fills rhs in place."""
    rhs.data_real[...], rhs.data_imag[...] = matrices.build_rhs_cnab2(
        (un.data_real, un.data_imag), (nl.data_real, nl.data_imag), (nl_prev.data_real, nl_prev.data_imag), dt)
    return rhs


def solve_implicit_step(solution: SHTnsSpectralField, rhs: SHTnsSpectralField, matrices: SHTnsImplicitMatrices):
    """solve_implicit_step! (src/timestep.jl:692-730): fills solution in place."""
    solution.data_real[...], solution.data_imag[...] = matrices.solve_implicit_step((rhs.data_real, rhs.data_imag))
    return solution


def compute_kinetic_energy(state: SimulationState):
    return state.config.energy()[0]


def compute_magnetic_energy(state: SimulationState):
    return state.config.energy()[1]


# -- restart files (restart.py): write_restart! / read_restart!
#    (src/outputs_writer.jl:1221-1371) -------------------------------------------
def write_restart(model: SHTnsKitConfig, filename, **kw):
    """The model's spectral state (and physical temperature) in the reference's
    restart layout; keywords as ``restart.write_restart``."""
    from . import restart
    return restart.write_restart(model, filename, **kw)


def read_restart(filename):
    """``(restart_data, metadata)`` of a restart file, as read_restart! returns them."""
    from . import restart
    return restart.read_restart(filename)


def load_restart(model: SHTnsKitConfig, filename):
    """Sets a fresh model's five spectral fields from a restart file; the run
    continues as a new run (AB1 start), like the reference's restarted run."""
    from . import restart
    return restart.load_restart(model, filename)

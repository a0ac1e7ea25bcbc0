"""ctypes binding of the C ABI (``include/solprop_b200.h``).

The structures mirror the header field for field.  Nothing here computes: every call
forwards to ``libsolprop_b200.so``, which must have been built (``python -m
solprop_b200.build``); a missing library is an error, never a fallback.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIBRARY_PATH = Path(__file__).resolve().parent / "libsolprop_b200.so"

SP_OK = 0
STATUS_NAMES = {1: "argument", 2: "refused", 3: "cuda", 4: "state", 5: "convergence"}


class SpTable(C.Structure):
    _fields_ = [("n_intervals", C.c_int32), ("n_deg", C.c_int32), ("n_values", C.c_int32),
                ("breakpoints", C.POINTER(C.c_double)), ("coefficients", C.POINTER(C.c_double))]


class SpPlasmaChannel(C.Structure):
    _fields_ = [("charge_mass_ratio", C.c_double), ("ionisation_potential", C.c_double),
                ("rate_intervals", C.c_int32), ("rate_coefficients", C.POINTER(C.c_double)),
                ("log_field_min", C.c_double), ("d_log_field", C.c_double), ("field_min", C.c_double),
                ("field_max", C.c_double), ("rate_max", C.c_double),
                ("plasma_density", SpTable), ("preionisation", SpTable)]


class SpRamanComponent(C.Structure):
    _fields_ = [("terms", C.c_int32), ("undamped", C.POINTER(C.c_double)), ("rates", SpTable * 4),
                ("fraction", C.c_double), ("density", SpTable), ("tensor_weights", C.POINTER(C.c_double))]


class SpProblemDesc(C.Structure):
    _fields_ = [
        ("grid_kind", C.c_int32),
        ("n_modes", C.c_int32), ("n_pol", C.c_int32), ("n_omega", C.c_int32), ("n_t", C.c_int32),
        ("n_to", C.c_int32), ("n_nodes", C.c_int32), ("n_pol_transform", C.c_int32),
        ("omega0", C.c_double), ("dt", C.c_double), ("dt_fine", C.c_double), ("z_end", C.c_double),
        ("omega", C.POINTER(C.c_double)), ("crop_index", C.POINTER(C.c_int64)),
        ("active_mask", C.POINTER(C.c_uint8)), ("norm_mask", C.POINTER(C.c_uint8)),
        ("omega_window", C.POINTER(C.c_double)), ("t_window", C.POINTER(C.c_double)),
        ("t_window_derivative", C.POINTER(C.c_double)), ("carrier", C.POINTER(C.c_double)),
        ("phi_expansion", C.c_int32), ("n_phi_terms", C.c_int32),
        ("phi_terms", C.POINTER(C.c_double)), ("phi_weights", SpTable), ("phi_rate", SpTable),
        ("n_prefactor_terms", C.c_int32), ("prefactor_terms", C.POINTER(C.c_double)),
        ("prefactor_weights", SpTable),
        ("density", SpTable), ("kerr_density", SpTable), ("plasma_density", SpTable),
        ("preionisation", SpTable), ("taper_scale", SpTable),
        ("synthesis", C.POINTER(C.c_double)), ("projection", C.POINTER(C.c_double)),
        ("kerr_enabled", C.c_int32), ("kerr_analytic", C.c_int32),
        ("kerr_coefficient", C.c_double), ("kerr_self", C.c_double),
        ("kerr_conjugate", C.c_double), ("kerr_harmonic", C.c_double),
        ("kerr_take_real", C.c_int32),
        ("plasma_enabled", C.c_int32), ("charge_mass_ratio", C.c_double),
        ("ionisation_potential", C.c_double), ("rate_intervals", C.c_int32),
        ("rate_coefficients", C.POINTER(C.c_double)),
        ("log_field_min", C.c_double), ("d_log_field", C.c_double), ("field_min", C.c_double),
        ("field_max", C.c_double), ("rate_max", C.c_double),
        ("band", C.c_int32), ("n_taps", C.c_int32), ("taps", C.POINTER(C.c_double)),
        ("raman_enabled", C.c_int32), ("raman_terms", C.c_int32), ("raman_thg", C.c_int32),
        ("raman_undamped", C.POINTER(C.c_double)), ("raman_rates", SpTable * 4),
        ("raman_fraction", C.c_double), ("raman_density", SpTable),
        ("absorber_in_stage", C.c_int32), ("temporal_absorber_fine", C.POINTER(C.c_double)),
        ("n_extra_channels", C.c_int32), ("extra_channels", C.POINTER(SpPlasmaChannel)),
        ("n_extra_raman", C.c_int32), ("extra_raman", C.POINTER(SpRamanComponent)),
        ("raman_tensor_weights", C.POINTER(C.c_double)),
    ]


class SpRunDesc(C.Structure):
    _fields_ = [
        ("method", C.c_int32), ("field0", C.POINTER(C.c_double)),
        ("z_start", C.c_double), ("proposal", C.c_double), ("rtol", C.c_double), ("atol", C.c_double),
        ("dz_min", C.c_double), ("dz_max", C.c_double), ("stretch", C.c_double), ("z_end", C.c_double),
        ("save_planes", C.POINTER(C.c_double)), ("n_save_planes", C.c_int32),
        ("hard_kinks", C.POINTER(C.c_double)), ("n_hard_kinks", C.c_int32),
        ("breakpoints", C.POINTER(C.c_double)), ("n_breakpoints", C.c_int32),
        ("schedule", C.POINTER(C.c_double)), ("n_schedule", C.c_int32),
        ("order", C.c_int32), ("variable_order", C.c_int32), ("restart_after", C.c_int32),
        ("equal_approach", C.c_int32),
        ("safety", C.c_double), ("max_growth", C.c_double), ("min_factor", C.c_double),
        ("rejection_growth", C.c_double), ("hysteresis", C.c_double),
        ("collar_stability", C.c_double), ("collar_rate", C.c_double),
        ("real_intervals", C.c_double * 8),
        ("beta1", C.c_double), ("beta2", C.c_double), ("max_factor", C.c_double),
        ("lag", C.c_int32), ("estimator_order", C.c_int32),
        ("auto_init", C.c_int32), ("start_growth", C.c_double),
    ]


class SpBatch(C.Structure):
    _fields_ = [("event", C.c_int32), ("plane_index", C.c_int32), ("z", C.c_double),
                ("attempts", C.c_int64), ("rejected", C.c_int64), ("evaluations", C.c_int64),
                ("reason", C.c_int32), ("category", C.c_int32),
                ("rows", C.POINTER(C.c_double)), ("rows_capacity", C.c_int32),
                ("n_rows", C.c_int32)]


class SpMarchState(C.Structure):
    _fields_ = [("z", C.c_double), ("proposal", C.c_double), ("attempts", C.c_int64),
                ("rejected", C.c_int64), ("evaluations", C.c_int64), ("order", C.c_int32),
                ("history_rows", C.c_int32), ("rejections", C.c_int32),
                ("plane_index", C.c_int32), ("outcome", C.c_int32)]


# sp_batch.event, .reason and .category (include/solprop_b200.h)
EVENTS = {0: "none", 1: "plane", 2: "finished", 3: "failed", 4: "stopped", 5: "halted"}
REASONS = {0: "reached", 3: "bound", 5: "floor", 6: "error", 7: "diverged", 11: "stopped",
           12: "halted"}
CATEGORIES = {0: "none", 1: "convergence", 2: "backend", 3: "value", 4: "refused"}


class SpStatistics(C.Structure):
    _fields_ = [("energy", C.POINTER(C.c_double)), ("omega0", C.POINTER(C.c_double)),
                ("peak_power", C.POINTER(C.c_double)), ("peak_power_total", C.POINTER(C.c_double)),
                ("spectrum", C.POINTER(C.c_double))]


def statistics_call(fn, rec, power_weight=None) -> dict:
    """Run an ``sp_*_statistics`` entry point ``fn(power_weight_ptr, out_ptr)`` into fresh
    host arrays: energy and omega0 per (mode, polarisation), peak_power per mode,
    peak_power_total, and the energy per bin."""
    out = {"energy": np.empty((rec.n_modes, rec.n_pol)), "omega0": np.empty((rec.n_modes, rec.n_pol)),
           "peak_power": np.empty(rec.n_modes), "peak_power_total": np.empty(1),
           "spectrum": np.empty(rec.n_omega)}
    st = SpStatistics(*(out[name].ctypes.data_as(C.POINTER(C.c_double)) for name in
                        ("energy", "omega0", "peak_power", "peak_power_total", "spectrum")))
    pw = None
    if power_weight is not None:
        pw = np.ascontiguousarray(np.broadcast_to(power_weight, (rec.n_modes, rec.n_pol, rec.n_omega)),
                                  dtype=np.float64)
    check(fn(_ptr(pw), C.byref(st)))
    out["peak_power_total"] = float(out["peak_power_total"][0])
    return out


class SpScanStatus(C.Structure):
    _fields_ = [("active", C.c_int32), ("attempts", C.c_int64), ("rejected", C.c_int64),
                ("evaluations", C.c_int64), ("batch_steps", C.c_int64)]


# the exported functions: name -> (restype, argtypes)
SIGNATURES = {
    "sp_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "sp_version": (C.c_char_p, []),
    "sp_device_count": (C.c_int, []),
    "sp_problem_create": (C.c_int, [C.POINTER(SpProblemDesc), C.POINTER(C.c_void_p)]),
    "sp_problem_destroy": (C.c_int, [C.c_void_p]),
    "sp_workspace_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "sp_workspace_create_ex": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sp_workspace_create_ex2": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    # the scan surrogate's perceptron kernels (device pointers, stream may be NULL)
    "sp_mlp_gemm": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                              C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                              C.c_void_p]),
    "sp_mlp_gemm_tc": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                 C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                 C.c_void_p]),
    "sp_mlp_gemm_tc_batch": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p), C.c_int,
                                       C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_void_p,
                                       C.c_void_p]),
    "sp_mlp_to_bf16": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                 C.c_void_p]),
    "sp_mlp_transpose_bf16": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                        C.c_int, C.c_void_p]),
    "sp_mlp_gelu_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "sp_mlp_bias_grad": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "sp_mlp_mse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p]),
    "sp_mlp_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float,
                              C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "sp_mlp_ensemble_stats": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "sp_workspace_destroy": (C.c_int, [C.c_void_p]),
    "sp_workspace_source": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_int,
                                      C.POINTER(C.c_double)]),
    "sp_workspace_source_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p]),
    "sp_workspace_launches_per_source": (C.c_int, [C.c_void_p]),
    "sp_session_start": (C.c_int, [C.c_void_p, C.POINTER(SpRunDesc), C.POINTER(C.c_void_p)]),
    "sp_session_advance": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.POINTER(SpBatch)]),
    "sp_session_request_stop": (C.c_int, [C.c_void_p]),
    "sp_session_request_snapshot": (C.c_int, [C.c_void_p]),
    "sp_session_march_state": (C.c_int, [C.c_void_p, C.POINTER(SpMarchState)]),
    "sp_session_snapshot": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "sp_session_restore": (C.c_int, [C.c_void_p, C.POINTER(SpRunDesc), C.c_void_p, C.c_size_t,
                                     C.POINTER(C.c_void_p)]),
    "sp_session_export": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "sp_session_statistics": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(SpStatistics)]),
    "sp_scan_statistics": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                     C.POINTER(SpStatistics)]),
    "sp_session_destroy": (C.c_int, [C.c_void_p]),
    "sp_workspace_stream": (C.c_void_p, [C.c_void_p]),
    "sp_session_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "sp_session_timing": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]),
    "sp_source_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                    C.c_void_p]),
    "sp_scan_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p), C.POINTER(SpRunDesc), C.c_int,
                                 C.POINTER(C.c_void_p)]),
    "sp_scan_create_ex": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p), C.POINTER(SpRunDesc), C.c_int, C.c_int,
                                 C.POINTER(C.c_void_p)]),
    "sp_scan_advance": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(SpScanStatus)]),
    "sp_scan_describe": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sp_scan_set_column": (C.c_int, [C.c_void_p, C.c_int32]),
    "sp_scan_set_alone": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double]),
    "sp_scan_set_transforms": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "sp_scan_run": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(SpBatch)]),
    "sp_scan_stream": (C.c_void_p, [C.c_void_p]),
    "sp_scan_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "sp_scan_timing": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]),
    "sp_scan_destroy": (C.c_int, [C.c_void_p]),
}

KERNEL_NAMES = ("adams_predict", "inverse_fft", "response_column", "project", "forward_fft",
                "stage_output", "adams_correct", "adams_accept", "adams_start", "rk_stage_input",
                "rk_finish")

_LIB: C.CDLL | None = None


class NativeError(RuntimeError):
    """A failure the library reported, with its status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{STATUS_NAMES.get(status, status)}] {message}")
        self.status = status


class BackendRefusal(NativeError):
    """The library refuses this problem by name (``SP_ERR_REFUSED``)."""


class ConvergenceError(NativeError):
    """Step control fell below its floor or a replayed step diverged
    (``SP_ERR_CONVERGENCE``; solprop's ``ConvergenceError`` category)."""


class BackendError(NativeError):
    """A device failure (``SP_ERR_CUDA``; solprop's ``BackendError`` category)."""


class SessionLifecycleError(NativeError):
    """A call out of the session's lifecycle (``SP_ERR_STATE``; native
    ``_core.SessionLifecycleError``): after a failure, a stop or a close."""


ERRORS = {2: BackendRefusal, 3: BackendError, 4: SessionLifecycleError, 5: ConvergenceError}


def library() -> C.CDLL:
    """Load ``libsolprop_b200.so`` once; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIBRARY_PATH.exists():
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `python -m solprop_b200.build` "
                "(this package has no CPU path)")
        lib = C.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _LIB = lib
    return _LIB


def check(status: int) -> None:
    if status != SP_OK:
        buf = C.create_string_buffer(4096)
        library().sp_last_error(buf, 4096)
        message = buf.value.decode(errors="replace")
        raise ERRORS.get(status, NativeError)(status, message)


def _ptr(array: np.ndarray | None, ctype=C.c_double):
    if array is None:
        return C.POINTER(ctype)()
    return array.ctypes.data_as(C.POINTER(ctype))


class Marshalled:
    """A record's arrays converted to the C layout, kept alive beside the descriptor."""

    def __init__(self):
        self.keep: list = []  # arrays and ctypes arrays

    def f64(self, a) -> C.POINTER(C.c_double):
        if a is None:
            return C.POINTER(C.c_double)()
        arr = np.ascontiguousarray(a, dtype=np.float64)
        self.keep.append(arr)
        return _ptr(arr)

    def c128(self, a) -> C.POINTER(C.c_double):
        if a is None:
            return C.POINTER(C.c_double)()
        arr = np.ascontiguousarray(a, dtype=np.complex128)
        self.keep.append(arr)
        return arr.ctypes.data_as(C.POINTER(C.c_double))

    def u8(self, a):
        arr = np.ascontiguousarray(np.asarray(a).astype(np.uint8))
        self.keep.append(arr)
        return _ptr(arr, C.c_uint8)

    def i64(self, a):
        arr = np.ascontiguousarray(a, dtype=np.int64)
        self.keep.append(arr)
        return _ptr(arr, C.c_int64)

    def table(self, t) -> SpTable:
        out = SpTable()
        if t is None:
            return out
        c = np.ascontiguousarray(t.coefficients, dtype=np.float64)
        out.n_intervals, out.n_deg, out.n_values = c.shape
        out.breakpoints = self.f64(t.breakpoints)
        out.coefficients = self.f64(c)
        return out


def problem_desc(rec) -> tuple[SpProblemDesc, Marshalled]:
    """The C descriptor of a :class:`solprop_b200.record.ProblemRecord`."""
    m = Marshalled()
    d = SpProblemDesc()
    d.grid_kind = 0 if rec.grid_kind == "field" else 1
    d.n_modes, d.n_pol, d.n_omega = rec.n_modes, rec.n_pol, rec.n_omega
    d.n_t, d.n_to, d.n_nodes, d.n_pol_transform = rec.n_t, rec.n_to, rec.n_nodes, rec.n_pol_transform
    d.omega0, d.dt, d.dt_fine, d.z_end = rec.omega0, rec.dt, rec.dt_fine, rec.z_end
    d.omega = m.f64(rec.omega)
    d.crop_index = m.i64(rec.crop_index)
    d.active_mask = m.u8(rec.active_mask)
    d.norm_mask = m.u8(rec.norm_mask)
    d.omega_window = m.f64(rec.omega_window)
    d.t_window = m.f64(rec.t_window)
    d.t_window_derivative = m.f64(rec.t_window_derivative)
    d.carrier = m.c128(rec.carrier)
    d.phi_expansion = int(rec.phi_representation == "expansion")
    d.n_phi_terms = rec.n_phi_terms
    d.phi_terms = m.c128(rec.phi_terms)
    d.phi_weights = m.table(rec.phi_weights)
    d.phi_rate = m.table(rec.phi_rate)
    d.n_prefactor_terms = rec.n_prefactor_terms
    d.prefactor_terms = m.c128(rec.prefactor_terms)
    d.prefactor_weights = m.table(rec.prefactor_weights)
    d.density = m.table(rec.density)
    d.kerr_density = m.table(rec.kerr_density)
    d.plasma_density = m.table(rec.plasma_density)
    d.preionisation = m.table(rec.preionisation)
    d.taper_scale = m.table(rec.taper_scale)
    d.synthesis = m.f64(rec.synthesis)
    d.projection = m.f64(rec.projection)
    d.kerr_enabled = int(rec.kerr_enabled)
    d.kerr_analytic = int(rec.kerr_form != "real")
    d.kerr_coefficient = rec.kerr_coefficient
    d.kerr_self, d.kerr_conjugate, d.kerr_harmonic = rec.kerr_self, rec.kerr_conjugate, rec.kerr_harmonic
    d.kerr_take_real = int(rec.kerr_take_real)
    d.plasma_enabled = int(rec.plasma_enabled)
    if rec.plasma_enabled:
        d.charge_mass_ratio = rec.charge_mass_ratio
        d.ionisation_potential = rec.ionisation_potential
        d.rate_intervals = rec.rate_coefficients.shape[1]
        d.rate_coefficients = m.f64(rec.rate_coefficients)
        d.log_field_min, d.d_log_field = rec.log_field_min, rec.d_log_field
        d.field_min, d.field_max, d.rate_max = rec.field_min, rec.field_max, rec.rate_max
        d.band = int(rec.integral_policy == "band")
        d.n_taps = rec.taps.size
        d.taps = m.f64(rec.taps)
    d.raman_enabled = int(rec.raman_enabled)
    if rec.raman_enabled:
        d.raman_terms = rec.raman_undamped.shape[0]
        d.raman_thg = int(rec.raman_thg)
        d.raman_undamped = m.f64(rec.raman_undamped)
        for i, t in enumerate(rec.raman_rates[:4]):
            d.raman_rates[i] = m.table(t)
        d.raman_fraction = rec.raman_fraction
        d.raman_density = m.table(rec.raman_density)
        d.raman_tensor_weights = m.f64(rec.raman_tensor_weights)
    d.absorber_in_stage = int(rec.absorber_scheme == "nonlinear")
    d.temporal_absorber_fine = m.f64(rec.temporal_absorber_fine)
    if rec.extra_channels:
        channels = (SpPlasmaChannel * len(rec.extra_channels))()
        for i, ch in enumerate(rec.extra_channels):
            c = channels[i]
            c.charge_mass_ratio, c.ionisation_potential = ch.charge_mass_ratio, ch.ionisation_potential
            c.rate_intervals = ch.rate_coefficients.shape[1]
            c.rate_coefficients = m.f64(ch.rate_coefficients)
            c.log_field_min, c.d_log_field = ch.log_field_min, ch.d_log_field
            c.field_min, c.field_max, c.rate_max = ch.field_min, ch.field_max, ch.rate_max
            c.plasma_density = m.table(ch.plasma_density)
            c.preionisation = m.table(ch.preionisation)
        m.keep.append(channels)
        d.n_extra_channels = len(rec.extra_channels)
        d.extra_channels = C.cast(channels, C.POINTER(SpPlasmaChannel))
    if rec.extra_raman:
        components = (SpRamanComponent * len(rec.extra_raman))()
        for i, comp in enumerate(rec.extra_raman):
            c = components[i]
            c.terms = comp.undamped.shape[0]
            c.undamped = m.f64(comp.undamped)
            for j, t in enumerate(comp.rates[:4]):
                c.rates[j] = m.table(t)
            c.fraction = comp.fraction
            c.density = m.table(comp.density)
            c.tensor_weights = m.f64(comp.tensor_weights)
        m.keep.append(components)
        d.n_extra_raman = len(rec.extra_raman)
        d.extra_raman = C.cast(components, C.POINTER(SpRamanComponent))
    return d, m


def run_desc(rec, policy: dict, *, field0=None, schedule=None) -> tuple[SpRunDesc, Marshalled]:
    """The C run descriptor from a march policy dict (``MarchPolicy`` / ``RungeKuttaPolicy``)."""
    m = Marshalled()
    r = SpRunDesc()
    adams = policy.get("march", "HostAdamsMarch") == "HostAdamsMarch"
    r.method = 0 if adams else 1
    r.field0 = m.c128(rec.launch_field() if field0 is None else field0)
    r.z_start = 0.0
    r.proposal = float(policy["proposal"])
    control = policy.get("controller", policy)
    r.rtol, r.atol = float(control["rtol"]), float(control["atol"])
    r.dz_min, r.dz_max = float(policy["dz_min"]), float(policy["dz_max"])
    r.stretch, r.z_end = float(policy["stretch"]), float(policy["z_end"])
    planes = np.asarray(policy.get("save_planes", []), dtype=np.float64)
    kinks = np.asarray(policy.get("hard_kinks", []), dtype=np.float64)
    edges = np.asarray(policy.get("breakpoints", [0.0, r.z_end]), dtype=np.float64)
    r.save_planes, r.n_save_planes = m.f64(planes), planes.size
    r.hard_kinks, r.n_hard_kinks = m.f64(kinks), kinks.size
    r.breakpoints, r.n_breakpoints = m.f64(edges), edges.size
    if schedule is not None:
        steps = np.asarray(schedule, dtype=np.float64)
        r.schedule, r.n_schedule = m.f64(steps), steps.size
    if adams:
        r.order = int(policy["order"])
        r.variable_order = int(policy["variable_order"])
        r.restart_after = int(policy["restart_after"])
        r.equal_approach = int(policy["equal_approach"])
        r.safety = float(policy["safety"])
        r.max_growth = float(policy["max_growth"])
        r.min_factor = float(policy["min_factor"])
        r.rejection_growth = float(policy["rejection_growth"])
        r.hysteresis = float(policy["hysteresis"])
        r.collar_stability = float(policy["collar_stability"])
        r.collar_rate = float(policy["collar_rate"])
        for i, v in enumerate(policy["real_intervals"][:8]):
            r.real_intervals[i] = float(v)
    else:
        r.safety = float(control["safety"])
        r.min_factor = float(control["min_factor"])
        r.max_factor = float(control["max_factor"])
        r.beta1, r.beta2 = float(control["beta1"]), float(control["beta2"])
        r.lag = int(control["lag"])
        r.estimator_order = int(control["estimator_order"])
        r.auto_init = int(bool(policy.get("auto_init", False)))
        r.start_growth = float(policy.get("start_growth", 100.0))
    return r, m


class Problem:
    """A problem owned by the library (``sp_problem``)."""

    def __init__(self, rec):
        self.handle = None
        self._lib = library()
        lib = library()
        self.record = rec
        desc, self._keep = problem_desc(rec)
        handle = C.c_void_p()
        check(lib.sp_problem_create(C.byref(desc), C.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sp_problem_destroy(self.handle)
            self.handle = None

    __del__ = close


PRECISIONS = {"fp64": 0, "mixed": 1}


def precision_code(precision: str) -> int:
    """``SP_PRECISION_*`` of a precision name: "fp64" (the plain form) or "mixed"."""
    try:
        return PRECISIONS[precision]
    except KeyError:
        raise ValueError(f"unknown precision {precision!r}; expected one of {sorted(PRECISIONS)}") from None


class Workspace:
    """Device buffers of one problem (``sp_workspace``; native ``_core.Workspace``)."""

    MODAL = {"auto": 0, "fused": 1, "gemm": 2}

    def __init__(self, problem: Problem, device: int = 0, precision: str = "fp64", modal: str = "auto"):
        """``modal``: the modal transform inside the response column ("fused", up to 8
        columns), as dense products ("gemm": FP64 products, or tcgen05 products of
        three-part BF16 splits in the mixed form), or "auto" (fused up to 8 columns)."""
        self.handle = None
        self._lib = library()
        self.problem = problem
        self.precision = precision
        if modal not in self.MODAL:
            raise ValueError(f"modal transform {modal!r}: expected one of {sorted(self.MODAL)}")
        handle = C.c_void_p()
        check(library().sp_workspace_create_ex2(problem.handle, device, precision_code(precision),
                                                self.MODAL[modal], C.byref(handle)))
        self.handle = handle
        self.shape = (problem.record.n_modes, problem.record.n_pol, problem.record.n_omega)

    def source(self, lab: np.ndarray, z: float, quiet: bool = False) -> np.ndarray:
        """One source evaluation at a lab-frame field (numpy_ref ``lab_source``)."""
        lab = np.ascontiguousarray(np.broadcast_to(lab, self.shape), dtype=np.complex128)
        out = np.empty(self.shape, dtype=np.complex128)
        check(library().sp_workspace_source(
            self.handle, lab.ctypes.data_as(C.POINTER(C.c_double)), float(z), int(quiet),
            out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def source_device(self, lab_ptr: int, z: float, out_ptr: int, quiet: bool = False) -> None:
        check(library().sp_workspace_source_device(self.handle, C.c_void_p(lab_ptr), float(z),
                                                   int(quiet), C.c_void_p(out_ptr)))

    @property
    def stream(self) -> int:
        """The ``cudaStream_t`` of every launch of this workspace, as an integer."""
        return int(library().sp_workspace_stream(self.handle) or 0)

    @property
    def launches_per_source(self) -> int:
        return int(library().sp_workspace_launches_per_source(self.handle))

    def start(self, policy: dict, *, field0=None, schedule=None) -> "Session":
        return Session(self, policy, field0=field0, schedule=schedule)

    def restore(self, policy: dict, snapshot: bytes, *, schedule=None) -> "Session":
        """A session continuing ``snapshot`` (``Session.snapshot``) under ``policy``."""
        return Session(self, policy, schedule=schedule, snapshot=snapshot)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sp_workspace_destroy(self.handle)
            self.handle = None

    __del__ = close


class Session:
    """One run on a workspace (``sp_session``; native ``_core.Session``)."""

    def __init__(self, ws: Workspace, policy: dict, *, field0=None, schedule=None, snapshot=None):
        self.handle = None
        self._lib = library()
        self.ws = ws
        desc, keep = run_desc(ws.problem.record, policy, field0=field0, schedule=schedule)
        handle = C.c_void_p()
        if snapshot is None:
            check(library().sp_session_start(ws.handle, C.byref(desc), C.byref(handle)))
        else:
            check(library().sp_session_restore(ws.handle, C.byref(desc), snapshot, len(snapshot),
                                                C.byref(handle)))
        self.handle = handle
        self.batch = SpBatch()

    def advance(self, work_limit: int = 256, deadline: float = 0.0, *, rows: bool = False) -> SpBatch:
        """Step until a save plane, the end, ``work_limit`` attempts or ``deadline`` host
        seconds (0: none).  With ``rows`` the batch's ``attempt_rows`` holds one row per
        attempt of this call: end, step, norm, accepted, wall seconds."""
        b = self.batch
        if rows:
            buf = np.zeros((max(int(work_limit), 1), 5))
            b.rows = buf.ctypes.data_as(C.POINTER(C.c_double))
            b.rows_capacity = buf.shape[0]
        else:
            buf = None
            b.rows = C.POINTER(C.c_double)()
            b.rows_capacity = 0
        try:
            check(library().sp_session_advance(self.handle, int(work_limit), float(deadline),
                                               C.byref(b)))
        finally:
            b.attempt_rows = None if buf is None else buf[: b.n_rows].copy()
            b.rows = C.POINTER(C.c_double)()
            b.rows_capacity = 0
        return b

    def request_stop(self) -> None:
        """Stop at the next attempt boundary; safe from another thread."""
        check(library().sp_session_request_stop(self.handle))

    def request_snapshot(self) -> None:
        """Return at the next accepted endpoint (event "halted") for a snapshot."""
        check(library().sp_session_request_snapshot(self.handle))

    def march_state(self) -> dict:
        st = SpMarchState()
        check(library().sp_session_march_state(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in SpMarchState._fields_}

    def statistics(self, power_weight=None) -> dict:
        """The current state's plane statistics, formed on the device
        (``sp_session_statistics``)."""
        return statistics_call(
            lambda pw, out: library().sp_session_statistics(self.handle, pw, out),
            self.ws.problem.record, power_weight)

    def snapshot(self) -> bytes:
        """The run's resumable state (``Workspace.restore`` continues it)."""
        size = C.c_size_t()
        check(library().sp_session_snapshot(self.handle, None, 0, C.byref(size)))
        buf = C.create_string_buffer(size.value)
        check(library().sp_session_snapshot(self.handle, buf, size.value, C.byref(size)))
        return buf.raw[: size.value]

    def set_timing(self, enable: bool) -> None:
        check(library().sp_session_set_timing(self.handle, int(enable)))

    def timing(self, reset: bool = False) -> dict:
        """Accumulated device milliseconds and launch counts per kernel family."""
        n = len(KERNEL_NAMES)
        ms = (C.c_double * n)()
        counts = (C.c_int64 * n)()
        check(library().sp_session_timing(self.handle, ms, counts, int(reset)))
        return {name: (ms[i], counts[i]) for i, name in enumerate(KERNEL_NAMES)}

    def export(self) -> np.ndarray:
        out = np.empty(self.ws.shape, dtype=np.complex128)
        check(library().sp_session_export(self.handle, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sp_session_destroy(self.handle)
            self.handle = None

    __del__ = close


class Scan:
    """Many independent runs stepped together on one device (``sp_scan``)."""

    def __init__(self, records, policies, device: int = 0, precision: str = "fp64"):
        self.handle = None
        self._lib = library()
        self.precision = precision
        self.records = list(records)
        self.problems = [Problem(r) for r in self.records]
        descs, self._keep = [], []
        for rec, pol in zip(self.records, policies):
            d, k = run_desc(rec, pol)
            descs.append(d)
            self._keep.append(k)
        n = len(descs)
        handles = (C.c_void_p * n)(*[p.handle.value for p in self.problems])
        runs = (SpRunDesc * n)(*descs)
        handle = C.c_void_p()
        check(library().sp_scan_create_ex(n, handles, runs, device, precision_code(precision),
                                          C.byref(handle)))
        self.handle = handle
        self.status = SpScanStatus()

    def describe(self) -> str:
        """The transform plan the autotuner chose, one line per grid size."""
        buf = C.create_string_buffer(8192)
        self._lib.sp_scan_describe(self.handle, buf, 8192)
        return buf.value.decode()

    COLUMN_FORMS = {"tiles": 1, "sweep": 2}

    def set_column(self, form: str) -> None:
        """Fix the response column's form: ``"tiles"`` (one CTA per tile and node group,
        the running integrals handed over between CTAs) or ``"sweep"`` (one CTA per run and
        node group walking the tiles).  The autotuner's choice stands otherwise."""
        if form not in self.COLUMN_FORMS:
            raise ValueError(f"column form {form!r}: expected one of {sorted(self.COLUMN_FORMS)}")
        check(library().sp_scan_set_column(self.handle, self.COLUMN_FORMS[form]))

    def set_alone(self, max_runs: int = 6, min_remaining: float = 2000.0, factor: float = 4.0) -> None:
        """Let runs whose remaining attempts exceed ``factor`` x the batch's median and
        ``min_remaining`` go on as single runs beside the batch (``max_runs`` at a time; 0
        keeps every run in the batch)."""
        check(library().sp_scan_set_alone(self.handle, int(max_runs), float(min_remaining), float(factor)))

    def set_transforms(self, n_to: int, inverse: int, forward: int) -> None:
        """Fix the transforms' forms for the runs with ``n_to`` fine samples: 0 for one CTA
        per row, or a cluster of 2, 4 or 8 CTAs."""
        check(library().sp_scan_set_transforms(self.handle, int(n_to), int(inverse), int(forward)))

    def advance(self, steps: int = 1) -> SpScanStatus:
        check(library().sp_scan_advance(self.handle, int(steps), C.byref(self.status)))
        return self.status

    def run(self, index: int, state: bool = True):
        rec = self.records[index]
        info = SpBatch()
        out = np.empty((rec.n_modes, rec.n_pol, rec.n_omega), dtype=np.complex128) if state else None
        ptr = out.ctypes.data_as(C.POINTER(C.c_double)) if state else C.POINTER(C.c_double)()
        check(library().sp_scan_run(self.handle, int(index), ptr, C.byref(info)))
        return out, info

    @property
    def stream(self) -> int:
        return int(library().sp_scan_stream(self.handle) or 0)

    def statistics(self, index: int, power_weight=None) -> dict:
        """Run ``index``'s plane statistics at its current state, formed on the device:
        no state leaves it (``sp_scan_statistics``)."""
        return statistics_call(
            lambda pw, out: library().sp_scan_statistics(self.handle, int(index), pw, out),
            self.records[index], power_weight)

    def set_timing(self, enable: bool) -> None:
        """Events around every batched launch family of the batch steps that follow."""
        check(library().sp_scan_set_timing(self.handle, int(enable)))

    def timing(self, reset: bool = False) -> dict:
        """Accumulated device milliseconds and launch counts per kernel family."""
        n = len(KERNEL_NAMES)
        ms = (C.c_double * n)()
        counts = (C.c_int64 * n)()
        check(library().sp_scan_timing(self.handle, ms, counts, int(reset)))
        return {name: (ms[i], counts[i]) for i, name in enumerate(KERNEL_NAMES)}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.sp_scan_destroy(self.handle)
            self.handle = None

    __del__ = close

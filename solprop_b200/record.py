"""The flat problem record: every array and scalar one run's hot path reads.

A :class:`ProblemRecord` is the lowered form of solprop's ``PropagationProblem``
(``src/solprop/translate/problem.py:465``) restricted to what the modal field and
envelope routes execute: grids and masks (``translate/masks.py:72``), the stage terms
of ``Phi`` and of the prefactor with their scalar weight tables
(``translate/stage.py:345-413``), the static synthesis and projection
(``translate/modal.py:187-191``), the compiled Kerr, plasma and Raman leaves
(``translate/responses.py:1749``) and the initial state.  It plays the part of the
native backend's ``_core.Problem`` record (``native/src/solprop_native/_core.pyi:51``):
plain NumPy arrays and scalars, with no solprop object inside, so that it can be saved
to an ``.npz`` file, rebuilt on a machine without solprop, and handed to the C ABI.

Scalar paths along z (density, the Kerr density, a plasma channel's density and
pre-ionisation, the taper scale) and the weight rows of an expansion are
:class:`PiecewiseTable` objects, the arrays of solprop's ``PiecewiseChebyshev``
(``translate/chebyshev.py:236``).
"""

from __future__ import annotations

import dataclasses
import io
import json
from dataclasses import dataclass, field

import numpy as np

__all__ = ["PiecewiseTable", "PlasmaChannelRecord", "ProblemRecord", "RamanComponentRecord", "load_record",
           "save_record"]

# Fraction of a table's span a position may lie outside it (translate/chebyshev.py,
# EDGE_SLACK_FRACTION): positions reached by summing steps arrive a few ulp off.
EDGE_SLACK_FRACTION = 1e-10


@dataclass
class PiecewiseTable:
    """A piecewise Chebyshev series in z with array values.

    On interval ``i`` the value is ``sum_j c[i, j] T_j(x)``, ``x = (2z - lo - hi) /
    (hi - lo)``, the representation of ``translate/chebyshev.py:236-300``; a position
    takes the interval ``searchsorted(edges, z, side="right") - 1`` clamped to the
    intervals (``translate/chebyshev.py:171-180``).

    Attributes
    ----------
    breakpoints : numpy.ndarray
        Interval edges, float64, shape ``(n_intervals + 1,)``.
    coefficients : numpy.ndarray
        Coefficients, float64, shape ``(n_intervals, n_deg, n_values)``.
    """

    breakpoints: np.ndarray
    coefficients: np.ndarray

    def __post_init__(self) -> None:
        self.breakpoints = np.ascontiguousarray(self.breakpoints, dtype=np.float64)
        c = np.asarray(self.coefficients, dtype=np.float64)
        if c.ndim == 2:
            c = c[:, :, None]
        self.coefficients = np.ascontiguousarray(c.reshape(c.shape[0], c.shape[1], -1))

    @classmethod
    def constant(cls, value: float | np.ndarray, z0: float, z1: float) -> PiecewiseTable:
        values = np.atleast_1d(np.asarray(value, dtype=np.float64))
        return cls(np.array([z0, z1]), values.reshape(1, 1, -1))

    @property
    def n_values(self) -> int:
        return int(self.coefficients.shape[2])

    def interval(self, z: float) -> int:
        edges = self.breakpoints
        k = int(np.searchsorted(edges, z, side="right")) - 1
        return min(max(k, 0), edges.shape[0] - 2)

    def __call__(self, z: float) -> np.ndarray:
        """Evaluate by the Clenshaw recursion of ``chebval`` (chebyshev.py:178-198)."""
        k = self.interval(z)
        lo, hi = self.breakpoints[k], self.breakpoints[k + 1]
        x = (2.0 * z - lo - hi) / (hi - lo)
        c = self.coefficients[k]
        n = c.shape[0]
        if n == 1:
            return c[0] + 0.0 * x
        if n == 2:
            return c[0] + c[1] * x
        x2 = 2.0 * x
        c0 = c[n - 2].copy()
        c1 = c[n - 1].copy()
        for i in range(3, n + 1):
            tmp = c0
            c0 = c[n - i] - c1
            c1 = tmp + c1 * x2
        return c0 + c1 * x

    def derivative(self) -> PiecewiseTable:
        """Return the table of d/dz, interval by interval (Chebyshev derivative)."""
        n_int, n_deg, n_val = self.coefficients.shape
        out = np.zeros((n_int, max(n_deg - 1, 1), n_val))
        for k in range(n_int):
            lo, hi = self.breakpoints[k], self.breakpoints[k + 1]
            scale = 2.0 / (hi - lo)
            for j in range(n_val):
                d = np.polynomial.chebyshev.chebder(self.coefficients[k, :, j])
                if d.size == 0:
                    d = np.zeros(1)
                out[k, : d.size, j] = d * scale
        return PiecewiseTable(self.breakpoints.copy(), out)


@dataclass
class PlasmaChannelRecord:
    """A further field-plasma channel of a gas mixture (``passes/plasma.py:326-485``): its
    own rate table (``translate/ionisation.py:242-323``), population and path tables."""

    charge_mass_ratio: float  # times the electrons per event
    ionisation_potential: float
    rate_coefficients: np.ndarray  # (4, n_intervals)
    log_field_min: float
    d_log_field: float
    field_min: float
    field_max: float
    rate_max: float
    plasma_density: PiecewiseTable | None = None
    preionisation: PiecewiseTable | None = None


@dataclass
class RamanComponentRecord:
    """A further Raman-active component of a gas mixture (``passes/responses.py:293-334``):
    rows damped at their own rates, weighted by the fraction and the density."""

    undamped: np.ndarray  # (n_terms, 2 n_to)
    rates: list[PiecewiseTable]
    fraction: float = 1.0
    density: PiecewiseTable | None = None
    tensor_weights: np.ndarray | None = None  # (n_terms, 2), two components only


@dataclass
class ProblemRecord:
    """One trajectory's lowered problem (see the module docstring).

    Array shapes use ``n_cols = n_modes * n_pol`` for the state's columns and
    ``n_rows = n_nodes * n_pol_transform`` for the synthesis rows.
    """

    # ---- dimensions and grid (kernel-contract.md sections 1-2)
    grid_kind: str  # "field" | "envelope"
    n_modes: int
    n_pol: int
    n_omega: int
    n_t: int
    n_to: int
    n_nodes: int
    n_pol_transform: int
    omega0: float
    dt: float
    dt_fine: float
    pad_scale: float
    crop_scale: float
    z_end: float
    omega: np.ndarray
    crop_index: np.ndarray
    active_mask: np.ndarray
    norm_mask: np.ndarray
    omega_window: np.ndarray
    t_window: np.ndarray
    t_window_derivative: np.ndarray
    carrier: np.ndarray | None = None
    # ---- linear operator and prefactor as stage terms (stage.py:345-411)
    phi_representation: str = "constant"  # "constant" | "expansion"
    phi_terms: np.ndarray | None = None  # (n_phi, n_modes, n_pol, n_omega) c128
    phi_weights: PiecewiseTable | None = None  # expansion: Phi(z) weights
    phi_rate: PiecewiseTable | None = None  # expansion: D(z) = dPhi/dz weights
    hard_kinks: np.ndarray = field(default_factory=lambda: np.zeros(0))
    breakpoints: np.ndarray = field(default_factory=lambda: np.zeros(0))
    prefactor_terms: np.ndarray | None = None  # (n_pre, n_modes, n_pol, n_omega) c128
    prefactor_weights: PiecewiseTable | None = None  # expansion only
    # ---- scalar paths along z
    density: PiecewiseTable | None = None
    kerr_density: PiecewiseTable | None = None
    plasma_density: PiecewiseTable | None = None
    preionisation: PiecewiseTable | None = None
    taper_scale: PiecewiseTable | None = None
    # ---- transform (kernel-contract.md section 4)
    synthesis: np.ndarray | None = None
    projection: np.ndarray | None = None
    projection_coarse: np.ndarray | None = None
    # ---- Kerr (translate/responses.py:235-275)
    kerr_enabled: bool = False
    kerr_coefficient: float = 0.0
    kerr_form: str = "real"  # "real" | "analytic"
    kerr_self: float = 0.0
    kerr_conjugate: float = 0.0
    kerr_harmonic: float = 0.0
    kerr_analytic_signal: bool = False
    kerr_take_real: bool = True
    # ---- plasma (translate/ionisation.py:95-323; nonlinear/ionisation.py:410-675)
    plasma_enabled: bool = False
    charge_mass_ratio: float = 0.0
    ionisation_potential: float = 0.0
    rate_coefficients: np.ndarray | None = None  # (4, n_intervals)
    log_field_min: float = 0.0
    d_log_field: float = 1.0
    field_min: float = 0.0
    field_max: float = 0.0
    rate_max: float = 0.0
    integral_policy: str = "trapezoid"  # "band" | "trapezoid"
    taps: np.ndarray = field(default_factory=lambda: np.ones(1))
    # ---- Raman (translate/raman.py; kernel-contract.md section 5)
    raman_enabled: bool = False
    raman_undamped: np.ndarray | None = None  # (n_terms, 2 n_to)
    raman_rates: list[PiecewiseTable] = field(default_factory=list)
    raman_fraction: float = 1.0
    raman_thg: bool = False
    raman_density: PiecewiseTable | None = None
    raman_tensor_weights: np.ndarray | None = None  # (n_terms, 2): trace, traceless (two components)
    # ---- a gas mixture: the plasma channels and Raman components after the first
    extra_channels: list[PlasmaChannelRecord] = field(default_factory=list)
    extra_raman: list[RamanComponentRecord] = field(default_factory=list)
    # ---- temporal absorber (stepping.py:286-369)
    absorber_scheme: str = "none"  # "nonlinear" | "split_step" | "none"
    temporal_absorber_fine: np.ndarray | None = None
    temporal_absorber: np.ndarray | None = None
    # ---- initial state (kernel-contract.md section 6)
    field0: np.ndarray | None = None
    noise0: np.ndarray | None = None
    noise_model: str = "none"  # "input": added to the launch field; "modified": every stage

    def launch_field(self) -> np.ndarray:
        """The state a run starts from: ``field0``, plus the ``input`` noise draw
        (``backends/numpy_ref/workspace.py:260-306``); the device masks it to the band."""
        field = np.broadcast_to(self.field0, (self.n_modes, self.n_pol, self.n_omega))
        if self.noise0 is not None and self.noise_model == "input":
            return field + self.noise0
        return np.array(field)

    @property
    def n_cols(self) -> int:
        return self.n_modes * self.n_pol

    @property
    def n_omega_fine(self) -> int:
        return self.n_to // 2 + 1 if self.grid_kind == "field" else self.n_to

    @property
    def n_phi_terms(self) -> int:
        return 0 if self.phi_terms is None else int(self.phi_terms.shape[0])

    @property
    def n_prefactor_terms(self) -> int:
        return 0 if self.prefactor_terms is None else int(self.prefactor_terms.shape[0])

    # ---------------------------------------------------------------- stage scalars
    def phi_delta_weights(self, z0: float, z1: float) -> np.ndarray:
        """Weights of ``Phi(z1) - Phi(z0)`` (``translate/stage.py:709-742``)."""
        if self.phi_representation == "constant":
            return np.array([z1 - z0])
        assert self.phi_weights is not None
        return self.phi_weights(z1) - self.phi_weights(z0)

    def phi_rate_weights(self, z: float, before: bool = False) -> np.ndarray:
        """Weights of ``D(z) = dPhi/dz`` (``translate/linop.py:2286-2423``).

        A position on an interval edge reads the interval starting there unless
        ``before`` asks for the one ending there (``linop.py:2402-2405``).
        """
        if self.phi_representation == "constant":
            return np.array([1.0])
        table = self.phi_rate if self.phi_rate is not None else self.phi_weights.derivative()
        k = table.interval(z)
        if before and k > 0 and z <= table.breakpoints[k]:
            k -= 1
        lo, hi = table.breakpoints[k], table.breakpoints[k + 1]
        one = PiecewiseTable(np.array([lo, hi]), table.coefficients[k:k + 1])
        return one(z)

    def prefactor_weights_at(self, z: float) -> np.ndarray:
        """Weights of the prefactor at ``z`` (``translate/stage.py:745-761``)."""
        if self.prefactor_weights is None:
            return np.array([1.0])
        return self.prefactor_weights(z)

    def scalar(self, table: PiecewiseTable | None, z: float, default: float) -> float:
        return default if table is None else float(table(z)[0])


def _table_arrays(prefix: str, table: PiecewiseTable | None, out: dict) -> None:
    if table is not None:
        out[f"{prefix}.bp"] = table.breakpoints
        out[f"{prefix}.c"] = table.coefficients


_CHANNEL_SCALARS = ("charge_mass_ratio", "ionisation_potential", "log_field_min", "d_log_field",
                    "field_min", "field_max", "rate_max")


def _read_table(data, names, prefix: str) -> PiecewiseTable | None:
    if f"{prefix}.bp" not in names:
        return None
    return PiecewiseTable(np.array(data[f"{prefix}.bp"]), np.array(data[f"{prefix}.c"]))


def save_record(record: ProblemRecord, path) -> None:
    """Write a record to an ``.npz`` file: arrays by name, scalars as one JSON entry."""
    arrays: dict[str, np.ndarray] = {}
    meta: dict[str, object] = {}
    for f in dataclasses.fields(record):
        value = getattr(record, f.name)
        if isinstance(value, PiecewiseTable):
            _table_arrays(f.name, value, arrays)
        elif f.name == "raman_rates":
            for i, table in enumerate(value):
                _table_arrays(f"raman_rates.{i}", table, arrays)
            meta["n_raman_rates"] = len(value)
        elif f.name == "extra_channels":
            scalars = []
            for i, ch in enumerate(value):
                arrays[f"extra_channels.{i}.rate_coefficients"] = ch.rate_coefficients
                _table_arrays(f"extra_channels.{i}.plasma_density", ch.plasma_density, arrays)
                _table_arrays(f"extra_channels.{i}.preionisation", ch.preionisation, arrays)
                scalars.append({k: getattr(ch, k) for k in _CHANNEL_SCALARS})
            meta["extra_channels"] = scalars
        elif f.name == "extra_raman":
            scalars = []
            for i, comp in enumerate(value):
                arrays[f"extra_raman.{i}.undamped"] = comp.undamped
                if comp.tensor_weights is not None:
                    arrays[f"extra_raman.{i}.tensor_weights"] = comp.tensor_weights
                for j, table in enumerate(comp.rates):
                    _table_arrays(f"extra_raman.{i}.rates.{j}", table, arrays)
                _table_arrays(f"extra_raman.{i}.density", comp.density, arrays)
                scalars.append({"fraction": comp.fraction, "n_rates": len(comp.rates)})
            meta["extra_raman"] = scalars
        elif isinstance(value, np.ndarray):
            arrays[f.name] = value
        elif value is None:
            continue
        else:
            meta[f.name] = value
    arrays["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrays)


def load_record(path) -> ProblemRecord:
    """Read a record :func:`save_record` wrote."""
    data = np.load(path) if not isinstance(path, dict) else path
    meta = json.loads(bytes(data["__meta__"]).decode())
    kwargs: dict[str, object] = {}
    names = set(data.keys()) if isinstance(data, dict) else set(data.files)
    n_rates = int(meta.pop("n_raman_rates", 0))
    channels = meta.pop("extra_channels", [])
    components = meta.pop("extra_raman", [])
    for f in dataclasses.fields(ProblemRecord):
        if f.name in meta:
            kwargs[f.name] = meta[f.name]
        elif f.name in names:
            kwargs[f.name] = np.array(data[f.name])
        elif f"{f.name}.bp" in names:
            kwargs[f.name] = PiecewiseTable(
                np.array(data[f"{f.name}.bp"]), np.array(data[f"{f.name}.c"])
            )
    kwargs["raman_rates"] = [
        PiecewiseTable(np.array(data[f"raman_rates.{i}.bp"]), np.array(data[f"raman_rates.{i}.c"]))
        for i in range(n_rates)
    ]
    kwargs["extra_channels"] = [
        PlasmaChannelRecord(
            rate_coefficients=np.array(data[f"extra_channels.{i}.rate_coefficients"]),
            plasma_density=_read_table(data, names, f"extra_channels.{i}.plasma_density"),
            preionisation=_read_table(data, names, f"extra_channels.{i}.preionisation"),
            **scalars,
        )
        for i, scalars in enumerate(channels)
    ]
    kwargs["extra_raman"] = [
        RamanComponentRecord(
            undamped=np.array(data[f"extra_raman.{i}.undamped"]),
            rates=[_read_table(data, names, f"extra_raman.{i}.rates.{j}") for j in range(c["n_rates"])],
            fraction=float(c["fraction"]),
            density=_read_table(data, names, f"extra_raman.{i}.density"),
            tensor_weights=(np.array(data[f"extra_raman.{i}.tensor_weights"])
                            if f"extra_raman.{i}.tensor_weights" in names else None),
        )
        for i, c in enumerate(components)
    ]
    return ProblemRecord(**kwargs)


def record_bytes(record: ProblemRecord) -> bytes:
    buf = io.BytesIO()
    save_record(record, buf)
    return buf.getvalue()

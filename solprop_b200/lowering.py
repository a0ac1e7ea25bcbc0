"""Lower solprop's ``PropagationProblem`` into a :class:`~solprop_b200.record.ProblemRecord`.

The counterpart of the native backend's lowering (``native/src/solprop_native/
_lowering.py:334-926``), for the routes this backend executes: the modal route on a
field or envelope grid (and the radial free-space route), Kerr, the field-plasma
channels and scalar Raman components of a gas mixture (up to four of each), under a
constant or expansion representation of ``Phi`` and of the prefactor.  Anything else is
refused by name, before anything is allocated, as the contract asks
(``docs/dev/kernel-contract.md`` section 1).  solprop itself is imported by duck typing
only: the record has no solprop object inside.
"""

from __future__ import annotations

import numpy as np

from solprop_b200.record import PiecewiseTable, PlasmaChannelRecord, ProblemRecord, RamanComponentRecord

__all__ = ["BackendRefusal", "lower"]


class BackendRefusal(Exception):
    """A problem this backend does not execute, refused by name before allocation."""


def _table(chebyshev) -> PiecewiseTable | None:
    if chebyshev is None:
        return None
    return PiecewiseTable(
        np.asarray(chebyshev.breakpoints, dtype=np.float64),
        np.asarray(chebyshev.coefficients, dtype=np.float64),
    )


def lower(problem) -> ProblemRecord:
    """Return the record of a validated ``PropagationProblem``.

    Raises
    ------
    BackendRefusal
        Naming the part of the problem this backend does not step.
    """
    grids, linear, transform = problem.grids, problem.linear, problem.transform
    responses, initial = problem.responses, problem.initial
    n_modes, n_pol, n_omega = problem.shape
    geometry = transform.geometry
    if transform.modal_tables is not None:
        raise BackendRefusal("the general modal route's tables are not lowered")
    if geometry is not None:
        # the radial free-space route is the modal route's arithmetic on a square Hankel
        # pair (its plasma projected after the nodes' transforms: the same linear maps in
        # another order, backends/numpy_ref/source.py:702-735); Cartesian, line and slab
        # grids transform in space instead, and the radial collar adds a spatial matrix
        if geometry.kind != "radial":
            raise BackendRefusal(f"route {transform.kind!r}: the modal and radial routes are lowered")
        if np.any(np.asarray(geometry.absorber_rate)):
            raise BackendRefusal("the radial spatial absorber (a spectral-space matrix) is not executed")
    if responses.temporal_absorber_fine is not None and responses.absorber_scheme != "nonlinear":
        raise BackendRefusal(
            f"the {responses.absorber_scheme!r} temporal absorber: the device march takes the "
            "in-stage (nonlinear) scheme")
    if linear.coupled_flow is not None:
        raise BackendRefusal("a coupled flow is not executed by this backend")
    if linear.phi_representation not in ("constant", "expansion"):
        raise BackendRefusal(
            f"Phi as a {linear.phi_representation!r}: a device build needs a constant "
            "or an expansion (translate/stage.py require_device_ready)"
        )
    if responses.prefactor_representation not in ("constant", "expansion"):
        raise BackendRefusal(f"prefactor as a {responses.prefactor_representation!r}")
    if responses.dispersive_kerr is not None or responses.envelope_plasma is not None:
        raise BackendRefusal("dispersive Kerr and envelope plasma are not executed")
    if len(responses.plasma_channels) > 4:
        raise BackendRefusal("more than four plasma channels")
    if len(responses.raman_terms) > 4:
        raise BackendRefusal("more than four Raman components")
    if getattr(problem.route, "tdse", None) is not None:
        raise BackendRefusal("a TDSE response is not executed by this backend")

    if linear.phi_constant is not None:
        phi_terms = np.asarray(linear.phi_constant)[np.newaxis]
        phi_weights = None
        phi_rep = "constant"
        phi_rate = None
    else:
        expansion = linear.phi_expansion
        phi_terms = np.asarray(expansion.terms)
        phi_weights = _table(expansion.weights)
        phi_rep = "expansion"
        phi_rate = _table(linear.rate)
    if responses.prefactor_constant is not None:
        pre_terms = np.asarray(responses.prefactor_constant)[np.newaxis]
        pre_weights = None
    else:
        expansion = responses.prefactor_expansion
        pre_terms = np.asarray(expansion.terms)
        pre_weights = _table(expansion.weights)

    kerr = responses.kerr_coefficients
    record = ProblemRecord(
        grid_kind=problem.grid_kind,
        n_modes=int(n_modes),
        n_pol=int(n_pol),
        n_omega=int(n_omega),
        n_t=int(grids.n_t),
        n_to=int(grids.n_to),
        n_nodes=int(transform.synthesis.shape[0] // transform._n_pol),
        n_pol_transform=int(transform._n_pol),
        omega0=float(grids.omega0),
        dt=float(grids.dt),
        dt_fine=float(grids.dt_fine),
        pad_scale=float(grids.pad_scale),
        crop_scale=float(grids.crop_scale),
        z_end=float(linear.phi_breakpoints[-1]),
        omega=np.asarray(grids.omega, dtype=np.float64),
        crop_index=np.asarray(grids.crop_index, dtype=np.int64),
        active_mask=np.asarray(grids.active_mask, dtype=bool),
        norm_mask=np.asarray(grids.norm_mask, dtype=bool),
        omega_window=np.asarray(grids.omega_window, dtype=np.float64),
        t_window=np.asarray(grids.t_window_fine, dtype=np.float64),
        t_window_derivative=np.asarray(grids.t_window_fine_derivative, dtype=np.float64),
        carrier=None if grids.carrier_2w0 is None else np.asarray(grids.carrier_2w0),
        phi_representation=phi_rep,
        phi_terms=np.ascontiguousarray(phi_terms, dtype=np.complex128),
        phi_weights=phi_weights,
        phi_rate=phi_rate,
        hard_kinks=np.asarray(linear.hard_kinks, dtype=np.float64),
        breakpoints=np.asarray(linear.phi_breakpoints, dtype=np.float64),
        prefactor_terms=np.ascontiguousarray(pre_terms, dtype=np.complex128),
        prefactor_weights=pre_weights,
        density=_table(responses.density),
        taper_scale=_table(transform.taper_scale),
        synthesis=np.ascontiguousarray(transform.synthesis, dtype=np.float64),
        projection=np.ascontiguousarray(transform.projection, dtype=np.float64),
        projection_coarse=np.ascontiguousarray(transform.projection_coarse, dtype=np.float64),
        absorber_scheme=(
            "none" if responses.temporal_absorber_fine is None else responses.absorber_scheme
        ),
        temporal_absorber_fine=None
        if responses.temporal_absorber_fine is None
        else np.asarray(responses.temporal_absorber_fine, dtype=np.float64),
        temporal_absorber=None
        if responses.temporal_absorber is None
        else np.asarray(responses.temporal_absorber, dtype=np.float64),
        field0=np.ascontiguousarray(np.broadcast_to(initial.field0, problem.shape), dtype=np.complex128),
        noise0=None if initial.noise0 is None else np.asarray(initial.noise0, dtype=np.complex128),
        noise_model=str(getattr(initial, "noise_model", "none") or "none"),
    )
    if record.noise0 is not None and record.noise_model == "modified":
        raise BackendRefusal("the modified noise model (a draw added at every stage)")
    if np.iscomplexobj(transform.synthesis):
        raise BackendRefusal("a complex synthesis matrix")
    if kerr is not None:
        record.kerr_enabled = True
        record.kerr_coefficient = float(kerr.coefficient)
        record.kerr_form = str(kerr.cubic_form)
        record.kerr_self = float(kerr.self_factor)
        record.kerr_conjugate = float(kerr.conjugate_factor)
        record.kerr_harmonic = float(kerr.harmonic_factor)
        record.kerr_analytic_signal = bool(kerr.analytic_signal)
        record.kerr_take_real = bool(kerr.take_real)
        record.kerr_density = _table(kerr.density) if kerr.density is not None else None
        if kerr.analytic_signal:
            raise BackendRefusal("the analytic-signal Kerr form on a field grid")
    if responses.plasma_channels:
        channel = responses.plasma_channels[0]
        table = channel.rate
        integral = responses.plasma_integral
        record.plasma_enabled = True
        record.charge_mass_ratio = float(channel.charge_mass_ratio * channel.electrons_per_event)
        record.ionisation_potential = float(channel.ionisation_potential)
        record.rate_coefficients = np.ascontiguousarray(table.coefficients, dtype=np.float64)
        record.log_field_min = float(table.log_field_min)
        record.d_log_field = float(table.d_log_field)
        record.field_min = float(table.field_min)
        record.field_max = float(table.field_max)
        record.rate_max = float(table.rate_max)
        record.integral_policy = str(integral.policy)
        record.taps = np.asarray(integral.taps, dtype=np.float64)
        record.plasma_density = _table(channel.density)
        record.preionisation = _table(channel.preionisation)
        if problem.grid_kind != "field":
            raise BackendRefusal("field plasma on an envelope grid")
    if responses.raman_terms:
        term = responses.raman_terms[0]
        record.raman_enabled = True
        record.raman_undamped = np.ascontiguousarray(term.undamped, dtype=np.float64)
        record.raman_rates = [_table(t) for t in term.decay_rates]
        record.raman_fraction = float(term.fraction)
        record.raman_thg = bool(term.thg)
        record.raman_density = _table(term.density) if term.density is not None else None
        if n_pol != 1:
            raise BackendRefusal("a state with two polarisation columns is not executed")
        if transform._n_pol == 2:  # two Cartesian components: the tensor response
            if not all(t.tensor_capable for t in responses.raman_terms):
                raise BackendRefusal("vector Raman needs tensor-capable Raman components")
            record.raman_tensor_weights = np.ascontiguousarray(term.tensor_weights, dtype=np.float64)
        for term in responses.raman_terms:
            if len(term.decay_rates) > 4:
                raise BackendRefusal("a Raman component with more than four damped rows")
        for term in responses.raman_terms[1:]:
            if bool(term.thg) != record.raman_thg:
                raise BackendRefusal("Raman components with different drives")
            record.extra_raman.append(RamanComponentRecord(
                undamped=np.ascontiguousarray(term.undamped, dtype=np.float64),
                rates=[_table(t) for t in term.decay_rates],
                fraction=float(term.fraction),
                density=_table(term.density) if term.density is not None else None,
                tensor_weights=(np.ascontiguousarray(term.tensor_weights, dtype=np.float64)
                                if transform._n_pol == 2 else None),
            ))
    for channel in responses.plasma_channels[1:]:
        table = channel.rate
        record.extra_channels.append(PlasmaChannelRecord(
            charge_mass_ratio=float(channel.charge_mass_ratio * channel.electrons_per_event),
            ionisation_potential=float(channel.ionisation_potential),
            rate_coefficients=np.ascontiguousarray(table.coefficients, dtype=np.float64),
            log_field_min=float(table.log_field_min),
            d_log_field=float(table.d_log_field),
            field_min=float(table.field_min),
            field_max=float(table.field_max),
            rate_max=float(table.rate_max),
            plasma_density=_table(channel.density),
            preionisation=_table(channel.preionisation),
        ))
    return record

"""One source evaluation of the modal route, restated from the reference's passes.

The pipeline of ``backends/numpy_ref/source.py:204-300`` (``StageSource.evaluate``) and
``source.py:599-700`` (``_over_nodes``) on a :class:`solprop_b200.record.ProblemRecord`:
inverse transform, synthesis, the fused response column (ionisation rate, plasma scans
and currents, Kerr, Raman), projection, forward transform and crop, the held plasma
assembly, the in-stage absorber and the stage output.  Test infrastructure (see the
package docstring).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.fft

EPS0 = 8.8541878188e-12  # solprop.constants.EPS0 (CODATA 2022)

__all__ = ["StageScalars", "lab_source", "stage_scalars"]


@dataclass
class StageScalars:
    """The host floats of one stage (``translate/stage.py:170-290``, a subset)."""

    z0: float
    z1: float
    phi_delta: np.ndarray
    prefactor: np.ndarray
    density: float
    taper: float
    kerr_density: float
    plasma_density: float
    preionisation: float
    raman_rates: tuple
    raman_density: float
    channel_densities: tuple = ()  # every plasma channel of a mixture, in order
    channel_preionisation: tuple = ()
    raman_rates_by_component: tuple = ()  # every Raman component's rates, in order
    raman_densities: tuple = ()


def stage_scalars(rec, z0: float, z1: float) -> StageScalars:
    """``translate/stage.py:413-503`` (``scalars``) on the lowered tables."""
    density = rec.scalar(rec.density, z1, 1.0)
    return StageScalars(
        z0=z0,
        z1=z1,
        phi_delta=rec.phi_delta_weights(z0, z1),
        prefactor=rec.prefactor_weights_at(z1),
        density=density,
        taper=rec.scalar(rec.taper_scale, z1, 1.0),
        kerr_density=density if rec.kerr_density is None else rec.scalar(rec.kerr_density, z1, 1.0),
        plasma_density=rec.scalar(rec.plasma_density, z1, density),
        preionisation=rec.scalar(rec.preionisation, z1, 0.0),
        raman_rates=tuple(float(t(z1)[0]) for t in rec.raman_rates),
        raman_density=density if rec.raman_density is None else rec.scalar(rec.raman_density, z1, 1.0),
        channel_densities=tuple(rec.scalar(ch.plasma_density, z1, density) for ch in rec.extra_channels),
        channel_preionisation=tuple(rec.scalar(ch.preionisation, z1, 0.0) for ch in rec.extra_channels),
        raman_rates_by_component=tuple(tuple(float(t(z1)[0]) for t in comp.rates) for comp in rec.extra_raman),
        raman_densities=tuple(density if comp.density is None else rec.scalar(comp.density, z1, 1.0)
                              for comp in rec.extra_raman),
    )


def combine(weights: np.ndarray, terms: np.ndarray) -> np.ndarray:
    """``translate/stage.py:292-342``: one term is multiplied, several contracted."""
    if terms.shape[0] == 1:
        return terms[0] if weights[0] == 1.0 else weights[0] * terms[0]
    return np.tensordot(weights, terms, axes=1)


# ------------------------------------------------------------------- transforms
def to_time(rec, spectrum: np.ndarray) -> np.ndarray:
    """``passes/transforms.py:31-84``: pad at ``crop_index``, inverse transform, no scale."""
    n_cols = rec.n_cols
    fine = np.zeros((n_cols, rec.n_omega_fine), dtype=np.complex128)
    fine[:, rec.crop_index] = spectrum.reshape(n_cols, -1)
    if rec.grid_kind == "field":
        out = scipy.fft.irfft(fine, n=rec.n_to, axis=-1)
    else:
        out = scipy.fft.ifft(fine, axis=-1)
    return out.reshape(rec.n_modes, rec.n_pol, rec.n_to)


def to_frequency(rec, samples: np.ndarray) -> np.ndarray:
    """``passes/transforms.py:190-233``: forward transform and crop, no scale."""
    flat = samples.reshape(-1, rec.n_to)
    if rec.grid_kind == "field":
        spec = scipy.fft.rfft(flat, axis=-1)
    else:
        spec = scipy.fft.fft(flat, axis=-1)
    return spec[:, rec.crop_index].reshape(*samples.shape[:-1], -1)


def synthesise(rec, modal_t: np.ndarray, taper: float) -> np.ndarray:
    """``passes/transforms.py:87-139``: ``E[i,p,t] = tau sum_m S[i n_pol + p, m] a[m,t]``."""
    scaled = rec.synthesis * taper
    nodes = np.tensordot(scaled, modal_t, axes=([1], [0]))
    n_rows, n_pol_state, n_to = nodes.shape
    npt = rec.n_pol_transform
    return nodes.reshape(n_rows // npt, npt * n_pol_state, n_to)


def project(rec, node_values: np.ndarray, taper: float) -> np.ndarray:
    """``passes/transforms.py:142-187``: ``P[m,t] = sum W[m, i n_pol + p] P[i,p,t] / tau``."""
    n_chunk, n_pol_node, n_to = node_values.shape
    npt = rec.n_pol_transform
    rows = node_values.reshape(n_chunk * npt, n_pol_node // npt, n_to)
    return np.tensordot(rec.projection / taper, rows, axes=([1], [0]))


# ------------------------------------------------------------------- the plasma column
def magnitude(field_t: np.ndarray) -> np.ndarray:
    """``passes/plasma.py:621-631``: ``|E|``, or ``hypot`` of two components."""
    if field_t.shape[-2] == 1:
        return np.abs(field_t[..., 0, :])
    return np.hypot(field_t[..., 0, :], field_t[..., 1, :])


def rate_lookup(rec, field_amplitude: np.ndarray) -> np.ndarray:
    """``translate/ionisation.py:242-323``: exp of a cubic in ``log|E|`` on uniform knots.

    Exactly zero below ``field_min`` and ``rate_max`` above ``field_max``.  ``rec`` is the
    record (its first channel's table) or a further channel's record.
    """
    flat = np.abs(field_amplitude).ravel()
    rate = np.zeros_like(flat)
    above = flat > rec.field_max
    inside = (flat >= rec.field_min) & ~above
    if np.any(inside):
        lf = np.log(flat[inside])
        c = rec.rate_coefficients
        index = np.clip(((lf - rec.log_field_min) / rec.d_log_field).astype(np.intp), 0, c.shape[1] - 1)
        local = lf - (rec.log_field_min + index * rec.d_log_field)
        log_rate = ((c[0, index] * local + c[1, index]) * local + c[2, index]) * local + c[3, index]
        rate[inside] = np.exp(log_rate)
    rate[above] = rec.rate_max
    return rate.reshape(field_amplitude.shape)


def band_filter(rec, values: np.ndarray) -> np.ndarray:
    """``nonlinear/ionisation.py:612-653``: symmetric taps, point-reflected ends.

    Centre first, then each pair ``y[n-k] + y[n+k]`` added before it is weighted.
    """
    taps = rec.taps
    half = taps.size - 1
    n = values.shape[-1]
    reach = np.arange(half, 0, -1)
    head = 2.0 * values[..., :1] - values[..., reach]
    tail = 2.0 * values[..., -1:] - values[..., n - 1 - reach[::-1]]
    ext = np.concatenate([head, values, tail], axis=-1)
    out = taps[0] * values
    for k in range(1, half + 1):
        out = out + taps[k] * (ext[..., half - k: half - k + n] + ext[..., half + k: half + k + n])
    return out


def running_integral(rec, values: np.ndarray, dt: float) -> np.ndarray:
    """``nonlinear/ionisation.py:566-610``: cumulative trapezoid of the filtered values.

    The trapezoid is scipy's ``cumulative_trapezoid(dx=dt, initial=0)``: the running
    sum of ``dt * (y[n] + y[n+1]) / 2``.
    """
    y = band_filter(rec, values) if (rec.integral_policy == "band" and rec.taps.size > 1) else values
    inc = dt * (y[..., 1:] + y[..., :-1]) / 2.0
    out = np.zeros_like(y)
    out[..., 1:] = np.cumsum(inc, axis=-1)
    return out


def floor(rec, exposure: np.ndarray) -> np.ndarray:
    """``nonlinear/ionisation.py:655-675``: floor at zero under the band rule."""
    return exposure if rec.integral_policy == "trapezoid" else np.maximum(exposure, 0.0)


def plasma_column(rec, field_t: np.ndarray, sc: StageScalars):
    """``passes/plasma.py:104-191`` and ``:280-323``: rate, fraction, free and total current.

    Returns the rate, the fraction and the ungated total current ``rho J``.
    """
    dt = rec.dt_fine
    mag = magnitude(field_t)
    rate = rate_lookup(rec, mag)
    exposure = floor(rec, running_integral(rec, rate, dt))
    fraction = 1.0 - (1.0 - sc.preionisation) * np.exp(-exposure)
    integrand = fraction[..., None, :] * rec.charge_mass_ratio * field_t
    free = running_integral(rec, integrand, dt)
    squared = mag ** 2
    scale = np.zeros_like(squared)
    np.divide(rec.ionisation_potential * rate * (1.0 - fraction), squared, out=scale,
              where=(rate > 0.0) & (squared > 0.0))
    current = sc.plasma_density * (free + scale[..., None, :] * field_t)
    return rate, fraction, current


def channels_current(rec, field_t: np.ndarray, sc: StageScalars) -> np.ndarray:
    """``passes/plasma.py:326-372`` and ``:426-485``: a mixture's channels, each with its own
    rate and exposure scan, their weights summed before the one free-current integral.

    Returns the ungated total current, the channel densities inside.
    """
    dt = rec.dt_fine
    mag = magnitude(field_t)
    channels = [rec, *rec.extra_channels]
    densities = (sc.plasma_density, *sc.channel_densities)
    initial = (sc.preionisation, *sc.channel_preionisation)
    weight = np.zeros_like(mag)
    work = np.zeros_like(mag)
    for channel, density, f0 in zip(channels, densities, initial):
        rate = rate_lookup(channel, mag)
        exposure = floor(rec, running_integral(rec, rate, dt))
        fraction = 1.0 - (1.0 - f0) * np.exp(-exposure)
        weight += density * fraction * channel.charge_mass_ratio
        work += density * channel.ionisation_potential * rate * (1.0 - fraction)
    free = running_integral(rec, weight[..., None, :] * field_t, dt)
    squared = mag ** 2
    guard = np.zeros_like(work)
    np.divide(work, squared, out=guard, where=squared > 0.0)
    return free + guard[..., None, :] * field_t


def kerr_polarisation(rec, field_t: np.ndarray, density: float, carrier=None) -> np.ndarray:
    """``passes/responses.py:65-139``: the real or analytic cubic."""
    factor = rec.kerr_coefficient * density
    values = field_t
    if rec.kerr_form == "real":
        pol = factor * np.sum(values ** 2, axis=-2, keepdims=True) * values
    else:
        squares = np.sum(values ** 2, axis=-2, keepdims=True)
        moduli = np.sum(np.abs(values) ** 2, axis=-2, keepdims=True)
        pol = factor * (rec.kerr_self * moduli * values + rec.kerr_conjugate * squares * np.conj(values))
        if carrier is not None:
            pol = pol + factor * rec.kerr_harmonic * carrier * squares * values
    return pol.real if rec.kerr_take_real else pol


def raman_spectrum(rec, rates) -> np.ndarray:
    """``passes/responses.py:218-290``: damp each row, sum, scale, ``rfft * dt``."""
    n2 = rec.raman_undamped.shape[1]
    t = np.arange(n2) * rec.dt_fine
    kernel = np.zeros(n2)
    for row, rate in zip(rec.raman_undamped, rates):
        kernel = kernel + row * np.exp(-rate * t)
    return np.fft.rfft(rec.raman_fraction * kernel) * rec.dt_fine


def mixture_raman_spectrum(rec, sc: StageScalars) -> np.ndarray:
    """``passes/responses.py:293-334``: every component's rows damped at their own rates,
    weighted by its density and fraction, summed, ``rfft * dt`` (the densities inside)."""
    n2 = rec.raman_undamped.shape[1]
    t = np.arange(n2) * rec.dt_fine
    total = np.zeros(n2)
    parts = [(rec.raman_undamped, sc.raman_rates, rec.raman_fraction, sc.raman_density)]
    parts += [(c.undamped, r, c.fraction, d)
              for c, r, d in zip(rec.extra_raman, sc.raman_rates_by_component, sc.raman_densities)]
    for undamped, rates, fraction, density in parts:
        amplitude = np.zeros(n2)
        for row, rate in zip(undamped, rates):
            amplitude += row * np.exp(-rate * t)
        total += density * fraction * amplitude
    return np.fft.rfft(total) * rec.dt_fine


def tensor_raman_spectrum(rec, sc: StageScalars) -> np.ndarray:
    """``passes/responses.py:337-392``: the trace and (when any row has one) the traceless
    kernels of two Cartesian components, every component's rows weighted, the densities
    inside for a mixture and 1 for one component (its density multiplies outside)."""
    n2 = rec.raman_undamped.shape[1]
    t = np.arange(n2) * rec.dt_fine
    parts = [(rec.raman_undamped, rec.raman_tensor_weights, sc.raman_rates, rec.raman_fraction,
              sc.raman_density)]
    parts += [(c.undamped, c.tensor_weights, r, c.fraction, d)
              for c, r, d in zip(rec.extra_raman, sc.raman_rates_by_component, sc.raman_densities)]
    n_kernels = 2 if any(np.any(w[:, 1]) for _, w, _, _, _ in parts) else 1
    mixture = len(parts) > 1
    total = np.zeros((n_kernels, n2))
    for undamped, weights, rates, fraction, density in parts:
        amplitude = np.zeros_like(total)
        for row, w, rate in zip(undamped, weights, rates):
            damped = row * np.exp(-rate * t)
            for k in range(n_kernels):
                amplitude[k] += w[k] * damped
        total += (density if mixture else 1.0) * fraction * amplitude
    return np.fft.rfft(total, axis=-1) * rec.dt_fine


def vector_raman_polarisation(rec, field_t: np.ndarray, spectrum: np.ndarray, density: float) -> np.ndarray:
    """``passes/responses.py:501-550``: the trace, difference and coherence drives of two
    Cartesian components convolved with the trace and traceless kernels, the symmetric
    matrix they make applied to the field (on the envelope grid, drives of ``|a|^2 / 2``)."""
    n_to = field_t.shape[-1]
    if rec.grid_kind != "envelope":
        raise NotImplementedError("vector Raman on a field grid")
    x, y = field_t[:, 0], field_t[:, 1]
    half = 0.5
    xx = half * (np.real(x) ** 2 + np.imag(x) ** 2)
    yy = half * (np.real(y) ** 2 + np.imag(y) ** 2)
    n_drives = 1 if spectrum.shape[0] == 1 else 3
    drive = np.zeros((field_t.shape[0], n_drives, 2 * n_to))
    drive[:, 0, :n_to] = xx + yy
    if n_drives == 3:
        drive[:, 1, :n_to] = xx - yy
        drive[:, 2, :n_to] = 2 * half * (np.real(x) * np.real(y) + np.imag(x) * np.imag(y))
    kernels = spectrum if n_drives == 1 else spectrum[[0, 1, 1]]
    conv = np.fft.irfft(kernels * np.fft.rfft(drive, axis=-1), n=2 * n_to, axis=-1)[..., :n_to]
    if n_drives == 1:
        return (EPS0 * density) * field_t * conv
    u, v, w = conv[:, 0], conv[:, 1], conv[:, 2]
    out = np.empty_like(field_t)
    out[:, 0] = (u + v) * field_t[:, 0] + w * field_t[:, 1]
    out[:, 1] = w * field_t[:, 0] + (u - v) * field_t[:, 1]
    return (EPS0 * density) * out


def raman_polarisation(rec, field_t: np.ndarray, spectrum: np.ndarray, density: float) -> np.ndarray:
    """``passes/responses.py:395-498`` (scalar): ``eps0 rho E irfft(H rfft(D))`` doubled."""
    n_to = field_t.shape[-1]
    drive = np.zeros((field_t.shape[0], 2 * n_to))
    if rec.grid_kind == "envelope":
        d = 0.5 * np.abs(field_t[:, 0, :]) ** 2
    elif rec.raman_thg:
        d = field_t[:, 0, :] ** 2
    else:
        raise NotImplementedError("analytic-signal Raman drive on a field grid")
    drive[:, :n_to] = d
    conv = np.fft.irfft(spectrum * np.fft.rfft(drive, axis=-1), n=2 * n_to, axis=-1)[..., :n_to]
    return (EPS0 * density) * field_t * conv[:, None, :]


def held_spectrum(rec, gated: np.ndarray, edge: np.ndarray) -> np.ndarray:
    """``passes/plasma.py:579-613``: ``DFT[gJ]/(i w) - DFT[g'J]/(i w)^2`` on active bins."""
    current = np.fft.rfft(gated, axis=-1)[..., rec.crop_index]
    derivative = np.fft.rfft(edge, axis=-1)[..., rec.crop_index]
    result = np.zeros_like(current)
    active = rec.active_mask
    q = 1j * rec.omega[active]
    result[..., active] = current[..., active] / q - derivative[..., active] / q ** 2
    return result


def lab_source(rec, lab: np.ndarray, z: float, *, quiet: bool = False, out: dict | None = None):
    """``backends/numpy_ref/workspace.py:819-859`` for the modal route.

    The untransported source ``F`` at a lab-frame field: the stage at ``(z, z)`` with
    a unit inverse propagator.  ``quiet`` leaves out a quiet in-stage collar
    (``source.py:858-890``).  ``out`` receives the intermediates when given.
    """
    sc = stage_scalars(rec, z, z)
    field_in = lab
    modal_t = to_time(rec, field_in)
    field_t = synthesise(rec, modal_t, sc.taper)
    total = np.zeros_like(field_t)
    current = rate = fraction = None
    if rec.plasma_enabled and rec.extra_channels:
        current = channels_current(rec, field_t, sc)
    elif rec.plasma_enabled:
        rate, fraction, current = plasma_column(rec, field_t, sc)
    if rec.kerr_enabled:
        total = total + kerr_polarisation(rec, field_t, sc.kerr_density, rec.carrier)
    if rec.raman_enabled and field_t.shape[-2] == 2:  # two Cartesian components: the tensor
        density = 1.0 if rec.extra_raman else sc.raman_density
        total = total + vector_raman_polarisation(rec, field_t, tensor_raman_spectrum(rec, sc), density)
    elif rec.raman_enabled:
        if rec.extra_raman:  # a mixture: one spectrum, the densities inside it
            spectrum, density = mixture_raman_spectrum(rec, sc), 1.0
        else:
            spectrum, density = raman_spectrum(rec, sc.raman_rates), sc.raman_density
        total = total + raman_polarisation(rec, field_t, spectrum, density)
    polarisation = total * rec.t_window
    projected = project(rec, polarisation, sc.taper)
    spectrum = to_frequency(rec, projected)
    if current is not None:
        gated = project(rec, rec.t_window * current, sc.taper)
        edge = project(rec, rec.t_window_derivative * current, sc.taper)
        spectrum = spectrum + held_spectrum(rec, gated, edge)
    absorber = None
    if rec.absorber_scheme == "nonlinear" and not quiet:
        term = -0.5 * rec.temporal_absorber_fine * modal_t
        absorber = to_frequency(rec, term) * rec.active_mask
    prefactor = combine(sc.prefactor, rec.prefactor_terms)
    normalised = prefactor * rec.omega_window * spectrum
    if absorber is not None:
        normalised = normalised + absorber
    if out is not None:
        out.update(modal_t=modal_t, field_t=field_t, polarisation=polarisation,
                   projected=projected, spectrum=spectrum, absorber=absorber)
        if current is not None:
            out.update(rate=rate, fraction=fraction, current=current, gated=gated, edge=edge)
    return normalised

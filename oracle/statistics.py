"""Plane statistics of a stored state, restated from solprop's definitions.

``src/solprop/stats/definitions.py``: ``analytic_field`` (148-178: an irfft on a field
grid, then ``fourier.analytic_signal``, scipy.signal.hilbert's weights; the ifft on an
envelope grid), ``omega0`` (268-362), ``energy`` (363-390, ``fourier.energy_omega``
805-855), ``peak_power`` (443-478) and ``peak_power_total`` (479-510); the energy per
bin is ``fourier.energy_weights`` (857-904) times the columns' summed ``|a|^2``.  Test
infrastructure (see the package docstring).
"""

from __future__ import annotations

import numpy as np
import scipy.fft

__all__ = ["statistics"]


def _weights(n_omega: int, n_t: int, dt: float, envelope: bool) -> np.ndarray:
    if envelope:
        return np.full(n_omega, dt / n_t)
    w = np.full(n_omega, 4.0 * dt / n_t)
    w[0] = w[-1] = dt / n_t
    return w


def _analytic(state: np.ndarray, n_t: int, envelope: bool) -> np.ndarray:
    if envelope:
        return scipy.fft.ifft(state, n=n_t, axis=-1)
    samples = scipy.fft.irfft(state, n=n_t, axis=-1)
    spectrum = scipy.fft.fft(samples, axis=-1)
    h = np.zeros(n_t)
    h[0] = h[n_t // 2] = 1.0
    h[1 : n_t // 2] = 2.0
    return scipy.fft.ifft(spectrum * h, axis=-1)


def statistics(rec, state: np.ndarray) -> dict:
    """energy and omega0 per (mode, polarisation), peak_power per mode, peak_power_total,
    and the energy per bin summed over the columns, of ``state`` (n_modes, n_pol, n_omega)."""
    envelope = rec.grid_kind == "envelope"
    power = np.abs(state) ** 2
    w = _weights(rec.n_omega, rec.n_t, rec.dt, envelope)
    density = power.sum(axis=-1)
    with np.errstate(invalid="ignore", divide="ignore"):
        omega0 = np.where(density > 0, (rec.omega * power).sum(axis=-1) / density, np.nan)
    p_t = np.abs(_analytic(state, rec.n_t, envelope)) ** 2
    return {"energy": (w * power).sum(axis=-1), "omega0": omega0,
            "peak_power": p_t.sum(axis=1).max(axis=-1),
            "peak_power_total": p_t.sum(axis=(0, 1)).max(),
            "spectrum": w * power.sum(axis=(0, 1))}

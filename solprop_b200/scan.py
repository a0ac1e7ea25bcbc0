"""Seeded capillary problems for parameter scans (configs 4 and 5: the batched scan and its surrogate).

A scan point is a gas-filled capillary run: core radius, length, gas, constant pressure,
pulse energy and duration at 800 nm, mode count and fine time-grid size.  This module
builds the :class:`~solprop_b200.record.ProblemRecord` of such a run from the physics
the reference's capillary route uses, restated here so that scans can be generated on a
machine without solprop:

* the field grid of ``grid.py`` (fine spacing fixed, the window growing with the grid),
  active band ``omega_min / 2 < omega < 1.1 omega_max`` (``translate/masks.py``);
* Marcatili HE_1m modes of a dielectric capillary filled with the gas (Marcatili and
  Schmeltzer, Bell Syst. Tech. J. 43, 1783 (1964)), gas index from Börzsönyi et al.'s
  two-pole fits (Appl. Opt. 47, 4856 (2008)) scaled with density, the operator
  ``D = -i (beta - beta0 - beta1 (omega - omega0)) - alpha / 2`` in the FFT convention of
  ``docs/dev/conventions.md`` (a constant representation: one term, weight ``dz``);
* the prefactor ``-i omega / (2 eps0 c Re n_eff)`` times the crop scale, zero off band;
* a Gauss-Legendre radial quadrature of the J0(u_m r / a) mode fields, normalised to one
  watt, with the pad scale in the synthesis and the weights in the projection
  (``modes/quadrature.py``);
* the real-field Kerr cubic with the gas's gamma3, and field plasma with the quasistatic
  ADK rate (Ammosov, Delone and Krainov, Sov. Phys. JETP 64, 1191 (1986)) tabulated as a
  cubic in log |E| on uniform knots (``translate/ionisation.py``), the trapezoid running
  integral;
* an in-stage temporal collar, a Gaussian input pulse in HE11 and one photon per mode
  per frequency bin of input shot noise, seeded: the reference's draw
  (``noise.py:195-294``), which the tests hold bit for bit to the reference's own
  realisation on the same grid and seed.

The scan's parameter distribution is config 4's (:func:`draw_points`).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy.interpolate import CubicSpline
from scipy.special import gamma as gamma_fn
from scipy.special import j0, j1

from solprop_b200.record import PiecewiseTable, ProblemRecord

C0 = 299792458.0
EPS0 = 8.8541878188e-12
HBAR = 6.62607015e-34 / (2 * math.pi)  # h / 2 pi, as scipy.constants defines it
E_CHARGE = 1.602176634e-19
M_E = 9.1093837139e-31
K_B = 1.380649e-23
AU_FIELD = 5.14220674763e11      # V/m
AU_TIME = 2.4188843265857e-17    # s
AU_ENERGY = 4.3597447222060e-18  # J
ROOM = 294.15                    # K

# (B1, C1 um^2, B2, C2 um^2) at 1 bar and 273.15 K; (Ip hartree, l, Z); gamma3 m^5/V^2
BORZSONYI = {
    "He": (4977.77e-8, 28.54e-6, 1856.94e-8, 7.76e-3),
    "Ne": (9154.48e-8, 656.97e-6, 4018.63e-8, 5.728e-3),
    "Ar": (20332.29e-8, 206.12e-6, 34458.31e-8, 8.066e-3),
}
ATOMS = {"He": (0.9036, 0, 1.0), "Ne": (0.7925, 1, 1.0), "Ar": (0.5792, 1, 1.0)}
GAMMA3 = {"He": 3.43e-53, "Ne": 6.8e-53, "Ar": 1.2e-51}
GASES = ("He", "Ne", "Ar")
HE1M_ZEROS = (2.404825557695773, 5.520078110286311, 8.653727912911012, 11.791534439014281,
              14.930917708487787, 18.071063967910924, 21.21163662987926, 24.352471530749302)
CLADDING = 1.45
DT_FINE = 0.09e-15               # s: the fine spacing; the coarse one is twice it
LAMBDA0 = 800e-9
BAND = (150e-9, 4e-6)


@dataclass(frozen=True)
class ScanPoint:
    radius: float     # m
    length: float     # m
    gas: str
    pressure: float   # bar
    energy: float     # J
    fwhm: float       # s
    modes: int
    n_to: int
    seed: int

    @property
    def features(self) -> np.ndarray:
        """The surrogate's six inputs: radius, length, gas id, pressure, energy, FWHM."""
        return np.array([self.radius, self.length, GASES.index(self.gas), self.pressure,
                         self.energy, self.fwhm])


def draw_points(n: int, seed: int, *, modes=(1, 8), grids=(12, 13, 14, 15)) -> list[ScanPoint]:
    """Config 4's distribution: radius U[50, 150] um, length U[0.5, 2] m, gas from
    {He, Ne, Ar}, pressure U[0.2, 3] bar, energy log-U[20, 500] uJ, FWHM U[5, 30] fs,
    mode count U{modes}, n_to uniform over 2**grids."""
    rng = np.random.default_rng(seed)
    points = []
    for i in range(n):
        points.append(ScanPoint(
            radius=float(rng.uniform(50e-6, 150e-6)),
            length=float(rng.uniform(0.5, 2.0)),
            gas=GASES[int(rng.integers(0, 3))],
            pressure=float(rng.uniform(0.2, 3.0)),
            energy=float(math.exp(rng.uniform(math.log(20e-6), math.log(500e-6)))),
            fwhm=float(rng.uniform(5e-15, 30e-15)),
            modes=int(rng.integers(modes[0], modes[1] + 1)),
            n_to=int(2 ** grids[int(rng.integers(0, len(grids)))]),
            seed=int(rng.integers(0, 2**31 - 1)),
        ))
    return points


def gas_index_minus_one(gas: str, omega: np.ndarray, density: float) -> np.ndarray:
    """n - 1 of the gas at ``density`` (m^-3), from the 1 bar, 0 C fit scaled by density."""
    lam_um2 = (2 * np.pi * C0 / omega * 1e6) ** 2
    b1, c1, b2, c2 = BORZSONYI[gas]
    n2m1 = b1 * lam_um2 / (lam_um2 - c1) + b2 * lam_um2 / (lam_um2 - c2)
    rho0 = 1e5 / (K_B * 273.15)
    return (np.sqrt(1.0 + n2m1) - 1.0) * (density / rho0)


def adk_rate(gas: str, field: np.ndarray) -> np.ndarray:
    """Quasistatic ADK rate per atom (s^-1), summed over m, at field amplitudes in V/m."""
    ip, l, z = ATOMS[gas]
    ns = z / math.sqrt(2 * ip)
    ls = ns - 1.0
    c2 = 2 ** (2 * ns) / (ns * gamma_fn(ns + ls + 1) * gamma_fn(ns - ls))
    f = np.abs(np.asarray(field, dtype=np.float64)) / AU_FIELD
    k = (2 * ip) ** 1.5
    total = np.zeros_like(f)
    for m in range(-l, l + 1):
        am = abs(m)
        flm = (2 * l + 1) * math.factorial(l + am) / (2**am * math.factorial(am) * math.factorial(l - am))
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            w = c2 * flm * ip * (2 * k / f) ** (2 * ns - am - 1) * np.exp(-2 * k / (3 * f))
        total += np.where(f > 0, w, 0.0)
    return total / AU_TIME


def rate_table(gas: str, intervals: int = 512):
    """The rate as exp of a cubic in log|E| on uniform knots (translate/ionisation.py)."""
    field_min = 1e9
    for _ in range(60):  # the field where the rate reaches 1 s^-1
        if adk_rate(gas, np.array([field_min]))[0] > 1.0:
            break
        field_min *= 1.2
    field_max = 1.0e12
    log_min, log_max = math.log(field_min), math.log(field_max)
    knots = np.linspace(log_min, log_max, intervals + 1)
    spline = CubicSpline(knots, np.log(adk_rate(gas, np.exp(knots))))
    return dict(rate_coefficients=np.ascontiguousarray(spline.c), log_field_min=log_min,
                d_log_field=(log_max - log_min) / intervals, field_min=field_min,
                field_max=field_max, rate_max=float(adk_rate(gas, np.array([field_max]))[0]))


def input_noise(omega: np.ndarray, active: np.ndarray, dt: float, d_omega: float,
                rng: np.random.Generator, *, n_modes: int = 1, n_pol: int = 1,
                kind: str = "field") -> np.ndarray:
    """One photon per mode, polarisation and active bin, with a random phase (the input
    shot-noise model, ``noise.py:195-294``): amplitude ``sqrt(hbar omega / d_omega)
    sqrt(2 pi) / dt``, halved on a field grid (its one-sided spectrum); the phase drawn
    uniform on [0, 2 pi) over every bin, active or not, so that a seed means the same
    realisation whatever the band."""
    amplitude = np.zeros(len(omega))
    scale = np.sqrt(2.0 * np.pi) / dt
    if kind == "field":
        scale = 0.5 * scale
    amplitude[active] = scale * np.sqrt(HBAR * omega[active] / d_omega)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(n_modes, n_pol, len(omega)))
    return amplitude * np.exp(1j * phase)


def collar(t: np.ndarray, half_window: float):
    """The temporal collar: one on the central 80 %, a cos^2 taper over each 10 % edge."""
    edge = 0.2 * half_window
    inner = half_window - edge
    u = np.clip((np.abs(t) - inner) / edge, 0.0, 1.0)
    g = np.cos(0.5 * np.pi * u) ** 2
    dg = np.where((u > 0) & (u < 1), -np.sign(t) * (np.pi / (2 * edge)) * np.sin(np.pi * u), 0.0)
    return g, dg


def capillary_record(p: ScanPoint) -> tuple[ProblemRecord, dict]:
    """The record of one scan point and its exponential-Adams march policy."""
    n_to = p.n_to
    n_t = n_to // 2
    dt = 2 * DT_FINE
    n_omega = n_t // 2 + 1
    omega = 2 * np.pi * np.arange(n_omega) / (n_t * dt)
    omega0 = 2 * np.pi * C0 / LAMBDA0
    w_min, w_max = 2 * np.pi * C0 / BAND[1], 2 * np.pi * C0 / BAND[0]
    active = (omega > w_min / 2) & (omega < 1.1 * w_max)
    density = p.pressure * 1e5 / (K_B * ROOM)
    n_modes = p.modes
    # Marcatili HE_1m propagation constants (complex), on the active band
    nu = (CLADDING**2 + 1) / (2 * math.sqrt(CLADDING**2 - 1))
    beta = np.zeros((n_modes, n_omega))
    alpha = np.zeros((n_modes, n_omega))
    w_act = omega[active]
    ngas = 1.0 + gas_index_minus_one(p.gas, w_act, density)
    k = w_act / C0 * ngas
    for m in range(n_modes):
        u = HE1M_ZEROS[m]
        gam = k * (1.0 - 0.5 * (u / (k * p.radius)) ** 2 * (1.0 - 1j * nu / (k * p.radius)))
        beta[m, active] = gam.real
        alpha[m, active] = np.minimum(2.0 * gam.imag, 2 * 708.0 / p.length)
    # frame: beta0 + beta1 (omega - omega0) of HE11 at the carrier
    b_of = lambda w: (w / C0 * (1 + gas_index_minus_one(p.gas, np.array([w]), density))
                      * (1 - 0.5 * (HE1M_ZEROS[0] / (w / C0 * p.radius)) ** 2))[0]
    h = omega0 * 1e-6
    beta0 = b_of(omega0)
    beta1 = (b_of(omega0 + h) - b_of(omega0 - h)) / (2 * h)
    D = np.zeros((n_modes, 1, n_omega), dtype=np.complex128)
    D[:, 0, :] = np.where(active, -1j * (beta - beta0 - beta1 * (omega - omega0)) - 0.5 * alpha, 0.0)
    crop_scale = n_t / n_to
    neff = np.where(active, beta * C0 / np.maximum(omega, 1e-300), 1.0)
    pre = np.zeros_like(D)
    pre[:, 0, :] = np.where(active, -1j * omega / (2 * EPS0 * C0 * neff) * crop_scale, 0.0)
    # radial quadrature of the mode fields
    n_r = max(8, 8 * n_modes)
    x, w = np.polynomial.legendre.leggauss(n_r)
    r = 0.5 * p.radius * (x + 1.0)
    wr = 0.5 * p.radius * w
    pad_scale = n_to / n_t
    norm = np.array([1.0 / (p.radius * abs(j1(HE1M_ZEROS[m])) * math.sqrt(math.pi * EPS0 * C0 / 2))
                     for m in range(n_modes)])
    fields = np.array([norm[m] * j0(HE1M_ZEROS[m] * r / p.radius) for m in range(n_modes)])
    synthesis = np.ascontiguousarray((pad_scale * fields).T)                 # (n_r, n_modes)
    projection = np.ascontiguousarray((EPS0 * C0 / 2) * fields * (2 * np.pi * r * wr)[None, :])
    # grids in time: centred, the fine axis twice as dense
    t_fine = (np.arange(n_to) - n_to // 2) * DT_FINE
    half = 0.5 * n_to * DT_FINE
    g, dg = collar(t_fine, half)
    alpha_max = 60.0 / p.length
    absorber = alpha_max * (1.0 - g)
    # input pulse in HE11: Gaussian, real field, energy normalised on the coarse grid
    t = (np.arange(n_t) - n_t // 2) * dt
    env = np.exp(-2 * math.log(2) * (t / p.fwhm) ** 2)
    a = env * np.cos(omega0 * t)
    a *= math.sqrt(p.energy / (np.sum(a * a) * dt))
    field0 = np.zeros((n_modes, 1, n_omega), dtype=np.complex128)
    field0[0, 0] = np.fft.rfft(a) * active
    # the state is the vacuum-normalised amplitude: true-power spectra divided by the root
    # of the modes' power weight Re n_eff (fourier.py:300-340, driver/inputs.py:484-488)
    root_weight = np.sqrt(np.where(active, beta * C0 / np.maximum(omega, 1e-300), 1.0))[:, None, :]
    field0 /= root_weight
    noise0 = input_noise(omega, active, dt, 2 * np.pi / (n_t * dt), np.random.default_rng(p.seed),
                         n_modes=n_modes) / root_weight
    rt = rate_table(p.gas)
    rec = ProblemRecord(
        grid_kind="field", n_modes=n_modes, n_pol=1, n_omega=n_omega, n_t=n_t, n_to=n_to,
        n_nodes=n_r, n_pol_transform=1, omega0=omega0, dt=dt, dt_fine=DT_FINE,
        pad_scale=pad_scale, crop_scale=crop_scale, z_end=p.length, omega=omega,
        crop_index=np.arange(n_omega, dtype=np.int64), active_mask=active, norm_mask=active.copy(),
        omega_window=np.ones(n_omega), t_window=g, t_window_derivative=dg,
        phi_representation="constant", phi_terms=D[None], prefactor_terms=pre[None],
        breakpoints=np.array([0.0, 1.05 * p.length]),
        density=PiecewiseTable.constant(density, 0.0, 1.05 * p.length),
        kerr_density=PiecewiseTable.constant(density, 0.0, 1.05 * p.length),
        plasma_density=PiecewiseTable.constant(density, 0.0, 1.05 * p.length),
        preionisation=PiecewiseTable.constant(0.0, 0.0, 1.05 * p.length),
        synthesis=synthesis, projection=projection, projection_coarse=projection.copy(),
        kerr_enabled=True, kerr_coefficient=EPS0 * GAMMA3[p.gas], kerr_form="real",
        plasma_enabled=True, charge_mass_ratio=E_CHARGE**2 / M_E,
        ionisation_potential=ATOMS[p.gas][0] * AU_ENERGY, integral_policy="trapezoid",
        taps=np.ones(1), absorber_scheme="nonlinear", temporal_absorber_fine=absorber,
        field0=field0, noise0=noise0, noise_model="input", **rt)
    policy = {
        "march": "HostAdamsMarch", "order": 5, "variable_order": True, "safety": 0.8,
        "max_growth": 2.0, "min_factor": 0.2, "rejection_growth": 0.9, "hysteresis": 1.2,
        "restart_after": 3, "collar_stability": 1.0,
        "real_intervals": [1.0, 0.545, 0.3, 0.163, 0.0877, 0.0465],
        "collar_rate": alpha_max / 2, "equal_approach": True, "interval_cap": False,
        "dz_min": 1e-9 * p.length, "dz_max": 0.5 * p.length, "stretch": 1.1,
        "z_end": p.length, "save_planes": [p.length], "hard_kinks": [],
        "breakpoints": [0.0, 1.05 * p.length], "landing_ulps": 8, "interpolate": False,
        "rtol": 1e-6, "atol": 1e-10, "proposal": 1e-4 * p.length,
    }
    return rec, policy


def shard(points, rank: int, world: int) -> list[int]:
    """The indices of the points rank ``rank`` of ``world`` solves: the runs sorted by their
    cost (fine samples x modes, the response column's work) and dealt round-robin, so every
    rank gets a like share of each size.  Runs are independent: no exchange while they run."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    order = sorted(range(len(points)), key=lambda i: (-points[i].n_to * points[i].modes, i))
    return sorted(i for k, i in enumerate(order) if k % world == rank)


def gather_by_index(indices, values, n_total: int, group=None):
    """Every rank's per-point rows, assembled in point order on rank 0 (None elsewhere):
    the scan's one collective, after all runs have finished."""
    import torch.distributed as dist

    payload = (list(indices), np.asarray(values))
    gathered = [None] * dist.get_world_size(group) if dist.get_rank(group) == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if gathered is None:
        return None
    first = next(v for _, v in gathered if len(v))
    out = np.zeros((n_total,) + first.shape[1:], dtype=first.dtype)
    seen = np.zeros(n_total, bool)
    for idx, vals in gathered:
        for i, v in zip(idx, vals):
            if seen[i]:
                raise ValueError(f"point {i} solved twice")
            out[i], seen[i] = v, True
    if not seen.all():
        raise ValueError(f"{int((~seen).sum())} points solved by no rank")
    return out


def exit_log_spectrum(rec: ProblemRecord, state: np.ndarray, bins: int = 2048) -> np.ndarray:
    """The surrogate's target: log10 of the exit energy spectral density, summed over modes,
    on ``bins`` wavelengths from 100 nm to 4 um (interpolated), floored at 1e-30."""
    power = np.sum(np.abs(state) ** 2, axis=(0, 1))[1:]
    lam = 2 * np.pi * C0 / rec.omega[1:]  # the DC bin has no wavelength
    grid = np.linspace(100e-9, 4e-6, bins)
    order = np.argsort(lam)
    values = np.interp(grid, lam[order], power[order], left=0.0, right=0.0)
    return np.log10(np.maximum(values, 1e-30))

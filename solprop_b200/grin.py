"""Seeded graded-index fibre problems on the envelope grid (config 3's workload).

A multimode graded-index fibre: parabolic index, core diameter 62.5 um, NA 0.275, the
lowest mode groups of its Hermite-Gauss modes in both polarisations (30 vector modes)
sampled on a Cartesian quadrature of the core (128 x 128 nodes), a 10 ps envelope window
at 1030 nm (2^14 samples), Kerr (n2 = 2.7e-20 m^2/W) and a silica-like tensor Raman response (f_R 0.18,
tau_1 12.2 fs, tau_2 32 fs), 500 nJ of a 200 fs Gaussian split equally over the first ten
modes with seeded phases.  The reference builds graded-index fibres on its field-grid
general modal route only, so this record is the envelope route restated from published
physics, for throughput measurement at config 3's size:

* fused silica's index from Malitson's Sellmeier fit (J. Opt. Soc. Am. 55, 1205 (1965));
* the parabolic fibre's Hermite-Gauss modes, waist ``w^2 = a lambda / (pi NA)`` and
  propagation constants ``beta_g^2 = (k n)^2 - 2 k n sqrt(2 Delta) (g + 1) / a`` for the
  mode group ``g = m + n`` (e.g. Agrawal, Nonlinear Fiber Optics, ch. 2), normalised to one
  watt, ``(eps0 c / 2) sum |f|^2 dA = 1``; the synthesis holds the two Cartesian
  components of each node (rows x, y), the projection ``(eps0 c / 2) f dA``;
* the operator ``D = -i (beta - beta0 - beta1 (omega - omega0))`` of the envelope grid
  (absolute frequencies ``omega0 + 2 pi fftfreq``) and the prefactor
  ``-i omega / (2 eps0 c n_eff)``, zero off the band, as the capillary records of
  ``scan.py``;
* the analytic Kerr cubic ``eps0 chi3 (|E|^2 E / 2 + E^2 E* / 4)``, summed over the
  components, ``chi3 = 4 eps0 c n^2 n2 / 3``; the Raman kernel
  ``K (tau1^2 + tau2^2) / (tau1 tau2^2) e^(-t / tau2) sin(t / tau1)`` with ``K`` giving it
  the fraction f_R of the nonlinear index, trace weight 1 and a traceless weight 0.5;
* an in-stage temporal collar and a DOPRI5 march at rtol 1e-6.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.special import eval_hermite

from solprop_b200.record import PiecewiseTable, ProblemRecord

C0 = 299792458.0
EPS0 = 8.8541878188e-12

CORE_RADIUS = 31.25e-6
NA = 0.275
LAMBDA0 = 1030e-9
WINDOW = 10e-12
LENGTH = 0.5
N2 = 2.7e-20
F_R, TAU1, TAU2 = 0.18, 12.2e-15, 32e-15
ENERGY, FWHM, LAUNCHED = 500e-9, 200e-15, 10


def silica_index(omega: np.ndarray) -> np.ndarray:
    """Malitson's three-pole Sellmeier fit of fused silica (wavelength in um)."""
    lam = 2 * np.pi * C0 / np.asarray(omega) * 1e6
    l2 = lam * lam
    n2m1 = (0.6961663 * l2 / (l2 - 0.0684043**2) + 0.4079426 * l2 / (l2 - 0.1162414**2)
            + 0.8974794 * l2 / (l2 - 9.896161**2))
    return np.sqrt(1.0 + n2m1)


def mode_orders(n_groups: int = 5) -> list[tuple[int, int]]:
    """Hermite-Gauss orders (m, n) of the mode groups g = m + n < n_groups, lowest first."""
    return [(m, g - m) for g in range(n_groups) for m in range(g, -1, -1)]


def grin_record(n_to: int = 16384, grid: int = 128, seed: int = 3) -> tuple[ProblemRecord, dict]:
    """The record and DOPRI5 policy of the graded-index workload: 2 x 15 modes on
    ``grid x grid`` Cartesian nodes, ``n_to`` envelope samples over the 10 ps window."""
    dt = WINDOW / n_to
    omega0 = 2 * np.pi * C0 / LAMBDA0
    omega = omega0 + 2 * np.pi * np.fft.fftfreq(n_to, dt)
    lam = 2 * np.pi * C0 / omega
    active = (lam > 700e-9) & (lam < 1600e-9)
    orders = mode_orders()
    n_spatial = len(orders)
    n_modes = 2 * n_spatial
    # propagation constants on the band
    n_core = silica_index(np.where(active, omega, omega0))
    delta = NA**2 / (2 * silica_index(np.array([omega0]))[0] ** 2)
    k = omega / C0
    beta = np.zeros((n_spatial, n_to))
    for s, (m, n) in enumerate(orders):
        g = m + n
        b2 = (k * n_core) ** 2 - 2 * k * n_core * math.sqrt(2 * delta) * (g + 1) / CORE_RADIUS
        beta[s] = np.where(active, np.sqrt(np.maximum(b2, 0.0)), 0.0)

    def beta_of(w: float) -> float:
        nc = silica_index(np.array([w]))[0]
        return math.sqrt((w / C0 * nc) ** 2 - 2 * w / C0 * nc * math.sqrt(2 * delta) / CORE_RADIUS)

    h = omega0 * 1e-6
    beta0 = beta_of(omega0)
    beta1 = (beta_of(omega0 + h) - beta_of(omega0 - h)) / (2 * h)
    D = np.zeros((n_modes, 1, n_to), dtype=np.complex128)
    pre = np.zeros_like(D)
    for c in range(n_modes):
        b = beta[c // 2]
        D[c, 0] = np.where(active, -1j * (b - beta0 - beta1 * (omega - omega0)), 0.0)
        neff = np.where(active, b * C0 / omega, 1.0)
        pre[c, 0] = np.where(active, -1j * omega / (2 * EPS0 * C0 * neff), 0.0)
    # Hermite-Gauss fields on the Cartesian nodes, one watt each
    waist = math.sqrt(CORE_RADIUS * LAMBDA0 / (math.pi * NA))
    half = 4.5 * waist
    x = (np.arange(grid) + 0.5) / grid * 2 * half - half
    area = (2 * half / grid) ** 2
    X, Y = np.meshgrid(x, x, indexing="ij")
    X, Y = X.ravel(), Y.ravel()
    n_nodes = grid * grid
    synthesis = np.zeros((2 * n_nodes, n_modes))
    for s, (m, n) in enumerate(orders):
        f = (eval_hermite(m, math.sqrt(2) * X / waist) * eval_hermite(n, math.sqrt(2) * Y / waist)
             * np.exp(-(X * X + Y * Y) / waist**2))
        f /= math.sqrt(EPS0 * C0 / 2 * np.sum(f * f) * area)
        synthesis[0::2, 2 * s] = f      # x-polarised: the x rows
        synthesis[1::2, 2 * s + 1] = f  # y-polarised: the y rows
    projection = np.ascontiguousarray((EPS0 * C0 / 2) * area * synthesis.T)
    # the temporal collar and its in-stage absorber
    t = (np.arange(n_to) - n_to // 2) * dt
    edge = 0.1 * WINDOW
    ramp = np.clip((np.abs(t) - (0.5 * WINDOW - edge)) / edge, 0.0, 1.0)
    g_win = np.cos(0.5 * np.pi * ramp) ** 2
    dg = np.gradient(g_win, dt)
    alpha = 60.0 / LENGTH * (1.0 - g_win)
    # nonlinearity: Kerr and the Raman kernel (trace and traceless weights)
    n0 = silica_index(np.array([omega0]))[0]
    chi3 = 4 * EPS0 * C0 * n0**2 * N2 / 3
    coefficient = EPS0 * chi3
    strength = 1.5 * chi3 * F_R / (1 - F_R)
    tk = np.arange(2 * n_to) * dt
    undamped = strength * (TAU1**2 + TAU2**2) / (TAU1 * TAU2**2) * np.sin(tk / TAU1)
    undamped[n_to:] = 0.0
    # the launch: the first ten modes, a Gaussian of ENERGY in all, seeded phases
    rng = np.random.default_rng(seed)
    env = np.exp(-2 * math.log(2) * (t / FWHM) ** 2)
    env *= math.sqrt(ENERGY / LAUNCHED / (np.sum(env * env) * dt))
    field0 = np.zeros((n_modes, 1, n_to), dtype=np.complex128)
    for c in range(LAUNCHED):
        field0[c, 0] = np.fft.fft(env * np.exp(1j * rng.uniform(0, 2 * np.pi))) * active
    span = (0.0, 1.05 * LENGTH)
    rec = ProblemRecord(
        grid_kind="envelope", n_modes=n_modes, n_pol=1, n_omega=n_to, n_t=n_to, n_to=n_to,
        n_nodes=n_nodes, n_pol_transform=2, omega0=omega0, dt=dt, dt_fine=dt, pad_scale=1.0,
        crop_scale=1.0, z_end=LENGTH, omega=omega, crop_index=np.arange(n_to, dtype=np.int64),
        active_mask=active, norm_mask=active.copy(), omega_window=np.ones(n_to),
        t_window=g_win, t_window_derivative=dg,
        phi_representation="constant", phi_terms=D[None], prefactor_terms=pre[None],
        breakpoints=np.array(span), density=PiecewiseTable.constant(1.0, *span),
        kerr_density=PiecewiseTable.constant(1.0, *span), taper_scale=None,
        synthesis=np.ascontiguousarray(synthesis), projection=projection,
        projection_coarse=projection.copy(), kerr_enabled=True, kerr_coefficient=coefficient,
        kerr_form="analytic", kerr_self=0.5, kerr_conjugate=0.25, kerr_harmonic=0.0,
        kerr_take_real=False, raman_enabled=True, raman_undamped=undamped[None],
        raman_rates=[PiecewiseTable.constant(1.0 / TAU2, *span)], raman_fraction=1.0,
        raman_thg=False, raman_density=PiecewiseTable.constant(1.0, *span),
        raman_tensor_weights=np.array([[1.0, 0.5]]), absorber_scheme="nonlinear",
        temporal_absorber_fine=alpha, field0=field0)
    policy = {
        "march": "RungeKuttaMarch",
        "controller": {"rtol": 1e-6, "atol": 1e-10, "safety": 0.8, "max_factor": 1.1, "min_factor": 0.2,
                       "beta1": 0.12, "beta2": -0.04, "lag": 1, "reject_free": False,
                       "estimator_order": 4},
        "dz_min": 1e-10, "dz_max": 0.05, "auto_init": True, "stretch": 1.1, "z_end": LENGTH,
        "save_planes": [LENGTH], "hard_kinks": [], "breakpoints": list(span), "landing_ulps": 8,
        "start_growth": 100.0, "rtol": 1e-6, "atol": 1e-10, "proposal": 1e-5,
    }
    return rec, policy

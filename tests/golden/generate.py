"""Generate the golden fixtures of this directory from the reference's own NumPy backend.

Run by hand, in a container that holds the reference checkout (``SOLPROP_REFERENCE``,
default ``/root/reference``): ``python tests/golden/generate.py``.  It backports the
reference package into a temporary directory (``backport.py`` beside this file),
builds small problems through the reference's own translation layer with
caller-supplied species data (the reference's material library is not installed), runs
the reference's ``numpy_ref`` backend on them, and writes for each case

* ``<case>.problem.npz`` -- the lowered problem record (``solprop_b200.lowering``);
* ``<case>.golden.npz``  -- the reference's outputs: one source evaluation per
  listed lab field with its intermediate passes, a fixed-schedule run's planes, and an
  adaptive run's planes and step history.

The species data are published fits (Börzsönyi et al., Appl. Opt. 47, 4856 (2008) for
the refractive index), the reference's own test-only ADK rate oracle
(``tests/rate_oracles.py``) and literature hyperpolarisabilities; absolute physics
differs from a solprop install with its material library, which does not matter for
parity: the build and the reference are compared on identical problem arrays.
"""

from __future__ import annotations

import os
import sys
import time
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT))

import backport  # noqa: E402

backport.activate()
sys.path.insert(0, str(backport.REFERENCE / "tests"))

from rate_oracles import HISTORICAL_ATOMS, adk_oracle  # noqa: E402
from solprop.backends.events import ObservationReady, Progress  # noqa: E402
from solprop.backends.numpy_ref import NumpyRefBackend  # noqa: E402
from solprop.backends.numpy_ref.passes.plasma import (  # noqa: E402
    held_plasma_spectrum,
    ionisation_rate,
    plasma_scan,
)
from solprop.backends.numpy_ref.passes.responses import nonlinear_sources  # noqa: E402
from solprop.backends.numpy_ref.passes.stepping import absorber_term, stage_output  # noqa: E402
from solprop.backends.numpy_ref.passes.transforms import (  # noqa: E402
    project,
    synthesise,
    to_frequency,
    to_time,
)
from solprop.backends.session import Start  # noqa: E402
from solprop.constants import AU_ENERGY, K_B  # noqa: E402
from solprop.constants import C as C0  # noqa: E402
from solprop.driver.simulation import Simulation  # noqa: E402
from solprop.grid import EnvelopeGrid, FieldGrid  # noqa: E402
from solprop.physdata.mixtures import Mixture  # noqa: E402
from solprop.physdata.species import (  # noqa: E402
    IdealGas,
    IonisationData,
    Species,
    TabulatedSusceptibility,
)
from solprop.stepper import FixedSchedule, RungeKutta  # noqa: E402

from solprop_b200.lowering import lower  # noqa: E402
from solprop_b200.record import save_record  # noqa: E402

warnings.simplefilter("ignore")

# Börzsönyi two-pole fits (B1, C1 um^2, B2, C2 um^2) at 1 bar, 0 C.
BORZSONYI = {
    "He": (4977.77e-8, 28.54e-6, 1856.94e-8, 7.76e-3),
    "Ne": (9154.48e-8, 656.97e-6, 4018.63e-8, 5.728e-3),
    "Ar": (20332.29e-8, 206.12e-6, 34458.31e-8, 8.066e-3),
}
# Hyperpolarisabilities gamma3 in m^5/V^2 of the order the literature gives.
GAMMA3 = {"He": 3.43e-53, "Ne": 6.8e-53, "Ar": 1.2e-51}


def gas_species(name: str, deep_uv: bool = False) -> Species:
    """A species of supplied data; ``deep_uv`` keeps only the fit's far pole, so that the
    table reaches 40 nm (a grid limited at 90 nm samples below the fit's second pole)."""
    shortest = 40e-9 if deep_uv else 120e-9
    lam = np.geomspace(shortest, 200e-6, 4000)[::-1]
    om = 2 * np.pi * C0 / lam
    l2 = (lam * 1e6) ** 2
    b1, c1, b2, c2 = BORZSONYI[name]
    n2m1 = b1 * l2 / (l2 - c1) + (0.0 if deep_uv else b2 * l2 / (l2 - c2))
    rho0 = 1e5 / (K_B * 273.15)
    refr = (np.sqrt(1 + n2m1) - 1) / rho0
    sus = TabulatedSusceptibility(
        om, refr, np.zeros_like(om), (shortest * 1.01, 199e-6), f"Borzsonyi 2008 {name}"
    )
    ip = HISTORICAL_ATOMS[name][0] * AU_ENERGY
    return Species(name, sus, IdealGas(), gamma3=GAMMA3[name], ionisation=IonisationData(ip))


def capillary(name, *, gas, pressure, length, n_t_limits, trange, energy, fwhm, modes,
              n_r=None, radial_rule="gauss_kronrod", absorber=None, schedule=None,
              n_save=3, rtol=1e-6, deep_uv=False):
    species = gas_species(gas, deep_uv)
    fill = Mixture.fill({species: 1.0}, pressure, length=length if not np.isscalar(pressure) else None)
    grid = FieldGrid.from_limits(length, 800e-9, n_t_limits, trange, fft_size="pow2")
    kwargs = dict(
        wavelength=800e-9, grid=grid, fwhm=fwhm, energy=energy, cladding=1.45 + 0j,
        modes=modes, plasma=adk_oracle(gas), noise=None, rtol=rtol, n_save=n_save,
        backend="numpy_ref", boundary_check=None,
    )
    if n_r is not None:
        kwargs.update(n_r=n_r, radial_rule=radial_rule)
    if absorber is not None:
        kwargs["absorber"] = absorber
    if schedule is not None:
        kwargs["schedule"] = schedule
    return Simulation.from_capillary(125e-6, length, fill, None, **kwargs)


def policy_record(session, request):
    """The march's policy and first proposal, as JSON bytes for the golden file."""
    import dataclasses
    import json

    march = session._method.march
    policy = march._policy
    values = {}
    for f in dataclasses.fields(policy):
        v = getattr(policy, f.name)
        if dataclasses.is_dataclass(v):
            v = {g.name: getattr(v, g.name) for g in dataclasses.fields(v)
                 if not isinstance(getattr(v, g.name), np.ndarray)}
        elif isinstance(v, np.ndarray):
            v = v.tolist()
        elif isinstance(v, tuple):
            v = list(v)
        values[f.name] = v
    control = request.stepper.controller
    values["rtol"], values["atol"] = float(control.rtol), float(control.atol)
    values["march"] = type(march).__name__
    values["proposal"] = float(march.state.proposal)
    return np.frombuffer(json.dumps(values, default=float).encode(), dtype=np.uint8)


def drive(sim):
    """Run the reference backend's session; return plane positions, states, history."""
    problem, request = sim.translate(), sim.run_request()
    backend = NumpyRefBackend(problem, request, grid=sim.grid, modes=sim.modes,
                              profiles=sim.profiles)
    session = backend.prepare(problem, request).start(Start.entrance(problem))
    drive.policy = policy_record(session, request)
    ws = backend._workspace
    zs, states, hist = [], [], []
    t0 = time.time()
    while not session.finished:
        batch = session.advance()
        for ev in batch.events:
            if isinstance(ev, Progress):
                continue
            h = getattr(ev, "history", None)
            if h is not None and len(h.z):
                hist.append(np.stack([h.z, h.dz, h.error_norm, h.accepted.astype(float)], 1))
            if isinstance(ev, ObservationReady):
                zs.append(ev.z if hasattr(ev, "z") else np.nan)
                states.append(np.array(ws.committed()))
            err = getattr(ev, "error", None)
            if err is not None:
                raise err
        session.acknowledge(batch.receipt)
    wall = time.time() - t0
    status = session.status()
    counts = np.array([getattr(status, "attempts", -1), getattr(status, "rejected", -1)])
    history = np.concatenate(hist) if hist else np.zeros((0, 4))
    return problem, np.array(zs), np.array(states), (history, counts), wall


def source_passes(problem, ws, lab, z, keep_nodes):
    """One source evaluation, pass by pass, checked against ``lab_source``."""
    grids, transform, responses = problem.grids, problem.transform, problem.responses
    kind = problem.grid_kind
    bundle = ws.stage_scalars(z, z)
    src = ws.stage_source
    modal_t = to_time(lab, grids.crop_index, grids.n_to, kind=kind)
    n_pol = transform._n_pol
    field_t = synthesise(modal_t, transform.synthesis, bundle.taper_scale, n_pol)
    raman = src._raman_spectrum(bundle.raman_rates, bundle.raman_densities)
    sources = nonlinear_sources(
        field_t, responses, grids.t_window_fine, kind=kind, density=bundle.density,
        preionisation=bundle.preionisation, dt=grids.dt_fine, carrier=grids.carrier_2w0,
        raman_spectrum=raman, scalars=bundle,
    )
    out = {"modal_t": modal_t, "field_nodes": field_t[keep_nodes],
           "polarisation_nodes": sources.polarisation[keep_nodes]}
    projected = project(sources.polarisation, transform.projection, bundle.taper_scale, n_pol)
    spectrum = to_frequency(projected, grids.crop_index, kind=kind)
    out["projected"] = projected
    if sources.current is not None:
        out["current_nodes"] = sources.current[keep_nodes]
        rate = ionisation_rate(field_t, responses.ionisation_table[0])
        frac, _ = plasma_scan(field_t, rate, responses.plasma_channels[0],
                              preionisation=bundle.preionisation, dt=grids.dt_fine,
                              integral=responses.plasma_integral)
        out["rate_nodes"] = rate[keep_nodes]
        out["fraction_nodes"] = frac[keep_nodes]
        gated = project(grids.t_window_fine * sources.current, transform.projection,
                        bundle.taper_scale, n_pol)
        edge = project(grids.t_window_fine_derivative * sources.current, transform.projection,
                       bundle.taper_scale, n_pol)
        out["gated"], out["edge"] = gated, edge
        spectrum = spectrum + held_plasma_spectrum(gated, edge, grids.omega, grids.crop_index,
                                                   grids.active_mask)
    if raman is not None:
        out["raman_spectrum"] = np.asarray(raman)
    out["spectrum"] = spectrum
    absorb = None
    if responses.temporal_absorber_fine is not None and responses.absorber_scheme == "nonlinear":
        absorb = absorber_term(modal_t, responses.temporal_absorber_fine, None,
                               grids.crop_index, grids.active_mask, kind=kind)
        out["absorber"] = absorb
    prefactor = ws.prefactor(bundle)
    k = stage_output(spectrum, prefactor, grids.omega_window, np.ones(problem.shape), absorb)
    ref = ws.lab_source(lab, z)
    err = np.linalg.norm(k - ref) / max(np.linalg.norm(ref), 1e-300)
    assert err < 1e-13, f"pass-by-pass source differs from lab_source: {err}"
    out["source"] = ref
    return out


def source_fixture(sim, problem, zs_eval, seed):
    request = sim.run_request()
    backend = NumpyRefBackend(problem, request, grid=sim.grid, modes=sim.modes,
                              profiles=sim.profiles)
    ws = backend._workspace
    rng = np.random.default_rng(seed)
    field0 = np.broadcast_to(problem.initial.field0, problem.shape)
    n_nodes = problem.transform.synthesis.shape[0] // problem.transform._n_pol
    keep = np.unique(np.linspace(0, n_nodes - 1, min(3, n_nodes)).astype(int))
    golden = {"src.keep_nodes": keep}
    labs = [field0.copy()]
    phase = np.exp(1j * rng.uniform(-0.3, 0.3, size=problem.shape))
    scale = 1.0 + 0.2 * rng.standard_normal(problem.shape)
    labs.append(field0 * phase * scale * problem.grids.active_mask)
    for i, (lab, z) in enumerate(zip(labs, zs_eval)):
        passes = source_passes(problem, ws, lab, z, keep)
        golden[f"src{i}.lab"] = lab
        golden[f"src{i}.z"] = np.array(z)
        for key, value in passes.items():
            if i == 0 or key == "source":
                golden[f"src{i}.{key}"] = value
    return golden


def write(case, problem, golden):
    record = lower(problem)
    save_record(record, HERE / f"{case}.problem.npz")
    np.savez_compressed(HERE / f"{case}.golden.npz", **golden)
    size = sum((HERE / f"{case}.{k}.npz").stat().st_size for k in ("problem", "golden"))
    print(f"{case}: wrote {size / 1024:.0f} KiB")


def cap_case(case, *, gas, pressure, length, limits, trange, energy, fwhm, modes, n_r,
             radial_rule, fixed_dz, n_fixed_planes, seed):
    common = dict(gas=gas, pressure=pressure, length=length, n_t_limits=limits,
                  trange=trange, energy=energy, fwhm=fwhm, modes=modes, n_r=n_r,
                  radial_rule=radial_rule)
    sim = capillary(case, **common)
    problem = sim.translate()
    golden = source_fixture(sim, problem, [0.0, 0.37 * length], seed)
    # Adaptive run with the route's defaults (in-stage collar, exponential Adams).
    _, zs, states, (hist, counts), wall = drive(capillary(case, **common, n_save=3))
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s")
    # Fixed schedule without the collar, so that steps of physical size are stable.
    planes = np.linspace(0.0, length, n_fixed_planes)
    schedule = FixedSchedule.uniform(0.0, length, fixed_dz, save_planes=planes)
    fixed_sim = capillary(case, **common, absorber=False, schedule=schedule,
                          n_save=n_fixed_planes)
    fixed_problem, zs, states, (hist, counts), wall = drive(fixed_sim)
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")
    print(f"{case}: fixed run {len(hist)} steps in {wall:.2f} s")


def gnlse_case(case, seed):
    """An envelope GNLSE with Kerr, self-steepening and a Blow-Wood Raman line, DOPRI5."""
    from solprop.nonlinear.gnlse import problem_from, raman_susceptibility
    from solprop.nonlinear.raman import RamanResponse, normalised_damped_oscillator
    from solprop.pulses import GaussianPulse
    from solprop.stepper import PIController
    from solprop.translate.assembly import assemble

    length = 0.05
    grid = EnvelopeGrid.from_limits(length, 1030e-9, (700e-9, 1600e-9), 4e-12, fft_size="pow2")
    betas = [0.0, 0.0, 2.2e-26, 8e-41]
    gnlse = problem_from(betas, omega_ref=grid.omega0, gamma=0.01, raman=False,
                         raman_fraction=0.18, shock=True)
    n2 = 0.01 * 1.0 / (grid.omega0 / C0)
    line = normalised_damped_oscillator(raman_susceptibility(n2), 1.0 / 12.2e-15, 32e-15)
    raman = RamanResponse(models=(line,), fraction=0.18, thg=False)
    start = GaussianPulse(wavelength=1030e-9, fwhm=200e-15, energy=20e-9).build(grid)

    def build(save_planes, schedule=None):
        return assemble(grid, gnlse.mode, [gnlse.kerr, raman], start,
                        controller=PIController(rtol=1e-6, atol=1e-14),
                        save_planes=save_planes, dz_max=0.01, dz_init=1e-4,
                        density=1.0, shock=True, prefactor_index=1.0, schedule=schedule)

    def run(problem, request):
        backend = NumpyRefBackend(problem, request, grid=grid, modes=[gnlse.mode])
        session = backend.prepare(problem, request).start(Start.entrance(problem))
        run.policy = policy_record(session, request)
        ws = backend._workspace
        zs, states = [], []
        while not session.finished:
            batch = session.advance()
            for ev in batch.events:
                if isinstance(ev, ObservationReady):
                    zs.append(ev.z)
                    states.append(np.array(ws.committed()))
                err = getattr(ev, "error", None)
                if err is not None:
                    raise err
            session.acknowledge(batch.receipt)
        status = session.status()
        return np.array(zs), np.array(states), np.array([status.attempts, status.rejected])

    class _Sim:
        pass

    problem, request = build([0.025, length])
    sim = _Sim()
    sim.run_request = lambda: request
    sim.grid, sim.modes, sim.profiles = grid, [gnlse.mode], None
    golden = source_fixture(sim, problem, [0.0, 0.02], seed)
    zs, states, counts = run(problem, request)
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.counts": counts,
                   "adaptive.policy": run.policy})
    print(f"{case}: adaptive RK run {counts} attempts/rejected")
    planes = np.linspace(0.0, length, 11)[1:]
    fixed_problem, fixed_request = build(
        planes, FixedSchedule.uniform(0.0, length, 0.0005, save_planes=planes))
    zs, states, counts = run(fixed_problem, fixed_request)
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.policy": run.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def radial_case(case, *, n_r, length, seed):
    """The radial free-space route (``Simulation.from_free`` on a ``RadialGrid``): an
    argon filament with Kerr (the real cubic form) and ADK plasma, the in-stage collar,
    exponential Adams at the route's default rtol; the Hankel pair is square, n_r x n_r.
    The fixed schedule steps with DOPRI5, whose stability interval admits its steps under
    the in-stage collar."""
    from solprop.driver.settings import SimulationSettings
    from solprop.grid import RadialGrid
    from solprop.nonlinear.responses import KerrResponse, PlasmaResponse
    from solprop.pulses import GaussianPulse, SpatialPulse
    from solprop.spatial import SpatialMedium
    from solprop.stats import StatsSpec

    species = gas_species("Ar")
    medium = SpatialMedium(Mixture.fill({species: 1.0}, 1.0))
    eps0 = 8.8541878188e-12

    def build(schedule=None, n_save=3, integrator=None):
        grid = FieldGrid.from_limits(length, 800e-9, (350e-9, 2e-6), 150e-15, fft_size="pow2")
        responses = [KerrResponse(GAMMA3["Ar"] * eps0, thg=True), PlasmaResponse(species, adk_oracle("Ar"))]
        pulse = SpatialPulse(GaussianPulse(wavelength=800e-9, fwhm=30e-15, energy=0.5e-3), 100e-6)
        settings = SimulationSettings(backend="numpy_ref", absorber_scheme="nonlinear", boundary_check=None,
                                      ionisation_field_range=(1e7, 1e11), stats=StatsSpec(names=()),
                                      schedule=schedule, n_save=n_save, integrator=integrator)
        return Simulation.from_free(grid, RadialGrid(1.5e-3, n_r), medium, responses, pulse, settings=settings)

    sim = build()
    problem = sim.translate()
    golden = source_fixture(sim, problem, [0.0, 0.4 * length], seed)
    _, zs, states, (hist, counts), wall = drive(build())
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s", flush=True)
    # the fixed schedule: 50 DOPRI5 steps, inside the in-stage collar's stability limit for
    # that method (the explicit Adams march's is about 7 um here)
    planes = np.linspace(0.0, length, 6)
    fixed_problem, zs, states, (hist, counts), wall = drive(
        build(FixedSchedule.uniform(0.0, length, length / 50, save_planes=planes), n_save=6,
              integrator=RungeKutta()))
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def raman_case(case, *, seed):
    """A nitrogen-filled capillary with the gas's rotational and vibrational Raman response
    on the field grid (the drive E^2, the harmonic kept) and the real Kerr cubic, no plasma:
    the reference's test-only molecular constants (``tests/former_raman.py``), Börzsönyi et
    al.'s nitrogen index; two modes, n_to 4096."""
    from former_raman import FORMER_N2

    lam = np.geomspace(120e-9, 200e-6, 4000)[::-1]
    om = 2 * np.pi * C0 / lam
    l2 = (lam * 1e6) ** 2
    b1, c1, b2, c2 = 39209.95e-8, 1146.24e-6, 18806.48e-8, 13.476e-3  # N2, 1 bar, 0 C
    n2m1 = b1 * l2 / (l2 - c1) + b2 * l2 / (l2 - c2)
    rho0 = 1e5 / (K_B * 273.15)
    sus = TabulatedSusceptibility(om, (np.sqrt(1 + n2m1) - 1) / rho0, np.zeros_like(om),
                                  (121e-9, 199e-6), "Borzsonyi 2008 N2")
    nitrogen = Species("N2", sus, IdealGas(), gamma3=1.1e-52, raman=FORMER_N2)
    length = 0.05

    def build(**kw):
        fill = Mixture.fill({nitrogen: 1.0}, 3.0)
        grid = FieldGrid.from_limits(length, 800e-9, (300e-9, 3e-6), 300e-15, fft_size="pow2")
        return Simulation.from_capillary(
            125e-6, length, fill, None, wavelength=800e-9, grid=grid, fwhm=30e-15, energy=80e-6,
            cladding=1.45 + 0j, modes=2, plasma=False, raman=True, thg=True, noise=None, rtol=1e-6,
            backend="numpy_ref", boundary_check=None, **kw)

    sim = build(n_save=3)
    problem = sim.translate()
    golden = source_fixture(sim, problem, [0.0, 0.37 * length], seed)
    _, zs, states, (hist, counts), wall = drive(build(n_save=3))
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s", flush=True)
    planes = np.linspace(0.0, length, 6)
    schedule = FixedSchedule.uniform(0.0, length, length / 50, save_planes=planes)
    fixed_problem, zs, states, (hist, counts), wall = drive(build(absorber=False, schedule=schedule, n_save=6))
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def mixture_case(case, *, seed):
    """A helium-argon mixture (0.7 : 0.3 at 1 bar) in a capillary: two field-plasma
    channels, each with its own quasi-static ADK rate (the reference's test-only oracle),
    exposure scan and population, their currents formed by the reference's multi-channel
    pass; two modes, n_to 2048."""
    he, ar = gas_species("He"), gas_species("Ar")
    length = 0.02

    def build(**kw):
        fill = Mixture.fill({he: 0.7, ar: 0.3}, 1.0)
        grid = FieldGrid.from_limits(length, 800e-9, (200e-9, 4e-6), 100e-15, fft_size="pow2")
        return Simulation.from_capillary(
            125e-6, length, fill, None, wavelength=800e-9, grid=grid, fwhm=10e-15, energy=60e-6,
            cladding=1.45 + 0j, modes=2, plasma={"He": adk_oracle("He"), "Ar": adk_oracle("Ar")},
            noise=None, rtol=1e-6, backend="numpy_ref", boundary_check=None, **kw)

    sim = build(n_save=3)
    problem = sim.translate()
    assert len(problem.responses.plasma_channels) == 2
    golden = source_fixture(sim, problem, [0.0, 0.37 * length], seed)
    _, zs, states, (hist, counts), wall = drive(build(n_save=3))
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s", flush=True)
    planes = np.linspace(0.0, length, 6)
    schedule = FixedSchedule.uniform(0.0, length, length / 20, save_planes=planes)
    fixed_problem, zs, states, (hist, counts), wall = drive(build(absorber=False, schedule=schedule, n_save=6))
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def raman_mixture_case(case, *, seed):
    """A nitrogen-hydrogen mixture (0.6 : 0.4 at 3 bar) with both gases' rotational and
    vibrational Raman lines on the field grid -- two Raman components, one kernel spectrum
    with the densities inside -- beside the real Kerr cubic, no plasma: the reference's
    test-only molecular constants (``tests/former_raman.py``); Börzsönyi et al.'s
    nitrogen index and Peck and Hung's hydrogen index (J. Opt. Soc. Am. 67, 1550 (1977));
    two modes, n_to 4096."""
    from former_raman import FORMER_H2, FORMER_N2

    lam = np.geomspace(120e-9, 200e-6, 4000)[::-1]
    om = 2 * np.pi * C0 / lam
    l2 = (lam * 1e6) ** 2
    rho0 = 1e5 / (K_B * 273.15)
    b1, c1, b2, c2 = 39209.95e-8, 1146.24e-6, 18806.48e-8, 13.476e-3  # N2, 1 bar, 0 C
    n2m1 = b1 * l2 / (l2 - c1) + b2 * l2 / (l2 - c2)
    sus_n2 = TabulatedSusceptibility(om, (np.sqrt(1 + n2m1) - 1) / rho0, np.zeros_like(om),
                                     (121e-9, 199e-6), "Borzsonyi 2008 N2")
    inv = 1.0 / l2
    h2m1 = 0.0148956 / (180.7 - inv) + 0.0049037 / (92.0 - inv)  # H2, 1 atm, 0 C
    sus_h2 = TabulatedSusceptibility(om, h2m1 / (101325.0 / (K_B * 273.15)), np.zeros_like(om),
                                     (121e-9, 199e-6), "Peck and Hung 1977 H2")
    nitrogen = Species("N2", sus_n2, IdealGas(), gamma3=1.1e-52, raman=FORMER_N2)
    hydrogen = Species("H2", sus_h2, IdealGas(), gamma3=6.4e-53, raman=FORMER_H2)
    length = 0.05

    def build(**kw):
        fill = Mixture.fill({nitrogen: 0.6, hydrogen: 0.4}, 3.0)
        grid = FieldGrid.from_limits(length, 800e-9, (300e-9, 3e-6), 300e-15, fft_size="pow2")
        return Simulation.from_capillary(
            125e-6, length, fill, None, wavelength=800e-9, grid=grid, fwhm=30e-15, energy=80e-6,
            cladding=1.45 + 0j, modes=2, plasma=False, raman=True, thg=True, noise=None, rtol=1e-6,
            backend="numpy_ref", boundary_check=None, **kw)

    sim = build(n_save=3)
    problem = sim.translate()
    assert len(problem.responses.raman_terms) == 2
    golden = source_fixture(sim, problem, [0.0, 0.37 * length], seed)
    _, zs, states, (hist, counts), wall = drive(build(n_save=3))
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s", flush=True)
    planes = np.linspace(0.0, length, 6)
    schedule = FixedSchedule.uniform(0.0, length, length / 50, save_planes=planes)
    fixed_problem, zs, states, (hist, counts), wall = drive(build(absorber=False, schedule=schedule, n_save=6))
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def vector_envelope_case(case, *, seed):
    """A nitrogen-filled capillary on the envelope grid with two Cartesian field components:
    HE11 polarised along x and along y, and HE12 -- the reference's vector route, with the
    analytic Kerr cubic summed over the components and nitrogen's tensor Raman response
    (the trace and traceless kernels, three drives per node)."""
    from solprop.modes import MarcatiliMode

    he11 = MarcatiliMode(100e-6, kind="HE", n=1, m=1, cladding=1.45 + 0j)
    modes = [he11, he11.orthogonal_polarisation, MarcatiliMode(100e-6, kind="HE", n=1, m=2, cladding=1.45 + 0j)]
    envelope_modal_case(case, seed=seed, modes=modes)


def envelope_modal_case(case, *, seed, modes, integrator=None, limits=(550e-9, 1300e-9), trange=800e-15,
                        length=0.1, trim=False):
    """A nitrogen-filled capillary on the envelope grid: several modes on the radial rule's
    nodes, the analytic Kerr cubic, the gas's rotational and vibrational Raman response
    (the drive |A|^2 / 2) and the in-stage collar -- the multimode generalised NLSE of the
    reference's envelope modal route.  ``integrator`` None is the route's default march
    (exponential Adams); the fixed schedule runs without the collar."""
    from former_raman import FORMER_N2

    lam = np.geomspace(120e-9, 200e-6, 4000)[::-1]
    om = 2 * np.pi * C0 / lam
    l2 = (lam * 1e6) ** 2
    b1, c1, b2, c2 = 39209.95e-8, 1146.24e-6, 18806.48e-8, 13.476e-3  # N2, 1 bar, 0 C
    n2m1 = b1 * l2 / (l2 - c1) + b2 * l2 / (l2 - c2)
    rho0 = 1e5 / (K_B * 273.15)
    sus = TabulatedSusceptibility(om, (np.sqrt(1 + n2m1) - 1) / rho0, np.zeros_like(om),
                                  (121e-9, 199e-6), "Borzsonyi 2008 N2")
    nitrogen = Species("N2", sus, IdealGas(), gamma3=1.1e-52, raman=FORMER_N2)
    def build(**kw):
        fill = Mixture.fill({nitrogen: 1.0}, 2.0)
        grid = EnvelopeGrid.from_limits(length, 800e-9, limits, trange, fft_size="pow2")
        extra = {} if integrator is None else {"integrator": integrator}
        return Simulation.from_capillary(
            100e-6, length, fill, None, wavelength=800e-9, grid=grid, fwhm=40e-15, energy=150e-6,
            cladding=1.45 + 0j, modes=modes, raman=True, noise=None, rtol=1e-6, backend="numpy_ref",
            boundary_check=None, envelope=True, **extra, **kw)

    sim = build(n_save=3)
    problem = sim.translate()
    assert problem.grid_kind == "envelope" and problem.shape[0] == (modes if np.isscalar(modes) else len(modes))
    print(f"{case}: n_to {problem.grids.n_to}, nodes {problem.transform.synthesis.shape[0]}", flush=True)
    golden = source_fixture(sim, problem, [0.0, 0.37 * length], seed)
    _, zs, states, (hist, counts), wall = drive(build(n_save=3))
    golden.update({"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                   "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                   "adaptive.policy": drive.policy})
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.2f} s", flush=True)
    planes = np.linspace(0.0, length, 6)
    schedule = FixedSchedule.uniform(0.0, length, length / 50, save_planes=planes)
    fixed_problem, zs, states, (hist, counts), wall = drive(build(absorber=False, schedule=schedule, n_save=6))
    golden.update({"fixed.z": zs, "fixed.states": states, "fixed.history": hist,
                   "fixed.policy": drive.policy})
    if trim:  # long rows: the sources and the runs, without the first source's passes
        golden = {k: v for k, v in golden.items()
                  if not k.startswith("src0.") or k in ("src0.lab", "src0.z", "src0.source")}
    write(case, problem, golden)
    save_record(lower(fixed_problem), HERE / f"{case}_fixed.problem.npz")


def workload_case(case, *, seed, n_save=3, **common):
    """A full-size configuration: the problem, the march policy, two reference source
    evaluations, and the reference's whole adaptive run (exponential Adams at the route's
    defaults) with its states at ``n_save`` planes, its step history and its counts."""
    sim = capillary(case, **common)
    problem, request = sim.translate(), sim.run_request()
    _, zs, states, (hist, counts), wall = drive(capillary(case, **common, n_save=n_save))
    adaptive = {"adaptive.z": zs, "adaptive.states": states, "adaptive.history": hist,
                "adaptive.counts": counts, "adaptive.wall": np.array(wall),
                "adaptive.policy": drive.policy}
    print(f"{case}: adaptive run {counts} attempts/rejected in {wall:.1f} s", flush=True)
    backend = NumpyRefBackend(problem, request, grid=sim.grid, modes=sim.modes,
                              profiles=sim.profiles)
    session = backend.prepare(problem, request).start(Start.entrance(problem))
    policy = policy_record(session, request)
    ws = backend._workspace
    field0 = np.broadcast_to(problem.initial.field0, problem.shape).copy()
    rng = np.random.default_rng(seed)
    lab1 = field0 * np.exp(1j * rng.uniform(-0.3, 0.3, problem.shape)) * problem.grids.active_mask
    golden = {"adaptive.policy": policy, "fixed.policy": policy}
    for i, (lab, z) in enumerate([(field0, 0.0), (lab1, 0.4 * problem.linear.phi_breakpoints[-1])]):
        golden[f"src{i}.lab"] = lab
        golden[f"src{i}.z"] = np.array(z)
        golden[f"src{i}.source"] = ws.lab_source(lab, z)
    golden.update(adaptive)
    write(case, problem, golden)


# Config-4 scan points built by the reference's own capillary translation (its defaults:
# Gauss-Kronrod radial rule, band-rule running integrals, in-stage collar), with the
# reference's input shot noise drawn from each point's seed.  The corner of the scan's
# distribution is here: eight modes on a 32768-sample grid.
SCAN_POINTS = [
    # radius, length, gas, pressure (bar), energy, fwhm, modes, n_to, seed
    (100e-6, 1.2, "He", 1.5, 150e-6, 12e-15, 8, 32768, 11),
    (60e-6, 0.6, "Ar", 2.5, 300e-6, 8e-15, 1, 4096, 12),
    (140e-6, 1.8, "Ne", 0.5, 60e-6, 25e-15, 4, 16384, 13),
    (110e-6, 1.0, "Ar", 1.0, 40e-6, 20e-15, 3, 8192, 14),
]
SCAN_ATTEMPTS = 24


def scan_point_sim(radius, length, gas, pressure, energy, fwhm, modes, n_to, seed, n_save=2):
    """One scan point through ``Simulation.from_capillary``: constant pressure, 800 nm,
    the 150 nm - 4 um band on a pow2 field grid of ``n_to`` fine samples."""
    omega_max = 2 * np.pi * C0 / 150e-9
    dt_fine = 2 * np.pi / (6.0 * omega_max)  # the grid's default ffac of 6
    # a request 0.75 n_to dt_fine wide after the outside collars rounds up to n_to
    trange = 0.8 * 0.75 * n_to * dt_fine
    grid = FieldGrid.from_limits(length, 800e-9, (150e-9, 4e-6), trange, fft_size="pow2")
    assert grid.n_to == n_to, (grid.n_to, n_to)
    fill = Mixture.fill({gas_species(gas): 1.0}, pressure)
    return Simulation.from_capillary(
        radius, length, fill, None, wavelength=800e-9, grid=grid, fwhm=fwhm, energy=energy,
        cladding=1.45 + 0j, modes=modes, plasma=adk_oracle(gas), noise="input", seed=seed,
        rtol=1e-6, n_save=n_save, backend="numpy_ref", boundary_check=None)


def scan_case(index, params):
    """The lowered problem, the launch state, one source evaluation and the state after
    ``SCAN_ATTEMPTS`` adaptive exponential-Adams attempts of one scan point."""
    case = f"scan{index}"
    sim = scan_point_sim(*params)
    problem, request = sim.translate(), sim.run_request()
    backend = NumpyRefBackend(problem, request, grid=sim.grid, modes=sim.modes,
                              profiles=sim.profiles)
    session = backend.prepare(problem, request).start(Start.entrance(problem))
    golden = {"adaptive.policy": policy_record(session, request), "params": np.array(params[:2] + params[3:], float),
              "gas": np.frombuffer(params[2].encode(), np.uint8)}
    from solprop.translate.linop import power_weight_at

    # the draw enters the problem divided by the root of this row (driver/inputs.py:484-488)
    golden["power_weight"] = np.asarray(power_weight_at(problem, 0.0))
    ws = backend._workspace
    golden["launch"] = np.array(ws.committed())
    golden["src0.lab"] = golden["launch"]
    golden["src0.z"] = np.array(0.0)
    golden["src0.source"] = ws.lab_source(golden["launch"], 0.0)
    t0 = time.time()
    done = 0
    while done < SCAN_ATTEMPTS:
        batch = session.advance(work_limit=SCAN_ATTEMPTS - done)
        session.acknowledge(batch.receipt)
        done = int(session.status().attempts)
    status = session.status()
    golden["attempts.state"] = np.array(ws.committed())
    golden["attempts.counts"] = np.array([status.attempts, status.rejected])
    print(f"{case}: {status.attempts} attempts ({status.rejected} rejected) in "
          f"{time.time() - t0:.1f} s, {problem.transform.synthesis.shape[0]} nodes", flush=True)
    write(case, problem, golden)


def stats_case(case):
    """The reference's own plane statistics (``stats/definitions.py``: energy, omega0,
    peak_power, peak_power_total; ``fourier.energy_weights`` times the columns' summed
    |a|^2 for the energy per bin) of a fixture's last stored state -- the adaptive run's
    last plane, or a scan point's state after its attempts -- added to its golden file as
    ``stats.*``."""
    from solprop import fourier
    from solprop.stats import definitions as D

    path = HERE / f"{case}.golden.npz"
    golden = dict(np.load(path))
    if case == "gnlse_raman":
        grid = EnvelopeGrid.from_limits(0.05, 1030e-9, (700e-9, 1600e-9), 4e-12, fft_size="pow2")
        state = golden["adaptive.states"][-1]
    elif case.startswith("scan"):
        grid = scan_point_sim(*SCAN_POINTS[int(case[4:])]).grid
        state = golden["attempts.state"]
    else:
        params = {"cap4_he": dict(gas="He", pressure=(0.8, 0.0), length=0.05, n_t_limits=(150e-9, 4e-6),
                                  trange=150e-15, energy=100e-6, fwhm=7.5e-15, modes=4, n_r=16,
                                  radial_rule="gauss"),
                  "config2": dict(gas="He", pressure=(0.8, 0.0), length=1.5, n_t_limits=(90e-9, 4e-6),
                                  trange=400e-15, energy=275e-6, fwhm=7.5e-15, modes=4, n_r=64,
                                  radial_rule="gauss", deep_uv=True)}[case]
        grid = capillary(case, **params).grid
        state = golden["adaptive.states"][-1]
    golden["stats.energy"] = np.asarray(D.energy(grid, state))
    golden["stats.omega0"] = np.asarray(D.omega0(grid, state))
    golden["stats.peak_power"] = np.asarray(D.peak_power(grid, state))
    golden["stats.peak_power_total"] = np.asarray(D.peak_power_total(grid, state))
    weights = fourier.energy_weights(grid.n_omega, grid.dt, kind=grid.kind)
    golden["stats.spectrum"] = weights * np.sum(np.abs(state) ** 2, axis=(0, 1))
    np.savez_compressed(path, **golden)
    print(f"{case}: statistics added", flush=True)


if __name__ == "__main__":
    only = set(sys.argv[1:])
    if not only or "cap1_ar" in only:
        cap_case("cap1_ar", gas="Ar", pressure=1.0, length=0.02, limits=(200e-9, 4e-6),
                 trange=100e-15, energy=30e-6, fwhm=10e-15, modes=1, n_r=None,
                 radial_rule="gauss_kronrod", fixed_dz=0.001, n_fixed_planes=11, seed=1)
    if not only or "cap4_he" in only:
        cap_case("cap4_he", gas="He", pressure=(0.8, 0.0), length=0.05, limits=(150e-9, 4e-6),
                 trange=150e-15, energy=100e-6, fwhm=7.5e-15, modes=4, n_r=16,
                 radial_rule="gauss", fixed_dz=0.005, n_fixed_planes=11, seed=2)
    if not only or "cap12_ne" in only:
        # twelve modes: more modal columns than the fused column holds (the GEMM route)
        cap_case("cap12_ne", gas="Ne", pressure=1.5, length=0.02, limits=(200e-9, 4e-6),
                 trange=100e-15, energy=60e-6, fwhm=10e-15, modes=12, n_r=96,
                 radial_rule="gauss", fixed_dz=0.001, n_fixed_planes=6, seed=6)
    if not only or "raman_n2" in only:
        raman_case("raman_n2", seed=8)
    if not only or "mix_hear" in only:
        mixture_case("mix_hear", seed=9)
    if not only or "raman_mix" in only:
        raman_mixture_case("raman_mix", seed=10)
    if not only or "env4_n2" in only:
        envelope_modal_case("env4_n2", seed=11, modes=4)
    if not only or "envv_n2" in only:
        vector_envelope_case("envv_n2", seed=13)
    if not only or "env2_8k" in only:
        # rows of 8192 envelope samples: the products route's longest
        envelope_modal_case("env2_8k", seed=14, modes=2, limits=(400e-9, 2000e-9), trange=6.4e-12, length=0.05)
    if not only or "env2_16k" in only:
        # rows of 16384 envelope samples: FP64 rows split into halves through a scratch
        envelope_modal_case("env2_16k", seed=15, modes=2, limits=(400e-9, 2000e-9), trange=12.8e-12, length=0.02,
                            trim=True)
    if not only or "env3_rk" in only:
        envelope_modal_case("env3_rk", seed=12, modes=3, integrator=RungeKutta())
    if not only or "radial_ar" in only:
        # the radial free-space route on 48 radial nodes (a 48 x 48 Hankel pair)
        radial_case("radial_ar", n_r=48, length=0.01, seed=7)
    if not only or "gnlse_raman" in only:
        gnlse_case("gnlse_raman", seed=3)
    if not only or "config2" in only:
        # config 2: He 125 um, 1.5 m, 0.8 -> 0 bar, 800 nm, 7.5 fs, 275 uJ,
        # HE11-HE14, 90 nm - 4 um, 400 fs, pow2 grid (n_to 16384), 64 Gauss nodes
        workload_case("config2", seed=4, gas="He", pressure=(0.8, 0.0), length=1.5,
                      n_t_limits=(90e-9, 4e-6), trange=400e-15, energy=275e-6, fwhm=7.5e-15,
                      modes=4, n_r=64, radial_rule="gauss", deep_uv=True)
    if not only or "config1" in only:
        # config 1: Ar 125 um, 1 m, 1 bar, 800 nm, 10 fs, 100 uJ, HE11,
        # 150 nm - 4 um, 400 fs, pow2 grid (n_to 8192)
        workload_case("config1", seed=5, gas="Ar", pressure=1.0, length=1.0,
                      n_t_limits=(150e-9, 4e-6), trange=400e-15, energy=100e-6, fwhm=10e-15,
                      modes=1)
    for i, params in enumerate(SCAN_POINTS):
        if not only or f"scan{i}" in only or "scan" in only:
            scan_case(i, params)
    for case in ("cap4_he", "config2", "gnlse_raman", "scan0"):
        if not only or f"stats_{case}" in only or "stats" in only:
            stats_case(case)

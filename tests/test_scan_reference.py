"""Scan points built by the reference's own translation: the batched solver against them.

``tests/golden/generate.py`` builds four config-4 scan points through the reference's
``Simulation.from_capillary`` (its defaults: Gauss-Kronrod radial rule, band-rule running
integrals, in-stage collar, input shot noise drawn from the point's seed), including the
distribution's corner -- eight modes on a 32768-sample grid -- and records the launch
state, one source evaluation and the state after 24 adaptive exponential-Adams attempts
of the reference's ``numpy_ref`` backend.

On the CPU: the restated shot-noise draw (``scan.input_noise``) gives the reference's
realisation bit for bit, and the oracle reproduces the reference's launch state, source
evaluation and attempts.  On the GPU: a batched scan of the four runs, in both column
forms and with the transforms in one CTA per row or over clusters, lands every run on
the reference's state after 24 attempts at 1e-10 relative L2, with the reference's
attempt and rejection counts.
"""

import numpy as np
import pytest

from oracle import march as M
from oracle import source as S
from solprop_b200 import scan
from tests._cases import golden, policy, record, rel

CASES = ("scan0", "scan1", "scan2", "scan3")
STEP_TOL = 1e-10


def _point(case):
    g = golden(case)
    radius, length, pressure, energy, fwhm, modes, n_to, seed = g["params"]
    return g, int(modes), int(n_to), int(seed)


@pytest.mark.parametrize("case", CASES)
def test_shot_noise_is_the_references_draw(case):
    rec = record(case)
    g, modes, n_to, seed = _point(case)
    assert rec.n_modes == modes and rec.n_to == n_to and rec.noise_model == "input"
    d_omega = float(rec.omega[1] - rec.omega[0])
    draw = scan.input_noise(rec.omega, rec.active_mask, rec.dt, d_omega,
                            np.random.default_rng(seed), n_modes=rec.n_modes, n_pol=rec.n_pol)
    # the problem holds it in the vacuum-normalised amplitude: divided by the root of the
    # modes' power weight at the entrance
    assert np.array_equal(draw / np.sqrt(g["power_weight"]), rec.noise0)
    # the launch state is the pulse plus the draw, as the reference starts it
    assert rel(rec.launch_field(), g["launch"]) < 1e-14


@pytest.mark.parametrize("case", CASES)
def test_oracle_source_matches_the_reference(case):
    rec = record(case)
    g = golden(case)
    assert rel(S.lab_source(rec, g["src0.lab"], 0.0), g["src0.source"]) < 1e-13


@pytest.mark.parametrize("case", ["scan1", "scan3"])
def test_oracle_attempts_match_the_reference(case):
    rec = record(case)
    g = golden(case)
    pol = policy(g, "adaptive")
    ws = M.Workspace(rec)
    march = M.AdamsMarch(M.AdamsEngine(ws, pol), pol, pol["proposal"])
    while march.attempts < int(g["attempts.counts"][0]):
        march.attempt_towards(rec.z_end)
    assert march.rejected == int(g["attempts.counts"][1])
    assert rel(ws.state, g["attempts.state"]) < 1e-13


# the transforms' forms per grid size, (inverse, forward): 0 is one CTA per row, k a
# cluster of k CTAs; an FP64 row of 32768 samples needs 2 CTAs inverse and 4 forward
NARROW = {4096: (0, 0), 8192: (0, 0), 16384: (0, 0), 32768: (2, 4)}
WIDE = {8192: (2, 2), 16384: (4, 4), 32768: (4, 8)}


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["tiles", "sweep"])
@pytest.mark.parametrize("transforms", ["narrow", "wide"])
def test_batched_scan_matches_the_reference_after_24_attempts(form, transforms):
    from solprop_b200 import _lib

    recs = [record(c) for c in CASES]
    pols = [policy(golden(c), "adaptive") for c in CASES]
    sc = _lib.Scan(recs, pols)
    sc.set_column(form)
    for n_to, (inverse, forward) in (NARROW if transforms == "narrow" else WIDE).items():
        sc.set_transforms(n_to, inverse, forward)
    steps = int(golden(CASES[0])["attempts.counts"][0])
    sc.advance(steps)
    for i, case in enumerate(CASES):
        g = golden(case)
        state, info = sc.run(i)
        assert info.attempts == int(g["attempts.counts"][0]), case
        assert info.rejected == int(g["attempts.counts"][1]), case
        assert rel(state, g["attempts.state"]) < STEP_TOL, case
    sc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_single_run_matches_the_reference_after_24_attempts(case):
    from solprop_b200 import _lib

    rec = record(case)
    g = golden(case)
    problem = _lib.Problem(rec)
    ws = _lib.Workspace(problem)
    session = ws.start(policy(g, "adaptive"))
    for _ in range(int(g["attempts.counts"][0])):
        batch = session.advance(1)
    assert batch.attempts == int(g["attempts.counts"][0])
    assert batch.rejected == int(g["attempts.counts"][1])
    assert rel(session.export(), g["attempts.state"]) < STEP_TOL

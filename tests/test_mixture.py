"""Gas mixtures against the reference: several plasma channels, several Raman components.

``mix_hear`` is a helium-argon capillary with two field-plasma channels: each channel has
its own rate table and exposure scan, the channels' weights and works are summed before
the one free-current integral (``passes/plasma.py:326-485``).  ``raman_mix`` is a
nitrogen-hydrogen capillary with two Raman components folded into one kernel spectrum,
their densities inside it (``passes/responses.py:293-334``).  The oracle's own pins are in
``tests/test_oracle_golden.py``; here the record, the refusals and the device.
"""

import ctypes as C
import io

import numpy as np
import pytest

from solprop_b200.record import load_record, save_record
from tests._cases import fixed_schedule, golden, policy, record, rel

SOURCE_TOL = 1e-10  # the plain form, as every source test
MIXED_TOL = 2e-6  # the mixed form's source tolerance (tests/test_mixed.py)


def test_the_record_keeps_every_channel_and_component():
    for case, n_channels, n_raman in (("mix_hear", 1, 0), ("raman_mix", 0, 1)):
        rec = record(case)
        assert len(rec.extra_channels) == n_channels and len(rec.extra_raman) == n_raman
        buf = io.BytesIO()
        save_record(rec, buf)
        buf.seek(0)
        back = load_record(buf)
        for a, b in zip(rec.extra_channels, back.extra_channels):
            assert np.array_equal(a.rate_coefficients, b.rate_coefficients)
            assert a.ionisation_potential == b.ionisation_potential
            assert np.array_equal(a.plasma_density.coefficients, b.plasma_density.coefficients)
        for a, b in zip(rec.extra_raman, back.extra_raman):
            assert np.array_equal(a.undamped, b.undamped) and a.fraction == b.fraction
            assert len(a.rates) == len(b.rates)


def test_mixtures_are_refused_where_one_channel_is_built():
    from solprop_b200 import _lib

    rec, g = record("mix_hear"), golden("mix_hear")
    problem = _lib.Problem(rec)
    with pytest.raises(_lib.BackendRefusal, match="one plasma channel"):
        _lib.Scan([rec], [policy(g, "adaptive")])
    lab = np.zeros(rec.n_cols * rec.n_omega * 2)
    with pytest.raises(_lib.BackendRefusal, match="one plasma channel"):
        _lib.check(_lib.library().sp_source_noalloc(problem.handle, C.c_void_p(lab.ctypes.data), 0.0, 0,
                                                    C.c_void_p(lab.ctypes.data), None))
    rec = record("raman_mix")
    with pytest.raises(_lib.BackendRefusal, match="field-grid Raman takes the modal"):
        _lib.Workspace(_lib.Problem(rec), 0, "fp64", modal="fused")


@pytest.mark.gpu
@pytest.mark.parametrize("case,modal", [("mix_hear", "fused"), ("mix_hear", "gemm"), ("raman_mix", "auto")])
@pytest.mark.parametrize("index", [0, 1])
def test_source_matches_the_reference(case, modal, index):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec), 0, "fp64", modal=modal)
    got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
    assert rel(got, g[f"src{index}.source"]) < SOURCE_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case,modal", [("mix_hear", "fused"), ("mix_hear", "gemm"), ("raman_mix", "auto")])
def test_mixed_source_matches_the_reference_to_fp32(case, modal):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec), 0, "mixed", modal=modal)
    for index in (0, 1):
        got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
        assert rel(got, g[f"src{index}.source"]) < MIXED_TOL, index


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["mix_hear", "raman_mix"])
def test_mixture_runs_step_with_the_reference(case):
    """A fixed schedule plane by plane at 1e-10, and the adaptive run within its rtol with
    the reference's attempt count (to +-3)."""
    from solprop_b200 import _lib

    rec, g = record(case, fixed=True), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec))
    steps, _ = fixed_schedule(g)
    session = ws.start(policy(g, "fixed"), schedule=steps)
    zs, states = g["fixed.z"], g["fixed.states"]
    plane = 1
    while True:
        batch = session.advance(1)
        if plane < len(zs) and abs(batch.z - zs[plane]) < 1e-12:
            assert rel(session.export(), states[plane]) < 1e-10, plane
            plane += 1
        if batch.event in (2, 3):
            break
    assert plane == len(zs)
    rec = record(case)
    ws = _lib.Workspace(_lib.Problem(rec))
    pol = policy(g, "adaptive")
    session = ws.start(pol)
    zs, states = g["adaptive.z"], g["adaptive.states"]
    seen = 1
    while True:
        batch = session.advance(256)
        assert batch.event != 3
        if batch.event in (1, 2):
            assert rel(session.export(), states[seen]) < pol["rtol"]
            seen += 1
        if batch.event == 2:
            break
    assert seen == len(zs)
    assert abs(batch.attempts - int(g["adaptive.counts"][0])) <= 3

"""The gas's Raman response on the field grid against the reference.

``raman_n2`` is a nitrogen-filled capillary (two modes, 33 nodes, n_to 4096) with the
rotational and vibrational Raman lines on the field grid -- the drive ``E^2`` with the
harmonic kept, the convolution on the doubled grid -- beside the real Kerr cubic.  The
response is added node by node to the polarisation the response column writes, so the run
takes the modal transform's products (the route that keeps the node field in HBM): a
workspace chooses it by itself and the fused column refuses the problem by name.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import source as S
from tests._cases import fixed_schedule, golden, policy, record, rel

SOURCE_TOL = 1e-10  # the plain form, as every source test
MIXED_TOL = 2e-6  # the mixed form's source tolerance (tests/test_mixed.py)


def test_oracle_matches_the_reference():
    rec, g = record("raman_n2"), golden("raman_n2")
    assert rec.raman_enabled and rec.raman_thg and rec.grid_kind == "field"
    for i in (0, 1):
        assert rel(S.lab_source(rec, g[f"src{i}.lab"], float(g[f"src{i}.z"])), g[f"src{i}.source"]) < 1e-13


def test_oracle_kernel_spectrum_matches_the_reference():
    rec, g = record("raman_n2"), golden("raman_n2")
    sc = S.stage_scalars(rec, float(g["src0.z"]), float(g["src0.z"]))
    assert rel(S.raman_spectrum(rec, sc.raman_rates), g["src0.raman_spectrum"]) < 1e-13


def test_field_raman_is_refused_where_the_fused_transform_is_the_only_one():
    from solprop_b200 import _lib

    rec, g = record("raman_n2"), golden("raman_n2")
    problem = _lib.Problem(rec)  # the problem itself is taken
    with pytest.raises(_lib.BackendRefusal, match="field-grid Raman takes the modal"):
        _lib.Workspace(problem, 0, "fp64", modal="fused")
    with pytest.raises(_lib.BackendRefusal, match="no field-grid Raman"):
        _lib.Scan([rec], [policy(g, "adaptive")])
    lab = np.zeros(rec.n_cols * rec.n_omega * 2)
    with pytest.raises(_lib.BackendRefusal, match="no field-grid Raman"):
        _lib.check(_lib.library().sp_source_noalloc(problem.handle, C.c_void_p(lab.ctypes.data), 0.0, 0,
                                                    C.c_void_p(lab.ctypes.data), None))


@pytest.mark.gpu
@pytest.mark.parametrize("index", [0, 1])
def test_source_matches_the_reference(index):
    from solprop_b200 import _lib

    rec, g = record("raman_n2"), golden("raman_n2")
    ws = _lib.Workspace(_lib.Problem(rec))  # field-grid Raman: the products, by itself
    got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
    assert rel(got, g[f"src{index}.source"]) < SOURCE_TOL


@pytest.mark.gpu
def test_mixed_source_matches_the_reference_to_fp32():
    from solprop_b200 import _lib

    rec, g = record("raman_n2"), golden("raman_n2")
    ws = _lib.Workspace(_lib.Problem(rec), 0, "mixed")
    for index in (0, 1):
        got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
        assert rel(got, g[f"src{index}.source"]) < MIXED_TOL, index


@pytest.mark.gpu
def test_raman_run_steps_with_the_reference():
    """A fixed schedule plane by plane at 1e-10, and the adaptive run within its rtol with
    the reference's attempt count (to +-3)."""
    from solprop_b200 import _lib

    rec, g = record("raman_n2", fixed=True), golden("raman_n2")
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
    rec = record("raman_n2")
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

"""The radial free-space route (the reference's ``Simulation.from_free`` on a RadialGrid).

Its transform is a square Hankel pair -- 48 radial nodes, 48 spectral columns here -- so
the workspace takes the modal transform's products by itself.  The reference projects the
radial plasma after the nodes' transforms (``backends/numpy_ref/source.py:702-735``); the
device projects in time and transforms per column, the same linear maps in the other order,
equal to rounding.  The fixture (``tests/golden/generate.py radial_ar``): an argon filament
with the real cubic Kerr form and ADK plasma under the in-stage collar; source evaluations,
a DOPRI5 fixed schedule and an exponential-Adams adaptive run of the reference.
"""

import numpy as np
import pytest

from oracle import source as S
from tests._cases import fixed_schedule, golden, policy, record, rel


def test_oracle_matches_the_reference():
    rec, g = record("radial_ar"), golden("radial_ar")
    assert rec.n_modes == rec.n_nodes == 48
    for i in (0, 1):
        assert rel(S.lab_source(rec, g[f"src{i}.lab"], float(g[f"src{i}.z"])), g[f"src{i}.source"]) < 1e-13


def test_the_radial_collar_and_split_step_absorbers_are_refused_by_name():
    from solprop_b200.lowering import BackendRefusal, lower

    class _Stub:  # only the fields the refusals read
        pass

    problem = _Stub()
    problem.grids = problem.linear = problem.route = None
    problem.shape = (1, 1, 3)
    problem.transform = _Stub()
    problem.transform.modal_tables = None
    problem.transform.kind = "radial"
    problem.transform.geometry = _Stub()
    problem.transform.geometry.kind = "radial"
    problem.transform.geometry.absorber_rate = np.array([0.0, 1.0])
    problem.responses = _Stub()
    problem.initial = None
    with pytest.raises(BackendRefusal, match="radial spatial absorber"):
        lower(problem)
    problem.transform.geometry.absorber_rate = np.zeros(2)
    problem.responses.temporal_absorber_fine = np.ones(4)
    problem.responses.absorber_scheme = "split_step"
    with pytest.raises(BackendRefusal, match="split_step"):
        lower(problem)


@pytest.mark.gpu
@pytest.mark.parametrize("index", [0, 1])
def test_source_matches_the_reference(index):
    from solprop_b200 import _lib

    rec, g = record("radial_ar"), golden("radial_ar")
    problem = _lib.Problem(rec)
    ws = _lib.Workspace(problem)  # 48 columns: the products, by itself
    assert rel(ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"])), g[f"src{index}.source"]) < 1e-10
    mixed = _lib.Workspace(problem, 0, "mixed")
    assert rel(mixed.source(g[f"src{index}.lab"], float(g[f"src{index}.z"])), g[f"src{index}.source"]) < 1e-5


@pytest.mark.gpu
def test_fixed_schedule_and_adaptive_run_match_the_reference():
    from solprop_b200 import _lib

    g = golden("radial_ar")
    ws = _lib.Workspace(_lib.Problem(record("radial_ar", fixed=True)))
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
    ws = _lib.Workspace(_lib.Problem(record("radial_ar")))
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

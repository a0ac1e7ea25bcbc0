"""Pin the oracle to the reference: its outputs against the golden vectors.

The golden vectors are the reference's own ``numpy_ref`` backend run on the fixture
problems (``tests/golden/generate.py``); the oracle restates that arithmetic, so the
bar is rounding: 1e-13 relative L2 for one source evaluation and per fixed step, and
identical step decisions on the adaptive runs.
"""

import numpy as np
import pytest

from oracle import march as M
from oracle import source as S
from tests._cases import CASES, fixed_schedule, golden, policy, record, rel


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("index", [0, 1])
def test_source_matches_reference(case, index):
    rec, g = record(case), golden(case)
    got = S.lab_source(rec, g[f"src{index}.lab"], float(g[f"src{index}.z"]))
    assert rel(got, g[f"src{index}.source"]) < 1e-13


def test_source_passes_match_reference():
    rec, g = record("cap1_ar"), golden("cap1_ar")
    out = {}
    S.lab_source(rec, g["src0.lab"], float(g["src0.z"]), out=out)
    keep = g["src.keep_nodes"]
    assert rel(out["modal_t"], g["src0.modal_t"]) < 1e-14
    assert rel(out["field_t"][keep], g["src0.field_nodes"]) < 1e-14
    assert rel(out["rate"][keep], g["src0.rate_nodes"]) < 1e-13
    assert rel(out["fraction"][keep], g["src0.fraction_nodes"]) < 1e-13
    assert rel(out["current"][keep], g["src0.current_nodes"]) < 1e-13
    assert rel(out["projected"], g["src0.projected"]) < 1e-13
    assert rel(out["gated"], g["src0.gated"]) < 1e-13
    assert rel(out["edge"], g["src0.edge"]) < 1e-13
    assert rel(out["spectrum"], g["src0.spectrum"]) < 1e-13
    assert rel(out["absorber"], g["src0.absorber"]) < 1e-13


def _march(rec, pol):
    ws = M.Workspace(rec)
    if pol["march"] == "HostAdamsMarch":
        return ws, M.AdamsMarch(M.AdamsEngine(ws, pol), pol, pol["proposal"])
    return ws, M.RungeKuttaMarch(M.RungeKuttaEngine(ws, pol["controller"]), pol, pol["proposal"])


@pytest.mark.parametrize("case", CASES)
def test_fixed_schedule_matches_reference(case):
    g = golden(case)
    rec, pol = record(case, fixed=True), policy(g, "fixed")
    ws, march = _march(rec, pol)
    steps, edges = fixed_schedule(g)
    zs, states = g["fixed.z"], g["fixed.states"]
    plane = 1
    for i, dz in enumerate(steps):
        march.replay(steps[i:i + 1], edges[i:i + 2])
        if plane < len(zs) and abs(march.z - zs[plane]) < 1e-12:
            assert rel(ws.state, states[plane]) < 1e-13, (case, plane)
            plane += 1
    assert plane == len(zs)


@pytest.mark.parametrize("case", CASES)
def test_adaptive_run_matches_reference(case):
    g = golden(case)
    rec, pol = record(case), policy(g, "adaptive")
    ws, march = _march(rec, pol)
    for i, zt in enumerate(g["adaptive.z"]):
        if i:
            march.march_to(float(zt))
        assert rel(ws.state, g["adaptive.states"][i]) < 1e-13
    assert [march.attempts, march.rejected] == list(g["adaptive.counts"])


def test_phi_functions_near_and_far_agree_with_augmented_exponential():
    # phi_k(x) by the definition's recurrence at a point where both branches are exact
    from scipy.linalg import expm
    for x in (0.3 + 0.2j, -2.9 + 0.1j, 3.1 - 1j, -40 + 5j, 1e-6j):
        phi = M.phi_functions(np.array([x]), 4)[:, 0]
        aug = np.zeros((5, 5), dtype=complex)
        aug[0, 0] = x
        for k in range(4):
            aug[k, k + 1] = 1.0
        e = expm(aug)
        ref = np.array([e[0, 0], *e[0, 1:5]])
        assert np.allclose(phi, ref, rtol=1e-13, atol=1e-15)


def test_lagrange_basis_is_cardinal():
    nodes = [1.0, 0.0, -0.7, -1.9, -2.4]
    c = M.lagrange_coefficients(nodes)
    vander = np.vander(np.array(nodes), increasing=True)
    assert np.allclose(c @ vander.T, np.eye(5), atol=1e-12)
    assert np.allclose(M.integrated_weights([1.0, 0.0, -1.0, -2.0]) * 24, [9, 19, -5, 1])

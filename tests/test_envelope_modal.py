"""The envelope grid's modal route with many modes and nodes, against the reference.

``env4_n2`` and ``env3_rk`` are nitrogen-filled capillaries on the envelope grid: four and
three modes on 33 radial nodes, n_to 1024, the analytic Kerr cubic, the gas's Raman
response (drive |A|^2 / 2) and the in-stage collar -- the multimode generalised NLSE,
stepped by exponential Adams and by DOPRI5.  ``envv_n2`` has two Cartesian field
components (HE11 along x and along y, HE12): the Kerr cubic summed over the components and
nitrogen's tensor Raman response (trace and traceless kernels, three drives per node).
``env2_8k`` and ``env2_16k`` have rows of 8 192 and 16 384 samples (config 3's count): the
FP64 rows of 16 384 take two halves of shared memory and a global scratch.  A workspace takes the modal transform's
products for them by itself (complex rows interleaved, N = 2 n_to); the single-CTA
envelope kernel, which holds one column on one node, refuses them by name.
"""

import pytest

from tests._cases import fixed_schedule, golden, policy, record, rel

SOURCE_TOL = 1e-10  # the plain form, as every source test
MIXED_TOL = 2e-6  # the mixed form's source tolerance (tests/test_mixed.py)


def test_oracle_matches_the_reference_on_rows_of_8192():
    """The oracle on ``env2_8k``: sources at 1e-13, the fixed schedule's planes at 1e-13, and
    the adaptive run with the reference's attempt and rejection counts, its planes within
    1e-7 (the other cases agree to 1e-13: at this length the run's sensitivity carries
    rounding differences of the transforms to the 1e-8 level)."""
    from oracle import march as M
    from oracle import source as S

    rec, g = record("env2_8k"), golden("env2_8k")
    for i in (0, 1):
        assert rel(S.lab_source(rec, g[f"src{i}.lab"], float(g[f"src{i}.z"])), g[f"src{i}.source"]) < 1e-13
    pol = policy(g, "adaptive")
    ws = M.Workspace(rec)
    march = M.AdamsMarch(M.AdamsEngine(ws, pol), pol, pol["proposal"])
    for i, zt in enumerate(g["adaptive.z"]):
        if i:
            march.march_to(float(zt))
        assert rel(ws.state, g["adaptive.states"][i]) < 1e-7
    assert [march.attempts, march.rejected] == list(g["adaptive.counts"])


def test_oracle_matches_the_reference_on_rows_of_16384():
    from oracle import source as S

    rec, g = record("env2_16k"), golden("env2_16k")
    assert rec.n_to == 16384
    for i in (0, 1):
        assert rel(S.lab_source(rec, g[f"src{i}.lab"], float(g[f"src{i}.z"])), g[f"src{i}.source"]) < 1e-13


def test_two_components_are_taken_on_the_envelope_grid_only():
    from solprop_b200 import _lib

    rec = record("envv_n2")
    assert rec.n_pol_transform == 2 and rec.raman_tensor_weights.shape == (2, 2)
    _lib.Problem(rec).close()
    rec.grid_kind = "field"
    with pytest.raises(_lib.BackendRefusal, match="two field components on the field grid"):
        _lib.Problem(rec)


def test_many_modes_are_refused_by_the_single_cta_form():
    from solprop_b200 import _lib

    problem = _lib.Problem(record("env4_n2"))
    with pytest.raises(_lib.BackendRefusal, match="envelope grid's modes, nodes, in-stage absorber"):
        _lib.Workspace(problem, 0, "fp64", modal="fused")
    single = _lib.Problem(record("gnlse_raman"))
    with pytest.raises(_lib.BackendRefusal, match="mixed precision of the envelope route takes"):
        _lib.Workspace(single, 0, "mixed", modal="fused")


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["env4_n2", "env3_rk", "envv_n2", "env2_8k", "env2_16k"])
@pytest.mark.parametrize("index", [0, 1])
def test_source_matches_the_reference(case, index):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec))
    got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
    assert rel(got, g[f"src{index}.source"]) < SOURCE_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["env4_n2", "env3_rk", "envv_n2", "env2_8k", "env2_16k", "gnlse_raman"])
def test_split_bf16_products_match_the_reference_to_fp32(case):
    """The mixed form: tcgen05 products of three-part BF16 splits, FP32 responses."""
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec), 0, "mixed")
    for index in (0, 1):
        got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
        assert rel(got, g[f"src{index}.source"]) < MIXED_TOL, index


@pytest.mark.gpu
def test_mixed_envelope_run_stays_near_the_reference():
    """The adaptive Adams run in the mixed form: every plane within 1e-5 of the reference."""
    from solprop_b200 import _lib

    rec, g = record("env4_n2"), golden("env4_n2")
    session = _lib.Workspace(_lib.Problem(rec), 0, "mixed").start(policy(g, "adaptive"))
    zs, states = g["adaptive.z"], g["adaptive.states"]
    seen = 1
    while True:
        batch = session.advance(256)
        assert batch.event != 3
        if batch.event in (1, 2):
            assert rel(session.export(), states[seen]) < 1e-5
            seen += 1
        if batch.event == 2:
            break
    assert seen == len(zs)


@pytest.mark.gpu
def test_the_single_mode_envelope_gives_the_same_source_on_either_form():
    """The GNLSE fixture (one column, one node) through the single CTA and the products."""
    from solprop_b200 import _lib

    rec, g = record("gnlse_raman"), golden("gnlse_raman")
    problem = _lib.Problem(rec)
    got = [_lib.Workspace(problem, 0, "fp64", modal=m).source(g["src1.lab"], float(g["src1.z"]))
           for m in ("fused", "gemm")]
    assert rel(got[1], g["src1.source"]) < SOURCE_TOL
    assert rel(got[1], got[0]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["env4_n2", "env3_rk", "envv_n2", "env2_8k", "env2_16k"])
def test_envelope_runs_step_with_the_reference(case):
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

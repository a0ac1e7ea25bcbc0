"""The modal transform as dense products (the GEMM route) against the reference.

The route takes the synthesis and the projection out of the response column: FP64
products in the plain form; in the mixed form tcgen05 products of three-part BF16 splits of
every operand, accumulated in FP32.  ``cap12_ne`` has twelve modes -- more modal columns than
the fused column holds -- so a workspace takes the route by itself; the other cases are
forced onto it and compared with the reference and with the fused route.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import source as S
from tests._cases import fixed_schedule, golden, policy, record, rel

SOURCE_TOL = 1e-10  # the plain form, as every source test
MIXED_TOL = 2e-6  # the mixed form's source tolerance (tests/test_mixed.py)


def test_oracle_matches_the_reference_on_twelve_modes():
    rec, g = record("cap12_ne"), golden("cap12_ne")
    for i in (0, 1):
        assert rel(S.lab_source(rec, g[f"src{i}.lab"], float(g[f"src{i}.z"])), g[f"src{i}.source"]) < 1e-13


def test_twelve_columns_are_refused_where_the_fused_transform_is_the_only_one():
    from solprop_b200 import _lib

    rec = record("cap12_ne")
    problem = _lib.Problem(rec)  # the problem itself is taken
    with pytest.raises(_lib.BackendRefusal, match="8 modal columns"):
        _lib.Workspace(problem, 0, "fp64", modal="fused")
    with pytest.raises(_lib.BackendRefusal, match="8 modal columns"):
        _lib.Scan([rec], [policy(golden("cap12_ne"), "adaptive")])
    lab = np.zeros(rec.n_cols * rec.n_omega * 2)
    with pytest.raises(_lib.BackendRefusal, match="8 modal columns"):
        _lib.check(_lib.library().sp_source_noalloc(problem.handle, C.c_void_p(lab.ctypes.data), 0.0, 0,
                                                    C.c_void_p(lab.ctypes.data), None))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cap12_ne", "cap4_he", "cap1_ar", "config2"])
@pytest.mark.parametrize("index", [0, 1])
def test_products_match_the_reference(case, index):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec), 0, "fp64", modal="gemm")
    got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
    assert rel(got, g[f"src{index}.source"]) < SOURCE_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["cap12_ne", "cap4_he", "config2"])
def test_split_bf16_products_match_the_reference_to_fp32(case):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    ws = _lib.Workspace(_lib.Problem(rec), 0, "mixed", modal="gemm")
    for index in (0, 1):
        got = ws.source(g[f"src{index}.lab"], float(g[f"src{index}.z"]))
        assert rel(got, g[f"src{index}.source"]) < MIXED_TOL, index


@pytest.mark.gpu
def test_twelve_modes_step_with_the_reference():
    """A fixed schedule plane by plane at 1e-10, and the adaptive run within its rtol with
    the reference's attempt count (to +-3)."""
    from solprop_b200 import _lib

    rec, g = record("cap12_ne", fixed=True), golden("cap12_ne")
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
    rec = record("cap12_ne")
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


@pytest.mark.gpu
def test_products_and_the_fused_column_take_the_same_steps():
    """Config 2 (four modes, 64 nodes, n_to 16384): five Adams steps on either route."""
    from solprop_b200 import _lib

    rec = record("config2")
    pol = policy(golden("config2"), "adaptive")
    problem = _lib.Problem(rec)
    steps = np.full(5, 2e-5)
    out = {}
    for modal in ("fused", "gemm"):
        session = _lib.Workspace(problem, 0, "fp64", modal=modal).start(pol, schedule=steps)
        for _ in range(5):
            session.advance(1)
        out[modal] = session.export()
    assert rel(out["gemm"], out["fused"]) < 1e-12

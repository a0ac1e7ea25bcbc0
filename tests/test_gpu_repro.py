"""Whole runs are reproducible bit for bit within one process, whatever ran before them.

The benchmark's runs leg solves configs 1 and 2 from start to end, plain FP64 then mixed
precision, each on a workspace of its own that the next one replaces.  This test repeats
that order twice in one process and requires the same attempt counts and the same final
states, bit for bit, on both passes: nothing a run leaves behind -- freed device or pinned
host memory, the response column's tickets and flags, kernel attributes set once per
device -- may reach the next run's arithmetic.
"""

import numpy as np
import pytest

from tests._cases import golden, policy, record

pytestmark = pytest.mark.gpu


def _runs_in_the_benchmarks_order():
    from solprop_b200 import _lib

    out = []
    for case in ("config1", "config2"):
        rec = record(case)
        pol = policy(golden(case), "adaptive")
        problem = _lib.Problem(rec)
        for precision in ("fp64", "mixed"):
            ws = _lib.Workspace(problem, 0, precision)
            session = ws.start(pol)
            while True:
                batch = session.advance(4096)
                if batch.event in (2, 3):
                    break
            assert batch.event == 2, (case, precision)
            out.append((case, precision, int(batch.attempts), int(batch.rejected), session.export()))
    return out


def test_runs_repeat_bit_for_bit_in_one_process():
    first = _runs_in_the_benchmarks_order()
    second = _runs_in_the_benchmarks_order()
    for a, b in zip(first, second):
        assert a[:4] == b[:4]
        assert np.array_equal(a[4], b[4]), a[:2]

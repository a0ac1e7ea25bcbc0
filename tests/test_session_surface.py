"""The session's surface beside stepping: bounds, attempt rows, stop, snapshot and resume.

These mirror the native ``_core.Session`` calls (``native/src/solprop_native/_core.pyi``:
``advance(work_limit, deadline)`` with its attempt rows, reason and category,
``request_stop``, ``request_snapshot``, ``march_state``, ``snapshot``) through the C ABI.
The resume test takes a run's snapshot part-way, lets the original finish, restores the
snapshot on a fresh workspace and requires the restored run to end on the same bits
after the same attempts -- for the exponential Adams march with a constant operator, with
a varying one (its history of states and rates rides in the snapshot too), and for the
DOPRI5 march.
"""

import threading
import time

import numpy as np
import pytest

from tests._cases import golden, policy, record

pytestmark = pytest.mark.gpu


def _session(case, **kw):
    from solprop_b200 import _lib

    rec = record(case)
    problem = _lib.Problem(rec)
    ws = _lib.Workspace(problem)
    return rec, ws, ws.start(policy(golden(case), "adaptive"), **kw)


def _to_end(session, limit=4096):
    while True:
        b = session.advance(limit)
        if b.event in (2, 3):
            return b


def test_deadline_bounds_a_call():
    _, _, session = _session("cap1_ar")
    b = session.advance(100000, 1e-9)
    assert b.event == 0 and b.reason == 3  # none, bound
    assert b.attempts == 1  # the deadline is checked after each attempt


def test_attempt_rows_follow_the_march():
    from solprop_b200 import _lib

    _, _, session = _session("cap4_he")
    rows = []
    last = session.march_state()
    while True:
        b = session.advance(40, rows=True)
        assert b.n_rows == len(b.attempt_rows) == b.attempts - last["attempts"]
        assert int((b.attempt_rows[:, 3] == 0).sum()) == b.rejected - last["rejected"]
        rows.append(b.attempt_rows)
        last = session.march_state()
        if b.event == 2:
            break
    rows = np.concatenate(rows)
    assert _lib.EVENTS[b.event] == "finished" and _lib.REASONS[b.reason] == "reached"
    accepted = rows[rows[:, 3] == 1]
    # every accepted attempt starts where the previous accepted one ended
    assert np.allclose(accepted[1:, 0] - accepted[1:, 1], accepted[:-1, 0], rtol=0, atol=1e-12)
    assert np.all(rows[rows[:, 3] == 1, 2] <= 1.0) and np.all(rows[rows[:, 3] == 0, 2] > 1.0)
    assert np.all(rows[:, 4] > 0)
    assert abs(accepted[-1, 0] - last["z"]) < 1e-12 and last["outcome"] == 1


def test_stop_from_another_thread_ends_the_run():
    from solprop_b200 import _lib

    _, _, session = _session("config2")
    timer = threading.Timer(0.05, session.request_stop)
    timer.start()
    t0 = time.perf_counter()
    b = session.advance(1_000_000)
    timer.join()
    assert _lib.EVENTS[b.event] == "stopped" and _lib.REASONS[b.reason] == "stopped"
    assert 0 < b.attempts < 1408 and time.perf_counter() - t0 < 5.0
    assert session.march_state()["outcome"] == 2
    with pytest.raises(_lib.SessionLifecycleError):
        session.advance(1)


def test_a_floor_failure_maps_to_convergence():
    from solprop_b200 import _lib

    rec = record("cap1_ar")
    pol = dict(policy(golden("cap1_ar"), "adaptive"))
    pol["dz_min"] = 1.0  # every proposal falls below it
    ws = _lib.Workspace(_lib.Problem(rec))
    session = ws.start(pol)
    with pytest.raises(_lib.ConvergenceError, match="dz_min"):
        session.advance(10)
    b = session.batch
    assert _lib.EVENTS[b.event] == "failed"
    assert _lib.REASONS[b.reason] == "floor" and _lib.CATEGORIES[b.category] == "convergence"
    with pytest.raises(_lib.SessionLifecycleError):
        session.advance(1)


@pytest.mark.parametrize("case", ["config1", "cap4_he", "gnlse_raman"])
def test_snapshot_resumes_bit_for_bit(case):
    from solprop_b200 import _lib

    rec, ws, session = _session(case)
    session.request_snapshot()
    b = session.advance(4096)
    assert _lib.EVENTS[b.event] in ("halted", "plane")
    while b.attempts < 40 and b.event not in (2, 3):  # part-way into the run
        b = session.advance(1)
    session.request_snapshot()
    b = session.advance(4096)
    assert _lib.EVENTS[b.event] in ("halted", "plane"), b.event
    snap = session.snapshot()
    state_then = session.march_state()
    end_a = _to_end(session)
    final_a = session.export()
    # a fresh workspace of the same problem continues the snapshot
    ws2 = _lib.Workspace(_lib.Problem(rec))
    resumed = ws2.restore(policy(golden(case), "adaptive"), snap)
    assert resumed.march_state() == state_then
    end_b = _to_end(resumed)
    assert end_b.event == 2 and end_a.event == 2
    assert (end_b.attempts, end_b.rejected) == (end_a.attempts, end_a.rejected)
    assert np.array_equal(resumed.export(), final_a)


def test_a_snapshot_of_another_problem_is_refused():
    from solprop_b200 import _lib

    _, _, session = _session("cap1_ar")
    session.advance(5)
    snap = session.snapshot()
    rec = record("cap4_he")
    ws = _lib.Workspace(_lib.Problem(rec))
    with pytest.raises(_lib.NativeError, match="another problem"):
        ws.restore(policy(golden("cap4_he"), "adaptive"), snap)
    with pytest.raises(_lib.NativeError, match="not a snapshot"):
        ws.restore(policy(golden("cap4_he"), "adaptive"), b"x" * len(snap))


@pytest.mark.parametrize("case", ["config1", "cap4_he"])
def test_reads_between_attempts_leave_the_run_unchanged(case):
    """A single run's accepted trial leaves its accept (the new state and the history's
    source row) to the next trial's predictor; every other reader of the state or the rows
    writes it first.  Exports, plane statistics, snapshots and workspace source calls after
    every attempt must see the accepted state and leave the run on the bits of an
    undisturbed run."""
    from solprop_b200 import _lib

    rec, ws, session = _session(case)
    end_a = _to_end(session)
    final_a = session.export()

    ws2 = _lib.Workspace(_lib.Problem(rec))
    session2 = ws2.start(policy(golden(case), "adaptive"))
    lab = np.asarray(rec.field0, dtype=np.complex128)
    states = []
    while True:
        b = session2.advance(1)
        state = session2.export()  # the accepted state, whatever the next trial does
        assert np.array_equal(session2.export(), state)
        states.append(state)
        k = len(states)
        if k % 3 == 0:
            session2.statistics()
        if k % 5 == 0:
            ws2.source(lab, b.z)
        if k % 7 == 0:
            session2.snapshot()
        if b.event in (2, 3):
            break
    assert b.event == 2 and (b.attempts, b.rejected) == (end_a.attempts, end_a.rejected)
    assert np.array_equal(session2.export(), final_a)
    # a rejected trial leaves the state as it was; an accepted one moves it
    assert any(not np.array_equal(states[i], states[i + 1]) for i in range(len(states) - 1))

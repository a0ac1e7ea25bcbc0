"""The scan workload: the seeded problem builder (CPU) and the batched solver (GPU)."""

import numpy as np
import pytest

from oracle import march as M
from oracle import source as S
from solprop_b200 import scan
from tests._cases import rel


def test_draw_points_follows_the_stated_distribution():
    pts = scan.draw_points(400, 11)
    r = np.array([p.radius for p in pts])
    e = np.array([p.energy for p in pts])
    assert r.min() >= 50e-6 and r.max() <= 150e-6
    assert e.min() >= 20e-6 and e.max() <= 500e-6
    assert {p.gas for p in pts} == {"He", "Ne", "Ar"}
    assert {p.n_to for p in pts} == {4096, 8192, 16384, 32768}
    assert {p.modes for p in pts} == set(range(1, 9))
    assert scan.draw_points(5, 11) == pts[:5]  # seeded


def test_capillary_record_is_a_consistent_problem():
    p = scan.ScanPoint(100e-6, 1.0, "Ar", 1.0, 50e-6, 20e-15, 3, 4096, 7)
    rec, pol = scan.capillary_record(p)
    # projection @ synthesis = pad_scale I on the orthonormal set (kernel-contract.md 4)
    ps = rec.projection @ rec.synthesis
    assert np.allclose(ps, rec.pad_scale * np.eye(3), atol=1e-12)
    # operator and prefactor vanish off the active band
    assert np.all(rec.phi_terms[..., ~rec.active_mask] == 0)
    assert np.all(rec.prefactor_terms[..., ~rec.active_mask] == 0)
    # the pulse carries its energy (Parseval on the coarse grid, half spectrum)
    x = np.fft.irfft(rec.field0[0, 0], n=rec.n_t)
    assert abs(np.sum(x * x) * rec.dt / 50e-6 - 1) < 1e-3
    out = {}
    k = S.lab_source(rec, rec.launch_field() * rec.active_mask, 0.0, out=out)
    assert np.all(np.isfinite(k)) and np.abs(k).max() > 0
    assert out["rate"].max() > 0  # the pulse ionises


SMALL_SCAN = [
    scan.ScanPoint(120e-6, 1.0, "He", 1.0, 60e-6, 20e-15, 2, 4096, 1),
    scan.ScanPoint(90e-6, 0.8, "Ar", 0.5, 30e-6, 25e-15, 1, 8192, 2),
    scan.ScanPoint(140e-6, 1.5, "Ne", 2.0, 100e-6, 12e-15, 3, 4096, 3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["tiles", "sweep"])
def test_batched_runs_match_single_runs(form):
    from solprop_b200 import _lib

    built = [scan.capillary_record(p) for p in SMALL_SCAN]
    sc = _lib.Scan([r for r, _ in built], [q for _, q in built])
    sc.set_column(form)
    steps = 12
    sc.advance(steps)
    assert "attempt phase: one CUDA graph" in sc.describe()
    assert f"column: {'sweep' if form == 'sweep' else 'tile-parallel'}" in sc.describe()
    for i, (rec, pol) in enumerate(built):
        state, info = sc.run(i)
        problem = _lib.Problem(rec)
        ws = _lib.Workspace(problem)
        session = ws.start(pol)
        for _ in range(int(info.attempts)):
            session.advance(1)
        assert rel(state, session.export()) < 1e-12, i
        assert info.attempts == steps


@pytest.mark.gpu
def test_batched_run_matches_the_oracle():
    from solprop_b200 import _lib

    p = scan.ScanPoint(110e-6, 1.0, "Ar", 1.0, 40e-6, 20e-15, 2, 4096, 5)
    rec, pol = scan.capillary_record(p)
    sc = _lib.Scan([rec], [pol])
    sc.advance(6)
    state, info = sc.run(0)
    ws = M.Workspace(rec)
    march = M.AdamsMarch(M.AdamsEngine(ws, pol), pol, pol["proposal"])
    for _ in range(int(info.attempts)):
        march.attempt_towards(rec.z_end)
    assert march.attempts == info.attempts
    assert rel(state, ws.state) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_column_forms_give_the_same_bits(precision):
    """The sweep carries each node's running sums in the order the tile-parallel column
    adds its predecessors' sums, and the forward transform adds the node groups' partial
    rows in the order the tile's last CTA does: the runs come out bit for bit equal."""
    from solprop_b200 import _lib

    built = [scan.capillary_record(p) for p in SMALL_SCAN]
    states = {}
    for form in ("tiles", "sweep"):
        sc = _lib.Scan([r for r, _ in built], [q for _, q in built], 0, precision)
        for n_to in sorted({p.n_to for p in SMALL_SCAN}):  # the same transforms in both scans
            sc.set_transforms(n_to, 0, 0)
        sc.set_column(form)
        sc.advance(8)
        states[form] = [sc.run(i)[0] for i in range(len(built))]
        sc.close()
    for a, b in zip(states["tiles"], states["sweep"]):
        assert np.array_equal(a, b)


def test_unknown_column_form_is_refused():
    from solprop_b200 import _lib

    with pytest.raises(ValueError):
        object.__new__(_lib.Scan).set_column("rows")


@pytest.mark.gpu
def test_transform_forms_are_checked_and_all_agree():
    """Every transform form a grid admits gives the same run to rounding; a form that does
    not hold the rows, or a grid the scan does not have, is refused."""
    from solprop_b200 import _lib

    p = scan.ScanPoint(100e-6, 1.0, "Ar", 1.0, 40e-6, 20e-15, 2, 16384, 7)
    rec, pol = scan.capillary_record(p)
    states = []
    for width in (0, 2, 4, 8):
        sc = _lib.Scan([rec], [pol])
        sc.set_transforms(16384, width, width)
        sc.advance(6)
        states.append(sc.run(0)[0])
        sc.close()
    for s in states[1:]:
        assert rel(s, states[0]) < 1e-12
    sc = _lib.Scan([rec], [pol])
    with pytest.raises(_lib.NativeError):
        sc.set_transforms(8192, 0, 0)
    with pytest.raises(_lib.NativeError):
        sc.set_transforms(16384, 3, 0)


@pytest.mark.gpu
def test_scan_to_completion_replans_and_matches_single_runs():
    """Runs of different lengths finish at different batch steps; the scan re-plans its
    work lists as they do (only the running runs are launched, the forms tuned again), the
    last few go on as single runs side by side, and every run still ends where it ends
    alone."""
    from solprop_b200 import _lib

    lengths = (0.02, 0.025, 0.03, 0.035, 0.04, 0.05, 0.06, 0.08, 0.1, 0.12, 0.14, 0.16)
    points = [scan.ScanPoint(120e-6, length, "He", 1.0, 60e-6, 20e-15, 1, 4096, 11 + k)
              for k, length in enumerate(lengths)]
    built = [scan.capillary_record(p) for p in points]
    sc = _lib.Scan([r for r, _ in built], [q for _, q in built])
    sc.set_alone(0)
    for _ in range(200):
        if sc.advance(500).active == 0:
            break
    assert sc.advance(0).active == 0
    text = sc.describe()
    assert "re-planned 0 times" not in text, text
    assert "alone from batch step -1" not in text, text  # the last runs went on alone
    for i, (rec, pol) in enumerate(built):
        state, info = sc.run(i)
        assert info.event == 2  # finished
        ws = _lib.Workspace(_lib.Problem(rec))
        session = ws.start(pol)
        while session.advance(4096).event != 2:
            pass
        assert session.batch.attempts == info.attempts, i
        assert rel(state, session.export()) < 1e-12, i



@pytest.mark.gpu
def test_long_runs_go_on_alone_and_match_single_runs():
    """With a low threshold the longest runs leave the batch and step on host threads of
    their own beside it; every run still ends where it ends alone."""
    from solprop_b200 import _lib

    lengths = (0.02, 0.02, 0.025, 0.03, 0.03, 0.035, 0.2, 0.3)
    points = [scan.ScanPoint(120e-6, length, "He", 1.0, 60e-6, 20e-15, 1, 4096, 31 + k)
              for k, length in enumerate(lengths)]
    built = [scan.capillary_record(p) for p in points]
    sc = _lib.Scan([r for r, _ in built], [q for _, q in built])
    sc.set_alone(2, 20.0, 2.0)
    for _ in range(400):
        if sc.advance(16).active == 0:
            break
    assert sc.advance(0).active == 0
    text = sc.describe()
    assert "0 long runs went on alone" not in text, text
    for i, (rec, pol) in enumerate(built):
        state, info = sc.run(i)
        assert info.event == 2
        ws = _lib.Workspace(_lib.Problem(rec))
        session = ws.start(pol)
        while session.advance(4096).event != 2:
            pass
        assert session.batch.attempts == info.attempts, i
        assert rel(state, session.export()) < 1e-12, i
    with pytest.raises(_lib.NativeError):
        sc.set_alone(-1)

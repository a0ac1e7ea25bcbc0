"""Plane statistics: the oracle against the reference's own values, the device against both.

``tests/golden/generate.py`` evaluates solprop's statistics (``stats/definitions.py``)
on fixture states: a four-mode capillary (field grid, n_t 2048), config 2 (n_t 8192),
the eight-mode scan point (n_t 16384, which the device transforms as two residue
classes of 8192 points) and the envelope GNLSE.  The energies, centroids and the energy
per bin are sums; the peak powers come from the analytic signal.
"""

import numpy as np
import pytest

from oracle import statistics as O
from tests._cases import golden, policy, record, rel

CASES = ("cap4_he", "config2", "scan0", "gnlse_raman")
NAMES = ("energy", "omega0", "peak_power", "peak_power_total", "spectrum")


def _state(case, g):
    return g["attempts.state"] if case.startswith("scan") else g["adaptive.states"][-1]


@pytest.mark.parametrize("case", CASES)
def test_oracle_statistics_match_the_reference(case):
    rec, g = record(case), golden(case)
    got = O.statistics(rec, _state(case, g))
    for name in NAMES:
        assert rel(np.ravel(got[name]), np.ravel(g[f"stats.{name}"])) < 1e-13, name


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_device_statistics_match_the_reference(case):
    from solprop_b200 import _lib

    rec, g = record(case), golden(case)
    state = _state(case, g)
    ws = _lib.Workspace(_lib.Problem(rec))
    session = ws.start(policy(g, "adaptive"), field0=state)  # the session holds the state
    got = session.statistics()
    for name in NAMES:
        assert rel(np.ravel(got[name]), np.ravel(g[f"stats.{name}"])) < 1e-12, name


@pytest.mark.gpu
def test_scan_statistics_match_the_oracle_without_exporting_states():
    from solprop_b200 import _lib

    cases = ("scan0", "scan1", "scan2", "scan3")
    recs = [record(c) for c in cases]
    sc = _lib.Scan(recs, [policy(golden(c), "adaptive") for c in cases])
    sc.advance(6)
    for i, rec in enumerate(recs):
        got = sc.statistics(i)
        want = O.statistics(rec, sc.run(i)[0])
        for name in NAMES:
            assert rel(np.ravel(got[name]), np.ravel(want[name])) < 1e-12, (i, name)
    sc.close()

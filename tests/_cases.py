"""Shared helpers for the parity tests: fixture loading and relative errors."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from solprop_b200.record import load_record

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("cap1_ar", "cap4_he", "gnlse_raman", "raman_n2", "mix_hear", "raman_mix", "env4_n2", "env3_rk", "envv_n2")


def rel(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def record(case: str, fixed: bool = False):
    return load_record(GOLDEN / f"{case}{'_fixed' if fixed else ''}.problem.npz")


def golden(case: str):
    return np.load(GOLDEN / f"{case}.golden.npz")


def policy(g, kind: str) -> dict:
    return json.loads(bytes(g[f"{kind}.policy"]).decode())


def fixed_schedule(g):
    """The fixed run's steps: uniform between the first and last plane, of the size the
    history records (its rows may be one per step or one per plane)."""
    zs = g["fixed.z"]
    if "fixed.history" in g.files:
        n = int(round(zs[-1] / g["fixed.history"][0, 1]))
    else:
        n = 100
    edges = np.linspace(0.0, zs[-1], n + 1)
    return np.diff(edges), edges

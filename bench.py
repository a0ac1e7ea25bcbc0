"""Benchmark of the B200 propagation hot path (one JSON line on stdout, rank 0).

Workload: config 2, the four-mode (HE11-HE14) helium capillary with a 0.8 -> 0
bar gradient, 1.5 m, 800 nm, 7.5 fs, 275 uJ, 90 nm - 4 um, n_to = 16384 fine samples,
64 Gauss nodes, Kerr + field plasma (band rule) + the in-stage collar, exponential
Adams at rtol 1e-6 -- lowered from the reference's own translation
(``tests/golden/config2.problem.npz``, made by ``tests/golden/generate.py``).

A step is one exponential-Adams attempt of that run: predictor, one source evaluation
(inverse FFT, synthesis + plasma/Kerr column, projection, forward FFT, stage output),
corrector with its defect norms, and the accept -- FP64 throughout.  ``value`` is
attempts per second with the state resident in HBM, timed with CUDA events on the
library's stream, L2 flushed (a 256 MiB write) between steps.  ``e2e`` is the same
through the public C ABI from host memory: session start (host field upload), the
attempts, and the export of the final field.  Multi-GPU: the run does not shard
(z is sequential), so N ranks run N independent replicas (weak scaling).

``--impl reference`` times the reference's CPU implementation of the path -- the
oracle port of ``numpy_ref`` (``oracle/``), pinned bit for bit to it by the tests --
on the host cores, on the same workload and unit.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "config2"
# DRAM bytes read + written per k_column launch on this workload, from one ncu capture
# (profiles/k_column_config2.md: 945 920 B read, 2 048 B written; the rest stays in L2)
COLUMN_TRAFFIC = 947_968
METRIC = "steps/s (exponential-Adams attempts, plain FP64, config 2 four-mode He capillary)"
UNIT = "steps/s"


def load_workload():
    from tests._cases import golden, policy, record

    rec = record(WORKLOAD)
    pol = policy(golden(WORKLOAD), "adaptive")
    return rec, pol


def algorithmic_bytes(rec) -> dict:
    """Bytes each kernel family must move per launch (reads + writes of its operands).

    The response column reads the modal field and the two temporal windows once and writes
    the projected streams (and its tiles' running-integral sums); nothing node-sized is
    stored, and the node groups' partial rows beyond one (added by the forward transform)
    are not counted.  The forward transform reads the projected streams and writes the
    spectra.  The corrector forms the stage output itself (its streams, prefactor terms and
    source row are counted with it), and the predictor applies the accept of the trial
    before (its rows are counted with it).
    """
    n = rec.n_cols * rec.n_omega
    c128, f64 = 16, 8
    nt, nn, nc = rec.n_to, rec.n_nodes, rec.n_cols
    k = (len(rec.taps) - 1) if rec.plasma_enabled else 0
    owned = 256 - 2 * (2 * k + 1)
    tiles = -(-nt // owned)
    streams = 3 if rec.plasma_enabled else 1
    absorber = 1 if rec.absorber_scheme == "nonlinear" else 0
    projected = streams * nc * nt * f64
    return {
        "adams_predict": 14 * n * c128 + 4 * n * c128,
        "inverse_fft": n * c128 + (1 + absorber) * nc * nt * f64 + absorber * nt * f64,
        "response_column": nc * nt * f64 + 2 * nt * f64 + 2 * nn * tiles * f64 + projected,
        "forward_fft": projected + absorber * nc * nt * f64 + (streams + absorber) * n * c128,
        "adams_correct": 15 * n * c128 + (streams + absorber) * n * c128
        + rec.n_prefactor_terms * n * c128 + n * c128,
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self) -> dict:
        rows = []
        for line in self.path.read_text().splitlines() if self.path.exists() else []:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_arm(rec, pol, steps: int, warmup: int, budget_s: float, threads: int | None):
    """The oracle march on the host: one attempt per step, wall-clock timed."""
    from threadpoolctl import threadpool_limits

    from oracle import march as M

    with threadpool_limits(limits=threads):
        ws = M.Workspace(rec)
        march = M.AdamsMarch(M.AdamsEngine(ws, pol), pol, pol["proposal"])
        target = float(pol["save_planes"][0]) if pol["save_planes"] else rec.z_end
        for _ in range(warmup):
            march.attempt_towards(target)
        done, t0 = 0, time.perf_counter()
        while done < steps and (time.perf_counter() - t0) < budget_s:
            march.attempt_towards(target)
            done += 1
        elapsed = time.perf_counter() - t0
    return done, elapsed


def runs_leg(device: int) -> dict:
    """Configs 1 and 2 run start to end, plain FP64 and mixed precision: runs per second,
    attempts per second, and the mixed run's relative L2 error against the FP64 run in
    the final spectrum and in time (each run takes its own adaptive steps)."""
    import torch

    from solprop_b200 import _lib
    from tests._cases import golden, policy, record

    out = {}
    for case in ("config1", "config2"):
        rec = record(case)
        pol = policy(golden(case), "adaptive")
        problem = _lib.Problem(rec)
        finals = {}
        for precision in ("fp64", "mixed"):
            ws = _lib.Workspace(problem, device, precision)
            stream = torch.cuda.ExternalStream(ws.stream, device=torch.device("cuda", device))
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s_ev.record(stream)
            session = ws.start(pol)
            while True:
                batch = session.advance(4096)
                if batch.event in (2, 3):
                    break
            e_ev.record(stream)
            torch.cuda.synchronize()
            sec = s_ev.elapsed_time(e_ev) / 1e3
            finals[precision] = session.export()
            out.setdefault(case, {})[precision] = {
                "finished": batch.event == 2, "attempts": int(batch.attempts), "seconds": sec,
                "runs_per_s": 1.0 / sec, "attempts_per_s": batch.attempts / sec}
        a64, a32 = finals["fp64"], finals["mixed"]
        t64 = np.fft.irfft(a64.reshape(-1, a64.shape[-1]), axis=-1)
        t32 = np.fft.irfft(a32.reshape(-1, a32.shape[-1]), axis=-1)
        out[case]["mixed_vs_fp64_spectral_rel_l2"] = float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64))
        out[case]["mixed_vs_fp64_temporal_rel_l2"] = float(np.linalg.norm(t32 - t64) / np.linalg.norm(t64))
    return out


def surrogate_leg(device: int, points: int = 16384, members: int = 5, repeats: int = 5) -> dict:
    """The surrogate's inference: ``members`` perceptrons (6 -> 4 x 512 -> 2048) over
    ``points`` inputs, device time per pass (CUDA events) and the FLOP rate against the
    measured BF16 peak -- on the tcgen05 path (TMA tiles, tensor-memory accumulators, BF16
    activations) and, for comparison, on the mma.sync path the training uses."""
    import torch

    from solprop_b200 import surrogate

    ens = surrogate.Ensemble(members=members, seed=1, device=device)
    x = torch.rand((points, 6), device=f"cuda:{device}") * 2 - 1
    sizes = (6,) + surrogate.HIDDEN + (surrogate.N_OUT,)
    flops = 2.0 * points * members * sum(a * b for a, b in zip(sizes[:-1], sizes[1:]))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    status = torch.zeros(1, dtype=torch.int32, device=f"cuda:{device}")

    def timed(run) -> float:
        run()
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ev.record()
        for _ in range(repeats):
            run()
        e_ev.record()
        torch.cuda.synchronize()
        return s_ev.elapsed_time(e_ev) / repeats

    ms_tc = timed(lambda: ens.infer(x, status))  # each layer: every member in one launch
    ms_mma = timed(lambda: [m.forward(x) for m in ens.members])
    if int(status.item()):
        raise RuntimeError("a tensor-core product's wait gave up")
    achieved = flops / (ms_tc * 1e-3) / 1e12
    return {"points": points, "members": members, "ms_per_pass": ms_tc, "points_per_s": points / (ms_tc * 1e-3),
            "mma_sync_ms_per_pass": ms_mma,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"}}


def modal_products_record(n_modes: int = 30, n_nodes: int = 16384):
    """A config-3-sized modal transform on config 2's field grid (n_to 16 384): n_modes
    columns on n_nodes nodes.  Synthetic operands with config 2's magnitudes -- node i,
    mode m takes config 2's synthesis and projection weights of node i mod 64 and mode
    m mod 4, the projection divided by the node multiple, each times a seeded factor in
    [0.9, 1.1] -- and config 2's operator and prefactor per mode m mod 4; the launch field
    is config 2's in the first four modes."""
    rec, pol = load_workload()
    rng = np.random.default_rng(7)
    base_s, base_w = rec.synthesis, rec.projection
    modes = np.arange(n_modes) % rec.n_modes
    nodes = np.arange(n_nodes) % rec.n_nodes
    rec.synthesis = np.ascontiguousarray(base_s[nodes][:, modes] * rng.uniform(0.9, 1.1, (n_nodes, n_modes)))
    rec.projection = np.ascontiguousarray(base_w[modes][:, nodes] * (rec.n_nodes / n_nodes)
                                          * rng.uniform(0.9, 1.1, (n_modes, n_nodes)))
    rec.projection_coarse = rec.projection.copy()
    rec.phi_terms = np.ascontiguousarray(rec.phi_terms[:, modes])
    rec.prefactor_terms = np.ascontiguousarray(rec.prefactor_terms[:, modes])
    field0 = np.zeros((n_modes,) + rec.field0.shape[1:], dtype=np.complex128)
    field0[: rec.n_modes] = rec.field0
    rec.field0 = field0
    rec.n_modes, rec.n_nodes = n_modes, n_nodes
    return rec, pol


def modal_products_leg(device: int, repeats: int = 3, n_nodes: int = 16384) -> dict:
    """The modal transform as products at a config-3 size (30 modes, 16 384 nodes, 16 384
    samples; config 3's own route -- envelope grid, vector modes, tensor Raman -- is not
    built): per source evaluation, the products' device time (synthesis and the three
    streams' projections, the mixed form's splits included) and their FLOP rate against
    the measured BF16 peak, in the mixed form (tcgen05, three-part BF16 splits) and the
    plain FP64 form.  FLOPs counted are the product's own, 2 N_q n_m n_to for the synthesis
    and 2 x 3 n_m N_q n_to for the projections; the split form executes six BF16 products
    for each."""
    from solprop_b200 import _lib

    rec, pol = modal_products_record(n_nodes=n_nodes)
    flops = 2.0 * rec.n_nodes * rec.n_modes * rec.n_to * (1 + 3)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops", 1590.0)
    problem = _lib.Problem(rec)
    out = {"workload": f"modal transform: 30 modes x {n_nodes} nodes x 16384 samples, config 2 grid and "
                       "response (synthetic operands)", "flops_per_evaluation": flops}
    lab = rec.field0
    for precision in ("mixed", "fp64"):
        ws = _lib.Workspace(problem, device, precision, modal="gemm")
        session = ws.start(pol, field0=lab)  # the timing switch lives on a session
        ws.source(lab, 0.0)  # warm-up
        session.set_timing(True)
        session.timing(reset=True)
        for _ in range(repeats):
            ws.source(lab, 0.0)
        fams = session.timing(reset=True)
        session.set_timing(False)
        prod_ms = fams["project"][0] / repeats
        total_ms = sum(v[0] for v in fams.values()) / repeats
        achieved = flops / (prod_ms * 1e-3) / 1e12
        out[precision] = {"products_ms": prod_ms, "column_ms": fams["response_column"][0] / repeats,
                          "evaluation_ms": total_ms, "products_tflops": achieved,
                          "frac_of_bf16_peak": achieved / peak}
        session.close()
        ws.close()
    out["roofline"] = {"bound": "tensor", "kernel": "modal products (tcgen05, split BF16)",
                       "achieved": out["mixed"]["products_tflops"], "peak": peak, "unit": "TFLOP/s",
                       "frac": out["mixed"]["frac_of_bf16_peak"],
                       "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"}
    return out


def config3_leg(device: int, attempts: int = 3, grid: int = 128) -> dict:
    """Config 3's route at its mode and node counts: 30 vector graded-index modes on
    ``grid x grid`` Cartesian nodes (two field components per node), the envelope grid
    with config 3's 2^14 samples, the analytic Kerr cubic
    and the tensor Raman response, DOPRI5 -- ``solprop_b200.grin``'s seeded synthetic
    workload.  Per precision: DOPRI5 attempts per second and, per source evaluation, the
    device time of its kernel families (session timing, CUDA events); the products' roofline
    in HBM bytes -- the node field written and the node stream read, N_rows x 2 n_to
    elements each -- since with K = 30 modes the products are bound by those bytes, not by
    the tensor pipe."""
    from solprop_b200 import _lib, grin

    rec, pol = grin.grin_record(n_to=16384, grid=grid)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    rows = rec.n_nodes * rec.n_pol_transform
    problem = _lib.Problem(rec)
    out = {"workload": f"config 3 (synthetic graded-index fibre): {rec.n_modes} vector modes on {grid}x{grid} "
                       f"nodes x 2 components, envelope n_to {rec.n_to}, Kerr + tensor Raman, DOPRI5",
           "modes": rec.n_modes, "nodes": rec.n_nodes, "n_to": rec.n_to}
    for precision in ("mixed", "fp64"):
        ws = _lib.Workspace(problem, device, precision)
        session = ws.start(pol)
        session.advance(1)  # warm-up: the first attempt
        session.set_timing(True)
        session.timing(reset=True)
        t0 = time.perf_counter()
        batch = session.advance(attempts)
        wall = time.perf_counter() - t0
        fams = session.timing(reset=True)
        session.set_timing(False)
        done = int(batch.attempts) - 1
        evaluations = max(fams.get("response_column", (0.0, 1))[1], 1)
        elem = 4 if precision == "mixed" else 8
        algorithmic = 2.0 * rows * 2 * rec.n_to * elem
        prod_ms = fams["project"][0] / evaluations
        out[precision] = {
            "attempts": done, "attempts_per_s": done / wall,
            "evaluation_ms": sum(v[0] for v in fams.values()) / evaluations,
            "families_ms_per_evaluation": {k: v[0] / evaluations for k, v in fams.items()},
            "products_ms": prod_ms, "products_gbs": algorithmic / (prod_ms * 1e-3) / 1e9,
            "products_frac_of_hbm": algorithmic / (prod_ms * 1e-3) / 1e9 / hbm}
        session.close()
        ws.close()
    out["roofline"] = {"bound": "hbm", "kernel": "modal products (tcgen05, split BF16)",
                       "achieved": out["mixed"]["products_gbs"], "peak": hbm, "unit": "GB/s",
                       "frac": out["mixed"]["products_frac_of_hbm"],
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    return out


def scan_leg(device: int, n_runs: int, steps: int, warmup: int, seed: int = 2024,
             rank: int = 0, world: int = 1) -> dict:
    """The parameter-scan workload (config 4): n_runs seeded uneven capillary runs, stepped together.

    Reports attempts per second of the batched solver at full batch (every batch step gives
    every run one exponential-Adams attempt; no run leaves the batch to go on alone) and of
    the plain path on the same runs one at a time (one session per run, its attempts back
    to back), on the device's clock.  With
    several ranks each solves its cost-balanced share of the runs (``scan.shard``, no
    exchange); attempts add over ranks and the time is the slowest rank's.
    """
    import torch

    from solprop_b200 import _lib, scan

    points = scan.draw_points(n_runs, seed)
    points = [points[i] for i in scan.shard(points, rank, world)]
    built = [scan.capillary_record(p) for p in points]

    def across_ranks(attempts: float, ms: float) -> tuple[float, float]:
        if world == 1:
            return attempts, ms
        import torch.distributed as dist

        a = torch.tensor([attempts], dtype=torch.float64, device=f"cuda:{device}")
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(a, op=dist.ReduceOp.SUM)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(a.item()), float(t.item())
    records, policies = [b[0] for b in built], [b[1] for b in built]
    batched = {}
    for precision in ("fp64", "mixed"):
        sc = _lib.Scan(records, policies, device, precision)
        sc.set_alone(0)
        stream = torch.cuda.ExternalStream(sc.stream, device=torch.device("cuda", device))
        sc.advance(warmup)
        before = sc.advance(0).attempts
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ev.record(stream)
        status = sc.advance(steps)
        e_ev.record(stream)
        torch.cuda.synchronize()
        attempts, ms = across_ranks(status.attempts - before, s_ev.elapsed_time(e_ev))
        # the families' device times over a few more batch steps, events around each
        sc.set_timing(True)
        sc.timing(reset=True)
        timed_steps = 5
        sc.advance(timed_steps)
        families = sc.timing(reset=True)
        sc.set_timing(False)
        batched[precision] = {"attempts_per_s": attempts / (ms / 1e3),
                              "ms_per_batch_step": ms / steps, "active_runs_at_end": status.active,
                              "roofline": scan_roofline(records, families, timed_steps, precision),
                              "transform_plan": sc.describe().strip().splitlines()}
        sc.close()
    # the plain path: each run alone, three attempts after one warm-up
    plain_ms, plain_attempts = 0.0, 0
    sample = list(range(0, len(points), max(1, n_runs // 64)))
    for i in sample:
        problem = _lib.Problem(records[i])
        ws = _lib.Workspace(problem, device)
        st = torch.cuda.ExternalStream(ws.stream, device=torch.device("cuda", device))
        session = ws.start(policies[i])
        session.advance(1)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(3):
            session.advance(1)
        b.record(st)
        torch.cuda.synchronize()
        plain_ms += a.elapsed_time(b)
        plain_attempts += 3
        session.close()
        ws.close()
        problem.close()
    plain_attempts, plain_ms = across_ranks(plain_attempts, plain_ms)
    plain = plain_attempts / (plain_ms / 1e3)
    return {"workload": f"config 4: {n_runs} seeded capillary runs (radius 50-150 um, length "
                        "0.5-2 m, He/Ne/Ar, 0.2-3 bar, 20-500 uJ, 5-30 fs, 1-8 modes, "
                        "n_to 2^12-2^15), Kerr + plasma + input shot noise, exp. Adams rtol 1e-6",
            "ranks": world, "batch_steps": steps, "batched": batched,
            "plain_fp64_attempts_per_s": plain, "plain_sample_runs": len(sample),
            "speedup_vs_plain": {k: v["attempts_per_s"] / plain for k, v in batched.items()}}


def scan_roofline(records, families: dict, steps: int, precision: str) -> dict:
    """Achieved bandwidth of each batched family over the timed batch steps: its
    algorithmic bytes per batch step (every run in the batch, the byte counts below) over
    its CUDA-event time, against the measured copy bandwidth.  Per run, with n the state's
    complex elements, c its modal columns, T its fine samples, r the transforms' and the
    column's real size (8 in FP64, 4 in the mixed form), P its prefactor terms:
    predict 14 x 16 n (state, five history rows, lab, six moments, flow, exponent),
    correct 15 x 16 n, accept 4 x 16 n; inverse 16 n + 2 x 8 c T (lab in, the modal field
    and the collar's stream out, FP64 in both forms); column 8 c T + 3 r c T (modal field
    in, three projected streams out); forward 4 r c T + 8 r n (four streams in, four
    spectra out); output 8 r n + (P + 2) 16 n."""
    r = 8 if precision == "fp64" else 4
    bytes_ = dict.fromkeys(("adams_predict", "inverse_fft", "response_column", "forward_fft",
                            "stage_output", "adams_correct", "adams_accept"), 0.0)
    for rec in records:
        n, c, T, P = rec.n_cols * rec.n_omega, rec.n_cols, rec.n_to, rec.prefactor_terms.shape[0]
        bytes_["adams_predict"] += 14 * 16 * n
        bytes_["adams_correct"] += 15 * 16 * n
        bytes_["adams_accept"] += 4 * 16 * n
        bytes_["inverse_fft"] += 16 * n + 2 * 8 * c * T
        bytes_["response_column"] += 8 * c * T + 3 * r * c * T
        bytes_["forward_fft"] += 4 * r * c * T + 8 * r * n
        bytes_["stage_output"] += 8 * r * n + (P + 2) * 16 * n
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    out = {}
    for name, b in bytes_.items():
        ms, launches = families.get(name, (0.0, 0))
        if not launches:
            continue
        per_step_ms = ms / steps
        achieved = b / (per_step_ms * 1e-3) / 1e9
        out[name] = {"algorithmic_bytes": b, "ms_per_batch_step": per_step_ms,
                     "achieved_gbs": achieved, "frac": achieved / peak}
    top = max(out, key=lambda k: out[k]["ms_per_batch_step"])
    return {"bound": "hbm", "kernel": top, "achieved": out[top]["achieved_gbs"], "peak": peak,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback", "unit": "GB/s",
            "frac": out[top]["frac"], "families": out}


def run_errors(mixed: list, reference: list, records) -> dict:
    """Relative L2 of each mixed-precision run's final state against the plain FP64 run of
    the same point: in the spectrum, and in time (the fields the states make)."""
    spectral, temporal = [], []
    for a, b, rec in zip(mixed, reference, records):
        spectral.append(float(np.linalg.norm(a - b) / np.linalg.norm(b)))
        ta = np.fft.irfft(a.reshape(-1, a.shape[-1]), n=rec.n_t, axis=-1)
        tb = np.fft.irfft(b.reshape(-1, b.shape[-1]), n=rec.n_t, axis=-1)
        temporal.append(float(np.linalg.norm(ta - tb) / np.linalg.norm(tb)))
    spectral, temporal = np.array(spectral), np.array(temporal)
    return {"spectral_max": float(spectral.max()), "spectral_median": float(np.median(spectral)),
            "temporal_max": float(temporal.max()), "temporal_median": float(np.median(temporal)),
            "runs_at_most_1e-6": int((spectral <= 1e-6).sum()), "runs": int(spectral.size)}


def complete_scan_leg(device: int, n_runs: int, seed: int = 2024, rank: int = 0, world: int = 1,
                      batched_fp64: bool = True) -> dict:
    """The scan's first n_runs points solved to the end, in runs per second: the batched
    mixed solver (re-planning as runs finish, long runs going on alone), and the batched
    FP64 solver, against the plain FP64 path solving the same runs one after another.
    Host wall time around the stepping (creation excluded on all sides), slowest rank's
    for the batched sides; every mixed run's final state against its plain FP64 run's."""
    import time

    import torch

    from solprop_b200 import _lib, scan

    points = scan.draw_points(n_runs, seed)
    points = [points[i] for i in scan.shard(points, rank, world)]
    built = [scan.capillary_record(p) for p in points]
    records, policies = [b[0] for b in built], [b[1] for b in built]
    sides = {}
    finals = {}
    for precision in ("mixed", "fp64") if batched_fp64 else ("mixed",):
        sc = _lib.Scan(records, policies, device, precision)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        while sc.advance(1000).active:
            pass
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
        runs = [sc.run(i) for i in range(len(records))]
        finals[precision] = [state for state, _ in runs]
        sides[precision] = {
            "seconds": seconds, "attempts": sum(int(i.attempts) for _, i in runs),
            "finished": sum(int(i.event) == 2 for _, i in runs),
            "plan": [line for line in sc.describe().splitlines() if line.startswith("work lists")]}
        sc.close()
    batched_s = sides["mixed"]["seconds"]
    finished = sides["mixed"]["finished"]
    plain_s, plain_attempts, plain_finals = 0.0, 0, []
    for rec, pol in zip(records, policies):
        problem = _lib.Problem(rec)
        ws = _lib.Workspace(problem, device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        session = ws.start(pol)
        while session.advance(4096).event not in (2, 3):
            pass
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
        plain_attempts += int(session.batch.attempts)
        plain_finals.append(session.export())
        session.close()
        ws.close()
        problem.close()
    errors = run_errors(finals["mixed"], plain_finals, records)
    batched64_s = sides["fp64"]["seconds"] if "fp64" in sides else None
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([batched_s, batched64_s or 0.0, plain_s], dtype=torch.float64,
                         device=f"cuda:{device}")
        dist.all_reduce(t[:2], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[2:], op=dist.ReduceOp.SUM)
        batched_s, plain_s = float(t[0].item()), float(t[2].item())
        batched64_s = float(t[1].item()) if batched64_s is not None else None
    out = {"runs": n_runs, "finished": finished * world if world > 1 else finished,
           "batched_mixed": {"seconds": batched_s, "runs_per_s": n_runs / batched_s,
                             "attempts": sides["mixed"]["attempts"], "plan": sides["mixed"]["plan"]},
           "plain_fp64": {"seconds": plain_s, "runs_per_s": n_runs / plain_s, "attempts": plain_attempts},
           "runs_per_s_ratio": plain_s / batched_s,
           "mixed_vs_fp64": errors}
    if batched64_s is not None:
        out["batched_fp64"] = {"seconds": batched64_s, "runs_per_s": n_runs / batched64_s,
                               "attempts": sides["fp64"]["attempts"], "plan": sides["fp64"]["plan"],
                               "runs_per_s_ratio": plain_s / batched64_s}
    return out


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=200)
    parser.add_argument("--warmup", type=int, default=10)
    parser.add_argument("--impl", default="ours", choices=["ours", "reference"])
    parser.add_argument("--cpu-budget", type=float, default=20.0)
    parser.add_argument("--scan-runs", type=int, default=256)
    parser.add_argument("--scan-steps", type=int, default=30)
    parser.add_argument("--complete-runs", type=int, default=256,
                        help="scan runs solved to the end for the runs/s comparison (0: skip)")
    parser.add_argument("--config2-only", action="store_true",
                        help="measure config 2 alone (no runs, surrogate or scan legs), e.g. under ncu")
    parser.add_argument("--scan-only", type=int, default=0, metavar="RUNS",
                        help="only the full-batch scan leg over RUNS runs (--scan-steps batch "
                             "steps after --warmup), e.g. under ncu; prints its JSON")
    parser.add_argument("--surrogate-only", type=int, default=0, metavar="POINTS",
                        help="only the surrogate's tcgen05 inference over POINTS points; prints its JSON")
    parser.add_argument("--config3-only", type=int, nargs="?", const=128, default=0, metavar="GRID",
                        help="only config 3's route (30 vector modes on GRID x GRID nodes, default 128); "
                             "prints its JSON")
    parser.add_argument("--modal-only", type=int, nargs="?", const=16384, default=0, metavar="NODES",
                        help="only the modal transform's products (30 modes, NODES nodes, default 16384: "
                             "config 3's size); prints its JSON")
    args = parser.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.scan_only or args.surrogate_only or args.modal_only or args.config3_only:
        import torch

        torch.cuda.set_device(local)
        if args.scan_only:
            result = scan_leg(local, args.scan_only, args.scan_steps, warmup=args.warmup)
        elif args.config3_only:
            result = config3_leg(local, grid=args.config3_only)
        elif args.modal_only:
            result = modal_products_leg(local, n_nodes=args.modal_only)
        else:
            result = surrogate_leg(local, points=args.surrogate_only)
        print(json.dumps(result), flush=True)
        return 0
    rec, pol = load_workload()
    config = {"workload": "config2: 4-mode He capillary 1.5 m 0.8->0 bar, n_to 16384, 64 nodes",
              "state": [rec.n_modes, rec.n_pol, rec.n_omega], "n_to": rec.n_to,
              "n_nodes": rec.n_nodes, "phi_terms": rec.n_phi_terms, "rtol": pol["rtol"],
              "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = os.cpu_count()
        done, elapsed = cpu_arm(rec, pol, args.steps, args.warmup, budget_s=150.0, threads=None)
        value = done / elapsed
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": args.gpus, "steps": done, "warmup": args.warmup,
                "ms_per_step": 1e3 * elapsed / done, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                                 "sample": f"{done} attempts of the config-2 run from z=0 "
                                           "(oracle port of numpy_ref, all host threads)"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch

    from solprop_b200 import _lib

    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    problem = _lib.Problem(rec)
    ws = _lib.Workspace(problem, local)
    stream = torch.cuda.ExternalStream(ws.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    # ---- device-resident throughput
    session = ws.start(pol)
    for _ in range(max(args.warmup, 3)):
        session.advance(1)
    times = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
            batch = session.advance(1)
            end.record(stream)
            times.append((start, end))
            if batch.event == 2:
                session = ws.start(pol)  # the run ended: start it again
        torch.cuda.synchronize()
    total_ms = sum(s.elapsed_time(e) for s, e in times)
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms / 1e3)

    # ---- per-kernel device times over a second timed pass (same steps, events per launch)
    session.set_timing(True)
    session.timing(reset=True)
    kernel_steps = min(args.steps, 100)
    for _ in range(kernel_steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        if session.advance(1).event == 2:
            session = ws.start(pol)
            session.set_timing(True)
    kernels = session.timing(reset=True)
    session.set_timing(False)
    launches_per_step = sum(c for c in (v[1] for v in kernels.values())) / kernel_steps
    top = max(kernels, key=lambda k: kernels[k][0])
    top_ms = kernels[top][0] / max(kernels[top][1], 1)
    algo = algorithmic_bytes(rec)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo.get(top, 0) / (top_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "unit": "GB/s", "frac": achieved / peak, "traffic": COLUMN_TRAFFIC if top == "response_column" else None,
                "algorithmic_bytes": algo.get(top, 0), "avg_launch_ms": top_ms,
                "kernels_ms_per_step": {k: v[0] / kernel_steps for k, v in kernels.items() if v[1]}}

    # ---- end to end through the C ABI from host memory
    field_host = torch.from_numpy(np.ascontiguousarray(rec.field0).view(np.float64)).pin_memory()
    out_host = torch.empty_like(field_host).pin_memory()
    e2e_steps = args.steps
    torch.cuda.synchronize()
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_ev.record(stream)
    s2 = ws.start(pol, field0=field_host.numpy().view(np.complex128).reshape(rec.field0.shape))
    for _ in range(e2e_steps):
        if s2.advance(1).event == 2:
            break
    result = s2.export()
    e_ev.record(stream)
    torch.cuda.synchronize()
    e2e_ms = s_ev.elapsed_time(e_ev)
    state_bytes = rec.n_cols * rec.n_omega * 16
    per_attempt_h2d = 2 * 1200 + 4000  # two stage-scalar slots and the Adams tables
    e2e = {"value": world * e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(state_bytes / e2e_steps + per_attempt_h2d),
           "d2h_bytes_per_step": int(state_bytes / e2e_steps + 32)}
    assert np.all(np.isfinite(result))

    cpu = None
    if rank == 0:
        done, elapsed = cpu_arm(rec, pol, steps=1000, warmup=1, budget_s=args.cpu_budget, threads=1)
        cpu = {"value": done / elapsed, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{done} attempts of the config-2 run from z=0 on one host thread "
                         f"({os.cpu_count()} cores on the box)"}

    runs_result = None if args.config2_only else runs_leg(local)
    surrogate_result = None if args.config2_only else surrogate_leg(local)
    modal_result = None if args.config2_only else modal_products_leg(local)
    config3_result = None if args.config2_only else config3_leg(local)
    scan_result = None
    if args.scan_runs > 0 and not args.config2_only:
        scan_result = scan_leg(local, args.scan_runs, args.scan_steps, warmup=3, rank=rank, world=world)
    if args.complete_runs > 0 and scan_result is not None:
        scan_result["complete"] = complete_scan_leg(local, args.complete_runs, rank=rank, world=world)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "clocks": clocks.summary(), "runs": runs_result, "scan": scan_result,
            "surrogate": surrogate_result, "modal_products": modal_result, "config3": config3_result}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del session, s2
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

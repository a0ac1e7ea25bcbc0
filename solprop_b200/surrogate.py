"""The scan surrogate: an ensemble of perceptrons from scan parameters to exit spectra.

Six inputs (core radius, length, gas id, pressure, pulse energy, FWHM) -> four hidden
layers of 512 GELU units -> the log10 exit spectral density on 2048 wavelengths from
100 nm to 4 um (``scan.exit_log_spectrum``).  Five members trained from different seeds
and shuffles form an ensemble; a point whose members disagree by more than a threshold
(the standard deviation over members of each output in log10 units, weighted by the mean
spectrum's energy there) is routed to the solver, whose solutions remain the measure of the
surrogate's error.  Targets are the exit log10 spectra floored at ``DECADES`` below each spectrum's
peak: the error measure weights bins by energy, and the floor keeps the empty bins' noise
out of the fit.

Every forward, backward and optimiser step runs in this library's kernels
(``csrc/mlp_kernels.cu``: BF16 tensor-core products with FP32 accumulation, FP32 master
weights and Adam); PyTorch only holds the device tensors.  Training data come from the
batched solver (``solve_points``).
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib, scan

HIDDEN = (512, 512, 512, 512)
N_IN = 6
N_OUT = 2048
DECADES = 6.0


def floored(y: np.ndarray) -> np.ndarray:
    """Log10 spectra floored at DECADES below each row's peak."""
    return np.maximum(y, np.max(y, axis=-1, keepdims=True) - DECADES).astype(np.float32)


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _check(status: int) -> None:
    _lib.check(status)


def _bind():
    return _lib.library()


def gemm(a, b, c, *, trans_a=False, trans_b=False, bias=None, epilogue=0, pre=None, stream=None):
    """c = op(a) op(b) (+ bias) (GELU) on the tensor cores; shapes from the tensors."""
    lib = _bind()
    m = a.shape[1] if trans_a else a.shape[0]
    k = a.shape[0] if trans_a else a.shape[1]
    n = b.shape[0] if trans_b else b.shape[1]
    kb = b.shape[1] if trans_b else b.shape[0]
    if kb != k or tuple(c.shape) != (m, n):
        raise ValueError(f"gemm shapes: op(a) {m}x{k}, op(b) {kb}x{n}, c {tuple(c.shape)}")
    _check(lib.sp_mlp_gemm(_ptr(a), a.stride(0), int(trans_a), _ptr(b), b.stride(0), int(trans_b),
                           _ptr(c), c.stride(0), m, n, k,
                           _ptr(bias) if bias is not None else None, epilogue,
                           _ptr(pre) if pre is not None else None, stream))


def gemm_tc(a16, w16, *, out=None, out16=None, bias=None, epilogue=0, status=None, stream=None):
    """out / out16 = a16 w16^T (+ bias) (GELU) on the tcgen05 tensor cores; a16 (M, K) and
    w16 (N, K) are BF16 tensors with K a multiple of 64 and N a multiple of 256."""
    import torch

    lib = _bind()
    m, k = a16.shape
    n, kw = w16.shape
    if kw != k:
        raise ValueError(f"gemm_tc shapes: a {tuple(a16.shape)}, w {tuple(w16.shape)}")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=a16.device)
    _check(lib.sp_mlp_gemm_tc(_ptr(a16), a16.stride(0), _ptr(w16), w16.stride(0),
                              _ptr(out) if out is not None else None, out.stride(0) if out is not None else 0,
                              _ptr(out16) if out16 is not None else None,
                              out16.stride(0) if out16 is not None else 0, m, n, k,
                              _ptr(bias) if bias is not None else None, epilogue, _ptr(status), stream))
    return status


def gemm_tc_batch(a16s, w16s, *, outs=None, outs16=None, biases=None, epilogue=0, status=None, stream=None):
    """gemm_tc for several operand sets of one shape (an ensemble's members through one
    layer) in one launch: out[q] / out16[q] = a16s[q] w16s[q]^T (+ biases[q]) (GELU)."""
    import ctypes as C

    import torch

    lib = _bind()
    count = len(a16s)
    m, k = a16s[0].shape
    n, kw = w16s[0].shape
    if kw != k or len(w16s) != count or any(a.shape != (m, k) or a.stride(0) != a16s[0].stride(0) for a in a16s) \
            or any(w.shape != (n, k) or w.stride(0) != w16s[0].stride(0) for w in w16s):
        raise ValueError("gemm_tc_batch: every product takes the same shapes and pitches")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=a16s[0].device)

    def pointers(ts):
        return (C.c_void_p * count)(*[_ptr(t) if t is not None else None for t in ts]) if ts is not None else None

    ld = outs[0].stride(0) if outs is not None else 0
    ld16 = outs16[0].stride(0) if outs16 is not None else 0
    _check(lib.sp_mlp_gemm_tc_batch(count, pointers(a16s), a16s[0].stride(0), pointers(w16s), w16s[0].stride(0),
                                    pointers(outs), ld, pointers(outs16), ld16, m, n, k, pointers(biases),
                                    epilogue, _ptr(status), stream))
    return status


def to_bf16(x, cols_out: int):
    """BF16 copy of an FP32 (rows, cols) tensor, zero-padded to cols_out columns."""
    import torch

    out = torch.empty((x.shape[0], cols_out), dtype=torch.bfloat16, device=x.device)
    _check(_bind().sp_mlp_to_bf16(_ptr(x), x.stride(0), x.shape[0], x.shape[1], _ptr(out), out.stride(0),
                                  cols_out, None))
    return out


def transpose_bf16(x, rows_pad: int):
    """The (cols, rows_pad) BF16 transpose of an FP32 or BF16 (rows, cols) tensor, zero-padded."""
    import torch

    out = torch.empty((x.shape[1], rows_pad), dtype=torch.bfloat16, device=x.device)
    _check(_bind().sp_mlp_transpose_bf16(_ptr(x), int(x.dtype == torch.bfloat16), x.stride(0), x.shape[0],
                                         x.shape[1], _ptr(out), out.stride(0), rows_pad, None))
    return out


def _pad64(n: int) -> int:
    return -(-n // 64) * 64


# ------------------------------------------------------------------ features and targets
def features(points) -> np.ndarray:
    """The six inputs of each point, each mapped onto [-1, 1] over the scan's ranges."""
    x = np.array([p.features for p in points], dtype=np.float64)
    lo = np.array([50e-6, 0.5, 0.0, 0.2, math.log(20e-6), 5e-15])
    hi = np.array([150e-6, 2.0, 2.0, 3.0, math.log(500e-6), 30e-15])
    x[:, 4] = np.log(x[:, 4])
    return (2.0 * (x - lo) / (hi - lo) - 1.0).astype(np.float32)


def energy_weighted_error(pred_log: np.ndarray, true_log: np.ndarray) -> np.ndarray:
    """Per point: sum_b P_b |log10 P^_b - log10 P_b| / sum_b P_b with P the solver's spectrum."""
    p = 10.0 ** (np.asarray(true_log, np.float64) - np.max(true_log, axis=-1, keepdims=True))
    return np.sum(p * np.abs(pred_log - true_log), axis=-1) / np.sum(p, axis=-1)


# ------------------------------------------------------------------ the solver's side
def solve_points(points, *, precision: str = "fp64", device: int = 0, chunk: int = 256,
                 max_batch_steps: int = 20000):
    """Exit log-spectra of the points from the batched solver; (spectra, finished mask,
    attempts per point).  Runs that have not finished after ``max_batch_steps`` attempts
    (or that failed) are marked unfinished."""
    spectra = np.zeros((len(points), N_OUT), np.float32)
    done = np.zeros(len(points), bool)
    attempts = np.zeros(len(points), np.int64)
    for s in range(0, len(points), chunk):
        part = points[s:s + chunk]
        built = [scan.capillary_record(p) for p in part]
        sc = _lib.Scan([b[0] for b in built], [b[1] for b in built], device, precision)
        steps = 0
        while steps < max_batch_steps:
            st = sc.advance(256)
            steps += 256
            if st.active == 0:
                break
        for j, (rec, _) in enumerate(built):
            state, info = sc.run(j)
            attempts[s + j] = info.attempts
            if info.event == 2:
                spectra[s + j] = scan.exit_log_spectrum(rec, state, N_OUT)
                done[s + j] = True
        sc.close()
    return spectra, done, attempts


# ------------------------------------------------------------------ one perceptron
class Perceptron:
    """One ensemble member: FP32 master weights and Adam moments on the device."""

    def __init__(self, seed: int, device: int = 0):
        import torch

        self.device = torch.device("cuda", device)
        sizes = (N_IN,) + HIDDEN + (N_OUT,)
        rng = np.random.default_rng(seed)
        self.weights, self.biases = [], []
        for fan_in, fan_out in zip(sizes[:-1], sizes[1:]):
            bound = math.sqrt(6.0 / (fan_in + fan_out)) if fan_out != N_OUT else math.sqrt(3.0 / fan_in)
            w = rng.uniform(-bound, bound, (fan_out, fan_in)).astype(np.float32)
            self.weights.append(torch.tensor(w, device=self.device))
            self.biases.append(torch.zeros(fan_out, dtype=torch.float32, device=self.device))
        self.params = [t for pair in zip(self.weights, self.biases) for t in pair]
        self.m1 = [torch.zeros_like(t) for t in self.params]
        self.m2 = [torch.zeros_like(t) for t in self.params]
        self.step = 0
        self.w16 = None  # BF16 copies for the tensor-core inference (K padded to 64)

    def refresh_bf16(self):
        """BF16 copies of the weights for ``infer`` (after initialisation or training)."""
        self.w16 = [to_bf16(w, -(-w.shape[1] // 64) * 64) for w in self.weights]

    def infer(self, x, status=None):
        """Outputs for x (rows) through the tcgen05 products: BF16 activations between the
        layers, FP32 accumulation, the output layer in FP32."""
        import torch

        if self.w16 is None:
            self.refresh_bf16()
        a = to_bf16(x, self.w16[0].shape[1])
        last = len(self.weights) - 1
        for i, (w16, b) in enumerate(zip(self.w16, self.biases)):
            if i == last:
                out = torch.empty((a.shape[0], w16.shape[0]), dtype=torch.float32, device=self.device)
                status = gemm_tc(a, w16, out=out, bias=b, epilogue=1, status=status)
                return out, status
            nxt = torch.empty((a.shape[0], w16.shape[0]), dtype=torch.bfloat16, device=self.device)
            status = gemm_tc(a, w16, out16=nxt, bias=b, epilogue=2, status=status)
            a = nxt

    def forward(self, x, keep: bool = False):
        """Outputs for x (rows); with ``keep`` the layers' inputs and pre-activations."""
        import torch

        a, cache = x, []
        last = len(self.weights) - 1
        for i, (w, b) in enumerate(zip(self.weights, self.biases)):
            out = torch.empty((a.shape[0], w.shape[0]), dtype=torch.float32, device=self.device)
            pre = torch.empty_like(out) if (keep and i != last) else None
            gemm(a, w, out, trans_b=True, bias=b, epilogue=1 if i == last else 2, pre=pre)
            cache.append((a, pre))
            a = out
        return a, cache

    def forward_tc(self, x, keep: bool = False, status=None):
        """The training's forward pass on the tcgen05 products (``gemm_tc``): BF16 operands,
        FP32 accumulation; the hidden layers write their pre-activations in FP32 and their
        activations in BF16 (epilogue 3).  Returns the output, the cache and the status."""
        import torch

        a = to_bf16(x, _pad64(x.shape[1]))
        cache = []
        last = len(self.weights) - 1
        for i, (w, b) in enumerate(zip(self.weights, self.biases)):
            w16 = to_bf16(w, _pad64(w.shape[1]))
            if i == last:
                out = torch.empty((a.shape[0], w.shape[0]), dtype=torch.float32, device=self.device)
                status = gemm_tc(a, w16, out=out, bias=b, epilogue=1, status=status)
                cache.append((x if i == 0 else a, None))
                return out, cache, status
            pre = torch.empty((a.shape[0], w.shape[0]), dtype=torch.float32, device=self.device)
            nxt = torch.empty((a.shape[0], w.shape[0]), dtype=torch.bfloat16, device=self.device)
            status = gemm_tc(a, w16, out=pre, out16=nxt, bias=b, epilogue=3, status=status)
            cache.append((x if i == 0 else a, pre if keep else None))
            a = nxt

    def gradients_tc(self, cache, dy, status=None):
        """dW, db of every layer from dL/dy on the tcgen05 products: the weight gradient
        dz^T a and the input gradient dz W as products C = A W^T of BF16 transposes (the
        batch zero-padded to a multiple of 64); the first layer's 6-input weight gradient,
        below the products' 256-column tiles, on the FP32 path.  Returns (grads, status)."""
        import torch

        lib = _bind()
        grads = [None] * len(self.params)
        g = dy
        rows = _pad64(dy.shape[0])
        for i in range(len(self.weights) - 1, -1, -1):
            a, pre = cache[i]
            w = self.weights[i]
            if pre is not None:
                dz = torch.empty_like(g)
                _check(lib.sp_mlp_gelu_backward(_ptr(g), _ptr(pre), _ptr(dz), g.numel(), None))
                g = dz
            dw = torch.empty_like(w)
            if w.shape[1] % 256 == 0:
                status = gemm_tc(transpose_bf16(g, rows), transpose_bf16(a, rows), out=dw, status=status)
            else:
                gemm(g, a, dw, trans_a=True)
            db = torch.empty_like(self.biases[i])
            _check(lib.sp_mlp_bias_grad(_ptr(g), g.shape[0], g.shape[1], _ptr(db), None))
            grads[2 * i], grads[2 * i + 1] = dw, db
            if i:
                da = torch.empty((g.shape[0], w.shape[1]), dtype=torch.float32, device=self.device)
                status = gemm_tc(to_bf16(g, g.shape[1]), transpose_bf16(w, w.shape[0]), out=da, status=status)
                g = da
        return grads, status

    def gradients(self, cache, dy):
        """dW, db of every layer from dL/dy (the backward pass)."""
        import torch

        lib = _bind()
        grads = [None] * len(self.params)
        g = dy
        for i in range(len(self.weights) - 1, -1, -1):
            a, pre = cache[i]
            w = self.weights[i]
            if pre is not None:
                dz = torch.empty_like(g)
                _check(lib.sp_mlp_gelu_backward(_ptr(g), _ptr(pre), _ptr(dz), g.numel(), None))
                g = dz
            dw = torch.empty_like(w)
            gemm(g, a, dw, trans_a=True)
            db = torch.empty_like(self.biases[i])
            _check(lib.sp_mlp_bias_grad(_ptr(g), g.shape[0], g.shape[1], _ptr(db), None))
            grads[2 * i], grads[2 * i + 1] = dw, db
            if i:
                da = torch.empty((g.shape[0], w.shape[1]), dtype=torch.float32, device=self.device)
                gemm(g, w, da)
                g = da
        return grads

    def adam(self, grads, lr: float, betas=(0.9, 0.999), eps: float = 1e-8):
        lib = _bind()
        self.step += 1
        for p, g, m1, m2 in zip(self.params, grads, self.m1, self.m2):
            _check(lib.sp_mlp_adam(_ptr(p), _ptr(g), _ptr(m1), _ptr(m2), p.numel(), lr, betas[0],
                                   betas[1], eps, self.step, None))


def mse(y, t):
    """(loss tensor on the device, dL/dy)."""
    import torch

    lib = _bind()
    dy = torch.empty_like(y)
    rows = torch.empty(y.shape[0], dtype=torch.float32, device=y.device)
    loss = torch.empty(1, dtype=torch.float32, device=y.device)
    _check(lib.sp_mlp_mse(_ptr(y), _ptr(t), y.shape[0], y.shape[1], _ptr(dy), _ptr(rows), _ptr(loss),
                          None))
    return loss, dy


# ------------------------------------------------------------------ the ensemble
@dataclass
class Screen:
    prediction: np.ndarray  # (n, 2048) log10 spectra: the surrogate's, or the solver's if flagged
    spread: np.ndarray      # (n,) ensemble disagreement
    flagged: np.ndarray     # (n,) bool: routed to the solver


class Ensemble:
    def __init__(self, members: int = 5, seed: int = 0, device: int = 0):
        self.members = [Perceptron(seed + 1000 * k, device) for k in range(members)]
        self.device = device
        self.y_mean = None
        self.y_scale = None

    def fit(self, x: np.ndarray, y: np.ndarray, *, epochs: int = 200, batch: int = 256,
            lr: float = 1e-3, seed: int = 0, log=None):
        """Train every member on (features, log10 spectra); returns the last epoch's mean loss."""
        import torch

        dev = torch.device("cuda", self.device)
        y = floored(y)
        self.y_mean = y.mean(axis=0).astype(np.float32)
        self.y_scale = np.maximum(y.std(axis=0), 1e-3).astype(np.float32)
        xt = torch.tensor(x, device=dev)
        yt = torch.tensor((y - self.y_mean) / self.y_scale, device=dev)
        n = x.shape[0]
        last = 0.0
        for k, member in enumerate(self.members):
            rng = np.random.default_rng(seed + k)
            for epoch in range(epochs):
                order = torch.tensor(rng.permutation(n), device=dev)
                total, count = torch.zeros((), device=dev), 0
                rate = lr * 0.5 * (1.0 + math.cos(math.pi * epoch / epochs))  # cosine decay
                status = torch.zeros(1, dtype=torch.int32, device=dev)
                for s in range(0, n - batch + 1, batch):
                    idx = order[s:s + batch]
                    xb, yb = xt[idx].contiguous(), yt[idx].contiguous()
                    out, cache, status = member.forward_tc(xb, keep=True, status=status)
                    loss, dy = mse(out, yb)
                    grads, status = member.gradients_tc(cache, dy, status=status)
                    member.adam(grads, rate)
                    total += loss[0]
                    count += 1
                if int(status.item()):
                    raise RuntimeError("a tensor-core product's wait gave up during training")
                if log and (epoch % 50 == 0 or epoch == epochs - 1):
                    log(f"member {k} epoch {epoch} loss {float(total) / max(count, 1):.4e}")
            last = float(total) / max(count, 1)
            member.refresh_bf16()
        return last

    def infer(self, x, status=None):
        """Every member's outputs for x (rows), (members, rows, N_OUT) in FP32: the tcgen05
        products with all members through a layer in one launch (BF16 activations between
        the layers, FP32 accumulation), the same arithmetic as Perceptron.infer."""
        import torch

        for member in self.members:
            if member.w16 is None:
                member.refresh_bf16()
        first = self.members[0]
        a = to_bf16(x, first.w16[0].shape[1])
        acts = [a] * len(self.members)
        last = len(first.weights) - 1
        for i in range(last + 1):
            ws = [member.w16[i] for member in self.members]
            bs = [member.biases[i] for member in self.members]
            if i == last:
                out = torch.empty((len(self.members), a.shape[0], ws[0].shape[0]), dtype=torch.float32,
                                  device=first.device)
                status = gemm_tc_batch(acts, ws, outs=list(out), biases=bs, epilogue=1, status=status)
                return out, status
            nxt = torch.empty((len(self.members), a.shape[0], ws[0].shape[0]), dtype=torch.bfloat16,
                              device=first.device)
            status = gemm_tc_batch(acts, ws, outs16=list(nxt), biases=bs, epilogue=2, status=status)
            acts = list(nxt)

    def predict(self, x: np.ndarray, chunk: int = 16384):
        """Ensemble mean (log10 spectra) and disagreement of every row of x."""
        import torch

        lib = _bind()
        dev = torch.device("cuda", self.device)
        n, e = x.shape[0], len(self.members)
        mean = np.empty((n, N_OUT), np.float32)
        spread = np.empty(n, np.float32)
        scale = torch.tensor(self.y_scale, device=dev)
        offset = torch.tensor(self.y_mean, device=dev)
        for s in range(0, n, chunk):
            xb = torch.tensor(x[s:s + chunk], device=dev)
            m = xb.shape[0]
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            if m >= 128:
                ys, status = self.infer(xb, status)
                ys = ys * scale + offset
            else:
                ys = torch.stack([member.forward(xb)[0] for member in self.members]) * scale + offset
            if int(status.item()):
                raise RuntimeError("a tensor-core product's wait gave up")
            mu = torch.empty((m, N_OUT), dtype=torch.float32, device=dev)
            sd = torch.empty(m, dtype=torch.float32, device=dev)
            _check(lib.sp_mlp_ensemble_stats(_ptr(ys), e, m, N_OUT, _ptr(mu), _ptr(sd), None))
            mean[s:s + m] = mu.cpu().numpy()
            spread[s:s + m] = sd.cpu().numpy()
        return mean, spread

    def screen(self, points, *, threshold: float = 5e-3, precision: str = "fp64",
               device: int = 0) -> Screen:
        """Predict every point; re-solve the points whose disagreement exceeds the threshold."""
        mean, spread = self.predict(features(points))
        flagged = spread > threshold
        out = mean.copy()
        if flagged.any():
            idx = np.flatnonzero(flagged)
            spectra, done, _ = solve_points([points[i] for i in idx], precision=precision, device=device)
            out[idx[done]] = spectra[done]
        return Screen(out, spread, flagged)


# ------------------------------------------------------------------ the screening study
def plain_seconds_per_point(points, device: int = 0, max_attempts: int = 8192):
    """Mean device time of whole plain FP64 solves, one run at a time (the path a scan
    without the surrogate takes), over the points that finish within ``max_attempts``."""
    import time

    import torch

    total, count = 0.0, 0
    for p in points:
        rec, pol = scan.capillary_record(p)
        problem = _lib.Problem(rec)
        ws = _lib.Workspace(problem, device)
        session = ws.start(pol)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch = session.advance(max_attempts)
        torch.cuda.synchronize()
        if batch.event == 2:
            total += time.perf_counter() - t0
            count += 1
        session.close()
        ws.close()
        problem.close()
    return total / max(count, 1), count


def study(*, n_train: int = 4096, n_screen: int = 100_000, threshold: float = 5e-3, epochs: int = 600,
          max_batch_steps: int = 4096, resolve_cap: int = 256, device: int = 0, seed: int = 2025,
          log=print) -> dict:
    """Train the ensemble on solver runs, screen ``n_screen`` seeded points, score a held-out
    1 % against plain FP64 solves.  Returns the figures as a dict."""
    import time

    import torch

    train_pts = scan.draw_points(n_train, seed, modes=(1, 4), grids=(13,))
    t0 = time.perf_counter()
    y_train, ok, att = solve_points(train_pts, precision="mixed", device=device,
                                    max_batch_steps=max_batch_steps)
    t_gen = time.perf_counter() - t0
    log(f"training runs: {int(ok.sum())} of {n_train} finished in {t_gen:.1f} s")
    x_train = features(train_pts)
    ens = Ensemble(members=5, seed=seed, device=device)
    t0 = time.perf_counter()
    loss = ens.fit(x_train[ok], y_train[ok], epochs=epochs, batch=128, lr=1e-3, seed=seed, log=log)
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0
    screen_pts = scan.draw_points(n_screen, seed + 1, modes=(1, 4), grids=(13,))
    x_screen = features(screen_pts)
    ens.predict(x_screen[:4096])  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mean, spread = ens.predict(x_screen)
    torch.cuda.synchronize()
    t_infer = time.perf_counter() - t0
    flagged = spread > threshold
    # held-out 1 %: every 100th screened point, re-solved with plain FP64
    held = np.arange(0, n_screen, 100)
    t0 = time.perf_counter()
    y_held, ok_held, _ = solve_points([screen_pts[i] for i in held], precision="fp64", device=device,
                                      max_batch_steps=max_batch_steps)
    t_held = time.perf_counter() - t0
    err = energy_weighted_error(mean[held], floored(y_held))
    routed = np.where(flagged[held], 0.0, err)  # flagged points take the solver's spectrum
    # the flagged points' re-solve: every one up to the cap, the cost measured on those
    idx = np.flatnonzero(flagged)[:resolve_cap]
    t0 = time.perf_counter()
    _, ok_flag, _ = solve_points([screen_pts[i] for i in idx], precision="fp64", device=device,
                                 max_batch_steps=max_batch_steps)
    t_resolve = time.perf_counter() - t0
    plain_s, plain_n = plain_seconds_per_point([screen_pts[i] for i in held[:16]], device)
    # what the network gains over no network: the training set's mean spectrum as the guess
    mean_guess = energy_weighted_error(np.broadcast_to(ens.y_mean, y_held.shape), floored(y_held))
    per_point = t_infer / n_screen
    sweep = []
    for thr in (5e-3, 1e-2, 2e-2, 5e-2, 1e-1, 2e-1):
        flag = spread > thr
        keep = ok_held & ~flag[held]
        sweep.append({
            "threshold": thr, "flagged_fraction": float(flag.mean()),
            "unflagged_held_out": int(keep.sum()),
            "unflagged_error_median": float(np.median(err[keep])) if keep.any() else None,
            "unflagged_error_p90": float(np.percentile(err[keep], 90)) if keep.any() else None,
            "speedup_vs_plain": plain_s / (per_point + float(flag.mean()) * plain_s),
        })
    result = {
        "n_train": n_train, "train_finished": int(ok.sum()), "train_generation_s": t_gen,
        "train_attempts_median": float(np.median(att)), "fit_s": t_fit, "final_loss": loss,
        "n_screen": n_screen, "inference_s": t_infer, "points_per_s": n_screen / t_infer,
        "threshold": threshold, "flagged": int(flagged.sum()),
        "held_out": int(ok_held.sum()), "held_out_total": len(held), "held_out_s": t_held,
        "surrogate_error_median": float(np.median(err[ok_held])),
        "surrogate_error_p90": float(np.percentile(err[ok_held], 90)),
        "screened_error_median": float(np.median(routed[ok_held])),
        "screened_error_p90": float(np.percentile(routed[ok_held], 90)),
        "screened_error_max": float(np.max(routed[ok_held])),
        "unflagged_error_max": float(np.max(err[ok_held & ~flagged[held]])) if np.any(ok_held & ~flagged[held]) else None,
        "resolved_flagged": int(len(idx)), "resolved_flagged_finished": int(ok_flag.sum()),
        "resolve_s": t_resolve,
        "plain_seconds_per_point": plain_s, "plain_points_timed": plain_n,
        "speedup_screen_vs_plain": plain_s / (t_infer / n_screen),
        "mean_spectrum_error_median": float(np.median(mean_guess[ok_held])),
        "threshold_sweep": sweep,
    }
    log(str(result))
    return result


def main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Train the scan surrogate and screen a scan.")
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--screen", type=int, default=100_000)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--threshold", type=float, default=5e-3)
    ap.add_argument("--max-batch-steps", type=int, default=4096)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    res = study(n_train=args.train, n_screen=args.screen, epochs=args.epochs, threshold=args.threshold,
                max_batch_steps=args.max_batch_steps)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

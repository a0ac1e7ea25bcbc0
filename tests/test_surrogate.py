"""The scan surrogate: its CPU oracle (gradient-checked by differences) and the device
kernels against the oracle; then a small surrogate trained on solver runs, screened."""

import numpy as np
import pytest

from oracle import mlp as O


def _small_net(seed=0, sizes=(6, 32, 32, 16)):
    rng = np.random.default_rng(seed)
    ws = [rng.normal(0, 1 / np.sqrt(a), (b, a)) for a, b in zip(sizes[:-1], sizes[1:])]
    bs = [rng.normal(0, 0.1, b) for b in sizes[1:]]
    return ws, bs


def test_oracle_gradients_match_central_differences():
    ws, bs = _small_net()
    rng = np.random.default_rng(1)
    x, t = rng.normal(size=(9, 6)), rng.normal(size=(9, 16))
    y, cache = O.forward(ws, bs, x, rounded=False)
    _, dy = O.mse(y, t)
    grads = O.backward(ws, cache, dy, rounded=False)
    for layer, index in [(0, (3, 2)), (1, (7, 30)), (2, (15, 0)), (2, (4, 11))]:
        num = O.numeric_gradient(ws, bs, x, t, layer, index)
        assert abs(grads[layer][0][index] - num) <= 1e-6 * max(1.0, abs(num)), (layer, index)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0078125, 1e-3], np.float32)
    r = O.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway: to the even mantissa
    assert r[2] == 1.0078125            # above halfway: up
    assert r[3] == -3.0                 # halfway below: to even
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8


# ---------------------------------------------------------------------------- device
gpu = pytest.mark.gpu


def _torch():
    import torch

    return torch


@gpu
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("shape", [(200, 130, 70), (5, 2048, 512), (512, 6, 3)])
def test_gemm_matches_bf16_oracle(ta, tb, shape):
    from solprop_b200 import surrogate as S

    torch = _torch()
    m, n, k = shape
    rng = np.random.default_rng(m + n + k + 2 * ta + tb)
    a = rng.normal(size=(k, m) if ta else (m, k)).astype(np.float32)
    b = rng.normal(size=(n, k) if tb else (k, n)).astype(np.float32)
    bias = rng.normal(size=n).astype(np.float32)
    A = torch.tensor(a, device="cuda")
    B = torch.tensor(b, device="cuda")
    Cd = torch.empty((m, n), device="cuda")
    S.gemm(A, B, Cd, trans_a=bool(ta), trans_b=bool(tb), bias=torch.tensor(bias, device="cuda"), epilogue=1)
    opa = a.T if ta else a
    opb = b.T if tb else b
    ref = O.bf16(opa) @ O.bf16(opb) + bias
    got = Cd.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref)) + 1e-6


@gpu
@pytest.mark.parametrize("shape", [(300, 512, 512), (1000, 2048, 512), (128, 512, 64), (4096, 256, 128)])
def test_tcgen05_gemm_matches_bf16_oracle(shape):
    """The tcgen05 product (TMA tiles, tensor-memory accumulator) against the same BF16
    operands multiplied in float64: FP32 accumulation error only."""
    from solprop_b200 import surrogate as S

    torch = _torch()
    m, n, k = shape
    rng = np.random.default_rng(m + n + k)
    a = rng.normal(size=(m, k)).astype(np.float32)
    w = rng.normal(size=(n, k)).astype(np.float32)
    bias = rng.normal(size=n).astype(np.float32)
    a16 = torch.tensor(a, device="cuda").to(torch.bfloat16)
    w16 = torch.tensor(w, device="cuda").to(torch.bfloat16)
    out = torch.empty((m, n), device="cuda")
    out16 = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    status = S.gemm_tc(a16, w16, out=out, out16=out16, bias=torch.tensor(bias, device="cuda"), epilogue=2)
    assert int(status.item()) == 0
    ref = O.gelu(O.bf16(a) @ O.bf16(w).T + bias)
    got = out.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 2e-5 * np.max(np.abs(ref)) + 1e-5
    assert np.allclose(out16.float().cpu().numpy(), got, rtol=1e-2, atol=1e-2)


@gpu
def test_inference_on_tcgen05_matches_the_training_path():
    from solprop_b200 import surrogate as S

    torch = _torch()
    net = S.Perceptron(seed=11)
    x = torch.tensor(np.random.default_rng(1).uniform(-1, 1, (700, 6)).astype(np.float32), device="cuda")
    y_train, _ = net.forward(x)
    y_infer, status = net.infer(x)
    assert int(status.item()) == 0
    a, b = y_infer.cpu().numpy(), y_train.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b)


@gpu
def test_ensemble_products_in_one_launch_match_each_member():
    """Every member through a layer in one launch (the persistent kernel walks all their
    tiles) gives each member's own products bit for bit, on a row count that leaves a
    partial last row tile."""
    from solprop_b200 import surrogate as S

    torch = _torch()
    ens = S.Ensemble(members=3, seed=4)
    x = torch.tensor(np.random.default_rng(2).uniform(-1, 1, (700, 6)).astype(np.float32), device="cuda")
    ys, status = ens.infer(x)
    assert int(status.item()) == 0 and tuple(ys.shape) == (3, 700, S.N_OUT)
    for k, member in enumerate(ens.members):
        y, st = member.infer(x)
        assert int(st.item()) == 0
        assert torch.equal(ys[k], y)


@gpu
def test_gelu_epilogue_and_preactivation():
    from solprop_b200 import surrogate as S

    torch = _torch()
    rng = np.random.default_rng(3)
    a, w, b = rng.normal(size=(64, 40)), rng.normal(size=(96, 40)) / 6, rng.normal(size=96)
    A, W, Bv = (torch.tensor(v, dtype=torch.float32, device="cuda") for v in (a, w, b))
    out, pre = torch.empty((64, 96), device="cuda"), torch.empty((64, 96), device="cuda")
    S.gemm(A, W, out, trans_b=True, bias=Bv, epilogue=2, pre=pre)
    z = O.bf16(a.astype(np.float32)) @ O.bf16(w.astype(np.float32)).T + b.astype(np.float32)
    assert np.allclose(pre.cpu().numpy(), z, rtol=1e-5, atol=1e-5)
    assert np.allclose(out.cpu().numpy(), O.gelu(z), rtol=1e-5, atol=1e-5)


@gpu
def test_backward_matches_oracle_gradients():
    """Forward and backward of a full-size member (6 -> 4 x 512 -> 2048) on a batch of 64:
    the device gradients against the oracle's, both with BF16 operands (the device
    accumulates in FP32, the oracle in FP64, so a product's rounding to BF16 can differ
    by one unit in rare elements): relative L2 per tensor at most 2e-2."""
    from solprop_b200 import surrogate as S

    torch = _torch()
    net = S.Perceptron(seed=7)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (64, 6)).astype(np.float32)
    t = rng.normal(size=(64, 2048)).astype(np.float32)
    xt, tt = torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda")
    y, cache = net.forward(xt, keep=True)
    loss, dy = S.mse(y, tt)
    grads = net.gradients(cache, dy)
    ws = [w.cpu().numpy().astype(np.float64) for w in net.weights]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.biases]
    yo, co = O.forward(ws, bs, x)
    lo, dyo = O.mse(yo, t)
    go = O.backward(ws, co, dyo)
    assert np.linalg.norm(y.cpu().numpy() - yo) <= 1e-3 * np.linalg.norm(yo)
    assert abs(float(loss.cpu()[0]) - lo) <= 1e-4 * lo
    for i, (dw, db) in enumerate(go):
        gw, gb = grads[2 * i].cpu().numpy(), grads[2 * i + 1].cpu().numpy()
        assert np.linalg.norm(gw - dw) <= 2e-2 * np.linalg.norm(dw), i
        assert np.linalg.norm(gb - db) <= 2e-2 * np.linalg.norm(db), i


@gpu
def test_tcgen05_training_pass_matches_oracle_gradients():
    """The training's forward and backward on the tcgen05 products (``forward_tc``,
    ``gradients_tc``: BF16 transposes, the batch zero-padded) for a full-size member on a
    batch of 40: output within 1e-3 and every gradient within 2e-2 (relative L2) of the
    oracle's with BF16 operands."""
    from solprop_b200 import surrogate as S

    torch = _torch()
    net = S.Perceptron(seed=7)
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, (40, 6)).astype(np.float32)
    t = rng.normal(size=(40, 2048)).astype(np.float32)
    xt, tt = torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda")
    y, cache, status = net.forward_tc(xt, keep=True)
    loss, dy = S.mse(y, tt)
    grads, status = net.gradients_tc(cache, dy, status=status)
    assert int(status.item()) == 0
    ws = [w.cpu().numpy().astype(np.float64) for w in net.weights]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.biases]
    yo, co = O.forward(ws, bs, x)
    lo, dyo = O.mse(yo, t)
    go = O.backward(ws, co, dyo)
    assert np.linalg.norm(y.cpu().numpy() - yo) <= 1e-3 * np.linalg.norm(yo)
    for i, (dw, db) in enumerate(go):
        gw, gb = grads[2 * i].cpu().numpy(), grads[2 * i + 1].cpu().numpy()
        assert np.linalg.norm(gw - dw) <= 2e-2 * np.linalg.norm(dw), i
        assert np.linalg.norm(gb - db) <= 2e-2 * np.linalg.norm(db), i


@gpu
def test_adam_step_matches_its_formula():
    from solprop_b200 import _lib
    from solprop_b200.surrogate import _ptr

    torch = _torch()
    rng = np.random.default_rng(2)
    w, g = rng.normal(size=1000).astype(np.float32), rng.normal(size=1000).astype(np.float32)
    m1, m2 = rng.normal(size=1000).astype(np.float32), rng.uniform(0, 1, 1000).astype(np.float32)
    W, G, M1, M2 = (torch.tensor(v, device="cuda") for v in (w, g, m1, m2))
    _lib.check(_lib.library().sp_mlp_adam(_ptr(W), _ptr(G), _ptr(M1), _ptr(M2), 1000, 1e-3, 0.9, 0.999,
                                          1e-8, 3, None))
    a = 0.9 * m1 + 0.1 * g
    b = 0.999 * m2 + 0.001 * g * g
    ref = w - 1e-3 * (a / (1 - 0.9 ** 3)) / (np.sqrt(b / (1 - 0.999 ** 3)) + 1e-8)
    assert np.allclose(W.cpu().numpy(), ref, rtol=1e-5, atol=1e-7)


@gpu
def test_ensemble_statistics():
    from solprop_b200 import _lib
    from solprop_b200.surrogate import _ptr

    torch = _torch()
    rng = np.random.default_rng(4)
    y = rng.normal(size=(5, 33, 70)).astype(np.float32)
    Y = torch.tensor(y, device="cuda")
    mu, sd = torch.empty((33, 70), device="cuda"), torch.empty(33, device="cuda")
    _lib.check(_lib.library().sp_mlp_ensemble_stats(_ptr(Y), 5, 33, 70, _ptr(mu), _ptr(sd), None))
    mean = y.mean(0)
    weight = 10.0 ** (mean - mean.max(axis=1, keepdims=True))
    assert np.allclose(mu.cpu().numpy(), mean, atol=1e-6)
    assert np.allclose(sd.cpu().numpy(), (weight * y.std(0)).sum(1) / weight.sum(1), rtol=1e-4)


@gpu
def test_training_fits_and_screening_routes_disagreement():
    """A small ensemble trained on the device on a smooth stand-in target (a fixed random
    perceptron): its held-out error falls far below the untrained network's, and points far
    outside the training range are the ones the ensemble flags."""
    from solprop_b200 import surrogate as S

    rng = np.random.default_rng(0)
    teacher_w, teacher_b = _small_net(9, sizes=(6, 64, 2048))
    x = rng.uniform(-1, 1, (2048, 6)).astype(np.float32)
    y = (np.tanh(x @ teacher_w[0].T + teacher_b[0]) @ teacher_w[1].T / 4).astype(np.float32)
    ens = S.Ensemble(members=3, seed=1)
    ens.fit(x[:1792], y[:1792], epochs=40, batch=128, lr=2e-3)
    mean, spread = ens.predict(x[1792:])
    err = np.sqrt(np.mean((mean - y[1792:]) ** 2))
    untrained = S.Ensemble(members=1, seed=5)
    untrained.y_mean, untrained.y_scale = ens.y_mean, ens.y_scale
    base, _ = untrained.predict(x[1792:])
    assert err < 0.25 * np.sqrt(np.mean((base - y[1792:]) ** 2))
    far = rng.uniform(4, 6, (64, 6)).astype(np.float32)
    _, far_spread = ens.predict(far)
    assert np.median(far_spread) > 3 * np.median(spread)


@pytest.mark.gpu
def test_trained_network_gains_over_the_method_without_it():
    """On the solver's own data (config 5's distribution: 1-4 modes, n_to 8192, exit
    spectra from the batched mixed solver): without the network, the best guess of a
    point's exit spectrum is the training runs' mean spectrum; the trained ensemble beats
    that guess on held-out points."""
    from solprop_b200 import scan
    from solprop_b200 import surrogate as S

    points = scan.draw_points(160, 11, modes=(1, 4), grids=(13,))
    spectra, done, _ = S.solve_points(points, precision="mixed", max_batch_steps=4096)
    keep = np.flatnonzero(done)
    assert keep.size >= 100
    x, y = S.features([points[i] for i in keep]), spectra[keep]
    n_train = keep.size - 24
    ens = S.Ensemble(members=3, seed=2)
    ens.fit(x[:n_train], y[:n_train], epochs=150, batch=32, lr=2e-3)
    mean, _ = ens.predict(x[n_train:])
    trained = S.energy_weighted_error(mean, y[n_train:])
    without = S.energy_weighted_error(np.broadcast_to(S.floored(y[:n_train]).mean(axis=0), mean.shape),
                                      y[n_train:])
    print(f"held-out energy-weighted error: trained median {np.median(trained):.3f}, "
          f"without the network {np.median(without):.3f}")
    assert np.median(trained) < 0.8 * np.median(without)

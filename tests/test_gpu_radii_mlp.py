"""Tensor-core learned-radii network kernels (no reference counterpart) against the numpy
oracle of the same network: forward output, input gradient (used for forces), training
gradient and Adam training.  The oracle applies BF16 rounding at the same points as the
kernels (inputs, weights, first-layer activations, backward deltas) and sums in f64, so the
remaining differences are FP32 accumulation order, tanhf, and rare BF16 rounding flips."""
import numpy as np
import pytest

import oracle as O
import ommb200

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def random_params(rng, features, targets=None):
    p = np.zeros(O.LR_N_PARAMS, np.float32)
    o = O.LR_OFF
    p[o["W1"]:o["b1"]] = rng.normal(0, 1 / np.sqrt(32), 2048)
    p[o["b1"]:o["W2"]] = rng.normal(0, 0.1, 64)
    p[o["W2"]:o["b2"]] = rng.normal(0, 1 / np.sqrt(64), 4096)
    p[o["b2"]:o["w3"]] = rng.normal(0, 0.1, 64)
    p[o["w3"]:o["b3"]] = rng.normal(0, 1 / np.sqrt(64), 64)
    p[o["b3"]] = 0.05
    p[o["mean"]:o["inv_std"]] = features.mean(0)
    p[o["inv_std"]:o["t_mean"]] = 1.0 / (features.std(0) + 1e-3)
    if targets is None:
        p[o["t_mean"]], p[o["t_scale"]] = 0.01, 0.02
    else:
        p[o["t_mean"]], p[o["t_scale"]] = targets.mean(), targets.std()
    return p


def synthetic_features(rng, n):
    return np.abs(rng.normal(2.0, 1.5, (n, 32))).astype(np.float32)


def dev(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("n", [1, 129, 1000, 20000])
def test_forward_and_input_gradient_match_oracle(n):
    rng = np.random.default_rng(n)
    g = synthetic_features(rng, n)
    p = random_params(rng, g)
    tail, dt = ommb200.radii_mlp_forward(dev(g), dev(p))
    torch.cuda.synchronize()
    tail, dt = tail.cpu().numpy().astype(np.float64), dt.cpu().numpy().astype(np.float64)
    y, cache = O.mlp_forward(p, g)
    P = O.mlp_unpack(p)
    ref_tail = y * float(P["t_scale"]) + float(P["t_mean"])
    ref_dt = O.mlp_input_grad(cache) * float(P["t_scale"])
    # normalised output error (units of the target scale)
    err_y = np.abs(tail - ref_tail) / float(P["t_scale"])
    print(f"n={n}: y max {err_y.max():.2e} rms {np.sqrt((err_y ** 2).mean()):.2e}; "
          f"dtail rms rel {rms_rel(dt, ref_dt):.2e}")
    assert np.sqrt((err_y ** 2).mean()) < 2e-3
    assert err_y.max() < 2e-2
    assert rms_rel(dt, ref_dt) < 5e-3
    # and against the unrounded f64 network: BF16-level agreement
    y64, c64 = O.mlp_forward(p, g, quantize=False)
    assert np.sqrt((((tail - float(P["t_mean"])) / float(P["t_scale"]) - y64) ** 2).mean()) < 3e-2
    assert rms_rel(dt, O.mlp_input_grad(c64) * float(P["t_scale"])) < 5e-2


def test_forward_without_gradient_gives_the_same_output():
    rng = np.random.default_rng(3)
    g = synthetic_features(rng, 700)
    p = random_params(rng, g)
    a, _ = ommb200.radii_mlp_forward(dev(g), dev(p), with_gradient=True)
    b, none = ommb200.radii_mlp_forward(dev(g), dev(p), with_gradient=False)
    assert none is None
    assert torch.equal(a, b)


@pytest.mark.parametrize("n", [128, 512])
def test_training_gradient_matches_oracle(n):
    rng = np.random.default_rng(10 + n)
    g = synthetic_features(rng, n)
    t = (0.02 * np.tanh(g[:, :4].sum(1) / 8.0) + rng.normal(0, 0.002, n)).astype(np.float32)
    p = random_params(rng, g, t)
    params = dev(p)
    moments = torch.zeros(2, ommb200.RADII_MLP_TRAINABLE, dtype=torch.float32, device="cuda")
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    loss, grad = ommb200.radii_mlp_train(dev(g), dev(t), params, moments, step, steps=1,
                                         batch=n, learning_rate=0.0, with_gradient=True)
    torch.cuda.synchronize()
    ref_loss, ref_grad = O.mlp_loss_grad(p, g, t)
    grad = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss[0]) - ref_loss) < 2e-3 * ref_loss
    o = O.LR_OFF
    for name, lo, hi in [("W1", o["W1"], o["b1"]), ("b1", o["b1"], o["W2"]),
                         ("W2", o["W2"], o["b2"]), ("b2", o["b2"], o["w3"]),
                         ("w3", o["w3"], o["b3"]), ("b3", o["b3"], o["b3"] + 1)]:
        e = rms_rel(grad[lo:hi], ref_grad[lo:hi])
        print(f"{name}: grad rms rel {e:.2e}")
        assert e < 1e-2, name
    assert np.array_equal(params.cpu().numpy(), p)  # lr 0 leaves the parameters unchanged
    assert int(step.cpu()[0]) == 1


def test_adam_step_matches_oracle_update():
    rng = np.random.default_rng(21)
    n = 256
    g = synthetic_features(rng, n)
    t = (0.02 * np.tanh(g[:, :4].sum(1) / 8.0)).astype(np.float32)
    p = random_params(rng, g, t)
    params = dev(p)
    moments = torch.zeros(2, ommb200.RADII_MLP_TRAINABLE, dtype=torch.float32, device="cuda")
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    _, grad = ommb200.radii_mlp_train(dev(g), dev(t), params, moments, step, steps=1, batch=n,
                                      learning_rate=1e-3, with_gradient=True)
    torch.cuda.synchronize()
    # apply the oracle's Adam to the kernel's own gradient: the update rule must agree
    pr = p.astype(np.float64).copy()
    m = np.zeros(O.LR_N_PARAMS)
    v = np.zeros(O.LR_N_PARAMS)
    O.adam_update(pr, m, v, grad.cpu().numpy().astype(np.float64), 1, 1e-3)
    got = params.cpu().numpy().astype(np.float64)
    assert np.abs(got - pr).max() < 1e-6
    mo = moments.cpu().numpy()
    assert np.abs(mo[0] - m[:O.LR_N_TRAIN]).max() < 1e-9 + 1e-6 * np.abs(m).max()


def test_training_fits_a_smooth_target_and_is_deterministic():
    rng = np.random.default_rng(5)
    n = 4096
    g = synthetic_features(rng, n)
    t = (0.02 * np.tanh((g[:, :8].sum(1) - g[:, 8:16].sum(1)) / 6.0) + 0.01).astype(np.float32)
    p = random_params(rng, g, t)
    runs = []
    for _ in range(2):
        params = dev(p)
        moments = torch.zeros(2, ommb200.RADII_MLP_TRAINABLE, dtype=torch.float32, device="cuda")
        step = torch.zeros(1, dtype=torch.int32, device="cuda")
        losses = []
        for _ in range(4):
            loss, _ = ommb200.radii_mlp_train(dev(g), dev(t), params, moments, step, steps=100,
                                              batch=1024, learning_rate=1e-3, seed=9)
            losses.append(loss.cpu().numpy())
        runs.append((params.cpu().numpy(), np.concatenate(losses)))
        assert int(step.cpu()[0]) == 400
    assert np.array_equal(runs[0][0], runs[1][0])
    losses = runs[0][1]
    print(f"loss {losses[:5].mean():.4f} -> {losses[-5:].mean():.4f}")
    assert losses[-20:].mean() < 0.2 * losses[:5].mean()
    # the trained network, evaluated by the inference kernel, predicts the targets
    tail, _ = ommb200.radii_mlp_forward(dev(g), dev(runs[0][0]), with_gradient=False)
    resid = tail.cpu().numpy() - t
    assert np.sqrt((resid ** 2).mean()) < 0.45 * t.std()

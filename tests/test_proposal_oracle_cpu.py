"""The FP64 oracle of the learned tile proposal on the CPU: its gradients against central finite differences, its
bfloat16 rounding against torch's, the vectorised features against the per-block definition, and Adam's first step
against its closed form."""

import numpy as np
import torch

import proposal


def small_case(seed=3, n=2, size=2 * proposal.HALO + proposal.TILE):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 2, size, size))
    labels = rng.normal(0.5, 0.3, (n, 1, 1))
    params = proposal.init_params(seed)
    # non-zero biases so every term of the gradient is exercised
    params = [(w, (0.1 * rng.normal(size=b.shape)).astype(np.float32)) for w, b in params]
    return x, labels, params


def test_gradients_match_finite_differences():
    x, labels, params = small_case()
    _, grads = proposal.loss_and_grads(x, labels, params, round_weights=False)
    rng = np.random.default_rng(9)
    eps = 1e-6
    checked = 0
    for li, (w, b) in enumerate(params):
        for which, arr in ((0, w), (1, b)):
            flat = arr.reshape(-1)
            for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
                def loss_at(delta):
                    p2 = [(ww.astype(np.float64).copy(), bb.astype(np.float64).copy()) for ww, bb in params]
                    p2[li][which].reshape(-1)[idx] += delta
                    return proposal.loss_and_grads(x, labels, p2, round_weights=False)[0]
                fd = (loss_at(eps) - loss_at(-eps)) / (2 * eps)
                an = grads[li][which].reshape(-1)[idx]
                assert abs(fd - an) <= 1e-8 + 1e-4 * abs(fd), (li, which, idx, fd, an)
                checked += 1
    assert checked >= 40


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-3, 1000), [0.0, -0.0, 1.0, 65504.0, 1.00390625, 1.01171875]])
    v = v.astype(np.float32)
    want = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(proposal.bf16(v), want)


def test_fast_features_equal_the_definition():
    rng = np.random.default_rng(2)
    words = (rng.integers(60, 900, (37, 53)) | (rng.integers(0, 2, (37, 53)) << 15)).astype(np.uint16)
    for x0, y0, fw, fh in ((0, 0, 13, 9), (-16, -16, 24, 24), (20, 8, 12, 10)):
        assert np.array_equal(proposal.features(words, x0, y0, fw, fh), proposal.features_fast(words, x0, y0, fw, fh))


def test_flat_parameters_round_trip():
    params = proposal.init_params(4)
    flat = proposal.flatten(params)
    assert flat.size == proposal.N_PARAMS
    back = proposal.unflatten(flat)
    assert all(np.array_equal(a, c) and np.array_equal(b, d) for (a, b), (c, d) in zip(params, back))


def test_adam_first_step_moves_each_weight_by_lr():
    x, labels, params = small_case()
    _, grads = proposal.loss_and_grads(x, labels, params)
    opt = proposal.Adam(params, lr=1e-3)
    new = opt.step(params, grads)
    for (w, b), (nw, nb), (gw, gb) in zip(params, new, grads):
        # after one step m / c1 = g and v / c2 = g^2: the update is lr * g / (|g| + eps)
        want = w.astype(np.float64) - 1e-3 * gw / (np.abs(gw) + 1e-8)
        assert np.allclose(nw, want.astype(np.float32), rtol=0, atol=1e-7)


def test_training_lowers_the_loss():
    x, labels, params = small_case(n=4)
    opt = proposal.Adam(params, lr=3e-3)
    l0 = proposal.loss_and_grads(x, labels, params)[0]
    for _ in range(30):
        _, g = proposal.loss_and_grads(x, labels, params)
        params = opt.step(params, g)
    assert proposal.loss_and_grads(x, labels, params)[0] < 0.5 * l0


def test_budget_threshold_known_answers():
    """Two scale-0 tiles of a 128 x 64 picture predicted at 0.5 and 2.0: a budget below the first tile's predicted
    contribution stops at the first tile's bin (0.5), one between the first and both stops at the second's (2.0), one
    above both skips everything (infinity); the threshold is a floor throughout, and tiles without a prediction add
    nothing."""
    import math

    w, h, k0, window = 128, 64, 4915, 9
    scale = 16.0 / (k0 * window * window)
    c1, c2 = scale * math.expm1(0.5) * 4096, scale * math.expm1(2.0) * 4096
    pred = np.array([0.5, 2.0], np.float32)
    assert proposal.budget_threshold(pred, w, h, k0, window, -1e30, 0.5 * c1) == 0.5
    assert proposal.budget_threshold(pred, w, h, k0, window, -1e30, c1 + 0.5 * c2) == 2.0
    assert proposal.budget_threshold(pred, w, h, k0, window, -1e30, 2 * (c1 + c2)) == np.inf
    assert proposal.budget_threshold(pred, w, h, k0, window, 1.0, 0.5 * c1) == 1.0
    assert proposal.budget_threshold(np.array([-np.inf, 2.0], np.float32), w, h, k0, window, -1e30, 0.5 * c2) == 2.0

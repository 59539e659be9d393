"""CPU checks of the proposal-network oracle (oracle/mlp.py): its backward
pass equals finite differences of its loss, and its BF16 rounding is the
round-to-nearest-even of the format."""
import numpy as np

import mlp as M


def test_bf16_rounding_is_nearest_even():
    # the bf16 spacing at 1 is 2^-7
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -3.14159265, 1e-30, 1.0 + 3 * 2 ** -8],
                 np.float64)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[3] == 1.0  # the tie 1 + 2^-8 goes to the even neighbour 1
    assert r[2] == 1.0 + 2 ** -7
    assert r[6] == 1.0 + 2 ** -6  # the tie 1 + 1.5 ulp goes to the even neighbour
    assert abs(r[4] + 3.140625) < 1e-12
    u = np.float32(r).view(np.uint32)
    assert np.all(u & 0xFFFF == 0)


def test_backward_matches_finite_differences():
    dims = (12, 64, 64, 12)
    rng = np.random.default_rng(1)
    p = M.init(dims, std=0.3, seed=2)
    for k in ("b1", "b2", "b3"):
        p[k] = rng.normal(0, 0.1, p[k].shape)
    X = rng.choice([-1.0, 1.0], size=(9, dims[0]))
    T = (rng.random((9, dims[3])) < 0.3).astype(np.float64)
    f = M.forward(p, X, bf=False)
    g = M.backward(f, T, bf=False)
    eps = 1e-6
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = p[k].ravel()
        for idx in rng.choice(flat.size, 6, replace=False):
            old = flat[idx]
            flat[idx] = old + eps
            lp = M.loss(M.forward(p, X, bf=False)["logits"], T)
            flat[idx] = old - eps
            lm = M.loss(M.forward(p, X, bf=False)["logits"], T)
            flat[idx] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[k].ravel()[idx]) < 1e-7 * max(1.0, abs(fd)), (k, idx, fd, g[k].ravel()[idx])


def test_soft_backward_matches_finite_differences():
    """The softmax cross entropy against soft targets (the learned proposals'
    loss over a move dictionary)."""
    dims = (12, 64, 64, 20)
    rng = np.random.default_rng(4)
    p = M.init(dims, std=0.3, seed=5)
    for k in ("b1", "b2", "b3"):
        p[k] = rng.normal(0, 0.1, p[k].shape)
    X = rng.choice([-1.0, 1.0], size=(7, dims[0]))
    T = rng.random((7, dims[3]))
    T /= T.sum(axis=1, keepdims=True)
    g = M.backward(M.forward(p, X, bf=False), T, bf=False, soft=True)
    eps = 1e-6
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = p[k].ravel()
        for idx in rng.choice(flat.size, 6, replace=False):
            old = flat[idx]
            flat[idx] = old + eps
            lp = M.loss_soft(M.forward(p, X, bf=False)["logits"], T)
            flat[idx] = old - eps
            lm = M.loss_soft(M.forward(p, X, bf=False)["logits"], T)
            flat[idx] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[k].ravel()[idx]) < 1e-7 * max(1.0, abs(fd)), (k, idx, fd, g[k].ravel()[idx])


def test_spins_to_input_convention():
    bits = np.array([[0b101, 0, 0, 0]], np.uint32)
    x = M.spins_to_input(bits, 4)
    assert x.tolist() == [[-1.0, 1.0, -1.0, 1.0]]

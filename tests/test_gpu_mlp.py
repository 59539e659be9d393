"""Proposal network on the GPU (tcgen05 BF16 GEMMs, FP32 accumulation)
against the CPU oracle oracle/mlp.py.  Layer by layer on the GPU's own BF16
inputs (FP32 accumulation order is the only difference: 1e-5 relative),
elementwise stages within one BF16 rounding step, and the full gradient
against the oracle's BF16-emulating backward pass."""
import numpy as np
import pytest

import mlp as M
import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

DIMS = [(128, 256, 256, 128), (32, 128, 64, 32), (18, 64, 64, 18)]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


def bf_close(a, b):
    """within one BF16 rounding step (2^-8 relative) plus a tiny absolute slack"""
    return np.all(np.abs(a - b) <= 2.0 ** -8 * np.abs(b) + 1e-6)


def setup(dims, B, seed=3, std=0.05, max_batch=None):
    rng = np.random.default_rng(seed)
    net = rbmnqs.ProposalNet(*dims, max_batch=max_batch or B)
    p = M.init(dims, std=std, seed=seed)
    for k in ("b1", "b2", "b3"):
        p[k] = rng.normal(0, 0.05, p[k].shape)
    net.set_params(rbmnqs.mlp_flatten(p))
    p = rbmnqs.mlp_unflatten(net.get_params(), dims)  # the FP32 values the GPU holds
    spins = O.random_spins(rng, B, dims[0])
    tgt = O.random_spins(rng, B, min(dims[3], 128))
    return net, p, spins, tgt


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("B", [256, 300])
def test_forward_layers_match_oracle(dims, B):
    net, p, spins, _ = setup(dims, B)
    logits = net.forward(spins)
    X = M.spins_to_input(spins, dims[0])
    W1, W2, W3 = (M.bf16(p[k]) for k in ("W1", "W2", "W3"))
    z1 = net.intermediate(2, B)[:, :dims[1]]
    a1 = net.intermediate(0, B)[:, :dims[1]]
    z2 = net.intermediate(3, B)[:, :dims[2]]
    a2 = net.intermediate(1, B)[:, :dims[2]]
    assert rel(z1, X @ W1.T + p["b1"]) < 1e-5
    assert bf_close(a1, M.bf16(M.gelu(z1.astype(np.float64))))
    assert rel(z2, a1 @ W2.T + p["b2"]) < 1e-5
    assert bf_close(a2, M.bf16(M.gelu(z2.astype(np.float64))))
    assert rel(logits, a2 @ W3.T + p["b3"]) < 1e-5
    # end to end against the BF16-emulating oracle
    f = M.forward(p, X)
    assert rel(logits, f["logits"]) < 2e-2


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("B,cap", [(512, 512), (300, 1024)])
def test_backward_layers_and_gradients_match_oracle(dims, B, cap):
    net, p, spins, tgt = setup(dims, B, max_batch=cap)
    loss, g = net.train_step(spins, tgt, apply=False)
    X = M.spins_to_input(spins, dims[0])
    T = M.spins_to_input(tgt, dims[3]) < 0  # bit set = 1
    T = T.astype(np.float64)
    W2, W3 = M.bf16(p["W2"]), M.bf16(p["W3"])
    logits = net.forward(spins)  # same weights: apply=False
    z1 = net.intermediate(2, B)[:, :dims[1]].astype(np.float64)
    z2 = net.intermediate(3, B)[:, :dims[2]].astype(np.float64)
    a1 = net.intermediate(0, B)[:, :dims[1]].astype(np.float64)
    a2 = net.intermediate(1, B)[:, :dims[2]].astype(np.float64)
    loss2, _ = net.train_step(spins, tgt, apply=False)
    g3 = net.intermediate(6, B)[:, :dims[3]].astype(np.float64)
    g2 = net.intermediate(5, B)[:, :dims[2]].astype(np.float64)
    g1 = net.intermediate(4, B)[:, :dims[1]].astype(np.float64)
    L = logits.astype(np.float64)
    assert abs(loss - M.loss(L, T)) < 1e-5 * abs(M.loss(L, T))
    assert bf_close(g3, M.bf16((1 / (1 + np.exp(-L)) - T) / B))
    assert bf_close(g2, M.bf16((g3 @ W3) * M.gelu_grad(z2)))
    assert bf_close(g1, M.bf16((g2 @ W2) * M.gelu_grad(z1)))
    grads = rbmnqs.mlp_unflatten(g, dims)
    ref = dict(W3=g3.T @ a2, b3=g3.sum(0), W2=g2.T @ a1, b2=g2.sum(0), W1=g1.T @ X, b1=g1.sum(0))
    for k in ref:
        assert rel(grads[k], ref[k]) < 1e-5, k
    # against the oracle's own BF16 backward pass from the same parameters
    f = M.forward(p, X)
    go = M.backward(f, T)
    for k in ("W1", "W2", "W3", "b1", "b2", "b3"):
        err = np.linalg.norm(grads[k] - go[k]) / np.linalg.norm(go[k])
        assert err < 2e-2, (k, err)


@pytest.mark.parametrize("dims,B", [((128, 256, 256, 256), 512), ((18, 64, 64, 27), 300)])
def test_soft_target_gradients_match_oracle(dims, B):
    """Softmax cross entropy over a move dictionary (the learned proposals'
    loss): dL/dlogits and the parameter gradients against the oracle."""
    net, p, spins, _ = setup(dims, B, max_batch=1024)
    rng = np.random.default_rng(8)
    T = rng.random((B, dims[3])) ** 4
    T /= T.sum(axis=1, keepdims=True)
    loss, g = net.train_step_soft(spins, T, apply=False)
    L = net.forward(spins).astype(np.float64)
    X = M.spins_to_input(spins, dims[0])
    T32 = T.astype(np.float32).astype(np.float64)
    assert abs(loss - M.loss_soft(L, T32)) < 1e-5 * abs(M.loss_soft(L, T32))
    net.train_step_soft(spins, T, apply=False)
    g3 = net.intermediate(6, B)[:, :dims[3]].astype(np.float64)
    assert bf_close(g3, M.bf16((np.exp(M.log_softmax(L)) - T32) / B))
    grads = rbmnqs.mlp_unflatten(g, dims)
    go = M.backward(M.forward(p, X), T32, soft=True)
    for k in ("W1", "W2", "W3", "b1", "b2", "b3"):
        err = np.linalg.norm(grads[k] - go[k]) / np.linalg.norm(go[k])
        assert err < 2e-2, (k, err)


def test_adam_steps_follow_oracle_and_reduce_loss():
    dims = (32, 128, 64, 32)
    B = 512
    net, p, spins, _ = setup(dims, B, std=0.1)
    # a learnable target: flip site i where sites i and i+1 agree
    n = dims[0]
    s0 = spins[:, 0].astype(np.uint64)
    rot = ((s0 >> 1) | ((s0 & 1) << (n - 1))) & ((1 << n) - 1)
    tgt = np.zeros_like(spins)
    tgt[:, 0] = (~(s0 ^ rot) & ((1 << n) - 1)).astype(np.uint32)
    X = M.spins_to_input(spins, dims[0])
    T = (M.spins_to_input(tgt, dims[3]) < 0).astype(np.float64)
    st = {}
    losses, ref = [], []
    for _ in range(30):
        l, _ = net.train_step(spins, tgt, lr=1e-2, apply=True, grads=False)
        losses.append(l)
        f = M.forward(p, X)
        ref.append(M.loss(f["logits"], T))
        p = M.adam(p, M.backward(f, T), st, lr=1e-2)
    assert losses[-1] < 0.6 * losses[0]
    # the GPU (FP32 master weights, BF16 GEMMs) follows the oracle's Adam trajectory
    assert np.all(np.abs(np.array(losses) - np.array(ref)) < 0.05 * np.array(ref))

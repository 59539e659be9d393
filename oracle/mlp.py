"""CPU oracle of the proposal network (test infrastructure only).

The learned-proposal extension has no counterpart in the reference; this is
the FP64 statement of the network the GPU kernels implement, used by the
tests to check the CUDA forward and backward passes:

    x (spins as +-1, n_in) -> z1 = W1 x + b1 -> a1 = GELU(z1)   (h1)
                           -> z2 = W2 a1 + b2 -> a2 = GELU(z2)  (h2)
                           -> l  = W3 a2 + b3                    (n_out flip logits)
    loss = (1/B) sum_b sum_i softplus(l_bi) - t_bi l_bi          (BCE with logits)
    or, for the learned proposals over a move dictionary,
    loss = -(1/B) sum_b sum_m t_bm log softmax(l_b)_m           (soft targets)

GELU is the erf form.  With bf16=True the values are rounded to bfloat16
(round to nearest even) at the points where the GPU stores them in BF16: the
weights, the activations a1 / a2 and the back-propagated dL/dz gradients;
everything else stays in FP64 here (FP32 on the GPU).
"""
import numpy as np
from math import sqrt

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(__import__("math").erf)

INV_SQRT2 = 1.0 / sqrt(2.0)
INV_SQRT2PI = 1.0 / sqrt(2.0 * np.pi)


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z * INV_SQRT2))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z * INV_SQRT2)) + z * INV_SQRT2PI * np.exp(-0.5 * z * z)


def init(dims=(128, 256, 256, 128), std=0.02, seed=0):
    """Weights N(0, std), biases zero; W_l has shape [out, in]."""
    rng = np.random.default_rng(seed)
    p = {}
    for l in range(3):
        p[f"W{l + 1}"] = rng.normal(0.0, std, (dims[l + 1], dims[l]))
        p[f"b{l + 1}"] = np.zeros(dims[l + 1])
    return p


def spins_to_input(bits, n):
    """[B] rows of 128-bit configurations (uint32[B, 4]) -> +-1 matrix [B, n]
    (bit set = spin down = -1, spin_state.cpp:44-62)."""
    bits = np.asarray(bits, dtype=np.uint64)
    idx = np.arange(n)
    b = (bits[:, idx // 32] >> (idx % 32).astype(np.uint64)) & 1
    return np.where(b == 1, -1.0, 1.0)


def forward(p, X, bf=True):
    r = (lambda v: bf16(v)) if bf else (lambda v: v)
    W1, W2, W3 = (r(p["W1"]), r(p["W2"]), r(p["W3"]))
    z1 = X @ W1.T + p["b1"]
    a1 = r(gelu(z1))
    z2 = a1 @ W2.T + p["b2"]
    a2 = r(gelu(z2))
    l = a2 @ W3.T + p["b3"]
    return dict(X=X, z1=z1, a1=a1, z2=z2, a2=a2, logits=l, W1=W1, W2=W2, W3=W3)


def loss(logits, T):
    B = logits.shape[0]
    return float(np.sum(np.logaddexp(0.0, logits) - T * logits) / B)


def log_softmax(logits):
    m = logits.max(axis=1, keepdims=True)
    return logits - m - np.log(np.exp(logits - m).sum(axis=1, keepdims=True))


def loss_soft(logits, T):
    """Soft-target softmax cross entropy -(1/B) sum_b sum_m T_bm log softmax(l_b)_m
    (the learned proposals' training loss; rows of T sum to 1)."""
    B = logits.shape[0]
    return float(-np.sum(T * log_softmax(logits)) / B)


def backward(f, T, bf=True, soft=False):
    """Gradients of loss() (soft=False) or loss_soft() (soft=True) with
    respect to W1..W3, b1..b3."""
    r = (lambda v: bf16(v)) if bf else (lambda v: v)
    B = f["logits"].shape[0]
    if soft:
        g3 = r((np.exp(log_softmax(f["logits"])) - T) / B)
    else:
        g3 = r((1.0 / (1.0 + np.exp(-f["logits"])) - T) / B)
    da2 = g3 @ f["W3"]
    g2 = r(da2 * gelu_grad(f["z2"]))
    da1 = g2 @ f["W2"]
    g1 = r(da1 * gelu_grad(f["z1"]))
    return dict(W3=g3.T @ f["a2"], b3=g3.sum(0), W2=g2.T @ f["a1"], b2=g2.sum(0), W1=g1.T @ f["X"], b1=g1.sum(0),
                g3=g3, g2=g2, g1=g1, da2=da2, da1=da1)


def adam(p, g, state, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on FP64 master weights (state: dict with t, m, v)."""
    state["t"] = state.get("t", 0) + 1
    t = state["t"]
    for k in p:
        m = state.setdefault("m" + k, np.zeros_like(p[k]))
        v = state.setdefault("v" + k, np.zeros_like(p[k]))
        m[...] = b1 * m + (1 - b1) * g[k]
        v[...] = b2 * v + (1 - b2) * g[k] ** 2
        mh = m / (1 - b1 ** t)
        vh = v / (1 - b2 ** t)
        p[k] = p[k] - lr * mh / (np.sqrt(vh) + eps)
    return p

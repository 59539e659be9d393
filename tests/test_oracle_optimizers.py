"""CPU checks of the oracle's restatements used by the optimizer, direct
solver and full-enumeration parity tests: the weighted aggregator against
the unweighted one, the full sampler's visiting order, the direct solve
against a dense solve, and the plugins' defining properties."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("n_bins", [1, 4, 32])
def test_weighted_aggregate_with_unit_weights_is_the_plain_aggregate(n_bins):
    rng = np.random.default_rng(0)
    x = rng.normal(size=256) + 1j * rng.normal(size=256)
    a = O.weighted_aggregate(x, np.ones(256), n_bins)
    b = O.stats(x, n_bins)
    assert abs(a["mean"] - b["mean"]) < 1e-13
    assert abs(a["var"] - b["var"]) < 1e-12
    assert abs(a["stddev"] - b["stddev"]) < 1e-12
    assert abs(a["tau"] - b["tau"]) < 1e-11


def test_weighted_aggregate_is_scale_invariant():
    rng = np.random.default_rng(1)
    x = rng.normal(size=128) + 0j
    w = rng.random(128)
    a, b = O.weighted_aggregate(x, w, 8), O.weighted_aggregate(x, 1e6 * w, 8)
    for k in ("mean", "var", "stddev", "tau"):
        assert abs(a[k] - b[k]) < 1e-9 * max(1.0, abs(a[k]))


@pytest.mark.parametrize("n,bits", [(6, 0), (6, 2), (8, 3), (5, 5)])
def test_full_order_is_a_gray_code_per_block(n, bits):
    nums = O.full_order(n, bits)
    assert sorted(nums.tolist()) == list(range(1 << n))
    per = 1 << (n - bits)
    for b in range(1 << bits):
        blk = nums[b * per:(b + 1) * per]
        assert blk[0] == b
        flips = blk[1:] ^ blk[:-1]
        assert np.all((flips & (flips - 1)) == 0)  # one bit per step
        assert np.all(flips >> bits > 0)            # only the high bits move


def test_direct_solve_matches_dense_solve():
    rng = np.random.default_rng(2)
    N, P = 64, 12
    Om = rng.normal(size=(N, P)) + 1j * rng.normal(size=(N, P))
    d = Om.mean(0)
    F = rng.normal(size=P) + 1j * rng.normal(size=P)
    diag = np.var(Om, axis=0, ddof=1)
    x = O.direct_solve(Om, d, F, 0.5, 1e-3, 0.1, diag, n_neural=8)
    S = Om.conj().T @ Om / N - np.outer(d.conj(), d)
    idx = np.arange(P)
    S[idx[:8], idx[:8]] *= 1.5
    S[idx[8:], idx[8:]] *= 1.6
    S[idx, idx] += 1e-3 * diag.max()
    assert np.allclose(S @ x, F, atol=1e-10)


def test_adam_first_step_is_lr_per_component():
    g = np.array([0.3 - 2j, -1e-3 + 5j, 4.0 + 0j])
    st = O.AdamPlugin(3, eps=1e-14).apply(g, 0.01)
    assert np.allclose(np.abs(st.real[g.real != 0]), 0.01)
    assert np.allclose(np.abs(st.imag[g.imag != 0]), 0.01)


def test_momentum_dialup_ramps_the_factor():
    m = O.MomentumPlugin(2, alpha=0.9, dialup=10.0)
    g = np.array([1.0 + 0j, 2.0 + 0j])
    s1 = m.apply(g, 1.0)  # dup 1e-2 after the first step: nearly plain SGD
    assert np.allclose(s1, g)
    m.apply(2 * g, 1.0)
    assert abs(m.dup - 1e-1) < 1e-15


def test_sgd_direction_divides_the_real_part():
    F = np.array([2.0 + 3j, -4.0 - 1j])
    assert np.allclose(O.sgd_direction(F, 4.0), [0.5 + 3j, -1.0 - 1j])

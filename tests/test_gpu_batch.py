"""Batched independent trainings (one CUDA-graph launch for several sessions
of different lattices and sizes; the FP32 sweeps of one entries-per-lane
class in one launch, the matrix-free CG systems of one precision in one
multi-system launch) and the launch-shape autotuner: both must leave every
session's trajectory bit-for-bit what its own epochs produce."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

PROBLEMS = [
    # (model, L, rbm_type, alpha, precision, chains, spc)
    ("toric", 3, 0, 2, 0, 32, 8),     # 702 parameters, tensor-core Gram
    ("toric", 4, 0, 2, 1, 16, 8),     # 2144 parameters: matrix-free CG (cooperative launch)
    ("toric", 4, 0, 2, 0, 24, 4),     # matrix-free, FP32 O: the three FP32 matrix-free
    ("kitaev", 3, 0, 1, 1, 16, 8),
    ("kitaev", 4, 1, 4, 0, 64, 4),
    ("toric", 4, 0, 2, 0, 16, 8),     # systems share one multi-system CG launch
    ("toric", 5, 0, 2, 0, 8, 8),      # 5150 parameters
]
# matrix-free CG systems merged into one launch (the FP64 one stays alone):
# each session's own epoch graph has two kernels for its solve (barrier
# reset, CG), the batch two for all three
MERGED = 3
# FP32 sweeps in the batch's sweep launches, one per entries-per-lane class:
# toric L = 3, 4, 4 (2 entries per lane) and the 32-spin symmetric Kitaev
# machine with toric L = 5 (4 entries per lane): five session sweeps, two
# launches
SWEPT, SWEEP_LAUNCHES = 5, 2


def make(spec, seed):
    model, L, rt, alpha, prec, chains, spc = spec
    gm = rbmnqs.Model.kitaev(L) if model == "kitaev" else rbmnqs.Model.toric(L, symmetry=1.0)
    cfg = rbmnqs.default_config(rbm_type=rt, alpha=alpha, n_chains=chains, samples_per_chain=spc, warmup=2,
                                seed=seed, precision=prec, bond_flips=0.5 if model == "kitaev" else 0.0,
                                max_iterations=60)
    s = rbmnqs.Session(gm, cfg)
    rng = np.random.default_rng(seed)
    s.set_weights(0.05 * (rng.normal(size=s.n_params) + 1j * rng.normal(size=s.n_params)))
    return s


def test_batch_epochs_equal_individual_epochs():
    a = [make(p, 100 + i) for i, p in enumerate(PROBLEMS)]
    b = [make(p, 100 + i) for i, p in enumerate(PROBLEMS)]
    batch = rbmnqs.Batch(a)
    for _ in range(3):
        sa, oa = batch.epoch()
        for i, s in enumerate(b):
            sb, ob = s.epoch()
            assert sa[i]["energy"] == sb["energy"] and oa[i]["iterations"] == ob["iterations"]
            assert oa[i]["status"] == 0
    for x, y in zip(a, b):
        assert np.array_equal(x.get_weights(), y.get_weights())
        assert np.array_equal(x.spins(), y.spins())
    assert batch.graph_kernels() == (sum(s.graph_kernels() for s in b) - 2 * (MERGED - 1) - SWEPT
                                     + SWEEP_LAUNCHES)


def test_autotune_keeps_the_trajectory():
    spec = ("kitaev", 4, 1, 4, 0, 256, 4)
    a, b = make(spec, 7), make(spec, 7)
    sw, ew, ms = a.autotune(sweeps=3)
    assert sw >= 1 and 1 <= ew <= 8 and ms > 0
    for _ in range(2):
        a.epoch()
        b.epoch()
    assert np.array_equal(a.get_weights(), b.get_weights())
    assert np.array_equal(a.spins(), b.spins())


def test_autotune_sr_keeps_S_within_tolerance():
    """The solver-stage autotuner (Gram split count, CG kernel) on the
    32-spin symmetric machine: the tuned tensor-core Gram still matches the
    oracle's S on the same samples at the FP32-path tolerance, and the
    session keeps training with the tuned choices."""
    spec = ("kitaev", 4, 1, 4, 0, 1024, 4)
    a = make(spec, 11)
    a.epoch()
    gs, kern, ms = a.autotune_sr()
    assert gs >= 1 and kern in (0, 1) and ms > 0
    a.sample()
    a.optimize()
    Eg, Og = a.samples()
    d, F, diag, S = a.sr_moments()
    So = O.sr_matrix(Og, O.sr_moments(Og, Eg)[0])
    assert np.linalg.norm(S - So) / np.linalg.norm(So) < 1e-5
    for _ in range(2):
        st, sr = a.epoch()
        assert sr["status"] == 0

"""Parity at the benchmark shapes.

* The mixed-precision SR epoch of the 32-spin Kitaev benchmark (4096 chains,
  symmetric RBM alpha=4, FP32 sweep, FP16x3 split-precision tensor-core Gram, cluster CG):
  the step dw = lr x of every epoch against the oracle's CG
  (cg_solver.cpp:260-334) on the GPU's own samples, FP32-path tolerance.
* The toric-code shapes of the batched benchmark at L = 5 and 8 (basic RBM
  alpha=2, 5150 and 33152 parameters): evaluation (E_loc, O_k), the FP32
  sweep against the oracle's chains (metropolis_sampler.cpp:118-273), and the
  matrix-free CG (cg_solver.cpp:301-318) in FP64 and inside the FP32 epoch.
* Statistics at benchmark scale: acceptance and energy of all chains against
  the oracle on a subsample of the same Philox streams, within error bars.
"""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-5


def relmax(a, b):
    """max |a - b| / max |b| (no floor: the steps are small numbers)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def kitaev32_session(std, seed=1234, chains=4096, spc=1, warmup=63, step=1):
    rng = np.random.default_rng(99)
    om = O.Model.kitaev(4)
    mach = O.Machine(om, "symmetry", 4, symm=0.5)
    P = mach.n_params
    w0 = rng.normal(0, std, P) + 1j * rng.normal(0, std, P)
    mach.set_params(w0)
    cfg = rbmnqs.default_config(rbm_type=1, alpha=4, n_chains=chains, samples_per_chain=spc, warmup=warmup,
                                step=step, bond_flips=0.5, seed=seed, precision=0, gram=0, reinit_chains=0,
                                reg2=(1e-4, 1e-4, 1.0))
    s = rbmnqs.Session(rbmnqs.Model.kitaev(4, symmetry=0.5), cfg)
    s.set_weights(w0)
    return om, mach, s


@pytest.mark.parametrize("std", [1e-4, 0.05])
def test_fp32_sr_epochs_at_kitaev32_bench_shape_match_oracle_cg(std):
    """Three captured epochs at the benchmark's shape: each epoch's step
    (weights before minus after) against lr x of the oracle's CG on that
    epoch's GPU samples, warm-started like the reference (x0 = lr x_prev),
    within 1e-5 of max |dw|."""
    om, mach, s = kitaev32_session(std)
    P = s.n_params
    x = np.zeros(P, np.complex128)
    errs = []
    for ep in range(3):
        w_before = s.get_weights()
        sst, ost = s.epoch()
        assert ost["status"] == 0
        E, Om = s.samples()
        d, F, diag = O.sr_moments(Om, E)
        x, it, rs = O.cg_solve(Om, d, F, x, ost["reg1"], ost["reg2"], ost["deltareg1"], diag)
        x = x * ost["lr"]
        dw_g = w_before - s.get_weights()
        err = relmax(dw_g, x)
        errs.append(err)
        assert err < TOL32, (ep, err)
        assert abs(ost["iterations"] - it) <= max(3, it // 10), (ep, ost["iterations"], it)
    print("dw relative error per epoch:", errs)


def toric_pair(L, precision, chains, spc, warmup, seed, std=0.05, **kw):
    rng = np.random.default_rng(L)
    om = O.Model.toric(L)
    mach = O.Machine(om, "basic", 2, symm=1.0).init_random(rng, std)
    cfg = rbmnqs.default_config(rbm_type=0, alpha=2, n_chains=chains, samples_per_chain=spc, warmup=warmup,
                                bond_flips=0.0, seed=seed, precision=precision, **kw)
    s = rbmnqs.Session(rbmnqs.Model.toric(L, symmetry=1.0), cfg)
    assert s.n_params == mach.n_params == 3 * 2 * L * L + 2 * (2 * L * L) ** 2
    s.set_weights(mach.params())
    return om, mach, s, rng


@pytest.mark.parametrize("L", [5, 8])
@pytest.mark.parametrize("precision,tol", [(1, TOL64), (0, TOL32)])
def test_toric_alpha2_eval_matches_oracle(L, precision, tol):
    """E_loc (L^2 four-spin star ratios) and O_k of the basic alpha=2 RBM on
    2 L^2 spins at given configurations."""
    om, mach, s, rng = toric_pair(L, precision, chains=8, spc=1, warmup=1, seed=3, std=0.1)
    spins = O.random_spins(rng, 24, mach.n)
    lg, eg, Og = s.eval_batch(spins)
    lo, eo, Oo = O.eval_batch(mach, om, spins)
    assert np.max(np.abs(eg - eo)) < tol * max(1.0, np.max(np.abs(eo)))
    assert np.max(np.abs(Og - Oo)) < tol * max(1.0, np.max(np.abs(Oo)))
    d = lg - lo
    assert np.max(np.abs(d.real)) < tol * max(1.0, np.max(np.abs(lo.real)))


@pytest.mark.parametrize("L", [5, 8])
def test_toric_alpha2_fp32_sweep_follows_oracle_chains(L):
    """The FP32 sweep (gathered flip rows; W from L2 at L = 8) against the
    FP64 oracle chains on the same Philox streams: the samples coincide
    except after acceptance ties; O_k and E_loc of the coinciding samples
    agree at the FP32 tolerance."""
    chains, spc, warm = 32, 6, 4
    om, mach, s, rng = toric_pair(L, 0, chains=chains, spc=spc, warmup=warm, seed=41)
    st = s.sample()
    Eg, Og = s.samples()
    Eo, Oo, acc, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=41)
    same = np.abs(Eg - Eo) < 1e-4 * np.maximum(1, np.abs(Eo))
    assert np.mean(same) > 0.9
    assert np.max(np.abs(Og[same] - Oo[same])) < TOL32 * max(1.0, np.max(np.abs(Oo)))
    assert abs(st["acceptance"] - acc.mean()) < 0.02


@pytest.mark.parametrize("L", [5, 8])
def test_toric_alpha2_matrix_free_solve_matches_oracle_cg(L):
    """The matrix-free FP64 CG (no S formed above 2048 parameters) against the
    oracle's CG on the same O store, both run to ||r||^2 < 1e-20 (a capped,
    unconverged CG amplifies summation-order differences from step to
    step, so only converged solves are compared)."""
    om, mach, s, rng = toric_pair(L, 1, chains=64, spc=2, warmup=3, seed=9, max_iterations=600, rtol=1e-20)
    s.sample()
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    P = mach.n_params
    x0 = 1e-3 * (rng.normal(size=P) + 1j * rng.normal(size=P))
    xo, ito, rso = O.cg_solve(Om, d, F, x0, 0.9, 9e-4, 1e-2, diag, max_iterations=600, rtol=1e-20)
    xg, itg, rsg = s.sr_solve(Om, d, F, x0, 0.9, 9e-4, 1e-2, diag)
    assert ito < 600 and rso < 1e-20 and rsg < 1e-20, (ito, rso, itg, rsg)
    assert abs(itg - ito) <= max(2, ito // 20)
    err = relmax(xg, xo)
    print(f"L={L} P={P} iterations {itg}/{ito}: max|dx|/max|x| = {err:.2e}")
    assert err < 1e-8


@pytest.mark.parametrize("L", [5, 8])
def test_toric_alpha2_fp32_epoch_step_matches_oracle_cg(L):
    """One captured FP32 epoch with the matrix-free CG (FP32 O store read as
    FP64): its step against lr x of the oracle's CG on the GPU's own samples,
    both converged to ||r||^2 < 1e-12."""
    om, mach, s, rng = toric_pair(L, 0, chains=64, spc=2, warmup=8, seed=13, max_iterations=400, rtol=1e-12,
                                  reinit_chains=0)
    w_before = s.get_weights()
    sst, ost = s.epoch()
    assert ost["status"] == 0
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    x, it, rs = O.cg_solve(Om, d, F, np.zeros(mach.n_params), ost["reg1"], ost["reg2"], ost["deltareg1"], diag,
                           max_iterations=400, rtol=1e-12)
    assert it < 400 and rs < 1e-12 and ost["residual"] < 1e-12, (it, rs, ost["iterations"], ost["residual"])
    dw_g = w_before - s.get_weights()
    err = relmax(dw_g, ost["lr"] * x)
    print(f"L={L} iterations {ost['iterations']}/{it}: max|d dw|/max|dw| = {err:.2e}")
    assert err < TOL32
    assert abs(ost["iterations"] - it) <= max(2, it // 20)


def test_kitaev32_bench_scale_statistics_agree_with_oracle_subsample():
    """All 4096 chains of the benchmark shape (16 samples per chain, 4 sweeps
    apart after 63 warm-up sweeps) against the oracle on the first 256 chains
    of the same Philox streams: acceptance and mean energy agree within error
    bars."""
    om, mach, s = kitaev32_session(0.05, chains=4096, spc=16, warmup=63, step=4)
    st = s.sample()
    Eg, _ = s.samples(with_O=False)
    sub = 256
    Eo, _, acc, _ = O.metropolis(mach, om, sub, 16, warmup=63, step=4, bond_flips=0.5, seed=1234, with_O=False)
    # chain-major samples: the first sub * 16 GPU samples are the oracle's chains
    same = np.abs(Eg[: sub * 16] - Eo) < 1e-4 * np.maximum(1, np.abs(Eo))
    assert np.mean(same) > 0.5
    ref = O.stats(Eo)
    err = np.hypot(st["stddev"], ref["stddev"])
    assert abs(st["energy"].real - ref["mean"].real) < 4 * err
    # acceptance per chain: binomial spread of the subsample's mean
    acc_err = np.std(acc) / np.sqrt(sub)
    assert abs(st["acceptance"] - acc.mean()) < 4 * acc_err + 1e-3


def test_kitaev128_bench_scale_statistics_agree_with_oracle_subsample():
    """The 128-spin benchmark lattice (symmetric alpha=4, 16384 chains, the
    gathered-row sweep) against the oracle on its first 96 chains."""
    rng = np.random.default_rng(5)
    om = O.Model.kitaev(8)
    mach = O.Machine(om, "symmetry", 4, symm=0.5).init_random(rng, 0.03)
    cfg = rbmnqs.default_config(rbm_type=1, alpha=4, n_chains=16384, samples_per_chain=8, warmup=16, step=2,
                                bond_flips=0.5, seed=777, precision=0, reinit_chains=1)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(8, symmetry=0.5), cfg)
    s.set_weights(mach.params())
    st = s.sample()
    Eg, _ = s.samples(with_O=False)
    sub = 96
    Eo, _, acc, _ = O.metropolis(mach, om, sub, 8, warmup=16, step=2, bond_flips=0.5, seed=777, with_O=False)
    same = np.abs(Eg[: sub * 8] - Eo) < 1e-4 * np.maximum(1, np.abs(Eo))
    assert np.mean(same) > 0.5
    ref = O.stats(Eo)
    err = np.hypot(st["stddev"], ref["stddev"])
    assert abs(st["energy"].real - ref["mean"].real) < 4 * err
    acc_err = np.std(acc) / np.sqrt(sub)
    assert abs(st["acceptance"] - acc.mean()) < 4 * acc_err + 1e-3

"""GPU parity of the RBM + Pfaffian machine (machine/pfaffian.cpp) against the
FP64 oracle on identical weights and configurations: log psi (modulo 2 pi i),
psi ratios, E_loc and O_k at 1e-10 (precision 1; the Pfaffian is FP64 in
both precisions, the RBM part FP32 at 1e-5 in precision 0), Metropolis
chains with the rank-2 X^{-1} updates and periodic refreshes reproduced
configuration for configuration, exact enumeration against the oracle and
exact diagonalisation."""
import numpy as np
import pytest

import ed
import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-5

CASES = {
    # name: (model, n_cells, rbm kind, alpha, Pfaffian symmetry)
    "kitaev2_basic_a1_pf0": ("kitaev", 2, "basic", 1, 0.0),
    "kitaev3_symm_a2_pf05": ("kitaev", 3, "symmetry", 2, 0.5),
    "kitaev4_symm_a2_pf05": ("kitaev", 4, "symmetry", 2, 0.5),
    "toric3_basic_a1_pf05": ("toric", 3, "basic", 1, 0.5),
}


def make_pair(case, precision=1, chains=8, spc=16, warmup=4, bond_flips=0.0, seed=123, std=0.1, std_pf=0.3,
              refresh=0, wseed=11, **cfgkw):
    model, L, kind, alpha, psym = CASES[case]
    rng = np.random.default_rng(wseed)
    symm = 0.5 if model == "kitaev" else 1.0
    om = O.Model.kitaev(L) if model == "kitaev" else O.Model.toric(L)
    mach = O.Machine(om, kind, alpha, symm=symm, pfaffian=True, pf_symm=psym)
    mach.init_random(rng, std, std_pf)
    gm = rbmnqs.Model.kitaev(L, symmetry=symm) if model == "kitaev" else rbmnqs.Model.toric(L, symmetry=symm)
    cfg = rbmnqs.default_config(rbm_type=1 if kind == "symmetry" else 0, alpha=alpha, n_chains=chains,
                                samples_per_chain=spc, warmup=warmup, bond_flips=bond_flips, seed=seed,
                                precision=precision, pfaffian=1, pfaffian_symmetry=psym, pfaffian_refresh=refresh,
                                **cfgkw)
    s = rbmnqs.Session(gm, cfg)
    assert s.n_params == mach.n_params
    s.set_weights(mach.params())
    return om, mach, s, rng


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


def logpsi_close(lg, lo, tol):
    d = lg - lo
    assert np.max(np.abs(d.real)) < tol * max(1.0, np.max(np.abs(lo.real)))
    assert np.max(np.abs(np.angle(np.exp(1j * d.imag)))) < tol * max(1.0, np.max(np.abs(lo.imag)))


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("precision,tol", [(1, TOL64), (0, TOL32)])
def test_pf_eval_batch_matches_oracle(case, precision, tol):
    om, mach, s, rng = make_pair(case, precision=precision, std=0.2)
    spins = O.random_spins(rng, 64, mach.n)
    lg, eg, Og = s.eval_batch(spins)
    lo, eo, Oo = O.eval_batch(mach, om, spins)
    logpsi_close(lg, lo, tol)
    assert rel(eg, eo) < tol
    assert rel(Og, Oo) < tol
    # the pair-parameter block is FP64 arithmetic in both precisions (stored
    # as FP32 in precision 0)
    P0 = mach.n_neural
    assert rel(Og[:, P0:], Oo[:, P0:]) < (TOL64 if precision == 1 else 1e-6)


@pytest.mark.parametrize("case", ["kitaev3_symm_a2_pf05", "kitaev4_symm_a2_pf05", "toric3_basic_a1_pf05"])
@pytest.mark.parametrize("nflip", [1, 2, 3, 4])
def test_pf_log_psi_over_psi_matches_oracle(case, nflip):
    om, mach, s, rng = make_pair(case, precision=1, std=0.2)
    B = 40
    spins = O.random_spins(rng, B, mach.n)
    flips = np.stack([rng.choice(mach.n, nflip, replace=False) for _ in range(B)]).astype(np.int32)
    rg = s.log_psi_over_psi(spins, flips)
    ro = np.array([O.log_psi_over_psi(mach, spins[b], flips[b]) for b in range(B)])
    assert rel(np.exp(rg), np.exp(ro)) < TOL64


@pytest.mark.parametrize("case,bond_flips,refresh", [
    ("kitaev2_basic_a1_pf0", 0.0, 0),
    ("kitaev3_symm_a2_pf05", 0.5, 4),
    ("kitaev4_symm_a2_pf05", 0.5, 32),
    ("kitaev4_symm_a2_pf05", 0.0, 0),
    ("toric3_basic_a1_pf05", 0.0, 8),
])
def test_pf_metropolis_fp64_reproduces_oracle_chains(case, bond_flips, refresh):
    """Rank-1/rank-2 X^{-1} updates between refreshes every `refresh`
    accepted moves (abstract_sampler.cpp:103-113): identical chains."""
    om, mach, s, rng = make_pair(case, precision=1, chains=8, spc=10, warmup=3, bond_flips=bond_flips,
                                 std=0.3, refresh=refresh)
    st = s.sample()
    Eg, Og = s.samples()
    Eo, Oo, acc, spo = O.metropolis(mach, om, 8, 10, warmup=3, bond_flips=bond_flips, seed=123, epoch=0,
                                    pf_refresh=refresh)
    assert np.array_equal(s.spins(), spo)
    assert rel(Eg, Eo) < TOL64
    assert rel(Og, Oo) < TOL64
    assert abs(st["acceptance"] - acc.mean()) < 1e-12


def test_pf_metropolis_fp32_statistics_agree():
    """Mixed precision (FP32 RBM ratios, FP64 Pfaffian): the chains follow
    the FP64 ones except after acceptance ties."""
    om, mach, s, rng = make_pair("kitaev3_symm_a2_pf05", precision=0, chains=32, spc=40, warmup=5,
                                 bond_flips=0.5, std=0.3, refresh=32)
    s.sample()
    Eg, _ = s.samples(with_O=False)
    Eo, _, _, _ = O.metropolis(mach, om, 32, 40, warmup=5, bond_flips=0.5, seed=123, pf_refresh=32,
                               with_O=False)
    same = np.mean(np.abs(Eg - Eo) < 1e-4 * np.maximum(1, np.abs(Eo)))
    assert same > 0.9


def test_pf_metropolis_fp64_at_bench_shape_reproduces_oracle_chains():
    """The 2048-chain shape of the 32-spin Pfaffian benchmark: 14 chains per
    block sharing the tables, X^{-1} in circulant form, the fresh inverse
    every 4 accepted moves in each warp's global scratch.  Every chain's
    configurations, E_loc and the acceptance match the FP64 oracle."""
    chains, spc, warm = 2048, 2, 3
    om, mach, s, rng = make_pair("kitaev4_symm_a2_pf05", precision=1, chains=chains, spc=spc, warmup=warm,
                                 bond_flips=0.5, std=0.1, refresh=4)
    st = s.sample()
    Eg, _ = s.samples(with_O=False)
    Eo, _, acc, spo = O.metropolis(mach, om, chains, spc, warmup=warm, bond_flips=0.5, seed=123, epoch=0,
                                   pf_refresh=4, with_O=False)
    assert np.array_equal(s.spins(), spo)
    assert rel(Eg, Eo) < TOL64
    assert abs(st["acceptance"] - acc.mean()) < 1e-12


def test_pf_metropolis_fp32_at_bench_shape_follows_oracle():
    """The benchmark's own path at its shape (FP32 RBM ratios, FP64 Pfaffian,
    2048 chains, refresh every 32 accepted moves): the samples follow the
    FP64 oracle's except after acceptance ties."""
    chains, spc, warm = 2048, 2, 3
    om, mach, s, rng = make_pair("kitaev4_symm_a2_pf05", precision=0, chains=chains, spc=spc, warmup=warm,
                                 bond_flips=0.5, std=0.1, refresh=32)
    s.sample()
    Eg, _ = s.samples(with_O=False)
    Eo, _, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, bond_flips=0.5, seed=123, epoch=0,
                               pf_refresh=32, with_O=False)
    same = np.mean(np.abs(Eg - Eo) < 1e-4 * np.maximum(1, np.abs(Eo)))
    assert same > 0.9


@pytest.mark.parametrize("case", ["kitaev2_basic_a1_pf0", "kitaev3_symm_a2_pf05"])
def test_pf_full_enumeration_matches_oracle_and_ed(case):
    om, mach, s, rng = make_pair(case, precision=1, std=0.3)
    Eg, dg, dhg = s.full_sample()
    ref = O.full(mach, om)
    assert abs(Eg - ref["E"]) < 1e-8 * abs(ref["E"])
    assert rel(dg, ref["d"]) < 1e-8
    assert rel(dhg, ref["dh"]) < 1e-8
    H = ed.hamiltonian(om)
    N = 1 << mach.n
    bits = ((np.arange(N)[:, None] >> np.arange(mach.n)[None, :]) & 1)
    lp, _, _ = s.eval_batch(O.spins_from_bits(bits), eloc=False, O=False)
    psi = np.exp(lp - lp.real.max())
    e = np.vdot(psi, H @ psi) / np.vdot(psi, psi)
    assert abs(Eg - e) < 1e-8 * abs(e)


def test_pf_sr_epochs_match_oracle():
    """Two SR epochs of the RBM + Pfaffian machine (FP64) against the oracle
    driving the reference loop: the pair parameters are updated with the rest."""
    chains, spc, warm = 8, 16, 3
    om, mach, s, rng = make_pair("kitaev3_symm_a2_pf05", precision=1, chains=chains, spc=spc, warmup=warm,
                                 std=0.05, std_pf=0.3, refresh=8)
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    x = np.zeros(mach.n_params, np.complex128)
    for ep in range(2):
        sst, ost = s.epoch()
        E, Om, acc, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=123, epoch=ep, pf_refresh=8)
        d, F, diag = O.sr_moments(Om, E)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        x, it, rs = O.cg_solve(Om, d, F, x, r1v, r2v, rdv, diag, n_neural=mach.n_neural)
        assert abs(ost["iterations"] - it) <= 1
        x = x * lrv
        mach.set_params(mach.params() - x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep

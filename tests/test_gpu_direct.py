"""GPU parity of the direct SR solver (optimizer.sr.method = direct,
optimizer/direct_solver.cpp:31-59): the multiplicative diagonal
regularisation and the exact solve (blocked Cholesky on the GPU, minimum-norm
least squares in the oracle) on the same O, d, F, and FP64 training epochs
against the oracle driving the reference loop; above 2048 parameters the
solve runs in sample space (the N x N system of the Woodbury identity)."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


def session(model, L, kind, alpha, chains=16, spc=12, **kw):
    rng = np.random.default_rng(8)
    om = O.Model.kitaev(L) if model == "kitaev" else O.Model.toric(L)
    symm = 0.5 if model == "kitaev" else 1.0
    mach = O.Machine(om, "symmetry" if kind else "basic", alpha, symm=symm).init_random(rng, 0.05)
    gm = rbmnqs.Model.kitaev(L, symmetry=symm) if model == "kitaev" else rbmnqs.Model.toric(L, symmetry=symm)
    cfg = rbmnqs.default_config(rbm_type=kind, alpha=alpha, n_chains=chains, samples_per_chain=spc, warmup=3,
                                seed=9, precision=1, solver=2, bond_flips=0.0, **kw)
    s = rbmnqs.Session(gm, cfg)
    s.set_weights(mach.params())
    return om, mach, s


@pytest.mark.parametrize("model,L,kind,alpha", [
    ("kitaev", 2, 1, 4),     # 20 parameters: one partial panel
    ("kitaev", 3, 0, 1),     # 360
    ("toric", 3, 0, 2),      # 702
    ("kitaev", 4, 0, 1),     # 1088: 34 panels, trailing updates over many blocks
])
def test_direct_solve_matches_oracle(model, L, kind, alpha):
    om, mach, s = session(model, L, kind, alpha)
    s.sample()
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    r1, r2, rd = 0.9, 9e-4, 1e-2
    xo = O.direct_solve(Om, d, F, r1, r2, rd, diag)
    xg, itg, _ = s.sr_solve(Om, d, F, np.zeros(mach.n_params), r1, r2, rd, diag)
    assert itg == 0
    assert rel(xg, xo) < 1e-9
    # and it solves the regularised system itself
    P = mach.n_params
    S = Om.conj().T @ Om / len(E) - np.outer(np.conj(d), d)
    S[np.arange(P), np.arange(P)] *= 1 + r1
    S[np.arange(P), np.arange(P)] += r2 * np.max(np.abs(diag))
    assert np.linalg.norm(S @ xg - F) < 1e-9 * max(1.0, np.linalg.norm(F))


def test_direct_sr_epochs_match_oracle():
    chains, spc, warm = 8, 24, 3
    om, mach, s = session("kitaev", 3, 0, 1, chains=chains, spc=spc)
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    for ep in range(3):
        _, ost = s.epoch()
        E, Om, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=9, epoch=ep)
        d, F, diag = O.sr_moments(Om, E)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        x = O.direct_solve(Om, d, F, r1v, r2v, rdv, diag)
        assert ost["status"] == 0 and ost["iterations"] == 0
        mach.set_params(mach.params() - lrv * x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep


def test_sample_space_direct_solve_matches_oracle():
    """2144 parameters (S not formed), 192 samples: the direct solve through
    the N x N system of the Woodbury identity against the oracle's
    minimum-norm least-squares solve of the P x P system."""
    om, mach, s = session("toric", 4, 0, 2)
    assert s.n_params == 2144
    s.sample()
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    r1, r2, rd = 0.9, 9e-4, 1e-2
    xo = O.direct_solve(Om, d, F, r1, r2, rd, diag)
    xg, itg, _ = s.sr_solve(Om, d, F, np.zeros(mach.n_params), r1, r2, rd, diag)
    assert itg == 0
    assert rel(xg, xo) < 1e-9
    P = mach.n_params
    S = Om.conj().T @ Om / len(E) - np.outer(np.conj(d), d)
    S[np.arange(P), np.arange(P)] *= 1 + r1
    S[np.arange(P), np.arange(P)] += r2 * np.max(np.abs(diag))
    assert np.linalg.norm(S @ xg - F) < 1e-9 * max(1.0, np.linalg.norm(F))


def test_sample_space_direct_epochs_match_oracle():
    """Two FP64 epochs of the 2144-parameter toric machine with the direct
    solver inside the captured epoch (schedules and var(O) on the device)
    against the oracle driving the reference loop."""
    chains, spc, warm = 8, 16, 3
    om, mach, s = session("toric", 4, 0, 2, chains=chains, spc=spc)
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    for ep in range(2):
        _, ost = s.epoch()
        E, Om, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=9, epoch=ep)
        d, F, diag = O.sr_moments(Om, E)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        x = O.direct_solve(Om, d, F, r1v, r2v, rdv, diag)
        assert ost["status"] == 0 and ost["iterations"] == 0
        mach.set_params(mach.params() - lrv * x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep


def test_direct_solver_rejects_too_many_samples_above_the_formed_sizes():
    gm = rbmnqs.Model.toric(4)
    cfg = rbmnqs.default_config(rbm_type=0, alpha=2, n_chains=512, samples_per_chain=16, precision=1, solver=2)
    with pytest.raises(rbmnqs.RbmNqsError, match="sample space"):
        rbmnqs.Session(gm, cfg)

"""Learned multi-spin proposals (proposal network + exact Metropolis-Hastings
acceptance): the stationary distribution is unchanged, so energies agree
with exact enumeration within error bars; the trained network lowers the
autocorrelation time of E_loc compared with plain single-flip Metropolis
at the same sweeps per sample."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def session(L, kind, alpha, std, proposal, chains, spc, step, warmup, seed=5, bond_flips=0.0, **kw):
    rng = np.random.default_rng(seed)
    om = O.Model.kitaev(L)
    mach = O.Machine(om, kind, alpha, symm=0.5).init_random(rng, std)
    gm = rbmnqs.Model.kitaev(L)
    cfg = rbmnqs.default_config(rbm_type=1 if kind == "symmetry" else 0, alpha=alpha, n_chains=chains,
                                samples_per_chain=spc, step=step, warmup=warmup, seed=seed, precision=0,
                                bond_flips=bond_flips, proposal=proposal, reinit_chains=0, **kw)
    s = rbmnqs.Session(gm, cfg)
    s.set_weights(mach.params())
    return s, mach, om


def test_learned_chains_sample_psi_squared():
    """Energies from learned-proposal chains (several epochs, weights fixed)
    against exact enumeration of the same 18-spin wavefunction."""
    s, mach, om = session(3, "basic", 1, 0.3, 1, chains=512, spc=16, step=1, warmup=10, learned_steps=2,
                          learned_train=2, learned_lr=3e-3)
    ex = O.full(mach, om, with_O=False)["E"].real
    es, errs, accs = [], [], []
    for _ in range(6):
        st = s.sample()
        es.append(st["energy"].real)
        errs.append(st["stddev"])
        accs.append(st["learned_acceptance"])
    E = np.mean(es[1:])
    err = np.sqrt(np.sum(np.square(errs[1:]))) / len(errs[1:])
    assert abs(E - ex) < 4 * err + 1e-6, (E, ex, err)
    assert min(accs) > 0.0


def lag1(E, chains, spc):
    """mean over chains of the lag-1 autocorrelation of E_loc along the chain"""
    x = np.asarray(E).real.reshape(chains, spc)
    x = x - x.mean(axis=1, keepdims=True)
    num = np.sum(x[:, 1:] * x[:, :-1], axis=1)
    den = np.sum(x * x, axis=1) + 1e-300
    return float(np.mean(num / den))


def test_learned_proposals_lower_autocorrelation():
    """Same lattice, weights and sweeps per sample (one sweep between
    samples): the learned form decorrelates faster (smaller lag-1
    autocorrelation of E_loc along the chains)."""
    chains, spc = 256, 64
    kw = dict(chains=chains, spc=spc, step=1, warmup=8)
    plain, _, _ = session(4, "symmetry", 2, 0.05, 0, **kw)
    learned, _, _ = session(4, "symmetry", 2, 0.05, 1, learned_steps=1, learned_train=4, learned_lr=3e-3, **kw)
    rp, rl, acc = [], [], []
    for ep in range(4):
        a = plain.sample()
        b = learned.sample()
        if ep > 0:  # after the first training
            rp.append(lag1(plain.samples(with_O=False)[0], chains, spc))
            rl.append(lag1(learned.samples(with_O=False)[0], chains, spc))
            acc.append(b["learned_acceptance"])
    assert np.mean(acc) > 0.3
    assert np.mean(rl) < 0.8 * np.mean(rp), (rl, rp)
    # both sample the same distribution
    ea, eb = a["energy"].real, b["energy"].real
    assert abs(ea - eb) < 5 * np.hypot(a["stddev"], b["stddev"]) + 1e-6

"""Learned proposals (dictionary moves drawn from the proposal network, exact
Metropolis-Hastings acceptance).

* Exactness: chains moved by learned moves alone sample |psi|^2 -- the
  energy agrees with exact enumeration within error bars and the visited
  configurations follow |psi|^2 over all 2^8 states of a small lattice.
* Gain: on a correlated state (a toric-code closed-loop state: plaquette
  hidden units W = 0.05 + i pi/4 suppress configurations that break a
  plaquette, as in the toric-code ground state) single-spin Metropolis
  accepts about 0.1 % of its proposals; the trained network learns to
  propose star moves (acceptance about 0.9 against about 0.35 untrained),
  learned moves added to the sweeps lower the binned autocorrelation time
  of E_loc, and the energy still matches exact enumeration.
* The 32-spin Kitaev machine runs with learned moves and agrees with plain
  Metropolis.
"""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def kitaev_session(L, kind, alpha, std, proposal, chains, spc, step, warmup, seed=5, bond_flips=0.0, **kw):
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


def test_learned_moves_alone_sample_psi_squared():
    """Only learned moves (no sweeps) on the 18-spin Kitaev lattice: energy
    against exact enumeration of the same wavefunction."""
    s, mach, om = kitaev_session(3, "basic", 1, 0.1, 1, chains=1024, spc=16, step=0, warmup=0, learned_steps=8,
                                 learned_train=2, learned_lr=3e-3)
    ex = O.full(mach, om, with_O=False)["E"].real
    es, errs, accs = [], [], []
    for ep in range(8):
        st = s.sample()
        if ep >= 2:  # after burn-in
            es.append(st["energy"].real)
            errs.append(st["stddev"])
            accs.append(st["learned_acceptance"])
    E = np.mean(es)
    err = np.sqrt(np.sum(np.square(errs))) / len(errs)
    assert abs(E - ex) < 4 * err + 1e-6, (E, ex, err)
    assert min(accs) > 0.1


def test_learned_chains_follow_psi_squared_over_all_states():
    """2^8 states of the 8-spin Kitaev lattice: the histogram of the
    configurations visited by learned moves alone against |psi|^2."""
    s, mach, om = kitaev_session(2, "basic", 2, 0.15, 1, chains=2048, spc=32, step=0, warmup=0, learned_steps=2,
                                 learned_train=2, learned_lr=3e-3)
    n = 8
    states = np.arange(1 << n)
    bits = ((states[:, None] >> np.arange(n)[None, :]) & 1)
    lp, _, _ = s.eval_batch(O.spins_from_bits(bits), eloc=False, O=False)
    p = np.exp(2 * (lp.real - lp.real.max()))
    p /= p.sum()
    counts = np.zeros(1 << n)
    for ep in range(6):
        s.sample()
        if ep >= 2:
            conf = s.sample_configs()[:, 0]
            counts += np.bincount(conf, minlength=1 << n)
    q = counts / counts.sum()
    tv = 0.5 * np.abs(p - q).sum()
    assert tv < 0.04, tv


def toric_loop_gas(L, eps=0.05):
    """Basic RBM (alpha 1) on the L x L toric code whose first L^2 hidden units
    sit on the plaquettes with W = eps + i pi / 4: |cosh|^2 is sinh^2(2 eps)
    for a violated plaquette (odd number of down spins) and about 1
    otherwise, so |psi|^2 is concentrated on the plaquette-satisfying
    (closed-loop) configurations, as in the toric-code ground state."""
    gm = rbmnqs.Model.toric(L, symmetry=1.0)
    n = gm.n
    plaqs = []
    for o in range(gm.n_ops):
        k, acts, mat = gm.op(o)
        if k == 4 and np.allclose(mat, np.diag(np.diag(mat))):
            plaqs.append(acts)
    assert len(plaqs) == L * L
    M = n
    W = np.zeros((n, M), np.complex128)
    for p, acts in enumerate(plaqs):
        for i in acts:
            W[i, p] = eps + 1j * np.pi / 4
    w = np.concatenate([np.zeros(n), np.zeros(M), W.ravel(order="F")])
    return gm, w


def test_learned_star_moves_lower_tau_on_a_closed_loop_state():
    """Closed-loop state of the 18-spin toric code: a single flip breaks two
    plaquettes (|psi'/psi|^2 about 1e-4), so single-flip Metropolis
    accepts about 0.1 % of its proposals.  The network, trained on
    |psi'/psi|^2 of every dictionary move, learns to propose stars
    (sigma^x on the four bonds of a vertex, which keep every plaquette):
    its acceptance rises from that of the untrained network (about a third
    of the dictionary are stars) to about 0.9.  With six learned moves added
    to each sweep, the binned autocorrelation time of E_loc (the
    reference's estimator) falls below two thirds of the plain chains'
    from the same starting configurations, and the energy matches exact
    enumeration."""
    L = 3
    gm, w = toric_loop_gas(L)
    om = O.Model.toric(L)
    mach = O.Machine(om, "basic", 1, symm=1.0)
    mach.set_params(w)
    ex = O.full(mach, om, with_O=False)["E"].real
    chains, spc = 256, 64
    common = dict(rbm_type=0, alpha=1, n_chains=chains, samples_per_chain=spc, warmup=0, seed=9, precision=0,
                  bond_flips=0.0, reinit_chains=0, step=1)
    plain = rbmnqs.Session(gm, rbmnqs.default_config(proposal=0, **common))
    learned = rbmnqs.Session(gm, rbmnqs.default_config(proposal=1, learned_steps=6, learned_train=4,
                                                       learned_lr=3e-3, **common))
    untrained = rbmnqs.Session(gm, rbmnqs.default_config(proposal=1, learned_steps=6, learned_train=0, **common))
    for s in (plain, learned, untrained):
        s.set_weights(w)
    for _ in range(3):  # plain sweeps remove the broken plaquettes of the random start
        plain.sample()
    for s in (learned, untrained):
        s.sample()  # first epoch: fresh chains, replaced by the plain chains' configurations
        s.set_spins(plain.spins())
    tp, tl, el, errs, lacc, uacc = [], [], [], [], [], []
    for ep in range(8):
        a = plain.sample()
        b = learned.sample()
        c = untrained.sample()
        if ep >= 2:  # after the network's first trainings
            tp.append(a["tau"])
            tl.append(b["tau"])
            el.append(b["energy"].real)
            errs.append(b["stddev"])
            lacc.append(b["learned_acceptance"])
            uacc.append(c["learned_acceptance"])
    assert np.mean(lacc) > 0.7 and np.mean(lacc) > np.mean(uacc) + 0.3, (lacc, uacc)
    assert np.mean(tl) < np.mean(tp) / 1.5, (tl, tp)
    E = np.mean(el)
    err = np.sqrt(np.sum(np.square(errs))) / len(errs)
    assert abs(E - ex) < 5 * err + 1e-4 * abs(ex), (E, ex, err)


def test_learned_moves_on_the_32_spin_kitaev_machine_agree_with_plain():
    kw = dict(chains=1024, spc=8, step=1, warmup=4)
    plain, _, _ = kitaev_session(4, "symmetry", 4, 0.05, 0, bond_flips=0.5, **kw)
    learned, _, _ = kitaev_session(4, "symmetry", 4, 0.05, 1, bond_flips=0.5, learned_steps=2, learned_train=2,
                                   learned_lr=3e-3, **kw)
    ea, eb, sa, sb, acc = [], [], [], [], []
    for ep in range(5):
        a = plain.sample()
        b = learned.sample()
        if ep >= 1:
            ea.append(a["energy"].real)
            eb.append(b["energy"].real)
            sa.append(a["stddev"])
            sb.append(b["stddev"])
            acc.append(b["learned_acceptance"])
    err = np.hypot(np.sqrt(np.sum(np.square(sa))), np.sqrt(np.sum(np.square(sb)))) / len(sa)
    assert abs(np.mean(ea) - np.mean(eb)) < 5 * err + 1e-6
    assert np.mean(acc) > 0.05

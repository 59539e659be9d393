"""GPU parity of the update rules around the solve: the Adam, momentum and
Heun plugins (optimizer/plugin.cpp:29-115) on SR and on plain gradient
descent (optimizer/gradient_descent.cpp:42-60), three FP64 epochs each
against the oracle driving the reference loop (abstract_optimizer.cpp:
150-177)."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def make_pair(L=3, kind="basic", alpha=1, chains=8, spc=24, warmup=4, seed=123, std=0.05, **cfgkw):
    rng = np.random.default_rng(7)
    om = O.Model.kitaev(L)
    mach = O.Machine(om, kind, alpha, symm=0.5)
    mach.init_random(rng, std)
    cfg = rbmnqs.default_config(rbm_type=1 if kind == "symmetry" else 0, alpha=alpha, n_chains=chains,
                                samples_per_chain=spc, warmup=warmup, seed=seed, precision=1, reinit_chains=1, bond_flips=0.0,
                                **cfgkw)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(L, symmetry=0.5), cfg)
    s.set_weights(mach.params())
    return om, mach, s


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


PLUGINS = {
    "none": (0, {}, lambda P: None),
    "adam": (1, dict(adam_beta1=0.8, adam_beta2=0.99, adam_eps=1e-6),
             lambda P: O.AdamPlugin(P, 0.8, 0.99, 1e-6)),
    "momentum": (2, dict(mom_alpha=0.7), lambda P: O.MomentumPlugin(P, 0.7)),
    "momentum_dialup": (2, dict(mom_alpha=0.9, mom_dialup=20.0), lambda P: O.MomentumPlugin(P, 0.9, 20.0)),
}


def run_epochs(optimizer_type, plugin, kind="basic", alpha=1, epochs=3, real_factor=1.0):
    code, kw, mk = PLUGINS[plugin]
    chains, spc, warm = 8, 24, 4
    om, mach, s = make_pair(kind=kind, alpha=alpha, chains=chains, spc=spc, warmup=warm,
                            optimizer_type=optimizer_type, plugin=code, sgd_real_factor=real_factor, **kw)
    plug = mk(mach.n_params)
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    x = np.zeros(mach.n_params, np.complex128)
    for ep in range(epochs):
        _, ost = s.epoch()
        E, Om, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=123, epoch=ep)
        d, F, diag = O.sr_moments(Om, E)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        if optimizer_type == 1:
            x = O.sgd_direction(F, real_factor)
            assert ost["iterations"] == 0
        else:
            x, it, _ = O.cg_solve(Om, d, F, x, r1v, r2v, rdv, diag)
            assert abs(ost["iterations"] - it) <= 1
        x = O.optimize_tail(x, lrv, plug)
        assert x is not None and ost["status"] == 0
        mach.set_params(mach.params() - x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep
    return s, mach


@pytest.mark.parametrize("plugin", ["adam", "momentum", "momentum_dialup"])
def test_sr_with_plugin_matches_oracle(plugin):
    run_epochs(0, plugin)


@pytest.mark.parametrize("plugin", ["none", "adam", "momentum"])
def test_sgd_matches_oracle(plugin):
    run_epochs(1, plugin)


def test_sgd_real_factor_and_symmetric_machine():
    run_epochs(1, "none", kind="symmetry", alpha=2, real_factor=4.0)


@pytest.mark.parametrize("optimizer_type", [0, 1])
def test_heun_matches_oracle(optimizer_type):
    """Heun: SR (or SGD) step x1, half step (lr/2) x1, a second sample and
    gradient (the regularisers decay again), then x2 (cbrt(eps/err) - 1/2) lr
    with err from the metric O of the second sample (SR) or |delta| (SGD)."""
    chains, spc, warm = 8, 24, 4
    om, mach, s = make_pair(chains=chains, spc=spc, warmup=warm, optimizer_type=optimizer_type, plugin=3,
                            heun_eps=1e-3)
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    x = np.zeros(mach.n_params, np.complex128)
    for ep in range(3):
        sst, ost = s.epoch()
        E, Om, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=123, epoch=2 * ep)
        # the reported sample statistics are the first sample's
        assert abs(sst["energy"] - E.mean()) < 1e-10 * abs(E.mean())
        d, F, diag = O.sr_moments(Om, E)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        x1 = O.sgd_direction(F) if optimizer_type else O.cg_solve(Om, d, F, x, r1v, r2v, rdv, diag)[0]
        assert np.max(np.abs(x1)) <= 30
        delta = O.heun_begin(x1, lrv)
        mach.set_params(mach.params() - delta)
        E, Om, _, _ = O.metropolis(mach, om, chains, spc, warmup=warm, seed=123, epoch=2 * ep + 1)
        d, F, diag = O.sr_moments(Om, E)
        if optimizer_type == 0:
            r1v, r2v, rdv = r1.get(), r2.get(), rd.get()
            x2, it, _ = O.cg_solve(Om, d, F, x1, r1v, r2v, rdv, diag)
            assert abs(ost["iterations"] - it) <= 1
            x = O.heun_finish(delta, x2, lrv, 1e-3, Om, d)
        else:
            x = O.heun_finish(delta, O.sgd_direction(F), lrv, 1e-3)
        assert ost["status"] == 0
        mach.set_params(mach.params() - x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep
    assert s.n_updates() == 3


def test_adam_step_is_lr_times_sign_on_first_epoch():
    """Adam's first bias-corrected step is lr * dw / (|dw| + eps) per real
    and imaginary part: every parameter moves by about lr."""
    om, mach, s = make_pair(optimizer_type=1, plugin=1, adam_eps=1e-12)
    w0 = s.get_weights()
    s.epoch()
    dw = w0 - s.get_weights()
    big = np.abs(dw.real) > 1e-6
    assert big.mean() > 0.9
    assert np.allclose(np.abs(dw.real[big]), 1e-2, rtol=1e-6)

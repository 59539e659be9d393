"""GPU parity of the full-enumeration sampler (sampler.type = full,
full_sampler.cpp:43-186) inside the epoch: the state order, per-state E_loc
and O_k, the |psi|^2-weighted aggregators (aggregator.cpp:190-239) and the
weighted SR system, against the oracle on the same weights; SR epochs
against the oracle driving the reference loop; the state vector against
exact diagonalisation."""
import numpy as np
import pytest

import ed
import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b)))


def make(model="kitaev", L=2, Lb=-1, kind=0, alpha=1, precision=1, bits=2, std=0.3, pf=False, **kw):
    rng = np.random.default_rng(5)
    if model == "kitaev":
        om, gm = O.Model.kitaev(L, Lb), rbmnqs.Model.kitaev(L, Lb)
    else:
        om, gm = O.Model.toric(L), rbmnqs.Model.toric(L)
    symm = 0.5 if model == "kitaev" else 1.0
    mach = O.Machine(om, "symmetry" if kind else "basic", alpha, symm=symm, pfaffian=pf, pf_symm=0.5)
    if pf:
        mach.init_random(rng, std, 0.3)
    else:
        mach.init_random(rng, std)
    cfg = rbmnqs.default_config(rbm_type=kind, alpha=alpha, precision=precision, sampler_type=1,
                                full_parallel_bits=bits, pfaffian=int(pf), pfaffian_symmetry=0.5, **kw)
    s = rbmnqs.Session(gm, cfg)
    s.set_weights(mach.params())
    return om, mach, s


def oracle_states(mach, om, bits):
    nums = O.full_order(mach.n, bits)
    bits_ = (nums[:, None] >> np.arange(mach.n)[None, :]) & 1
    spins = O.spins_from_bits(bits_)
    lp, E, Om = O.eval_batch(mach, om, spins)
    p = np.exp(2 * lp.real - np.max(2 * lp.real))
    return nums, spins, lp, E, Om, p


def weighted_sr(E, Om, p):
    W, W2 = p.sum(), (p * p).sum()
    d = (p[:, None] * Om).sum(0) / W
    em = (p * E).sum() / W
    F = (p[:, None] * E[:, None] * Om.conj()).sum(0) / W - em * d.conj()
    X = Om - d
    S = (p[:, None] * X).T.conj() @ X / W
    diag = (p[:, None] * np.abs(X) ** 2).sum(0) / (W - W2 / W)
    return em, d, F, S, diag


@pytest.mark.parametrize("case", [
    dict(model="kitaev", L=2, kind=0, alpha=1, bits=2),
    dict(model="kitaev", L=2, kind=1, alpha=3, bits=0),
    dict(model="toric", L=2, kind=0, alpha=2, bits=3),
    dict(model="kitaev", L=2, kind=0, alpha=1, bits=1, pf=True),
])
def test_full_sample_matches_oracle(case):
    om, mach, s = make(**case)
    st = s.sample()
    so = s.optimize()
    nums, spins, lp, Eo, Oo, p = oracle_states(mach, om, case["bits"])
    assert np.array_equal(s.sample_configs(), spins)
    Eg, Og = s.samples()
    assert rel(Eg, Eo) < TOL64
    em, d, F, S, diag = weighted_sr(Eo, Oo, p)
    dg, Fg, diagg, Sg = s.sr_moments(with_S=True)
    assert rel(dg, d) < TOL64 and rel(Fg, F) < TOL64
    assert rel(diagg, diag) < TOL64
    assert rel(Sg, S) < TOL64
    ref = O.weighted_aggregate(Eo, p, st["n_bins"])
    assert abs(st["energy"] - ref["mean"]) < TOL64 * max(1, abs(ref["mean"]))
    assert abs(st["var"] - ref["var"]) < 1e-9 * max(1e-12, ref["var"])
    assert abs(st["stddev"] - ref["stddev"]) < 1e-8 * max(1e-12, ref["stddev"])
    assert abs(st["tau"] - ref["tau"]) < 1e-8 * max(1, ref["tau"])
    # the exact expectation of the Hamiltonian
    assert abs(st["energy"] - O.full(mach, om)["E"]) < 1e-10 * abs(st["energy"])
    assert so["status"] == 0


@pytest.mark.parametrize("case", [
    dict(model="kitaev", L=2, kind=0, alpha=2, bits=2),
    dict(model="kitaev", L=2, kind=1, alpha=2, bits=2, solver=2),
    dict(model="kitaev", L=2, Lb=3, kind=0, alpha=14, bits=2),   # 2196 parameters: matrix-free CG
])
def test_full_sr_epochs_match_oracle(case):
    om, mach, s = make(std=0.05, **case)
    bits = case["bits"]
    lr, r1, r2, rd = O.Decay(1e-2), O.Decay(1, 1e-4, 0.9), O.Decay(1e-3, 1e-6, 0.9), O.Decay(1e-2)
    x = np.zeros(mach.n_params, np.complex128)
    for ep in range(3):
        _, ost = s.epoch()
        _, _, _, Eo, Oo, p = oracle_states(mach, om, bits)
        em, d, F, S, diag = weighted_sr(Eo, Oo, p)
        lrv, r1v, r2v, rdv = lr.get(), r1.get(), r2.get(), rd.get()
        if case.get("solver") == 2:
            x = O.direct_solve(np.sqrt(p)[:, None] * Oo, d, F, r1v, r2v, rdv, diag, norm=p.sum())
        else:
            # the reference's sqrt(p) O store with norm sum p
            x, it, _ = O.cg_solve(np.sqrt(p)[:, None] * Oo, d, F, x, r1v, r2v, rdv, diag, norm=p.sum())
            assert abs(ost["iterations"] - it) <= max(2, it // 20)
        assert ost["status"] == 0
        x = x * lrv
        mach.set_params(mach.params() - x)
        assert rel(s.get_weights(), mach.params()) < 1e-9, ep


def test_full_state_vector_matches_eval_and_ed():
    om, mach, s = make(model="kitaev", L=2, kind=1, alpha=2, bits=2)
    st = s.sample()
    psi = s.full_state()
    n = mach.n
    allbits = (np.arange(1 << n)[:, None] >> np.arange(n)[None, :]) & 1
    lp, _, _ = O.eval_batch(mach, om, O.spins_from_bits(allbits), with_O=False)
    ref = np.exp(lp - lp.real.max())
    ref /= np.linalg.norm(ref)
    assert rel(psi, ref) < TOL64
    assert abs(np.linalg.norm(psi) - 1) < 1e-12
    H = ed.hamiltonian(om)
    e = np.vdot(psi, H @ psi)
    assert abs(st["energy"] - e) < 1e-8 * abs(e)


def test_full_fp32_tracks_fp64():
    """Mixed precision (FP32 ratios, FP16x3 split-precision tensor-core Gram) on the full
    sampler follows the FP64 training within the FP32 tolerance."""
    _, _, a = make(model="kitaev", L=2, kind=1, alpha=2, precision=0, std=0.05)
    _, _, b = make(model="kitaev", L=2, kind=1, alpha=2, precision=1, std=0.05)
    for _ in range(2):
        sa, _ = a.epoch()
        sb, _ = b.epoch()
        assert abs(sa["energy"] - sb["energy"]) < 1e-5 * abs(sb["energy"])
    assert rel(a.get_weights(), b.get_weights()) < 1e-5


def test_full_observables_are_weighted():
    """Evaluation mode on the full sampler: <W_p> per hexagon weighted by
    |psi|^2 over all states, with the weighted aggregator statistics."""
    rng = np.random.default_rng(3)
    om = O.Model.kitaev(2)
    mach = O.Machine(om, "basic", 1, symm=0.5).init_random(rng, 0.3)
    gm = rbmnqs.Model.kitaev(2)
    gm.add_hexagons()
    s = rbmnqs.Session(gm, rbmnqs.default_config(rbm_type=0, alpha=1, precision=1, sampler_type=1))
    s.set_weights(mach.params())
    st = s.sample()
    vals = s.observables()
    _, spins, _, _, _, p = oracle_states(mach, om, 2)
    hx = O.Model.hexagons(2)
    assert vals.shape == (hx.n_ops, 4)
    for o in range(hx.n_ops):
        one = O.Model(hx.n, hx.k[o:o + 1], hx.sites[o:o + 1], np.array([0], np.int32),
                      hx.mats[2 * hx.mat_off[o]: 2 * (hx.mat_off[o] + 64 * 64)])
        _, lo, _ = O.eval_batch(mach, one, spins, with_O=False)
        ref = O.weighted_aggregate(lo, p, st["n_bins"])
        assert abs(vals[o, 0] + 1j * vals[o, 1] - ref["mean"]) < TOL64
        assert abs(vals[o, 2] - ref["stddev"]) < 1e-8 * max(1e-12, ref["stddev"])

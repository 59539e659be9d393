"""Failure detection without a GPU fault.

The reference's failure handling is the max|dw| > 30 guard of the
optimizer (abstract_optimizer.cpp:157-159) and exceptions that end the run
(main.cpp:610-615).  Here every such condition comes back as a status code:

* non-finite weights: the epoch reports RBMNQS_ERR_NONFINITE and the
  update is not applied;
* a step with max|dw| > 30: RBMNQS_ERR_MASSIVE_STEP, weights unchanged;
* a CG that hits its iteration cap: the residual and the iteration count
  are reported, the step is applied as the reference does;
* bounded device waits that run out (test hook rbmnqs_test_fault): the
  cooperative solvers' grid barriers and the proposal network's TMA wait give
  up after a short limit and the call reports RBMNQS_ERR_CUDA; no GPU fault,
  and the same session works again once the hook is off.
"""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def session(model="kitaev", L=3, kind=0, alpha=1, std=0.1, seed=4, **kw):
    rng = np.random.default_rng(seed)
    om = O.Model.kitaev(L) if model == "kitaev" else O.Model.toric(L)
    mach = O.Machine(om, "symmetry" if kind else "basic", alpha,
                     symm=0.5 if model == "kitaev" else 1.0).init_random(rng, std)
    gm = rbmnqs.Model.kitaev(L) if model == "kitaev" else rbmnqs.Model.toric(L, symmetry=1.0)
    cfg = rbmnqs.default_config(rbm_type=kind, alpha=alpha, n_chains=16, samples_per_chain=8, warmup=2, seed=seed,
                                **kw)
    s = rbmnqs.Session(gm, cfg)
    s.set_weights(mach.params())
    return s, mach


@pytest.mark.parametrize("precision", [1, 0])
def test_nonfinite_weights_are_reported_and_not_applied(precision):
    s, mach = session(precision=precision)
    w = mach.params().copy()
    w[3] = np.nan
    s.set_weights(w)
    st = s.sample()
    assert st["status"] == rbmnqs.ERR_NONFINITE
    sr = s.optimize()
    assert sr["status"] == rbmnqs.ERR_NONFINITE
    w_after = s.get_weights()
    assert np.array_equal(np.isnan(w_after), np.isnan(w))
    assert np.array_equal(w_after[~np.isnan(w)], w[~np.isnan(w)])
    # a finite state again: the next epoch is normal
    s.set_weights(mach.params())
    st, sr = s.epoch()
    assert st["status"] == 0 and sr["status"] == 0


def test_massive_step_is_reported_and_not_applied():
    """SGD direction Re F / real_factor with real_factor 1e-9: max|dw| far
    above 30 whatever the samples (gradient_descent.cpp:42-60 feeding the
    guard of abstract_optimizer.cpp:157-159)."""
    s, mach = session(precision=1, optimizer_type=1, sgd_real_factor=1e-9)
    w0 = s.get_weights()
    s.sample()
    sr = s.optimize()
    assert sr["max_dw"] > 30
    assert sr["status"] == rbmnqs.ERR_MASSIVE_STEP
    assert np.array_equal(s.get_weights(), w0)


def test_cg_iteration_cap_reports_the_residual():
    s, mach = session(precision=1, max_iterations=1)
    s.sample()
    sr = s.optimize()
    assert sr["status"] == 0
    assert sr["iterations"] == 1
    assert sr["residual"] > 1e-16  # the default tolerance was not reached
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    x, it, rs = O.cg_solve(Om, d, F, np.zeros(mach.n_params), sr["reg1"], sr["reg2"], sr["deltareg1"], diag,
                           max_iterations=1)
    assert it == 1 and abs(rs - sr["residual"]) < 1e-8 * rs


@pytest.mark.parametrize("model,L,alpha", [("kitaev", 3, 1), ("toric", 4, 2)])
def test_cooperative_barrier_wait_runs_out(model, L, alpha):
    """The formed-S cooperative CG (360 parameters) and the matrix-free CG
    (2144 parameters): with the barrier fault the solve gives up, reports
    RBMNQS_ERR_CUDA and leaves the weights as they were; with the fault off
    the same session solves again."""
    s, mach = session(model=model, L=L, alpha=alpha, precision=1, max_iterations=50)
    s.sample()
    w0 = s.get_weights()
    rbmnqs.test_fault(1)
    try:
        sr = s.optimize()
    finally:
        rbmnqs.test_fault(0)
    assert sr["status"] == -2  # RBMNQS_ERR_CUDA
    assert np.array_equal(s.get_weights(), w0)
    s.sample()
    sr = s.optimize()
    assert sr["status"] == 0 and sr["iterations"] > 0
    assert not np.array_equal(s.get_weights(), w0)


def test_proposal_network_wait_runs_out():
    """The proposal network's GEMM issues no copies under the fault: its
    bounded wait runs out and the epoch fails with RBMNQS_ERR_CUDA; with
    the fault off the session samples again."""
    s, mach = session(L=2, alpha=2, precision=0, proposal=1, learned_steps=1, learned_train=1)
    s.sample()
    rbmnqs.test_fault(2)
    try:
        with pytest.raises(rbmnqs.RbmNqsError) as e:
            s.sample()
    finally:
        rbmnqs.test_fault(0)
    assert e.value.code == -2
    assert "proposal network" in str(e.value)
    st = s.sample()
    assert st["status"] == 0 and st["learned_acceptance"] > 0


def test_standalone_network_wait_runs_out():
    net = rbmnqs.ProposalNet(32, 64, 64, 32, max_batch=256)
    net.init(0.02, 1)
    spins = O.random_spins(np.random.default_rng(2), 256, 32)
    ref = net.forward(spins)
    rbmnqs.test_fault(2)
    try:
        with pytest.raises(rbmnqs.RbmNqsError) as e:
            net.forward(spins)
    finally:
        rbmnqs.test_fault(0)
    assert e.value.code == -2
    assert np.array_equal(net.forward(spins), ref)

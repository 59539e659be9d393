"""Pins the FP64 CPU oracle against the reference's own golden data and
invariants (notebook ED outputs, lattice golden lists, gtest tolerances)."""
import numpy as np
import pytest

import ed
import oracle as O


# ------------------------------------------------------------------ RNG --
def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10.
    assert O.philox([0, 0, 0, 0], [0, 0]).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2).tolist() == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]).tolist() == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


# -------------------------------------------------------------- lattice --
def test_honeycomb_nns_golden(golden):
    for site, want in golden["honeycomb3_nns"].items():
        site = int(site)
        # test_lattice.cpp:255-258 states the site-17 list for honeycomb(5)
        n_cells = 5 if site == 17 else 3
        assert O.honeycomb_nns(n_cells, site).tolist() == want


@pytest.mark.parametrize("n_cells,key", [(2, "bonds2"), (3, "bonds3")])
def test_honeycomb_bonds_match_notebook(golden, n_cells, key):
    want = [(a, b, t) for (a, b), t in golden[key]]
    got = [tuple(x) for x in O.honeycomb_bonds(n_cells).tolist()]
    assert got == want


@pytest.mark.parametrize("n_cells,key", [(2, "plaqs2"), (3, "plaqs3")])
def test_hexagons_match_notebook(golden, n_cells, key):
    want = [tuple(h) for h, _ in golden[key]]
    got = [tuple(x) for x in O.honeycomb_hexagons(n_cells).tolist()]
    assert got == want


def test_bravais_up_down_with_shift_and_2nd_dim():
    # test_lattice.cpp:178-215 (N=5, Nb=3, shift 2)
    N, Nb, sh = 5, 3, 2
    _, up, down = O.up(N, 0, n_uc_b=Nb, h_shift=sh)
    mat = np.arange(N * Nb).reshape(N, Nb).T  # Eigen column-major (Nb, N)
    for s in range(1, Nb):
        for i in range(Nb):
            for j in range(N):
                assert up(mat[i, j], 0, s) == mat[(i + s) % Nb, j]
                assert down(mat[i, j], 0, s) == mat[(i - s + Nb) % Nb, j]
    for s in range(1, N):
        for i in range(Nb):
            for j in range(N):
                inew = (Nb + i - (sh if j + s >= N else 0)) % Nb
                assert up(mat[i, j], 1, s) == mat[inew, (j + s) % N]
                inew = (i + (sh if j - s < 0 else 0)) % Nb
                assert down(mat[i, j], 1, s) == mat[inew, (j - s + N) % N]


def test_symmetry_tables():
    perm, basis = O.symmetry("honeycomb", 4, 0.5)
    n = 32
    assert perm.shape == (n, n) and basis.tolist() == [0]
    for p in perm:
        assert sorted(p.tolist()) == list(range(n))
    # the orbit of the basis site covers every site exactly once
    assert sorted(perm[:, 0].tolist()) == list(range(n))
    perm1, basis1 = O.symmetry("toric", 3, 1.0)
    assert perm1.shape == (9, 18) and basis1.tolist() == [0, 1]


def test_toric_plaqs():
    p = O.toric_plaqs(3)
    assert p.shape == (18, 5)
    # every spin sits on exactly two plaquettes and two stars
    for t in (0, 1):
        cnt = np.bincount(p[p[:, 4] == t, :4].ravel(), minlength=18)
        assert (cnt == 2).all()


# ------------------------------------------------------------------- ED --
@pytest.mark.parametrize("n_cells,key,wkey", [(2, "ed_energy_per_site_2x2", "ed_wp_2x2"),
                                              (3, "ed_energy_per_site_3x3", "ed_wp_3x3")])
def test_ed_matches_notebook(golden, n_cells, key, wkey):
    model = O.Model.kitaev(n_cells)
    H = ed.hamiltonian(model)
    e0, v = ed.ground_state(H)
    assert abs(e0 / model.n - golden[key]) < 1e-10
    hexm = O.Model.hexagons(n_cells)
    for o, want in enumerate(golden[wkey]):
        Wp = ed.hamiltonian(O.Model(hexm.n, hexm.k[o:o + 1], hexm.sites[o:o + 1], [0],
                                    hexm.mats[2 * hexm.mat_off[o]: 2 * (hexm.mat_off[o] + 4096)]))
        assert abs(np.vdot(v, Wp @ v).real - want) < 1e-8


def test_kitaev_exact_energy_3x3(golden):
    assert abs(O.kitaev_exact_energy(3) - golden["ed_energy_per_site_3x3"]) < 1e-10


def test_toric_ground_energy():
    model = O.Model.toric(2)
    e0, _ = ed.ground_state(ed.hamiltonian(model))
    assert abs(e0 / model.n + 1.0) < 1e-10


# ------------------------------------------------------- wavefunctions --
def _machine(kind, n_cells=3, alpha=1, std=0.2, seed=1, pf=False, model="kitaev"):
    rng = np.random.default_rng(seed)
    mdl = O.Model.kitaev(n_cells) if model == "kitaev" else O.Model.toric(n_cells)
    m = O.Machine(mdl, kind, alpha, symm=0.5 if model == "kitaev" else 1.0, pfaffian=pf)
    m.init_random(rng, std, std_pf=0.1)
    return mdl, m, rng


@pytest.mark.parametrize("kind", ["basic", "symmetry"])
def test_ratio_consistent_with_log_psi(kind):
    mdl, m, rng = _machine(kind)
    s = O.random_spins(rng, 8, m.n)
    lp, _, _ = O.eval_batch(m, mdl, s, with_O=False)
    for b in range(8):
        fl = rng.choice(m.n, 2, replace=False)
        s2 = s[b].copy()
        for f in fl:
            s2[f // 32] ^= np.uint32(1 << (f % 32))
        lp2, _, _ = O.eval_batch(m, mdl, s2[None], with_O=False)
        r = O.log_psi_over_psi(m, s[b], fl)
        assert abs(np.exp(r) - np.exp(lp2[0] - lp[b])) < 1e-12 * abs(np.exp(r))


@pytest.mark.parametrize("kind", ["basic", "symmetry"])
def test_derivative_finite_difference(golden, kind):
    # test_derivative.cpp:78-112: psi(w + dw) ~ psi(w)(1 + dw.O), per-parameter
    # relative tolerance 1e-15 at |dw| ~ 1e-7 (honeycomb(5), alpha 10, std 0.2)
    g = golden["test_derivative"]
    rng = np.random.default_rng(g["seed"])
    mdl = O.Model.kitaev(5)
    # rbm_base{10, lat} -> alpha 10; honeycomb(5)'s default symmetry is {1}
    m = O.Machine(mdl, kind, alpha=g["n_hidden"], symm=1.0)
    m.init_random(rng, g["weight_std"])
    s = O.random_spins(rng, 1, m.n)[0]
    # The reference's forward difference carries the second-order term
    # (dw.O)^2/2 ~ 3e-10, which alone exceeds 1e-15 * P at alpha 10; the
    # central difference below cancels it and keeps the reference tolerance.
    for _ in range(10):
        dw = g["rbm_fd_dw_scale"] * (rng.normal(size=m.n_params) + 1j * rng.normal(size=m.n_params))
        lp, _, Od = O.eval_batch(m, mdl, s[None])
        w = m.params()
        m.set_params(w + dw)  # rbm.update_weights(-dw) subtracts -dw
        lpp, _, _ = O.eval_batch(m, mdl, s[None], with_O=False)
        m.set_params(w - dw)
        lpm, _, _ = O.eval_batch(m, mdl, s[None], with_O=False)
        m.set_params(w)
        central = 0.5 * (np.exp(lpp[0] - lp[0]) - np.exp(lpm[0] - lp[0]))
        assert abs(central - dw @ Od[0]) / m.n_params < g["rbm_fd_tol_per_param"]
        f = int(rng.integers(m.n))
        s[f // 32] ^= np.uint32(1 << (f % 32))


def test_pfaffian_against_determinant():
    rng = np.random.default_rng(3)
    A = rng.normal(size=(10, 10)) + 1j * rng.normal(size=(10, 10))
    A = A - A.T
    mant, e = O.pfaffian10(A)
    pf = mant * 10.0 ** e
    assert abs(pf * pf - np.linalg.det(A)) < 1e-10 * abs(np.linalg.det(A))


def test_pfaffian_update_drift(golden):
    # test_derivative.cpp:120-154: 100 two-site updates vs a fresh context
    g = golden["test_derivative"]
    rng = np.random.default_rng(g["seed"])
    mdl = O.Model.kitaev(3)
    m = O.Machine(mdl, "basic", 1, pfaffian=True)
    m.fs[:] = rng.normal(0, g["pf_weight_std"], m.fs.shape) + 1j * rng.normal(0, g["pf_weight_std"], m.fs.shape)
    s = O.random_spins(rng, 1, m.n)[0]
    ctx, inv = O.pf_context(m, s)
    for _ in range(g["n_updates"]):
        fl = rng.choice(m.n, 2, replace=False)
        O.pf_update(m, s, fl, ctx)
        for f in fl:
            s[f // 32] ^= np.uint32(1 << (f % 32))
    ctx2, inv2 = O.pf_context(m, s)
    assert np.mean(np.abs(inv - inv2)) < g["pf_inv_drift_tol"]
    pf1 = complex(*ctx.pf_mant)
    pf2 = complex(*ctx2.pf_mant) * 10.0 ** (ctx2.pf_exp10 - ctx.pf_exp10)
    assert abs(pf1 - pf2) * 10.0 ** ctx.pf_exp10 < g["pf_pfaffian_drift_tol"] * max(1.0, 10.0 ** ctx.pf_exp10)


def test_pfaffian_derivative_finite_difference(golden):
    g = golden["test_derivative"]
    rng = np.random.default_rng(g["seed"] + 1)
    mdl = O.Model.kitaev(3)
    m = O.Machine(mdl, "basic", 1, pfaffian=True)
    m.init_random(rng, 1e-2, std_pf=g["pf_weight_std"])
    s = O.random_spins(rng, 1, m.n)[0]
    for _ in range(5):
        dw = np.zeros(m.n_params, np.complex128)
        npf = 4 * m.n_indep
        dw[-npf:] = g["pf_fd_dw_scale"] * (rng.normal(size=npf) + 1j * rng.normal(size=npf))
        lp, _, Od = O.eval_batch(m, mdl, s[None])
        w = m.params()
        m.set_params(w + dw)  # pfaff.update_weights(-dw)
        lpp, _, _ = O.eval_batch(m, mdl, s[None], with_O=False)
        m.set_params(w - dw)
        lpm, _, _ = O.eval_batch(m, mdl, s[None], with_O=False)
        m.set_params(w)
        central = 0.5 * (np.exp(lpp[0] - lp[0]) - np.exp(lpm[0] - lp[0]))
        assert abs(central - dw @ Od[0]) / m.n_params < g["pf_fd_tol_per_param"]
        f = int(rng.integers(m.n))
        s[f // 32] ^= np.uint32(1 << (f % 32))


# ------------------------------------------------------ full sampling --
@pytest.mark.parametrize("kind,n_cells", [("basic", 2), ("symmetry", 2), ("basic", 3)])
def test_full_enumeration_energy_matches_ed(kind, n_cells):
    mdl, m, rng = _machine(kind, n_cells=n_cells, std=0.3)
    res = O.full(m, mdl, with_O=False)
    H = ed.hamiltonian(mdl)
    N = 1 << m.n
    bits = ((np.arange(N)[:, None] >> np.arange(m.n)[None, :]) & 1)
    lp, _, _ = O.eval_batch(m, mdl, O.spins_from_bits(bits), with_O=False)
    psi = np.exp(lp - lp.real.max())
    e = np.vdot(psi, H @ psi) / np.vdot(psi, psi)
    assert abs(res["E"] - e) < 1e-8 * abs(e)


def test_toric_eloc_full():
    mdl, m, rng = _machine("basic", n_cells=2, std=0.3, model="toric")
    res = O.full(m, mdl, with_O=False)
    H = ed.hamiltonian(mdl)
    N = 1 << m.n
    bits = ((np.arange(N)[:, None] >> np.arange(m.n)[None, :]) & 1)
    lp, _, _ = O.eval_batch(m, mdl, O.spins_from_bits(bits), with_O=False)
    psi = np.exp(lp - lp.real.max())
    e = np.vdot(psi, H @ psi) / np.vdot(psi, psi)
    assert abs(res["E"] - e) < 1e-8 * abs(e)


# ------------------------------------------------------------ sampler --
def test_metropolis_estimates_energy():
    mdl, m, rng = _machine("basic", n_cells=2, std=0.3)
    ex = O.full(m, mdl, with_O=False)["E"].real
    E, _, acc, _ = O.metropolis(m, mdl, 8, 2000, warmup=50, seed=7, with_O=False)
    st = O.stats(E)
    assert 0 < acc.mean() <= 1
    assert abs(st["mean"].real - ex) < 5 * max(st["stddev"], 1e-3)


def test_metropolis_bond_flips_and_determinism():
    mdl, m, rng = _machine("symmetry", n_cells=2, std=0.3)
    a = O.metropolis(m, mdl, 4, 50, warmup=5, bond_flips=0.5, seed=11)
    b = O.metropolis(m, mdl, 4, 50, warmup=5, bond_flips=0.5, seed=11)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[3], b[3])


# -------------------------------------------------------------- stats --
def test_stats_formulas():
    rng = np.random.default_rng(5)
    x = rng.normal(size=1000) + 1j * rng.normal(size=1000)
    st = O.stats(x)
    assert st["n_bins"] == 50
    mu = x.mean()
    assert abs(st["mean"] - mu) < 1e-14
    assert abs(st["var"] - np.sum(np.abs(x - mu) ** 2) / 999) < 1e-12
    bm = x.reshape(50, 20).mean(1)
    vb = 20 * np.sum(np.abs(bm - mu) ** 2)
    assert abs(st["var_binned"] - vb / 999) < 1e-12
    assert abs(st["tau"] - 0.5 * (max(20 * vb / np.sum(np.abs(x - mu) ** 2), 1) - 1)) < 1e-12
    assert O.n_bins_for(262144) == 32


# ------------------------------------------------------------------ SR --
def test_cg_solves_regularised_system():
    rng = np.random.default_rng(9)
    N, P = 400, 30
    Om = rng.normal(size=(N, P)) + 1j * rng.normal(size=(N, P))
    E = rng.normal(size=N) + 1j * rng.normal(size=N)
    d, F, diag = O.sr_moments(Om, E)
    S = O.sr_matrix(Om, d)
    r1, r2 = 0.9, 1e-3
    x, it, rs = O.cg_solve(Om, d, F, np.zeros(P), r1, r2, 0.0, diag)
    A = S + np.diag(diag * r1 + diag.max() * r2)
    assert np.linalg.norm(A @ x - F) < 1e-7
    assert 0 < it <= 2 * P
    assert np.allclose(S, S.conj().T, atol=1e-13)


def qlp_system(N, P, k, s, seed):
    """Random O whose last k columns are scaled by s (1..k): S has k
    eigenvalues near s^2 next to a bulk of order 1."""
    rng = np.random.default_rng(seed)
    Om = rng.normal(size=(N, P)) + 1j * rng.normal(size=(N, P))
    if k:
        Om[:, P - k:] *= s * (1 + np.arange(k))
    E = rng.normal(size=N) + 1j * rng.normal(size=N)
    d, F, diag = O.sr_moments(Om, E)
    return Om, d, F, diag


def sr_operator(Om, d, diag, r1, r2, rd, n_neural, norm):
    S = Om.conj().T @ Om / norm - np.outer(d.conj(), d)
    f = np.where(np.arange(Om.shape[1]) < n_neural, r1, r1 + rd)
    return S + np.diag(diag * f + diag.max() * r2)


def test_minresqlp_solves_the_regularised_system():
    """The system of debug.cpp:215-262 (500 parameters, 500 samples, 50
    neural parameters, norm 0.1, d = column sums / sqrt(norm), e1 = de = e2
    = 1, itnlim 1000): the operator is indefinite (d d^H is not the outer
    product of the mean), which MINRES-QLP handles; it stops on the
    relative residual, in the MINRES phase (condition about 4e4)."""
    rng = np.random.default_rng(1)
    Om = rng.uniform(-1, 1, (500, 500)) + 1j * rng.uniform(-1, 1, (500, 500))
    d = Om.sum(0) / np.sqrt(0.1)
    diag = np.sum(np.abs(Om) ** 2, 0) / 0.1 - np.abs(d) ** 2
    F = rng.uniform(-1, 1, 500) + 1j * rng.uniform(-1, 1, 500)
    x, it, rn, info = O.minres_solve(Om, d, F, 1.0, 1.0, 1.0, diag, n_neural=50, norm=0.1, info=True,
                                     max_iterations=1000)
    A = sr_operator(Om, d, diag, 1.0, 1.0, 1.0, 50, 0.1)
    scale = np.linalg.norm(A, 2) * np.linalg.norm(x) + np.linalg.norm(F)
    assert np.linalg.norm(A @ x - F) < 1e-14 * scale  # the relative residual MINRES-QLP bounds
    assert info["istop"] in (4, 5) and info["qlp"] == 0 and info["acond"] < 1e7
    assert 0 < it < 1000 and rn < 1e-14 * scale


def test_minresqlp_switches_to_qlp_on_an_ill_conditioned_system():
    """Four eigenvalues near 1e-10 beside an O(1) bulk (condition 3e10):
    the condition estimate passes trancond = 1e7, the QLP updates take over
    and the solution still agrees with the dense solve to cond * eps."""
    Om, d, F, diag = qlp_system(300, 80, 4, 1e-5, 3)
    x, it, rn, info = O.minres_solve(Om, d, F, 0.0, 0.0, 0.0, diag, info=True)
    A = sr_operator(Om, d, diag, 0.0, 0.0, 0.0, 80, 300)
    xs = np.linalg.solve(A, F)
    assert info["qlp"] > 0 and info["acond"] > 1e7 and info["istop"] in (4, 5), info
    assert np.linalg.norm(A @ x - F) < 1e-10 * np.linalg.norm(F)
    assert np.linalg.norm(x - xs) < 1e-4 * np.linalg.norm(xs)


def test_minresqlp_singular_system_gives_near_minimum_length():
    """40 samples, 120 parameters, no regularisation: S has rank 39 and F
    lies in its range.  MINRES-QLP solves it to rounding and its solution is
    within 1 % of the minimum-length (pseudo-inverse) solution's norm."""
    Om, d, F, diag = qlp_system(40, 120, 0, 1.0, 4)
    x, it, rn, info = O.minres_solve(Om, d, F, 0.0, 0.0, 0.0, diag, info=True)
    A = sr_operator(Om, d, diag, 0.0, 0.0, 0.0, 120, 40)
    xp = np.linalg.pinv(A, rcond=1e-10, hermitian=True) @ F
    assert np.linalg.norm(A @ x - F) < 1e-12 * np.linalg.norm(F)
    assert np.linalg.norm(x) < 1.01 * np.linalg.norm(xp)
    assert info["qlp"] > 0


def test_minresqlp_stopping_rules():
    """itnlim reached: istop 8 after exactly max_iterations steps; a loose
    rtol: istop 4 (relative residual <= rtol) long before rounding level;
    b = 0: istop 3, x = 0, no iterations."""
    Om, d, F, diag = qlp_system(300, 80, 4, 1e-5, 3)
    x, it, rn, info = O.minres_solve(Om, d, F, 0.0, 0.0, 0.0, diag, max_iterations=7, info=True)
    assert it == 7 and info["istop"] == 8
    x, it, rn, info = O.minres_solve(Om, d, F, 0.0, 0.0, 0.0, diag, rtol=1e-3, info=True)
    assert info["istop"] == 4 and it < 40
    x, it, rn, info = O.minres_solve(Om, d, np.zeros_like(F), 0.0, 0.0, 0.0, diag, info=True)
    assert it == 0 and info["istop"] == 3 and not np.any(x)


def test_decay_schedule():
    d = O.Decay(1.0, 1e-4, 0.9)
    assert abs(d.get() - 0.9) < 1e-15  # decays before first use
    c = O.Decay(1e-2)
    assert c.get() == 1e-2 and c.get() == 1e-2

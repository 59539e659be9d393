"""GPU exact diagonalisation (Lanczos on the full 2^n basis) against the
reference notebook's ED energies (2x2 and 3x3 Kitaev), scipy on the same
Hamiltonian (with a complex field term), the toric code's exact ground
energy, and the analytic flux-free Kitaev energy at 24 sites."""
import json
import os

import numpy as np
import pytest

import ed
import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.json")))


@pytest.mark.parametrize("L,key", [(2, "ed_energy_per_site_2x2"), (3, "ed_energy_per_site_3x3")])
def test_kitaev_ground_energy_matches_reference_notebook(L, key):
    gm = rbmnqs.Model.kitaev(L)
    e, it = gm.ground_state()
    assert abs(e / gm.n - GOLD[key]) < 1e-10 * abs(GOLD[key])
    assert it < 400


def test_toric_ground_energy_is_exact():
    gm = rbmnqs.Model.toric(2)
    e, _ = gm.ground_state()
    assert abs(e - (-gm.n)) < 1e-10 * gm.n


@pytest.mark.parametrize("h", [0.0, 0.1])
def test_ground_state_matches_scipy(h):
    """Including a field with sigma^y terms (a complex Hamiltonian): the
    energy and the eigenvector's residual |H psi - E psi|."""
    gm = rbmnqs.Model.kitaev(2, h=h)
    om = O.Model.kitaev(2, h=h)
    H = ed.hamiltonian(om)
    eref, _ = ed.ground_state(H)
    e, it, psi = gm.ground_state(vector=True)
    assert abs(e - eref) < 1e-10 * abs(eref)
    assert abs(np.linalg.norm(psi) - 1) < 1e-12
    assert np.linalg.norm(H @ psi - e * psi) < 1e-6
    assert abs(np.vdot(psi, H @ psi).real - e) < 1e-9 * abs(e)


def test_24_site_kitaev_matches_flux_free_energy():
    """3 x 4 unit cells (2^24 states): the GPU ground energy against the
    analytic flux-free energy of the same lattice."""
    gm = rbmnqs.Model.kitaev(3, 4)
    e, it = gm.ground_state(max_iter=600)
    ex = O.kitaev_exact_energy(3, 4)
    assert abs(e / gm.n - ex) < 1e-9 * abs(ex), (e / gm.n, ex, it)

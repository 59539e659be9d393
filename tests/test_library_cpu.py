"""CPU checks of the C-ABI library: it loads, exports every symbol the header
declares, its host-side lattice/model tables equal the oracle's bit for bit,
and compute entry points fail loudly (never fall back) without a GPU."""
import ctypes
import subprocess

import numpy as np
import pytest

import oracle as O
import rbmnqs


def test_exports_every_declared_symbol():
    L = rbmnqs.lib()
    declared = rbmnqs.header_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", rbmnqs.LIBPATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported


@pytest.mark.parametrize("n_cells", [2, 3, 4, 8])
def test_kitaev_tables_match_oracle(n_cells):
    m = rbmnqs.Model.kitaev(n_cells)
    ref = O.Model.kitaev(n_cells)
    assert m.n == ref.n and m.n_ops == ref.n_ops
    assert np.array_equal(m.bonds(), O.honeycomb_bonds(n_cells))
    for o in range(m.n_ops):
        k, acts, mat = m.op(o)
        assert k == ref.k[o] and list(acts) == list(ref.sites[o, :k])
        assert np.array_equal(mat, ref.op_matrix(o))
    perm, basis = m.symmetry()
    rp, rb = O.symmetry("honeycomb", n_cells, 0.5)
    assert np.array_equal(perm, rp) and np.array_equal(basis, rb)


@pytest.mark.parametrize("symm", [0.0, 1.0])
def test_kitaev_symmetry_variants(symm):
    m = rbmnqs.Model.kitaev(4, symmetry=symm)
    perm, basis = m.symmetry()
    rp, rb = O.symmetry("honeycomb", 4, symm)
    assert np.array_equal(perm, rp) and np.array_equal(basis, rb)


def test_kitaev_field_ops_match_oracle():
    m = rbmnqs.Model.kitaev(2, h=0.3, J=(-1.0, -0.5, 0.7))
    ref = O.Model.kitaev(2, h=0.3, J=(-1.0, -0.5, 0.7))
    assert m.n_ops == ref.n_ops
    for o in range(m.n_ops):
        k, acts, mat = m.op(o)
        assert np.array_equal(mat, ref.op_matrix(o))


@pytest.mark.parametrize("L", [2, 3, 5, 8])
def test_toric_tables_match_oracle(L):
    m = rbmnqs.Model.toric(L)
    ref = O.Model.toric(L)
    assert m.n == ref.n and m.n_ops == ref.n_ops
    for o in range(m.n_ops):
        k, acts, mat = m.op(o)
        assert list(acts) == list(ref.sites[o, :4])
        assert np.array_equal(mat, ref.op_matrix(o))
    perm, basis = m.symmetry()
    rp, rb = O.symmetry("toric", L, 1.0)
    assert np.array_equal(perm, rp) and np.array_equal(basis, rb)


@pytest.mark.parametrize("kind,L", [("kitaev", 2), ("kitaev", 3), ("kitaev", 4), ("toric", 3), ("toric", 4)])
@pytest.mark.parametrize("psym", [0.0, 0.5, 1.0])
def test_pfaffian_classes_match_oracle(kind, L, psym):
    """Pair-class matrix bs_ and n_indep of pfaffian.cpp:31-85, bit for bit."""
    m = rbmnqs.Model.kitaev(L) if kind == "kitaev" else rbmnqs.Model.toric(L)
    om = O.Model.kitaev(L) if kind == "kitaev" else O.Model.toric(L)
    ref = O.Machine(om, "basic", 1, pfaffian=True, pf_symm=psym)
    bs, ni = m.pfaffian_classes(psym)
    assert ni == ref.n_indep
    assert np.array_equal(bs, ref.bs)


def test_hexagon_observables_match_oracle():
    m = rbmnqs.Model.kitaev(3)
    m.add_hexagons()
    assert m.n_obs == 9
    hx = O.honeycomb_hexagons(3)
    for i in range(9):
        k, acts, mat = m.op(m.n_ops + i)
        assert list(acts) == hx[i].tolist()


def test_create_fails_loudly_without_gpu():
    try:
        ctypes.CDLL("libcuda.so.1")
        pytest.skip("a CUDA driver is present")
    except OSError:
        pass
    m = rbmnqs.Model.kitaev(2)
    cfg = rbmnqs.default_config()
    with pytest.raises(rbmnqs.RbmNqsError) as e:
        rbmnqs.Session(m, cfg)
    assert e.value.code == -6


def test_default_config_matches_reference_ini():
    c = rbmnqs.default_config()
    assert c.n_chains == 4 and c.warmup == 100 and c.step == 1 and c.bond_flips == 0.5
    assert list(c.reg1) == [1.0, 1e-4, 0.9] and list(c.reg2) == [1e-3, 1e-6, 0.9]
    assert list(c.lr)[:1] == [1e-2] and c.seed == 421390484

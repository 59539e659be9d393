"""The reference's .rbm checkpoint format (rbm_base::save / load,
rbm_base.cpp:219-288; matrices as eigen_fstream.cpp:25-51): files written by
the library read back with an independent reader of that layout, files
written by that layout load into a session, the update count restarts the
decay_t schedules."""
import struct

import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu


def write_mat(f, m):
    m = np.atleast_2d(np.asarray(m, np.complex128).T).T if np.ndim(m) == 1 else np.asarray(m, np.complex128)
    if m.ndim == 1:
        m = m[:, None]
    f.write(struct.pack("<QQ", m.shape[0], m.shape[1]))
    f.write(np.asfortranarray(m).ravel(order="F").astype(np.complex128).tobytes())


def read_mat(f):
    r, c = struct.unpack("<QQ", f.read(16))
    a = np.frombuffer(f.read(16 * r * c), np.complex128)
    return a.reshape(c, r).T


def session(kind="symmetry", pf=False, seed=3):
    rng = np.random.default_rng(seed)
    om = O.Model.kitaev(3)
    mach = O.Machine(om, kind, 2, symm=0.5, pfaffian=pf, pf_symm=0.5).init_random(rng, 0.1, 0.2)
    cfg = rbmnqs.default_config(rbm_type=1 if kind == "symmetry" else 0, alpha=2, n_chains=16, samples_per_chain=8,
                                warmup=2, pfaffian=1 if pf else 0, pfaffian_refresh=8, precision=1)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(3), cfg)
    s.set_weights(mach.params())
    return s, mach


@pytest.mark.parametrize("kind,pf", [("symmetry", False), ("basic", False), ("symmetry", True)])
def test_saved_file_has_the_reference_layout(tmp_path, kind, pf):
    s, mach = session(kind, pf)
    path = tmp_path / "m.rbm"
    s.save(path)
    with open(path, "rb") as f:
        W = read_mat(f)
        h = read_mat(f)
        v = read_mat(f)
        (nu,) = struct.unpack("<Q", f.read(8))
        fs = read_mat(f) if pf else None
        assert f.read() == b""
    assert W.shape == (mach.n, mach.nh) and h.shape == (mach.nh, 1) and v.shape == (mach.n_vb, 1)
    assert np.array_equal(W, mach.W.T) and np.array_equal(h[:, 0], mach.h) and np.array_equal(v[:, 0], mach.v)
    assert nu == 0
    if pf:
        assert np.array_equal(fs, mach.fs.T)


def test_load_sets_weights_and_restarts_schedules(tmp_path):
    s, mach = session()
    rng = np.random.default_rng(9)
    W = rng.normal(size=(mach.n, mach.nh)) + 1j * rng.normal(size=(mach.n, mach.nh))
    h = rng.normal(size=mach.nh) * 0.1 + 0j
    v = rng.normal(size=mach.n_vb) * 0.1 + 0j
    path = tmp_path / "w.rbm"
    with open(path, "wb") as f:
        write_mat(f, 0.01 * W)
        write_mat(f, h)
        write_mat(f, v)
        f.write(struct.pack("<Q", 7))
    s.load(path)
    w = s.get_weights()
    assert np.array_equal(w[:mach.n_vb], v)
    assert np.array_equal(w[mach.n_vb:mach.n_vb + mach.nh], h)
    assert np.array_equal(w[mach.n_vb + mach.nh:], (0.01 * W).T.ravel())
    assert s.n_updates() == 7
    s.sample()
    st = s.optimize()
    # decay_t(1, 1e-4, 0.9) constructed at offset 7 decays before its first use
    assert abs(st["reg1"] - 0.9 ** 8) < 1e-15
    assert s.n_updates() == 8
    # a round trip through the library's own writer
    s.save(tmp_path / "again.rbm")
    t, _ = session(seed=11)
    t.load(tmp_path / "again.rbm")
    assert np.array_equal(t.get_weights(), s.get_weights()) and t.n_updates() == 8


def test_load_rejects_other_shapes(tmp_path):
    s, _ = session("basic")
    other, _ = session("symmetry")
    other.save(tmp_path / "o.rbm")
    with pytest.raises(rbmnqs.RbmNqsError):
        s.load(tmp_path / "o.rbm")

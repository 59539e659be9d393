"""ctypes wrapper around the FP64 CPU oracle (oracle/liborc.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product library never
imports or calls anything in this directory.

The oracle restates the reference algorithm (dbucher97/rbm-nqs); the C
sources cite the reference file:line of every function.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liborc.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _declare(_LIB)
    return _LIB


P_I = C.POINTER(C.c_int)
P_D = C.POINTER(C.c_double)
P_U32 = C.POINTER(C.c_uint32)


class _Ops(C.Structure):
    _fields_ = [("n_ops", C.c_int), ("k", P_I), ("sites", P_I), ("mat_off", P_I), ("mats", P_D)]


class _Machine(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("n_vb", C.c_int), ("nh", C.c_int), ("S", C.c_int),
        ("symmetric", C.c_int), ("perm", P_I), ("basis", P_I),
        ("v", P_D), ("h", P_D), ("W", P_D),
        ("has_pf", C.c_int), ("n_indep", C.c_int), ("bs", P_I), ("fs", P_D),
    ]


class _Cfg(C.Structure):
    _fields_ = [
        ("n_chains", C.c_int), ("samples_per_chain", C.c_int), ("warmup", C.c_int),
        ("step", C.c_int), ("bond_flips", C.c_double), ("n_prop_bonds", C.c_int),
        ("prop_bonds", P_I), ("seed", C.c_uint64), ("pf_refresh", C.c_int),
    ]


class _Cplx(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class _PfCtx(C.Structure):
    _fields_ = [("inv", P_D), ("pf_mant", C.c_double * 2), ("pf_exp10", C.c_int),
                ("update_factor", C.c_double * 2)]


def _declare(L):
    L.orc_philox.argtypes = [P_U32, P_U32, P_U32]
    L.orc_up.restype = C.c_uint64
    L.orc_down.restype = C.c_uint64
    L.orc_honeycomb_bonds.argtypes = [C.c_int, C.c_int, P_I]
    L.orc_honeycomb_nns.argtypes = [C.c_int, C.c_int, C.c_int, P_I]
    L.orc_honeycomb_hexagons.argtypes = [C.c_int, C.c_int, P_I]
    L.orc_toric_plaqs.argtypes = [C.c_int, P_I]
    L.orc_symmetry.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, P_I, P_I, P_I]
    L.orc_kitaev_sizes.argtypes = [C.c_int, C.c_int, C.c_double, P_I, P_I]
    L.orc_kitaev_ops.argtypes = [C.c_int, C.c_int, P_D, C.c_double, P_I, P_I, P_I, P_D]
    L.orc_toric_sizes.argtypes = [C.c_int, P_I, P_I]
    L.orc_toric_ops.argtypes = [C.c_int, C.c_double, P_I, P_I, P_I, P_D]
    L.orc_hexagon_sizes.argtypes = [C.c_int, C.c_int, P_I, P_I]
    L.orc_hexagon_ops.argtypes = [C.c_int, C.c_int, P_I, P_I, P_I, P_D]
    L.orc_kitaev_exact_energy.argtypes = [C.c_int, C.c_int, P_D]
    L.orc_kitaev_exact_energy.restype = C.c_double
    L.orc_pfaffian_bs.argtypes = [C.c_int, C.c_int, P_I, C.c_int, P_I, P_I]
    L.orc_n_params.argtypes = [C.POINTER(_Machine)]
    L.orc_eval_batch.argtypes = [C.POINTER(_Machine), C.POINTER(_Ops), P_U32, C.c_int, P_D, P_D, P_D]
    L.orc_log_psi_over_psi.argtypes = [C.POINTER(_Machine), P_U32, P_I, C.c_int]
    L.orc_log_psi_over_psi.restype = _Cplx
    L.orc_theta.argtypes = [C.POINTER(_Machine), P_U32, P_D]
    L.orc_metropolis.argtypes = [C.POINTER(_Machine), C.POINTER(_Ops), C.POINTER(_Cfg), C.c_uint32,
                                 C.c_int, P_U32, P_D, P_D, P_D, C.c_int]
    L.orc_full.argtypes = [C.POINTER(_Machine), C.POINTER(_Ops), P_D, P_D, P_D, P_D, P_D, C.c_int]
    L.orc_stats.argtypes = [P_D, C.c_int, C.c_int, P_D, P_D, P_D, P_D, P_D]
    L.orc_sr_moments.argtypes = [P_D, P_D, C.c_int, C.c_int, P_D, P_D, P_D]
    L.orc_sr_matrix.argtypes = [P_D, P_D, C.c_int, C.c_int, P_D]
    L.orc_cg_solve.argtypes = [P_D, P_D, C.c_double, C.c_int, C.c_int, C.c_int, P_D, P_D,
                               C.c_double, C.c_double, C.c_double, P_D, C.c_int, C.c_double, P_D]
    L.orc_minresqlp_solve.argtypes = [P_D, P_D, C.c_double, C.c_int, C.c_int, C.c_int, P_D, P_D,
                                      C.c_double, C.c_double, C.c_double, P_D, C.c_int, C.c_double, P_D,
                                      P_I, P_D, P_I]
    L.orc_pf_context.argtypes = [C.POINTER(_Machine), P_U32, C.POINTER(_PfCtx)]
    L.orc_pf_update.argtypes = [C.POINTER(_Machine), P_U32, P_I, C.c_int, C.POINTER(_PfCtx)]
    L.orc_pf_matrix.argtypes = [C.POINTER(_Machine), P_U32, P_D]
    L.orc_pfaffian10.argtypes = [C.c_int, P_D, P_I]
    L.orc_pfaffian10.restype = _Cplx


def _p(a, t):
    return a.ctypes.data_as(t)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


# ------------------------------------------------------------------ RNG --
def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(_p(c, P_U32), _p(k, P_U32), _p(o, P_U32))
    return o


# -------------------------------------------------------------- lattice --
def honeycomb_bonds(n_cells, n_cells_b=-1):
    nb = n_cells * (n_cells if n_cells_b < 0 else n_cells_b) * 3
    out = np.zeros((nb, 3), dtype=np.int32)
    lib().orc_honeycomb_bonds(n_cells, n_cells_b, _p(out, P_I))
    return out


def honeycomb_nns(n_cells, site, n_cells_b=-1):
    out = np.zeros(3, dtype=np.int32)
    lib().orc_honeycomb_nns(n_cells, n_cells_b, site, _p(out, P_I))
    return out


def honeycomb_hexagons(n_cells, n_cells_b=-1):
    nh = n_cells * (n_cells if n_cells_b < 0 else n_cells_b)
    out = np.zeros((nh, 6), dtype=np.int32)
    lib().orc_honeycomb_hexagons(n_cells, n_cells_b, _p(out, P_I))
    return out


def toric_plaqs(n_cells):
    out = np.zeros((2 * n_cells * n_cells, 5), dtype=np.int32)
    lib().orc_toric_plaqs(n_cells, _p(out, P_I))
    return out


def symmetry(kind, n_cells, symm, n_cells_b=-1):
    """kind 'honeycomb' | 'toric'.  Returns (perm[S][n], basis[n_vb])."""
    kk = 0 if kind == "honeycomb" else 1
    nb = n_cells if n_cells_b < 0 else n_cells_b
    n = 2 * n_cells * nb
    perm = np.zeros(n * n, dtype=np.int32)
    basis = np.zeros(n, dtype=np.int32)
    nvb = C.c_int(0)
    S = lib().orc_symmetry(kk, n_cells, n_cells_b, float(symm), _p(perm, P_I), _p(basis, P_I), C.byref(nvb))
    return perm[: S * n].reshape(S, n).copy(), basis[: nvb.value].copy()


def up(n_uc, uc, dir=0, step=1, n_uc_b=0, h_shift=0, n_basis=1):
    class B(C.Structure):
        _fields_ = [(f, C.c_uint64) for f in
                    ("n_uc", "n_dim", "n_basis", "n_coord", "n_total_uc", "n_total", "n_uc_b", "h_shift")]
    b = B()
    lib().orc_bravais_init(C.byref(b), C.c_uint64(n_uc), C.c_uint64(2), C.c_uint64(n_basis), C.c_uint64(0),
                           C.c_uint64(n_uc_b), C.c_uint64(h_shift))
    return b, (lambda u, d=0, s=1: lib().orc_up(C.byref(b), C.c_uint64(u), C.c_uint64(d), C.c_uint64(s))), \
        (lambda u, d=0, s=1: lib().orc_down(C.byref(b), C.c_uint64(u), C.c_uint64(d), C.c_uint64(s)))


# --------------------------------------------------------------- models --
class Model:
    """Dense local-operator Hamiltonian plus lattice bookkeeping."""

    def __init__(self, n, k, sites, mat_off, mats, bonds=None, kind="honeycomb", n_cells=0, n_cells_b=-1):
        self.n = n
        self.k = np.ascontiguousarray(k, dtype=np.int32)
        self.sites = np.ascontiguousarray(sites, dtype=np.int32)
        self.mat_off = np.ascontiguousarray(mat_off, dtype=np.int32)
        self.mats = np.ascontiguousarray(mats, dtype=np.float64)
        self.bonds = bonds
        self.kind = kind
        self.n_cells = n_cells
        self.n_cells_b = n_cells_b
        if bonds is not None:
            pb = bonds[bonds[:, 2] != 2][:, :2]
            self.prop_bonds = np.ascontiguousarray(pb, dtype=np.int32)
        else:
            self.prop_bonds = np.zeros((0, 2), dtype=np.int32)

    @property
    def n_ops(self):
        return len(self.k)

    def c_ops(self):
        o = _Ops()
        o.n_ops = self.n_ops
        o.k = _p(self.k, P_I)
        o.sites = _p(self.sites, P_I)
        o.mat_off = _p(self.mat_off, P_I)
        o.mats = _p(self.mats, P_D)
        return o

    def op_matrix(self, o):
        d = 1 << int(self.k[o])
        off = int(self.mat_off[o])
        m = self.mats[2 * off: 2 * (off + d * d)].view(np.complex128)
        return m.reshape(d, d)

    @staticmethod
    def kitaev(n_cells, n_cells_b=-1, J=(-1.0, -1.0, -1.0), h=0.0):
        no, ne = C.c_int(), C.c_int()
        lib().orc_kitaev_sizes(n_cells, n_cells_b, h, C.byref(no), C.byref(ne))
        k = np.zeros(no.value, np.int32)
        sites = np.zeros((no.value, 6), np.int32)
        off = np.zeros(no.value, np.int32)
        mats = np.zeros(2 * ne.value, np.float64)
        Jv = np.asarray(J, dtype=np.float64)
        lib().orc_kitaev_ops(n_cells, n_cells_b, _p(Jv, P_D), h, _p(k, P_I), _p(sites, P_I), _p(off, P_I),
                             _p(mats, P_D))
        nb = n_cells if n_cells_b < 0 else n_cells_b
        return Model(2 * n_cells * nb, k, sites, off, mats, honeycomb_bonds(n_cells, n_cells_b), "honeycomb",
                     n_cells, n_cells_b)

    @staticmethod
    def toric(n_cells, J=-1.0):
        no, ne = C.c_int(), C.c_int()
        lib().orc_toric_sizes(n_cells, C.byref(no), C.byref(ne))
        k = np.zeros(no.value, np.int32)
        sites = np.zeros((no.value, 6), np.int32)
        off = np.zeros(no.value, np.int32)
        mats = np.zeros(2 * ne.value, np.float64)
        lib().orc_toric_ops(n_cells, J, _p(k, P_I), _p(sites, P_I), _p(off, P_I), _p(mats, P_D))
        return Model(2 * n_cells * n_cells, k, sites, off, mats, None, "toric", n_cells)

    @staticmethod
    def hexagons(n_cells, n_cells_b=-1):
        no, ne = C.c_int(), C.c_int()
        lib().orc_hexagon_sizes(n_cells, n_cells_b, C.byref(no), C.byref(ne))
        k = np.zeros(no.value, np.int32)
        sites = np.zeros((no.value, 6), np.int32)
        off = np.zeros(no.value, np.int32)
        mats = np.zeros(2 * ne.value, np.float64)
        lib().orc_hexagon_ops(n_cells, n_cells_b, _p(k, P_I), _p(sites, P_I), _p(off, P_I), _p(mats, P_D))
        nb = n_cells if n_cells_b < 0 else n_cells_b
        return Model(2 * n_cells * nb, k, sites, off, mats, None, "honeycomb", n_cells, n_cells_b)


def kitaev_exact_energy(n_cells, n_cells_b=-1, J=(-1.0, -1.0, -1.0)):
    Jv = np.asarray(J, dtype=np.float64)
    return lib().orc_kitaev_exact_energy(n_cells, n_cells_b, _p(Jv, P_D))


# -------------------------------------------------------------- machine --
class Machine:
    """RBM (basic or symmetric) with optional Pfaffian factor; FP64 weights."""

    def __init__(self, model, kind="basic", alpha=1, symm=0.5, pfaffian=False, pf_symm=0.5):
        self.model = model
        n = model.n
        self.n = n
        self.symmetric = kind == "symmetry"
        if self.symmetric:
            perm, basis = symmetry(model.kind, model.n_cells, symm, model.n_cells_b)
        else:
            perm = np.arange(n, dtype=np.int32)[None, :].copy()
            basis = np.arange(n, dtype=np.int32)
        self.perm = np.ascontiguousarray(perm, dtype=np.int32)
        self.basis = np.ascontiguousarray(basis, dtype=np.int32)
        self.S = self.perm.shape[0]
        self.n_vb = len(self.basis)
        self.nh = alpha * self.n_vb
        self.v = np.zeros(self.n_vb, np.complex128)
        self.h = np.zeros(self.nh, np.complex128)
        self.W = np.zeros((self.nh, n), np.complex128)  # W[k, i] == Eigen W(i, k)
        self.has_pf = bool(pfaffian)
        self.n_indep = 0
        self.bs = np.zeros((1, 1), np.int32)
        self.fs = np.zeros((0, 4), np.complex128)
        if pfaffian:
            pperm, pbasis = symmetry(model.kind, model.n_cells, pf_symm, model.n_cells_b)
            bs = np.zeros(n * n, np.int32)
            self.n_indep = lib().orc_pfaffian_bs(n, pperm.shape[0], _p(np.ascontiguousarray(pperm), P_I),
                                                 len(pbasis), _p(np.ascontiguousarray(pbasis), P_I),
                                                 _p(bs, P_I))
            self.bs = bs.reshape(n, n)
            self.fs = np.zeros((4, self.n_indep), np.complex128)  # fs[c, i] == Eigen fs_(i, c)

    @property
    def n_neural(self):
        return self.n_vb + self.nh + self.n * self.nh

    @property
    def n_params(self):
        return self.n_neural + 4 * self.n_indep

    def init_random(self, rng, std=1e-4, std_pf=1e-2):
        def cg(shape, s):
            return rng.normal(0, s, shape) + 1j * rng.normal(0, s, shape)
        self.v[:] = cg(self.v.shape, std)
        self.h[:] = cg(self.h.shape, std)
        self.W[:] = cg(self.W.shape, std)
        if self.has_pf:
            self.fs[:] = cg(self.fs.shape, std_pf)
        return self

    def params(self):
        """Flat parameter vector in the reference order."""
        parts = [self.v, self.h, self.W.reshape(-1)]
        if self.has_pf:
            parts.append(self.fs.reshape(-1))
        return np.concatenate(parts)

    def set_params(self, w):
        w = np.asarray(w, dtype=np.complex128)
        a = self.n_vb
        b = a + self.nh
        c = b + self.nh * self.n
        self.v[:] = w[:a]
        self.h[:] = w[a:b]
        self.W[:] = w[b:c].reshape(self.nh, self.n)
        if self.has_pf:
            self.fs[:] = w[c:].reshape(4, self.n_indep)

    def c_machine(self):
        m = _Machine()
        m.n, m.n_vb, m.nh, m.S = self.n, self.n_vb, self.nh, self.S
        m.symmetric = 1 if self.symmetric else 0
        self._keep = [np.ascontiguousarray(x) for x in (self.perm, self.basis, self.v, self.h, self.W,
                                                         self.bs, self.fs)]
        perm, basis, v, h, W, bs, fs = self._keep
        m.perm = _p(perm, P_I)
        m.basis = _p(basis, P_I)
        m.v = _p(v, P_D)
        m.h = _p(h, P_D)
        m.W = _p(W, P_D)
        m.has_pf = 1 if self.has_pf else 0
        m.n_indep = self.n_indep
        m.bs = _p(bs, P_I)
        m.fs = _p(fs, P_D)
        return m


def spins_from_bits(bits):
    """bits: (B, n) array of {0,1} -> (B, 4) uint32 words."""
    bits = np.asarray(bits, dtype=np.uint64)
    B, n = bits.shape
    out = np.zeros((B, 4), dtype=np.uint32)
    for i in range(n):
        out[:, i // 32] |= (bits[:, i].astype(np.uint32) << np.uint32(i % 32))
    return out


def random_spins(rng, B, n):
    return spins_from_bits(rng.integers(0, 2, size=(B, n)))


def eval_batch(machine, model, spins, with_O=True):
    spins = np.ascontiguousarray(spins, dtype=np.uint32)
    B = spins.shape[0]
    lp = np.zeros(B, np.complex128)
    el = np.zeros(B, np.complex128)
    O = np.zeros((B, machine.n_params), np.complex128) if with_O else None
    cm = machine.c_machine()
    co = model.c_ops()
    lib().orc_eval_batch(C.byref(cm), C.byref(co), _p(spins, P_U32), B, _p(lp, P_D), _p(el, P_D),
                         _p(O, P_D) if with_O else None)
    return lp, el, O


def theta(machine, spins):
    s = np.ascontiguousarray(spins, dtype=np.uint32)
    out = np.zeros(machine.nh * machine.S, np.complex128)
    cm = machine.c_machine()
    lib().orc_theta(C.byref(cm), _p(s, P_U32), _p(out, P_D))
    return out


def log_psi_over_psi(machine, spins, flips):
    s = np.ascontiguousarray(spins, dtype=np.uint32)
    f = np.ascontiguousarray(flips, dtype=np.int32)
    cm = machine.c_machine()
    r = lib().orc_log_psi_over_psi(C.byref(cm), _p(s, P_U32), _p(f, P_I), len(f))
    return complex(r.re, r.im)


def metropolis(machine, model, n_chains, spc, warmup=0, step=1, bond_flips=0.0, seed=1, epoch=0,
               init=True, spins=None, pf_refresh=0, threads=0, with_O=True):
    cfg = _Cfg()
    cfg.n_chains, cfg.samples_per_chain, cfg.warmup, cfg.step = n_chains, spc, warmup, step
    cfg.bond_flips = bond_flips
    pb = model.prop_bonds
    cfg.n_prop_bonds = len(pb)
    cfg.prop_bonds = _p(pb, P_I)
    cfg.seed = seed
    cfg.pf_refresh = pf_refresh
    if spins is None:
        spins = np.zeros((n_chains, 4), np.uint32)
    spins = np.ascontiguousarray(spins, dtype=np.uint32)
    N = n_chains * spc
    E = np.zeros(N, np.complex128)
    O = np.zeros((N, machine.n_params), np.complex128) if with_O else None
    acc = np.zeros(n_chains, np.float64)
    cm = machine.c_machine()
    co = model.c_ops()
    lib().orc_metropolis(C.byref(cm), C.byref(co), C.byref(cfg), epoch, 1 if init else 0, _p(spins, P_U32),
                         _p(E, P_D), _p(O, P_D) if with_O else None, _p(acc, P_D), threads)
    return E, O, acc, spins


def full_order(n, bits=2):
    """State numbers in full_sampler::sample's visiting order (one process,
    full_sampler.cpp:63-136): block b over the low `bits` bits, and within
    it the Gray code gray(i) = i ^ (i >> 1) over the high n - bits bits."""
    hb = n - bits
    k = np.arange(1 << n, dtype=np.int64)
    b, i = k >> hb, k & ((1 << hb) - 1)
    return b | ((i ^ (i >> 1)) << bits)


def weighted_aggregate(x, w, n_bins):
    """aggregator::aggregate / finalize (operators/aggregator.cpp:84-239, one
    process) for a scalar observable with weights w and n_bins bins:
    the weighted Welford mean and M2, the bin recurrences, tau and the binned
    standard deviation of the mean."""
    result, wsum, wsum2, var = 0j, 0.0, 0.0, 0.0
    bin_, wsum_bin, cur, rb, vb = 0j, 0.0, 0, 0j, 0.0
    bs = len(x) // n_bins
    for xi, wi in zip(x, w):
        wsum += wi
        wsum2 += wi * wi
        delta = wi * (xi - result)
        result += delta / wsum
        var += (np.conj(xi - result) * delta).real
        if n_bins > 1:
            cur += 1
            wsum_bin += wi
            bin_ += wi * xi
            if cur == bs:
                cur = 0
                bin_ /= wsum_bin
                delta = wsum_bin * (bin_ - rb)
                rb += delta / wsum
                vb += (np.conj(delta) * (bin_ - rb)).real
                bin_, wsum_bin = 0j, 0.0
    tau = 0.0
    if n_bins > 1 and not (var == 0 and vb == 0):
        tau = 0.5 * (max(bs * vb / var, 1.0) - 1)
    den = wsum - wsum2 / wsum
    vb = max(vb / den, 0.0)
    var = max(var / den, 0.0)
    sd = np.sqrt(vb / n_bins) if n_bins > 1 else np.sqrt(var / len(x))
    return dict(mean=result, var=var, var_binned=vb, tau=tau, stddev=sd)


def full(machine, model, threads=0, with_O=True):
    P = machine.n_params
    pt = C.c_double()
    em = np.zeros(1, np.complex128)
    d = np.zeros(P, np.complex128)
    dh = np.zeros(P, np.complex128)
    var = np.zeros(P, np.float64)
    cm = machine.c_machine()
    co = model.c_ops()
    lib().orc_full(C.byref(cm), C.byref(co), C.byref(pt), _p(em, P_D), _p(d, P_D) if with_O else None,
                   _p(dh, P_D) if with_O else None, _p(var, P_D) if with_O else None, threads)
    return dict(p_tot=pt.value, E=em[0], d=d, dh=dh, var=var)


def n_bins_for(N, k=50):
    """abstract_optimizer.cpp:184-192: largest k <= 50 dividing N."""
    while N % k:
        k -= 1
    return k


def stats(x, n_bins=None):
    x = _c128(x)
    N = len(x)
    nb = n_bins_for(N) if n_bins is None else n_bins
    mean = np.zeros(1, np.complex128)
    var, vb, tau, sd = (C.c_double() for _ in range(4))
    lib().orc_stats(_p(x, P_D), N, nb, _p(mean, P_D), C.byref(var), C.byref(vb), C.byref(tau), C.byref(sd))
    return dict(mean=mean[0], var=var.value, var_binned=vb.value, tau=tau.value, stddev=sd.value, n_bins=nb)


def sr_moments(O, E):
    O = _c128(O)
    E = _c128(E)
    N, P = O.shape
    d = np.zeros(P, np.complex128)
    F = np.zeros(P, np.complex128)
    diag = np.zeros(P, np.float64)
    lib().orc_sr_moments(_p(O, P_D), _p(E, P_D), N, P, _p(d, P_D), _p(F, P_D), _p(diag, P_D))
    return d, F, diag


def sr_matrix(O, d):
    O = _c128(O)
    d = _c128(d)
    N, P = O.shape
    S = np.zeros((P, P), np.complex128)
    lib().orc_sr_matrix(_p(O, P_D), _p(d, P_D), N, P, _p(S, P_D))
    return S


def cg_solve(O, d, F, x0, r1, r2, rd, diag, n_neural=None, max_iterations=0, rtol=0.0, norm=None):
    O = _c128(O)
    N, P = O.shape
    d = _c128(d)
    F = _c128(F)
    x = _c128(x0).copy()
    diag = np.ascontiguousarray(diag, dtype=np.float64)
    rs = C.c_double()
    it = lib().orc_cg_solve(_p(O, P_D), _p(d, P_D), float(N if norm is None else norm), N, P,
                            P if n_neural is None else n_neural, _p(F, P_D), _p(x, P_D), r1, r2, rd,
                            _p(diag, P_D), max_iterations, rtol, C.byref(rs))
    return x, it, rs.value


def minres_solve(O, d, F, r1, r2, rd, diag, n_neural=None, max_iterations=0, rtol=0.0, norm=None, info=False):
    """MINRES-QLP (zminresqlpModule.f90 through minresqlp_adapter.cpp:40-110)
    on the SR operator from x0 = 0 -> (x, iterations, rnorm), plus
    {"istop", "acond", "qlp"} when info is set."""
    O = _c128(O)
    N, P = O.shape
    d = _c128(d)
    F = _c128(F)
    x = np.zeros(P, np.complex128)
    diag = np.ascontiguousarray(diag, dtype=np.float64)
    rn = C.c_double()
    ist = C.c_int()
    ac = C.c_double()
    nq = C.c_int()
    it = lib().orc_minresqlp_solve(_p(O, P_D), _p(d, P_D), float(N if norm is None else norm), N, P,
                                   P if n_neural is None else n_neural, _p(F, P_D), _p(x, P_D), r1, r2, rd,
                                   _p(diag, P_D), max_iterations, rtol, C.byref(rn), C.byref(ist), C.byref(ac),
                                   C.byref(nq))
    if info:
        return x, it, rn.value, {"istop": ist.value, "acond": ac.value, "qlp": nq.value}
    return x, it, rn.value


def direct_solve(O, d, F, r1, r2, rd, diag, n_neural=None, norm=None):
    """direct_solver::solve (optimizer/direct_solver.cpp:31-59): S =
    conj(O)^T O / norm - conj(d) d^T, the diagonal scaled by (1 + r1)
    ((1 + r1) + rd on non-neural parameters), plus r2 max|diag| I, solved
    for the minimum-norm least-squares x (what Eigen's complete orthogonal
    decomposition returns)."""
    O = _c128(O)
    N, P = O.shape
    nn = P if n_neural is None else n_neural
    S = O.conj().T @ O / float(N if norm is None else norm)
    S -= np.outer(np.conj(d), d)
    idx = np.arange(P)
    S[idx[:nn], idx[:nn]] *= 1 + r1
    if P > nn:
        S[idx[nn:], idx[nn:]] *= 1 + r1 + rd
    S[idx, idx] += r2 * np.max(np.abs(diag))
    return np.linalg.lstsq(S, _c128(F), rcond=None)[0]


class Decay:
    """decay_t (abstract_optimizer.cpp:27-54): decays before first use."""

    def __init__(self, initial, mn=None, decay=1.0, offset=0):
        self.initial = initial
        self.min = initial if mn is None else mn
        self.decay = decay
        self.value = decay ** offset * initial
        self.min_reached = decay == 1.0

    def get(self):
        if not self.min_reached:
            self.value *= self.decay
            if self.value < self.min:
                self.min_reached = True
                self.value = self.min
        return self.value


class AdamPlugin:
    """adam_plugin (optimizer/plugin.cpp:29-59): first moment complex, second
    moment split into real and imaginary parts, bias-corrected with t counted
    from 1; the result is scaled by lr."""

    def __init__(self, P, beta1=0.9, beta2=0.999, eps=1e-8):
        self.b1, self.b2, self.eps, self.t = beta1, beta2, eps, 1
        self.m = np.zeros(P, np.complex128)
        self.wr = np.zeros(P)
        self.wi = np.zeros(P)

    def apply(self, dw, lr):
        self.m = self.b1 * self.m + (1 - self.b1) * dw
        self.wr = self.b2 * self.wr + (1 - self.b2) * dw.real ** 2
        self.wi = self.b2 * self.wi + (1 - self.b2) * dw.imag ** 2
        m = self.m / (1 - self.b1 ** self.t)
        wr = self.wr / (1 - self.b2 ** self.t)
        wi = self.wi / (1 - self.b2 ** self.t)
        self.t += 1
        out = m.real / (np.sqrt(wr) + self.eps) + 1j * (m.imag / (np.sqrt(wi) + self.eps))
        return out * lr


class MomentumPlugin:
    """momentum_plugin (optimizer/plugin.cpp:61-85): a zero momentum starts at
    dw; with dialup != 1 the momentum factor ramps up as alpha * dup, dup
    starting at 1e-3 and multiplied by dialup every step until it reaches 1."""

    def __init__(self, P, alpha=0.9, dialup=1.0):
        self.alpha, self.dialup = alpha, dialup
        self.dup = 1.0 if dialup == 1.0 else 1e-3
        self.m = np.zeros(P, np.complex128)

    def apply(self, dw, lr):
        ax = self.alpha
        if np.all(np.abs(self.m) <= 1e-12):
            self.m = dw.copy()
        if self.dup < 1.0:
            self.dup *= self.dialup
            ax *= self.dup
        self.m = ax * self.m + (1 - ax) * dw
        return lr * self.m


def heun_begin(x1, lr):
    """heun_plugin::apply (optimizer/plugin.cpp:87-91), first half: the
    weights move by delta = (lr/2) x1 (update_weights_nc, no update counted)
    before the second sample; returns delta."""
    return 0.5 * lr * x1


def heun_finish(delta, x2, lr, eps, O=None, d=None):
    """heun_plugin::apply (optimizer/plugin.cpp:92-115), second half, with x2
    the step direction of the second gradient() call.  SR registers the
    metric (O of the second sample, <O>; stochastic_reconfiguration.cpp:
    111-113), giving err = sqrt(sum_s |sum_k delta_k O_sk - d.delta|^2) / P;
    SGD has none, giving err = |delta|.  Returns the step x2 (cbrt(eps/err)
    - 1/2) lr."""
    delta = (delta - 0.5 * lr * x2) / 6
    if O is not None:
        e = np.asarray(O) @ delta - np.dot(d, delta)
        err = np.sqrt(np.sum(np.abs(e) ** 2)) / delta.size
    else:
        err = np.linalg.norm(delta)
    xx = (eps / err) ** (1.0 / 3)
    return x2 * ((xx - 0.5) * lr)


def sgd_direction(F, real_factor=1.0):
    """gradient_descent::gradient (optimizer/gradient_descent.cpp:42-60): the
    SR force F = <conj(O) E> - conj(<O>) <E> with its real part divided by
    real_factor."""
    F = _c128(F)
    return F.real / real_factor + 1j * F.imag


def optimize_tail(dw, lr, plugin=None):
    """abstract_optimizer::optimize tail (abstract_optimizer.cpp:157-176): None
    when max|dw| > 30 (no update), else the plugin's step or lr * dw."""
    if np.max(np.abs(dw)) > 30:
        return None
    return plugin.apply(dw, lr) if plugin is not None else dw * lr


def pf_context(machine, spins):
    n = machine.n
    inv = np.zeros(n * n, np.complex128)
    ctx = _PfCtx()
    ctx.inv = _p(inv, P_D)
    cm = machine.c_machine()
    s = np.ascontiguousarray(spins, dtype=np.uint32)
    lib().orc_pf_context(C.byref(cm), _p(s, P_U32), C.byref(ctx))
    return ctx, inv


def pf_update(machine, spins, flips, ctx):
    cm = machine.c_machine()
    s = np.ascontiguousarray(spins, dtype=np.uint32)
    f = np.ascontiguousarray(flips, dtype=np.int32)
    lib().orc_pf_update(C.byref(cm), _p(s, P_U32), _p(f, P_I), len(f), C.byref(ctx))


def pf_matrix(machine, spins):
    n = machine.n
    X = np.zeros(n * n, np.complex128)
    cm = machine.c_machine()
    s = np.ascontiguousarray(spins, dtype=np.uint32)
    lib().orc_pf_matrix(C.byref(cm), _p(s, P_U32), _p(X, P_D))
    return X.reshape(n, n).T.copy()  # column-major -> row-major numpy


def pfaffian10(A):
    """A: numpy (n, n) antisymmetric -> (mantissa, exp10)."""
    a = np.ascontiguousarray(np.asarray(A, dtype=np.complex128).T)  # column-major layout
    e = C.c_int()
    r = lib().orc_pfaffian10(a.shape[0], _p(a, P_D), C.byref(e))
    return complex(r.re, r.im), e.value

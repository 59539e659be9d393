"""Python binding of librbmnqs_b200.so (the C ABI in include/rbmnqs_b200.h).

A thin ctypes layer in the spirit of the reference's python_adapter: it
builds models, creates a GPU session and moves numpy arrays across the
boundary.  All compute runs in the CUDA library; if the library or a GPU is
missing, calls raise RbmNqsError instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "librbmnqs_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "rbmnqs_b200.h")

_LIB = None


class RbmNqsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rbmnqs error {code}: {msg}")
        self.code = code


ERR_MASSIVE_STEP = -4
ERR_NONFINITE = -5


class Config(C.Structure):
    _fields_ = [
        ("rbm_type", C.c_int32), ("alpha", C.c_int32), ("pfaffian", C.c_int32),
        ("pfaffian_symmetry", C.c_double), ("n_chains", C.c_int32), ("samples_per_chain", C.c_int32),
        ("warmup", C.c_int32), ("step", C.c_int32), ("bond_flips", C.c_double),
        ("pfaffian_refresh", C.c_int32), ("reinit_chains", C.c_int32), ("seed", C.c_uint64),
        ("lr", C.c_double * 3), ("reg1", C.c_double * 3), ("reg2", C.c_double * 3),
        ("deltareg1", C.c_double * 3), ("max_iterations", C.c_int32), ("rtol", C.c_double),
        ("precision", C.c_int32), ("n_updates", C.c_int32), ("gram", C.c_int32),
        ("proposal", C.c_int32), ("learned_steps", C.c_int32), ("learned_train", C.c_int32),
        ("learned_hidden", C.c_int32), ("learned_lr", C.c_double), ("solver", C.c_int32),
        ("optimizer_type", C.c_int32), ("sgd_real_factor", C.c_double), ("plugin", C.c_int32),
        ("adam_beta1", C.c_double), ("adam_beta2", C.c_double), ("adam_eps", C.c_double),
        ("mom_alpha", C.c_double), ("mom_dialup", C.c_double), ("heun_eps", C.c_double),
        ("sampler_type", C.c_int32), ("full_parallel_bits", C.c_int32),
    ]


class SampleStats(C.Structure):
    _fields_ = [("energy", C.c_double * 2), ("energy_var", C.c_double), ("energy_stddev", C.c_double),
                ("tau", C.c_double), ("acceptance", C.c_double), ("n_samples", C.c_int64),
                ("n_bins", C.c_int32), ("status", C.c_int32), ("learned_acceptance", C.c_double),
                ("learned_loss", C.c_double)]

    def as_dict(self):
        return dict(energy=complex(self.energy[0], self.energy[1]), var=self.energy_var,
                    stddev=self.energy_stddev, tau=self.tau, acceptance=self.acceptance,
                    n_samples=self.n_samples, n_bins=self.n_bins, status=self.status,
                    learned_acceptance=self.learned_acceptance, learned_loss=self.learned_loss)


class SrStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("residual", C.c_double),
                ("max_dw", C.c_double), ("lr", C.c_double), ("reg1", C.c_double), ("reg2", C.c_double),
                ("deltareg1", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


P_D = C.POINTER(C.c_double)
P_I = C.POINTER(C.c_int32)
P_U32 = C.POINTER(C.c_uint32)
P_I64 = C.POINTER(C.c_int64)
P_F = C.POINTER(C.c_float)
VP = C.c_void_p


def _declare(L):
    sig = {
        "rbmnqs_model_kitaev": [C.c_int32, C.c_int32, P_D, C.c_double, C.c_double, C.POINTER(VP)],
        "rbmnqs_model_toric": [C.c_int32, C.c_double, C.c_double, C.POINTER(VP)],
        "rbmnqs_model_add_hexagons": [VP],
        "rbmnqs_model_sizes": [VP, P_I, P_I, P_I, P_I],
        "rbmnqs_model_bonds": [VP, P_I],
        "rbmnqs_model_op": [VP, C.c_int32, P_I, P_I, P_D],
        "rbmnqs_model_symmetry": [VP, P_I, P_I, P_I, P_I],
        "rbmnqs_model_pfaffian_classes": [VP, C.c_double, P_I, P_I],
        "rbmnqs_model_destroy": [VP],
        "rbmnqs_config_default": [C.POINTER(Config)],
        "rbmnqs_create": [VP, C.POINTER(Config), C.POINTER(VP)],
        "rbmnqs_destroy": [VP],
        "rbmnqs_sizes": [VP, P_I, P_I, P_I, P_I, P_I],
        "rbmnqs_set_weights": [VP, P_D],
        "rbmnqs_get_weights": [VP, P_D],
        "rbmnqs_sample": [VP, C.POINTER(SampleStats)],
        "rbmnqs_optimize": [VP, C.POINTER(SrStats)],
        "rbmnqs_epoch": [VP, C.POINTER(SampleStats), C.POINTER(SrStats)],
        "rbmnqs_get_samples": [VP, P_D, P_D],
        "rbmnqs_get_sr": [VP, P_D, P_D, P_D, P_D],
        "rbmnqs_get_spins": [VP, P_U32],
        "rbmnqs_get_sample_configs": [VP, P_U32],
        "rbmnqs_set_spins": [VP, P_U32],
        "rbmnqs_eval_batch": [VP, P_U32, C.c_int32, P_D, P_D, P_D],
        "rbmnqs_log_psi_over_psi": [VP, P_U32, P_I, C.c_int32, C.c_int32, P_D],
        "rbmnqs_sr_solve": [VP, P_D, C.c_int32, P_D, C.c_double, P_D, P_D, C.c_double, C.c_double, C.c_double,
                            P_D, P_I, P_D],
        "rbmnqs_solve_info": [VP, P_I, P_D, P_I, P_D, P_I],
        "rbmnqs_log_open": [VP, C.c_char_p, C.c_int32],
        "rbmnqs_log_close": [VP],
        "rbmnqs_full_sample": [VP, P_D, P_D, P_D],
        "rbmnqs_get_observables": [VP, P_D],
        "rbmnqs_full_state": [VP, P_D],
        "rbmnqs_model_ground_state": [VP, C.c_int32, C.c_double, C.c_uint64, P_D, P_I, P_D],
        "rbmnqs_set_sweep_shape": [VP, C.c_int32, C.c_int32],
        "rbmnqs_get_sweep_shape": [VP, P_I, P_I],
        "rbmnqs_timing": [VP, P_D, P_I64, C.c_int32],
        "rbmnqs_timing_reset": [VP, C.c_int32],
        "rbmnqs_graph_kernels": [VP, P_I],
        "rbmnqs_autotune": [VP, C.c_int32, P_I, P_I, P_D],
        "rbmnqs_autotune_sr": [VP, P_I, P_I, P_D],
        "rbmnqs_save": [VP, C.c_char_p],
        "rbmnqs_load": [VP, C.c_char_p],
        "rbmnqs_n_updates": [VP, P_I64],
        "rbmnqs_batch_create": [C.POINTER(VP), C.c_int32, C.POINTER(VP)],
        "rbmnqs_batch_epoch": [VP, VP, VP],
        "rbmnqs_batch_graph_kernels": [VP, P_I],
        "rbmnqs_batch_destroy": [VP],
        "rbmnqs_mlp_create": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(VP)],
        "rbmnqs_mlp_n_params": [VP, C.POINTER(C.c_int64)],
        "rbmnqs_mlp_set_params": [VP, P_F],
        "rbmnqs_mlp_get_params": [VP, P_F],
        "rbmnqs_mlp_init": [VP, C.c_float, C.c_uint64],
        "rbmnqs_mlp_forward": [VP, P_U32, C.c_int32, P_F],
        "rbmnqs_mlp_train_step": [VP, P_U32, P_U32, C.c_int32, C.c_float, C.c_int32, P_F, P_F],
        "rbmnqs_mlp_train_step_soft": [VP, P_U32, P_F, C.c_int32, C.c_float, C.c_int32, P_F, P_F],
        "rbmnqs_mlp_intermediate": [VP, C.c_int32, C.c_int32, P_F, P_I],
        "rbmnqs_mlp_destroy": [VP],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = None if name in ("rbmnqs_model_destroy", "rbmnqs_destroy", "rbmnqs_batch_destroy",
                                     "rbmnqs_mlp_destroy") else C.c_int
    L.rbmnqs_sr_solve_noalloc.argtypes = [VP, C.c_int32, C.c_int32, C.c_int32, VP, C.c_double, VP, VP, C.c_double,
                                          C.c_double, C.c_double, VP, C.c_int32, C.c_double, VP, P_I, P_D]
    L.rbmnqs_sr_solve_noalloc.restype = C.c_int
    L.rbmnqs_test_fault.argtypes = [C.c_int32]
    L.rbmnqs_test_fault.restype = C.c_int
    L.rbmnqs_probe_mufu.argtypes = [C.c_int32, P_D]
    L.rbmnqs_probe_mufu.restype = C.c_int
    L.rbmnqs_last_error.restype = C.c_char_p
    L.rbmnqs_stream.argtypes = [VP]
    L.rbmnqs_stream.restype = VP
    L.rbmnqs_batch_stream.argtypes = [VP]
    L.rbmnqs_batch_stream.restype = VP


def lib():
    """Load the in-tree library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBPATH):
            raise RbmNqsError(-6, f"{LIBPATH} not built (run __graft_entry__.build())")
        _LIB = C.CDLL(LIBPATH)
        _declare(_LIB)
    return _LIB


def test_fault(kind):
    """rbmnqs_test_fault: 0 off, 1 cooperative-solve barriers never complete,
    2 the proposal network's GEMM copies are never issued (bounded waits run
    out and the calls report RBMNQS_ERR_CUDA)."""
    _ck(lib().rbmnqs_test_fault(kind))


def probe_mufu(iters=4096):
    """Measured MUFU (ex2/lg2/sin/cos) operations per second of this GPU."""
    v = C.c_double()
    _ck(lib().rbmnqs_probe_mufu(iters, C.byref(v)))
    return v.value


def sr_solve_noalloc(O_ptr, N, n_params, n_neural, d_ptr, norm, F_ptr, x_ptr, r1, r2, rd, diag_ptr,
                     max_iterations=0, rtol=0.0, stream=0):
    """rbmnqs_sr_solve_noalloc on caller-owned device buffers (raw device
    addresses).  The solve allocates no device memory; x is updated in
    place.  Returns (iterations, residual)."""
    it, rs = C.c_int32(), C.c_double()
    _ck(lib().rbmnqs_sr_solve_noalloc(O_ptr, N, n_params, n_neural, d_ptr, norm, F_ptr, x_ptr, r1, r2, rd, diag_ptr,
                                      max_iterations, rtol, stream, C.byref(it), C.byref(rs)))
    return it.value, rs.value


def header_symbols():
    """Function names declared in include/rbmnqs_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(rbmnqs_[a-z_0-9]+)\s*\(", txt)))


def _ck(rc):
    if rc != 0:
        raise RbmNqsError(rc, lib().rbmnqs_last_error().decode())
    return rc


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


class Model:
    """A lattice + Hamiltonian (model::kitaev / model::toric)."""

    def __init__(self, handle, kind):
        self._h = handle
        self.kind = kind
        n, o, b, ob = (C.c_int32() for _ in range(4))
        _ck(lib().rbmnqs_model_sizes(self._h, C.byref(n), C.byref(o), C.byref(b), C.byref(ob)))
        self.n, self.n_ops, self.n_bonds, self.n_obs = n.value, o.value, b.value, ob.value

    @staticmethod
    def kitaev(n_cells, n_cells_b=-1, J=(-1.0, -1.0, -1.0), h=0.0, symmetry=0.5):
        out = VP()
        Jv = np.asarray(J, dtype=np.float64)
        _ck(lib().rbmnqs_model_kitaev(n_cells, n_cells_b, _p(Jv, P_D), h, symmetry, C.byref(out)))
        return Model(out, "kitaev")

    @staticmethod
    def toric(n_cells, J=-1.0, symmetry=1.0):
        out = VP()
        _ck(lib().rbmnqs_model_toric(n_cells, J, symmetry, C.byref(out)))
        return Model(out, "toric")

    def ground_state(self, max_iter=400, tol=1e-13, seed=1, vector=False):
        """Exact diagonalisation on the GPU (Lanczos, n <= 28): (E0,
        iterations[, psi over the 2^n states])."""
        e, it = C.c_double(), C.c_int32()
        psi = np.zeros(1 << self.n, np.complex128) if vector else None
        _ck(lib().rbmnqs_model_ground_state(self._h, max_iter, tol, seed, C.byref(e), C.byref(it),
                                            _p(psi.view(np.float64), P_D) if vector else None))
        return (e.value, it.value, psi) if vector else (e.value, it.value)

    def bonds(self):
        a = np.zeros((self.n_bonds, 3), np.int32)
        _ck(lib().rbmnqs_model_bonds(self._h, _p(a, P_I)))
        return a

    def op(self, o):
        k = C.c_int32()
        acts = np.zeros(6, np.int32)
        _ck(lib().rbmnqs_model_op(self._h, o, C.byref(k), _p(acts, P_I), None))
        d = 1 << k.value
        mat = np.zeros(2 * d * d, np.float64)
        _ck(lib().rbmnqs_model_op(self._h, o, None, None, _p(mat, P_D)))
        return k.value, acts[: k.value].copy(), mat.view(np.complex128).reshape(d, d)

    def symmetry(self):
        S, nvb = C.c_int32(), C.c_int32()
        _ck(lib().rbmnqs_model_symmetry(self._h, C.byref(S), C.byref(nvb), None, None))
        perm = np.zeros(S.value * self.n, np.int32)
        basis = np.zeros(nvb.value, np.int32)
        _ck(lib().rbmnqs_model_symmetry(self._h, None, None, _p(perm, P_I), _p(basis, P_I)))
        return perm.reshape(S.value, self.n), basis

    def pfaffian_classes(self, symmetry=0.5):
        """(bs [n, n] signed 1-based pair classes, n_indep) of pfaffian.cpp:31-85."""
        ni = C.c_int32()
        _ck(lib().rbmnqs_model_pfaffian_classes(self._h, symmetry, None, C.byref(ni)))
        bs = np.zeros(self.n * self.n, np.int32)
        _ck(lib().rbmnqs_model_pfaffian_classes(self._h, symmetry, _p(bs, P_I), C.byref(ni)))
        return bs.reshape(self.n, self.n), ni.value

    def add_hexagons(self):
        _ck(lib().rbmnqs_model_add_hexagons(self._h))
        self.__init__(self._h, self.kind)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.rbmnqs_model_destroy(self._h)
            self._h = None


def default_config(**kw):
    c = Config()
    _ck(lib().rbmnqs_config_default(C.byref(c)))
    for k, v in kw.items():
        if isinstance(getattr(c, k), C.Array):
            vv = list(v) if hasattr(v, "__len__") else [v, v, 1.0]
            for i in range(3):
                getattr(c, k)[i] = vv[i]
        else:
            setattr(c, k, v)
    return c


class Session:
    """GPU sampler + SR optimizer for one machine on one model."""

    def __init__(self, model, cfg):
        self.model = model
        self.cfg = cfg
        h = VP()
        _ck(lib().rbmnqs_create(model._h, C.byref(cfg), C.byref(h)))
        self._h = h
        P, Pn, nvb, nh, S = (C.c_int32() for _ in range(5))
        _ck(lib().rbmnqs_sizes(h, C.byref(P), C.byref(Pn), C.byref(nvb), C.byref(nh), C.byref(S)))
        self.n_params, self.n_neural, self.n_vb, self.n_hidden, self.n_symm = \
            P.value, Pn.value, nvb.value, nh.value, S.value
        self.n = model.n
        # samples per epoch: 2^n states for full enumeration
        self.N = (1 << model.n) if cfg.sampler_type == 1 else cfg.n_chains * cfg.samples_per_chain

    def close(self):
        if getattr(self, "_h", None):
            lib().rbmnqs_destroy(self._h)
            self._h = None

    __del__ = close

    def set_weights(self, w):
        w = _c128(w)
        assert w.shape == (self.n_params,)
        _ck(lib().rbmnqs_set_weights(self._h, _p(w.view(np.float64), P_D)))

    def get_weights(self):
        w = np.zeros(self.n_params, np.complex128)
        _ck(lib().rbmnqs_get_weights(self._h, _p(w.view(np.float64), P_D)))
        return w

    def sample(self):
        s = SampleStats()
        _ck(lib().rbmnqs_sample(self._h, C.byref(s)))
        return s.as_dict()

    def optimize(self):
        o = SrStats()
        _ck(lib().rbmnqs_optimize(self._h, C.byref(o)))
        return o.as_dict()

    def epoch(self):
        s, o = SampleStats(), SrStats()
        _ck(lib().rbmnqs_epoch(self._h, C.byref(s), C.byref(o)))
        return s.as_dict(), o.as_dict()

    def samples(self, with_O=True):
        E = np.zeros(self.N, np.complex128)
        O = np.zeros((self.N, self.n_params), np.complex128) if with_O else None
        _ck(lib().rbmnqs_get_samples(self._h, _p(E.view(np.float64), P_D),
                                     _p(O.view(np.float64), P_D) if with_O else None))
        return E, O

    def sample_configs(self):
        """configurations of the last epoch's samples [N][4] (the order of samples())"""
        c = np.zeros((self.N, 4), np.uint32)
        _ck(lib().rbmnqs_get_sample_configs(self._h, _p(c, P_U32)))
        return c

    def sr_moments(self, with_S=None):
        """d, F, diag and (when formed: n_params <= 2048, or with_S) S."""
        P = self.n_params
        if with_S is None:
            with_S = P <= 2048
        d = np.zeros(P, np.complex128)
        F = np.zeros(P, np.complex128)
        diag = np.zeros(P, np.float64)
        S = np.zeros((P, P), np.complex128) if with_S else None
        _ck(lib().rbmnqs_get_sr(self._h, _p(d.view(np.float64), P_D), _p(F.view(np.float64), P_D),
                                _p(diag, P_D), _p(S.view(np.float64), P_D) if with_S else None))
        return d, F, diag, S

    def spins(self):
        s = np.zeros((self.cfg.n_chains, 4), np.uint32)
        _ck(lib().rbmnqs_get_spins(self._h, _p(s, P_U32)))
        return s

    def set_spins(self, s):
        s = np.ascontiguousarray(s, dtype=np.uint32)
        _ck(lib().rbmnqs_set_spins(self._h, _p(s, P_U32)))

    def eval_batch(self, spins, logpsi=True, eloc=True, O=True):
        spins = np.ascontiguousarray(spins, dtype=np.uint32)
        B = spins.shape[0]
        lp = np.zeros(B, np.complex128) if logpsi else None
        el = np.zeros(B, np.complex128) if eloc else None
        Od = np.zeros((B, self.n_params), np.complex128) if O else None
        _ck(lib().rbmnqs_eval_batch(self._h, _p(spins, P_U32), B,
                                    _p(lp.view(np.float64), P_D) if logpsi else None,
                                    _p(el.view(np.float64), P_D) if eloc else None,
                                    _p(Od.view(np.float64), P_D) if O else None))
        return lp, el, Od

    def log_psi_over_psi(self, spins, flips):
        spins = np.ascontiguousarray(spins, dtype=np.uint32)
        flips = np.ascontiguousarray(flips, dtype=np.int32)
        B, m = flips.shape
        out = np.zeros(B, np.complex128)
        _ck(lib().rbmnqs_log_psi_over_psi(self._h, _p(spins, P_U32), _p(flips, P_I), m, B,
                                          _p(out.view(np.float64), P_D)))
        return out

    def sr_solve(self, O, d, F, x0, r1, r2, rd, diag, norm=None):
        O = _c128(O)
        N = O.shape[0]
        d, F = _c128(d), _c128(F)
        x = _c128(x0).copy()
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        it, rs = C.c_int32(), C.c_double()
        _ck(lib().rbmnqs_sr_solve(self._h, _p(O.view(np.float64), P_D), N, _p(d.view(np.float64), P_D),
                                  float(N if norm is None else norm), _p(F.view(np.float64), P_D),
                                  _p(x.view(np.float64), P_D), r1, r2, rd, _p(diag, P_D), C.byref(it),
                                  C.byref(rs)))
        return x, it.value, rs.value

    def log_open(self, name, force=False):
        """Training log <name>.log (logger.cpp:31-74): one line per applied
        update, appended to an existing file unless force."""
        _ck(lib().rbmnqs_log_open(self._h, str(name).encode(), int(bool(force))))

    def log_close(self):
        _ck(lib().rbmnqs_log_close(self._h))

    def solve_info(self):
        """The last SR solve's outcome (minresqlp_adapter getItn / getRnorm /
        getAcond and the istop of apply): {"iterations", "residual",
        "istop", "acond", "qlp"}; istop, acond and qlp are 0 unless the
        solver is minresqlp."""
        it, rs, ist, ac, nq = C.c_int32(), C.c_double(), C.c_int32(), C.c_double(), C.c_int32()
        _ck(lib().rbmnqs_solve_info(self._h, C.byref(it), C.byref(rs), C.byref(ist), C.byref(ac), C.byref(nq)))
        return {"iterations": it.value, "residual": rs.value, "istop": ist.value, "acond": ac.value,
                "qlp": nq.value}

    def observables(self):
        """Evaluation mode: [n_obs] rows of (Re <O>, Im <O>, stddev, tau) over the
        last epoch's samples (hexagon W_p after Model.add_hexagons)."""
        v = np.zeros(4 * self.model.n_obs, np.float64)
        _ck(lib().rbmnqs_get_observables(self._h, _p(v, P_D)))
        return v.reshape(-1, 4)

    def set_sweep_shape(self, warps_per_block=0, chains_per_warp=1):
        _ck(lib().rbmnqs_set_sweep_shape(self._h, warps_per_block, chains_per_warp))

    def sweep_shape(self):
        w, c = C.c_int32(), C.c_int32()
        _ck(lib().rbmnqs_get_sweep_shape(self._h, C.byref(w), C.byref(c)))
        return w.value, c.value

    def full_state(self):
        """Full enumeration (sampler_type 1): the normalised psi over all 2^n
        states, indexed by the state number, of the last sample."""
        psi = np.zeros(1 << self.model.n, np.complex128)
        _ck(lib().rbmnqs_full_state(self._h, _p(psi.view(np.float64), P_D)))
        return psi

    def full_sample(self):
        P = self.n_params
        em = np.zeros(1, np.complex128)
        d = np.zeros(P, np.complex128)
        dh = np.zeros(P, np.complex128)
        _ck(lib().rbmnqs_full_sample(self._h, _p(em.view(np.float64), P_D), _p(d.view(np.float64), P_D),
                                     _p(dh.view(np.float64), P_D)))
        return em[0], d, dh

    def timing(self, n=6):
        ms = np.zeros(n, np.float64)
        cnt = np.zeros(n, np.int64)
        _ck(lib().rbmnqs_timing(self._h, _p(ms, P_D), _p(cnt, P_I64), n))
        return ms, cnt

    def timing_reset(self, enable=True):
        _ck(lib().rbmnqs_timing_reset(self._h, 1 if enable else 0))

    def graph_kernels(self):
        n = C.c_int32()
        _ck(lib().rbmnqs_graph_kernels(self._h, C.byref(n)))
        return n.value

    def stream(self):
        return lib().rbmnqs_stream(self._h)

    def save(self, path):
        """The reference's .rbm checkpoint (rbm_base::save)."""
        _ck(lib().rbmnqs_save(self._h, str(path).encode()))

    def load(self, path):
        _ck(lib().rbmnqs_load(self._h, str(path).encode()))

    def n_updates(self):
        n = C.c_int64()
        _ck(lib().rbmnqs_n_updates(self._h, C.byref(n)))
        return n.value

    def autotune(self, sweeps=4):
        """Launch-shape autotuning (rbmnqs_autotune): (sampler warps per
        block, evaluation warps per block, sampler ms for `sweeps` sweeps)."""
        sw, ew, ms = C.c_int32(), C.c_int32(), C.c_double()
        _ck(lib().rbmnqs_autotune(self._h, sweeps, C.byref(sw), C.byref(ew), C.byref(ms)))
        return sw.value, ew.value, ms.value

    def autotune_sr(self):
        """Solver-stage autotuning (rbmnqs_autotune_sr) on the current O:
        (Gram split count or 0, CG kernel 0 cluster / 1 cooperative / -1,
        best Gram + CG ms)."""
        gs, ck_, ms = C.c_int32(), C.c_int32(), C.c_double()
        _ck(lib().rbmnqs_autotune_sr(self._h, C.byref(gs), C.byref(ck_), C.byref(ms)))
        return gs.value, ck_.value, ms.value


class Batch:
    """Independent sessions advanced together: one CUDA-graph launch runs the
    epoch of every session (rbmnqs_batch_*)."""

    def __init__(self, sessions):
        self.sessions = list(sessions)
        arr = (VP * len(self.sessions))(*[x._h for x in self.sessions])
        h = VP()
        _ck(lib().rbmnqs_batch_create(arr, len(self.sessions), C.byref(h)))
        self._h = h

    def epoch(self):
        n = len(self.sessions)
        s, o = (SampleStats * n)(), (SrStats * n)()
        _ck(lib().rbmnqs_batch_epoch(self._h, C.cast(s, VP), C.cast(o, VP)))
        return [x.as_dict() for x in s], [x.as_dict() for x in o]

    def graph_kernels(self):
        k = C.c_int32()
        _ck(lib().rbmnqs_batch_graph_kernels(self._h, C.byref(k)))
        return k.value

    def stream(self):
        return lib().rbmnqs_batch_stream(self._h)

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.rbmnqs_batch_destroy(self._h)
            self._h = None


class ProposalNet:
    """The proposal network on the GPU (rbmnqs_mlp_*): BF16 weights and
    activations, FP32 accumulation, tcgen05 forward and backward, Adam."""

    def __init__(self, n_in=128, h1=256, h2=256, n_out=128, max_batch=16384):
        h = VP()
        _ck(lib().rbmnqs_mlp_create(n_in, h1, h2, n_out, max_batch, C.byref(h)))
        self._h = h
        self.dims = (n_in, h1, h2, n_out)
        n = C.c_int64()
        _ck(lib().rbmnqs_mlp_n_params(self._h, C.byref(n)))
        self.n_params = n.value

    def init(self, std=0.02, seed=0):
        _ck(lib().rbmnqs_mlp_init(self._h, std, seed))

    def set_params(self, flat):
        a = np.ascontiguousarray(flat, dtype=np.float32)
        assert a.size == self.n_params
        _ck(lib().rbmnqs_mlp_set_params(self._h, _p(a, P_F)))

    def get_params(self):
        a = np.zeros(self.n_params, np.float32)
        _ck(lib().rbmnqs_mlp_get_params(self._h, _p(a, P_F)))
        return a

    def forward(self, spins):
        s = np.ascontiguousarray(spins, dtype=np.uint32)
        out = np.zeros((s.shape[0], self.dims[3]), np.float32)
        _ck(lib().rbmnqs_mlp_forward(self._h, _p(s, P_U32), s.shape[0], _p(out, P_F)))
        return out

    def train_step(self, spins, targets, lr=1e-3, apply=True, grads=True):
        s = np.ascontiguousarray(spins, dtype=np.uint32)
        t = np.ascontiguousarray(targets, dtype=np.uint32)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32) if grads else None
        _ck(lib().rbmnqs_mlp_train_step(self._h, _p(s, P_U32), _p(t, P_U32), s.shape[0], lr, 1 if apply else 0,
                                        C.byref(loss), _p(g, P_F)))
        return loss.value, g

    def train_step_soft(self, spins, targets, lr=1e-3, apply=True, grads=True):
        """One step on the softmax cross entropy against soft targets [B][n_out]."""
        s = np.ascontiguousarray(spins, dtype=np.uint32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32) if grads else None
        _ck(lib().rbmnqs_mlp_train_step_soft(self._h, _p(s, P_U32), _p(t, P_F), s.shape[0], lr, 1 if apply else 0,
                                             C.byref(loss), _p(g, P_F)))
        return loss.value, g

    def intermediate(self, which, B):
        c = C.c_int32()
        _ck(lib().rbmnqs_mlp_intermediate(self._h, which, B, None, C.byref(c)))
        out = np.zeros((B, c.value), np.float32)
        _ck(lib().rbmnqs_mlp_intermediate(self._h, which, B, _p(out, P_F), C.byref(c)))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.rbmnqs_mlp_destroy(self._h)
            self._h = None


def mlp_unflatten(flat, dims):
    """flat [W1, b1, W2, b2, W3, b3] -> dict of float64 arrays (oracle layout)."""
    p, o = {}, 0
    for l in range(3):
        r, c = dims[l + 1], dims[l]
        p[f"W{l + 1}"] = np.asarray(flat[o:o + r * c], np.float64).reshape(r, c)
        o += r * c
        p[f"b{l + 1}"] = np.asarray(flat[o:o + r], np.float64)
        o += r
    return p


def mlp_flatten(p):
    return np.concatenate([np.ravel(p[k]) for k in ("W1", "b1", "W2", "b2", "W3", "b3")]).astype(np.float32)

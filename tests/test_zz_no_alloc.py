"""The allocation-free SR solve (rbmnqs_sr_solve_noalloc) against the
allocating one (rbmnqs_sr_solve).

Callers that cannot allocate device memory -- code inside a runtime that owns
all device memory through its own pool, latency-critical loops that cannot
take cudaMalloc's implicit synchronisation -- get the same solve with the
working memory in a fixed array inside the library.  This file is collected
last so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

TOL = 1e-10  # FP64 path tolerance used by the parity tests


def _system():
    rng = np.random.default_rng(11)
    om = O.Model.kitaev(4)
    mach = O.Machine(om, "symmetry", 4, symm=0.5).init_random(rng, 0.05)
    cfg = rbmnqs.default_config(rbm_type=1, alpha=4, n_chains=64, samples_per_chain=8, warmup=4, bond_flips=0.5,
                                seed=3, precision=1)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(4, symmetry=0.5), cfg)
    s.set_weights(mach.params())
    s.sample()
    E, Om = s.samples()
    d, F, diag = O.sr_moments(Om, E)
    x0 = 1e-3 * (rng.normal(size=mach.n_params) + 1j * rng.normal(size=mach.n_params))
    return s, Om, d, F, diag, x0


def test_noalloc_solve_matches_allocating_solve_twice():
    import torch

    s, Om, d, F, diag, x0 = _system()
    N, P = Om.shape
    r1, r2, rd = 0.9, 1e-4, 1e-2
    x_ref, it_ref, _ = s.sr_solve(Om, d, F, x0, r1, r2, rd, diag)

    dev = torch.device("cuda")

    def on_gpu(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).to(dev)

    tO, td, tF, tdiag = on_gpu(Om), on_gpu(d), on_gpu(F), on_gpu(diag)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # the second call reuses the array the first one left behind
        tx = on_gpu(x0)
        torch.cuda.synchronize()
        it, rs = rbmnqs.sr_solve_noalloc(tO.data_ptr(), N, P, s.n_neural, td.data_ptr(), float(N), tF.data_ptr(),
                                         tx.data_ptr(), r1, r2, rd, tdiag.data_ptr(), stream=stream)
        x = tx.cpu().numpy().view(np.complex128)
        err = np.max(np.abs(x - x_ref)) / max(1.0, np.max(np.abs(x_ref)))
        assert err < TOL, (call, err)
        assert abs(it - it_ref) <= max(2, it_ref // 20), (call, it, it_ref)
        assert rs < 1e-16


def test_noalloc_rejects_too_many_params():
    with pytest.raises(rbmnqs.RbmNqsError) as e:
        rbmnqs.sr_solve_noalloc(1, 16, 300, 300, 1, 16.0, 1, 1, 0.9, 1e-4, 0.0, 1)
    assert e.value.code == -1
    assert "256" in str(e.value)

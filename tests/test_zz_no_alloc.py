"""The allocation-free SR solve (rbmnqs_sr_solve_noalloc) against the
allocating one (rbmnqs_sr_solve).

Callers that cannot allocate device memory -- code inside a runtime that owns
all device memory through its own pool, latency-critical loops that cannot
take cudaMalloc's implicit synchronisation -- get the same solve with the
working memory in a fixed array inside the library.  The cases cover a small
parameter count and one close to the array's limit (where the CG status sits
at the end of the array and the CG needs more than 48 KB of shared memory),
the single-split Gram taken for very few samples, and a smaller solve after a
larger one (the array then holds the larger solve's leftovers).  This file is
collected last so that a run stopping at the first failure has run every
other test."""
import numpy as np
import pytest

import oracle as O
import rbmnqs

pytestmark = pytest.mark.gpu

TOL = 1e-10  # FP64 path tolerance used by the parity tests

# (n_cells of the Kitaev lattice, alpha) -> n_params of the symmetric RBM:
# (4, 4) -> 133, (3, 13) -> 248 (close to RBMNQS_NOALLOC_MAX_PARAMS = 256)
CASES = {"small": (4, 4), "near_limit": (3, 13)}


def _system(case, N, seed):
    n_cells, alpha = CASES[case]
    cfg = rbmnqs.default_config(rbm_type=1, alpha=alpha, n_chains=32, samples_per_chain=1, warmup=1,
                                bond_flips=0.5, seed=3, precision=1)
    s = rbmnqs.Session(rbmnqs.Model.kitaev(n_cells, symmetry=0.5), cfg)
    P = s.n_params
    rng = np.random.default_rng(seed)
    # a synthetic O store and local energies of N samples: the solve sees
    # only these arrays, not how they were sampled
    Om = rng.normal(size=(N, P)) + 1j * rng.normal(size=(N, P))
    E = rng.normal(size=N) + 1j * rng.normal(size=N)
    d, F, diag = O.sr_moments(Om, E)
    x0 = 1e-3 * (rng.normal(size=P) + 1j * rng.normal(size=P))
    return s, Om, d, F, diag, x0


def _noalloc(s, Om, d, F, diag, x0, r1, r2, rd):
    import torch

    dev = torch.device("cuda")

    def on_gpu(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).to(dev)

    N, P = Om.shape
    tO, td, tF, tdiag, tx = on_gpu(Om), on_gpu(d), on_gpu(F), on_gpu(diag), on_gpu(x0)
    torch.cuda.synchronize()
    it, rs = rbmnqs.sr_solve_noalloc(tO.data_ptr(), N, P, s.n_neural, td.data_ptr(), float(N), tF.data_ptr(),
                                     tx.data_ptr(), r1, r2, rd, tdiag.data_ptr(),
                                     stream=torch.cuda.current_stream().cuda_stream)
    return tx.cpu().numpy().view(np.complex128), it, rs


def _check(s, Om, d, F, diag, x0, tag):
    r1, r2, rd = 0.9, 1e-4, 1e-2
    x_ref, it_ref, _ = s.sr_solve(Om, d, F, x0, r1, r2, rd, diag)
    x, it, rs = _noalloc(s, Om, d, F, diag, x0, r1, r2, rd)
    err = np.max(np.abs(x - x_ref)) / max(1.0, np.max(np.abs(x_ref)))
    assert err < TOL, (tag, err)
    assert abs(it - it_ref) <= max(2, it_ref // 20), (tag, it, it_ref)
    assert rs < 1e-16, (tag, rs)


@pytest.mark.parametrize("case", ["small", "near_limit"])
@pytest.mark.parametrize("N", [16, 512])
def test_noalloc_solve_matches_allocating_solve_twice(case, N):
    sysm = _system(case, N, seed=11)
    for call in range(2):  # the second call reuses the array the first one left behind
        _check(*sysm, tag=(case, N, call))


def test_noalloc_smaller_solve_after_larger_one():
    big = _system("near_limit", 512, seed=21)
    small = _system("small", 512, seed=22)
    _check(*big, tag="near_limit")
    _check(*small, tag="small after near_limit")


def test_noalloc_rejects_too_many_params():
    with pytest.raises(rbmnqs.RbmNqsError) as e:
        rbmnqs.sr_solve_noalloc(1, 16, 300, 300, 1, 16.0, 1, 1, 0.9, 1e-4, 0.0, 1)
    assert e.value.code == -1
    assert "256" in str(e.value)


def test_noalloc_rejects_negative_max_iterations():
    with pytest.raises(rbmnqs.RbmNqsError) as e:
        rbmnqs.sr_solve_noalloc(1, 16, 100, 100, 1, 16.0, 1, 1, 0.9, 1e-4, 0.0, 1, max_iterations=-1)
    assert e.value.code == -1
    assert "max_iterations" in str(e.value)

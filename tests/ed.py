"""Exact diagonalisation helpers for the tests (scipy), mirroring the
reference's python_adapter/rbm/__init__.py:16-41 convention: site i <-> bit i
of the basis index, sigma^z|0> = +|0>, <x|H|y> = op[loc(x)][loc(y)]."""
import numpy as np
import scipy.sparse as sp


def hamiltonian(model):
    n = model.n
    N = 1 << n
    x = np.arange(N, dtype=np.int64)
    rows, cols, vals = [], [], []
    for o in range(model.n_ops):
        k = int(model.k[o])
        sites = model.sites[o, :k]
        M = model.op_matrix(o)
        loc = np.zeros(N, dtype=np.int64)
        for i, s in enumerate(sites):
            loc |= ((x >> int(s)) & 1) << i
        base = x.copy()
        for s in sites:
            base &= ~(np.int64(1) << int(s))
        for c in range(1 << k):
            v = M[loc, c]
            nz = v != 0
            if not nz.any():
                continue
            y = base.copy()
            for i, s in enumerate(sites):
                if (c >> i) & 1:
                    y |= np.int64(1) << int(s)
            rows.append(x[nz])
            cols.append(y[nz])
            vals.append(v[nz])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


def ground_state(H):
    from scipy.sparse.linalg import eigsh
    w, v = eigsh(H, k=1, which="SA")
    return w[0], v[:, 0]

"""Integral inputs for the selected-CI path.

``synthetic_integrals`` is the seeded integral recipe of the benchmark
workloads: orbital energies eps_p = -1.5 + 2.5 p/(n-1) Eh, one-electron
h_pq = eps_p delta_pq plus a symmetric off-diagonal N(0, 0.02^2), and
two-electron (pq|rs) = sum_{L<2n} B^L_pq B^L_rs with every B^L symmetric and
entries N(0, (0.3 exp(-L/n))^2) -- 8-fold symmetric and positive
semi-definite; core energy 0.

``fcidump_fill`` expands FCIDUMP lines into T and V with the same 8-fold fill
as the reference reader (src/macis/fcidump.cxx:141-174).

Both return flat column-major float64 arrays, T(p,q) = T[p + q n] and
V(p,q,r,s) = V[p + q n + r n^2 + s n^3] (include/macis/types.hpp:22-33).
"""
import numpy as np


def synthetic_integrals(norb, seed=0):
    n = int(norb)
    rng = np.random.default_rng(seed)
    eps = -1.5 + 2.5 * np.arange(n) / max(n - 1, 1)
    off = np.triu(rng.normal(0.0, 0.02, size=(n, n)), 1)
    T = off + off.T + np.diag(eps)
    B = np.empty((2 * n, n, n))
    for L in range(2 * n):
        M = rng.normal(0.0, 0.3 * np.exp(-L / n), size=(n, n))
        up = np.triu(M)
        B[L] = up + np.triu(M, 1).T
    Bf = B.reshape(2 * n, n * n)          # symmetric, so C/F order agree
    Vmat = Bf.T @ Bf                      # (pq, rs)
    Vmat = 0.5 * (Vmat + Vmat.T)          # exact (pq|rs) = (rs|pq)
    return (np.ascontiguousarray(T.ravel(order="F")),
            np.ascontiguousarray(Vmat.ravel(order="F")))


def fcidump_fill(idx, val, norb=None):
    """T, V, E_core from FCIDUMP lines (1-based p q r s, value)."""
    idx = np.asarray(idx, dtype=np.int64)
    val = np.asarray(val, dtype=np.float64)
    n = int(norb if norb is not None else idx.max())
    T = np.zeros((n, n), order="F")
    V = np.zeros((n, n, n, n), order="F")
    ecore = 0.0
    for (p, q, r, s), v in zip(idx, val):
        if p and q and r and s:
            p, q, r, s = p - 1, q - 1, r - 1, s - 1
            for a, b, c, d in ((p, q, r, s), (p, q, s, r), (q, p, r, s),
                               (q, p, s, r), (r, s, p, q), (s, r, p, q),
                               (r, s, q, p), (s, r, q, p)):
                V[a, b, c, d] = v
        elif p and q:
            T[p - 1, q - 1] = v
            T[q - 1, p - 1] = v
        elif not (p or q or r or s):
            ecore = v
    return (np.ascontiguousarray(T.ravel(order="F")),
            np.ascontiguousarray(V.ravel(order="F")), ecore)

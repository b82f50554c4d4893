"""Davidson eigensolver and selected-CI driver on the B200.

* ``SparseMatrixOperator`` -- include/macis/solvers/davidson.hpp:29-59
* ``diagonal_guess``       -- davidson.hpp:61-68
* ``davidson``             -- davidson.hpp:128-225 (FP64 or mixed precision)
* ``selected_ci_diag``     -- include/macis/solvers/selected_ci_diag.hpp:
  125-206 (H build + Davidson, logged under the reference logger names)
"""
import ctypes as C
import logging
import time

import numpy as np

from . import _lib
from ._lib import ECAPACITY, ENOMEM, LIB, MacisError, check
from .hamiltonian import (DeviceCSR, MatrixFreeHamiltonian,
                          make_csr_hamiltonian)

__all__ = ["SparseMatrixOperator", "diagonal_guess", "davidson",
           "selected_ci_diag", "small_syev", "davidson_stats", "FP64",
           "MIXED"]

FP64 = "fp64"
MIXED = "mixed"


class SparseMatrixOperator:
    """H.X hook of the Davidson solver: operator_action(m, alpha, V, LDV,
    beta, AV, LDAV) with column-major host blocks."""

    def __init__(self, H):
        self.H = H

    def operator_action(self, m, alpha, V, LDV, beta, AV, LDAV):
        V = np.asarray(V, dtype=np.float64)
        check(LIB.macis_b200_spmv(self.H.handle, m, alpha, V.ctypes.data, LDV,
                                  beta, AV.ctypes.data, LDAV, 0))


def diagonal_guess(N, A, X):
    """Unit vector at the first minimum of the diagonal."""
    D = A.diagonal()
    X[:] = 0.0
    X[int(np.argmin(D))] = 1.0


def davidson(N, max_m, op, D, tol, X, use_guess=True, restart_keep=0,
             max_iter=0):
    """Lowest eigenpair of op.H (a DeviceCSR or a MatrixFreeHamiltonian); X
    holds the guess and receives the Ritz vector. Returns (iterations, eigenvalue). D (the diagonal) is taken
    from the matrix itself, as extract_diagonal_elements would give it.
    restart_keep = 0 is the reference solver (at most max_m basis vectors);
    restart_keep > 0 adds a thick restart keeping that many Ritz vectors,
    bounded by max_iter iterations (0: unbounded).
    Raises RuntimeError("Davidson Did Not Converge!") like the reference."""
    H = op.H if isinstance(op, SparseMatrixOperator) else op
    if H.m != N:
        raise RuntimeError("Davidson: dimension mismatch")
    xs = np.ascontiguousarray(X, dtype=np.float64)
    E = C.c_double()
    it = C.c_int64()
    o = _lib.DavidsonOptsC(int(max_m), float(tol), int(use_guess),
                           int(restart_keep), int(max_iter))
    from .hamiltonian import MatrixFreeHamiltonian
    fn = (LIB.macis_b200_hop_davidson if isinstance(H, MatrixFreeHamiltonian)
          else LIB.macis_b200_davidson_ex)
    rc = fn(H.handle, C.byref(o), xs.ctypes.data, C.byref(E), C.byref(it), 0)
    if rc == _lib.ENOCONV:
        raise RuntimeError("Davidson Did Not Converge!")
    check(rc)
    X[:] = xs
    logging.getLogger("davidson").info("Davidson Converged! iter = %d E0 = %.12e",
                                       it.value, E.value)
    return it.value, E.value


def davidson_stats():
    """Per-phase device times (ms) of the last Davidson solve on this thread:
    apply (H products), rayleigh, residual, ortho (CGS2 and restarts), wall
    (host), and vector_bytes, the algorithmic bytes of the non-product
    phases."""
    st = _lib.DavidsonStatsC()
    check(LIB.macis_b200_davidson_last_stats(C.byref(st)))
    return {k: getattr(st, k) for k, _ in st._fields_}


def small_syev(lower, nwant=1):
    """Lowest `nwant` eigenpairs of a symmetric matrix from its lower
    triangle -- the Rayleigh-Ritz eigensolver used inside davidson."""
    A = np.asfortranarray(np.tril(np.asarray(lower, dtype=np.float64)))
    k = A.shape[0]
    W = np.empty(nwant)
    Vec = np.empty((nwant, k))
    check(LIB.macis_b200_small_syev(k, A.ctypes.data, nwant, W.ctypes.data,
                                    Vec.ctypes.data))
    return W, Vec.T


def selected_ci_diag(dets, ham_gen, h_el_tol, davidson_max_m,
                     davidson_res_tol, C=None, precision=FP64,
                     index_t=np.int32, timings=None, restart_keep=0,
                     max_iter=0, matrix_free=None):
    """Build H for `dets` and solve for the lowest root. Returns (E0, C).
    C is used as the guess when max|C| > 1/N (selected_ci_diag.hpp:96-101),
    else the diagonal guess is taken. precision MIXED stores the
    off-diagonal H in FP32 (FP64 diagonal) and keeps residuals, CGS2,
    Rayleigh-Ritz and the energy in FP64. matrix_free: True applies H
    without storing it (MatrixFreeHamiltonian), False always stores the
    CSR matrix, None (default) stores it unless the build runs out of
    device memory."""
    log = logging.getLogger("ci_solver")
    dets = np.ascontiguousarray(dets, dtype=np.uint64)
    ndets = dets.shape[0]
    log.info("[Selected CI Solver]: NDETS = %d, MATEL_TOL = %.5e, RES_TOL = "
             "%.5e, MAX_SUB = %d", ndets, h_el_tol, davidson_res_tol,
             davidson_max_m)
    value_t = np.float32 if precision == MIXED else np.float64
    t0 = time.perf_counter()
    H = None
    if matrix_free:
        H = MatrixFreeHamiltonian(dets, ham_gen, h_el_tol, value_t)
    else:
        try:
            H = _build_csr(dets, ham_gen, h_el_tol, index_t, value_t, log)
        except MacisError as e:
            if matrix_free is not None or e.code != ENOMEM:
                raise
            log.info("  the CSR matrix does not fit in device memory: "
                     "matrix-free H")
            H = MatrixFreeHamiltonian(dets, ham_gen, h_el_tol, value_t)
    t1 = time.perf_counter()
    if isinstance(H, MatrixFreeHamiltonian):
        log.info("  matrix-free H, setup %.5e ms", (t1 - t0) * 1e3)
    else:
        log.info("  NNZ = %d, H_DUR = %.5e ms", H.nnz, (t1 - t0) * 1e3)
        log.info("  HMEM_LOC = %.2e GiB", H.mem_footprint() / 1073741824.0)
    X = np.zeros(ndets)
    use_guess = False
    if C is not None and len(C) == ndets and ndets:
        if np.max(np.abs(C)) > 1.0 / ndets:
            X[:] = C
            use_guess = True
    it, E = davidson(ndets, davidson_max_m, H, None,
                     davidson_res_tol, X, use_guess=use_guess,
                     restart_keep=restart_keep, max_iter=max_iter)
    t2 = time.perf_counter()
    log.info("  DAV_NITER = %d, E0 = %.6e Eh, DAVIDSON_DUR = %.5e ms", it, E,
             (t2 - t1) * 1e3)
    if timings is not None:
        timings.update(h_ms=(t1 - t0) * 1e3, dav_ms=(t2 - t1) * 1e3,
                       nnz=getattr(H, "nnz", None), niter=it)
    return E, X


def _build_csr(dets, ham_gen, h_el_tol, index_t, value_t, log):
    """The CSR build of selected_ci_diag; index_t None picks int32 while nnz
    fits and int64 beyond."""
    ndets = dets.shape[0]
    if index_t is None:
        # int32 indices while nnz fits (2^31 - 1), else int64; the need for
        # int64 is remembered per generator so that later, larger spaces go
        # straight to it
        index_t = np.int64 if ndets >= getattr(
            ham_gen, "_int64_from_ndets", 1 << 62) else np.int32
        try:
            H = make_csr_hamiltonian(dets, ham_gen, h_el_tol, index_t, value_t)
        except MacisError as e:
            if index_t is not np.int32 or e.code != ECAPACITY:
                raise
            ham_gen._int64_from_ndets = ndets
            log.info("  nnz exceeds int32 indices: 64-bit indices")
            H = make_csr_hamiltonian(dets, ham_gen, h_el_tol, np.int64,
                                     value_t)
    else:
        H = make_csr_hamiltonian(dets, ham_gen, h_el_tol, index_t, value_t)
    return H

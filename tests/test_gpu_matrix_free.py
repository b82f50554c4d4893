"""Matrix-free H x (macis_b200_hop_*) against the CSR path: the same
elements and threshold, summed in enumeration order instead of column
order, so products agree to rounding (1e-12 relative here) and Davidson to
1e-9 Eh; the diagonal is the CSR diagonal exactly."""
import itertools

import numpy as np
import pytest

import macis_b200 as mb
from cases import embed, fci, shuffled

pytestmark = pytest.mark.gpu

EPS = float(np.finfo(float).eps)


def _selected(nbits, seed=2):
    T, V, d = fci(9, 4, 4, nbits, seed=5)
    sel = shuffled(d, seed=seed, frac=0.6).copy()
    sel[11] = 0                     # zero determinant: empty row and column
    sel[40] = sel[41]               # duplicate determinant
    return T, V, sel


def _check_product(A, Hm, n, seed=0):
    rng = np.random.default_rng(seed)
    for _ in range(2):
        x = rng.standard_normal(n)
        y0 = rng.standard_normal(n)
        ref = A.spmv(x, 0.7, 0.3, y0)
        got = Hm.spmv(x, 0.7, 0.3, y0)
        np.testing.assert_allclose(got, ref, rtol=1e-12,
                                   atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("nbits", [64, 128])
def test_apply_and_diagonal_match_csr(nbits):
    T, V, sel = _selected(nbits)
    H = mb.HamiltonianGenerator(T, V, nbits)
    A = mb.make_csr_hamiltonian(sel, H, EPS)
    Hm = mb.MatrixFreeHamiltonian(sel, H, EPS)
    assert Hm.m == A.m
    assert np.array_equal(Hm.diagonal(), A.diagonal())
    _check_product(A, Hm, A.m)
    for thr in (1e-3, 0.05):        # thresholds that drop elements
        _check_product(mb.make_csr_hamiltonian(sel, H, thr),
                       mb.MatrixFreeHamiltonian(sel, H, thr), A.m, seed=1)


def test_fp32_values_match_fp32_csr():
    """FP32 mode: the FP32-valued CSR's stored elements (diagonal kept in
    FP64) times the FP64 vector -- the product Davidson uses; the public
    SpMV of an FP32 matrix also rounds x, which this operator does not."""
    T, V, sel = _selected(64, seed=3)
    H = mb.HamiltonianGenerator(T, V, 64)
    A32 = mb.make_csr_hamiltonian(sel, H, EPS, value_t=np.float32)
    H32 = mb.MatrixFreeHamiltonian(sel, H, EPS, value_t=np.float32)
    x = np.random.default_rng(4).standard_normal(A32.m)
    rp, ci, nz = A32.to_host()
    rows = np.repeat(np.arange(A32.m), np.diff(rp))
    ref = np.zeros(A32.m)
    np.add.at(ref, rows, nz.astype(np.float64) * x[ci])
    ref += A32.diagonal() * x
    np.testing.assert_allclose(H32.spmv(x), ref, rtol=1e-12,
                               atol=1e-12 * np.abs(ref).max())


def test_large_groups_and_256_bit():
    """A 462-member alpha group (hash probes, beta-major alpha doubles) and
    the same problem in 256-bit words."""
    from macis_b200.integrals import synthetic_integrals
    rng = np.random.default_rng(3)
    n, k = 11, 5
    T, V = synthetic_integrals(n, 2)
    betas = [sum(1 << i for i in c)
             for c in itertools.combinations(range(n), k)]
    hf = (1 << k) - 1
    a_list, b_list = [hf] * len(betas), list(betas)
    for i in range(k):
        for x in range(k, n):
            for b in rng.choice(betas, 20, replace=False):
                a_list.append(hf ^ (1 << i) ^ (1 << x))
                b_list.append(int(b))
    d64 = shuffled(mb.sd.make_dets(a_list, b_list, 64), seed=5)
    for nbits, dets in ((64, d64), (256, embed(d64, 64, 256))):
        H = mb.HamiltonianGenerator(T, V, nbits)
        A = mb.make_csr_hamiltonian(dets, H, EPS)
        Hm = mb.MatrixFreeHamiltonian(dets, H, EPS)
        assert np.array_equal(Hm.diagonal(), A.diagonal())
        _check_product(A, Hm, A.m, seed=nbits)


def test_davidson_matches_csr():
    T, V, d = fci(8, 4, 4, 64, seed=2)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(d, H, EPS)
    Hm = mb.MatrixFreeHamiltonian(d, H, EPS)
    X0 = np.zeros(A.m)
    X1 = np.zeros(A.m)
    it0, E0 = mb.davidson(A.m, 60, mb.SparseMatrixOperator(A), None, 1e-8,
                          X0, use_guess=False)
    it1, E1 = mb.davidson(A.m, 60, Hm, None, 1e-8, X1, use_guess=False)
    assert abs(E1 - E0) < 1e-9 and abs(it1 - it0) <= 1
    assert abs(abs(X0 @ X1) - 1.0) < 1e-9


def test_selected_ci_diag_matrix_free_and_fallback(monkeypatch):
    """selected_ci_diag with matrix_free=True, and the default falling back
    to the matrix-free operator when the CSR build runs out of device
    memory (simulated: the build raises ENOMEM)."""
    from macis_b200 import _lib, solvers
    T, V, sel = _selected(64, seed=6)
    H = mb.HamiltonianGenerator(T, V, 64)
    E0, X0 = mb.selected_ci_diag(sel, H, EPS, 80, 1e-8)
    E1, X1 = mb.selected_ci_diag(sel, H, EPS, 80, 1e-8, matrix_free=True)
    assert abs(E1 - E0) < 1e-9

    def no_memory(*a, **k):
        raise _lib.MacisError(_lib.ENOMEM, "out of device memory")
    monkeypatch.setattr(solvers, "_build_csr", no_memory)
    t = {}
    E2, X2 = mb.selected_ci_diag(sel, H, EPS, 80, 1e-8, timings=t)
    assert abs(E2 - E0) < 1e-9 and t["nnz"] is None
    with pytest.raises(_lib.MacisError):
        mb.selected_ci_diag(sel, H, EPS, 80, 1e-8, matrix_free=False)

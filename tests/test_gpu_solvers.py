"""SpMV and Davidson on the GPU against the reference and the golden
energies (davidson.cxx:48, tolerance 1e-8 Eh), FP64 and mixed precision."""
import numpy as np
import pytest

import macis_b200 as mb
from cases import fci, shuffled
from golden_data import constants, water

pytestmark = pytest.mark.gpu
K = constants()


@pytest.fixture(scope="module")
def water_cisd(port):
    norb, T, V, ec = water()
    dets = port.cisd_space(64, norb, 5, 5)
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    return norb, T, V, ec, dets, H


def test_spmv_matches_reference(ref, water_cisd):
    norb, T, V, _, dets, H = water_cisd
    A = mb.make_csr_hamiltonian(dets, H, 1e-16)
    R = ref.csr(ref.ham(64, norb, T, V), dets, dets, 1e-16)
    rng = np.random.default_rng(0)
    for _ in range(3):
        x = rng.standard_normal(A.n)
        y = A.spmv(x)
        yr = R.spmv(x)
        np.testing.assert_allclose(y, yr, rtol=1e-12, atol=1e-12 * np.abs(yr).max())
    # alpha / beta and block of K = 3 columns
    X = rng.standard_normal((3, A.n))
    Y0 = rng.standard_normal((3, A.m))
    Y = Y0.copy()
    from macis_b200._lib import LIB, check
    check(LIB.macis_b200_spmv(A.handle, 3, 0.5, X.ctypes.data, A.n, -2.0,
                              Y.ctypes.data, A.m, 0))
    for k in range(3):
        np.testing.assert_allclose(Y[k], 0.5 * R.spmv(X[k]) - 2.0 * Y0[k],
                                   rtol=1e-11, atol=1e-10)


def test_davidson_water_golden(water_cisd):
    norb, T, V, ec, dets, H = water_cisd
    A = mb.make_csr_hamiltonian(dets, H, 1e-16)
    X = np.zeros(A.n)
    mb.diagonal_guess(A.n, A, X)
    it, E = mb.davidson(A.n, 15, mb.SparseMatrixOperator(A), A.diagonal(),
                        1e-8, X)
    assert abs(E + ec - K["water_cisd_e0_plus_ecore"]) < 1e-8
    assert abs(np.linalg.norm(X) - 1.0) < 1e-10
    assert abs(X @ A.spmv(X) - E) < 1e-8


def test_davidson_vs_reference_c1(ref):
    # The synthetic integrals are strongly correlated: the reference solver
    # (no restart) needs ~190 basis vectors at 1e-8, so both sides get 300.
    T, V, dets = fci(10, 5, 5, 64, seed=0)
    H = mb.HamiltonianGenerator(T, V, 64)
    E, X = mb.selected_ci_diag(dets, H, np.finfo(float).eps, 300, 1e-8)
    Er, Xr = ref.selected_ci_diag(ref.ham(64, 10, T, V), dets,
                                  np.finfo(float).eps, 300, 1e-8)
    assert abs(E - Er) < 1e-8
    assert abs(abs(X @ Xr) - 1.0) < 1e-7
    # thick restart reaches the same root with a 40-vector basis
    E2, X2 = mb.selected_ci_diag(dets, H, np.finfo(float).eps, 40, 1e-8,
                                 restart_keep=8, max_iter=2000)
    assert abs(E2 - Er) < 1e-8
    with pytest.raises(RuntimeError, match="Davidson Did Not Converge!"):
        mb.selected_ci_diag(dets, H, np.finfo(float).eps, 20, 1e-8)


def test_mixed_precision_energy():
    T, V, dets = fci(10, 5, 5, 64, seed=0)
    H = mb.HamiltonianGenerator(T, V, 64)
    kw = dict(restart_keep=8, max_iter=2000)
    E64, _ = mb.selected_ci_diag(dets, H, np.finfo(float).eps, 40, 1e-8, **kw)
    E32, X = mb.selected_ci_diag(dets, H, np.finfo(float).eps, 40, 1e-8,
                                 precision=mb.MIXED, **kw)
    assert abs(E32 - E64) < 1e-7          # north-star mixed target
    assert abs(np.linalg.norm(X) - 1.0) < 1e-10


def test_davidson_nonconvergence_raises():
    T, V, dets = fci(8, 4, 4, 64, seed=1)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, 1e-14)
    X = np.zeros(A.n)
    with pytest.raises(RuntimeError, match="Davidson Did Not Converge!"):
        mb.davidson(A.n, 3, mb.SparseMatrixOperator(A), None, 1e-14, X,
                    use_guess=False)


def test_guess_reuse_and_selected_space(ref):
    T, V, dets = fci(9, 4, 4, 128, seed=4)
    sel = shuffled(dets, seed=5, frac=0.5)
    H = mb.HamiltonianGenerator(T, V, 128)
    E, X = mb.selected_ci_diag(sel, H, 1e-12, 300, 1e-9)
    Er, _ = ref.selected_ci_diag(ref.ham(128, 9, T, V), sel, 1e-12, 300, 1e-9)
    assert abs(E - Er) < 1e-8
    E2, X2 = mb.selected_ci_diag(sel, H, 1e-12, 300, 1e-9, C=X)
    assert abs(E2 - E) < 1e-8

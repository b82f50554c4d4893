"""Row-distributed H and p_davidson on one GPU (world size 1, no process
group): the device product of DistCSR and the solver against the oracle.
The host logic with two ranks is covered on CPU over gloo."""
import numpy as np
import pytest

import macis_b200 as mb
from cases import fci

pytestmark = pytest.mark.gpu


def test_dist_csr_and_p_davidson(port):
    import torch

    from macis_b200 import dist as md
    T, V, dets = fci(8, 4, 3, 64, seed=2)
    N = len(dets)
    H = mb.HamiltonianGenerator(T, V, 64)
    dev = torch.device("cuda", 0)
    for src in (dets, torch.from_numpy(dets.view(np.int64)).to(dev)):
        A = md.make_dist_csr_hamiltonian(src, H, np.finfo(float).eps)
        assert (A.lo, A.hi, A.N) == (0, N, N)
        ref = port.build_csr(port.ham(64, 8, T, V), dets, dets,
                             np.finfo(float).eps)
        rp, ci, nz = A.local.to_host()
        assert np.array_equal(rp, ref[0]) and np.array_equal(ci, ref[1])
        assert np.array_equal(nz, ref[2])
        x = np.random.default_rng(0).standard_normal(N)
        y = A.local_spmv(torch.from_numpy(x).to(dev),
                         torch.empty(N, dtype=torch.float64, device=dev))
        np.testing.assert_allclose(y.cpu().numpy(), port.spmv(*ref, x),
                                   rtol=1e-12, atol=1e-12)
    D = A.diagonal(dev)
    X = torch.zeros(N, dtype=torch.float64, device=dev)
    g = int(torch.argmin(D).item())
    X[g] = 1.0
    it, E = md.p_davidson(N, 200, A.operator(), D, 1e-8, X)
    X0 = np.zeros(N)
    X0[g] = 1.0
    E_ref, it_ref, X_ref = port.davidson(*ref, 200, 1e-8, X0)
    assert abs(E - E_ref) < 1e-9 and abs(it - it_ref) <= 1
    Xg = X.cpu().numpy()
    assert abs(abs(Xg @ X_ref) / np.linalg.norm(Xg) / np.linalg.norm(X_ref)
               - 1) < 1e-10


def test_dist_csr_offset_block_diagonal(port):
    """On a rank with lo > 0 the preconditioner diagonal is H_ii of its rows
    (the diagonal tile), not the block's entries in column == local row."""
    from macis_b200 import dist as md
    T, V, dets = fci(8, 4, 4, 64, seed=7)
    N = len(dets)
    H = mb.HamiltonianGenerator(T, V, 64)
    full = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps).diagonal()
    for r in range(3):
        lo, hi = mb.row_bounds(N, 3, r)
        blk = mb.make_csr_hamiltonian_block(dets[lo:hi], dets, H,
                                            np.finfo(float).eps)
        D = md.DistCSR(blk, lo, hi, N, bra=dets[lo:hi]).diagonal().numpy()
        assert np.array_equal(D, full[lo:hi])


def test_dist_asci_grow_refine_water_golden():
    """The distributed ASCI drivers at world size 1 (no process group): the
    split search, the row-block H with p_davidson and the gathered vector
    reproduce the water grow and refine energies."""
    from golden_data import constants, water

    from macis_b200 import dist as md
    K = constants()
    norb, T, V, _ = water()
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    s = mb.ASCISettings()
    s.ntdets_max = K["water_asci_ntdets_max"]
    ci = mb.MCSCFSettings()
    hf = mb.canonical_hf_determinant(5, 5, 64)
    E0 = H.matrix_element(hf, hf)
    E, dets, X = md.asci_grow(s, ci, E0, hf, np.ones(1), H, norb)
    assert len(dets) == 10000 and abs(X @ X - 1) < 1e-10
    assert abs(E - K["water_asci_grow_e0"]) < 1e-8
    E, dets, X = md.asci_refine(s, ci, E, dets, X, H, norb)
    assert len(dets) == 10000
    assert abs(E - K["water_asci_refine_e0"]) < 1e-7
    ci.precision = mb.MIXED
    with pytest.raises(NotImplementedError):
        md.asci_iter(s, ci, 10000, E, dets, X, H, norb)

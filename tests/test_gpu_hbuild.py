"""H build on the GPU against the reference (compiled) and the oracle:
bit-exact rowptr / colind / nzval (double_loop.hpp:31-98 semantics)."""
import numpy as np
import pytest

import macis_b200 as mb
from cases import assert_csr_equal, embed, fci, shuffled
from golden_data import water, water_cisd_rowptr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wat():
    return water()


def test_water_cisd_exact(port, ref, wat):
    norb, T, V, _ = wat
    dets = port.cisd_space(64, norb, 5, 5)
    H = mb.HamiltonianGenerator(T, V, 64, norb)
    A = mb.make_csr_hamiltonian(dets, H, 1e-16)
    rp, ci, nz = A.to_host()
    assert np.array_equal(rp, water_cisd_rowptr())
    r = ref.build_csr(ref.ham(64, norb, T, V), dets, dets, 1e-16, nthreads=4)
    assert_csr_equal((rp, ci, nz), r)
    assert np.array_equal(A.diagonal(), ref.csr(ref.ham(64, norb, T, V), dets,
                                                dets, 1e-16).diagonal())


@pytest.mark.parametrize("nbits", [64, 128])
def test_fci_direct_product_exact(ref, nbits):
    T, V, dets = fci(8, 4, 3, nbits, seed=3)
    H = mb.HamiltonianGenerator(T, V, nbits)
    hr = ref.ham(nbits, 8, T, V)
    for thr in (np.finfo(float).eps, 1e-3, 0.05):   # 0.05 drops many entries
        A = mb.make_csr_hamiltonian(dets, H, thr)
        assert A.build_stats()["direct_product"] == 1
        assert_csr_equal(A.to_host(), ref.build_csr(hr, dets, dets, thr,
                                                    nthreads=4))
        A32 = mb.make_csr_hamiltonian(dets, H, thr, value_t=np.float32)
        assert np.array_equal(A32.to_host()[1], A.to_host()[1])
        assert np.array_equal(A32.diagonal(), A.diagonal())


@pytest.mark.parametrize("norb,na,nb", [(9, 3, 0), (8, 2, 8), (7, 1, 6),
                                         (12, 6, 1)])
def test_direct_product_edge_occupations(ref, norb, na, nb):
    """Empty / full / single-electron beta strings: beta lists of one entry
    (no beta excitation) and short lists."""
    T, V, dets = fci(norb, na, nb, 64, seed=5)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps)
    assert A.build_stats()["direct_product"] == 1
    assert_csr_equal(A.to_host(), ref.build_csr(
        ref.ham(64, norb, T, V), dets, dets, np.finfo(float).eps, nthreads=4))


def test_c1_fci_exact(ref):
    # CAS(10e,10o): 63,504 determinants
    T, V, dets = fci(10, 5, 5, 64, seed=0)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps)
    assert A.m == 63504
    r = ref.build_csr(ref.ham(64, 10, T, V), dets, dets, np.finfo(float).eps,
                      nthreads=16)
    assert_csr_equal(A.to_host(), r)


def test_row_blocks_of_direct_product(ref):
    # the row partition of make_dist_csr_hamiltonian (csr_hamiltonian.hpp:
    # 49-82): bra = contiguous slice of the ket list keeps the direct path
    T, V, dets = fci(8, 4, 4, 64, seed=12)
    H = mb.HamiltonianGenerator(T, V, 64)
    hr = ref.ham(64, 8, T, V)
    thr = np.finfo(float).eps
    for r in range(3):
        lo, hi = mb.row_bounds(len(dets), 3, r)
        A = mb.make_csr_hamiltonian_block(dets[lo:hi], dets, H, thr)
        assert A.build_stats()["direct_product"] == 1
        assert_csr_equal(A.to_host(), ref.build_csr(hr, dets[lo:hi], dets, thr))
        A32 = mb.make_csr_hamiltonian_block(dets[lo:hi], dets, H, thr,
                                            value_t=np.float32)
        assert np.array_equal(A32.to_host()[1], A.to_host()[1])


@pytest.mark.parametrize("nbits", [64, 128])
def test_general_path_shuffled_and_rectangular(ref, nbits):
    T, V, dets = fci(9, 4, 4, nbits, seed=5)
    sel = shuffled(dets, seed=2, frac=0.6)          # selected-CI style list
    H = mb.HamiltonianGenerator(T, V, nbits)
    hr = ref.ham(nbits, 9, T, V)
    thr = np.finfo(float).eps
    assert_csr_equal(mb.make_csr_hamiltonian(sel, H, thr).to_host(),
                     ref.build_csr(hr, sel, sel, thr, nthreads=8))
    bra, ket = sel[:500], shuffled(dets, seed=7, frac=0.5)
    assert_csr_equal(
        mb.make_csr_hamiltonian_block(bra, ket, H, thr).to_host(),
        ref.build_csr(hr, bra, ket, thr, nthreads=8))


def test_zero_dets_duplicates_and_threshold(ref):
    T, V, dets = fci(8, 3, 3, 64, seed=9)
    sel = shuffled(dets, seed=4, frac=0.5).copy()
    sel[5] = 0                  # zero determinants: empty rows / columns
    sel[17] = 0
    sel[30] = sel[31]           # duplicate determinant
    H = mb.HamiltonianGenerator(T, V, 64)
    hr = ref.ham(64, 8, T, V)
    for thr in (np.finfo(float).eps, 1e-3, 0.05):   # exercise compaction
        assert_csr_equal(mb.make_csr_hamiltonian(sel, H, thr).to_host(),
                         ref.build_csr(hr, sel, sel, thr))


def test_long_rows_path(ref):
    # every determinant three times: rows carry ~1083 candidates, more than
    # the shared-memory sort holds, so they go through the radix-sort pass
    T, V, d = fci(8, 4, 4, 64, seed=11)
    sel = shuffled(np.concatenate([d, d, d]), seed=3)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(sel, H, 0.0)
    rp = A.to_host()[0]
    assert np.diff(rp).max() > 1024
    assert_csr_equal(A.to_host(), ref.build_csr(ref.ham(64, 8, T, V), sel,
                                                sel, 0.0, nthreads=16))


def test_int64_index_and_empty(ref):
    T, V, dets = fci(7, 3, 3, 64, seed=1)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, 1e-12, index_t=np.int64)
    assert A.index_t == np.int64
    assert_csr_equal(A.to_host(), ref.build_csr(ref.ham(64, 7, T, V), dets,
                                                dets, 1e-12))
    E = mb.make_csr_hamiltonian_block(dets[:0], dets, H, 1e-12)
    assert E.m == 0 and E.nnz == 0
    E = mb.make_csr_hamiltonian_block(dets[:4], dets[:0], H, 1e-12)
    assert E.m == 4 and E.nnz == 0 and np.all(E.to_host()[0] == 0)


def test_fp32_storage_matches_fp64(ref):
    T, V, dets = fci(8, 4, 4, 64, seed=2)
    H = mb.HamiltonianGenerator(T, V, 64)
    A64 = mb.make_csr_hamiltonian(dets, H, 1e-14)
    A32 = mb.make_csr_hamiltonian(dets, H, 1e-14, value_t=np.float32)
    r64, c64, z64 = A64.to_host()
    r32, c32, z32 = A32.to_host()
    assert np.array_equal(r64, r32) and np.array_equal(c64, c32)
    rows = np.repeat(np.arange(A64.m), np.diff(r64))
    diag = c64 == rows
    assert np.all(z32[diag] == 0)
    assert np.array_equal(z32[~diag], z64[~diag].astype(np.float32))
    assert np.array_equal(A32.diagonal(), A64.diagonal())


def test_256bit_matches_embedded(port):
    # bitset<256> has no reference: the oracle restatement is the check, and
    # a 64-bit problem embedded in 256-bit words must give the same CSR.
    T, V, d64 = fci(8, 3, 3, 64, seed=6)
    d256 = embed(shuffled(d64, seed=1, frac=0.7), 64, 256)
    H = mb.HamiltonianGenerator(T, V, 256)
    A = mb.make_csr_hamiltonian(d256, H, 1e-14).to_host()
    hp = port.ham(256, 8, T, V)
    assert_csr_equal(A, port.build_csr(hp, d256, d256, 1e-14))
    d64s = embed(d256, 256, 64)
    H64 = mb.HamiltonianGenerator(T, V, 64)
    assert_csr_equal(A, mb.make_csr_hamiltonian(d64s, H64, 1e-14).to_host())


def test_256bit_large_orbital_count(port):
    # n = 70 orbitals crosses the 64-bit word boundary of each spin string
    from macis_b200.integrals import synthetic_integrals
    rng = np.random.default_rng(0)
    n = 70
    T, V = synthetic_integrals(n, 4)
    hf_a = (1 << 4) - 1
    a = [hf_a] + [hf_a ^ (1 << int(i)) ^ (1 << int(x)) for i, x in
                  zip(rng.integers(0, 4, 60), rng.integers(4, n, 60))]
    b = [hf_a ^ (1 << 3) ^ (1 << int(x)) for x in rng.integers(60, n, 61)]
    dets = mb.sd.make_dets(a, b, 256)
    dets = np.unique(dets, axis=0)
    H = mb.HamiltonianGenerator(T, V, 256)
    A = mb.make_csr_hamiltonian(dets, H, 1e-14).to_host()
    assert_csr_equal(A, port.build_csr(port.ham(256, n, T, V), dets, dets,
                                       1e-14))


def test_matrix_element_batch(ref):
    T, V, dets = fci(8, 4, 3, 128, seed=8)
    rng = np.random.default_rng(0)
    i, j = rng.integers(0, len(dets), 4000), rng.integers(0, len(dets), 4000)
    H = mb.HamiltonianGenerator(T, V, 128)
    got = H.matrix_element(dets[i], dets[j])
    exp = ref.matrix_element(ref.ham(128, 8, T, V), dets[i], dets[j])
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("nbits", [64, 128])
def test_general_path_large_groups(ref, nbits):
    """Rows whose alpha string is a single excitation of a large alpha group
    (here the HF alpha with all 462 betas) look their beta singles up in the
    group's hash table instead of testing every member; parity with the
    reference, with a duplicated determinant inside the large group."""
    from macis_b200.integrals import synthetic_integrals
    rng = np.random.default_rng(3)
    n, k = 11, 5
    T, V = synthetic_integrals(n, 2)
    betas = [sum(1 << i for i in c) for c in
             __import__("itertools").combinations(range(n), k)]
    hf = (1 << k) - 1
    a_list, b_list = [hf] * len(betas), list(betas)
    for i in range(k):
        for x in range(k, n):
            a = hf ^ (1 << i) ^ (1 << x)
            for b in rng.choice(betas, 20, replace=False):
                a_list.append(a)
                b_list.append(int(b))
    dets = mb.sd.make_dets(a_list, b_list, nbits)
    dets = np.concatenate([dets, dets[7:8]])          # duplicate in the group
    dets = shuffled(dets, seed=5)
    H = mb.HamiltonianGenerator(T, V, nbits)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps)
    assert A.build_stats()["direct_product"] == 0
    assert_csr_equal(A.to_host(), ref.build_csr(ref.ham(nbits, n, T, V), dets,
                                                dets, np.finfo(float).eps,
                                                nthreads=8))


def test_product_layout_with_many_orbitals_takes_general_path(ref):
    """A selected space in the product layout (one alpha string, distinct
    betas) at 48 orbitals: the direct-product fill's per-warp singles table
    would not fit in shared memory, so the general path builds it,
    bit-exact with the reference."""
    from macis_b200.integrals import synthetic_integrals
    n, k = 48, 12
    T, V = synthetic_integrals(n, 1)
    hf = (1 << k) - 1
    betas = sorted({hf} | {hf ^ (1 << i) ^ (1 << a) for i in range(k)
                           for a in range(k, n)})
    dets = mb.sd.make_dets([hf] * len(betas), betas, 128)
    H = mb.HamiltonianGenerator(T, V, 128)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps)
    assert A.build_stats()["direct_product"] == 0
    assert_csr_equal(A.to_host(), ref.build_csr(ref.ham(128, n, T, V), dets,
                                                dets, np.finfo(float).eps,
                                                nthreads=8))

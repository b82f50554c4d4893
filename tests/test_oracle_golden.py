"""The CPU oracle (C restatement) and the compiled reference against the
golden values of the reference's own tests (tests/double_loop.cxx,
tests/csr_hamiltonian.cxx, tests/davidson.cxx, tests/asci.cxx) on the water
cc-pVDZ integrals."""
import numpy as np
import pytest

import oracle
from golden_data import constants, water, water_cisd_rowptr

K = constants()
REL = K["catch2_approx_rel"]  # Catch2 Approx default


def approx(a, b, rel=REL):
    return abs(a - b) <= rel * (1.0 + max(abs(a), abs(b)))


@pytest.fixture(scope="module")
def wat():
    return water()


@pytest.fixture(scope="module")
def hp(port, wat):
    norb, T, V, _ = wat
    return port.ham(64, norb, T, V)


def test_hf_energy(port, ref, wat, hp):
    norb, T, V, ec = wat
    hf = port.hf_det(64, 5, 5)
    e_port = port.matrix_element(hp, hf, hf)[0]
    e_ref = ref.matrix_element(ref.ham(64, norb, T, V), hf, hf)[0]
    assert e_port == e_ref
    assert abs(e_port + ec - K["water_ehf_plus_ecore"]) < 1e-10


def _flip(det, *bits):
    d = det.copy()
    for b in bits:
        d[0, 0] ^= np.uint64(1) << np.uint64(b)
    return d


def test_excited_diagonals_and_fast_diag(port, ref, wat, hp):
    norb, T, V, _ = wat
    hr = ref.ham(64, norb, T, V)
    hf = port.hf_det(64, 5, 5)
    ehf = port.matrix_element(hp, hf, hf)[0]
    occ = np.arange(5, dtype=np.uint32)
    eps = port.single_orbital_ens(hp, occ, occ)
    P = port.L
    s1 = _flip(hf, 0, 5)
    es = port.matrix_element(hp, s1, s1)[0]
    assert approx(es, K["water_single_diag"])
    fs = P.orc_fast_diag_single(hp.p, eps[0], eps[5], 0, 5, ehf)
    assert approx(es, fs)
    assert fs == ref.fast_diag(hr, 1, occ, occ, [0, 5], ehf)
    d2 = _flip(hf, 0, 5, 1, 6)
    ed = port.matrix_element(hp, d2, d2)[0]
    assert approx(ed, K["water_ss_double_diag"])
    fd = P.orc_fast_diag_ss_double(hp.p, eps[0], eps[1], eps[5], eps[6], 0, 1,
                                   5, 6, ehf)
    assert approx(ed, fd)
    assert fd == ref.fast_diag(hr, 2, occ, occ, [0, 1, 5, 6], ehf)
    o2 = _flip(hf, 0, 5, 33, 38)
    eo = port.matrix_element(hp, o2, o2)[0]
    assert approx(eo, K["water_os_double_diag"])
    fo = P.orc_fast_diag_os_double(hp.p, eps[0], eps[1], eps[5], eps[6], 0, 1,
                                   5, 6, ehf)
    assert approx(eo, fo)
    assert fo == ref.fast_diag(hr, 3, occ, occ, [0, 1, 5, 6], ehf)


def test_brillouin_and_mp2(port, wat, hp):
    norb, T, V, _ = wat
    n2, n3 = norb * norb, norb ** 3
    hf = port.hf_det(64, 5, 5)
    eps = np.array([T[p * (norb + 1)] + sum(
        2 * V[p * (norb + 1) + i * (n2 + n3)] - V[p * (1 + n3) + i * (norb + n2)]
        for i in range(5)) for p in range(norb)])
    for shift in (0, 32):
        for i in range(5):
            for a in range(5, norb):
                s = _flip(hf, i + shift, a + shift)
                e1 = port.matrix_element(hp, hf, s)[0]
                e2 = port.matrix_element(hp, s, hf)[0]
                assert abs(e1) < 1e-6 and approx(e1, e2)
    emp2 = 0.0
    for shift in (0, 32):
        for a in range(5, norb):
            for b in range(a + 1, norb):
                for i in range(5):
                    for j in range(i + 1, 5):
                        s = _flip(hf, i + shift, j + shift, a + shift, b + shift)
                        h = port.matrix_element(hp, hf, s)[0]
                        emp2 += h * h / (eps[a] + eps[b] - eps[i] - eps[j])
    bra, ket, den = [], [], []
    for a in range(5, norb):
        for b in range(5, norb):
            for i in range(5):
                for j in range(5):
                    bra.append(hf[0])
                    ket.append(_flip(hf, i, j + 32, a, b + 32)[0])
                    den.append(eps[a] + eps[b] - eps[i] - eps[j])
    h = port.matrix_element(hp, np.array(bra), np.array(ket))
    emp2 += np.sum(h * h / np.array(den))
    assert approx(-emp2, K["water_mp2"])


@pytest.fixture(scope="module")
def cisd(port, ref, wat, hp):
    norb, T, V, _ = wat
    dets = port.cisd_space(64, norb, 5, 5)
    assert (dets == ref.cisd_space(64, norb, 5, 5)).all()
    return dets, port.build_csr(hp, dets, dets, 1e-16)


def test_cisd_csr_matches_reference_rowptr(cisd, ref, wat):
    dets, (rp, ci, nz) = cisd
    assert len(dets) == 12636
    assert np.array_equal(rp, water_cisd_rowptr())
    norb, T, V, _ = wat
    rr, cr, zr = ref.build_csr(ref.ham(64, norb, T, V), dets, dets, 1e-16,
                               nthreads=4)
    assert np.array_equal(rr, rp) and np.array_equal(cr, ci)
    assert np.array_equal(zr, nz)  # bit-exact values


def test_cisd_davidson(port, cisd, wat):
    _, (rp, ci, nz) = cisd
    E, it, X = port.davidson(rp, ci, nz, K["water_cisd_davidson_max_m"], 1e-8)
    assert abs(E + wat[3] - K["water_cisd_e0_plus_ecore"]) < 1e-8
    assert approx(np.linalg.norm(X), 1.0)
    assert approx(X @ port.spmv(rp, ci, nz, X), E)


def test_asci_grow_refine_water(port, ref, wat):
    norb, T, V, _ = wat
    hp = port.ham(64, norb, T, V)
    s = oracle.AsciSettings.default(ntdets_max=K["water_asci_ntdets_max"])
    ci = oracle.CiSettings.default()
    hf = port.hf_det(64, 5, 5)
    E0 = port.matrix_element(hp, hf, hf)[0]
    E, dets, X = port.asci_grow(hp, s, ci, E0, hf, np.ones(1))
    assert len(dets) == 10000 and approx(X @ X, 1.0)
    assert abs(E - K["water_asci_grow_e0"]) < 1e-8
    E, dets, X = port.asci_refine(hp, s, ci, E, dets, X)
    assert len(dets) == 10000
    assert abs(E - K["water_asci_refine_e0"]) < 1e-7


def test_singles_doubles_enumeration(port):
    # sd_operations.cxx: singles / doubles of HF(4 alpha) in 8 orbitals are
    # all 16 single and 36 double alpha excitations.
    for nbits in (64, 128, 256):
        d = port.cisd_space(nbits, 8, 4, 0)
        assert len(d) == 1 + 16 + 36
        a = [int(x[0]) for x in d]
        assert a[0] == 0b1111 and len(set(a)) == len(a)
        pc = [bin(x ^ 0b1111).count("1") for x in a]
        assert pc == [0] + [2] * 16 + [4] * 36


@pytest.mark.parametrize("nbits", [64, 128])
def test_asci_pairs_and_search_match_reference(port, ref, wat, nbits):
    """The oracle's ASCI restatement against the compiled reference
    (determinant_search.hpp:54-141, 395-663) on a water core set: the same
    accumulated candidates, scores to 1e-12 relative (the reference sums
    duplicates in its sort's order), and the same top-k except between
    candidates tied at the cut."""
    norb, T, V, _ = wat
    hp = port.ham(nbits, norb, T, V)
    s = oracle.AsciSettings.default()
    ci = oracle.CiSettings.default()
    hf = port.hf_det(nbits, 5, 5)
    E0 = port.matrix_element(hp, hf, hf)[0]
    E, dets, X = port.asci_iter(hp, s, ci, 800, E0, hf, np.ones(1))
    order = np.argsort(-np.abs(X), kind="stable")[:100]
    cd, cc = dets[order], X[order]
    hr = ref.ham(nbits, norb, T, V)
    so, ro = port.asci_pairs(hp, s, cd, E, cc)
    sr, rr = ref.asci_pairs(hr, s, cd, E, cc)
    assert np.array_equal(so, sr)
    assert np.all(np.abs(ro - rr) <= 1e-12 * np.abs(rr) + 1e-15 * np.abs(rr).max())
    score = {tuple(t): abs(v) for t, v in zip(so.tolist(), ro)}
    for ndets in (900, 5000):
        a = port.asci_search(hp, s, ndets, cd, E, cc)
        b = ref.asci_search(hr, s, ndets, cd, E, cc)
        assert len(a) == len(b) and np.array_equal(a[-len(cd):], cd)
        ta = set(map(tuple, a[:-len(cd)].tolist()))
        tb = set(map(tuple, b[:-len(cd)].tolist()))
        kth = min(score[t] for t in ta)
        for t in ta ^ tb:
            assert abs(score[t] - kth) <= 1e-12 * kth

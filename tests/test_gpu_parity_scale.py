"""Parity at the shapes of the large ASCI configurations, against the
compiled reference and the oracle port.

* n = 48, 12 alpha / 12 beta electrons and n = 64, 16 alpha / 16 beta, both
  as bitset<128>: every spin word uses bits 32..63, which the water-sized
  problems never reach. Checked against the compiled reference:
  - ASCI contributions of a core set (asci_contributions_standard +
    sort_and_accumulate_asci_pairs, determinant_search.hpp:54-141,
    determinant_sort.hpp:40-83): identical candidate sets; scores
    bit-identical to the port (same generation and summation order) and
    within 1e-13 of the sum of |contributions| of the reference's (whose
    unstable std::sort changes the summation order: sums that cancel differ
    by up to ~4e-11 relative between the two orders at n = 64, so a bound
    relative to the score itself does not hold for either implementation);
  - asci_search (determinant_search.hpp:395-663): identical to the port,
    identical to the reference outside near-ties at the k-th score;
  - the CSR Hamiltonian (double_loop.hpp:31-98) of the selected space that
    search returns: rowptr / colind / nzval bit-exact, square, rectangular
    and shuffled;
  - selected_ci_diag (selected_ci_diag.hpp:76-121) on that space: lowest
    energy within 1e-8 Eh.
* n = 100, 20 alpha / 20 beta as bitset<256> (the reference cannot
  instantiate bitset<256>): the port is the check; the port's 256-bit path
  is itself pinned to the reference by the n = 48 problem embedded in
  256-bit words (tests/test_oracle_scale.py).
"""
import numpy as np
import pytest

import macis_b200 as mb
import oracle
from cases import (abs_sums, assert_csr_equal, core_set,
                   reference_mpi_selection, shuffled)

pytestmark = pytest.mark.gpu

SHAPES = {"n48": (48, 12, 50), "n64": (64, 16, 20)}
NDETS = 20000


def _settings():
    return mb.ASCISettings()


@pytest.fixture(scope="module", params=sorted(SHAPES))
def shape(request, port, ref):
    n, k, ncore = SHAPES[request.param]
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, ncore, 128)
    hr = ref.ham(128, n, T, V)
    hp = port.ham(128, n, T, V)
    H = mb.HamiltonianGenerator(T, V, 128)
    E0 = float(H.matrix_element(cd[:1], cd[:1])) - 0.5
    return dict(n=n, T=T, V=V, cd=cd, C=C, hr=hr, hp=hp, H=H, E0=E0)


@pytest.fixture(scope="module")
def pairs(shape, port, ref):
    s = oracle.AsciSettings.default()
    g = mb.asci_pairs(_settings(), shape["cd"], shape["E0"], shape["C"],
                      shape["H"])
    p = port.asci_pairs(shape["hp"], s, shape["cd"], shape["E0"], shape["C"])
    r = ref.asci_pairs(shape["hr"], s, shape["cd"], shape["E0"], shape["C"])
    raw = port.asci_pairs(shape["hp"], s, shape["cd"], shape["E0"],
                          shape["C"], accumulate=False)
    u, scale = abs_sums(*raw)
    return g, p, r, u, scale


def test_pairs_match_port_and_reference(pairs):
    (gs, gr), (ps, pr), (rs, rr), u, scale = pairs
    assert len(gs) > 1_000_000
    assert np.array_equal(gs, ps) and np.array_equal(gr, pr)
    assert np.array_equal(gs, rs)
    assert np.array_equal(gs, u)
    assert np.all(np.abs(gr - rr) <= 1e-13 * scale)


def test_search_matches_port_and_reference(shape, pairs, port, ref):
    s = oracle.AsciSettings.default()
    got = mb.asci_search(_settings(), NDETS, shape["cd"], shape["E0"],
                         shape["C"], shape["n"], shape["H"])
    exp = port.asci_search(shape["hp"], s, NDETS, shape["cd"], shape["E0"],
                           shape["C"])
    assert np.array_equal(got, exp)
    r = ref.asci_search(shape["hr"], s, NDETS, shape["cd"], shape["E0"],
                        shape["C"])
    assert len(r) == len(got) == NDETS
    key = lambda a: set(map(tuple, np.asarray(a).tolist()))
    diff = key(got) ^ key(r)
    if diff:
        # only near-ties at the cut may differ: their scores equal the k-th
        # score within the summation error of both orders
        (gs, gr), _, _, _, scale = pairs
        idx = {t: i for i, t in enumerate(map(tuple, gs.tolist()))}
        kth = min(abs(gr[idx[t]])
                  for t in key(got[:NDETS - len(shape["cd"])]))
        for t in diff:
            i = idx[t]
            assert abs(abs(gr[i]) - kth) <= 2e-13 * scale[i] + 1e-14 * kth


@pytest.mark.parametrize("world", [2, 4])
def test_split_search_matches_reference_constraint_partition(shape, pairs,
                                                             world):
    """The hash-bin split search over `world` parts, merged, against the
    reference's MPI search over `world` ranks: each rank's pairs from the
    reference's own constraint-partitioned path (asci_contributions_
    constraint, determinant_search.hpp:143-391, rank split of
    dist_constraint_general) and the reference's distributed top-k over
    them (determinant_search.hpp:528-654). Identical selections outside
    near-ties at the k-th score."""
    if not oracle.ref_constraint_available():
        pytest.skip("compiled reference oracle/_ref not built")
    refc = oracle.ref_constraint()
    n, cd, C, E0, H = (shape[k] for k in ("n", "cd", "C", "E0", "H"))
    parts = [mb.asci_search_part(_settings(), NDETS, cd, E0, C, n, H, i,
                                 world) for i in range(world)]
    got = mb.merge_asci_parts(parts, NDETS, cd, 128)
    hc = refc.ham(128, n, shape["T"], shape["V"])
    so = oracle.AsciSettings.default()
    rparts = [refc.asci_pairs(hc, so, cd, E0, C, r, world)
              for r in range(world)]
    exp = reference_mpi_selection(rparts, cd, NDETS)
    assert len(got) == len(exp) == NDETS
    assert np.array_equal(got[NDETS - len(cd):], cd)
    key = lambda a: set(map(tuple, np.asarray(a).tolist()))
    diff = key(got) ^ key(exp)
    if diff:
        (gs, gr), _, _, _, scale = pairs
        idx = {t: i for i, t in enumerate(map(tuple, gs.tolist()))}
        kth = min(abs(gr[idx[t]]) for t in key(got[:NDETS - len(cd)]))
        for t in diff:
            i = idx[t]
            assert abs(abs(gr[i]) - kth) <= 2e-13 * scale[i] + 1e-14 * kth


@pytest.fixture(scope="module")
def space(shape):
    return mb.asci_search(_settings(), NDETS, shape["cd"], shape["E0"],
                          shape["C"], shape["n"], shape["H"])


def test_selected_space_csr_bit_exact(shape, space, ref):
    thr = 1e-16
    A = mb.make_csr_hamiltonian(space, shape["H"], thr)
    assert A.build_stats()["direct_product"] == 0
    r = ref.build_csr(shape["hr"], space, space, thr, nthreads=8)
    assert_csr_equal(A.to_host(), r)
    assert len(r[1]) > 20 * len(space)
    # rectangular block of a shuffled list, 64-bit indices, a coarse
    # threshold that drops most elements
    kets = shuffled(space, seed=3)
    bra = kets[:3000]
    for thr2, idx in ((thr, np.int64), (1e-3, np.int32)):
        B = mb.make_csr_hamiltonian_block(bra, kets, shape["H"], thr2,
                                          index_t=idx)
        assert_csr_equal(B.to_host(), ref.build_csr(shape["hr"], bra, kets,
                                                    thr2, nthreads=8))
    F = mb.make_csr_hamiltonian(space, shape["H"], thr, value_t=np.float32)
    assert np.array_equal(F.to_host()[1], r[1])
    assert np.array_equal(F.diagonal(), A.diagonal())


def test_selected_space_energy(shape, space, ref):
    if shape["n"] != 48:
        pytest.skip("one energy check (n = 48) keeps the module short")
    E, X = mb.selected_ci_diag(space, shape["H"], 1e-16, 100, 1e-8)
    Er, Xr = ref.selected_ci_diag(shape["hr"], space, 1e-16, 100, 1e-8)
    assert abs(E - Er) <= 1e-8
    assert abs(abs(np.dot(X, Xr)) - 1.0) <= 1e-6


@pytest.fixture(scope="module")
def n100(port):
    n, k = 100, 20
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, 3, 256)
    H = mb.HamiltonianGenerator(T, V, 256)
    hp = port.ham(256, n, T, V)
    E0 = float(H.matrix_element(cd[:1], cd[:1])) - 0.5
    return dict(n=n, T=T, V=V, cd=cd, C=C, H=H, hp=hp, E0=E0)


def test_256bit_n100_pairs_search_and_csr(n100, port):
    s = oracle.AsciSettings.default()
    cd, C, E0, H, hp = (n100[k] for k in ("cd", "C", "E0", "H", "hp"))
    gs, gr = mb.asci_pairs(_settings(), cd, E0, C, H)
    ps, pr = port.asci_pairs(hp, s, cd, E0, C)
    assert len(gs) > 5_000_000
    assert np.array_equal(gs, ps) and np.array_equal(gr, pr)
    got = mb.asci_search(_settings(), 5000, cd, E0, C, n100["n"], H)
    assert np.array_equal(got, port.asci_search(hp, s, 5000, cd, E0, C))
    A = mb.make_csr_hamiltonian(got, H, 1e-16)
    assert_csr_equal(A.to_host(), port.build_csr(hp, got, got, 1e-16))

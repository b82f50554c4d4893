"""The oracle port against the compiled reference on the CPU at the n = 48
(12 alpha / 12 beta) shape, where spin strings use bits 32..63 of their
words, and the port's bitset<256> path against the same problem embedded in
256-bit words. This pins the port that the n = 100 bitset<256> GPU tests
use as their only check (the reference cannot instantiate bitset<256>,
include/macis/bitset_operations.hpp:266-283)."""
import numpy as np
import pytest

import macis_b200 as mb
import oracle
from cases import abs_sums, assert_csr_equal, core_set, embed


@pytest.fixture(scope="module")
def n48(port, ref):
    n, k = 48, 12
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, 8, 128)
    hr = ref.ham(128, n, T, V)
    E0 = float(ref.matrix_element(hr, cd[:1], cd[:1])[0]) - 0.5
    return dict(n=n, T=T, V=V, cd=cd, C=C, hr=hr, E0=E0,
                hp=port.ham(128, n, T, V), hp256=port.ham(256, n, T, V))


def test_port_pairs_match_reference_n48(n48, port, ref):
    s = oracle.AsciSettings.default()
    args = (n48["cd"], n48["E0"], n48["C"])
    ps, pr = port.asci_pairs(n48["hp"], s, *args)
    rs, rr = ref.asci_pairs(n48["hr"], s, *args)
    u, scale = abs_sums(*port.asci_pairs(n48["hp"], s, *args,
                                         accumulate=False))
    assert len(ps) > 500_000
    assert np.array_equal(ps, rs) and np.array_equal(ps, u)
    assert np.all(np.abs(pr - rr) <= 1e-13 * scale)
    # 256-bit words, same problem: the same scores bit for bit
    s4, r4 = port.asci_pairs(n48["hp256"], s, embed(n48["cd"], 128, 256),
                             n48["E0"], n48["C"])
    assert np.array_equal(embed(s4, 256, 128), ps)
    assert np.array_equal(r4, pr)


def test_port_search_and_csr_match_reference_n48(n48, port, ref):
    s = oracle.AsciSettings.default()
    args = (n48["cd"], n48["E0"], n48["C"])
    got = port.asci_search(n48["hp"], s, 3000, *args)
    r = ref.asci_search(n48["hr"], s, 3000, *args)
    assert len(got) == len(r) == 3000
    key = lambda a: set(map(tuple, np.asarray(a).tolist()))
    assert len(key(got) ^ key(r)) <= 2      # at most one swapped near-tie
    g4 = port.asci_search(n48["hp256"], s, 3000, embed(n48["cd"], 128, 256),
                          n48["E0"], n48["C"])
    assert np.array_equal(embed(g4, 256, 128), got)
    A = ref.build_csr(n48["hr"], got, got, 1e-16, nthreads=4)
    assert_csr_equal(port.build_csr(n48["hp"], got, got, 1e-16), A)
    g256 = embed(got, 128, 256)
    assert_csr_equal(port.build_csr(n48["hp256"], g256, g256, 1e-16), A)

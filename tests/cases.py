"""Seeded synthetic problems shared by the parity tests."""
import numpy as np

from macis_b200.integrals import synthetic_integrals
from macis_b200.sd import generate_hilbert_space, make_dets, split_dets


def embed(dets, nbits_from, nbits_to):
    """Re-pack determinants into a wider bitset (same orbitals)."""
    a, b = split_dets(dets, nbits_from)
    return make_dets(a, b, nbits_to)


def fci(norb, na, nb, nbits=64, seed=0):
    T, V = synthetic_integrals(norb, seed)
    return T, V, generate_hilbert_space(norb, na, nb, nbits)


def shuffled(dets, seed=1, frac=1.0):
    rng = np.random.default_rng(seed)
    idx = rng.permutation(len(dets))[: int(len(dets) * frac)]
    return dets[idx]


def assert_csr_equal(a, b, exact=True):
    (ra, ca, za), (rb, cb, zb) = a, b
    assert np.array_equal(np.asarray(ra, np.int64), np.asarray(rb, np.int64))
    assert np.array_equal(np.asarray(ca, np.int64), np.asarray(cb, np.int64))
    if exact:
        assert np.array_equal(np.asarray(za, np.float64),
                              np.asarray(zb, np.float64))
    else:
        np.testing.assert_allclose(za, zb, rtol=1e-12, atol=1e-14)

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


def core_set(norb, nel, ncore, nbits=128, seed=0, nalpha=60, top=30):
    """A core set shaped like the ASCI core of a large active space: the HF
    determinant of `nel` alpha and `nel` beta electrons in `norb` orbitals
    and products of its low single / double excitations, ordered by total
    excitation degree, with decaying normalised coefficients. Returns
    (dets, C)."""
    rng = np.random.default_rng(seed)
    hf = (1 << nel) - 1
    strings = {hf}
    while len(strings) < nalpha:
        a = hf
        for _ in range(int(rng.integers(1, 3))):
            i, v = int(rng.integers(0, nel)), int(rng.integers(nel, norb))
            if a >> i & 1 and not a >> v & 1:
                a ^= (1 << i) ^ (1 << v)
        strings.add(a)
    strings = sorted(strings, key=lambda x: (bin(x ^ hf).count("1"), x))
    deg = lambda ab: (bin(ab[0] ^ hf).count("1") + bin(ab[1] ^ hf).count("1"),
                      ab)
    pairs = sorted(((a, b) for a in strings[:top] for b in strings[:top]),
                   key=deg)[:ncore]
    dets = make_dets([a for a, _ in pairs], [b for _, b in pairs], nbits)
    C = np.exp(-0.5 * np.arange(len(dets)) / 10.0)
    return dets, C / np.linalg.norm(C)


def abs_sums(states, rv):
    """Unique states of a raw contribution list in ascending bitset order
    (the order of sort_and_accumulate_asci_pairs) and, per state, the sum of
    |rv| over its contributions: the scale of the rounding error of any
    summation order of that state's score."""
    nw = states.shape[1]
    order = np.lexsort(tuple(states[:, w] for w in range(nw)))
    s, a = states[order], np.abs(rv[order])
    new = np.ones(len(s), dtype=bool)
    new[1:] = np.any(s[1:] != s[:-1], axis=1)
    idx = np.flatnonzero(new)
    return s[idx], np.add.reduceat(a, idx) if len(a) else a


def reference_mpi_selection(parts, cdets, ndets_max):
    """The selection of the reference's MPI asci_search (world size > 1,
    include/macis/asci/determinant_search.hpp:528-654) from every rank's
    accumulated (states, rv) pairs: per rank, rv -> -|rv| and the core
    determinants are dropped (keep_only_largest_copy_asci_pairs + partition);
    the k-th largest |rv| over all ranks (dist_quickselect,
    util/dist_quickselect.hpp) with k = ndets_max - ncore; every rank keeps
    its pairs with |rv| >= that score; the gathered states (rank order) are
    cut at k when ties at the score overflow it; the core determinants
    follow. Returns the determinant array."""
    cdets = np.ascontiguousarray(cdets)
    vt = np.dtype((np.void, cdets.shape[1] * 8))
    core = cdets.view(vt).ravel()
    kept = []
    for st, rv in parts:
        st = np.ascontiguousarray(st)
        keep = ~np.isin(st.view(vt).ravel(), core)
        kept.append((st[keep], np.abs(rv[keep])))
    k = ndets_max - len(cdets)
    allv = np.concatenate([v for _, v in kept])
    if len(allv) <= k:
        sel = [s for s, _ in kept]
    else:
        kth = np.sort(allv)[::-1][k - 1]
        sel = [s[v >= kth] for s, v in kept]
    sel = np.concatenate(sel)[:k] if sel else np.zeros((0, cdets.shape[1]),
                                                        dtype=np.uint64)
    return np.concatenate([sel, np.ascontiguousarray(cdets)])

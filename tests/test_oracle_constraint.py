"""The reference's MPI-only constraint-partitioned ASCI contributions
(asci_contributions_constraint, include/macis/asci/determinant_search.hpp:
143-391, with the rank split of dist_constraint_general,
asci/mask_constraints.hpp:486-605), run for every rank of a 1-, 2- and
4-rank job in one process against a serial MPI stand-in, on the CPU:
the ranks' candidate sets are disjoint and together are the standard path's
(asci_contributions_standard + sort_and_accumulate_asci_pairs), with scores
equal up to summation order on every candidate that is not itself a core
determinant (core determinants are dropped before the selection; on water
the constraint path scores the HF determinant differently). This pins the
partition that the split-search
GPU tests compare the hash-bin split against."""
import numpy as np
import pytest

import macis_b200 as mb
import oracle
from cases import abs_sums, core_set, reference_mpi_selection
from golden_data import water


@pytest.fixture(scope="module")
def refc():
    if not oracle.ref_constraint_available():
        pytest.skip("compiled reference oracle/_ref not built")
    return oracle.ref_constraint()


def _problems(port):
    n, k = 48, 12
    T, V = mb.synthetic_integrals(n, 0)
    cd, C = core_set(n, k, 8, 128)
    yield "n48", 128, n, T, V, cd, C
    norb, T, V, _ = water()
    cd = port.cisd_space(64, norb, 5, 5)[:60]
    yield "water", 64, norb, T, V, cd, np.linspace(1.0, 0.05, len(cd))


@pytest.mark.parametrize("world", [1, 2, 4])
def test_constraint_parts_partition_the_standard_pairs(ref, refc, port, world):
    s = oracle.AsciSettings.default()
    for name, nbits, n, T, V, cd, C in _problems(port):
        hr, hc = ref.ham(nbits, n, T, V), refc.ham(nbits, n, T, V)
        hp = port.ham(nbits, n, T, V)
        E0 = float(ref.matrix_element(hr, cd[:1], cd[:1])[0]) - 0.5
        parts = [refc.asci_pairs(hc, s, cd, E0, C, r, world)
                 for r in range(world)]
        assert all(len(p[0]) for p in parts), name
        st = np.concatenate([p[0] for p in parts])
        rv = np.concatenate([p[1] for p in parts])
        u, _ = abs_sums(st, rv)
        assert len(u) == len(st), name        # no state on two ranks
        rs, rr = ref.asci_pairs(hr, s, cd, E0, C)
        assert np.array_equal(u, rs), name
        order = np.lexsort(tuple(st[:, w] for w in range(st.shape[1])))
        us, scale = abs_sums(*port.asci_pairs(hp, s, cd, E0, C,
                                              accumulate=False))
        assert np.array_equal(us, rs)
        # scores agree up to summation order, except possibly on candidates
        # that are core determinants themselves (water: the HF determinant),
        # which both paths drop before the selection
        off = np.abs(rv[order] - rr) > 1e-13 * scale
        core = set(map(bytes, np.ascontiguousarray(cd)))
        assert all(bytes(x) in core for x in rs[off]), name
        # the MPI selection over the parts against the serial search
        ndets = 2000
        sel = reference_mpi_selection(parts, cd, ndets)
        whole = ref.asci_search(hr, s, ndets, cd, E0, C)
        key = lambda a: set(map(bytes, np.ascontiguousarray(a)))
        assert len(sel) == len(whole) == ndets
        assert len(key(sel) ^ key(whole)) <= 2, name

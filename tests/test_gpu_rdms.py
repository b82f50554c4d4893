"""1- and 2-RDMs (macis_b200_form_rdms) against the reference's own
DoubleLoopHamiltonianGenerator::form_rdms (double_loop.hpp:117-165),
compiled here: sums are atomic on the GPU, so the tolerance is 1e-12
(absolute, the RDM entries are O(1))."""
import numpy as np
import pytest

import macis_b200 as mb
from cases import fci, shuffled

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nbits", [64, 128])
def test_rdms_match_reference(ref, nbits):
    T, V, d = fci(7, 3, 3, nbits, seed=2)
    sel = shuffled(d, seed=3, frac=0.7).copy()
    sel[9] = 0                                  # zero determinant: skipped
    sel[20] = sel[21]                           # duplicate determinant
    C = np.random.default_rng(1).standard_normal(len(sel))
    C /= np.linalg.norm(C)
    C[5] = 1e-17                                # pairs below 1e-16 skipped
    H = mb.HamiltonianGenerator(T, V, nbits)
    hr = ref.ham(nbits, 7, T, V)
    for two in (True, False):
        o, t = H.form_rdms(sel, C, two=two)
        ro, rt = ref.form_rdms(hr, sel, C, two=two)
        np.testing.assert_allclose(o.ravel(order="F"), ro, rtol=0,
                                   atol=1e-12)
        if two:
            np.testing.assert_allclose(t.ravel(order="F"), rt, rtol=0,
                                       atol=1e-12)


def test_rdm_traces_and_energy(port):
    """Tr(1-RDM) = electrons; E = sum h D1 + 1/2 sum V D2 for the ground
    state (the reference's RDM-energy identity, cas.hpp)."""
    T, V, d = fci(6, 3, 2, 64, seed=4)
    H = mb.HamiltonianGenerator(T, V, 64)
    E, X = mb.selected_ci_diag(d, H, np.finfo(float).eps, 60, 1e-10)
    o, t = H.form_rdms(d, X)
    assert abs(np.trace(o) - 5) < 1e-10
    n = 6
    Tm = np.asarray(T).reshape(n, n, order="F")
    Vm = np.asarray(V).reshape(n, n, n, n, order="F")
    E_rdm = np.einsum("pq,pq", Tm, o) + np.einsum("pqrs,pqrs", Vm, t)
    assert abs(E_rdm - E) < 1e-8

"""Failure paths on the GPU, made to fail without a GPU fault.

* A barrier wait in the tensor-core kernels of the screening network that
  runs out: the wait limit (macis_b200_set_wait_limit_ns) is set to 1 ns, so
  the waits for weight chunks and MMA completions give up. The call returns
  MACIS_B200_ETIMEOUT after the kernel drained its copies and MMAs and freed
  its tensor memory; with the default limit the next calls reproduce the
  results from before, in the same process.
* Host-side injection (macis_b200_inject_fault): a device allocation that
  reports out-of-memory, and a lowered int32 index range. The C ABI returns
  MACIS_B200_ENOMEM / MACIS_B200_ECAPACITY with a message and leaves the
  library usable; selected_ci_diag falls back to the matrix-free operator on
  ENOMEM and to 64-bit indices on ECAPACITY (selected_ci_diag.hpp:146-171 is
  the reference step whose failure these replace).
"""
import ctypes as C

import numpy as np
import pytest

import macis_b200 as mb
from cases import fci, shuffled
from macis_b200 import _lib
from macis_b200._lib import LIB, check

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def _rand_rows(rng, n, din):
    X = np.zeros((n, din), dtype=np.float32)
    X[:, :din - 64] = rng.integers(0, 2, (n, din - 64))
    X[:, din - 64:] = rng.normal(0, 1, (n, 64))
    u = X.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


@pytest.fixture
def short_waits():
    def set_ns(ns):
        check(LIB.macis_b200_set_wait_limit_ns(ns))
    yield set_ns
    set_ns(0)


@pytest.fixture
def faults():
    def inject(kind, arg=0):
        check(LIB.macis_b200_inject_fault(kind, arg))
    yield inject
    inject(_lib.FAULT_NONE)


def test_network_wait_timeout_then_recovery(short_waits):
    rng = np.random.default_rng(4)
    net = mb.ScreeningNetwork(din=192, seed=2)
    X = _rand_rows(rng, 1 << 16, 192)
    t = rng.normal(0, 1, 4096).astype(np.float32)
    y0 = net.forward(X)
    g0, l0 = net.gradients(X[:4096], t)
    short_waits(1)
    with pytest.raises(mb.MacisError) as e:
        net.forward(X)
    assert e.value.code == _lib.ETIMEOUT
    assert "timed out" in str(e.value)
    # the training GEMMs bound their waits the same way: whether or not one
    # of them ran out, the call ends with a status and the next ones work
    try:
        net.gradients(X[:4096], t)
    except mb.MacisError as e2:
        assert e2.code == _lib.ETIMEOUT
    short_waits(0)
    for _ in range(2):
        assert np.array_equal(net.forward(X), y0)
    g1, l1 = net.gradients(X[:4096], t)
    assert np.array_equal(g1, g0) and abs(l1 - l0) <= 1e-12 * abs(l0)


def test_screened_search_wait_timeout_then_recovery(short_waits):
    T, V, dets = fci(10, 4, 4, 64, seed=3)
    H = mb.HamiltonianGenerator(T, V, 64)
    core = dets[:300]
    C = np.linspace(1.0, 0.1, len(core))
    net = mb.ScreeningNetwork(nbits=64, seed=0)
    sc = mb.ScreenSettings(network=net, keep_frac=0.5, explore_frac=0.0,
                           train=False)
    s = mb.ASCISettings()
    before = mb.asci_search(s, 2000, core, -5.0, C, 10, H, screen=sc,
                            use_net=True)
    short_waits(1)
    with pytest.raises(mb.MacisError) as e:
        mb.asci_search(s, 2000, core, -5.0, C, 10, H, screen=sc, use_net=True)
    assert e.value.code == _lib.ETIMEOUT
    short_waits(0)
    after = mb.asci_search(s, 2000, core, -5.0, C, 10, H, screen=sc,
                           use_net=True)
    assert np.array_equal(after, before)


def test_injected_out_of_memory(faults):
    T, V, d = fci(9, 4, 4, 64, seed=5)
    sel = shuffled(d, seed=2, frac=0.6).copy()
    H = mb.HamiltonianGenerator(T, V, 64)
    A0 = mb.make_csr_hamiltonian(sel, H, EPS)
    ref = A0.to_host()
    # the C ABI: the build's third allocation fails, with status and message
    faults(_lib.FAULT_ALLOC, 2)
    c = C.c_void_p()
    rc = LIB.macis_b200_build_csr(H.handle, sel.ctypes.data, len(sel),
                                  sel.ctypes.data, len(sel), EPS, 4, 8, 0,
                                  C.byref(c))
    assert rc == _lib.ENOMEM and not c.value
    assert b"out of memory" in LIB.macis_b200_last_error()
    # once fired, the injection is off: the same build now succeeds
    A1 = mb.make_csr_hamiltonian(sel, H, EPS)
    for a, b in zip(A1.to_host(), ref):
        assert np.array_equal(a, b)
    # an ASCI search that runs out of memory part way leaves no state behind
    s = mb.ASCISettings()
    core, Cc = sel[:40], np.linspace(1.0, 0.1, 40)
    whole = mb.asci_search(s, 3000, core, -20.0, Cc, 9, H)
    faults(_lib.FAULT_ALLOC, 6)
    with pytest.raises(mb.MacisError) as e:
        mb.asci_search(s, 3000, core, -20.0, Cc, 9, H)
    assert e.value.code == _lib.ENOMEM
    assert np.array_equal(mb.asci_search(s, 3000, core, -20.0, Cc, 9, H),
                          whole)
    # selected_ci_diag: the CSR build's failure sends it to the matrix-free
    # operator, with the same energy
    E0, X0 = mb.selected_ci_diag(sel, H, EPS, 80, 1e-8)
    faults(_lib.FAULT_ALLOC, 0)
    t = {}
    E1, X1 = mb.selected_ci_diag(sel, H, EPS, 80, 1e-8, timings=t)
    assert t["nnz"] is None and abs(E1 - E0) < 1e-9


def test_injected_int32_capacity(faults):
    T, V, d = fci(9, 4, 4, 64, seed=5)
    H = mb.HamiltonianGenerator(T, V, 64)
    dav = dict(restart_keep=8, max_iter=3000)
    E0, _ = mb.selected_ci_diag(d, H, EPS, 40, 1e-8, **dav)
    A = mb.make_csr_hamiltonian(d, H, EPS)
    faults(_lib.FAULT_INT32_LIMIT, A.nnz - 1)
    with pytest.raises(mb.MacisError) as e:
        mb.make_csr_hamiltonian(d, H, EPS)
    assert e.value.code == _lib.ECAPACITY and "int32" in str(e.value)
    A64 = mb.make_csr_hamiltonian(d, H, EPS, index_t=np.int64)
    assert A64.nnz == A.nnz
    # index_t=None: int32 first, int64 after the capacity error, remembered
    # for later spaces of this generator
    t = {}
    E1, _ = mb.selected_ci_diag(d, H, EPS, 40, 1e-8, index_t=None, timings=t,
                                **dav)
    assert abs(E1 - E0) < 1e-9 and t["nnz"] == A.nnz
    assert H._int64_from_ndets == len(d)

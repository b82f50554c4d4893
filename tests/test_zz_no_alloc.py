"""The allocation-free mixed-precision SpMV (macis_b200_spmv_mixed_noalloc)
against the regular entry point, through the C ABI.

It serves callers that may not allocate device memory while they run; its
scratch (the FP32 copy of x) is a fixed array inside the library. This file
is collected last so that a stop-at-first-failure run has already run every
other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import macis_b200 as mb
from macis_b200 import _lib
from macis_b200._lib import LIB, check

pytestmark = pytest.mark.gpu


def test_noalloc_spmv_matches_regular_entry_point():
    import torch
    T, V = mb.synthetic_integrals(9, seed=7)
    dets = mb.generate_hilbert_space(9, 4, 4, 64)             # 15,876 dets
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps,
                                value_t=np.float32)
    rng = np.random.default_rng(3)
    for call in range(2):                                     # two calls in a row
        x = torch.tensor(rng.standard_normal(A.n), dtype=torch.float64,
                         device="cuda")
        y0 = torch.tensor(rng.standard_normal(A.m), dtype=torch.float64,
                          device="cuda")
        y_ref, y_new = y0.clone(), y0.clone()
        check(LIB.macis_b200_spmv(A.handle, 1, 0.7, x.data_ptr(), A.n, 0.3,
                                  y_ref.data_ptr(), A.m, _lib.DEVICE_PTRS))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        check(LIB.macis_b200_spmv_mixed_noalloc(A.handle, 0.7, x.data_ptr(),
                                                0.3, y_new.data_ptr()))
        # once the SpMV code is resident on the device (the regular product
        # above), the call takes no device memory
        assert torch.cuda.mem_get_info()[0] == free0
        torch.cuda.synchronize()
        np.testing.assert_allclose(y_new.cpu().numpy(), y_ref.cpu().numpy(),
                                   rtol=1e-12, atol=1e-12)


def test_noalloc_spmv_column_limit_and_empty_ket_list():
    import torch
    T, V = mb.synthetic_integrals(14, seed=2)
    kets = mb.generate_hilbert_space(14, 7, 7, 64)     # 11,778,624 columns
    assert len(kets) > 4_194_304
    H = mb.HamiltonianGenerator(T, V, 64)
    big = mb.make_csr_hamiltonian_block(kets[:2], kets, H,
                                        np.finfo(float).eps,
                                        value_t=np.float32)
    x = torch.ones(big.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(big.m, dtype=torch.float64, device="cuda")
    rc = LIB.macis_b200_spmv_mixed_noalloc(big.handle, 1.0, x.data_ptr(), 0.0,
                                           y.data_ptr())
    assert rc == _lib.ECAPACITY
    assert b"4,194,304" in LIB.macis_b200_last_error()
    # the rejected call leaves the library usable: the regular product of
    # the same block, and an allocation-free product of a block with rows
    # but no columns (y = beta y)
    check(LIB.macis_b200_spmv(big.handle, 1, 1.0, x.data_ptr(), big.n, 0.0,
                              y.data_ptr(), big.m, _lib.DEVICE_PTRS))
    assert np.all(np.isfinite(y.cpu().numpy())) and y.abs().sum().item() > 0
    empty = mb.make_csr_hamiltonian_block(kets[:3], kets[:0], H,
                                          np.finfo(float).eps,
                                          value_t=np.float32)
    assert (empty.m, empty.n, empty.nnz) == (3, 0, 0)
    y3 = torch.tensor([1.0, -2.0, 4.0], dtype=torch.float64, device="cuda")
    check(LIB.macis_b200_spmv_mixed_noalloc(empty.handle, 0.5, x.data_ptr(),
                                            0.25, y3.data_ptr()))
    assert y3.cpu().tolist() == [0.25, -0.5, 1.0]


def test_noalloc_spmv_rejects_fp64_matrix():
    import torch
    T, V = mb.synthetic_integrals(6, seed=1)
    dets = mb.generate_hilbert_space(6, 3, 3, 64)
    H = mb.HamiltonianGenerator(T, V, 64)
    A = mb.make_csr_hamiltonian(dets, H, np.finfo(float).eps)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    rc = LIB.macis_b200_spmv_mixed_noalloc(A.handle, 1.0, x.data_ptr(), 0.0,
                                           y.data_ptr())
    assert rc == _lib.EINVAL
    assert b"FP32" in LIB.macis_b200_last_error()

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
    for _ in range(2):                                        # two calls in a row
        x = torch.tensor(rng.standard_normal(A.n), dtype=torch.float64,
                         device="cuda")
        y0 = torch.tensor(rng.standard_normal(A.m), dtype=torch.float64,
                          device="cuda")
        y_ref, y_new = y0.clone(), y0.clone()
        check(LIB.macis_b200_spmv(A.handle, 1, 0.7, x.data_ptr(), A.n, 0.3,
                                  y_ref.data_ptr(), A.m, _lib.DEVICE_PTRS))
        check(LIB.macis_b200_spmv_mixed_noalloc(A.handle, 0.7, x.data_ptr(),
                                                0.3, y_new.data_ptr()))
        torch.cuda.synchronize()
        np.testing.assert_allclose(y_new.cpu().numpy(), y_ref.cpu().numpy(),
                                   rtol=1e-12, atol=1e-12)


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

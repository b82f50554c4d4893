"""macis_b200 -- the selected-CI hot path of MACIS on one NVIDIA B200.

Hand-written sm_100a kernels behind a C ABI (include/macis_b200.h, built
into libmacis_b200.so by ``python macis_b200/build.py``), with this package
as the host side mirroring MACIS's own API:

    HamiltonianGenerator, make_csr_hamiltonian_block, make_csr_hamiltonian,
    SparseMatrixOperator, diagonal_guess, davidson, selected_ci_diag,
    ASCISettings, MCSCFSettings, asci_search, asci_iter, asci_grow,
    asci_refine

plus the learned screening of the ASCI search (ScreeningNetwork,
ScreenSettings), which has no MACIS counterpart.

Importing the package loads the native library and fails if it is missing.
"""
from ._lib import MacisError  # noqa: F401  (loads libmacis_b200.so)
from .asci import (ASCISettings, MCSCFSettings, asci_grow, asci_iter,  # noqa
                   asci_pairs, asci_refine, asci_search, asci_search_part,
                   last_search_stats, merge_asci_parts, reorder_ci_on_coeff,
                   topk_recall)
from .hamiltonian import (DeviceCSR, HamiltonianGenerator,  # noqa: F401
                          MatrixFreeHamiltonian, make_csr_hamiltonian,
                          make_csr_hamiltonian_block, row_bounds)
from .integrals import fcidump_fill, synthetic_integrals  # noqa: F401
from .screening import (ScreeningNetwork, ScreenSettings,  # noqa: F401
                        unit_features, unit_width)
from .sd import (canonical_hf_determinant, from_canonical_string,  # noqa
                 generate_cisd_hilbert_space, generate_hilbert_space,
                 to_canonical_string)
from .solvers import (FP64, MIXED, SparseMatrixOperator,  # noqa: F401
                      davidson, davidson_stats, diagonal_guess,
                      selected_ci_diag, small_syev)

__version__ = "0.1.0"

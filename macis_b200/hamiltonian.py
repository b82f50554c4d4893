"""Hamiltonian generator and CSR Hamiltonian on the B200.

Mirrors the reference API:

* ``HamiltonianGenerator`` -- DoubleLoopHamiltonianGenerator<N>
  (include/macis/hamiltonian_generator/double_loop.hpp:17) over HBM-resident
  integrals; ``make_csr_hamiltonian_block`` is the virtual build hook
  (include/macis/hamiltonian_generator.hpp:66-72, 143-156).
* ``make_csr_hamiltonian_block`` / ``make_csr_hamiltonian`` -- the free
  functions of include/macis/csr_hamiltonian.hpp:23-45.
* ``DeviceCSR`` -- the sparsexx::csr_matrix<double, index_t> result, kept in
  HBM (``to_host`` gives the by-value arrays of the reference).
* ``MatrixFreeHamiltonian`` -- H over one determinant list without storing
  it, for lists whose CSR matrix does not fit in device memory: the operator
  the reference's davidson accepts (include/macis/solvers/davidson.hpp:
  47-58, 129).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import LIB, check

__all__ = ["HamiltonianGenerator", "DeviceCSR", "make_csr_hamiltonian_block",
           "make_csr_hamiltonian", "row_bounds", "MatrixFreeHamiltonian"]


def row_bounds(M, world_size, rank):
    """Row block [lo, hi) of `rank`: M // world_size rows each, the last rank
    takes the remainder (the default partition of the reference's
    dist_sparse_matrix, sparsexx/matrix_types/dist_sparse_matrix.hpp:47-62,
    used by make_dist_csr_hamiltonian, csr_hamiltonian.hpp:49-82)."""
    per = M // world_size
    lo = rank * per
    hi = lo + per + (M % world_size if rank == world_size - 1 else 0)
    return lo, hi


def _dev_ptr(a):
    """Device pointer of a torch CUDA tensor, else None."""
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return a.data_ptr()
    return None


def _host_dets(d, nbits):
    d = np.ascontiguousarray(d, dtype=np.uint64)
    return d.reshape(-1, nbits // 64)


class HamiltonianGenerator:
    """Integrals T (n x n) and V (n^4), column-major, uploaded to HBM with
    the reference intermediates G, G_red, V_red, G2_red, V2_red
    (hamiltonian_generator/impl.hpp:26-70)."""

    def __init__(self, T, V, nbits=64, norb=None):
        T = np.asarray(T, dtype=np.float64)
        V = np.asarray(V, dtype=np.float64)
        if norb is None:
            norb = T.shape[0] if T.ndim == 2 else int(round(T.size ** 0.5))
        self.norb = int(norb)
        self.nbits = int(nbits)
        self.T = np.ascontiguousarray(T.reshape(-1, order="F") if T.ndim > 1
                                      else T)
        self.V = np.ascontiguousarray(V.reshape(-1, order="F") if V.ndim > 1
                                      else V)
        if self.T.size != self.norb ** 2 or self.V.size != self.norb ** 4:
            raise RuntimeError("V has incorrect dimensions")
        h = C.c_void_p()
        check(LIB.macis_b200_ham_create(
            self.nbits, self.norb, self.T.ctypes.data_as(_lib._pd), self.norb,
            self.V.ctypes.data_as(_lib._pd), self.norb, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            LIB.macis_b200_ham_destroy(h)
            self._h = None

    # -- matrix elements (matrix_elements.hpp:15-32)
    def matrix_element(self, bra, ket):
        bra = _host_dets(bra, self.nbits)
        ket = _host_dets(ket, self.nbits)
        out = np.empty(len(bra))
        check(LIB.macis_b200_matrix_element(
            self._h, bra.ctypes.data, ket.ctypes.data, len(bra),
            out.ctypes.data, 0))
        return out if len(out) > 1 else float(out[0])

    # -- form_rdms (double_loop.hpp:117-165, bra = ket = dets)
    def form_rdms(self, dets, C, two=True):
        """(ordm, trdm) of the wavefunction C over dets: norb x norb and
        norb^4 arrays indexed as the reference's spans (column-major);
        trdm is None when two is False. Contributions and their dispatch
        follow include/macis/util/rdms.hpp:15-131 (with two=False the
        reference routes higher excitations into its one-body branches,
        and so does this); sums are atomic, so values agree with the
        reference to rounding."""
        d = _host_dets(dets, self.nbits)
        C = np.ascontiguousarray(C, dtype=np.float64)
        if len(C) != len(d):
            raise RuntimeError("C and dets differ in length")
        n = self.norb
        o = np.zeros(n * n)
        t = np.zeros(n ** 4) if two else None
        check(LIB.macis_b200_form_rdms(self._h, d.ctypes.data, len(d),
                                       C.ctypes.data, o.ctypes.data,
                                       t.ctypes.data if two else None, 0))
        return (o.reshape(n, n, order="F"),
                t.reshape(n, n, n, n, order="F") if two else None)

    # -- CSR build hook (hamiltonian_generator.hpp:143-156)
    def make_csr_hamiltonian_block(self, bra, ket, H_thresh, index_t=np.int32,
                                   value_t=np.float64):
        return DeviceCSR.build(self, bra, ket, H_thresh, index_t, value_t)


class DeviceCSR:
    """CSR Hamiltonian held in HBM by libmacis_b200."""

    def __init__(self, handle, ham=None):
        self._c = handle
        self.ham = ham
        m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        ib, vb = C.c_int(), C.c_int()
        check(LIB.macis_b200_csr_info(handle, C.byref(m), C.byref(n),
                                      C.byref(nnz), C.byref(ib), C.byref(vb)))
        self.m, self.n, self.nnz = m.value, n.value, nnz.value
        self.index_t = np.int32 if ib.value == 4 else np.int64
        self.value_t = np.float64 if vb.value == 8 else np.float32

    @classmethod
    def build(cls, ham, bra, ket, H_thresh, index_t=np.int32,
              value_t=np.float64):
        ib = np.dtype(index_t).itemsize
        if ib not in (4, 8):
            raise RuntimeError("Unsupported index_t")
        vb = np.dtype(value_t).itemsize
        flags = 0
        pb, pk = _dev_ptr(bra), _dev_ptr(ket)
        if pb is not None:
            flags = _lib.DEVICE_PTRS
            nbra = bra.numel() * 8 // (ham.nbits // 8)
            nket = ket.numel() * 8 // (ham.nbits // 8)
            keep = (bra, ket)
        else:
            same = bra is ket
            bra = _host_dets(bra, ham.nbits)
            ket = bra if same else _host_dets(ket, ham.nbits)
            pb, pk = bra.ctypes.data, ket.ctypes.data
            nbra, nket = len(bra), len(ket)
            keep = (bra, ket)
        c = C.c_void_p()
        check(LIB.macis_b200_build_csr(ham.handle, pb, nbra, pk, nket,
                                       float(H_thresh), ib, vb, flags,
                                       C.byref(c)))
        del keep
        return cls(c, ham)

    @property
    def handle(self):
        return self._c

    def __del__(self):
        c = getattr(self, "_c", None)
        if c:
            LIB.macis_b200_csr_destroy(c)
            self._c = None

    def to_host(self):
        """(rowptr, colind, nzval) numpy arrays (sparsexx csr_matrix data)."""
        rp = np.empty(self.m + 1, dtype=self.index_t)
        ci = np.empty(max(self.nnz, 1), dtype=self.index_t)
        nz = np.empty(max(self.nnz, 1), dtype=self.value_t)
        check(LIB.macis_b200_csr_download(self._c, rp.ctypes.data,
                                          ci.ctypes.data, nz.ctypes.data, 0))
        return rp, ci[:self.nnz], nz[:self.nnz]

    def rows(self, r0, r1):
        """(rowptr, colind, nzval) of rows [r0, r1) as numpy arrays, rowptr
        rebased to start at 0 (the local CSR of that row block)."""
        if not 0 <= r0 <= r1 <= self.m:
            raise ValueError("row range outside the matrix")
        rp = np.empty(r1 - r0 + 1, dtype=self.index_t)
        check(LIB.macis_b200_csr_download_rows(self._c, r0, r1, rp.ctypes.data,
                                               None, None, 0))
        k = int(rp[-1] - rp[0])
        ci = np.empty(max(k, 1), dtype=self.index_t)
        nz = np.empty(max(k, 1), dtype=self.value_t)
        check(LIB.macis_b200_csr_download_rows(self._c, r0, r1, None,
                                               ci.ctypes.data, nz.ctypes.data,
                                               0))
        return rp - rp[0], ci[:k], nz[:k]

    def diagonal(self):
        """extract_diagonal_elements (sparsexx/util/submatrix.hpp:264-292)."""
        d = np.empty(self.m)
        check(LIB.macis_b200_csr_diagonal(self._c, d.ctypes.data, 0))
        return d

    def build_stats(self):
        """Timings and path of the build (CUDA events on the build stream)."""
        st = _lib.BuildStatsC()
        check(LIB.macis_b200_csr_build_stats(self._c, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def mem_footprint(self):
        ib = np.dtype(self.index_t).itemsize
        vb = np.dtype(self.value_t).itemsize
        return (self.m + 1) * ib + self.nnz * (ib + vb)

    def spmv(self, x, alpha=1.0, beta=0.0, y=None):
        """alpha * A x + beta * y (gespmbv with K = 1) on host vectors."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.m) if y is None else np.array(y, dtype=np.float64)
        check(LIB.macis_b200_spmv(self._c, 1, alpha, x.ctypes.data, self.n,
                                  beta, y.ctypes.data, self.m, 0))
        return y


def make_csr_hamiltonian_block(bra, ket, ham_gen, H_thresh, index_t=np.int32,
                               value_t=np.float64):
    """csr_hamiltonian.hpp:23-37 (the empty-input guard is in the library)."""
    return ham_gen.make_csr_hamiltonian_block(bra, ket, H_thresh, index_t,
                                              value_t)


def make_csr_hamiltonian(dets, ham_gen, H_thresh, index_t=np.int32,
                         value_t=np.float64):
    """csr_hamiltonian.hpp:39-45: square block over one determinant list."""
    return ham_gen.make_csr_hamiltonian_block(dets, dets, H_thresh, index_t,
                                              value_t)


class MatrixFreeHamiltonian:
    """H over one determinant list, applied without storing it: every
    product evaluates the elements again from the determinants and the
    integrals (same enumeration, Slater-Condon rules and threshold as the
    CSR build). value_t=np.float32 rounds the off-diagonal elements to FP32
    as an FP32-valued CSR matrix would (the diagonal stays FP64). Products
    agree with the CSR product to rounding (sums in enumeration order)."""

    def __init__(self, dets, ham_gen, H_thresh, value_t=np.float64):
        flags = _lib.HOP_FP32 if np.dtype(value_t) == np.float32 else 0
        p = _dev_ptr(dets)
        if p is not None:
            flags |= _lib.DEVICE_PTRS
            n = dets.numel() * 8 // (ham_gen.nbits // 8)
            keep = dets
        else:
            keep = _host_dets(dets, ham_gen.nbits)
            p, n = keep.ctypes.data, len(keep)
        h = C.c_void_p()
        check(LIB.macis_b200_hop_create(ham_gen.handle, p, n, float(H_thresh),
                                        flags, C.byref(h)))
        del keep
        self._h = h
        self.ham = ham_gen
        self.m = self.n = int(n)
        self.value_t = np.float32 if flags & _lib.HOP_FP32 else np.float64

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            LIB.macis_b200_hop_destroy(h)
            self._h = None

    def diagonal(self):
        d = np.empty(self.m)
        check(LIB.macis_b200_hop_diagonal(self._h, d.ctypes.data, 0))
        return d

    def spmv(self, x, alpha=1.0, beta=0.0, y=None):
        """alpha * H x + beta * y on host vectors."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.m) if y is None else np.array(y, dtype=np.float64)
        check(LIB.macis_b200_hop_apply(self._h, 1, alpha, x.ctypes.data,
                                       self.n, beta, y.ctypes.data, self.m, 0))
        return y

"""CPU oracle for the selected-CI hot path -- TEST INFRASTRUCTURE ONLY.

Two checkers, both CPU-only:

* ``port`` -- ``liboracle.so``, the plain-C restatement of the reference
  algorithms in ``macis_oracle.c`` (covers bitset<64/128/256>).
* ``ref``  -- ``_ref/libmacis_ref.so``, the unmodified reference MACIS headers
  compiled by ``ref/Makefile`` (bitset<64/128>; the reference cannot
  instantiate bitset<256>, include/macis/bitset_operations.hpp:267).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed
CPU baseline. The product package ``macis_b200`` never imports it.

Determinant arrays are numpy ``uint64`` of shape (ndets, nbits // 64) in the
std::bitset word layout; integrals are flat column-major float64 arrays.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libmacis_ref.so")
REFC_PATH = os.path.join(HERE, "_ref", "libmacis_ref_constraint.so")

_p64 = C.POINTER(C.c_uint64)
_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)
_pi32 = C.POINTER(C.c_int32)
_pu32 = C.POINTER(C.c_uint32)


class AsciSettings(C.Structure):
    """Mirror of macis::ASCISettings (asci/determinant_search.hpp:34-51)."""
    _fields_ = [("ntdets_max", C.c_uint64), ("ntdets_min", C.c_uint64),
                ("ncdets_max", C.c_uint64), ("h_el_tol", C.c_double),
                ("rv_prune_tol", C.c_double), ("pair_size_max", C.c_uint64),
                ("just_singles", C.c_int32), ("pad_", C.c_int32),
                ("grow_factor", C.c_uint64), ("max_refine_iter", C.c_uint64),
                ("refine_energy_tol", C.c_double)]

    @classmethod
    def default(cls, **kw):
        s = cls(ntdets_max=100000, ntdets_min=100, ncdets_max=100,
                h_el_tol=1e-8, rv_prune_tol=1e-8, pair_size_max=500000000,
                just_singles=0, pad_=0, grow_factor=8, max_refine_iter=6,
                refine_energy_tol=1e-6)
        for k, v in kw.items():
            setattr(s, k, v)
        return s


class CiSettings(C.Structure):
    """The CI fields of macis::MCSCFSettings (util/mcscf.hpp:27-29)."""
    _fields_ = [("ci_res_tol", C.c_double), ("ci_max_subspace", C.c_uint64),
                ("ci_matel_tol", C.c_double)]

    @classmethod
    def default(cls, **kw):
        s = cls(ci_res_tol=1e-8, ci_max_subspace=20,
                ci_matel_tol=float(np.finfo(np.float64).eps))
        for k, v in kw.items():
            setattr(s, k, v)
        return s


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _dets(d, nbits):
    d = np.ascontiguousarray(d, dtype=np.uint64)
    return d.reshape(-1, nbits // 64)


class Port:
    """ctypes front end of the C restatement (macis_oracle.h)."""

    def __init__(self, path=PORT_PATH):
        L = self.L = C.CDLL(path)
        L.orc_ham_create.restype = C.c_void_p
        L.orc_ham_create.argtypes = [C.c_int, C.c_size_t, _pd, _pd]
        L.orc_ham_free.argtypes = [C.c_void_p]
        L.orc_matrix_element.argtypes = [C.c_void_p, _p64, _p64, C.c_size_t, _pd]
        L.orc_build_csr.restype = C.c_int64
        L.orc_build_csr.argtypes = [C.c_void_p, _p64, C.c_size_t, _p64,
                                    C.c_size_t, C.c_double, _pi64, _pi64, _pd]
        L.orc_spmv.argtypes = [C.c_size_t, _pi64, _pi64, _pd, C.c_double, _pd,
                               C.c_double, _pd]
        L.orc_davidson.restype = C.c_int
        L.orc_davidson.argtypes = [C.c_size_t, _pi64, _pi64, _pd, C.c_int64,
                                   C.c_double, _pd, C.c_int, _pd, _pi64]
        L.orc_asci_pairs.restype = C.c_size_t
        L.orc_asci_pairs.argtypes = [C.c_void_p, C.POINTER(AsciSettings), _p64,
                                     C.c_size_t, C.c_double, _pd, C.c_int,
                                     _p64, _pd]
        L.orc_asci_search.restype = C.c_size_t
        L.orc_asci_search.argtypes = [C.c_void_p, C.POINTER(AsciSettings),
                                      C.c_size_t, _p64, C.c_size_t, C.c_double,
                                      _pd, _p64]
        L.orc_single_orbital_ens.argtypes = [C.c_void_p, _pu32, C.c_size_t,
                                             _pu32, C.c_size_t, _pd]
        for f in ("orc_fast_diag_single", "orc_fast_diag_ss_double",
                  "orc_fast_diag_os_double"):
            getattr(L, f).restype = C.c_double
        L.orc_fast_diag_single.argtypes = [C.c_void_p, C.c_double, C.c_double,
                                           C.c_uint32, C.c_uint32, C.c_double]
        L.orc_fast_diag_ss_double.argtypes = [C.c_void_p] + [C.c_double] * 4 + \
            [C.c_uint32] * 4 + [C.c_double]
        L.orc_fast_diag_os_double.argtypes = L.orc_fast_diag_ss_double.argtypes
        L.orc_hilbert_space.restype = C.c_size_t
        L.orc_hilbert_space.argtypes = [C.c_int, C.c_size_t, C.c_size_t,
                                        C.c_size_t, _p64]
        L.orc_cisd_space.restype = C.c_size_t
        L.orc_cisd_space.argtypes = L.orc_hilbert_space.argtypes
        L.orc_hf_det.argtypes = [C.c_int, C.c_size_t, C.c_size_t, _p64]

    # -- integrals / generator
    def ham(self, nbits, norb, T, V):
        T = np.ascontiguousarray(T, dtype=np.float64).ravel(order="K")
        V = np.ascontiguousarray(V, dtype=np.float64).ravel(order="K")
        h = self.L.orc_ham_create(nbits, norb, _ptr(T, _pd), _ptr(V, _pd))
        return Handle(h, self.L.orc_ham_free, nbits, norb)

    def matrix_element(self, h, bra, ket):
        bra, ket = _dets(bra, h.nbits), _dets(ket, h.nbits)
        out = np.empty(len(bra))
        self.L.orc_matrix_element(h.p, _ptr(bra, _p64), _ptr(ket, _p64),
                                  len(bra), _ptr(out, _pd))
        return out

    def build_csr(self, h, bra, ket, thresh):
        bra, ket = _dets(bra, h.nbits), _dets(ket, h.nbits)
        rp = np.zeros(len(bra) + 1, dtype=np.int64)
        nnz = self.L.orc_build_csr(h.p, _ptr(bra, _p64), len(bra),
                                   _ptr(ket, _p64), len(ket), thresh,
                                   _ptr(rp, _pi64), None, None)
        ci = np.empty(max(nnz, 1), dtype=np.int64)
        nz = np.empty(max(nnz, 1))
        r = self.L.orc_build_csr(h.p, _ptr(bra, _p64), len(bra),
                                 _ptr(ket, _p64), len(ket), thresh,
                                 _ptr(rp, _pi64), _ptr(ci, _pi64),
                                 _ptr(nz, _pd))
        assert r == nnz
        return rp, ci[:nnz], nz[:nnz]

    def spmv(self, rp, ci, nz, x, alpha=1.0, beta=0.0, y=None):
        rp = np.ascontiguousarray(rp, dtype=np.int64)
        ci = np.ascontiguousarray(ci, dtype=np.int64)
        nz = np.ascontiguousarray(nz, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        m = len(rp) - 1
        y = np.zeros(m) if y is None else np.array(y, dtype=np.float64)
        self.L.orc_spmv(m, _ptr(rp, _pi64), _ptr(ci, _pi64), _ptr(nz, _pd),
                        alpha, _ptr(x, _pd), beta, _ptr(y, _pd))
        return y

    def davidson(self, rp, ci, nz, max_m, tol, X=None):
        rp = np.ascontiguousarray(rp, dtype=np.int64)
        ci = np.ascontiguousarray(ci, dtype=np.int64)
        nz = np.ascontiguousarray(nz, dtype=np.float64)
        n = len(rp) - 1
        use = X is not None
        X = np.zeros(n) if X is None else np.array(X, dtype=np.float64)
        E = C.c_double()
        it = C.c_int64()
        rc = self.L.orc_davidson(n, _ptr(rp, _pi64), _ptr(ci, _pi64),
                                 _ptr(nz, _pd), max_m, tol, _ptr(X, _pd),
                                 int(use), C.byref(E), C.byref(it))
        if rc:
            raise RuntimeError("Davidson Did Not Converge!")
        return E.value, it.value, X

    def asci_pairs(self, h, s, cdets, E0, Cv, accumulate=True):
        cdets = _dets(cdets, h.nbits)
        Cv = np.ascontiguousarray(Cv, dtype=np.float64)
        n = self.L.orc_asci_pairs(h.p, C.byref(s), _ptr(cdets, _p64),
                                  len(cdets), E0, _ptr(Cv, _pd),
                                  int(accumulate), None, None)
        st = np.empty((max(n, 1), h.nbits // 64), dtype=np.uint64)
        rv = np.empty(max(n, 1))
        self.L.orc_asci_pairs(h.p, C.byref(s), _ptr(cdets, _p64), len(cdets),
                              E0, _ptr(Cv, _pd), int(accumulate),
                              _ptr(st, _p64), _ptr(rv, _pd))
        return st[:n], rv[:n]

    def asci_search(self, h, s, ndets_max, cdets, E0, Cv):
        cdets = _dets(cdets, h.nbits)
        Cv = np.ascontiguousarray(Cv, dtype=np.float64)
        out = np.empty((ndets_max + len(cdets), h.nbits // 64), dtype=np.uint64)
        n = self.L.orc_asci_search(h.p, C.byref(s), ndets_max,
                                   _ptr(cdets, _p64), len(cdets), E0,
                                   _ptr(Cv, _pd), _ptr(out, _p64))
        return out[:n]

    def single_orbital_ens(self, h, ss, os_):
        ss = np.ascontiguousarray(ss, dtype=np.uint32)
        os_ = np.ascontiguousarray(os_, dtype=np.uint32)
        eps = np.empty(h.norb)
        self.L.orc_single_orbital_ens(h.p, _ptr(ss, _pu32), len(ss),
                                      _ptr(os_, _pu32), len(os_),
                                      _ptr(eps, _pd))
        return eps

    def hilbert_space(self, nbits, norb, na, nb):
        n = self.L.orc_hilbert_space(nbits, norb, na, nb, None)
        out = np.empty((n, nbits // 64), dtype=np.uint64)
        self.L.orc_hilbert_space(nbits, norb, na, nb, _ptr(out, _p64))
        return out

    def cisd_space(self, nbits, norb, na, nb):
        n = self.L.orc_cisd_space(nbits, norb, na, nb, None)
        out = np.empty((n, nbits // 64), dtype=np.uint64)
        self.L.orc_cisd_space(nbits, norb, na, nb, _ptr(out, _p64))
        return out

    def hf_det(self, nbits, na, nb):
        out = np.zeros((1, nbits // 64), dtype=np.uint64)
        self.L.orc_hf_det(nbits, na, nb, _ptr(out, _p64))
        return out

    # -- drivers built from the primitives (selected_ci_diag.hpp:125-206,
    #    asci/iteration.hpp:17-68, grow.hpp:17-171, refine.hpp:15-66)
    def selected_ci_diag(self, h, dets, h_el_tol, max_m, tol):
        rp, ci, nz = self.build_csr(h, dets, dets, h_el_tol)
        E, it, X = self.davidson(rp, ci, nz, max_m, tol)
        return E, X

    def asci_iter(self, h, s, ci, ndets_max, E0, dets, X):
        dets = _dets(dets, h.nbits)
        X = np.asarray(X, dtype=np.float64)
        if len(dets) > 1:
            order = np.argsort(-np.abs(X), kind="stable")
            dets, X = dets[order], X[order]
        nkeep = min(s.ncdets_max, len(dets))
        dets = self.asci_search(h, s, ndets_max, dets[:nkeep], E0, X[:nkeep])
        E, X = self.selected_ci_diag(h, dets, ci.ci_matel_tol,
                                     ci.ci_max_subspace, ci.ci_res_tol)
        return E, dets, X

    def asci_grow(self, h, s, ci, E0, dets, X):
        dets = _dets(dets, h.nbits)
        while len(dets) < s.ntdets_max:
            nnew = min(max(s.ntdets_min, len(dets) * s.grow_factor),
                       s.ntdets_max)
            E, dets, X = self.asci_iter(h, s, ci, nnew, E0, dets, X)
            if nnew > len(dets):
                raise RuntimeError("Wavefunction didn't grow enough...")
            E0 = E
        return E0, dets, X

    def asci_refine(self, h, s, ci, E0, dets, X):
        ndets = len(dets)
        for _ in range(s.max_refine_iter):
            E, dets, X = self.asci_iter(h, s, ci, ndets, E0, dets, X)
            if len(dets) != ndets:
                raise RuntimeError("Wavefunction size can't change in refinement")
            dE = E - E0
            E0 = E
            if abs(dE) < s.refine_energy_tol:
                return E0, dets, X
        raise RuntimeError("ACCI Refine did not converge")


class Ref:
    """ctypes front end of the compiled reference (oracle/ref/ref_capi.cpp)."""

    def __init__(self, path=REF_PATH):
        L = self.L = C.CDLL(path)
        L.mref_last_error.restype = C.c_char_p
        L.mref_set_threads.argtypes = [C.c_int]
        L.mref_ham_create.restype = C.c_void_p
        L.mref_ham_create.argtypes = [C.c_int, C.c_size_t, _pd, _pd]
        L.mref_ham_free.argtypes = [C.c_void_p]
        L.mref_form_rdms.argtypes = [C.c_void_p, _p64, C.c_size_t, _pd, _pd,
                                     C.c_void_p]
        L.mref_matrix_element.argtypes = [C.c_void_p, _p64, _p64, C.c_size_t, _pd]
        L.mref_fast_diag.argtypes = [C.c_void_p, C.c_int, _pu32, C.c_size_t,
                                     _pu32, C.c_size_t, _pu32, C.c_double, _pd]
        L.mref_csr_build.restype = C.c_void_p
        L.mref_csr_build.argtypes = [C.c_void_p, _p64, C.c_size_t, _p64,
                                     C.c_size_t, C.c_double, C.c_int]
        L.mref_csr_nnz.restype = C.c_int64
        L.mref_csr_nnz.argtypes = [C.c_void_p]
        L.mref_csr_copy.argtypes = [C.c_void_p, _pi32, _pi32, _pd]
        L.mref_csr_free.argtypes = [C.c_void_p]
        L.mref_spmv.argtypes = [C.c_void_p, C.c_int64, C.c_double, _pd,
                                C.c_int64, C.c_double, _pd, C.c_int64]
        L.mref_csr_diagonal.argtypes = [C.c_void_p, _pd]
        L.mref_davidson.argtypes = [C.c_void_p, C.c_int64, C.c_double, _pd,
                                    _pd, _pi64]
        L.mref_selected_ci_diag.argtypes = [C.c_void_p, _p64, C.c_size_t,
                                            C.c_double, C.c_size_t, C.c_double,
                                            _pd, _pd]
        L.mref_asci_pairs.restype = C.c_void_p
        L.mref_asci_pairs.argtypes = [C.c_void_p, C.POINTER(AsciSettings), _p64,
                                      C.c_size_t, C.c_double, _pd, C.c_int]
        L.mref_pairs_size.restype = C.c_size_t
        L.mref_pairs_size.argtypes = [C.c_void_p]
        L.mref_pairs_copy.argtypes = [C.c_void_p, _p64, _pd]
        L.mref_pairs_free.argtypes = [C.c_void_p]
        L.mref_asci_search.argtypes = [C.c_void_p, C.POINTER(AsciSettings),
                                       C.c_size_t, _p64, C.c_size_t,
                                       C.c_double, _pd, _p64,
                                       C.POINTER(C.c_size_t)]
        L.mref_asci_run.argtypes = [C.c_void_p, C.c_int, C.POINTER(AsciSettings),
                                    C.POINTER(CiSettings), _pd, _p64, _pd,
                                    C.c_size_t, C.POINTER(C.c_size_t)]
        L.mref_hilbert_space.restype = C.c_size_t
        L.mref_hilbert_space.argtypes = [C.c_int, C.c_size_t, C.c_size_t,
                                         C.c_size_t, _p64]
        L.mref_cisd_space.restype = C.c_size_t
        L.mref_cisd_space.argtypes = L.mref_hilbert_space.argtypes
        L.mref_read_wavefunction.restype = C.c_long
        L.mref_read_wavefunction.argtypes = [C.c_char_p, _p64, _pd, C.c_size_t]
        L.mref_write_wavefunction.argtypes = [C.c_char_p, C.c_size_t, _p64, _pd,
                                              C.c_size_t, C.c_size_t]
        L.mref_read_fcidump.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), _pd,
                                        _pd, _pd]
        L.mref_write_fcidump.argtypes = [C.c_char_p, C.c_size_t, _pd, _pd,
                                         C.c_double]
        L.mref_read_rdms_binary.argtypes = [C.c_char_p, C.c_size_t, _pd, _pd]
        L.mref_write_rdms_binary.argtypes = [C.c_char_p, C.c_size_t, _pd, _pd]

    def _err(self):
        return self.L.mref_last_error().decode()

    def set_threads(self, n):
        self.L.mref_set_threads(n)

    def ham(self, nbits, norb, T, V):
        T = np.ascontiguousarray(T, dtype=np.float64).ravel(order="K")
        V = np.ascontiguousarray(V, dtype=np.float64).ravel(order="K")
        h = self.L.mref_ham_create(nbits, norb, _ptr(T, _pd), _ptr(V, _pd))
        if not h:
            raise RuntimeError(self._err())
        return Handle(h, self.L.mref_ham_free, nbits, norb)

    def read_wavefunction(self, fname, cap=1 << 16):
        """(dets, coeffs) from the reference's read_wavefunction<64>;
        RuntimeError with its message when it throws."""
        d = np.zeros(cap, dtype=np.uint64)
        c = np.zeros(cap)
        n = self.L.mref_read_wavefunction(str(fname).encode(), _ptr(d, _p64),
                                          _ptr(c, _pd), cap)
        if n < 0:
            raise RuntimeError(self._err())
        return d[:n].reshape(-1, 1), c[:n]

    def read_fcidump(self, fname):
        """(norb, T, V, E_core) from the reference's FCIDUMP readers (flat
        column-major, zero where the file has no line)."""
        n = C.c_uint32()
        if self.L.mref_read_fcidump(str(fname).encode(), C.byref(n), None,
                                    None, None) != 0:
            raise RuntimeError(self._err())
        T, V, core = np.zeros(n.value ** 2), np.zeros(n.value ** 4), C.c_double()
        if self.L.mref_read_fcidump(str(fname).encode(), C.byref(n),
                                    _ptr(T, _pd), _ptr(V, _pd),
                                    C.byref(core)) != 0:
            raise RuntimeError(self._err())
        return n.value, T, V, core.value

    def write_fcidump(self, fname, norb, T, V, E_core):
        """The reference's write_fcidump."""
        T = np.ascontiguousarray(T, dtype=np.float64).ravel(order="K")
        V = np.ascontiguousarray(V, dtype=np.float64).ravel(order="K")
        if self.L.mref_write_fcidump(str(fname).encode(), int(norb),
                                     _ptr(T, _pd), _ptr(V, _pd),
                                     float(E_core)) != 0:
            raise RuntimeError(self._err())

    def read_rdms_binary(self, fname, norb):
        """(ordm, trdm) from the reference's read_rdms_binary."""
        o, t = np.zeros(norb ** 2), np.zeros(norb ** 4)
        if self.L.mref_read_rdms_binary(str(fname).encode(), int(norb),
                                        _ptr(o, _pd), _ptr(t, _pd)) != 0:
            raise RuntimeError(self._err())
        return o, t

    def write_rdms_binary(self, fname, norb, ordm, trdm):
        """The reference's write_rdms_binary."""
        o = np.ascontiguousarray(ordm, dtype=np.float64).ravel(order="K")
        t = np.ascontiguousarray(trdm, dtype=np.float64).ravel(order="K")
        if self.L.mref_write_rdms_binary(str(fname).encode(), int(norb),
                                         _ptr(o, _pd), _ptr(t, _pd)) != 0:
            raise RuntimeError(self._err())

    def write_wavefunction(self, fname, norb, dets, coeffs):
        """The reference's write_wavefunction<64>."""
        d = np.ascontiguousarray(dets, dtype=np.uint64).ravel()
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        if self.L.mref_write_wavefunction(str(fname).encode(), int(norb),
                                          _ptr(d, _p64), _ptr(c, _pd),
                                          len(d), len(c)) != 0:
            raise RuntimeError(self._err())

    def form_rdms(self, h, dets, C, two=True):
        """(1-RDM, 2-RDM or None) of C over dets from the reference's
        form_rdms, both column-major flattened."""
        dets = _dets(dets, h.nbits)
        C = np.ascontiguousarray(C, dtype=np.float64).copy()
        o = np.zeros(h.norb ** 2)
        t = np.zeros(h.norb ** 4) if two else None
        self.L.mref_form_rdms(h.p, _ptr(dets, _p64), len(dets), _ptr(C, _pd),
                              _ptr(o, _pd),
                              t.ctypes.data if two else None)
        return o, t

    def matrix_element(self, h, bra, ket):
        bra, ket = _dets(bra, h.nbits), _dets(ket, h.nbits)
        out = np.empty(len(bra))
        self.L.mref_matrix_element(h.p, _ptr(bra, _p64), _ptr(ket, _p64),
                                   len(bra), _ptr(out, _pd))
        return out

    def fast_diag(self, h, kind, ss, os_, orbs, hii):
        ss = np.ascontiguousarray(ss, dtype=np.uint32)
        os_ = np.ascontiguousarray(os_, dtype=np.uint32)
        orbs = np.ascontiguousarray(orbs, dtype=np.uint32)
        out = C.c_double()
        self.L.mref_fast_diag(h.p, kind, _ptr(ss, _pu32), len(ss),
                              _ptr(os_, _pu32), len(os_), _ptr(orbs, _pu32),
                              hii, C.byref(out))
        return out.value

    def csr(self, h, bra, ket, thresh, nthreads=1):
        bra, ket = _dets(bra, h.nbits), _dets(ket, h.nbits)
        c = self.L.mref_csr_build(h.p, _ptr(bra, _p64), len(bra),
                                  _ptr(ket, _p64), len(ket), thresh, nthreads)
        if not c:
            raise RuntimeError(self._err())
        return RefCsr(self, c, len(bra), len(ket))

    def build_csr(self, h, bra, ket, thresh, nthreads=1):
        A = self.csr(h, bra, ket, thresh, nthreads)
        return A.arrays()

    def selected_ci_diag(self, h, dets, h_el_tol, max_m, tol, X=None):
        dets = _dets(dets, h.nbits)
        X = np.zeros(len(dets)) if X is None else np.array(X, dtype=np.float64)
        E = C.c_double()
        if self.L.mref_selected_ci_diag(h.p, _ptr(dets, _p64), len(dets),
                                        h_el_tol, max_m, tol, _ptr(X, _pd),
                                        C.byref(E)):
            raise RuntimeError(self._err())
        return E.value, X

    def asci_pairs(self, h, s, cdets, E0, Cv, accumulate=True):
        cdets = _dets(cdets, h.nbits)
        Cv = np.ascontiguousarray(Cv, dtype=np.float64)
        p = self.L.mref_asci_pairs(h.p, C.byref(s), _ptr(cdets, _p64),
                                   len(cdets), E0, _ptr(Cv, _pd),
                                   int(accumulate))
        if not p:
            raise RuntimeError(self._err())
        n = self.L.mref_pairs_size(p)
        st = np.empty((max(n, 1), h.nbits // 64), dtype=np.uint64)
        rv = np.empty(max(n, 1))
        self.L.mref_pairs_copy(p, _ptr(st, _p64), _ptr(rv, _pd))
        self.L.mref_pairs_free(p)
        return st[:n], rv[:n]

    def asci_search(self, h, s, ndets_max, cdets, E0, Cv):
        cdets = _dets(cdets, h.nbits)
        Cv = np.ascontiguousarray(Cv, dtype=np.float64)
        out = np.empty((ndets_max + len(cdets), h.nbits // 64), dtype=np.uint64)
        n = C.c_size_t()
        if self.L.mref_asci_search(h.p, C.byref(s), ndets_max,
                                   _ptr(cdets, _p64), len(cdets), E0,
                                   _ptr(Cv, _pd), _ptr(out, _p64), C.byref(n)):
            raise RuntimeError(self._err())
        return out[:n.value]

    def asci_run(self, h, refine, s, ci, E0, dets, X, cap):
        dets0 = _dets(dets, h.nbits)
        cap = max(cap, len(dets0))
        D = np.zeros((cap, h.nbits // 64), dtype=np.uint64)
        D[:len(dets0)] = dets0
        Xb = np.zeros(cap)
        Xb[:len(dets0)] = X
        E = C.c_double(E0)
        n = C.c_size_t()
        if self.L.mref_asci_run(h.p, int(refine), C.byref(s), C.byref(ci),
                                C.byref(E), _ptr(D, _p64), _ptr(Xb, _pd),
                                len(dets0), C.byref(n)):
            raise RuntimeError(self._err())
        return E.value, D[:n.value], Xb[:n.value]

    def hilbert_space(self, nbits, norb, na, nb):
        n = self.L.mref_hilbert_space(nbits, norb, na, nb, None)
        out = np.empty((n, nbits // 64), dtype=np.uint64)
        self.L.mref_hilbert_space(nbits, norb, na, nb, _ptr(out, _p64))
        return out

    def cisd_space(self, nbits, norb, na, nb):
        n = self.L.mref_cisd_space(nbits, norb, na, nb, None)
        out = np.empty((n, nbits // 64), dtype=np.uint64)
        self.L.mref_cisd_space(nbits, norb, na, nb, _ptr(out, _p64))
        return out


class Handle:
    def __init__(self, p, free, nbits, norb):
        self.p, self._free, self.nbits, self.norb = p, free, nbits, norb

    def __del__(self):
        if self.p:
            self._free(self.p)
            self.p = None


class RefCsr:
    """A reference sparsexx::csr_matrix<double,int32_t> held by the library."""

    def __init__(self, ref, c, m, n):
        self.ref, self.c, self.m, self.n = ref, c, m, n
        self.nnz = ref.L.mref_csr_nnz(c)

    def arrays(self):
        rp = np.empty(self.m + 1, dtype=np.int32)
        ci = np.empty(max(self.nnz, 1), dtype=np.int32)
        nz = np.empty(max(self.nnz, 1))
        self.ref.L.mref_csr_copy(self.c, _ptr(rp, _pi32), _ptr(ci, _pi32),
                                 _ptr(nz, _pd))
        return rp, ci[:self.nnz], nz[:self.nnz]

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.m)
        self.ref.L.mref_spmv(self.c, 1, 1.0, _ptr(x, _pd), self.n, 0.0,
                             _ptr(y, _pd), self.m)
        return y

    def diagonal(self):
        d = np.empty(self.m)
        self.ref.L.mref_csr_diagonal(self.c, _ptr(d, _pd))
        return d

    def davidson(self, max_m, tol):
        X = np.zeros(self.n)
        E = C.c_double()
        it = C.c_int64()
        if self.ref.L.mref_davidson(self.c, max_m, tol, _ptr(X, _pd),
                                    C.byref(E), C.byref(it)):
            raise RuntimeError(self.ref._err())
        return E.value, it.value, X

    def __del__(self):
        if self.c:
            self.ref.L.mref_csr_free(self.c)
            self.c = None


class RefConstraint:
    """The reference's MPI-only constraint-partitioned ASCI contributions
    (asci_contributions_constraint, determinant_search.hpp:143-391), compiled
    against a serial MPI stand-in so that one call runs one rank of a job of
    `world` ranks (_ref/libmacis_ref_constraint.so, bitset<64/128>)."""

    def __init__(self, path=REFC_PATH):
        L = C.CDLL(path)
        L.mrefc_last_error.restype = C.c_char_p
        L.mrefc_ham_create.restype = C.c_void_p
        L.mrefc_ham_create.argtypes = [C.c_int, C.c_size_t, _pd, _pd]
        L.mrefc_ham_free.argtypes = [C.c_void_p]
        L.mrefc_asci_pairs.restype = C.c_void_p
        L.mrefc_asci_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _p64,
                                       C.c_size_t, C.c_double, _pd, C.c_int,
                                       C.c_int]
        L.mrefc_pairs_size.restype = C.c_size_t
        L.mrefc_pairs_size.argtypes = [C.c_void_p]
        L.mrefc_pairs_copy.argtypes = [C.c_void_p, _p64, _pd]
        L.mrefc_pairs_free.argtypes = [C.c_void_p]
        self.L = L

    def ham(self, nbits, norb, T, V):
        T = np.ascontiguousarray(T, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        p = self.L.mrefc_ham_create(nbits, norb, _ptr(T, _pd), _ptr(V, _pd))
        if not p:
            raise RuntimeError(self.L.mrefc_last_error().decode())
        return Handle(p, self.L.mrefc_ham_free, nbits, norb)

    def asci_pairs(self, h, s, cdets, E0, Cv, rank, world, constraint_level=2):
        """This rank's accumulated (state, rv) pairs, per constraint in the
        reference's order (each constraint's block sorted on its own)."""
        cdets = _dets(cdets, h.nbits)
        Cv = np.ascontiguousarray(Cv, dtype=np.float64)
        p = self.L.mrefc_asci_pairs(h.p, C.byref(s), int(constraint_level),
                                    _ptr(cdets, _p64), len(cdets), E0,
                                    _ptr(Cv, _pd), int(rank), int(world))
        if not p:
            raise RuntimeError(self.L.mrefc_last_error().decode())
        n = self.L.mrefc_pairs_size(p)
        st = np.empty((max(n, 1), h.nbits // 64), dtype=np.uint64)
        rv = np.empty(max(n, 1))
        self.L.mrefc_pairs_copy(p, _ptr(st, _p64), _ptr(rv, _pd))
        self.L.mrefc_pairs_free(p)
        return st[:n], rv[:n]


_port = None
_ref = None
_refc = None


def port():
    global _port
    if _port is None:
        _port = Port()
    return _port


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        _ref = Ref()
    return _ref


def ref_constraint_available():
    return os.path.exists(REFC_PATH)


def ref_constraint():
    global _refc
    if _refc is None:
        _refc = RefConstraint()
    return _refc

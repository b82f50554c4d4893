"""ctypes binding of libmacis_b200.so (declarations in include/macis_b200.h).

The library is loaded from this package directory; importing the package
fails loudly when it is missing or cannot be loaded -- there is no CPU
fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmacis_b200.so")

OK, EINVAL, ENOMEM, ECAPACITY, ETIMEOUT, ENOCONV, ECUDA, ENOGROW = range(8)
DEVICE_PTRS = 1
FAULT_NONE, FAULT_ALLOC, FAULT_INT32_LIMIT = 0, 1, 2
HOP_FP32 = 2  # matrix-free H: off-diagonal elements rounded to FP32
FP64, MIXED = 0, 1

_p64 = C.POINTER(C.c_uint64)
_pd = C.POINTER(C.c_double)
_vp = C.c_void_p
_sz = C.c_size_t


class AsciSettingsC(C.Structure):
    _fields_ = [("ntdets_max", C.c_uint64), ("ntdets_min", C.c_uint64),
                ("ncdets_max", C.c_uint64), ("h_el_tol", C.c_double),
                ("rv_prune_tol", C.c_double), ("pair_size_max", C.c_uint64),
                ("just_singles", C.c_int32), ("pad_", C.c_int32),
                ("grow_factor", C.c_uint64), ("max_refine_iter", C.c_uint64),
                ("refine_energy_tol", C.c_double)]


class AsciStatsC(C.Structure):
    _fields_ = [("raw_pairs", C.c_uint64), ("unique_pairs", C.c_uint64),
                ("kept_pairs", C.c_uint64), ("batches", C.c_uint64),
                ("pairs_ms", C.c_double), ("sort_ms", C.c_double),
                ("keep_ms", C.c_double), ("topk_ms", C.c_double),
                ("total_ms", C.c_double), ("units_total", C.c_uint64),
                ("units_kept", C.c_uint64), ("samples", C.c_uint64),
                ("screen_ms", C.c_double), ("predict_ms", C.c_double),
                ("sort_pass_items", C.c_uint64),
                ("alpha_strings", C.c_uint64), ("key_bits", C.c_uint64),
                ("rank_ms", C.c_double)]


class AsciScreenC(C.Structure):
    _fields_ = [("net", C.c_void_p), ("use_net", C.c_int32),
                ("pad_", C.c_int32), ("keep_frac", C.c_double),
                ("explore_frac", C.c_double), ("max_samples", C.c_uint64),
                ("seed", C.c_uint64)]


class DavidsonOptsC(C.Structure):
    _fields_ = [("max_m", C.c_int64), ("tol", C.c_double),
                ("use_guess", C.c_int32), ("restart_keep", C.c_int32),
                ("max_iter", C.c_int64)]


class DavidsonStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("apply_ms", C.c_double),
                ("rayleigh_ms", C.c_double), ("residual_ms", C.c_double),
                ("ortho_ms", C.c_double), ("wall_ms", C.c_double),
                ("vector_bytes", C.c_double)]


class BuildStatsC(C.Structure):
    _fields_ = [("build_ms", C.c_double), ("fill_ms", C.c_double),
                ("nnz_candidates", C.c_int64), ("direct_product", C.c_int32),
                ("long_rows", C.c_int32)]


class MacisError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_SIGS = {
    "macis_b200_last_error": (C.c_char_p, []),
    "macis_b200_version": (C.c_int, []),
    "macis_b200_launch_count": (C.c_ulonglong, []),
    "macis_b200_set_wait_limit_ns": (C.c_int, [C.c_uint64]),
    "macis_b200_inject_fault": (C.c_int, [C.c_int, C.c_int64]),
    "macis_b200_ham_create": (C.c_int, [C.c_int, _sz, _pd, _sz, _pd, _sz,
                                        C.POINTER(_vp)]),
    "macis_b200_ham_destroy": (C.c_int, [_vp]),
    "macis_b200_matrix_element": (C.c_int, [_vp, _vp, _vp, _sz, _vp,
                                            C.c_uint]),
    "macis_b200_build_csr": (C.c_int, [_vp, _vp, _sz, _vp, _sz, C.c_double,
                                       C.c_int, C.c_int, C.c_uint,
                                       C.POINTER(_vp)]),
    "macis_b200_csr_destroy": (C.c_int, [_vp]),
    "macis_b200_csr_info": (C.c_int, [_vp, C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "macis_b200_csr_download": (C.c_int, [_vp, _vp, _vp, _vp, C.c_uint]),
    "macis_b200_csr_download_rows": (C.c_int, [_vp, C.c_int64, C.c_int64,
                                               _vp, _vp, _vp, C.c_uint]),
    "macis_b200_csr_diagonal": (C.c_int, [_vp, _vp, C.c_uint]),
    "macis_b200_spmv": (C.c_int, [_vp, C.c_int64, C.c_double, _vp, C.c_int64,
                                  C.c_double, _vp, C.c_int64, C.c_uint]),
    "macis_b200_spmv_mixed_noalloc": (C.c_int, [_vp, C.c_double, _vp,
                                                C.c_double, _vp]),
    "macis_b200_davidson": (C.c_int, [_vp, C.c_int64, C.c_double, C.c_int,
                                      _vp, C.POINTER(C.c_double),
                                      C.POINTER(C.c_int64), C.c_uint]),
    "macis_b200_davidson_ex": (C.c_int, [_vp, C.POINTER(DavidsonOptsC), _vp,
                                         C.POINTER(C.c_double),
                                         C.POINTER(C.c_int64), C.c_uint]),
    "macis_b200_davidson_last_stats": (C.c_int, [C.POINTER(DavidsonStatsC)]),
    "macis_b200_small_syev": (C.c_int, [C.c_int, _vp, C.c_int, _vp, _vp]),
    "macis_b200_csr_build_stats": (C.c_int, [_vp, C.POINTER(BuildStatsC)]),
    "macis_b200_asci_search": (C.c_int, [_vp, C.POINTER(AsciSettingsC), _sz,
                                         _vp, _sz, C.c_double, _vp, _vp,
                                         C.POINTER(_sz), C.c_uint]),
    "macis_b200_asci_pairs": (C.c_int, [_vp, C.POINTER(AsciSettingsC), _vp,
                                        _sz, C.c_double, _vp, _vp, _vp,
                                        C.POINTER(_sz)]),
    "macis_b200_asci_last_stats": (C.c_int, [_vp, C.POINTER(AsciStatsC)]),
    "macis_b200_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "macis_b200_mlp_destroy": (C.c_int, [_vp]),
    "macis_b200_mlp_num_params": (C.c_int, [_vp, C.POINTER(_sz)]),
    "macis_b200_mlp_get_params": (C.c_int, [_vp, _vp]),
    "macis_b200_mlp_set_params": (C.c_int, [_vp, _vp]),
    "macis_b200_mlp_forward": (C.c_int, [_vp, _vp, _sz, _vp, C.c_uint]),
    "macis_b200_mlp_gradients": (C.c_int, [_vp, _vp, _vp, _sz, _vp,
                                           C.POINTER(C.c_double), C.c_uint]),
    "macis_b200_mlp_train": (C.c_int, [_vp, _vp, _vp, _sz, C.c_int, C.c_int,
                                       C.c_double, C.c_uint64,
                                       C.POINTER(C.c_double), C.c_uint]),
    "macis_b200_mlp_samples": (C.c_int, [_vp, C.POINTER(_sz), _vp, _vp]),
    "macis_b200_mlp_clamp_samples": (C.c_int, [_vp, C.c_double,
                                               C.POINTER(C.c_float)]),
    "macis_b200_asci_unit_width": (C.c_int, [C.c_int]),
    "macis_b200_asci_search_screened": (C.c_int, [
        _vp, C.POINTER(AsciSettingsC), C.POINTER(AsciScreenC), _sz, _vp, _sz,
        C.c_double, _vp, _vp, C.POINTER(_sz), C.c_uint]),
    "macis_b200_asci_unit_features": (C.c_int, [_vp, _vp, _sz, C.c_double, _vp,
                                                _sz, _sz, _vp,
                                                C.POINTER(_sz)]),
    "macis_b200_form_rdms": (C.c_int, [_vp, _vp, _sz, _vp, _vp, _vp,
                                       C.c_uint]),
    "macis_b200_asci_search_part": (C.c_int, [_vp, C.POINTER(AsciSettingsC),
                                              _sz, _vp, _sz, C.c_double, _vp,
                                              C.c_uint32, C.c_uint32,
                                              C.POINTER(_sz), C.c_uint]),
    "macis_b200_asci_part_results": (C.c_int, [_vp, _vp, _vp]),
    "macis_b200_asci_search_part_screened": (C.c_int, [
        _vp, C.POINTER(AsciSettingsC), C.POINTER(AsciScreenC), _sz, _vp, _sz,
        C.c_double, _vp, C.c_uint32, C.c_uint32, C.POINTER(_sz), C.c_uint]),
    "macis_b200_mlp_set_sample_targets": (C.c_int, [_vp, _vp, _sz]),
    "macis_b200_hop_create": (C.c_int, [_vp, _vp, _sz, C.c_double, C.c_uint,
                                        C.POINTER(_vp)]),
    "macis_b200_hop_destroy": (C.c_int, [_vp]),
    "macis_b200_hop_apply": (C.c_int, [_vp, C.c_int64, C.c_double, _vp,
                                       C.c_int64, C.c_double, _vp, C.c_int64,
                                       C.c_uint]),
    "macis_b200_hop_diagonal": (C.c_int, [_vp, _vp, C.c_uint]),
    "macis_b200_hop_davidson": (C.c_int, [_vp, C.POINTER(DavidsonOptsC), _vp,
                                          C.POINTER(C.c_double),
                                          C.POINTER(C.c_int64), C.c_uint]),
}

EXPORTS = tuple(_SIGS)


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python macis_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = load()


def check(rc):
    if rc != OK:
        msg = LIB.macis_b200_last_error().decode()
        raise MacisError(rc, msg)

// C ABI of libmacis_b200 (declared in include/macis_b200.h). Every entry
// point converts exceptions into status codes and stages host buffers
// through HBM when MACIS_B200_DEVICE_PTRS is not set.
#include <cstring>
#include <string>

#include "internal.hpp"
#include "primitives.cuh"

namespace mb {
void ham_create(macis_b200_ham* h, int nbits, size_t norb, const double* T,
                size_t LDT, const double* V, size_t LDV);
void ham_destroy(macis_b200_ham* h);

static thread_local std::string g_err;
void set_error(const std::string& s) { g_err = s; }

template <class F>
static int guarded(F&& f) {
  try {
    f();
    return MACIS_B200_OK;
  } catch(const Error& e) {
    g_err = e.what();
    return e.code;
  } catch(const std::bad_alloc&) {
    g_err = "host allocation failed";
    return MACIS_B200_ENOMEM;
  } catch(const std::exception& e) {
    g_err = e.what();
    return MACIS_B200_EINVAL;
  }
}

// Device view of a possibly-host buffer.
template <typename T>
struct DevBuf {
  T* d = nullptr;
  bool owned = false;
  cudaStream_t s;
  DevBuf(const T* p, size_t n, unsigned flags, cudaStream_t st) : s(st) {
    if(flags & MACIS_B200_DEVICE_PTRS) {
      d = const_cast<T*>(p);
    } else {
      MB_CUDA(dev_malloc_async(&d, n * sizeof(T) + 16, s));
      owned = true;
      if(n && p)
        MB_CUDA(cudaMemcpyAsync(d, p, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
  }
  DevBuf(const DevBuf&) = delete;
  ~DevBuf() {
    if(owned) cudaFreeAsync(d, s);
  }
};

static void require_dets(const void* p, size_t n, unsigned flags = 0) {
  MB_REQUIRE(n == 0 || p != nullptr, MACIS_B200_EINVAL,
             "null determinant array");
  MB_REQUIRE(!(flags & MACIS_B200_DEVICE_PTRS) ||
                 (reinterpret_cast<uintptr_t>(p) & 15) == 0,
             MACIS_B200_EINVAL, "device determinant arrays must be 16-byte aligned");
}

}  // namespace mb

using namespace mb;

extern "C" {

const char* macis_b200_last_error(void) { return g_err.c_str(); }
int macis_b200_version(void) { return 1; }

int macis_b200_ham_create(int nbits, size_t norb, const double* T, size_t LDT,
                          const double* V, size_t LDV, macis_b200_ham** out) {
  return guarded([&] {
    MB_REQUIRE(out && T && V, MACIS_B200_EINVAL, "null argument");
    auto* h = new macis_b200_ham;
    try {
      ham_create(h, nbits, norb, T, LDT, V, LDV);
    } catch(...) {
      ham_destroy(h);
      delete h;
      throw;
    }
    *out = h;
  });
}

int macis_b200_ham_destroy(macis_b200_ham* h) {
  return guarded([&] {
    if(!h) return;
    ham_destroy(h);
    delete h;
  });
}

int macis_b200_matrix_element(macis_b200_ham* h, const uint64_t* bra,
                              const uint64_t* ket, size_t n, double* out,
                              unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(h, MACIS_B200_EINVAL, "null handle");
    require_dets(bra, n);
    require_dets(ket, n);
    const size_t nw = h->nbits / 64;
    DevBuf<uint64_t> b(bra, n * nw, flags, h->stream), k(ket, n * nw, flags,
                                                          h->stream);
    DevBuf<double> o(out, 0, flags | MACIS_B200_DEVICE_PTRS, h->stream);
    double* dout = out;
    if(!(flags & MACIS_B200_DEVICE_PTRS))
      MB_CUDA(dev_malloc_async(&dout, n * 8 + 8, h->stream));
    matrix_elements_device(h, b.d, k.d, n, dout);
    if(!(flags & MACIS_B200_DEVICE_PTRS)) {
      MB_CUDA(cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, h->stream));
      cudaFreeAsync(dout, h->stream);
    }
    MB_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int macis_b200_build_csr(macis_b200_ham* h, const uint64_t* bra, size_t nbra,
                         const uint64_t* ket, size_t nket, double H_thresh,
                         int idx_bytes, int val_bytes, unsigned flags,
                         macis_b200_csr** out) {
  return guarded([&] {
    MB_REQUIRE(h && out, MACIS_B200_EINVAL, "null argument");
    require_dets(bra, nbra, flags);
    require_dets(ket, nket, flags);
    const size_t nw = h->nbits / 64;
    // a bra list inside the ket array (same list, or a row block of it) is
    // uploaded once and passed as a sub-range, which keeps the square /
    // row-block fast paths
    const bool inside = bra >= ket && bra + nbra * nw <= ket + nket * nw &&
                        (bra - ket) % nw == 0;
    DevBuf<uint64_t> k(ket, nket * nw, flags, h->stream);
    const uint64_t* bd = nullptr;
    DevBuf<uint64_t>* bb = nullptr;
    if(inside && !(flags & MACIS_B200_DEVICE_PTRS)) {
      bd = k.d + (bra - ket);
    } else {
      bb = new DevBuf<uint64_t>(bra, nbra * nw, flags, h->stream);
      bd = bb->d;
    }
    try {
      *out = build_csr_device(h, bd, nbra, k.d, nket, H_thresh, idx_bytes,
                              val_bytes);
    } catch(...) {
      delete bb;
      throw;
    }
    delete bb;
  });
}

int macis_b200_csr_destroy(macis_b200_csr* A) {
  return guarded([&] {
    if(!A) return;
    cudaFreeAsync(A->rowptr, A->stream);
    cudaFreeAsync(A->colind, A->stream);
    cudaFreeAsync(A->nzval, A->stream);
    cudaFreeAsync(A->diag, A->stream);
    cudaStreamSynchronize(A->stream);
    if(A->own_stream) cudaStreamDestroy(A->stream);
    delete A;
  });
}

unsigned long long macis_b200_launch_count(void) { return launch_counter(); }

int macis_b200_inject_fault(int kind, int64_t arg) {
  return guarded([&] {
    switch(kind) {
      case MACIS_B200_FAULT_NONE:
        faults().alloc_countdown.store(-1);
        faults().int32_limit.store(INT32_MAX);
        break;
      case MACIS_B200_FAULT_ALLOC:
        MB_REQUIRE(arg >= 0, MACIS_B200_EINVAL, "allocation count must be >= 0");
        faults().alloc_countdown.store(arg);
        break;
      case MACIS_B200_FAULT_INT32_LIMIT:
        MB_REQUIRE(arg >= 0 && arg <= INT32_MAX, MACIS_B200_EINVAL,
                   "int32 limit must be in [0, 2^31 - 1]");
        faults().int32_limit.store(arg);
        break;
      default:
        MB_REQUIRE(false, MACIS_B200_EINVAL, "unknown fault kind");
    }
  });
}

int macis_b200_set_wait_limit_ns(uint64_t ns) {
  wait_limit_slot().store(ns ? ns : kDefaultWaitLimitNs);
  return MACIS_B200_OK;
}

int macis_b200_csr_info(const macis_b200_csr* A, int64_t* m, int64_t* n,
                        int64_t* nnz, int* idx_bytes, int* val_bytes) {
  return guarded([&] {
    MB_REQUIRE(A, MACIS_B200_EINVAL, "null handle");
    if(m) *m = A->m;
    if(n) *n = A->n;
    if(nnz) *nnz = A->nnz;
    if(idx_bytes) *idx_bytes = A->idx_bytes;
    if(val_bytes) *val_bytes = A->val_bytes;
  });
}

int macis_b200_csr_download(const macis_b200_csr* A, void* rowptr,
                            void* colind, void* nzval, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(A, MACIS_B200_EINVAL, "null handle");
    const cudaMemcpyKind k = (flags & MACIS_B200_DEVICE_PTRS)
                                 ? cudaMemcpyDeviceToDevice
                                 : cudaMemcpyDeviceToHost;
    if(rowptr)
      MB_CUDA(cudaMemcpyAsync(rowptr, A->rowptr, (A->m + 1) * A->idx_bytes, k,
                              A->stream));
    if(colind && A->nnz)
      MB_CUDA(cudaMemcpyAsync(colind, A->colind, A->nnz * A->idx_bytes, k,
                              A->stream));
    if(nzval && A->nnz)
      MB_CUDA(cudaMemcpyAsync(nzval, A->nzval, A->nnz * A->val_bytes, k,
                              A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
  });
}

int macis_b200_csr_download_rows(const macis_b200_csr* A, int64_t r0,
                                 int64_t r1, void* rowptr, void* colind,
                                 void* nzval, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(A, MACIS_B200_EINVAL, "null handle");
    MB_REQUIRE(0 <= r0 && r0 <= r1 && r1 <= A->m, MACIS_B200_EINVAL,
               "row range outside the matrix");
    const cudaMemcpyKind k = (flags & MACIS_B200_DEVICE_PTRS)
                                 ? cudaMemcpyDeviceToDevice
                                 : cudaMemcpyDeviceToHost;
    const size_t ib = size_t(A->idx_bytes);
    // the two bounding row offsets, as stored (int32 or int64)
    int64_t lo = 0, hi = 0;
    MB_CUDA(cudaMemcpyAsync(&lo, static_cast<char*>(A->rowptr) + r0 * ib, ib,
                            cudaMemcpyDeviceToHost, A->stream));
    MB_CUDA(cudaMemcpyAsync(&hi, static_cast<char*>(A->rowptr) + r1 * ib, ib,
                            cudaMemcpyDeviceToHost, A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
    if(ib == 4) {  // little-endian: the low word holds the int32 value
      lo = int64_t(int32_t(uint32_t(lo)));
      hi = int64_t(int32_t(uint32_t(hi)));
    }
    if(rowptr)
      MB_CUDA(cudaMemcpyAsync(rowptr, static_cast<char*>(A->rowptr) + r0 * ib,
                              size_t(r1 - r0 + 1) * ib, k, A->stream));
    if(colind && hi > lo)
      MB_CUDA(cudaMemcpyAsync(colind, static_cast<char*>(A->colind) + lo * ib,
                              size_t(hi - lo) * ib, k, A->stream));
    if(nzval && hi > lo)
      MB_CUDA(cudaMemcpyAsync(
          nzval, static_cast<char*>(A->nzval) + lo * A->val_bytes,
          size_t(hi - lo) * A->val_bytes, k, A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
  });
}

int macis_b200_csr_diagonal(const macis_b200_csr* A, double* D,
                            unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(A && D, MACIS_B200_EINVAL, "null argument");
    const cudaMemcpyKind k = (flags & MACIS_B200_DEVICE_PTRS)
                                 ? cudaMemcpyDeviceToDevice
                                 : cudaMemcpyDeviceToHost;
    if(A->m)
      MB_CUDA(cudaMemcpyAsync(D, A->diag, A->m * 8, k, A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
  });
}

int macis_b200_spmv(const macis_b200_csr* A, int64_t K, double alpha,
                    const double* V, int64_t LDV, double beta, double* AV,
                    int64_t LDAV, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(A && (K == 0 || (V && AV)), MACIS_B200_EINVAL, "null argument");
    MB_REQUIRE(K >= 0 && LDV >= A->n && LDAV >= A->m, MACIS_B200_EINVAL,
               "bad leading dimension");
    cudaStream_t s = A->stream;
    if(flags & MACIS_B200_DEVICE_PTRS) {
      for(int64_t k = 0; k < K; ++k)
        spmv_device(A, alpha, V + k * LDV, beta, AV + k * LDAV, s);
    } else {
      Arena W(s);
      double* dv = W.get<double>(size_t(A->n));
      double* dy = W.get<double>(size_t(A->m));
      for(int64_t k = 0; k < K; ++k) {
        MB_CUDA(cudaMemcpyAsync(dv, V + k * LDV, A->n * 8,
                                cudaMemcpyHostToDevice, s));
        if(beta != 0.0)
          MB_CUDA(cudaMemcpyAsync(dy, AV + k * LDAV, A->m * 8,
                                  cudaMemcpyHostToDevice, s));
        spmv_device(A, alpha, dv, beta, dy, s);
        MB_CUDA(cudaMemcpyAsync(AV + k * LDAV, dy, A->m * 8,
                                cudaMemcpyDeviceToHost, s));
      }
    }
    MB_CUDA(cudaStreamSynchronize(s));
  });
}

int macis_b200_davidson(const macis_b200_csr* A, int64_t max_m, double tol,
                        int use_guess, double* X, double* E, int64_t* niter,
                        unsigned flags) {
  int rc = MACIS_B200_OK;
  int st = guarded([&] {
    MB_REQUIRE(A && X && E && niter, MACIS_B200_EINVAL, "null argument");
    DevBuf<double> x(X, size_t(A->m), flags, A->stream);
    rc = davidson_device(A, max_m, tol, use_guess != 0, x.d, E, niter, 0, 0);
    if(!(flags & MACIS_B200_DEVICE_PTRS))
      MB_CUDA(cudaMemcpyAsync(X, x.d, A->m * 8, cudaMemcpyDeviceToHost, A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
  });
  if(st) return st;
  if(rc == MACIS_B200_ENOCONV) g_err = "Davidson Did Not Converge!";
  return rc;
}

int macis_b200_davidson_ex(const macis_b200_csr* A,
                           const macis_b200_davidson_opts* o, double* X,
                           double* E, int64_t* niter, unsigned flags) {
  int rc = MACIS_B200_OK;
  int st = guarded([&] {
    MB_REQUIRE(A && o && X && E && niter, MACIS_B200_EINVAL, "null argument");
    DevBuf<double> x(X, size_t(A->m), flags, A->stream);
    rc = davidson_device(A, o->max_m, o->tol, o->use_guess != 0, x.d, E, niter,
                         o->restart_keep, o->max_iter);
    if(!(flags & MACIS_B200_DEVICE_PTRS))
      MB_CUDA(cudaMemcpyAsync(X, x.d, A->m * 8, cudaMemcpyDeviceToHost, A->stream));
    MB_CUDA(cudaStreamSynchronize(A->stream));
  });
  if(st) return st;
  if(rc == MACIS_B200_ENOCONV) g_err = "Davidson Did Not Converge!";
  return rc;
}

int macis_b200_davidson_last_stats(macis_b200_davidson_stats* out) {
  return guarded([&] {
    MB_REQUIRE(out, MACIS_B200_EINVAL, "null argument");
    *out = davidson_last_stats();
  });
}

int macis_b200_small_syev(int k, const double* lower, int nwant, double* W,
                          double* Vec) {
  return guarded([&] {
    MB_REQUIRE(k >= 1 && nwant >= 1 && lower && W && Vec, MACIS_B200_EINVAL,
               "bad argument");
    small_syev_lowest(k, lower, nwant, W, Vec);
  });
}

int macis_b200_csr_build_stats(const macis_b200_csr* A,
                               macis_b200_build_stats* out) {
  return guarded([&] {
    MB_REQUIRE(A && out, MACIS_B200_EINVAL, "null argument");
    out->build_ms = A->build_ms;
    out->fill_ms = A->fill_ms;
    out->nnz_candidates = A->nnz_candidates;
    out->direct_product = A->direct_product ? 1 : 0;
    out->long_rows = int32_t(A->long_rows);
  });
}

int macis_b200_asci_search(macis_b200_ham* h,
                           const macis_b200_asci_settings* s,
                           size_t ndets_max, const uint64_t* cdets,
                           size_t ncdets, double E0, const double* C,
                           uint64_t* out_dets, size_t* nout, unsigned flags) {
  return macis_b200_asci_search_screened(h, s, nullptr, ndets_max, cdets,
                                         ncdets, E0, C, out_dets, nout, flags);
}

int macis_b200_asci_search_screened(macis_b200_ham* h,
                                    const macis_b200_asci_settings* s,
                                    const macis_b200_asci_screen* scr,
                                    size_t ndets_max, const uint64_t* cdets,
                                    size_t ncdets, double E0, const double* C,
                                    uint64_t* out_dets, size_t* nout,
                                    unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(h && s && out_dets && nout, MACIS_B200_EINVAL, "null argument");
    require_dets(cdets, ncdets, flags);
    require_dets(out_dets, 1, flags);
    const size_t nw = h->nbits / 64;
    DevBuf<uint64_t> cd(cdets, ncdets * nw, flags, h->stream);
    DevBuf<double> cc(C, ncdets, flags, h->stream);
    const size_t cap = ndets_max + ncdets;
    uint64_t* od = out_dets;
    if(!(flags & MACIS_B200_DEVICE_PTRS))
      MB_CUDA(dev_malloc_async(&od, cap * nw * 8 + 32, h->stream));
    try {
      asci_search_device(h, *s, scr, ndets_max, cd.d, ncdets, E0, cc.d, od,
                         nout, nullptr, nullptr, false);
    } catch(...) {
      if(!(flags & MACIS_B200_DEVICE_PTRS)) cudaFreeAsync(od, h->stream);
      throw;
    }
    if(!(flags & MACIS_B200_DEVICE_PTRS)) {
      MB_CUDA(cudaMemcpyAsync(out_dets, od, *nout * nw * 8,
                              cudaMemcpyDeviceToHost, h->stream));
      cudaFreeAsync(od, h->stream);
    }
    MB_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int macis_b200_asci_pairs(macis_b200_ham* h, const macis_b200_asci_settings* s,
                          const uint64_t* cdets, size_t ncdets, double E0,
                          const double* C, uint64_t* states, double* rv,
                          size_t* npairs) {
  return guarded([&] {
    MB_REQUIRE(h && s && npairs, MACIS_B200_EINVAL, "null argument");
    require_dets(cdets, ncdets);
    const size_t nw = h->nbits / 64;
    DevBuf<uint64_t> cd(cdets, ncdets * nw, 0, h->stream);
    DevBuf<double> cc(C, ncdets, 0, h->stream);
    std::vector<uint64_t> ps;
    std::vector<double> pr;
    size_t dummy = 0;
    asci_search_device(h, *s, nullptr, 0, cd.d, ncdets, E0, cc.d, nullptr,
                       &dummy, &ps, &pr, true);
    *npairs = pr.size();
    if(states) {
      std::memcpy(states, ps.data(), ps.size() * 8);
      std::memcpy(rv, pr.data(), pr.size() * 8);
    }
  });
}

int macis_b200_asci_last_stats(const macis_b200_ham* h,
                               macis_b200_asci_stats* out) {
  return guarded([&] {
    MB_REQUIRE(h && out, MACIS_B200_EINVAL, "null argument");
    *out = h->last_asci;
  });
}

int macis_b200_asci_unit_width(int nbits) { return asci_unit_din(nbits); }

int macis_b200_asci_unit_features(macis_b200_ham* h, const uint64_t* cdets,
                                  size_t ncdets, double E0, const double* C,
                                  size_t first, size_t n, uint16_t* X,
                                  size_t* nunits) {
  return guarded([&] {
    MB_REQUIRE(h && nunits, MACIS_B200_EINVAL, "null argument");
    require_dets(cdets, ncdets);
    const size_t nw = h->nbits / 64, din = size_t(asci_unit_din(h->nbits));
    DevBuf<uint64_t> cd(cdets, ncdets * nw, 0, h->stream);
    DevBuf<double> cc(C, ncdets, 0, h->stream);
    DevBuf<uint16_t> xd(nullptr, X ? n * din : 0, 0, h->stream);
    *nunits = size_t(asci_unit_features_device(h, cd.d, ncdets, E0, cc.d,
                                               first, X ? n : 0, xd.d));
    if(X && n) {
      MB_CUDA(cudaMemcpyAsync(X, xd.d, n * din * 2, cudaMemcpyDeviceToHost,
                              h->stream));
      MB_CUDA(cudaStreamSynchronize(h->stream));
    }
  });
}

// ------------------------------------------------------ screening network
int macis_b200_mlp_create(int din, uint64_t seed, macis_b200_mlp** out) {
  return guarded([&] {
    MB_REQUIRE(out, MACIS_B200_EINVAL, "null argument");
    *out = mlp_create(din, seed);
  });
}

int macis_b200_mlp_destroy(macis_b200_mlp* m) {
  return guarded([&] { mlp_destroy(m); });
}

int macis_b200_mlp_num_params(const macis_b200_mlp* m, size_t* n) {
  return guarded([&] {
    MB_REQUIRE(m && n, MACIS_B200_EINVAL, "null argument");
    *n = m->nparams;
  });
}

int macis_b200_mlp_get_params(const macis_b200_mlp* m, float* P) {
  return guarded([&] {
    MB_REQUIRE(m && P, MACIS_B200_EINVAL, "null argument");
    mlp_get_params(m, P);
  });
}

int macis_b200_mlp_set_params(macis_b200_mlp* m, const float* P) {
  return guarded([&] {
    MB_REQUIRE(m && P, MACIS_B200_EINVAL, "null argument");
    mlp_set_params(m, P);
  });
}

int macis_b200_mlp_forward(macis_b200_mlp* m, const uint16_t* X, size_t n,
                           float* y, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(m && (n == 0 || (X && y)), MACIS_B200_EINVAL, "null argument");
    const size_t din = size_t(m->din);
    DevBuf<uint16_t> xd(X, n * din, flags, m->stream);
    DevBuf<float> yd(nullptr, (flags & MACIS_B200_DEVICE_PTRS) ? 0 : n, 0,
                     m->stream);
    float* yp = (flags & MACIS_B200_DEVICE_PTRS) ? y : yd.d;
    mlp_forward_device(m, xd.d, int64_t(n), yp, m->stream);
    if(!(flags & MACIS_B200_DEVICE_PTRS) && n) {
      MB_CUDA(cudaMemcpyAsync(y, yp, n * 4, cudaMemcpyDeviceToHost, m->stream));
      MB_CUDA(cudaStreamSynchronize(m->stream));
    }
  });
}

int macis_b200_mlp_gradients(macis_b200_mlp* m, const uint16_t* X,
                             const float* t, size_t n, float* grad,
                             double* loss, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(m && X && t && grad && n > 0, MACIS_B200_EINVAL,
               "null argument or empty batch");
    const size_t din = size_t(m->din);
    DevBuf<uint16_t> xd(X, n * din, flags, m->stream);
    DevBuf<float> td(t, n, flags, m->stream);
    DevBuf<float> gd(nullptr, m->nparams, 0, m->stream);
    const double l = mlp_gradients_device(m, xd.d, td.d, int64_t(n), gd.d);
    MB_CUDA(cudaMemcpyAsync(grad, gd.d, m->nparams * 4,
                            (flags & MACIS_B200_DEVICE_PTRS)
                                ? cudaMemcpyDeviceToDevice
                                : cudaMemcpyDeviceToHost,
                            m->stream));
    MB_CUDA(cudaStreamSynchronize(m->stream));
    if(loss) *loss = l;
  });
}

int macis_b200_mlp_train(macis_b200_mlp* m, const uint16_t* X, const float* t,
                         size_t n, int epochs, int batch, double lr,
                         uint64_t seed, double* loss, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(m, MACIS_B200_EINVAL, "null argument");
    double l = 0;
    if(X == nullptr) {
      MB_REQUIRE(m->ns > 0, MACIS_B200_EINVAL, "no recorded samples");
      l = mlp_train_device(m, m->xs, m->ts, int64_t(m->ns), epochs, batch, lr,
                           seed);
    } else {
      MB_REQUIRE(t && n > 0, MACIS_B200_EINVAL, "null targets or no samples");
      const size_t din = size_t(m->din);
      DevBuf<uint16_t> xd(X, n * din, flags, m->stream);
      DevBuf<float> td(t, n, flags, m->stream);
      l = mlp_train_device(m, xd.d, td.d, int64_t(n), epochs, batch, lr, seed);
    }
    if(loss) *loss = l;
  });
}

int macis_b200_mlp_clamp_samples(macis_b200_mlp* m, double q, float* floor) {
  return guarded([&] {
    MB_REQUIRE(m, MACIS_B200_EINVAL, "null argument");
    const float f = mlp_clamp_samples(m, q);
    if(floor) *floor = f;
  });
}

int macis_b200_mlp_set_sample_targets(macis_b200_mlp* m, const float* t,
                                      size_t n) {
  return guarded([&] {
    MB_REQUIRE(m && (t || n == 0), MACIS_B200_EINVAL, "null argument");
    MB_REQUIRE(n == m->ns, MACIS_B200_EINVAL,
               "target count differs from the recorded sample count");
    if(n) {
      MB_CUDA(cudaMemcpyAsync(m->ts, t, n * 4, cudaMemcpyHostToDevice,
                              m->stream));
      MB_CUDA(cudaStreamSynchronize(m->stream));
    }
  });
}

int macis_b200_mlp_samples(const macis_b200_mlp* m, size_t* n, uint16_t* X,
                           float* t) {
  return guarded([&] {
    MB_REQUIRE(m && n, MACIS_B200_EINVAL, "null argument");
    *n = m->ns;
    if(X && m->ns) {
      MB_CUDA(cudaMemcpyAsync(X, m->xs, m->ns * size_t(m->din) * 2,
                              cudaMemcpyDeviceToHost, m->stream));
      if(t)
        MB_CUDA(cudaMemcpyAsync(t, m->ts, m->ns * 4, cudaMemcpyDeviceToHost,
                                m->stream));
      MB_CUDA(cudaStreamSynchronize(m->stream));
    }
  });
}

}  // extern "C"

// ---------------------------------------------------- matrix-free H
extern "C" {

int macis_b200_hop_create(const macis_b200_ham* h, const uint64_t* dets,
                          size_t ndets, double H_thresh, unsigned flags,
                          macis_b200_hop** out) {
  return guarded([&] {
    MB_REQUIRE(h && out, MACIS_B200_EINVAL, "null argument");
    require_dets(dets, ndets, flags);
    *out = hop_create(const_cast<macis_b200_ham*>(h), dets, ndets, H_thresh,
                      (flags & MACIS_B200_HOP_FP32) != 0,
                      (flags & MACIS_B200_DEVICE_PTRS) != 0);
  });
}

int macis_b200_hop_destroy(macis_b200_hop* op) {
  return guarded([&] { hop_destroy(op); });
}

int macis_b200_hop_apply(const macis_b200_hop* op, int64_t K, double alpha,
                         const double* V, int64_t LDV, double beta, double* AV,
                         int64_t LDAV, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(op && (K == 0 || (V && AV)), MACIS_B200_EINVAL, "null argument");
    const int64_t n = hop_size(op);
    MB_REQUIRE(K >= 0 && LDV >= n && LDAV >= n, MACIS_B200_EINVAL,
               "bad leading dimension");
    cudaStream_t s = hop_stream(op);
    if(flags & MACIS_B200_DEVICE_PTRS) {
      for(int64_t k = 0; k < K; ++k)
        hop_apply(op, alpha, V + k * LDV, beta, AV + k * LDAV);
    } else {
      Arena W(s);
      double* dv = W.get<double>(size_t(n));
      double* dy = W.get<double>(size_t(n));
      for(int64_t k = 0; k < K; ++k) {
        MB_CUDA(cudaMemcpyAsync(dv, V + k * LDV, n * 8, cudaMemcpyHostToDevice, s));
        if(beta != 0.0)
          MB_CUDA(cudaMemcpyAsync(dy, AV + k * LDAV, n * 8,
                                  cudaMemcpyHostToDevice, s));
        hop_apply(op, alpha, dv, beta, dy);
        MB_CUDA(cudaMemcpyAsync(AV + k * LDAV, dy, n * 8,
                                cudaMemcpyDeviceToHost, s));
      }
    }
    MB_CUDA(cudaStreamSynchronize(s));
  });
}

int macis_b200_hop_diagonal(const macis_b200_hop* op, double* D,
                            unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(op && D, MACIS_B200_EINVAL, "null argument");
    cudaStream_t s = hop_stream(op);
    const auto k = (flags & MACIS_B200_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice
                                                    : cudaMemcpyDeviceToHost;
    MB_CUDA(cudaMemcpyAsync(D, hop_diag(op), hop_size(op) * 8, k, s));
    MB_CUDA(cudaStreamSynchronize(s));
  });
}

int macis_b200_hop_davidson(const macis_b200_hop* op,
                            const macis_b200_davidson_opts* o, double* X,
                            double* E, int64_t* niter, unsigned flags) {
  int rc = MACIS_B200_OK;
  int st = guarded([&] {
    MB_REQUIRE(op && o && X && E && niter, MACIS_B200_EINVAL, "null argument");
    cudaStream_t s = hop_stream(op);
    const int64_t n = hop_size(op);
    DevBuf<double> x(X, size_t(n), flags, s);
    DavOperator dop;
    dop.n = n;
    dop.diag = hop_diag(op);
    dop.s = s;
    dop.apply = [op](const double* xin, double* y) {
      hop_apply(op, 1.0, xin, 0.0, y);
    };
    rc = davidson_op(dop, o->max_m, o->tol, o->use_guess != 0, x.d, E, niter,
                     o->restart_keep, o->max_iter);
    if(!(flags & MACIS_B200_DEVICE_PTRS))
      MB_CUDA(cudaMemcpyAsync(X, x.d, n * 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
  });
  if(st) return st;
  if(rc == MACIS_B200_ENOCONV) g_err = "Davidson Did Not Converge!";
  return rc;
}

}  // extern "C"

extern "C" int macis_b200_form_rdms(macis_b200_ham* h, const uint64_t* dets,
                                    size_t ndets, const double* C,
                                    double* ordm, double* trdm,
                                    unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(h && ordm && (ndets == 0 || C), MACIS_B200_EINVAL,
               "null argument");
    require_dets(dets, ndets, flags);
    const size_t nw = h->nbits / 64, n = size_t(h->norb);
    const size_t n2 = n * n, n4 = n2 * n2;
    cudaStream_t s = h->stream;
    DevBuf<uint64_t> d(dets, ndets * nw, flags, s);
    DevBuf<double> c(C, ndets, flags, s);
    DevBuf<double> o(ordm, n2, flags, s);  // accumulated into, as given
    DevBuf<double>* t = trdm ? new DevBuf<double>(trdm, n4, flags, s) : nullptr;
    try {
      form_rdms_device(h, d.d, ndets, c.d, o.d, t ? t->d : nullptr);
      if(!(flags & MACIS_B200_DEVICE_PTRS)) {
        MB_CUDA(cudaMemcpyAsync(ordm, o.d, n2 * 8, cudaMemcpyDeviceToHost, s));
        if(t)
          MB_CUDA(cudaMemcpyAsync(trdm, t->d, n4 * 8, cudaMemcpyDeviceToHost, s));
      }
      MB_CUDA(cudaStreamSynchronize(s));
    } catch(...) {
      delete t;
      throw;
    }
    delete t;
  });
}

extern "C" int macis_b200_asci_search_part(
    macis_b200_ham* h, const macis_b200_asci_settings* s, size_t ndets_max,
    const uint64_t* cdets, size_t ncdets, double E0, const double* C,
    uint32_t part_index, uint32_t part_count, size_t* nout, unsigned flags) {
  return macis_b200_asci_search_part_screened(h, s, nullptr, ndets_max, cdets,
                                              ncdets, E0, C, part_index,
                                              part_count, nout, flags);
}

extern "C" int macis_b200_asci_search_part_screened(
    macis_b200_ham* h, const macis_b200_asci_settings* s,
    const macis_b200_asci_screen* scr, size_t ndets_max, const uint64_t* cdets,
    size_t ncdets, double E0, const double* C, uint32_t part_index,
    uint32_t part_count, size_t* nout, unsigned flags) {
  return guarded([&] {
    MB_REQUIRE(h && s && nout, MACIS_B200_EINVAL, "null argument");
    MB_REQUIRE(part_count >= 1 && part_index < part_count, MACIS_B200_EINVAL,
               "part_index must be in [0, part_count)");
    require_dets(cdets, ncdets, flags);
    const size_t nw = h->nbits / 64;
    DevBuf<uint64_t> cd(cdets, ncdets * nw, flags, h->stream);
    DevBuf<double> cc(C, ncdets, flags, h->stream);
    AsciPart part;
    part.index = part_index;
    part.count = part_count;
    size_t dummy = 0;
    h->part_states.clear();
    h->part_scores.clear();
    asci_search_device(h, *s, scr, ndets_max, cd.d, ncdets, E0, cc.d,
                       nullptr, &dummy, nullptr, nullptr, false, &part);
    *nout = h->part_scores.size();
  });
}

extern "C" int macis_b200_asci_part_results(const macis_b200_ham* h,
                                            uint64_t* states, double* scores) {
  return guarded([&] {
    MB_REQUIRE(h && states && scores, MACIS_B200_EINVAL, "null argument");
    if(!h->part_scores.empty()) {
      std::memcpy(states, h->part_states.data(), h->part_states.size() * 8);
      std::memcpy(scores, h->part_scores.data(), h->part_scores.size() * 8);
    }
  });
}

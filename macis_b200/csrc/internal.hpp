// Internal handle types and cross-file entry points of libmacis_b200.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"

struct macis_b200_ham {
  int nbits = 64;
  int norb = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  // Device integrals + intermediates (column-major, compact leading dims).
  double *T = nullptr, *V = nullptr, *G = nullptr, *G_red = nullptr,
         *V_red = nullptr, *G2_red = nullptr, *V2_red = nullptr;
  // V with the two index pairs swapped, VT[(p + q n) n^2 + (r + s n)] =
  // V[(p + q n) + (r + s n) n^2]; built on first use by the direct-product
  // fill so that one alpha pair's row of V is contiguous
  double* VT = nullptr;
  macis_b200_asci_stats last_asci{};
  mb::Ints ints() const {
    return mb::Ints{norb, T, V, G, G_red, V_red, G2_red, V2_red};
  }
};

struct macis_b200_csr {
  int64_t m = 0, n = 0, nnz = 0;
  int idx_bytes = 4, val_bytes = 8;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  void* rowptr = nullptr;  // (m+1) x idx_bytes
  void* colind = nullptr;  // nnz x idx_bytes
  void* nzval = nullptr;   // nnz x val_bytes (FP32 mode: diagonal slots 0)
  double* diag = nullptr;  // m, FP64 stored diagonal (0 where absent)
  // build diagnostics
  bool direct_product = false;
  int64_t nnz_candidates = 0;
  int64_t long_rows = 0;
  float build_ms = 0.f;
  float fill_ms = 0.f;
};

namespace mb {

// Build the CSR block of H for device-resident bra/ket determinant arrays.
macis_b200_csr* build_csr_device(macis_b200_ham* h, const uint64_t* bra,
                                 size_t nbra, const uint64_t* ket, size_t nket,
                                 double thresh, int idx_bytes, int val_bytes);

// Batched matrix elements for device arrays.
void matrix_elements_device(macis_b200_ham* h, const uint64_t* bra,
                            const uint64_t* ket, size_t n, double* out);

// y = alpha*A*x + beta*y on device vectors (one column).
void spmv_device(const macis_b200_csr* A, double alpha, const double* x,
                 double beta, double* y, cudaStream_t s);

// Davidson on device-resident matrix; X is a device vector.
int davidson_device(const macis_b200_csr* A, int64_t max_m, double tol,
                    bool use_guess, double* X, double* E, int64_t* niter,
                    int restart_keep, int64_t max_iter);

// Lowest nwant eigenpairs of a k x k symmetric matrix (lower triangle).
void small_syev_lowest(int k, const double* lower, int nwant, double* W,
                       double* Vec);

// ASCI search on device-resident core dets (see macis_b200_asci_search).
void asci_search_device(macis_b200_ham* h, const macis_b200_asci_settings& s,
                        size_t ndets_max, const uint64_t* cdets, size_t ncdets,
                        double E0, const double* C, uint64_t* out_dets,
                        size_t* nout, std::vector<uint64_t>* pairs_states,
                        std::vector<double>* pairs_rv, bool pairs_only);

void set_error(const std::string& s);

}  // namespace mb

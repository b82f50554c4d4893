// Internal handle types and cross-file entry points of libmacis_b200.
#pragma once
#include <cuda_runtime.h>
#include <functional>

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
  // Per outer pair (i, a), p = a + i n: pairmax[p] = max_{b,j} |G(b,j,a,i)|
  // and pairmax[n^2 + p] = max_{b,j} |V(a,i,b,j)| -- upper bounds of the
  // same-spin / opposite-spin double elements of the ASCI units; built on
  // first use by the screened search
  double* pairmax = nullptr;
  macis_b200_asci_stats last_asci{};
  // result of the last macis_b200_asci_search_part (candidates, scores)
  std::vector<uint64_t> part_states;
  std::vector<double> part_scores;
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

// Screening network (mlp.cu). BF16 buffers are held as uint16_t.
struct macis_b200_mlp {
  int din = 192;
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0,
         off_b3 = 0, nparams = 0;
  float *P = nullptr, *G = nullptr, *Mo = nullptr, *Ve = nullptr;
  uint16_t *w1t = nullptr, *w2t = nullptr, *w2T = nullptr;
  int* err = nullptr;
  int64_t step = 0;  // Adam steps taken
  // training scratch for batches of B rows
  int64_t B = 0;
  std::vector<void*> scratch;
  uint16_t *xb = nullptr, *xbt = nullptr, *h1t = nullptr, *dz2t_b = nullptr,
           *dz2_b = nullptr, *dz1t_b = nullptr;
  float *tb = nullptr, *yb = nullptr, *z1t = nullptr, *z2t = nullptr,
        *dy = nullptr, *dz2t = nullptr, *p3t = nullptr, *dz1t = nullptr;
  int64_t* idx = nullptr;
  // (features, target) samples recorded by the last ASCI search
  uint16_t* xs = nullptr;
  float* ts = nullptr;
  size_t ns = 0, cap = 0;
  double last_loss = 0;
  double train_ms = 0;
};

namespace mb {

struct MlpWeights;
macis_b200_mlp* mlp_create(int din, uint64_t seed);
void mlp_destroy(macis_b200_mlp* m);
void mlp_set_params(macis_b200_mlp* m, const float* host);
void mlp_get_params(const macis_b200_mlp* m, float* host);
MlpWeights mlp_weights(const macis_b200_mlp* m);
// y[0..n) = network(X) for device X [n][din] BF16; synchronizes s.
void mlp_forward_device(macis_b200_mlp* m, const uint16_t* X, int64_t n,
                        float* y, cudaStream_t s);
// One forward + backward over all n rows; device gradient (nparams) -> grad.
double mlp_gradients_device(macis_b200_mlp* m, const uint16_t* X,
                            const float* t, int64_t n, float* grad);
// Adam on (X, t) device samples; returns the mean loss of the last epoch.
double mlp_train_device(macis_b200_mlp* m, const uint16_t* X, const float* t,
                        int64_t S, int epochs, int batch, double lr,
                        uint64_t seed);
void mlp_reserve_samples(macis_b200_mlp* m, size_t cap);
// Raise the recorded targets below their q-quantile to it; returns the floor.
float mlp_clamp_samples(macis_b200_mlp* m, double q);

// Build the CSR block of H for device-resident bra/ket determinant arrays.
macis_b200_csr* build_csr_device(macis_b200_ham* h, const uint64_t* bra,
                                 size_t nbra, const uint64_t* ket, size_t nket,
                                 double thresh, int idx_bytes, int val_bytes);

// Batched matrix elements for device arrays.
void matrix_elements_device(macis_b200_ham* h, const uint64_t* bra,
                            const uint64_t* ket, size_t n, double* out);

// y = alpha*A*x + beta*y on device vectors (one column).
// Davidson's product: on a mixed matrix, FP32 values times the FP64 x with
// FP64 sums (one fixed linear operator); FP64 matrices as spmv_device.
void spmv_device_x64(const macis_b200_csr* A, double alpha, const double* x,
                     double beta, double* y, cudaStream_t s);
void spmv_device(const macis_b200_csr* A, double alpha, const double* x,
                 double beta, double* y, cudaStream_t s);

// Davidson on device-resident matrix; X is a device vector.
int davidson_device(const macis_b200_csr* A, int64_t max_m, double tol,
                    bool use_guess, double* X, double* E, int64_t* niter,
                    int restart_keep, int64_t max_iter);

// The operator Davidson works with: y = H x on device vectors of length n,
// diag(H) in device memory, everything on stream s (the reference's
// davidson takes any functor with operator_action, davidson.hpp:47-58, 129).
struct DavOperator {
  int64_t n = 0;
  const double* diag = nullptr;
  cudaStream_t s = nullptr;
  std::function<void(const double* x, double* y)> apply;
};
int davidson_op(const DavOperator& op, int64_t max_m, double tol,
                bool use_guess, double* X, double* E, int64_t* niter,
                int restart_keep, int64_t max_iter);
const macis_b200_davidson_stats& davidson_last_stats();

// 1- and 2-RDM over one determinant list (device arrays; results added to
// ordm / trdm, trdm may be null).
void form_rdms_device(macis_b200_ham* h, const uint64_t* dets, size_t n,
                      const double* C, double* ordm, double* trdm);

// Matrix-free H over one determinant list (hbuild.cu).
macis_b200_hop* hop_create(macis_b200_ham* h, const uint64_t* dets, size_t n,
                           double thresh, bool mixed, bool device_ptrs);
void hop_apply(const macis_b200_hop* op, double alpha, const double* x,
               double beta, double* y);
void hop_destroy(macis_b200_hop* op);
int64_t hop_size(const macis_b200_hop* op);
const double* hop_diag(const macis_b200_hop* op);
cudaStream_t hop_stream(const macis_b200_hop* op);

// Lowest nwant eigenpairs of a k x k symmetric matrix (lower triangle).
void small_syev_lowest(int k, const double* lower, int nwant, double* W,
                       double* Vec);

// ASCI search on device-resident core dets (see macis_b200_asci_search).
// scr may be null (exact search, nothing recorded).
// One part of a search split over `count` parts (index in [0, count)): the
// part's candidates and scores go to h->part_states / part_scores.
struct AsciPart {
  uint32_t index = 0, count = 1;
};
// V with its index pairs swapped (macis_b200_ham::VT), built on first use.
const double* ham_vt(macis_b200_ham* h);

void asci_search_device(macis_b200_ham* h, const macis_b200_asci_settings& s,
                        const macis_b200_asci_screen* scr, size_t ndets_max,
                        const uint64_t* cdets, size_t ncdets, double E0,
                        const double* C, uint64_t* out_dets, size_t* nout,
                        std::vector<uint64_t>* pairs_states,
                        std::vector<double>* pairs_rv, bool pairs_only,
                        const AsciPart* part = nullptr);
// Network input rows of units [first, first + n) of the search over the core
// dets (device X [n][din]); returns the unit count.
int64_t asci_unit_features_device(macis_b200_ham* h, const uint64_t* cdets,
                                  size_t ncdets, double E0, const double* C,
                                  size_t first, size_t n, uint16_t* X);
int asci_unit_din(int nbits);

void set_error(const std::string& s);

}  // namespace mb

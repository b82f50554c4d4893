// C++ drop-in for MACIS's selected-CI hot path on a B200 (header-only).
//
// Include after the MACIS headers. It keeps MACIS's own template API:
//
//   macis_b200::HamiltonianGenerator<N>   a macis::HamiltonianGenerator<N>
//       whose virtual CSR hook (include/macis/hamiltonian_generator.hpp:
//       66-72) builds on the GPU, so macis::make_csr_hamiltonian[_block]
//       (include/macis/csr_hamiltonian.hpp:23-45) and everything above it
//       use the GPU build unchanged
//   macis_b200::SparseMatrixOperator       the H.X hook of macis::davidson
//       (include/macis/solvers/davidson.hpp:29-59) over a device CSR
//   macis_b200::selected_ci_diag           selected_ci_diag.hpp:125-206 with
//       H kept in HBM (build + Davidson on the GPU)
//   macis_b200::asci_search / asci_iter / asci_grow / asci_refine
//       include/macis/asci/{determinant_search.hpp:395,iteration.hpp:17,
//       grow.hpp:17,refine.hpp:15}; the reference drivers call asci_search
//       and selected_ci_diag directly, so same-signature drivers are shipped;
//       a trailing ScreenSettings* adds the learned screening of the search
//
// Link with libmacis_b200.so (C ABI in macis_b200.h). MPI world size 1.
#pragma once
#include <macis_b200.h>

#include <bitset>
#include <cstring>
#include <macis/asci/determinant_search.hpp>
#include <macis/hamiltonian_generator.hpp>
#include <macis/util/mcscf.hpp>
#include <sparsexx/matrix_types/csr_matrix.hpp>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace macis_b200 {

inline void check(int rc) {
  if(rc != MACIS_B200_OK) throw std::runtime_error(macis_b200_last_error());
}

template <size_t N>
inline const uint64_t* words(const std::bitset<N>* p) {
  static_assert(sizeof(std::bitset<N>) == N / 8, "bitset word layout");
  return reinterpret_cast<const uint64_t*>(p);
}

// Device CSR owned by the library.
class DeviceCSR {
  macis_b200_csr* A_ = nullptr;

 public:
  explicit DeviceCSR(macis_b200_csr* A) : A_(A) {}
  DeviceCSR(const DeviceCSR&) = delete;
  DeviceCSR(DeviceCSR&& o) noexcept : A_(o.A_) { o.A_ = nullptr; }
  ~DeviceCSR() {
    if(A_) macis_b200_csr_destroy(A_);
  }
  macis_b200_csr* get() const { return A_; }
  int64_t m() const {
    int64_t v;
    check(macis_b200_csr_info(A_, &v, nullptr, nullptr, nullptr, nullptr));
    return v;
  }
  int64_t nnz() const {
    int64_t v;
    check(macis_b200_csr_info(A_, nullptr, nullptr, &v, nullptr, nullptr));
    return v;
  }
  std::vector<double> diagonal() const {
    std::vector<double> d(m());
    check(macis_b200_csr_diagonal(A_, d.data(), 0));
    return d;
  }
  template <typename index_t>
  sparsexx::csr_matrix<double, index_t> to_host() const {
    int64_t m, n, nnz;
    int ib, vb;
    check(macis_b200_csr_info(A_, &m, &n, &nnz, &ib, &vb));
    if(ib != int(sizeof(index_t)) || vb != 8)
      throw std::runtime_error("Unsupported index_t");
    std::vector<index_t> rp(m + 1), ci(nnz);
    std::vector<double> nz(nnz);
    check(macis_b200_csr_download(A_, rp.data(), ci.data(), nz.data(), 0));
    return sparsexx::csr_matrix<double, index_t>(m, n, std::move(rp),
                                                 std::move(ci), std::move(nz));
  }
};

template <size_t N>
class HamiltonianGenerator : public macis::HamiltonianGenerator<N> {
  using base = macis::HamiltonianGenerator<N>;
  macis_b200_ham* h_ = nullptr;

 public:
  using full_det_iterator = typename base::full_det_iterator;
  using matrix_span_t = typename base::matrix_span_t;
  using rank4_span_t = typename base::rank4_span_t;

  HamiltonianGenerator(matrix_span_t T, rank4_span_t V) : base(T, V) {
    check(macis_b200_ham_create(int(N), T.extent(0), T.data_handle(),
                                T.extent(0), V.data_handle(), V.extent(0),
                                &h_));
  }
  ~HamiltonianGenerator() noexcept override {
    if(h_) macis_b200_ham_destroy(h_);
  }
  macis_b200_ham* handle() const { return h_; }

  // Device-resident build (no download): the selected_ci_diag path.
  DeviceCSR build_device(full_det_iterator bb, full_det_iterator be,
                         full_det_iterator kb, full_det_iterator ke,
                         double thresh, int idx_bytes = 4,
                         int val_bytes = 8) {
    const size_t nb = std::distance(bb, be), nk = std::distance(kb, ke);
    macis_b200_csr* A = nullptr;
    check(macis_b200_build_csr(h_, nb ? words<N>(&*bb) : nullptr, nb,
                               nk ? words<N>(&*kb) : nullptr, nk, thresh,
                               idx_bytes, val_bytes, 0, &A));
    return DeviceCSR(A);
  }

  // form_rdms (double_loop.hpp:117-165) for bra = ket, the way
  // compute_casci_rdms calls it (cas.hpp:52-56); results are added to the
  // contiguous column-major spans, trdm may be empty (1-RDM alone).
  void form_rdms(full_det_iterator bb, full_det_iterator be,
                 full_det_iterator kb, full_det_iterator ke, double* C,
                 matrix_span_t ordm, rank4_span_t trdm) override {
    if(bb != kb || be != ke)
      throw std::logic_error(
          "form_rdms on the B200 path takes the same bra and ket range");
    const size_t n = std::distance(bb, be);
    check(macis_b200_form_rdms(h_, n ? words<N>(&*bb) : nullptr, n, C,
                               ordm.data_handle(), trdm.data_handle(), 0));
  }

 protected:
  template <typename index_t>
  sparsexx::csr_matrix<double, index_t> build_host(full_det_iterator bb,
                                                   full_det_iterator be,
                                                   full_det_iterator kb,
                                                   full_det_iterator ke,
                                                   double thresh) {
    return build_device(bb, be, kb, ke, thresh, int(sizeof(index_t)))
        .template to_host<index_t>();
  }
  sparsexx::csr_matrix<double, int32_t> make_csr_hamiltonian_block_32bit_(
      full_det_iterator bb, full_det_iterator be, full_det_iterator kb,
      full_det_iterator ke, double thresh) override {
    return build_host<int32_t>(bb, be, kb, ke, thresh);
  }
  sparsexx::csr_matrix<double, int64_t> make_csr_hamiltonian_block_64bit_(
      full_det_iterator bb, full_det_iterator be, full_det_iterator kb,
      full_det_iterator ke, double thresh) override {
    return build_host<int64_t>(bb, be, kb, ke, thresh);
  }
};

// operator_action(m, alpha, V, LDV, beta, AV, LDAV) on host blocks.
class SparseMatrixOperator {
  const DeviceCSR& A_;

 public:
  explicit SparseMatrixOperator(const DeviceCSR& A) : A_(A) {}
  void operator_action(size_t m, double alpha, const double* V, size_t LDV,
                       double beta, double* AV, size_t LDAV) const {
    check(macis_b200_spmv(A_.get(), int64_t(m), alpha, V, int64_t(LDV), beta,
                          AV, int64_t(LDAV), 0));
  }
};

// Matrix-free H over one determinant list (macis_b200_hop_*), for lists
// whose CSR matrix does not fit in device memory. operator_action has the
// signature MACIS's own davidson (davidson.hpp:129) calls on its functor, so
// macis::davidson(N, max_m, op, D, tol, X) runs with it directly (D from
// diagonal()). The generator must outlive the operator's products.
template <size_t N>
class MatrixFreeOperator {
  macis_b200_hop* op_ = nullptr;
  int64_t n_ = 0;

 public:
  MatrixFreeOperator(const HamiltonianGenerator<N>& ham,
                     macis::wavefunction_iterator_t<N> b,
                     macis::wavefunction_iterator_t<N> e, double thresh,
                     bool fp32_values = false) {
    n_ = std::distance(b, e);
    check(macis_b200_hop_create(ham.handle(), n_ ? words<N>(&*b) : nullptr,
                                size_t(n_), thresh,
                                fp32_values ? MACIS_B200_HOP_FP32 : 0u, &op_));
  }
  MatrixFreeOperator(const MatrixFreeOperator&) = delete;
  MatrixFreeOperator& operator=(const MatrixFreeOperator&) = delete;
  ~MatrixFreeOperator() {
    if(op_) macis_b200_hop_destroy(op_);
  }
  const macis_b200_hop* get() const { return op_; }
  int64_t size() const { return n_; }
  std::vector<double> diagonal() const {
    std::vector<double> d(n_);
    check(macis_b200_hop_diagonal(op_, d.data(), 0));
    return d;
  }
  void operator_action(size_t m, double alpha, const double* V, size_t LDV,
                       double beta, double* AV, size_t LDAV) const {
    check(macis_b200_hop_apply(op_, int64_t(m), alpha, V, int64_t(LDV), beta,
                               AV, int64_t(LDAV), 0));
  }
};

// davidson(N, max_m, op, D, tol, X) for a device operator: the reference
// signature; D is taken from the matrix. Throws "Davidson Did Not Converge!".
inline std::pair<int64_t, double> davidson(int64_t, int64_t max_m,
                                           const SparseMatrixOperator& op,
                                           const DeviceCSR& A, double tol,
                                           double* X, bool use_guess = true) {
  double E = 0;
  int64_t it = 0;
  check(macis_b200_davidson(A.get(), max_m, tol, use_guess, X, &E, &it, 0));
  (void)op;
  return {it, E};
}

template <size_t N, typename index_t = int32_t>
double selected_ci_diag(macis::wavefunction_iterator_t<N> dets_begin,
                        macis::wavefunction_iterator_t<N> dets_end,
                        HamiltonianGenerator<N>& ham_gen, double h_el_tol,
                        size_t davidson_max_m, double davidson_res_tol,
                        std::vector<double>& C_local,
                        const bool /*quiet*/ = false) {
  const size_t ndets = std::distance(dets_begin, dets_end);
  DeviceCSR H = ham_gen.build_device(dets_begin, dets_end, dets_begin,
                                     dets_end, h_el_tol, sizeof(index_t));
  C_local.resize(ndets, 0);
  double max_c = 0;
  for(double c : C_local) max_c = std::max(max_c, std::abs(c));
  const bool guess = ndets && max_c > 1. / ndets;  // selected_ci_diag.hpp:96
  double E = 0;
  int64_t it = 0;
  check(macis_b200_davidson(H.get(), int64_t(davidson_max_m),
                            davidson_res_tol, guess, C_local.data(), &E, &it,
                            0));
  return E;
}

inline macis_b200_asci_settings to_c(const macis::ASCISettings& s) {
  macis_b200_asci_settings c{};
  c.ntdets_max = s.ntdets_max;
  c.ntdets_min = s.ntdets_min;
  c.ncdets_max = s.ncdets_max;
  c.h_el_tol = s.h_el_tol;
  c.rv_prune_tol = s.rv_prune_tol;
  c.pair_size_max = s.pair_size_max;
  c.just_singles = s.just_singles;
  c.grow_factor = s.grow_factor;
  c.max_refine_iter = s.max_refine_iter;
  c.refine_energy_tol = s.refine_energy_tol;
  return c;
}

// asci_search with the reference signature (world size 1). The integral
// pointers are accepted for signature compatibility; the generator's
// device copies are used.
template <size_t N>
std::vector<macis::wfn_t<N>> asci_search(
    macis::ASCISettings asci_settings, size_t ndets_max,
    macis::wavefunction_iterator_t<N> cdets_begin,
    macis::wavefunction_iterator_t<N> cdets_end, const double E_ASCI,
    const std::vector<double>& C, size_t /*norb*/, const double* /*T_pq*/,
    const double* /*G_red*/, const double* /*V_red*/,
    const double* /*G_pqrs*/, const double* /*V_pqrs*/,
    HamiltonianGenerator<N>& ham_gen) {
  const size_t nc = std::distance(cdets_begin, cdets_end);
  const auto s = to_c(asci_settings);
  std::vector<macis::wfn_t<N>> out(ndets_max + nc);
  size_t nout = 0;
  check(macis_b200_asci_search(ham_gen.handle(), &s, ndets_max,
                               nc ? words<N>(&*cdets_begin) : nullptr, nc,
                               E_ASCI, C.data(),
                               reinterpret_cast<uint64_t*>(out.data()), &nout,
                               0));
  out.resize(nout);
  return out;
}

// Learned screening of the ASCI search (no MACIS counterpart). A search
// "unit" is one core determinant with one excitation class and, for
// doubles, one outer (occupied, virtual) pair; the network predicts each
// unit's largest log |score|, and a screened search scores exactly only the
// top keep_frac of the units (plus a random explore_frac).
class ScreeningNetwork {
  macis_b200_mlp* m_ = nullptr;
  size_t trained_steps_ = 0;

 public:
  explicit ScreeningNetwork(int nbits, uint64_t seed = 0) {
    check(macis_b200_mlp_create(macis_b200_asci_unit_width(nbits), seed, &m_));
  }
  ScreeningNetwork(const ScreeningNetwork&) = delete;
  ScreeningNetwork& operator=(const ScreeningNetwork&) = delete;
  ~ScreeningNetwork() {
    if(m_) macis_b200_mlp_destroy(m_);
  }
  macis_b200_mlp* handle() const { return m_; }
  size_t trained_steps() const { return trained_steps_; }
  // Adam over the samples the last recording search stored; returns the
  // mean loss of the last epoch.
  double train_on_samples(int epochs, int batch, double lr, uint64_t seed) {
    double loss = 0;
    check(macis_b200_mlp_train(m_, nullptr, nullptr, 0, epochs, batch, lr,
                               seed, &loss, 0));
    ++trained_steps_;
    return loss;
  }
  // Raise the stored targets below their q-quantile to that value.
  float clamp_samples(double q) {
    float f = 0;
    check(macis_b200_mlp_clamp_samples(m_, q, &f));
    return f;
  }
};

// How the ASCI drivers use a ScreeningNetwork: every search records
// samples of the units it scores and the network is retrained after it;
// searches after the first warmup_searches, with at least min_units units,
// prune by prediction.
struct ScreenSettings {
  ScreeningNetwork* network = nullptr;
  double keep_frac = 0.2;
  double explore_frac = 0.02;
  uint64_t max_samples = 1000000;  // samples recorded per search
  int epochs = 2;
  double lr = 1e-3;
  int batch = 1024;
  double clamp_quantile = 0.6;  // 0: no clamping
  uint64_t min_units = 20000;
  uint64_t warmup_searches = 1;
  bool train = true;
  uint64_t seed = 0;
  uint64_t searches = 0;  // searches run so far (updated)

  bool prune_next() const {
    return network && network->trained_steps() > 0 &&
           searches >= warmup_searches;
  }
  macis_b200_asci_screen to_c(bool use_net) const {
    macis_b200_asci_screen c{};
    c.net = network ? network->handle() : nullptr;
    c.use_net = use_net;
    c.keep_frac = keep_frac;
    c.explore_frac = explore_frac;
    c.max_samples = train ? max_samples : 0;
    c.seed = seed + 7919 * searches;
    return c;
  }
};

// asci_search with learned screening (use_net: prune by prediction).
template <size_t N>
std::vector<macis::wfn_t<N>> asci_search(
    macis::ASCISettings asci_settings, size_t ndets_max,
    macis::wavefunction_iterator_t<N> cdets_begin,
    macis::wavefunction_iterator_t<N> cdets_end, const double E_ASCI,
    const std::vector<double>& C, HamiltonianGenerator<N>& ham_gen,
    ScreenSettings& screen, bool use_net) {
  if(!screen.network) throw std::logic_error("ScreenSettings without network");
  const size_t nc = std::distance(cdets_begin, cdets_end);
  const auto s = to_c(asci_settings);
  const auto sc = screen.to_c(use_net);
  std::vector<macis::wfn_t<N>> out(ndets_max + nc);
  size_t nout = 0;
  check(macis_b200_asci_search_screened(
      ham_gen.handle(), &s, &sc, ndets_max,
      nc ? words<N>(&*cdets_begin) : nullptr, nc, E_ASCI, C.data(),
      reinterpret_cast<uint64_t*>(out.data()), &nout, 0));
  ++screen.searches;
  out.resize(nout);
  return out;
}

// Statistics of the last search on a generator.
template <size_t N>
macis_b200_asci_stats last_search_stats(const HamiltonianGenerator<N>& h) {
  macis_b200_asci_stats st{};
  check(macis_b200_asci_last_stats(h.handle(), &st));
  return st;
}

// asci_iter (include/macis/asci/iteration.hpp:17-68). With a screen whose
// network is set, the search records samples / prunes units and the network
// is retrained on the recorded samples before the diagonalisation.
template <size_t N, typename index_t = int32_t>
auto asci_iter(macis::ASCISettings asci_settings,
               macis::MCSCFSettings mcscf_settings, size_t ndets_max,
               double E0, std::vector<macis::wfn_t<N>> wfn,
               std::vector<double> X, HamiltonianGenerator<N>& ham_gen,
               size_t norb, ScreenSettings* screen = nullptr) {
  if(wfn.size() > 1) {  // reorder_ci_on_coeff, ties kept in order
    std::vector<size_t> idx(X.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](size_t i, size_t j) {
      return std::abs(X[i]) > std::abs(X[j]);
    });
    std::vector<macis::wfn_t<N>> w2(wfn.size());
    std::vector<double> x2(X.size());
    for(size_t i = 0; i < idx.size(); ++i) {
      w2[i] = wfn[idx[i]];
      x2[i] = X[idx[i]];
    }
    wfn = std::move(w2);
    X = std::move(x2);
  }
  const size_t nkeep = std::min(asci_settings.ncdets_max, wfn.size());
  if(screen && screen->network) {
    bool use_net = screen->prune_next();
    if(use_net && screen->min_units) {  // small searches run exact
      size_t nunits = 0;
      check(macis_b200_asci_unit_features(
          ham_gen.handle(), nkeep ? words<N>(wfn.data()) : nullptr, nkeep, E0,
          X.data(), 0, 0, nullptr, &nunits));
      use_net = nunits >= screen->min_units;
    }
    wfn = asci_search<N>(asci_settings, ndets_max, wfn.begin(),
                         wfn.begin() + nkeep, E0, X, ham_gen, *screen,
                         use_net);
    if(screen->train && last_search_stats(ham_gen).samples > 0) {
      if(screen->clamp_quantile > 0)
        screen->network->clamp_samples(screen->clamp_quantile);
      screen->network->train_on_samples(screen->epochs, screen->batch,
                                        screen->lr,
                                        screen->seed + screen->searches);
    }
  } else {
    wfn = asci_search<N>(asci_settings, ndets_max, wfn.begin(),
                         wfn.begin() + nkeep, E0, X, norb, nullptr, nullptr,
                         nullptr, nullptr, nullptr, ham_gen);
  }
  std::vector<double> X_local;
  const double E = selected_ci_diag<N, index_t>(
      wfn.begin(), wfn.end(), ham_gen, mcscf_settings.ci_matel_tol,
      mcscf_settings.ci_max_subspace, mcscf_settings.ci_res_tol, X_local);
  return std::make_tuple(E, wfn, std::move(X_local));
}

// asci_grow (include/macis/asci/grow.hpp:17-171, without grow_with_rot)
template <size_t N, typename index_t = int32_t>
auto asci_grow(macis::ASCISettings asci_settings,
               macis::MCSCFSettings mcscf_settings, double E0,
               std::vector<macis::wfn_t<N>> wfn, std::vector<double> X,
               HamiltonianGenerator<N>& ham_gen, size_t norb,
               ScreenSettings* screen = nullptr) {
  if(asci_settings.grow_with_rot)
    throw std::logic_error("grow_with_rot is not part of the B200 path");
  while(wfn.size() < asci_settings.ntdets_max) {
    const size_t ndets_new = std::min(
        std::max(asci_settings.ntdets_min,
                 wfn.size() * asci_settings.grow_factor),
        asci_settings.ntdets_max);
    double E;
    std::tie(E, wfn, X) = asci_iter<N, index_t>(
        asci_settings, mcscf_settings, ndets_new, E0, std::move(wfn),
        std::move(X), ham_gen, norb, screen);
    if(ndets_new > wfn.size())
      throw std::runtime_error("Wavefunction didn't grow enough...");
    E0 = E;
  }
  return std::make_tuple(E0, wfn, X);
}

// asci_refine (include/macis/asci/refine.hpp:15-66)
template <size_t N, typename index_t = int32_t>
auto asci_refine(macis::ASCISettings asci_settings,
                 macis::MCSCFSettings mcscf_settings, double E0,
                 std::vector<macis::wfn_t<N>> wfn, std::vector<double> X,
                 HamiltonianGenerator<N>& ham_gen, size_t norb,
                 ScreenSettings* screen = nullptr) {
  const size_t ndets = wfn.size();
  for(size_t iter = 0; iter < asci_settings.max_refine_iter; ++iter) {
    double E;
    std::tie(E, wfn, X) =
        asci_iter<N, index_t>(asci_settings, mcscf_settings, ndets, E0,
                              std::move(wfn), std::move(X), ham_gen, norb,
                              screen);
    if(wfn.size() != ndets)
      throw std::runtime_error("Wavefunction size can't change in refinement");
    const double dE = E - E0;
    E0 = E;
    if(std::abs(dE) < asci_settings.refine_energy_tol)
      return std::make_tuple(E0, wfn, X);
  }
  throw std::runtime_error("ACCI Refine did not converge");
}

}  // namespace macis_b200

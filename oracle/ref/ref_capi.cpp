// C entry points over the UNMODIFIED reference MACIS headers, compiled from
// the reference sources in place (see oracle/ref/Makefile). This is test
// infrastructure: the parity tests and the CPU baseline call it as the
// reference implementation of the hot path. Nothing in the product links it.
//
// Every entry point wraps one public reference API:
//   mref_csr_build       -> macis::make_csr_hamiltonian_block<int32_t>
//                           (include/macis/csr_hamiltonian.hpp:23-37) on a
//                           DoubleLoopHamiltonianGenerator<N>
//                           (include/macis/hamiltonian_generator/double_loop.hpp:17)
//                           optionally over row blocks on several threads, the
//                           same split as make_dist_csr_hamiltonian
//                           (csr_hamiltonian.hpp:49-82)
//   mref_spmv            -> sparsexx::spblas::gespmbv (spblas/spmbv.hpp:39)
//   mref_davidson        -> macis::davidson (solvers/davidson.hpp:129)
//   mref_selected_ci_diag-> macis::selected_ci_diag (selected_ci_diag.hpp:125)
//   mref_asci_pairs      -> macis::asci_contributions_standard +
//                           sort_and_accumulate_asci_pairs
//                           (asci/determinant_search.hpp:54, determinant_sort.hpp:40)
//   mref_asci_search     -> macis::asci_search (determinant_search.hpp:395)
//   mref_asci_grow/refine-> macis::asci_grow / asci_refine (asci/grow.hpp:17,
//                           asci/refine.hpp:15)
#include <spdlog/sinks/null_sink.h>
#include <spdlog/spdlog.h>

#include <cstring>
#include <macis/asci/grow.hpp>
#include <macis/asci/refine.hpp>
#include <macis/csr_hamiltonian.hpp>
#include <macis/hamiltonian_generator/double_loop.hpp>
#include <macis/solvers/davidson.hpp>
#include <macis/solvers/selected_ci_diag.hpp>
#include <macis/util/mcscf.hpp>
#include <macis/util/binary_rdms.hpp>
#include <macis/util/fcidump.hpp>
#include <macis/wavefunction_io.hpp>
#include <sparsexx/spblas/spmbv.hpp>
#include <sparsexx/util/submatrix.hpp>
#include <atomic>
#include <string>
#include <thread>
#include <vector>

extern "C" void openblas_set_num_threads(int);

namespace {

thread_local std::string g_err;

void quiet_loggers() {
  for(const char* n :
      {"davidson", "ci_solver", "asci_search", "asci_grow", "asci_refine"})
    if(!spdlog::get(n)) spdlog::null_logger_mt(n);
}

template <size_t N>
std::vector<std::bitset<N>> to_dets(const uint64_t* w, size_t n) {
  constexpr size_t W = N / 64;
  static_assert(sizeof(std::bitset<N>) == W * 8, "bitset layout");
  std::vector<std::bitset<N>> d(n);
  if(n) std::memcpy(d.data(), w, n * W * 8);
  return d;
}

template <size_t N>
void from_dets(const std::vector<std::bitset<N>>& d, uint64_t* w) {
  if(!d.empty()) std::memcpy(w, d.data(), d.size() * (N / 64) * 8);
}

struct HamBase {
  int nbits;
  size_t norb;
  std::vector<double> T, V;
  HamBase(int b, size_t n, std::vector<double> t, std::vector<double> v)
      : nbits(b), norb(n), T(std::move(t)), V(std::move(v)) {}
  virtual ~HamBase() = default;
};

template <size_t N>
struct Ham : HamBase {
  macis::DoubleLoopHamiltonianGenerator<N> gen;
  Ham(size_t n, std::vector<double> t, std::vector<double> v)
      : HamBase(int(N), n, std::move(t), std::move(v)),
        gen(macis::matrix_span<double>(T.data(), n, n),
            macis::rank4_span<double>(V.data(), n, n, n, n)) {}
};

struct Csr {
  sparsexx::csr_matrix<double, int32_t> A;
};

struct AsciSettingsC {
  uint64_t ntdets_max, ntdets_min, ncdets_max;
  double h_el_tol, rv_prune_tol;
  uint64_t pair_size_max;
  int32_t just_singles, pad_;
  uint64_t grow_factor, max_refine_iter;
  double refine_energy_tol;
};

struct CiSettingsC {
  double ci_res_tol;
  uint64_t ci_max_subspace;
  double ci_matel_tol;
};

macis::ASCISettings to_asci(const AsciSettingsC* s) {
  macis::ASCISettings a;
  a.ntdets_max = s->ntdets_max;
  a.ntdets_min = s->ntdets_min;
  a.ncdets_max = s->ncdets_max;
  a.h_el_tol = s->h_el_tol;
  a.rv_prune_tol = s->rv_prune_tol;
  a.pair_size_max = s->pair_size_max;
  a.just_singles = s->just_singles != 0;
  a.grow_factor = s->grow_factor;
  a.max_refine_iter = s->max_refine_iter;
  a.refine_energy_tol = s->refine_energy_tol;
  return a;
}

macis::MCSCFSettings to_ci(const CiSettingsC* s) {
  macis::MCSCFSettings m;
  m.ci_res_tol = s->ci_res_tol;
  m.ci_max_subspace = s->ci_max_subspace;
  m.ci_matel_tol = s->ci_matel_tol;
  return m;
}

template <size_t N>
Csr* build_csr(Ham<N>* h, const uint64_t* bra, size_t nbra,
               const uint64_t* ket, size_t nket, double thresh, int nthreads) {
  auto B = to_dets<N>(bra, nbra);
  auto K = to_dets<N>(ket, nket);
  if(nthreads <= 1 || nbra < size_t(4 * nthreads)) {
    auto A = macis::make_csr_hamiltonian_block<int32_t>(
        B.begin(), B.end(), K.begin(), K.end(), h->gen, thresh);
    return new Csr{std::move(A)};
  }
  // Row blocks on separate threads, each through the reference API.
  std::vector<sparsexx::csr_matrix<double, int32_t>> parts(nthreads);
  std::vector<std::thread> th;
  // Interleaved small blocks balance the cost of rows of different length.
  const size_t nblk = size_t(nthreads) * 16;
  std::vector<sparsexx::csr_matrix<double, int32_t>> blocks(nblk);
  std::atomic<size_t> next{0};
  for(int t = 0; t < nthreads; ++t)
    th.emplace_back([&]() {
      for(size_t b; (b = next.fetch_add(1)) < nblk;) {
        size_t lo = nbra * b / nblk, hi = nbra * (b + 1) / nblk;
        blocks[b] = macis::make_csr_hamiltonian_block<int32_t>(
            B.begin() + lo, B.begin() + hi, K.begin(), K.end(), h->gen,
            thresh);
      }
    });
  for(auto& x : th) x.join();
  size_t nnz = 0;
  for(auto& b : blocks) nnz += b.nnz();
  std::vector<int32_t> rp(nbra + 1), ci;
  std::vector<double> nz;
  ci.reserve(nnz);
  nz.reserve(nnz);
  size_t row = 0;
  rp[0] = 0;
  for(auto& b : blocks) {
    const int32_t base = int32_t(ci.size());
    for(int64_t i = 0; i < b.m(); ++i) rp[row + i + 1] = base + b.rowptr()[i + 1];
    ci.insert(ci.end(), b.colind().begin(), b.colind().end());
    nz.insert(nz.end(), b.nzval().begin(), b.nzval().end());
    row += b.m();
  }
  return new Csr{sparsexx::csr_matrix<double, int32_t>(
      nbra, nket, std::move(rp), std::move(ci), std::move(nz))};
}

}  // namespace

extern "C" {

const char* mref_last_error() { return g_err.c_str(); }

void mref_set_threads(int n) {
  openblas_set_num_threads(n);
}

void* mref_ham_create(int nbits, size_t norb, const double* T,
                      const double* V) {
  quiet_loggers();
  std::vector<double> t(T, T + norb * norb),
      v(V, V + norb * norb * norb * norb);
  if(nbits == 64) return new Ham<64>(norb, std::move(t), std::move(v));
  if(nbits == 128) return new Ham<128>(norb, std::move(t), std::move(v));
  g_err = "reference supports nbits 64 or 128 only";
  return nullptr;
}

void mref_ham_free(void* h) { delete static_cast<HamBase*>(h); }

// DoubleLoopHamiltonianGenerator::form_rdms (double_loop.hpp:117-165) with
// bra = ket = dets, the compute_casci_rdms form (cas.hpp:52-56); results are
// added to ordm (norb^2) and trdm (norb^4, or NULL).
int mref_form_rdms(void* hv, const uint64_t* dets, size_t n, double* C,
                   double* ordm, double* trdm) {
  auto* hb = static_cast<HamBase*>(hv);
  const size_t m = hb->norb;
  macis::matrix_span<double> o(ordm, m, m);
  macis::rank4_span<double> t(trdm, m, m, m, m);
  if(hb->nbits == 64) {
    auto D = to_dets<64>(dets, n);
    static_cast<Ham<64>*>(hb)->gen.form_rdms(D.begin(), D.end(), D.begin(),
                                             D.end(), C, o, t);
  } else {
    auto D = to_dets<128>(dets, n);
    static_cast<Ham<128>*>(hb)->gen.form_rdms(D.begin(), D.end(), D.begin(),
                                              D.end(), C, o, t);
  }
  return 0;
}

// Batched matrix_element(bra, ket) (hamiltonian_generator/matrix_elements.hpp:15)
int mref_matrix_element(void* hv, const uint64_t* bra, const uint64_t* ket,
                        size_t n, double* out) {
  auto* hb = static_cast<HamBase*>(hv);
  if(hb->nbits == 64) {
    auto* h = static_cast<Ham<64>*>(hb);
    auto B = to_dets<64>(bra, n), K = to_dets<64>(ket, n);
    for(size_t i = 0; i < n; ++i) out[i] = h->gen.matrix_element(B[i], K[i]);
  } else {
    auto* h = static_cast<Ham<128>*>(hb);
    auto B = to_dets<128>(bra, n), K = to_dets<128>(ket, n);
    for(size_t i = 0; i < n; ++i) out[i] = h->gen.matrix_element(B[i], K[i]);
  }
  return 0;
}

// fast_diag_{single,ss_double,os_double} with orbital-energy recomputation
// (hamiltonian_generator/fast_diagonals.hpp:236,261,288). kind: 1 single,
// 2 same-spin double, 3 opposite-spin double. occ lists are ascending.
int mref_fast_diag(void* hv, int kind, const uint32_t* ss_occ, size_t nss,
                   const uint32_t* os_occ, size_t nos, const uint32_t* orbs,
                   double hii, double* out) {
  auto* hb = static_cast<HamBase*>(hv);
  std::vector<uint32_t> ss(ss_occ, ss_occ + nss), os(os_occ, os_occ + nos);
  auto run = [&](auto& gen) {
    if(kind == 1)
      *out = gen.fast_diag_single(ss, os, orbs[0], orbs[1], hii);
    else if(kind == 2)
      *out = gen.fast_diag_ss_double(ss, os, orbs[0], orbs[1], orbs[2],
                                     orbs[3], hii);
    else
      *out = gen.fast_diag_os_double(ss, os, orbs[0], orbs[1], orbs[2],
                                     orbs[3], hii);
  };
  if(hb->nbits == 64)
    run(static_cast<Ham<64>*>(hb)->gen);
  else
    run(static_cast<Ham<128>*>(hb)->gen);
  return 0;
}

void* mref_csr_build(void* hv, const uint64_t* bra, size_t nbra,
                     const uint64_t* ket, size_t nket, double thresh,
                     int nthreads) {
  try {
    auto* hb = static_cast<HamBase*>(hv);
    if(hb->nbits == 64)
      return build_csr(static_cast<Ham<64>*>(hb), bra, nbra, ket, nket,
                       thresh, nthreads);
    return build_csr(static_cast<Ham<128>*>(hb), bra, nbra, ket, nket, thresh,
                     nthreads);
  } catch(std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

int64_t mref_csr_nnz(void* c) { return static_cast<Csr*>(c)->A.nnz(); }

void mref_csr_copy(void* c, int32_t* rowptr, int32_t* colind, double* nzval) {
  auto& A = static_cast<Csr*>(c)->A;
  std::memcpy(rowptr, A.rowptr().data(), A.rowptr().size() * 4);
  std::memcpy(colind, A.colind().data(), A.colind().size() * 4);
  std::memcpy(nzval, A.nzval().data(), A.nzval().size() * 8);
}

void mref_csr_free(void* c) { delete static_cast<Csr*>(c); }

// AV = alpha * A * V + beta * AV, K columns.
void mref_spmv(void* c, int64_t K, double alpha, const double* V, int64_t LDV,
               double beta, double* AV, int64_t LDAV) {
  auto& A = static_cast<Csr*>(c)->A;
  sparsexx::spblas::gespmbv(K, alpha, A, V, LDV, beta, AV, LDAV);
}

// extract_diagonal_elements (sparsexx/util/submatrix.hpp:264)
void mref_csr_diagonal(void* c, double* D) {
  auto d = sparsexx::extract_diagonal_elements(static_cast<Csr*>(c)->A);
  std::copy(d.begin(), d.end(), D);
}

// diagonal_guess + davidson on a built CSR (tests/davidson.cxx:56-60 order).
int mref_davidson(void* c, int64_t max_m, double tol, double* X, double* E,
                  int64_t* niter) {
  try {
    quiet_loggers();
    auto& A = static_cast<Csr*>(c)->A;
    std::fill_n(X, A.n(), 0.0);
    macis::diagonal_guess(A.n(), A, X);
    auto D = sparsexx::extract_diagonal_elements(A);
    auto [it, e] = macis::davidson(A.n(), max_m,
                                   macis::SparseMatrixOperator(A), D.data(),
                                   tol, X);
    *E = e;
    *niter = int64_t(it);
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

int mref_selected_ci_diag(void* hv, const uint64_t* dets, size_t ndets,
                          double h_el_tol, size_t max_m, double tol,
                          double* C, double* E) {
  try {
    quiet_loggers();
    auto* hb = static_cast<HamBase*>(hv);
    auto run = [&](auto* h, auto D) {
      std::vector<double> X(C, C + ndets);
      *E = macis::selected_ci_diag(D.begin(), D.end(), h->gen, h_el_tol,
                                   max_m, tol, X);
      std::copy(X.begin(), X.end(), C);
    };
    if(hb->nbits == 64)
      run(static_cast<Ham<64>*>(hb), to_dets<64>(dets, ndets));
    else
      run(static_cast<Ham<128>*>(hb), to_dets<128>(dets, ndets));
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

struct Pairs {
  std::vector<uint64_t> states;
  std::vector<double> rv;
};

// Raw ASCI contributions followed by sort_and_accumulate (the pair list the
// top-k works on, before the core merge).
void* mref_asci_pairs(void* hv, const AsciSettingsC* s, const uint64_t* cdets,
                      size_t ncdets, double E0, const double* C,
                      int accumulate) {
  try {
    quiet_loggers();
    auto* hb = static_cast<HamBase*>(hv);
    auto* P = new Pairs;
    auto run = [&](auto* h, auto D) {
      constexpr size_t N = typename decltype(D)::value_type().size();
      std::vector<double> Cv(C, C + ncdets);
      auto pairs = macis::asci_contributions_standard<N>(
          to_asci(s), D.begin(), D.end(), E0, Cv, h->norb, h->gen.T(),
          h->gen.G_red(), h->gen.V_red(), h->gen.G(), h->gen.V(), h->gen);
      if(accumulate) macis::sort_and_accumulate_asci_pairs(pairs);
      P->states.resize(pairs.size() * (N / 64));
      P->rv.resize(pairs.size());
      for(size_t i = 0; i < pairs.size(); ++i) {
        std::memcpy(&P->states[i * (N / 64)], &pairs[i].state, N / 8);
        P->rv[i] = pairs[i].rv;
      }
    };
    if(hb->nbits == 64)
      run(static_cast<Ham<64>*>(hb), to_dets<64>(cdets, ncdets));
    else
      run(static_cast<Ham<128>*>(hb), to_dets<128>(cdets, ncdets));
    return P;
  } catch(std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

size_t mref_pairs_size(void* p) { return static_cast<Pairs*>(p)->rv.size(); }
void mref_pairs_copy(void* p, uint64_t* states, double* rv) {
  auto* P = static_cast<Pairs*>(p);
  std::copy(P->states.begin(), P->states.end(), states);
  std::copy(P->rv.begin(), P->rv.end(), rv);
}
void mref_pairs_free(void* p) { delete static_cast<Pairs*>(p); }

// asci_search: out_dets must hold ndets_max + ncdets determinants.
int mref_asci_search(void* hv, const AsciSettingsC* s, size_t ndets_max,
                     const uint64_t* cdets, size_t ncdets, double E0,
                     const double* C, uint64_t* out_dets, size_t* nout) {
  try {
    quiet_loggers();
    auto* hb = static_cast<HamBase*>(hv);
    auto run = [&](auto* h, auto D) {
      std::vector<double> Cv(C, C + ncdets);
      auto nd = macis::asci_search(to_asci(s), ndets_max, D.begin(), D.end(),
                                   E0, Cv, h->norb, h->gen.T(),
                                   h->gen.G_red(), h->gen.V_red(),
                                   h->gen.G(), h->gen.V(), h->gen);
      from_dets(nd, out_dets);
      *nout = nd.size();
    };
    if(hb->nbits == 64)
      run(static_cast<Ham<64>*>(hb), to_dets<64>(cdets, ncdets));
    else
      run(static_cast<Ham<128>*>(hb), to_dets<128>(cdets, ncdets));
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// asci_grow (refine=0) or asci_refine (refine=1). dets/C hold n_in on entry
// and must have room for the returned wavefunction (ntdets_max for grow).
int mref_asci_run(void* hv, int refine, const AsciSettingsC* s,
                  const CiSettingsC* ci, double* E0, uint64_t* dets,
                  double* C, size_t n_in, size_t* n_out) {
  try {
    quiet_loggers();
    auto* hb = static_cast<HamBase*>(hv);
    auto run = [&](auto* h, auto D) {
      std::vector<double> X(C, C + n_in);
      double e = *E0;
      if(refine)
        std::tie(e, D, X) = macis::asci_refine(to_asci(s), to_ci(ci), e,
                                               std::move(D), std::move(X),
                                               h->gen, h->norb);
      else
        std::tie(e, D, X) = macis::asci_grow(to_asci(s), to_ci(ci), e,
                                             std::move(D), std::move(X),
                                             h->gen, h->norb);
      *E0 = e;
      from_dets(D, dets);
      std::copy(X.begin(), X.end(), C);
      *n_out = D.size();
    };
    if(hb->nbits == 64)
      run(static_cast<Ham<64>*>(hb), to_dets<64>(dets, n_in));
    else
      run(static_cast<Ham<128>*>(hb), to_dets<128>(dets, n_in));
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// FCI space in the reference order (sd_operations.hpp:461).
size_t mref_hilbert_space(int nbits, size_t norb, size_t na, size_t nb,
                          uint64_t* out) {
  if(nbits == 64) {
    auto d = macis::generate_hilbert_space<64>(norb, na, nb);
    if(out) from_dets(d, out);
    return d.size();
  }
  auto d = macis::generate_hilbert_space<128>(norb, na, nb);
  if(out) from_dets(d, out);
  return d.size();
}

// CISD space around the canonical HF determinant (sd_operations.hpp:422).
size_t mref_cisd_space(int nbits, size_t norb, size_t na, size_t nb,
                       uint64_t* out) {
  if(nbits == 64) {
    auto hf = macis::canonical_hf_determinant<64>(na, nb);
    auto d = macis::generate_cisd_hilbert_space<64>(norb, hf);
    if(out) from_dets(d, out);
    return d.size();
  }
  auto hf = macis::canonical_hf_determinant<128>(na, nb);
  auto d = macis::generate_cisd_hilbert_space<128>(norb, hf);
  if(out) from_dets(d, out);
  return d.size();
}

// read_wavefunction<64> (wavefunction_io.hpp:39-74): the number of
// determinants (at most cap copied out), or -1 when the reader throws.
long mref_read_wavefunction(const char* fname, uint64_t* dets, double* coeffs,
                            size_t cap) {
  try {
    std::vector<std::bitset<64>> st;
    std::vector<double> c;
    macis::read_wavefunction<64>(fname, st, c);
    for(size_t i = 0; i < st.size() && i < cap; ++i) {
      dets[i] = st[i].to_ullong();
      coeffs[i] = c[i];
    }
    return long(st.size());
  } catch(std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// read_fcidump_norb / _core / _1body / _2body (fcidump.cxx:78-182): with
// T == NULL only *norb; else T (norb^2) and V (norb^4) must be zeroed by the
// caller, leading dimensions norb. -1 when the reader throws.
int mref_read_fcidump(const char* fname, uint32_t* norb, double* T, double* V,
                      double* core) {
  try {
    *norb = macis::read_fcidump_norb(fname);
    if(T) {
      *core = macis::read_fcidump_core(fname);
      macis::read_fcidump_1body(fname, T, *norb);
      macis::read_fcidump_2body(fname, V, *norb);
    }
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// write_fcidump (fcidump.cxx:184-207). The writer registers an spdlog
// logger named "fcidump"; it is dropped afterwards, which closes the file
// and lets the next call register it again.
int mref_write_fcidump(const char* fname, size_t norb, const double* T,
                       const double* V, double core) {
  try {
    macis::write_fcidump(fname, norb, T, norb, V, norb, core);
    spdlog::drop("fcidump");
    return 0;
  } catch(std::exception& e) {
    spdlog::drop("fcidump");
    g_err = e.what();
    return -1;
  }
}

// read_rdms_binary / write_rdms_binary (fcidump.cxx:209-276), leading
// dimensions norb; -1 when they throw.
int mref_read_rdms_binary(const char* fname, size_t norb, double* ORDM,
                          double* TRDM) {
  try {
    macis::read_rdms_binary(fname, norb, ORDM, norb, TRDM, norb);
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int mref_write_rdms_binary(const char* fname, size_t norb, const double* ORDM,
                           const double* TRDM) {
  try {
    macis::write_rdms_binary(fname, norb, ORDM, norb, TRDM, norb);
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// write_wavefunction<64> (wavefunction_io.hpp:88-114); -1 when it throws.
int mref_write_wavefunction(const char* fname, size_t norb,
                            const uint64_t* dets, const double* coeffs,
                            size_t n, size_t nc) {
  try {
    std::vector<std::bitset<64>> st(n);
    for(size_t i = 0; i < n; ++i) st[i] = std::bitset<64>(dets[i]);
    std::vector<double> c(coeffs, coeffs + nc);
    macis::write_wavefunction<64>(fname, norb, st, c);
    return 0;
  } catch(std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"

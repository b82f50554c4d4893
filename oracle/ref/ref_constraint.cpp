// The reference's constraint-partitioned ASCI contribution path, compiled
// from the UNMODIFIED reference headers with MPI enabled against the serial
// shim in shim_mpi/ (test infrastructure only; see oracle/ref/Makefile).
//
//   mrefc_asci_pairs -> macis::asci_contributions_constraint
//                       (include/macis/asci/determinant_search.hpp:143-391)
//                       as rank `rank` of a job of `world` ranks: the
//                       constraints that dist_constraint_general
//                       (asci/mask_constraints.hpp:486-605) assigns to that
//                       rank, each constraint's contributions sorted and
//                       accumulated on their own (the "Local S&A for each
//                       quad" of the reference).
// The reference's MPI asci_search runs this on every rank and selects the
// top-k over all ranks with dist_quickselect; this library gives the
// per-rank pair lists, so that a test can run every rank in one process.
#include <spdlog/sinks/null_sink.h>
#include <spdlog/spdlog.h>

#include <cstring>
#include <macis/asci/determinant_search.hpp>
#include <macis/hamiltonian_generator/double_loop.hpp>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

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

struct AsciSettingsC {
  uint64_t ntdets_max, ntdets_min, ncdets_max;
  double h_el_tol, rv_prune_tol;
  uint64_t pair_size_max;
  int32_t just_singles, pad_;
  uint64_t grow_factor, max_refine_iter;
  double refine_energy_tol;
};

struct Pairs {
  std::vector<uint64_t> states;
  std::vector<double> rv;
};

}  // namespace

#define MREFC_API extern "C" __attribute__((visibility("default")))

MREFC_API const char* mrefc_last_error(void) { return g_err.c_str(); }

MREFC_API void* mrefc_ham_create(int nbits, size_t norb, const double* T,
                       const double* V) {
  try {
    std::vector<double> t(T, T + norb * norb);
    std::vector<double> v(V, V + norb * norb * norb * norb);
    if(nbits == 64) return new Ham<64>(norb, std::move(t), std::move(v));
    if(nbits == 128) return new Ham<128>(norb, std::move(t), std::move(v));
    g_err = "nbits must be 64 or 128";
  } catch(std::exception& e) {
    g_err = e.what();
  }
  return nullptr;
}

MREFC_API void mrefc_ham_free(void* h) { delete static_cast<HamBase*>(h); }

MREFC_API void* mrefc_asci_pairs(void* hv, const AsciSettingsC* s, int constraint_level,
                       const uint64_t* cdets, size_t ncdets, double E0,
                       const double* C, int rank, int world) {
  try {
    if(!spdlog::get("asci_search")) spdlog::null_logger_mt("asci_search");
    if(world < 1 || rank < 0 || rank >= world || world > 0x7FFF) {
      g_err = "bad rank / world";
      return nullptr;
    }
    auto* hb = static_cast<HamBase*>(hv);
    auto* P = new Pairs;
    auto go = [&](auto* h, auto tag) {
      constexpr size_t N = decltype(tag)::value;
      std::vector<std::bitset<N>> D(ncdets);
      if(ncdets) std::memcpy(D.data(), cdets, ncdets * (N / 8));
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
      a.constraint_level = constraint_level;
      std::vector<double> Cv(C, C + ncdets);
      const MPI_Comm comm = (world << 16) | rank;
      auto pairs = macis::asci_contributions_constraint<N>(
          a, D.begin(), D.end(), E0, Cv, h->norb, h->gen.T(), h->gen.G_red(),
          h->gen.V_red(), h->gen.G(), h->gen.V(), h->gen, comm);
      P->states.resize(pairs.size() * (N / 64));
      P->rv.resize(pairs.size());
      for(size_t i = 0; i < pairs.size(); ++i) {
        std::memcpy(&P->states[i * (N / 64)], &pairs[i].state, N / 8);
        P->rv[i] = pairs[i].rv;
      }
    };
    if(hb->nbits == 64)
      go(static_cast<Ham<64>*>(hb), std::integral_constant<size_t, 64>{});
    else
      go(static_cast<Ham<128>*>(hb), std::integral_constant<size_t, 128>{});
    return P;
  } catch(std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

MREFC_API size_t mrefc_pairs_size(void* p) { return static_cast<Pairs*>(p)->rv.size(); }
MREFC_API void mrefc_pairs_copy(void* p, uint64_t* states, double* rv) {
  auto* P = static_cast<Pairs*>(p);
  std::copy(P->states.begin(), P->states.end(), states);
  std::copy(P->rv.begin(), P->rv.end(), rv);
}
MREFC_API void mrefc_pairs_free(void* p) { delete static_cast<Pairs*>(p); }

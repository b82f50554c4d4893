// Drop-in check (test infrastructure): the reference's own templates run
// with the B200 generator plugged into the HamiltonianGenerator virtual hook
// (include/macis/hamiltonian_generator.hpp:66-72), compared with the
// reference DoubleLoopHamiltonianGenerator on the same inputs.
//
//   dropin_check T.bin V.bin norb nalpha nbeta ntdets_max
//
// T.bin / V.bin are raw column-major float64 integrals. Prints one JSON line.
#include <spdlog/sinks/null_sink.h>
#include <spdlog/spdlog.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <macis/asci/grow.hpp>
#include <macis/csr_hamiltonian.hpp>
#include <macis/hamiltonian_generator/double_loop.hpp>
#include <macis/solvers/selected_ci_diag.hpp>
#include <macis_b200/macis_b200.hpp>

static std::vector<double> load(const char* f, size_t n) {
  std::vector<double> v(n);
  std::ifstream in(f, std::ios::binary);
  in.read(reinterpret_cast<char*>(v.data()), n * 8);
  if(!in) throw std::runtime_error(std::string("cannot read ") + f);
  return v;
}

int main(int argc, char** argv) {
  if(argc < 7) return 2;
  for(const char* n : {"davidson", "ci_solver", "asci_search", "asci_grow",
                       "asci_refine"})
    spdlog::null_logger_mt(n);
  const size_t norb = std::stoul(argv[3]), na = std::stoul(argv[4]),
               nb = std::stoul(argv[5]), ntdets = std::stoul(argv[6]);
  auto T = load(argv[1], norb * norb);
  auto V = load(argv[2], norb * norb * norb * norb);
  macis::matrix_span<double> Ts(T.data(), norb, norb);
  macis::rank4_span<double> Vs(V.data(), norb, norb, norb, norb);
  macis::DoubleLoopHamiltonianGenerator<64> cpu(Ts, Vs);
  macis_b200::HamiltonianGenerator<64> gpu(Ts, Vs);

  auto hf = macis::canonical_hf_determinant<64>(na, nb);
  auto dets = macis::generate_cisd_hilbert_space<64>(norb, hf);
  // 1. the reference free function through the virtual hook
  auto Hc = macis::make_csr_hamiltonian<int32_t>(dets.begin(), dets.end(),
                                                 cpu, 1e-16);
  auto Hg = macis::make_csr_hamiltonian<int32_t>(dets.begin(), dets.end(),
                                                 gpu, 1e-16);
  const bool csr_equal = Hc.rowptr() == Hg.rowptr() &&
                         Hc.colind() == Hg.colind() && Hc.nzval() == Hg.nzval();
  // 2. the reference selected_ci_diag on both generators (CPU Davidson),
  //    and the shim's GPU-resident selected_ci_diag
  std::vector<double> C1, C2, C3;
  const double e_cpu = macis::selected_ci_diag<64, int32_t>(
      dets.begin(), dets.end(), cpu, 1e-16, 15, 1e-8, C1);
  const double e_hook = macis::selected_ci_diag<64, int32_t>(
      dets.begin(), dets.end(), gpu, 1e-16, 15, 1e-8, C2);
  const double e_gpu = macis_b200::selected_ci_diag<64, int32_t>(
      dets.begin(), dets.end(), gpu, 1e-16, 15, 1e-8, C3);
  // 3. the reference's own davidson driving the matrix-free operator
  macis_b200::MatrixFreeOperator<64> mf(gpu, dets.begin(), dets.end(), 1e-16);
  const auto D = mf.diagonal();
  std::vector<double> X4(dets.size(), 0.0);
  X4[std::min_element(D.begin(), D.end()) - D.begin()] = 1.0;
  const double e_mf =
      macis::davidson(int64_t(dets.size()), 15, mf, D.data(), 1e-8, X4.data())
          .second;
  // 4. form_rdms through the virtual hook on both generators
  const size_t m = norb;
  std::vector<double> o1(m * m, 0.0), t1(m * m * m * m, 0.0), o2(o1), t2(t1);
  cpu.form_rdms(dets.begin(), dets.end(), dets.begin(), dets.end(), C1.data(),
                macis::matrix_span<double>(o1.data(), m, m),
                macis::rank4_span<double>(t1.data(), m, m, m, m));
  static_cast<macis::HamiltonianGenerator<64>&>(gpu).form_rdms(
      dets.begin(), dets.end(), dets.begin(), dets.end(), C1.data(),
      macis::matrix_span<double>(o2.data(), m, m),
      macis::rank4_span<double>(t2.data(), m, m, m, m));
  double rdm_diff = 0;
  for(size_t i = 0; i < o1.size(); ++i)
    rdm_diff = std::max(rdm_diff, std::abs(o1[i] - o2[i]));
  for(size_t i = 0; i < t1.size(); ++i)
    rdm_diff = std::max(rdm_diff, std::abs(t1[i] - t2[i]));
  // 5. ASCI grow with the shim drivers
  macis::ASCISettings as;
  as.ntdets_max = ntdets;
  macis::MCSCFSettings ms;
  std::vector<macis::wfn_t<64>> w = {hf};
  std::vector<double> X = {1.0};
  double E0 = gpu.matrix_element(hf, hf);
  std::tie(E0, w, X) = macis_b200::asci_grow<64>(as, ms, E0, w, X, gpu, norb);
  double nrm = 0;
  for(double x : X) nrm += x * x;
  // 6. the same grow with learned screening: (a) recording and training
  //    only, which must not change the searches; (b) pruning by prediction
  //    from the third search on
  auto screened_grow = [&](macis_b200::ScreenSettings& sc) {
    std::vector<macis::wfn_t<64>> ws = {hf};
    std::vector<double> Xs = {1.0};
    double Es = gpu.matrix_element(hf, hf);
    std::tie(Es, ws, Xs) =
        macis_b200::asci_grow<64>(as, ms, Es, ws, Xs, gpu, norb, &sc);
    return std::make_pair(Es, ws.size());
  };
  macis_b200::ScreeningNetwork net_rec(64, 0), net_scr(64, 0);
  macis_b200::ScreenSettings rec;
  rec.network = &net_rec;
  rec.warmup_searches = size_t(-1);
  const auto [e_rec, n_rec] = screened_grow(rec);
  macis_b200::ScreenSettings scr;
  scr.network = &net_scr;
  scr.keep_frac = 0.5;
  scr.epochs = 8;
  scr.min_units = 0;
  scr.warmup_searches = 2;
  const auto [e_scr, n_scr] = screened_grow(scr);
  const auto st = macis_b200::last_search_stats(gpu);
  std::printf(
      "{\"ndets\": %zu, \"nnz\": %ld, \"csr_equal\": %s, \"e_cpu\": %.15g, "
      "\"e_hook\": %.15g, \"e_gpu\": %.15g, \"e_matrix_free\": %.15g, "
      "\"rdm_max_diff\": %.3g, \"asci_e0\": %.15g, \"asci_size\": %zu, "
      "\"asci_norm\": %.15g, \"rec_e0\": %.15g, \"rec_size\": %zu, "
      "\"rec_trained\": %zu, \"rec_searches\": %zu, \"scr_e0\": %.15g, "
      "\"scr_size\": %zu, \"scr_trained\": %zu, \"scr_units_kept\": %llu, "
      "\"scr_units_total\": %llu}\n",
      dets.size(), long(Hg.nnz()), csr_equal ? "true" : "false", e_cpu,
      e_hook, e_gpu, e_mf, rdm_diff, E0, w.size(), nrm, e_rec, n_rec,
      net_rec.trained_steps(), size_t(rec.searches), e_scr, n_scr,
      net_scr.trained_steps(), (unsigned long long)st.units_kept,
      (unsigned long long)st.units_total);
  return 0;
}

/* CPU oracle for the selected-CI hot path: a plain-C restatement of the
 * reference MACIS algorithms. TEST INFRASTRUCTURE ONLY -- the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it as the
 * checker; the product never links or calls it.
 *
 * Determinants are arrays of little-endian uint64 words, nbits/64 words per
 * determinant, in the std::bitset<N> word layout the reference uses
 * (include/macis/bitset_operations.hpp:264-286): for nbits=64 the alpha string
 * is bits 0..31 and beta bits 32..63 of word 0; for nbits=128 alpha is word 0
 * and beta word 1; for nbits=256 (which the reference cannot instantiate,
 * bitset_operations.hpp:267) alpha is words 0-1 and beta words 2-3.
 * Integrals are column-major: T(p,q) = T[p + q*n], V(p,q,r,s) =
 * V[p + q*n + r*n^2 + s*n^3] (include/macis/types.hpp:22-33).
 */
#ifndef MACIS_ORACLE_H
#define MACIS_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ham orc_ham;

typedef struct {
  uint64_t ntdets_max, ntdets_min, ncdets_max;
  double h_el_tol, rv_prune_tol;
  uint64_t pair_size_max;
  int32_t just_singles, pad_;
  uint64_t grow_factor, max_refine_iter;
  double refine_energy_tol;
} orc_asci_settings;

orc_ham* orc_ham_create(int nbits, size_t norb, const double* T,
                        const double* V);
void orc_ham_free(orc_ham* h);

/* matrix_element(bra, ket) for n pairs (matrix_elements.hpp:15-134). */
void orc_matrix_element(const orc_ham* h, const uint64_t* bra,
                        const uint64_t* ket, size_t n, double* out);

/* DoubleLoop CSR (double_loop.hpp:31-98). Two calls: count (colind==NULL)
 * fills rowptr and returns nnz; fill writes colind/nzval. int64 indices. */
int64_t orc_build_csr(const orc_ham* h, const uint64_t* bra, size_t nbra,
                      const uint64_t* ket, size_t nket, double thresh,
                      int64_t* rowptr, int64_t* colind, double* nzval);

/* AV = alpha*A*V + beta*AV, one column, sequential row sums (spmbv.hpp:39). */
void orc_spmv(size_t m, const int64_t* rowptr, const int64_t* colind,
              const double* nzval, double alpha, const double* x, double beta,
              double* y);

/* diagonal_guess + davidson (davidson.hpp:62-225) with a Jacobi eigensolver
 * for the Rayleigh-Ritz step. Returns 0 on convergence, 1 otherwise. */
int orc_davidson(size_t n, const int64_t* rowptr, const int64_t* colind,
                 const double* nzval, int64_t max_m, double tol, double* X,
                 int use_guess, double* E, int64_t* niter);

/* ASCI contributions of the core dets (determinant_search.hpp:54-141,
 * determinant_contributions.hpp:26-160) followed by a STABLE sort by
 * determinant and accumulation (determinant_sort.hpp:40-83). Returns the
 * number of unique pairs; call with states==NULL for the count. */
size_t orc_asci_pairs(const orc_ham* h, const orc_asci_settings* s,
                      const uint64_t* cdets, size_t ncdets, double E0,
                      const double* C, int accumulate, uint64_t* states,
                      double* rv);

/* asci_search (determinant_search.hpp:395-663): out_dets holds up to
 * ndets_max + ncdets dets; top-k ties are broken by ascending determinant and
 * the top-k states are returned in ascending determinant order, followed by
 * the core dets. */
size_t orc_asci_search(const orc_ham* h, const orc_asci_settings* s,
                       size_t ndets_max, const uint64_t* cdets, size_t ncdets,
                       double E0, const double* C, uint64_t* out_dets);

/* Orbital energies and fast diagonals (fast_diagonals.hpp:15-128). */
void orc_single_orbital_ens(const orc_ham* h, const uint32_t* ss_occ,
                            size_t nss, const uint32_t* os_occ, size_t nos,
                            double* eps);
double orc_fast_diag_single(const orc_ham* h, double hol_en, double par_en,
                            uint32_t hol, uint32_t par, double hii);
double orc_fast_diag_ss_double(const orc_ham* h, double h1, double h2,
                               double p1, double p2, uint32_t oh1,
                               uint32_t oh2, uint32_t op1, uint32_t op2,
                               double hii);
double orc_fast_diag_os_double(const orc_ham* h, double hu, double hd,
                               double pu, double pd, uint32_t ohu,
                               uint32_t ohd, uint32_t opu, uint32_t opd,
                               double hii);

/* generate_hilbert_space (sd_operations.hpp:441-476); out may be NULL. */
size_t orc_hilbert_space(int nbits, size_t norb, size_t na, size_t nb,
                         uint64_t* out);
/* canonical_hf_determinant (sd_operations.hpp:32-37). */
void orc_hf_det(int nbits, size_t na, size_t nb, uint64_t* out);
/* generate_cisd_hilbert_space (sd_operations.hpp:422-430); out may be NULL */
size_t orc_cisd_space(int nbits, size_t norb, size_t na, size_t nb,
                      uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif

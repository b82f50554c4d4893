/* macis_b200 -- C ABI of the B200 (sm_100a) selected-CI hot path.
 *
 * Plain pointers and sizes only. Each entry point names the reference MACIS
 * interface it replaces (paths relative to the MACIS source tree). The C++
 * drop-in shim include/macis_b200/macis_b200.hpp wraps these calls behind
 * the reference's own template API.
 *
 * Determinants: arrays of little-endian uint64 words, nbits/64 words per
 * determinant, in the std::bitset<nbits> layout (nbits = 64, 128 or 256):
 *   nbits=64 : word0 bits 0..31 alpha, bits 32..63 beta
 *   nbits=128: word0 alpha, word1 beta
 *   nbits=256: words 0-1 alpha, words 2-3 beta
 * Integrals: column-major T(p,q) = T[p + q*LDT], V(p,q,r,s) =
 * V[p + LDV*(q + LDV*(r + LDV*s))] (include/macis/types.hpp:22-33).
 *
 * Memory: pointer arguments are host memory unless MACIS_B200_DEVICE_PTRS is
 * set in `flags`, in which case they are device (HBM) pointers on the
 * library's current device. All calls are synchronous at return and run on
 * one CUDA stream per handle. Handles are not thread-safe (neither is the
 * reference generator).
 *
 * Errors: every call returns 0 or one of the MACIS_B200_E* codes below;
 * macis_b200_last_error() returns the message of the last failure on the
 * calling thread. The C++ shim rethrows std::runtime_error with the
 * reference's messages.
 */
#ifndef MACIS_B200_H
#define MACIS_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MACIS_B200_OK 0
#define MACIS_B200_EINVAL 1    /* bad argument */
#define MACIS_B200_ENOMEM 2    /* device allocation failed */
#define MACIS_B200_ECAPACITY 3 /* result exceeds the index type / buffer */
#define MACIS_B200_ETIMEOUT 4  /* a bounded device wait gave up */
#define MACIS_B200_ENOCONV 5   /* Davidson did not converge */
#define MACIS_B200_ECUDA 6     /* CUDA runtime error */
#define MACIS_B200_ENOGROW 7   /* ASCI search returned too few dets */

#define MACIS_B200_DEVICE_PTRS 1u /* pointer arguments are device memory */

/* Davidson precision modes. */
#define MACIS_B200_FP64 0  /* FP64 H values and FP64 vectors */
#define MACIS_B200_MIXED 1 /* FP32 off-diagonal H, FP64 diagonal, FP64
                              residual / CGS2 / Rayleigh-Ritz / energy */

typedef struct macis_b200_ham macis_b200_ham;
typedef struct macis_b200_csr macis_b200_csr;

/* ASCI settings, field for field macis::ASCISettings
 * (include/macis/asci/determinant_search.hpp:34-51). */
typedef struct {
  uint64_t ntdets_max, ntdets_min, ncdets_max;
  double h_el_tol, rv_prune_tol;
  uint64_t pair_size_max;
  int32_t just_singles, pad_;
  uint64_t grow_factor, max_refine_iter;
  double refine_energy_tol;
} macis_b200_asci_settings;

/* Diagnostics of the last asci_search call on a handle. */
typedef struct {
  uint64_t raw_pairs;     /* contributions generated (after h_el_tol) */
  uint64_t unique_pairs;  /* after sort + accumulate */
  uint64_t kept_pairs;    /* after dropping core dets, zero scores and, in
                             ranges after the running top-k first filled,
                             scores below its k-th score */
  uint64_t batches;       /* core-det batches used */
  double pairs_ms, sort_ms, keep_ms, topk_ms, total_ms;
  uint64_t units_total;   /* work units of the search (see asci_screen) */
  uint64_t units_kept;    /* units scored exactly */
  uint64_t samples;       /* training samples recorded into the network */
  double screen_ms;       /* prediction + selection + recording */
  double predict_ms;      /* network forward over all units (device time) */
  uint64_t sort_pass_items; /* sum over the sorted candidate ranges of
                               (radix digit passes x records): each pass
                               reads and writes every record once */
  uint64_t alpha_strings;   /* alpha strings of the core dets whose alpha
                               doubles the candidate ranges read from
                               per-range lists (those shared by the most
                               core dets), else 0 */
  uint64_t key_bits;        /* bits of the ranked candidate keys (alpha and
                               beta string ranks) the candidates were sorted
                               by, 0 when sorted by the determinant bitset */
  double rank_ms;           /* building the string rank tables */
} macis_b200_asci_stats;

/* Learned screening (no MACIS counterpart). A "unit" of the ASCI search is
 * one core determinant with one excitation class and, for doubles, one outer
 * (occupied, virtual) pair: the singles of a spin, or the inner loop of
 * append_ss_doubles / append_os_doubles_asci_contributions
 * (determinant_contributions.hpp:68-160) for fixed (i, a). The network
 * predicts each unit's largest log |score|; with use_net the search scores
 * exactly only the top keep_frac of the units (plus a random explore_frac)
 * and drops the rest before any contribution is generated. With
 * max_samples > 0 the search records up to that many (unit input, exact
 * target) pairs of the units it scored into the network, for
 * macis_b200_mlp_train with X == NULL. Target = (ln max|rv| + 20) / 5 with
 * max|rv| floored at 1e-12. */
typedef struct macis_b200_mlp macis_b200_mlp;
typedef struct {
  macis_b200_mlp* net;   /* may be NULL: exact search, nothing recorded */
  int32_t use_net;       /* 1: prune units by prediction */
  int32_t pad_;
  double keep_frac;      /* fraction of units kept by prediction, (0, 1] */
  double explore_frac;   /* extra random fraction kept, [0, 1] */
  uint64_t max_samples;  /* samples recorded (0: none) */
  uint64_t seed;
} macis_b200_asci_screen;

const char* macis_b200_last_error(void);
int macis_b200_version(void);
/* Number of kernels this library has launched in the process (benchmark
 * diagnostics; no reference counterpart). */
unsigned long long macis_b200_launch_count(void);
/* Time limit, in nanoseconds, of every barrier wait inside the tensor-core
 * kernels of the screening network (0 restores the default of 2 s; no
 * reference counterpart). A wait that runs out makes the call return
 * MACIS_B200_ETIMEOUT after the kernel has drained its copies and MMAs in
 * flight and freed its tensor memory; later calls run normally. A limit far
 * below a kernel's own waits forces that path, which the tests use. */
int macis_b200_set_wait_limit_ns(uint64_t ns);
/* Host-side fault injection for tests of the error paths (no reference
 * counterpart; the C++ shim maps the resulting codes to the reference's
 * exceptions). MACIS_B200_FAULT_ALLOC: after `arg` more successful device
 * allocations by the library, the next one reports out-of-memory
 * (MACIS_B200_ENOMEM), once. MACIS_B200_FAULT_INT32_LIMIT: CSR builds with
 * int32 indices reject more than `arg` nonzeros (MACIS_B200_ECAPACITY).
 * MACIS_B200_FAULT_NONE clears both. Process-wide; nothing fails on the
 * device. */
#define MACIS_B200_FAULT_NONE 0
#define MACIS_B200_FAULT_ALLOC 1
#define MACIS_B200_FAULT_INT32_LIMIT 2
int macis_b200_inject_fault(int kind, int64_t arg);

/* --- Hamiltonian generator ------------------------------------------------
 * Replaces the HamiltonianGenerator<N> constructor and
 * generate_integral_intermediates (include/macis/hamiltonian_generator.hpp:75,
 * hamiltonian_generator/impl.hpp:26-70): uploads T, V and builds G, G_red,
 * V_red, G2_red, V2_red in HBM. T and V are host pointers. */
int macis_b200_ham_create(int nbits, size_t norb, const double* T, size_t LDT,
                          const double* V, size_t LDV, macis_b200_ham** out);
int macis_b200_ham_destroy(macis_b200_ham* h);

/* Batched HamiltonianGenerator::matrix_element(bra, ket)
 * (hamiltonian_generator/matrix_elements.hpp:15-32). */
int macis_b200_matrix_element(macis_b200_ham* h, const uint64_t* bra,
                              const uint64_t* ket, size_t n, double* out,
                              unsigned flags);

/* --- CSR Hamiltonian build ------------------------------------------------
 * Replaces the make_csr_hamiltonian_block_32bit_/64bit_ virtual hook of
 * HamiltonianGenerator (hamiltonian_generator.hpp:66-72) as implemented by
 * DoubleLoopHamiltonianGenerator::make_csr_hamiltonian_block_
 * (hamiltonian_generator/double_loop.hpp:31-98): rows follow the bra list,
 * columns are ascending ket indices, entries with |h| > H_thresh are kept,
 * zero determinants give empty rows/columns. idx_bytes = 4 (int32_t) or 8
 * (int64_t); val_bytes = 8 (FP64 values) or 4 (FP32 off-diagonal values
 * with the FP64 diagonal kept separately, the MIXED precision mode). The
 * matrix stays in HBM, owned by the returned handle. */
int macis_b200_build_csr(macis_b200_ham* h, const uint64_t* bra, size_t nbra,
                         const uint64_t* ket, size_t nket, double H_thresh,
                         int idx_bytes, int val_bytes, unsigned flags,
                         macis_b200_csr** out);
int macis_b200_csr_destroy(macis_b200_csr* A);
/* m, n, nnz, idx_bytes, val_bytes of a built matrix. */
int macis_b200_csr_info(const macis_b200_csr* A, int64_t* m, int64_t* n,
                        int64_t* nnz, int* idx_bytes, int* val_bytes);
/* Copy the CSR arrays out (the by-value sparsexx::csr_matrix return of the
 * hook, sparsexx/matrix_types/csr_matrix.hpp:67-76): rowptr (m+1) and colind
 * (nnz) of idx_bytes each, nzval (nnz) of val_bytes each. Any pointer may be
 * NULL to skip that array. */
int macis_b200_csr_download(const macis_b200_csr* A, void* rowptr,
                            void* colind, void* nzval, unsigned flags);
/* Copy rows [r0, r1) out: rowptr gets the r1 - r0 + 1 stored offsets
 * rowptr[r0..r1] (absolute, as in the whole matrix), colind and nzval the
 * entries rowptr[r0] .. rowptr[r1] - 1. The row block that
 * make_dist_csr_hamiltonian gives one rank (csr_hamiltonian.hpp:49-82),
 * read out of a matrix built whole. Any pointer may be NULL. */
int macis_b200_csr_download_rows(const macis_b200_csr* A, int64_t r0,
                                 int64_t r1, void* rowptr, void* colind,
                                 void* nzval, unsigned flags);
/* Diagonal of the matrix, FP64 (sparsexx/util/submatrix.hpp:264-292). */
int macis_b200_csr_diagonal(const macis_b200_csr* A, double* D,
                            unsigned flags);

/* AV = alpha * A * V + beta * AV for K column vectors (column-major, leading
 * dimensions LDV, LDAV). Replaces sparsexx::spblas::gespmbv
 * (sparsexx/spblas/spmbv.hpp:39-73) behind SparseMatrixOperator::
 * operator_action (include/macis/solvers/davidson.hpp:47-58). */
int macis_b200_spmv(const macis_b200_csr* A, int64_t K, double alpha,
                    const double* V, int64_t LDV, double beta, double* AV,
                    int64_t LDAV, unsigned flags);

/* y = alpha * A * x + beta * y for one column, FP32-value (mixed) matrices
 * only, without allocating device memory. It has no counterpart in the
 * reference. It is meant for callers that may not allocate device memory
 * once they run -- for instance a service whose memory manager takes all of
 * HBM at start-up -- and it produces the same result as macis_b200_spmv.
 * x and y are device pointers on the matrix's device; the call runs on that
 * device whatever device is current and restores the caller's device. The
 * FP32 copy of x is kept in a fixed array compiled into the library
 * (4,194,304 entries, 16 MiB): matrices with more columns are rejected with
 * MACIS_B200_ECAPACITY. The array and the SpMV code are made resident on a
 * device by the first use of the library's SpMV there (CUDA loads device
 * modules lazily), which can allocate device memory and looks up the
 * array's device address: make that first call during set-up, before the
 * caller's memory manager takes HBM and before any stream capture. Later
 * calls allocate nothing, and the array then stays on that device until the
 * process exits. Every call reuses the same array, so calls that overlap on
 * the GPU (from several host threads or handles at once) race; calls return
 * after the product completes. */
int macis_b200_spmv_mixed_noalloc(const macis_b200_csr* A, double alpha,
                                  const double* x, double beta, double* y);

/* Single-vector Davidson for the lowest eigenpair of A, replacing
 * macis::davidson (include/macis/solvers/davidson.hpp:129-225) with the
 * diagonal preconditioner and CGS2 of the reference. X holds the guess on
 * entry when use_guess != 0 (else the diagonal_guess unit vector,
 * davidson.hpp:62-68) and the Ritz vector on exit. The precision follows
 * the matrix: val_bytes=8 is MACIS_B200_FP64, val_bytes=4 MACIS_B200_MIXED.
 * Returns MACIS_B200_ENOCONV (message "Davidson Did Not Converge!") when the
 * residual stays above tol after max_m basis vectors. */
int macis_b200_davidson(const macis_b200_csr* A, int64_t max_m, double tol,
                        int use_guess, double* X, double* E, int64_t* niter,
                        unsigned flags);

/* Device time per phase of the last Davidson solve on the calling thread
 * (CSR or matrix-free; diagnostics, no reference counterpart): the H
 * products, the new row of the Rayleigh matrix (multi-dot), the Ritz vector
 * with residual and preconditioned correction, and CGS2 with the thick-
 * restart rotations; wall_ms is the host time of the whole solve (the
 * difference is host work: the k x k eigensolve and synchronisation).
 * vector_bytes: algorithmic bytes of the Rayleigh, residual and CGS2 phases
 * (each column of V / AV read once per pass, vectors read / written once). */
typedef struct {
  int64_t iterations;
  double apply_ms, rayleigh_ms, residual_ms, ortho_ms, wall_ms;
  double vector_bytes;
} macis_b200_davidson_stats;
int macis_b200_davidson_last_stats(macis_b200_davidson_stats* out);

/* Davidson options beyond the reference signature. restart_keep = 0 keeps
 * the reference behaviour (no restart: stop after max_m basis vectors);
 * restart_keep > 0 compresses a full basis to its lowest restart_keep Ritz
 * vectors and continues (thick restart) until max_iter total iterations
 * (0: unbounded). */
typedef struct {
  int64_t max_m;
  double tol;
  int32_t use_guess;
  int32_t restart_keep;
  int64_t max_iter;
} macis_b200_davidson_opts;
int macis_b200_davidson_ex(const macis_b200_csr* A,
                           const macis_b200_davidson_opts* opts, double* X,
                           double* E, int64_t* niter, unsigned flags);

/* Matrix-free Hamiltonian over one determinant list, for lists whose CSR
 * matrix would not fit in device memory: every application evaluates the
 * elements again from the determinants and the integrals (the same
 * enumeration, Slater-Condon rules and threshold as macis_b200_build_csr,
 * double_loop.hpp:31-98) and accumulates H x without storing H. It stands
 * where the reference hands Davidson a SparseMatrixOperator
 * (include/macis/solvers/davidson.hpp:47-58): the reference's davidson
 * (:129-225) accepts any functor with operator_action. flags: with
 * MACIS_B200_HOP_FP32 the off-diagonal elements are rounded to FP32 before
 * the product (the values of an FP32-valued CSR matrix; the diagonal stays
 * FP64), MACIS_B200_DEVICE_PTRS for a device determinant list. Sums run in
 * enumeration order, not column order, so results agree with the CSR
 * product to rounding (~1e-15 relative), not bit for bit. */
#define MACIS_B200_HOP_FP32 2u
typedef struct macis_b200_hop macis_b200_hop;
int macis_b200_hop_create(const macis_b200_ham* h, const uint64_t* dets,
                          size_t ndets, double H_thresh, unsigned flags,
                          macis_b200_hop** out);
int macis_b200_hop_destroy(macis_b200_hop* op);
/* AV = alpha * H * V + beta * AV for K columns, as macis_b200_spmv. */
int macis_b200_hop_apply(const macis_b200_hop* op, int64_t K, double alpha,
                         const double* V, int64_t LDV, double beta, double* AV,
                         int64_t LDAV, unsigned flags);
/* Diagonal of H, FP64 (submatrix.hpp:264-292 on the matrix it stands for). */
int macis_b200_hop_diagonal(const macis_b200_hop* op, double* D,
                            unsigned flags);
/* macis_b200_davidson_ex with the matrix-free operator. */
int macis_b200_hop_davidson(const macis_b200_hop* op,
                            const macis_b200_davidson_opts* opts, double* X,
                            double* E, int64_t* niter, unsigned flags);

/* One- and two-particle reduced density matrices of the wavefunction C over
 * dets, added to ordm (norb x norb) and trdm (norb^4; may be NULL for the
 * 1-RDM alone), column-major like the integrals. Replaces
 * DoubleLoopHamiltonianGenerator::form_rdms (include/macis/
 * hamiltonian_generator/double_loop.hpp:117-165) with bra = ket = dets, the
 * way compute_casci_rdms calls it (include/macis/util/cas.hpp:52-56); the
 * contributions are those of include/macis/util/rdms.hpp:15-131, dispatched
 * in the same order. The sums are atomic, so results agree with the
 * reference to rounding, not bit for bit. */
int macis_b200_form_rdms(macis_b200_ham* h, const uint64_t* dets,
                         size_t ndets, const double* C, double* ordm,
                         double* trdm, unsigned flags);

/* Lowest nwant eigenpairs (W ascending, eigenvectors in the columns of Vec,
 * ld k) of the symmetric k x k matrix whose lower triangle is `lower`
 * (column-major, ld k): the syev step of lobpcgxx::rayleigh_ritz
 * (src/lobpcgxx/include/lobpcgxx/rayleigh_ritz.hpp:70-77) used inside
 * Davidson. Host-only; needs no GPU. */
int macis_b200_small_syev(int k, const double* lower, int nwant, double* W,
                          double* Vec);

/* Timings of the last build of a CSR handle (CUDA events on the build
 * stream): whole build, the fill kernel (the HBM-bound writer of colind /
 * nzval), the candidate count before thresholding and the path taken. */
typedef struct {
  double build_ms, fill_ms;
  int64_t nnz_candidates;
  int32_t direct_product, long_rows;
} macis_b200_build_stats;
int macis_b200_csr_build_stats(const macis_b200_csr* A,
                               macis_b200_build_stats* out);

/* --- ASCI search ----------------------------------------------------------
 * Replaces macis::asci_search (include/macis/asci/determinant_search.hpp:
 * 395-663) at MPI world size 1: singles/doubles contributions of the core
 * dets (determinant_contributions.hpp:26-160), sort + accumulate
 * (determinant_sort.hpp:40-83), core merge (determinant_sort.hpp:86-120,
 * determinant_search.hpp:528-544) and top-k (determinant_search.hpp:622-626).
 * out_dets must hold ndets_max + ncdets determinants; *nout receives the
 * count. The top-k states come first in ascending determinant order (ties at
 * the k-th score resolved towards smaller determinants), followed by the core
 * dets in input order. C holds the ncdets core coefficients. */
int macis_b200_asci_search(macis_b200_ham* h,
                           const macis_b200_asci_settings* s,
                           size_t ndets_max, const uint64_t* cdets,
                           size_t ncdets, double E0, const double* C,
                           uint64_t* out_dets, size_t* nout, unsigned flags);
/* One part of an exact ASCI search split over part_count processes (one
 * per GPU; no data is exchanged during the search). The candidate
 * determinants are divided by a hash of their alpha string into 4096 bins;
 * every part computes the same contribution histogram over the bins and
 * takes the bins where its cumulative load crosses part_index / part_count
 * and (part_index + 1) / part_count of the total. The part's result is its
 * candidates with their scores, core determinants and zero scores removed,
 * cut at the (ndets_max - ncdets)-th |score| with every tie kept: the union
 * over all parts, ordered by |score| descending then by determinant
 * (bitset order) ascending and cut at ndets_max - ncdets, is exactly the
 * top-k that macis_b200_asci_search returns for the same inputs (it then
 * lists it in ascending determinant order, followed by the core dets).
 * This replaces the reference's MPI search, which splits the work by alpha
 * constraints and selects the top-k with a distributed quickselect
 * (include/macis/asci/determinant_search.hpp:145-391,
 * include/macis/util/dist_quickselect.hpp). *nout receives the number of
 * candidates; macis_b200_asci_part_results copies them (states: nout x
 * words, scores: nout) to host memory. */
int macis_b200_asci_search_part(macis_b200_ham* h,
                                const macis_b200_asci_settings* s,
                                size_t ndets_max, const uint64_t* cdets,
                                size_t ncdets, double E0, const double* C,
                                uint32_t part_index, uint32_t part_count,
                                size_t* nout, unsigned flags);
int macis_b200_asci_part_results(const macis_b200_ham* h, uint64_t* states,
                                 double* scores);
/* macis_b200_asci_search_part with learned screening / sample recording
 * (scr as in macis_b200_asci_search_screened; may be NULL). The network
 * runs over all units on every part, so parts holding equal networks keep
 * the same units and their union is the screened whole search. A recording
 * part stores the same sample rows as the whole search, each target taken
 * over the part's bins only: the elementwise maximum of the parts' targets
 * (macis_b200_mlp_samples, then macis_b200_mlp_set_sample_targets) is the
 * whole search's. */
int macis_b200_asci_search_part_screened(macis_b200_ham* h,
                                         const macis_b200_asci_settings* s,
                                         const macis_b200_asci_screen* scr,
                                         size_t ndets_max,
                                         const uint64_t* cdets, size_t ncdets,
                                         double E0, const double* C,
                                         uint32_t part_index,
                                         uint32_t part_count, size_t* nout,
                                         unsigned flags);
/* The accumulated (state, score) pairs before the core merge -- the list the
 * reference top-k works on (determinant_search.hpp:498). Two calls: with
 * states == NULL only *npairs is set. States ascend. */
int macis_b200_asci_pairs(macis_b200_ham* h, const macis_b200_asci_settings* s,
                          const uint64_t* cdets, size_t ncdets, double E0,
                          const double* C, uint64_t* states, double* rv,
                          size_t* npairs);
int macis_b200_asci_last_stats(const macis_b200_ham* h,
                               macis_b200_asci_stats* out);

/* --- Learned screening network (no MACIS counterpart) ---------------------
 * din -> 256 -> 256 -> 1 with GELU, BF16 tcgen05 GEMMs with FP32
 * accumulation, FP32 master weights and Adam. Parameters are one FP32 array:
 * W1 [256][din] row-major, b1 [256], W2 [256][256], b2 [256], w3 [256],
 * b3 [1]. BF16 inputs are passed as their uint16 bit patterns. */
int macis_b200_mlp_create(int din, uint64_t seed, macis_b200_mlp** out);
int macis_b200_mlp_destroy(macis_b200_mlp* m);
int macis_b200_mlp_num_params(const macis_b200_mlp* m, size_t* n);
int macis_b200_mlp_get_params(const macis_b200_mlp* m, float* P);
/* Sets the master weights and resets the Adam state. */
int macis_b200_mlp_set_params(macis_b200_mlp* m, const float* P);
/* y[i] = network(X[i]) for X [n][din]. */
int macis_b200_mlp_forward(macis_b200_mlp* m, const uint16_t* X, size_t n,
                           float* y, unsigned flags);
/* Gradient of L = sum_i (y_i - t_i)^2 / (2 n) over all n rows (host grad,
 * num_params floats); *loss = L. No update. */
int macis_b200_mlp_gradients(macis_b200_mlp* m, const uint16_t* X,
                             const float* t, size_t n, float* grad,
                             double* loss, unsigned flags);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over shuffled minibatches; X == NULL
 * trains on the samples the last screened search recorded. *loss = mean
 * loss of the last epoch (may be NULL). */
int macis_b200_mlp_train(macis_b200_mlp* m, const uint16_t* X, const float* t,
                         size_t n, int epochs, int batch, double lr,
                         uint64_t seed, double* loss, unsigned flags);
/* Raise the recorded targets below their q-quantile to that value (the
 * ranking below it does not matter to a search that keeps the top units);
 * *floor = the value (may be NULL). */
int macis_b200_mlp_clamp_samples(macis_b200_mlp* m, double q, float* floor);
/* Overwrite the targets of the n recorded samples (n must equal their
 * count), e.g. with the maximum over the parts of a split search. */
int macis_b200_mlp_set_sample_targets(macis_b200_mlp* m, const float* t,
                                      size_t n);
/* Recorded samples (host copies; X may be NULL to query *n). */
int macis_b200_mlp_samples(const macis_b200_mlp* m, size_t* n, uint16_t* X,
                           float* t);
/* Network input width of the ASCI units of nbits-wide determinants. */
int macis_b200_asci_unit_width(int nbits);
/* macis_b200_asci_search with learned screening / sample recording. */
int macis_b200_asci_search_screened(macis_b200_ham* h,
                                    const macis_b200_asci_settings* s,
                                    const macis_b200_asci_screen* scr,
                                    size_t ndets_max, const uint64_t* cdets,
                                    size_t ncdets, double E0, const double* C,
                                    uint64_t* out_dets, size_t* nout,
                                    unsigned flags);
/* Network input rows of units [first, first + n) of the search over the
 * core dets (X [n][width], host); *nunits = the search's unit count. */
int macis_b200_asci_unit_features(macis_b200_ham* h, const uint64_t* cdets,
                                  size_t ncdets, double E0, const double* C,
                                  size_t first, size_t n, uint16_t* X,
                                  size_t* nunits);

#ifdef __cplusplus
}
#endif
#endif

/* CPU oracle for the selected-CI hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference MACIS algorithms, written to check
 * the CUDA path and to stand in for the reference where it cannot run
 * (bitset<256>, include/macis/bitset_operations.hpp:267). Each function cites
 * the reference file:line it follows; paths are relative to the MACIS tree.
 * Only the parity tests, the smoke check and the CPU-baseline leg of the
 * benchmark may call it. Summation orders are those of the reference; where
 * the reference leaves an order unspecified (std::sort, std::nth_element) the
 * oracle uses the stable / ascending-determinant choice documented in
 * macis_oracle.h.
 */
#include "macis_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- spins */
/* Spin strings of up to 128 orbitals (std::bitset<N/2>). */
typedef struct {
  uint64_t w[2];
} spin_t;

static inline spin_t sp_zero(void) {
  spin_t s = {{0, 0}};
  return s;
}
static inline spin_t sp_xor(spin_t a, spin_t b) {
  spin_t s = {{a.w[0] ^ b.w[0], a.w[1] ^ b.w[1]}};
  return s;
}
static inline spin_t sp_and(spin_t a, spin_t b) {
  spin_t s = {{a.w[0] & b.w[0], a.w[1] & b.w[1]}};
  return s;
}
static inline int sp_popc(spin_t a) {
  return __builtin_popcountll(a.w[0]) + __builtin_popcountll(a.w[1]);
}
static inline int sp_any(spin_t a) { return (a.w[0] | a.w[1]) != 0; }
/* ffs(bits) - 1 (bitset_operations.hpp:153-172); -1 when empty. */
static inline int sp_lowest(spin_t a) {
  if(a.w[0]) return __builtin_ctzll(a.w[0]);
  if(a.w[1]) return 64 + __builtin_ctzll(a.w[1]);
  return -1;
}
static inline int sp_test(spin_t a, int i) {
  return (int)((a.w[i >> 6] >> (i & 63)) & 1u);
}
static inline spin_t sp_flip(spin_t a, int i) {
  a.w[i >> 6] ^= (uint64_t)1 << (i & 63);
  return a;
}
/* full_mask<N>(i): bits [0, i) (bitset_operations.hpp:136-141). */
static inline spin_t sp_prefix(int i) {
  spin_t s = sp_zero();
  if(i >= 128) {
    s.w[0] = s.w[1] = ~(uint64_t)0;
  } else if(i >= 64) {
    s.w[0] = ~(uint64_t)0;
    s.w[1] = (i == 64) ? 0 : ((~(uint64_t)0) >> (128 - i));
  } else if(i > 0) {
    s.w[0] = (~(uint64_t)0) >> (64 - i);
  }
  return s;
}
/* bitset_less on full determinants: most significant word first
 * (bitset_operations.hpp:289-306). */
static int det_cmp(const uint64_t* a, const uint64_t* b, int nw) {
  for(int i = nw - 1; i >= 0; --i) {
    if(a[i] < b[i]) return -1;
    if(a[i] > b[i]) return 1;
  }
  return 0;
}

static inline spin_t det_alpha(const uint64_t* d, int nbits) {
  spin_t s = sp_zero();
  if(nbits == 64)
    s.w[0] = d[0] & 0xffffffffull;
  else if(nbits == 128)
    s.w[0] = d[0];
  else {
    s.w[0] = d[0];
    s.w[1] = d[1];
  }
  return s;
}
static inline spin_t det_beta(const uint64_t* d, int nbits) {
  spin_t s = sp_zero();
  if(nbits == 64)
    s.w[0] = d[0] >> 32;
  else if(nbits == 128)
    s.w[0] = d[1];
  else {
    s.w[0] = d[2];
    s.w[1] = d[3];
  }
  return s;
}
static inline void det_make(uint64_t* d, int nbits, spin_t a, spin_t b) {
  if(nbits == 64)
    d[0] = (a.w[0] & 0xffffffffull) | (b.w[0] << 32);
  else if(nbits == 128) {
    d[0] = a.w[0];
    d[1] = b.w[0];
  } else {
    d[0] = a.w[0];
    d[1] = a.w[1];
    d[2] = b.w[0];
    d[3] = b.w[1];
  }
}
static inline int det_popc(const uint64_t* d, int nw) {
  int c = 0;
  for(int i = 0; i < nw; ++i) c += __builtin_popcountll(d[i]);
  return c;
}

/* bits_to_indices (bitset_operations.hpp:206-217). */
static int to_indices(spin_t s, uint32_t* idx) {
  int c = 0;
  for(int i; (i = sp_lowest(s)) >= 0; s = sp_flip(s, i)) idx[c++] = i;
  return c;
}
/* bitset_to_occ_vir (sd_operations.hpp:82-97). */
static void occ_vir(size_t norb, spin_t s, uint32_t* occ, int* nocc,
                    uint32_t* vir, int* nvir) {
  *nocc = to_indices(s, occ);
  *nvir = (int)norb - *nocc;
  spin_t ns = {{~s.w[0], ~s.w[1]}};
  for(int i = 0; i < *nvir; ++i) {
    int a = sp_lowest(ns);
    vir[i] = a;
    ns = sp_flip(ns, a);
  }
}

/* single_excitation_sign (sd_operations.hpp:503-513). */
static double ex_sign(spin_t state, unsigned p, unsigned q) {
  spin_t mask;
  if(p > q)
    mask = sp_and(state, sp_xor(sp_prefix(p), sp_prefix(q + 1)));
  else
    mask = sp_and(state, sp_xor(sp_prefix(q), sp_prefix(p + 1)));
  return (sp_popc(mask) % 2) ? -1. : 1.;
}
/* first_occupied_flipped (sd_operations.hpp:497-500). */
static inline uint32_t fof(spin_t state, spin_t ex) {
  return (uint32_t)sp_lowest(sp_and(state, ex));
}

/* ---------------------------------------------------------- hamiltonian */
struct orc_ham {
  int nbits;
  size_t n;
  double *T, *V, *G, *G_red, *V_red, *G2_red, *V2_red;
};

#define IDX4(p, q, r, s, n) ((p) + (q) * (n) + (r) * (n) * (n) + (s) * (n) * (n) * (n))

/* HamiltonianGenerator::generate_integral_intermediates
 * (hamiltonian_generator/impl.hpp:26-70). */
orc_ham* orc_ham_create(int nbits, size_t n, const double* T,
                        const double* V) {
  orc_ham* h = (orc_ham*)calloc(1, sizeof(orc_ham));
  const size_t n2 = n * n, n3 = n2 * n, n4 = n3 * n;
  h->nbits = nbits;
  h->n = n;
  h->T = (double*)malloc(n2 * 8);
  h->V = (double*)malloc(n4 * 8);
  h->G = (double*)malloc(n4 * 8);
  h->G_red = (double*)malloc(n3 * 8);
  h->V_red = (double*)malloc(n3 * 8);
  h->G2_red = (double*)malloc(n2 * 8);
  h->V2_red = (double*)malloc(n2 * 8);
  memcpy(h->T, T, n2 * 8);
  memcpy(h->V, V, n4 * 8);
  memcpy(h->G, V, n4 * 8);
  for(size_t i = 0; i < n; ++i)
    for(size_t j = 0; j < n; ++j)
      for(size_t k = 0; k < n; ++k)
        for(size_t l = 0; l < n; ++l)
          h->G[IDX4(i, j, k, l, n)] -= V[IDX4(i, l, k, j, n)];
  for(size_t j = 0; j < n; ++j)
    for(size_t i = 0; i < n; ++i)
      for(size_t k = 0; k < n; ++k) {
        h->G_red[k + i * n + j * n2] = h->G[IDX4(k, k, i, j, n)];
        h->V_red[k + i * n + j * n2] = V[IDX4(k, k, i, j, n)];
      }
  for(size_t j = 0; j < n; ++j)
    for(size_t i = 0; i < n; ++i) {
      h->G2_red[i + j * n] = 0.5 * h->G[IDX4(i, i, j, j, n)];
      h->V2_red[i + j * n] = V[IDX4(i, i, j, j, n)];
    }
  return h;
}

void orc_ham_free(orc_ham* h) {
  if(!h) return;
  free(h->T);
  free(h->V);
  free(h->G);
  free(h->G_red);
  free(h->V_red);
  free(h->G2_red);
  free(h->V2_red);
  free(h);
}

/* matrix_element_4 (matrix_elements.hpp:55-61) with doubles_sign_indices
 * (sd_operations.hpp:528-543). */
static double me_4(const orc_ham* h, spin_t bra, spin_t ket, spin_t ex) {
  const uint32_t o1 = fof(ket, ex), v1 = fof(bra, ex);
  double sign = ex_sign(ket, v1, o1);
  ket = sp_flip(sp_flip(ket, o1), v1);
  ex = sp_flip(sp_flip(ex, o1), v1);
  const uint32_t o2 = fof(ket, ex), v2 = fof(bra, ex);
  sign *= ex_sign(ket, v2, o2);
  return sign * h->G[IDX4(v1, o1, v2, o2, h->n)];
}
/* matrix_element_22 (matrix_elements.hpp:63-74). */
static double me_22(const orc_ham* h, spin_t ba, spin_t ka, spin_t xa,
                    spin_t bb, spin_t kb, spin_t xb) {
  const uint32_t o1 = fof(ka, xa), v1 = fof(ba, xa);
  const double sa = ex_sign(ka, v1, o1);
  const uint32_t o2 = fof(kb, xb), v2 = fof(bb, xb);
  const double sb = ex_sign(kb, v2, o2);
  const double sign = sa * sb;
  return sign * h->V[IDX4(v1, o1, v2, o2, h->n)];
}
/* matrix_element_2 (matrix_elements.hpp:76-96). */
static double me_2(const orc_ham* h, spin_t bra, spin_t ket, spin_t ex,
                   const uint32_t* occ_s, int ns, const uint32_t* occ_o,
                   int no) {
  const uint32_t o1 = fof(ket, ex), v1 = fof(bra, ex);
  const double sign = ex_sign(ket, v1, o1);
  const size_t n = h->n;
  double h_el = h->T[v1 + o1 * n];
  const double* Gov = h->G_red + v1 * n + o1 * n * n;
  for(int i = 0; i < ns; ++i) h_el += Gov[occ_s[i]];
  const double* Vov = h->V_red + v1 * n + o1 * n * n;
  for(int i = 0; i < no; ++i) h_el += Vov[occ_o[i]];
  return sign * h_el;
}
/* matrix_element_diag (matrix_elements.hpp:98-125). */
static double me_diag(const orc_ham* h, const uint32_t* oa, int na,
                      const uint32_t* ob, int nb) {
  const size_t n = h->n;
  double e = 0;
  for(int i = 0; i < na; ++i) e += h->T[oa[i] * (n + 1)];
  for(int i = 0; i < nb; ++i) e += h->T[ob[i] * (n + 1)];
  for(int j = 0; j < na; ++j)
    for(int i = 0; i < na; ++i) e += h->G2_red[oa[i] + oa[j] * n];
  for(int j = 0; j < nb; ++j)
    for(int i = 0; i < nb; ++i) e += h->G2_red[ob[i] + ob[j] * n];
  for(int j = 0; j < nb; ++j)
    for(int i = 0; i < na; ++i) e += h->V2_red[oa[i] + ob[j] * n];
  return e;
}
/* matrix_element dispatch (matrix_elements.hpp:22-53). */
static double me_dispatch(const orc_ham* h, spin_t ba, spin_t ka, spin_t bb,
                          spin_t kb, const uint32_t* oa, int na,
                          const uint32_t* ob, int nb) {
  const spin_t xa = sp_xor(ba, ka), xb = sp_xor(bb, kb);
  const int ca = sp_popc(xa), cb = sp_popc(xb);
  if(ca + cb > 4) return 0.;
  if(ca == 4) return me_4(h, ba, ka, xa);
  if(cb == 4) return me_4(h, bb, kb, xb);
  if(ca == 2 && cb == 2) return me_22(h, ba, ka, xa, bb, kb, xb);
  if(ca == 2) return me_2(h, ba, ka, xa, oa, na, ob, nb);
  if(cb == 2) return me_2(h, bb, kb, xb, ob, nb, oa, na);
  return me_diag(h, oa, na, ob, nb);
}

void orc_matrix_element(const orc_ham* h, const uint64_t* bra,
                        const uint64_t* ket, size_t n, double* out) {
  const int nb = h->nbits, nw = nb / 64;
  uint32_t oa[128], ob[128];
  for(size_t i = 0; i < n; ++i) {
    const uint64_t *b = bra + i * nw, *k = ket + i * nw;
    spin_t ba = det_alpha(b, nb), bb = det_beta(b, nb);
    int na = to_indices(ba, oa), nbe = to_indices(bb, ob);
    out[i] = me_dispatch(h, ba, det_alpha(k, nb), bb, det_beta(k, nb), oa,
                         na, ob, nbe);
  }
}

/* DoubleLoopHamiltonianGenerator::make_csr_hamiltonian_block_
 * (double_loop.hpp:31-98). */
int64_t orc_build_csr(const orc_ham* h, const uint64_t* bra, size_t nbra,
                      const uint64_t* ket, size_t nket, double thresh,
                      int64_t* rowptr, int64_t* colind, double* nzval) {
  const int nb = h->nbits, nw = nb / 64;
  uint32_t oa[128], ob[128];
  int64_t nnz = 0;
  rowptr[0] = 0;
  for(size_t i = 0; i < nbra; ++i) {
    const uint64_t* b = bra + i * nw;
    if(det_popc(b, nw)) {
      spin_t ba = det_alpha(b, nb), bb = det_beta(b, nb);
      int na = to_indices(ba, oa), nbe = to_indices(bb, ob);
      for(size_t j = 0; j < nket; ++j) {
        const uint64_t* k = ket + j * nw;
        if(!det_popc(k, nw)) continue;
        int ex = 0;
        for(int w = 0; w < nw; ++w) ex += __builtin_popcountll(b[w] ^ k[w]);
        if(ex > 4) continue;
        double v = me_dispatch(h, ba, det_alpha(k, nb), bb, det_beta(k, nb),
                               oa, na, ob, nbe);
        if(fabs(v) > thresh) {
          if(colind) {
            colind[nnz] = (int64_t)j;
            nzval[nnz] = v;
          }
          nnz++;
        }
      }
    }
    if(colind && rowptr[i + 1] != nnz) return -1; /* count/fill mismatch */
    rowptr[i + 1] = nnz;
  }
  return nnz;
}

/* gespmbv for one column (spblas/spmbv.hpp:39-73). */
void orc_spmv(size_t m, const int64_t* rp, const int64_t* ci,
              const double* nz, double alpha, const double* x, double beta,
              double* y) {
  for(size_t i = 0; i < m; ++i) {
    double av = 0.;
    for(int64_t j = rp[i]; j < rp[i + 1]; ++j) av += nz[j] * x[ci[j]];
    y[i] = alpha * av + beta * y[i];
  }
}

/* ------------------------------------------------------------- davidson */
/* Cyclic Jacobi eigensolver for a symmetric k x k matrix given by its lower
 * triangle (column-major, ld k). Eigenvalues ascending in W, eigenvectors in
 * the columns of A on exit (the role dsyev plays in
 * lobpcgxx/rayleigh_ritz.hpp:75). */
static void jacobi_syev(int k, double* A, double* W) {
  double* a = (double*)malloc((size_t)k * k * 8);
  double* v = (double*)calloc((size_t)k * k, 8);
  for(int j = 0; j < k; ++j)
    for(int i = j; i < k; ++i) a[i + j * k] = a[j + i * k] = A[i + j * k];
  for(int i = 0; i < k; ++i) v[i + i * k] = 1.;
  for(int sweep = 0; sweep < 100; ++sweep) {
    double off = 0, tot = 0;
    for(int j = 0; j < k; ++j)
      for(int i = 0; i < k; ++i) {
        tot += a[i + j * k] * a[i + j * k];
        if(i != j) off += a[i + j * k] * a[i + j * k];
      }
    if(off <= 1e-30 * tot || off == 0) break;
    for(int p = 0; p < k; ++p)
      for(int q = p + 1; q < k; ++q) {
        const double apq = a[p + q * k];
        if(apq == 0) continue;
        const double app = a[p + p * k], aqq = a[q + q * k];
        const double theta = (aqq - app) / (2 * apq);
        const double t = (theta >= 0 ? 1. : -1.) /
                         (fabs(theta) + sqrt(theta * theta + 1.));
        const double c = 1. / sqrt(t * t + 1.), s = t * c;
        for(int r = 0; r < k; ++r) {
          const double arp = a[r + p * k], arq = a[r + q * k];
          a[r + p * k] = c * arp - s * arq;
          a[r + q * k] = s * arp + c * arq;
        }
        for(int r = 0; r < k; ++r) {
          const double apr = a[p + r * k], aqr = a[q + r * k];
          a[p + r * k] = c * apr - s * aqr;
          a[q + r * k] = s * apr + c * aqr;
        }
        for(int r = 0; r < k; ++r) {
          const double vrp = v[r + p * k], vrq = v[r + q * k];
          v[r + p * k] = c * vrp - s * vrq;
          v[r + q * k] = s * vrp + c * vrq;
        }
      }
  }
  /* sort ascending */
  int* ord = (int*)malloc(k * sizeof(int));
  for(int i = 0; i < k; ++i) ord[i] = i;
  for(int i = 1; i < k; ++i)
    for(int j = i; j > 0 && a[ord[j] * (k + 1)] < a[ord[j - 1] * (k + 1)];
        --j) {
      int t = ord[j];
      ord[j] = ord[j - 1];
      ord[j - 1] = t;
    }
  for(int c = 0; c < k; ++c) {
    W[c] = a[ord[c] * (k + 1)];
    for(int r = 0; r < k; ++r) A[r + c * k] = v[r + ord[c] * k];
  }
  free(ord);
  free(a);
  free(v);
}

static double dotp(size_t n, const double* x, const double* y) {
  double s = 0;
  for(size_t i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}

/* gram_schmidt (davidson.hpp:111-126): CGS2 then normalise. */
static void cgs2(size_t n, int64_t K, const double* Vo, double* vn) {
  double* inner = (double*)malloc(K * 8);
  for(int pass = 0; pass < 2; ++pass) {
    for(int64_t j = 0; j < K; ++j) inner[j] = dotp(n, Vo + j * n, vn);
    for(size_t i = 0; i < n; ++i) {
      double s = 0;
      for(int64_t j = 0; j < K; ++j) s += Vo[i + j * n] * inner[j];
      vn[i] -= s;
    }
  }
  const double nrm = sqrt(dotp(n, vn, vn));
  for(size_t i = 0; i < n; ++i) vn[i] *= 1. / nrm;
  free(inner);
}

int orc_davidson(size_t N, const int64_t* rp, const int64_t* ci,
                 const double* nz, int64_t max_m, double tol, double* X,
                 int use_guess, double* E, int64_t* niter) {
  /* extract_diagonal_elements (sparsexx/util/submatrix.hpp:264-292) */
  double* D = (double*)malloc(N * 8);
  for(size_t i = 0; i < N; ++i) {
    D[i] = 0;
    for(int64_t j = rp[i]; j < rp[i + 1]; ++j)
      if(ci[j] == (int64_t)i) {
        D[i] = nz[j];
        break;
      }
  }
  if(!use_guess) { /* diagonal_guess (davidson.hpp:62-68) */
    size_t imin = 0;
    for(size_t i = 1; i < N; ++i)
      if(D[i] < D[imin]) imin = i;
    for(size_t i = 0; i < N; ++i) X[i] = 0;
    X[imin] = 1.;
  }
  if(max_m > (int64_t)N) max_m = (int64_t)N;
  double* V = (double*)calloc(N * (max_m + 1), 8);
  double* AV = (double*)calloc(N * (max_m + 1), 8);
  double* C = (double*)calloc((max_m + 1) * (max_m + 1), 8);
  double* LAM = (double*)calloc(max_m + 1, 8);
  memcpy(V, X, N * 8);
  orc_spmv(N, rp, ci, nz, 1., V, 0., AV);
  memcpy(V + N, AV, N * 8);
  cgs2(N, 1, V, V + N);
  int converged = 0;
  int64_t iter = 1;
  for(int64_t i = 1; i < max_m; ++i, ++iter) {
    const int64_t k = i + 1;
    orc_spmv(N, rp, ci, nz, 1., V + i * N, 0., AV + i * N);
    /* rayleigh_ritz: C = V^T AV (lower triangle used) */
    for(int64_t c = 0; c < k; ++c)
      for(int64_t r = c; r < k; ++r)
        C[r + c * k] = dotp(N, V + r * N, AV + c * N);
    jacobi_syev((int)k, C, LAM);
    double* R = V + (i + 1) * N;
    for(size_t r = 0; r < N; ++r) {
      double x = 0, av = 0;
      for(int64_t c = 0; c < k; ++c) x += V[r + c * N] * C[c];
      for(int64_t c = 0; c < k; ++c) av += AV[r + c * N] * C[c];
      X[r] = x;
      R[r] = av - LAM[0] * x;
    }
    const double res = sqrt(dotp(N, R, R));
    if(res < tol) {
      converged = 1;
      break;
    }
    for(size_t r = 0; r < N; ++r) R[r] = -R[r] / (D[r] - LAM[0]);
    cgs2(N, k, V, R);
  }
  *E = LAM[0];
  *niter = iter;
  free(D);
  free(V);
  free(AV);
  free(C);
  free(LAM);
  return converged ? 0 : 1;
}

/* ----------------------------------------------------------------- ASCI */
void orc_single_orbital_ens(const orc_ham* h, const uint32_t* ss, size_t nss,
                            const uint32_t* os, size_t nos, double* eps) {
  /* single_orbital_ens (fast_diagonals.hpp:34-53) */
  const size_t n = h->n;
  for(size_t i = 0; i < n; ++i) {
    double e = h->T[i * (n + 1)];
    for(size_t q = 0; q < nss; ++q)
      e += h->G2_red[i + ss[q] * n] + h->G2_red[ss[q] + i * n];
    e -= h->G2_red[i * (n + 1)];
    for(size_t q = 0; q < nos; ++q) e += h->V2_red[i + os[q] * n];
    eps[i] = e;
  }
}

#define G2(p, q) h->G2_red[(p) + (size_t)(q) * h->n]
#define V2(p, q) h->V2_red[(p) + (size_t)(q) * h->n]
/* fast_diag_single (fast_diagonals.hpp:55-62) */
double orc_fast_diag_single(const orc_ham* h, double hol_en, double par_en,
                            uint32_t hol, uint32_t par, double hii) {
  return hii + par_en - hol_en - G2(par, hol) - G2(hol, par);
}
/* fast_diag_ss_double (fast_diagonals.hpp:74-87) */
double orc_fast_diag_ss_double(const orc_ham* h, double h1, double h2,
                               double p1, double p2, uint32_t oh1,
                               uint32_t oh2, uint32_t op1, uint32_t op2,
                               double hii) {
  return hii + p1 + p2 - h1 - h2 + G2(oh1, oh2) + G2(oh2, oh1) +
         G2(op1, op2) + G2(op2, op1) - G2(op1, oh1) - G2(oh1, op1) -
         G2(op2, oh1) - G2(oh1, op2) - G2(op1, oh2) - G2(oh2, op1) -
         G2(op2, oh2) - G2(oh2, op2);
}
/* fast_diag_os_double (fast_diagonals.hpp:103-114) */
double orc_fast_diag_os_double(const orc_ham* h, double hu, double hd,
                               double pu, double pd, uint32_t ohu,
                               uint32_t ohd, uint32_t opu, uint32_t opd,
                               double hii) {
  return hii + pu + pd - hu - hd + V2(ohu, ohd) + V2(opu, opd) -
         G2(opu, ohu) - G2(ohu, opu) - G2(opd, ohd) - G2(ohd, opd) -
         V2(opu, ohd) - V2(ohu, opd);
}

typedef struct {
  uint64_t* st; /* nw words per entry */
  double* rv;
  size_t n, cap;
  int nw;
} pairvec;

static void pv_push(pairvec* p, const uint64_t* s, double rv) {
  if(p->n == p->cap) {
    p->cap = p->cap ? 2 * p->cap : 1024;
    p->st = (uint64_t*)realloc(p->st, p->cap * p->nw * 8);
    p->rv = (double*)realloc(p->rv, p->cap * 8);
  }
  memcpy(p->st + p->n * p->nw, s, p->nw * 8);
  p->rv[p->n++] = rv;
}

/* Stable merge sort of an index permutation by determinant. */
static const uint64_t* g_sort_st;
static int g_sort_nw;
static void msort(size_t* idx, size_t* tmp, size_t n) {
  if(n < 2) return;
  size_t m = n / 2;
  msort(idx, tmp, m);
  msort(idx + m, tmp, n - m);
  size_t i = 0, j = m, k = 0;
  while(i < m && j < n) {
    if(det_cmp(g_sort_st + idx[j] * g_sort_nw, g_sort_st + idx[i] * g_sort_nw,
               g_sort_nw) < 0)
      tmp[k++] = idx[j++];
    else
      tmp[k++] = idx[i++];
  }
  while(i < m) tmp[k++] = idx[i++];
  while(j < n) tmp[k++] = idx[j++];
  memcpy(idx, tmp, n * sizeof(size_t));
}
static void pv_sort(pairvec* p) {
  size_t* idx = (size_t*)malloc((p->n + 1) * sizeof(size_t));
  size_t* tmp = (size_t*)malloc((p->n + 1) * sizeof(size_t));
  for(size_t i = 0; i < p->n; ++i) idx[i] = i;
  g_sort_st = p->st;
  g_sort_nw = p->nw;
  msort(idx, tmp, p->n);
  uint64_t* st = (uint64_t*)malloc((p->n + 1) * p->nw * 8);
  double* rv = (double*)malloc((p->n + 1) * 8);
  for(size_t i = 0; i < p->n; ++i) {
    memcpy(st + i * p->nw, p->st + idx[i] * p->nw, p->nw * 8);
    rv[i] = p->rv[idx[i]];
  }
  free(p->st);
  free(p->rv);
  p->st = st;
  p->rv = rv;
  p->cap = p->n + 1;
  free(idx);
  free(tmp);
}
/* sort_and_accumulate_asci_pairs (determinant_sort.hpp:40-83), stable. */
static void pv_sort_accumulate(pairvec* p) {
  if(!p->n) return;
  pv_sort(p);
  size_t u = 0;
  for(size_t i = 1; i < p->n; ++i) {
    if(det_cmp(p->st + i * p->nw, p->st + u * p->nw, p->nw) == 0)
      p->rv[u] += p->rv[i];
    else {
      ++u;
      if(u != i) {
        memcpy(p->st + u * p->nw, p->st + i * p->nw, p->nw * 8);
        p->rv[u] = p->rv[i];
      }
    }
  }
  p->n = u + 1;
}

/* append_singles_asci_contributions (determinant_contributions.hpp:25-66) */
static void add_singles(const orc_ham* h, double coeff, const uint64_t* state,
                        spin_t same, int beta, const uint32_t* occ, int no,
                        const uint32_t* vir, int nv, const uint32_t* othr,
                        int nt, const double* eps, double tol, double root,
                        double E0, pairvec* out) {
  const size_t n = h->n;
  const int nb = h->nbits, nw = nb / 64;
  uint64_t ex[4];
  for(int ii = 0; ii < no; ++ii)
    for(int aa = 0; aa < nv; ++aa) {
      const uint32_t i = occ[ii], a = vir[aa];
      double h_el = h->T[a + i * n];
      const double* Gov = h->G_red + a * n + i * n * n;
      const double* Vov = h->V_red + a * n + i * n * n;
      for(int p = 0; p < no; ++p) h_el += Gov[occ[p]];
      for(int p = 0; p < nt; ++p) h_el += Vov[othr[p]];
      if(fabs(h_el) < tol) continue;
      spin_t sa = det_alpha(state, nb), sb = det_beta(state, nb);
      if(beta)
        sb = sp_flip(sp_flip(sb, i), a);
      else
        sa = sp_flip(sp_flip(sa, i), a);
      det_make(ex, nb, sa, sb);
      h_el *= ex_sign(same, a, i);
      const double hd = orc_fast_diag_single(h, eps[i], eps[a], i, a, root);
      h_el /= (E0 - hd);
      pv_push(out, ex, coeff * h_el);
    }
  (void)nw;
}

/* append_ss_doubles_asci_contributions (determinant_contributions.hpp:68-120) */
static void add_ss_doubles(const orc_ham* h, double coeff,
                           const uint64_t* state, spin_t spin, int beta,
                           const uint32_t* occ, int no, const uint32_t* vir,
                           int nv, const double* eps, double tol, double root,
                           double E0, pairvec* out) {
  const size_t n = h->n, n2 = n * n;
  const int nb = h->nbits;
  uint64_t ex[4];
  for(int ii = 0; ii < no; ++ii)
    for(int aa = 0; aa < nv; ++aa) {
      const uint32_t i = occ[ii], a = vir[aa];
      const double* G_ai = h->G + (a + i * n) * n2;
      for(int jj = ii + 1; jj < no; ++jj)
        for(int bb = aa + 1; bb < nv; ++bb) {
          const uint32_t j = occ[jj], b = vir[bb];
          const double G_aibj = G_ai[b + j * n];
          if(fabs(G_aibj) < tol) continue;
          spin_t fx = sp_flip(sp_flip(sp_flip(sp_flip(sp_zero(), i), j), a), b);
          spin_t exs = sp_xor(spin, fx);
          /* doubles_sign(state_spin, ex_det_spin, full_ex_spin) */
          spin_t bra = spin, ket = exs, e = fx;
          const uint32_t o1 = fof(ket, e), v1 = fof(bra, e);
          double sign = ex_sign(ket, v1, o1);
          ket = sp_flip(sp_flip(ket, o1), v1);
          e = sp_flip(sp_flip(e, o1), v1);
          const uint32_t o2 = fof(ket, e), v2 = fof(bra, e);
          sign *= ex_sign(ket, v2, o2);
          spin_t sa = det_alpha(state, nb), sb = det_beta(state, nb);
          if(beta)
            sb = sp_xor(sb, fx);
          else
            sa = sp_xor(sa, fx);
          det_make(ex, nb, sa, sb);
          double h_el = sign * G_aibj;
          const double hd = orc_fast_diag_ss_double(
              h, eps[i], eps[j], eps[a], eps[b], i, j, a, b, root);
          h_el /= (E0 - hd);
          pv_push(out, ex, coeff * h_el);
        }
    }
}

/* append_os_doubles_asci_contributions (determinant_contributions.hpp:122-160) */
static void add_os_doubles(const orc_ham* h, double coeff,
                           const uint64_t* state, spin_t sa0, spin_t sb0,
                           const uint32_t* oa, int noa, const uint32_t* ob,
                           int nob, const uint32_t* va, int nva,
                           const uint32_t* vb, int nvb, const double* ea,
                           const double* eb, double tol, double root,
                           double E0, pairvec* out) {
  const size_t n = h->n, n2 = n * n;
  const int nb = h->nbits;
  uint64_t ex[4];
  for(int ii = 0; ii < noa; ++ii)
    for(int aa = 0; aa < nva; ++aa) {
      const uint32_t i = oa[ii], a = va[aa];
      const double* V_ai = h->V + a + i * n;
      const double sign_a = ex_sign(sa0, a, i);
      for(int jj = 0; jj < nob; ++jj)
        for(int bb = 0; bb < nvb; ++bb) {
          const uint32_t j = ob[jj], b = vb[bb];
          const double V_aibj = V_ai[(b + j * n) * n2];
          if(fabs(V_aibj) < tol) continue;
          const double sign_b = ex_sign(sb0, b, j);
          const double sign = sign_a * sign_b;
          spin_t sa = sp_flip(sp_flip(sa0, a), i);
          spin_t sb = sp_flip(sp_flip(sb0, j), b);
          det_make(ex, nb, sa, sb);
          double h_el = sign * V_aibj;
          const double hd = orc_fast_diag_os_double(h, ea[i], eb[j], ea[a],
                                                    eb[b], i, j, a, b, root);
          h_el /= (E0 - hd);
          pv_push(out, ex, coeff * h_el);
        }
    }
  (void)state;
}

/* asci_contributions_standard (determinant_search.hpp:54-141), without the
 * pair_size_max pruning (the parity regime keeps every pair). */
static void asci_contribs(const orc_ham* h, const orc_asci_settings* s,
                          const uint64_t* cdets, size_t ncdets, double E0,
                          const double* C, pairvec* out) {
  const int nb = h->nbits, nw = nb / 64;
  const size_t n = h->n;
  uint32_t oa[128], va[128], ob[128], vb[128];
  double* ea = (double*)malloc(n * 8);
  double* eb = (double*)malloc(n * 8);
  for(size_t c = 0; c < ncdets; ++c) {
    const uint64_t* st = cdets + c * nw;
    spin_t sa = det_alpha(st, nb), sb = det_beta(st, nb);
    const double coeff = C[c];
    int noa, nva, nob, nvb;
    occ_vir(n, sa, oa, &noa, va, &nva);
    occ_vir(n, sb, ob, &nob, vb, &nvb);
    orc_single_orbital_ens(h, oa, noa, ob, nob, ea);
    orc_single_orbital_ens(h, ob, nob, oa, noa, eb);
    const double hd = me_diag(h, oa, noa, ob, nob);
    const double tol = s->h_el_tol;
    add_singles(h, coeff, st, sa, 0, oa, noa, va, nva, ob, nob, ea, tol, hd,
                E0, out);
    add_singles(h, coeff, st, sb, 1, ob, nob, vb, nvb, oa, noa, eb, tol, hd,
                E0, out);
    if(!s->just_singles) {
      add_ss_doubles(h, coeff, st, sa, 0, oa, noa, va, nva, ea, tol, hd, E0,
                     out);
      add_ss_doubles(h, coeff, st, sb, 1, ob, nob, vb, nvb, eb, tol, hd, E0,
                     out);
      add_os_doubles(h, coeff, st, sa, sb, oa, noa, ob, nob, va, nva, vb, nvb,
                     ea, eb, tol, hd, E0, out);
    }
  }
  free(ea);
  free(eb);
}

size_t orc_asci_pairs(const orc_ham* h, const orc_asci_settings* s,
                      const uint64_t* cdets, size_t ncdets, double E0,
                      const double* C, int accumulate, uint64_t* states,
                      double* rv) {
  pairvec p = {0};
  p.nw = h->nbits / 64;
  asci_contribs(h, s, cdets, ncdets, E0, C, &p);
  if(accumulate) pv_sort_accumulate(&p);
  if(states) {
    memcpy(states, p.st, p.n * p.nw * 8);
    memcpy(rv, p.rv, p.n * 8);
  }
  size_t n = p.n;
  free(p.st);
  free(p.rv);
  return n;
}

static int g_topk_nw;
static const uint64_t* g_topk_st;
static const double* g_topk_rv;
static int topk_cmp(const void* x, const void* y) {
  size_t a = *(const size_t*)x, b = *(const size_t*)y;
  double fa = fabs(g_topk_rv[a]), fb = fabs(g_topk_rv[b]);
  if(fa > fb) return -1;
  if(fa < fb) return 1;
  return det_cmp(g_topk_st + a * g_topk_nw, g_topk_st + b * g_topk_nw,
                 g_topk_nw);
}

size_t orc_asci_search(const orc_ham* h, const orc_asci_settings* s,
                       size_t ndets_max, const uint64_t* cdets, size_t ncdets,
                       double E0, const double* C, uint64_t* out_dets) {
  const int nw = h->nbits / 64;
  pairvec p = {0};
  p.nw = nw;
  asci_contribs(h, s, cdets, ncdets, E0, C, &p);
  pv_sort_accumulate(&p);
  /* determinant_search.hpp:528-544: finalise scores, add the core dets with
   * |C|, keep the largest copy, drop entries with rv >= 0. */
  for(size_t i = 0; i < p.n; ++i) p.rv[i] = -fabs(p.rv[i]);
  for(size_t i = 0; i < ncdets; ++i) pv_push(&p, cdets + i * nw, fabs(C[i]));
  pv_sort(&p);
  size_t u = 0;
  for(size_t i = 1; i < p.n; ++i) {
    if(det_cmp(p.st + i * nw, p.st + u * nw, nw) == 0) {
      /* cur_it->rv = std::max(cur_it->rv, it->rv) */
      if(p.rv[u] < p.rv[i]) p.rv[u] = p.rv[i];
    } else {
      ++u;
      memmove(p.st + u * nw, p.st + i * nw, nw * 8);
      p.rv[u] = p.rv[i];
    }
  }
  if(p.n) p.n = u + 1;
  size_t m = 0;
  for(size_t i = 0; i < p.n; ++i)
    if(p.rv[i] < 0.0) {
      memmove(p.st + m * nw, p.st + i * nw, nw * 8);
      p.rv[m++] = p.rv[i];
    }
  p.n = m;
  const size_t topk = ndets_max - ncdets; /* size_t arithmetic as in :547 */
  size_t nout = 0;
  if(p.n > topk) {
    size_t* idx = (size_t*)malloc(p.n * sizeof(size_t));
    for(size_t i = 0; i < p.n; ++i) idx[i] = i;
    g_topk_nw = nw;
    g_topk_st = p.st;
    g_topk_rv = p.rv;
    qsort(idx, p.n, sizeof(size_t), topk_cmp);
    char* keep = (char*)calloc(p.n, 1);
    for(size_t i = 0; i < topk; ++i) keep[idx[i]] = 1;
    for(size_t i = 0; i < p.n; ++i)
      if(keep[i]) memcpy(out_dets + (nout++) * nw, p.st + i * nw, nw * 8);
    free(keep);
    free(idx);
  } else {
    for(size_t i = 0; i < p.n; ++i)
      memcpy(out_dets + (nout++) * nw, p.st + i * nw, nw * 8);
  }
  memcpy(out_dets + nout * nw, cdets, ncdets * nw * 8);
  nout += ncdets;
  free(p.st);
  free(p.rv);
  return nout;
}

/* ------------------------------------------------------------- spaces */
/* std::prev_permutation on a 0/1 array. */
static int prev_perm(unsigned char* v, size_t n) {
  if(n < 2) return 0;
  size_t i = n - 1;
  while(i > 0 && !(v[i - 1] > v[i])) --i;
  if(i == 0) {
    for(size_t a = 0, b = n - 1; a < b; ++a, --b) {
      unsigned char t = v[a];
      v[a] = v[b];
      v[b] = t;
    }
    return 0;
  }
  size_t j = n - 1;
  while(!(v[j] < v[i - 1])) --j;
  unsigned char t = v[i - 1];
  v[i - 1] = v[j];
  v[j] = t;
  for(size_t a = i, b = n - 1; a < b; ++a, --b) {
    t = v[a];
    v[a] = v[b];
    v[b] = t;
  }
  return 1;
}

/* generate_combs (sd_operations.hpp:440-458) */
static size_t combs(size_t nbits, size_t nset, spin_t* out) {
  unsigned char v[128] = {0};
  for(size_t i = 0; i < nset; ++i) v[i] = 1;
  size_t c = 0;
  do {
    spin_t t = sp_zero();
    for(size_t i = 0; i < nbits; ++i)
      if(v[i]) t = sp_flip(t, (int)i);
    if(out) out[c] = t;
    ++c;
  } while(prev_perm(v, nbits));
  return c;
}

size_t orc_hilbert_space(int nbits, size_t norb, size_t na, size_t nb,
                         uint64_t* out) {
  const size_t ca = combs(norb, na, NULL), cb = combs(norb, nb, NULL);
  if(!out) return ca * cb;
  spin_t* A = (spin_t*)malloc(ca * sizeof(spin_t));
  spin_t* B = (spin_t*)malloc(cb * sizeof(spin_t));
  combs(norb, na, A);
  combs(norb, nb, B);
  const int nw = nbits / 64;
  for(size_t i = 0; i < ca; ++i)
    for(size_t j = 0; j < cb; ++j) det_make(out + (i * cb + j) * nw, nbits, A[i], B[j]);
  free(A);
  free(B);
  return ca * cb;
}

void orc_hf_det(int nbits, size_t na, size_t nb, uint64_t* out) {
  det_make(out, nbits, sp_prefix((int)na), sp_prefix((int)nb));
}

/* generate_singles / generate_doubles on one spin (sd_operations.hpp:129-187) */
static size_t spin_singles(size_t norb, spin_t s, spin_t* out) {
  uint32_t occ[128], vir[128];
  int no, nv;
  occ_vir(norb, s, occ, &no, vir, &nv);
  size_t c = 0;
  for(int a = 0; a < nv; ++a)
    for(int i = 0; i < no; ++i) {
      if(out) out[c] = sp_flip(sp_flip(s, occ[i]), vir[a]);
      ++c;
    }
  return c;
}
static size_t spin_doubles(size_t norb, spin_t s, spin_t* out) {
  uint32_t occ[128], vir[128];
  int no, nv;
  occ_vir(norb, s, occ, &no, vir, &nv);
  size_t c = 0;
  for(int a = 0; a < nv; ++a)
    for(int i = 0; i < no; ++i)
      for(int b = a + 1; b < nv; ++b)
        for(int j = i + 1; j < no; ++j) {
          if(out)
            out[c] = sp_flip(sp_flip(sp_flip(sp_flip(s, occ[i]), vir[a]),
                                     occ[j]),
                             vir[b]);
          ++c;
        }
  return c;
}

/* generate_cisd_hilbert_space (sd_operations.hpp:361-430) */
size_t orc_cisd_space(int nbits, size_t norb, size_t na, size_t nb,
                      uint64_t* out) {
  uint64_t hf[4];
  orc_hf_det(nbits, na, nb, hf);
  spin_t a = det_alpha(hf, nbits), b = det_beta(hf, nbits);
  size_t nsa = spin_singles(norb, a, NULL), nsb = spin_singles(norb, b, NULL);
  size_t nda = spin_doubles(norb, a, NULL), ndb = spin_doubles(norb, b, NULL);
  size_t tot = 1 + nsa + nsb + nda + ndb + nsa * nsb;
  if(!out) return tot;
  spin_t* SA = (spin_t*)malloc((nsa + 1) * sizeof(spin_t));
  spin_t* SB = (spin_t*)malloc((nsb + 1) * sizeof(spin_t));
  spin_t* DA = (spin_t*)malloc((nda + 1) * sizeof(spin_t));
  spin_t* DB = (spin_t*)malloc((ndb + 1) * sizeof(spin_t));
  spin_singles(norb, a, SA);
  spin_singles(norb, b, SB);
  spin_doubles(norb, a, DA);
  spin_doubles(norb, b, DB);
  const int nw = nbits / 64;
  size_t c = 0;
  det_make(out + (c++) * nw, nbits, a, b);
  for(size_t i = 0; i < nsa; ++i) det_make(out + (c++) * nw, nbits, SA[i], b);
  for(size_t i = 0; i < nsb; ++i) det_make(out + (c++) * nw, nbits, a, SB[i]);
  for(size_t i = 0; i < nda; ++i) det_make(out + (c++) * nw, nbits, DA[i], b);
  for(size_t i = 0; i < ndb; ++i) det_make(out + (c++) * nw, nbits, a, DB[i]);
  for(size_t i = 0; i < nsa; ++i)
    for(size_t j = 0; j < nsb; ++j)
      det_make(out + (c++) * nw, nbits, SA[i], SB[j]);
  free(SA);
  free(SB);
  free(DA);
  free(DB);
  return c;
}

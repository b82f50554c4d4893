// BLAS front end used only to compile the reference MACIS/lobpcgxx headers
// for the CPU oracle (test infrastructure). The reference builds against
// blaspp (pinned in src/lobpcgxx/CMakeLists.txt:22-28); this shim exposes the
// same call shapes and forwards the double-precision routines the hot path
// calls (gemm, nrm2, dot, scal, copy, axpy, swap) to a Fortran BLAS.
// Routines that the path never instantiates are declared only.
#pragma once
#include <cstdint>
#include <complex>
#include <vector>

extern "C" {
void dgemm_(const char*, const char*, const int*, const int*, const int*,
            const double*, const double*, const int*, const double*,
            const int*, const double*, double*, const int*);
double dnrm2_(const int*, const double*, const int*);
double ddot_(const int*, const double*, const int*, const double*,
             const int*);
void dscal_(const int*, const double*, double*, const int*);
void dcopy_(const int*, const double*, const int*, double*, const int*);
void daxpy_(const int*, const double*, const double*, const int*, double*,
            const int*);
void dswap_(const int*, double*, const int*, double*, const int*);
}

namespace blas {

enum class Layout : char { ColMajor = 'C', RowMajor = 'R' };
enum class Op : char { NoTrans = 'N', Trans = 'T', ConjTrans = 'C' };
enum class Uplo : char { Upper = 'U', Lower = 'L', General = 'G' };
enum class Side : char { Left = 'L', Right = 'R' };
enum class Diag : char { NonUnit = 'N', Unit = 'U' };

inline char op_char(Op o) { return o == Op::NoTrans ? 'N' : 'T'; }

template <typename Alpha, typename Beta>
void gemm(Layout, Op ta, Op tb, int64_t m, int64_t n, int64_t k, Alpha alpha,
          const double* A, int64_t lda, const double* B, int64_t ldb,
          Beta beta, double* C, int64_t ldc) {
  if(m == 0 || n == 0) return;
  const char a = op_char(ta), b = op_char(tb);
  const int M = int(m), N = int(n), K = int(k), LA = int(lda), LB = int(ldb),
            LC = int(ldc);
  const double al = double(alpha), be = double(beta);
  dgemm_(&a, &b, &M, &N, &K, &al, A, &LA, B, &LB, &be, C, &LC);
}

inline double nrm2(int64_t n, const double* x, int64_t incx) {
  const int N = int(n), I = int(incx);
  return dnrm2_(&N, x, &I);
}
inline double dot(int64_t n, const double* x, int64_t incx, const double* y,
                  int64_t incy) {
  const int N = int(n), I = int(incx), J = int(incy);
  return ddot_(&N, x, &I, y, &J);
}
template <typename Alpha>
void scal(int64_t n, Alpha alpha, double* x, int64_t incx) {
  const int N = int(n), I = int(incx);
  const double a = double(alpha);
  dscal_(&N, &a, x, &I);
}
inline void copy(int64_t n, const double* x, int64_t incx, double* y,
                 int64_t incy) {
  const int N = int(n), I = int(incx), J = int(incy);
  dcopy_(&N, x, &I, y, &J);
}
template <typename Alpha>
void axpy(int64_t n, Alpha alpha, const double* x, int64_t incx, double* y,
          int64_t incy) {
  const int N = int(n), I = int(incx), J = int(incy);
  const double a = double(alpha);
  daxpy_(&N, &a, x, &I, y, &J);
}
inline void swap(int64_t n, double* x, int64_t incx, double* y,
                 int64_t incy) {
  const int N = int(n), I = int(incx), J = int(incy);
  dswap_(&N, x, &I, y, &J);
}

// Declared for the LOBPCG driver templates, which MACIS never instantiates.
template <typename... Args>
void trsm(Args&&...);

}  // namespace blas

// LAPACK front end used only to compile the reference MACIS/lobpcgxx headers
// for the CPU oracle (test infrastructure). The reference builds against
// lapackpp (pinned in src/lobpcgxx/CMakeLists.txt:22-28); this shim exposes
// the call shapes and forwards the symmetric eigensolver (syev, used by
// lobpcgxx::rayleigh_ritz, rayleigh_ritz.hpp:75) to a Fortran LAPACK.
// Routines that the path never instantiates are declared only.
#pragma once
#include <blas.hh>
#include <cstdint>
#include <vector>

extern "C" {
void dsyev_(const char*, const char*, const int*, double*, const int*, double*,
            double*, const int*, int*);
}

namespace lapack {

using blas::Op;
using blas::Side;
using blas::Uplo;
enum class Job : char {
  NoVec = 'N',
  Vec = 'V',
  OverwriteVec = 'O',
  AllVec = 'A',
  SomeVec = 'S'
};
enum class MatrixType : char { General = 'G', Lower = 'L', Upper = 'U' };

inline int64_t syev(Job jobz, Uplo uplo, int64_t n, double* A, int64_t lda,
                    double* W) {
  const char j = char(jobz), u = char(uplo);
  const int N = int(n), LA = int(lda);
  int info = 0, lwork = -1;
  double wq = 0;
  dsyev_(&j, &u, &N, A, &LA, W, &wq, &lwork, &info);
  lwork = int(wq);
  std::vector<double> work(lwork > 1 ? lwork : 1);
  dsyev_(&j, &u, &N, A, &LA, W, work.data(), &lwork, &info);
  return info;
}

// Declared for the LOBPCG driver templates, which MACIS never instantiates.
template <typename... Args>
int64_t potrf(Args&&...);
template <typename... Args>
int64_t gesvd(Args&&...);
template <typename... Args>
int64_t lacpy(Args&&...);
template <typename... Args>
int64_t gelqf(Args&&...);
template <typename... Args>
int64_t ormlq(Args&&...);

}  // namespace lapack

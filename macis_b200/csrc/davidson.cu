// Single-vector Davidson on the GPU, replacing macis::davidson
// (include/macis/solvers/davidson.hpp:129-225) and diagonal_guess (:62-68).
//
// Basis V and A*V live in HBM (N x (max_m+1) FP64 each). Per iteration:
//   AV_i = H V_i                                  (spmv.cu)
//   row i of the Rayleigh matrix V^T AV           (multi-dot, FP64)
//   k x k symmetric eigenproblem on the host      (cyclic Jacobi, FP64)
//   X = V c, R = AV c - lambda X, |R|, W = -R/(D - lambda)   (one fused pass)
//   CGS2 of W against V, normalise                (davidson.hpp:111-126)
// The reference recomputes the full k x k product with gemm every
// iteration; only its lower triangle enters syev (rayleigh_ritz.hpp:73-75),
// and the entries of earlier rows do not change, so only the new row is
// formed. Reductions are two-stage with a fixed order (deterministic).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "internal.hpp"
#include "primitives.cuh"

namespace mb {

constexpr int DV_THREADS = 256;
constexpr int DV_CHUNK = 8;  // columns per multi-dot pass

// partial[b * ncol + c] = sum over block b's rows of A[:, c0+c] . v
__global__ void __launch_bounds__(DV_THREADS)
    multidot_k(const double* __restrict__ Acols, int64_t lda, int ncol,
               const double* __restrict__ v, int64_t n,
               double* __restrict__ partial) {
  __shared__ double sh[DV_THREADS / 32][DV_CHUNK];
  double acc[DV_CHUNK];
#pragma unroll
  for(int c = 0; c < DV_CHUNK; ++c) acc[c] = 0;
  for(int64_t i = int64_t(blockIdx.x) * DV_THREADS + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * DV_THREADS) {
    const double x = v[i];
#pragma unroll
    for(int c = 0; c < DV_CHUNK; ++c)
      if(c < ncol) acc[c] += Acols[i + c * lda] * x;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for(int c = 0; c < DV_CHUNK; ++c) {
    double a = acc[c];
#pragma unroll
    for(int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if(lane == 0) sh[wid][c] = a;
  }
  __syncthreads();
  if(threadIdx.x < ncol) {
    double a = 0;
    for(int w = 0; w < DV_THREADS / 32; ++w) a += sh[w][threadIdx.x];
    partial[size_t(blockIdx.x) * ncol + threadIdx.x] = a;
  }
}

__global__ void reduce_partials_k(const double* partial, int nb, int ncol,
                                  double* out) {
  // one warp per column, fixed order
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x;
  double a = 0;
  for(int b = lane; b < nb; b += 32) a += partial[size_t(b) * ncol + c];
#pragma unroll
  for(int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if(lane == 0) out[c] = a;
}

// v -= A[:, 0:k] * coef
__global__ void cgs_update_k(const double* __restrict__ A, int64_t lda, int k,
                             const double* __restrict__ coef, double* v,
                             int64_t n) {
  __shared__ double cf[1024];
  for(int c = threadIdx.x; c < k; c += blockDim.x) cf[c] = coef[c];
  __syncthreads();
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * blockDim.x) {
    double s = 0;
    for(int c = 0; c < k; ++c) s += A[i + c * lda] * cf[c];
    v[i] -= s;
  }
}

__global__ void scale_k(double* v, int64_t n, const double* nrm2) {
  const double inv = 1. / sqrt(*nrm2);
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * blockDim.x)
    v[i] *= inv;
}

// X = V c; R = AV c - lam X; partial |R|^2; W = -R / (D - lam) into Wout.
__global__ void __launch_bounds__(DV_THREADS)
    ritz_residual_k(const double* __restrict__ V, const double* __restrict__ AV,
                    int64_t n, int k, const double* __restrict__ c, double lam,
                    const double* __restrict__ D, double* __restrict__ X,
                    double* __restrict__ W, double* __restrict__ partial) {
  __shared__ double cf[1024];
  __shared__ double sh[DV_THREADS / 32];
  for(int j = threadIdx.x; j < k; j += blockDim.x) cf[j] = c[j];
  __syncthreads();
  double acc = 0;
  for(int64_t i = int64_t(blockIdx.x) * DV_THREADS + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * DV_THREADS) {
    double x = 0, av = 0;
    for(int j = 0; j < k; ++j) {
      x += V[i + j * n] * cf[j];
      av += AV[i + j * n] * cf[j];
    }
    const double r = av - lam * x;
    X[i] = x;
    W[i] = -r / (D[i] - lam);
    acc += r * r;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for(int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if(lane == 0) sh[wid] = acc;
  __syncthreads();
  if(threadIdx.x == 0) {
    double a = 0;
    for(int w = 0; w < DV_THREADS / 32; ++w) a += sh[w];
    partial[blockIdx.x] = a;
  }
}

// Lowest `nwant` eigenpairs of the k x k Rayleigh matrix, given by its lower
// triangle (column-major, ld k) as dsyev with Uplo::Lower reads it
// (lobpcgxx/rayleigh_ritz.hpp:75). Householder reduction to tridiagonal
// form, Sturm-sequence bisection for each wanted eigenvalue, inverse
// iteration on the tridiagonal matrix, back-transformation and modified
// Gram-Schmidt among the returned vectors. W ascending; Vec columns.
void small_syev_lowest(int k, const double* lower, int nwant, double* W,
                       double* Vec) {
  std::vector<double> a(size_t(k) * k);
  for(int j = 0; j < k; ++j)
    for(int i = j; i < k; ++i) a[i + size_t(j) * k] = a[j + size_t(i) * k] = lower[i + size_t(j) * k];
  std::vector<double> d(k), e(k, 0.0);
  std::vector<std::vector<double>> refl;  // Householder vectors (length k)
  // tridiagonalise: A <- H A H with H = I - 2 v v^T acting on rows/cols j+1..
  for(int j = 0; j + 2 < k; ++j) {
    double nrm = 0;
    for(int i = j + 1; i < k; ++i) nrm += a[i + size_t(j) * k] * a[i + size_t(j) * k];
    nrm = std::sqrt(nrm);
    std::vector<double> v(k, 0.0);
    const double x0 = a[j + 1 + size_t(j) * k];
    if(nrm == 0) {
      refl.push_back(v);
      continue;
    }
    const double alpha = x0 > 0 ? -nrm : nrm;
    v[j + 1] = x0 - alpha;
    for(int i = j + 2; i < k; ++i) v[i] = a[i + size_t(j) * k];
    double vn = 0;
    for(int i = j + 1; i < k; ++i) vn += v[i] * v[i];
    vn = std::sqrt(vn);
    if(vn == 0) {
      refl.push_back(std::vector<double>(k, 0.0));
      continue;
    }
    for(int i = j + 1; i < k; ++i) v[i] /= vn;
    // p = A v ; K = v.p ; q = p - K v ; A <- A - 2 v q^T - 2 q v^T
    std::vector<double> p(k, 0.0);
    for(int c = j; c < k; ++c) {
      double s2 = 0;
      for(int r = j + 1; r < k; ++r) s2 += a[c + size_t(r) * k] * v[r];
      p[c] = s2;
    }
    double K = 0;
    for(int r = j + 1; r < k; ++r) K += v[r] * p[r];
    for(int r = j; r < k; ++r) p[r] -= K * v[r];
    for(int c = j; c < k; ++c)
      for(int r = j; r < k; ++r)
        a[r + size_t(c) * k] -= 2 * (v[r] * p[c] + p[r] * v[c]);
    refl.push_back(v);
  }
  for(int i = 0; i < k; ++i) d[i] = a[i + size_t(i) * k];
  for(int i = 0; i + 1 < k; ++i) e[i] = a[i + 1 + size_t(i) * k];
  // Gershgorin bounds
  double lo = d[0], hi = d[0];
  for(int i = 0; i < k; ++i) {
    const double r = (i ? std::fabs(e[i - 1]) : 0) + (i + 1 < k ? std::fabs(e[i]) : 0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
  }
  const double span = std::max({hi - lo, std::fabs(lo), std::fabs(hi), 1e-30});
  lo -= 1e-12 * span;
  hi += 1e-12 * span;
  const double tiny = 1e-15 * span;  // pivot floor of the shifted solves
  auto count_below = [&](double x) {  // Sturm count of eigenvalues < x
    int c = 0;
    double q = d[0] - x;
    if(q < 0) ++c;
    for(int i = 1; i < k; ++i) {
      if(q == 0) q = 1e-300;
      q = d[i] - x - e[i - 1] * e[i - 1] / q;
      if(q < 0) ++c;
    }
    return c;
  };
  nwant = std::min(nwant, k);
  std::vector<std::vector<double>> ztri;  // eigenvectors of the tridiagonal
  for(int m = 0; m < nwant; ++m) {
    double l = lo, h = hi;  // the m-th eigenvalue has count_below(x) > m
    for(int it = 0; it < 200 && h - l > 4e-16 * std::max(std::fabs(l), std::fabs(h)) + 1e-300; ++it) {
      const double mid = 0.5 * (l + h);
      if(count_below(mid) > m)
        h = mid;
      else
        l = mid;
    }
    W[m] = 0.5 * (l + h);
    // inverse iteration on T - lambda I (tridiagonal LU with pivoting-free
    // elimination, shifted slightly to stay regular)
    const double lam = W[m] + 1e-14 * span;
    auto floor_piv = [&](double x) {
      return std::fabs(x) < tiny ? (x < 0 ? -tiny : tiny) : x;
    };
    // start vector: deterministic, different per wanted pair
    std::vector<double> z(k), w2(k);
    for(int i = 0; i < k; ++i)
      z[i] = 1.0 + 0.5 * std::sin(0.7 * (i + 1) * (m + 1) + 0.3 * m);
    for(int it = 0; it < 5; ++it) {
      std::vector<double> dd(k), rhs = z;
      dd[0] = floor_piv(d[0] - lam);
      for(int i = 1; i < k; ++i) {
        const double f = e[i - 1] / dd[i - 1];
        dd[i] = floor_piv(d[i] - lam - f * e[i - 1]);
        rhs[i] -= f * rhs[i - 1];
      }
      w2[k - 1] = rhs[k - 1] / dd[k - 1];
      for(int i = k - 2; i >= 0; --i) w2[i] = (rhs[i] - e[i] * w2[i + 1]) / dd[i];
      // keep it orthogonal to the vectors of (nearly) equal eigenvalues
      for(int p = 0; p < m; ++p) {
        if(std::fabs(W[p] - W[m]) > 1e-7 * span) continue;
        double s2 = 0;
        for(int i = 0; i < k; ++i) s2 += ztri[p][i] * w2[i];
        for(int i = 0; i < k; ++i) w2[i] -= s2 * ztri[p][i];
      }
      double nn = 0;
      for(double x : w2) nn += x * x;
      nn = std::sqrt(nn);
      if(!(nn > 0) || !std::isfinite(nn)) break;
      for(int i = 0; i < k; ++i) z[i] = w2[i] / nn;
    }
    ztri.push_back(z);
    // back-transform: y = H_0 H_1 ... H_{k-3} z
    for(int r = int(refl.size()) - 1; r >= 0; --r) {
      const auto& v = refl[r];
      double s2 = 0;
      for(int i = 0; i < k; ++i) s2 += v[i] * z[i];
      for(int i = 0; i < k; ++i) z[i] -= 2 * s2 * v[i];
    }
    double nn = 0;
    for(double x : z) nn += x * x;
    nn = std::sqrt(nn);
    for(int i = 0; i < k; ++i) Vec[i + size_t(m) * k] = z[i] / nn;
  }
}

// out[:, j] = Acols[:, 0:k] * Q[:, j] for j < keep (Q column-major, ld k)
__global__ void basis_rotate_k(const double* __restrict__ A, int64_t n, int k,
                               const double* __restrict__ Q, int keep,
                               double* __restrict__ out) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * blockDim.x) {
    for(int j = 0; j < keep; ++j) {
      double s = 0;
      for(int c = 0; c < k; ++c) s += A[i + c * n] * __ldg(Q + c + j * k);
      out[i + j * n] = s;
    }
  }
}

// Phase timings of the last solve on this host thread
// (macis_b200_davidson_last_stats).
static thread_local macis_b200_davidson_stats g_dav_stats{};
const macis_b200_davidson_stats& davidson_last_stats() { return g_dav_stats; }

namespace {
// Device time of one phase, accumulated over the solve: events recorded on
// the solver stream around the phase, read at the next synchronisation.
struct PhaseTimer {
  cudaEvent_t e[2];
  cudaStream_t s;
  double* acc = nullptr;
  bool open = false;
  explicit PhaseTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&e[0]);
    cudaEventCreate(&e[1]);
  }
  ~PhaseTimer() {
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
  }
  void begin(double* into) {
    collect();
    acc = into;
    cudaEventRecord(e[0], s);
  }
  void end() {
    cudaEventRecord(e[1], s);
    open = true;
  }
  // after a stream synchronisation (or at the end of the solve)
  void collect() {
    if(!open) return;
    float ms = 0.f;
    cudaEventSynchronize(e[1]);
    if(cudaEventElapsedTime(&ms, e[0], e[1]) == cudaSuccess) *acc += ms;
    open = false;
  }
};

struct DavCtx {
  cudaStream_t s;
  int64_t n;
  unsigned nb;
  double* partial;  // nb * DV_CHUNK
  double* dots;     // up to 128
  DavCtx(cudaStream_t st, int64_t nn, Arena& A) : s(st), n(nn) {
    nb = grid_for(size_t(nn), DV_THREADS, size_t(num_sms()) * 4);
    partial = A.get<double>(size_t(nb) * DV_CHUNK + 8);
    dots = A.get<double>(2048);
  }
  // dots[0:ncol) = Acols^T v (columns of length n, leading dim lda)
  void multidot(const double* Acols, int64_t lda, int ncol, const double* v,
                double* out) {
    for(int c0 = 0; c0 < ncol; c0 += DV_CHUNK) {
      const int nc = ncol - c0 < DV_CHUNK ? ncol - c0 : DV_CHUNK;
      multidot_k<<<nb, DV_THREADS, 0, s>>>(Acols + c0 * lda, lda, nc, v, n,
                                           partial), note_launch();
      reduce_partials_k<<<nc, 32, 0, s>>>(partial, nb, nc, out + c0), note_launch();
    }
  }
  // gram_schmidt (davidson.hpp:111-126): CGS2 against K columns, normalise
  void cgs2(const double* Vb, int K, double* w) {
    const unsigned g = grid_for(size_t(n), 256, size_t(num_sms()) * 8);
    for(int pass = 0; pass < 2; ++pass) {
      multidot(Vb, n, K, w, dots);
      cgs_update_k<<<g, 256, 0, s>>>(Vb, n, K, dots, w, n), note_launch();
    }
    multidot(w, n, 1, w, dots + 1100);
    scale_k<<<g, 256, 0, s>>>(w, n, dots + 1100), note_launch();
  }
};
}  // namespace

int davidson_device(const macis_b200_csr* A, int64_t max_m, double tol,
                    bool use_guess, double* X, double* E, int64_t* niter,
                    int restart_keep, int64_t max_iter) {
  MB_REQUIRE(A->m == A->n, MACIS_B200_EINVAL, "Davidson needs a square matrix");
  DavOperator op;
  op.n = A->m;
  op.diag = A->diag;
  op.s = A->stream;
  op.apply = [A](const double* x, double* y) {
    spmv_device_x64(A, 1.0, x, 0.0, y, A->stream);
  };
  return davidson_op(op, max_m, tol, use_guess, X, E, niter, restart_keep,
                     max_iter);
}

int davidson_op(const DavOperator& op, int64_t max_m, double tol,
                bool use_guess, double* X, double* E, int64_t* niter,
                int restart_keep, int64_t max_iter) {
  const int64_t N = op.n;
  MB_REQUIRE(N > 0, MACIS_B200_EINVAL, "Davidson: empty matrix");
  MB_REQUIRE(max_m >= 1 && max_m <= 1000, MACIS_B200_EINVAL,
             "Davidson: max_m must be in [1, 1000]");
  MB_REQUIRE(restart_keep >= 0 && restart_keep < max_m, MACIS_B200_EINVAL,
             "Davidson: restart_keep must be in [0, max_m)");
  NvtxRange nv("macis_b200: Davidson");
  cudaStream_t s = op.s;
  Arena Ar(s);
  const auto t_wall = std::chrono::steady_clock::now();
  macis_b200_davidson_stats st{};
  PhaseTimer t_op(s), t_ray(s), t_res(s), t_cgs(s);
  max_m = std::min<int64_t>(max_m, N);
  if(restart_keep >= max_m) restart_keep = int(max_m) - 1;
  const double* D = op.diag;
  if(!use_guess) {
    // diagonal_guess: unit vector at the first minimum of the diagonal
    std::vector<double> hD(N);
    MB_CUDA(cudaMemcpyAsync(hD.data(), D, N * 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    int64_t imin = 0;
    for(int64_t i = 1; i < N; ++i)
      if(hD[i] < hD[imin]) imin = i;
    MB_CUDA(cudaMemsetAsync(X, 0, N * 8, s));
    const double one = 1.0;
    MB_CUDA(cudaMemcpyAsync(X + imin, &one, 8, cudaMemcpyHostToDevice, s));
  }
  double* V = Ar.get<double>(size_t(N) * (max_m + 1));
  double* AV = Ar.get<double>(size_t(N) * (max_m + 1));
  double* tmp = restart_keep ? Ar.get<double>(size_t(N) * restart_keep) : nullptr;
  DavCtx ctx(s, N, Ar);
  MB_CUDA(cudaMemcpyAsync(V, X, N * 8, cudaMemcpyDeviceToDevice, s));
  op.apply(V, AV);
  MB_CUDA(cudaMemcpyAsync(V + N, AV, N * 8, cudaMemcpyDeviceToDevice, s));
  ctx.cgs2(V, 1, V + N);

  const int ld = int(max_m + 1);
  std::vector<double> Cl(size_t(ld) * ld, 0.0), rowdots(ld + 1), lower,
      W(ld), Vec;
  // first entry of the Rayleigh matrix, V_0 . AV_0
  ctx.multidot(AV, N, 1, V, ctx.dots);
  MB_CUDA(cudaMemcpyAsync(rowdots.data(), ctx.dots, 8, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  Cl[0] = rowdots[0];
  double* d_c = Ar.get<double>(size_t(ld) * ld + 2);
  bool converged = false;
  int64_t iter = 1;
  double lam0 = 0;
  int64_t i = 1;  // index of the newest basis vector (AV_i not yet formed)
  for(;; ++iter) {
    const int k = int(i + 1);
    t_op.begin(&st.apply_ms);
    op.apply(V + i * N, AV + i * N);
    t_op.end();
    // new row of V^T AV: V_i . AV_c for c <= i (lower triangle)
    t_ray.begin(&st.rayleigh_ms);
    ctx.multidot(AV, N, k, V + i * N, ctx.dots);
    t_ray.end();
    st.vector_bytes += double(N) * (k + 1) * 8;
    MB_CUDA(cudaMemcpyAsync(rowdots.data(), ctx.dots, k * 8,
                            cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    for(int c = 0; c < k; ++c) Cl[i + size_t(c) * ld] = rowdots[c];
    lower.assign(size_t(k) * k, 0.0);
    for(int c = 0; c < k; ++c)
      for(int r = c; r < k; ++r) lower[r + size_t(c) * k] = Cl[r + size_t(c) * ld];
    const int nwant = std::max(1, std::min(restart_keep, k));
    Vec.assign(size_t(k) * nwant, 0.0);
    small_syev_lowest(k, lower.data(), nwant, W.data(), Vec.data());
    lam0 = W[0];
    MB_CUDA(cudaMemcpyAsync(d_c, Vec.data(), size_t(k) * nwant * 8,
                            cudaMemcpyHostToDevice, s));
    double* R = V + size_t(k) * N;
    t_res.begin(&st.residual_ms);
    ritz_residual_k<<<ctx.nb, DV_THREADS, 0, s>>>(V, AV, N, k, d_c, lam0, D,
                                                  X, R, ctx.partial), note_launch();
    reduce_partials_k<<<1, 32, 0, s>>>(ctx.partial, ctx.nb, 1, ctx.dots + 1200), note_launch();
    t_res.end();
    st.vector_bytes += double(N) * (2.0 * k + 3) * 8;
    double rn2 = 0;
    MB_CUDA(cudaMemcpyAsync(&rn2, ctx.dots + 1200, 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if(std::sqrt(rn2) < tol) {
      converged = true;
      break;
    }
    if(k >= max_m) {
      // the reference stops here (davidson.hpp:161, 221)
      if(!restart_keep || (max_iter > 0 && iter >= max_iter)) break;
      // thick restart: keep the lowest restart_keep Ritz vectors
      const int keep = restart_keep;
      const unsigned g = grid_for(size_t(N), 256, size_t(num_sms()) * 8);
      t_cgs.begin(&st.ortho_ms);
      // two rotations (read k columns, write keep), the copies back and
      // of R, then CGS2 over keep columns
      st.vector_bytes += double(N) * (2.0 * k + 6.0 * keep + 2) * 8 +
                         double(N) * (4.0 * keep + 9) * 8;
      basis_rotate_k<<<g, 256, 0, s>>>(V, N, k, d_c, keep, tmp), note_launch();
      MB_CUDA(cudaMemcpyAsync(V, tmp, size_t(N) * keep * 8,
                              cudaMemcpyDeviceToDevice, s));
      basis_rotate_k<<<g, 256, 0, s>>>(AV, N, k, d_c, keep, tmp), note_launch();
      MB_CUDA(cudaMemcpyAsync(AV, tmp, size_t(N) * keep * 8,
                              cudaMemcpyDeviceToDevice, s));
      MB_CUDA(cudaMemcpyAsync(V + size_t(keep) * N, R, N * 8,
                              cudaMemcpyDeviceToDevice, s));
      std::fill(Cl.begin(), Cl.end(), 0.0);
      for(int c = 0; c < keep; ++c) Cl[c + size_t(c) * ld] = W[c];
      ctx.cgs2(V, keep, V + size_t(keep) * N);
      t_cgs.end();
      i = keep;
      continue;
    }
    if(max_iter > 0 && iter >= max_iter) break;
    t_cgs.begin(&st.ortho_ms);
    ctx.cgs2(V, k, R);
    t_cgs.end();
    st.vector_bytes += double(N) * (4.0 * k + 9) * 8;
    i = k;
  }
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(s));
  for(PhaseTimer* t : {&t_op, &t_ray, &t_res, &t_cgs}) t->collect();
  st.iterations = iter;
  st.wall_ms = std::chrono::duration<double, std::milli>(
                   std::chrono::steady_clock::now() - t_wall)
                   .count();
  g_dav_stats = st;
  *E = lam0;
  *niter = iter;
  return converged ? 0 : MACIS_B200_ENOCONV;
}

}  // namespace mb

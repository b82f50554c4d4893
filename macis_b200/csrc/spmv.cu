// CSR sparse matrix - vector products on the GPU, replacing
// sparsexx::spblas::gespmbv (src/sparsexx/include/sparsexx/spblas/spmbv.hpp:
// 39-73) behind SparseMatrixOperator::operator_action
// (include/macis/solvers/davidson.hpp:47-58).
//
// HBM-bound: each product streams colind + nzval once (12 B/nnz for FP64
// values with int32 indices, 8 B/nnz for the FP32 mixed mode) while x stays
// in L2. One warp per row; the index/value streams are loaded with an
// evict-first hint so that x keeps the cache. Row sums are warp trees in
// FP64. Mixed mode: FP32 off-diagonal values times an FP32 copy of x, each
// product formed exactly in FP64 (24x24-bit mantissas fit in 53 bits) and
// summed in FP64, plus the FP64 diagonal times the FP64 x.
#include "internal.hpp"
#include "primitives.cuh"

namespace mb {

constexpr int SPMV_THREADS = 256;

template <typename CI, typename VT, bool MIXED>
__global__ void __launch_bounds__(SPMV_THREADS)
    spmv_k(int64_t m, int64_t n, const CI* __restrict__ rowptr,
           const CI* __restrict__ colind, const VT* __restrict__ nzval,
           const double* __restrict__ diag, const double* __restrict__ x,
           const float* __restrict__ x32, double alpha, double beta,
           double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = int64_t(gridDim.x) * (SPMV_THREADS / 32);
  for(int64_t row = int64_t(blockIdx.x) * (SPMV_THREADS / 32) + (threadIdx.x >> 5);
      row < m; row += nwarp) {
    const int64_t b = int64_t(rowptr[row]), e = int64_t(rowptr[row + 1]);
    double acc0 = 0, acc1 = 0;
    int64_t j = b + lane;
    for(; j + 32 < e; j += 64) {
      const CI c0 = __ldcs(colind + j), c1 = __ldcs(colind + j + 32);
      const VT v0 = __ldcs(nzval + j), v1 = __ldcs(nzval + j + 32);
      if constexpr(MIXED) {
        acc0 += double(v0) * double(__ldg(x32 + c0));
        acc1 += double(v1) * double(__ldg(x32 + c1));
      } else {
        acc0 += double(v0) * __ldg(x + c0);
        acc1 += double(v1) * __ldg(x + c1);
      }
    }
    if(j < e) {
      const CI c0 = __ldcs(colind + j);
      const VT v0 = __ldcs(nzval + j);
      if constexpr(MIXED)
        acc0 += double(v0) * double(__ldg(x32 + c0));
      else
        acc0 += double(v0) * __ldg(x + c0);
    }
    double acc = acc0 + acc1;
#pragma unroll
    for(int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if(lane == 0) {
      if constexpr(MIXED)
        if(row < n) acc += diag[row] * x[row];
      y[row] = beta == 0.0 ? alpha * acc : alpha * acc + beta * y[row];
    }
  }
}

__global__ void to_f32_k(const double* x, float* y, int64_t n) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * blockDim.x)
    y[i] = float(x[i]);
}

static unsigned spmv_grid(int64_t m) {
  // enough resident warps to cover HBM latency: 16 blocks of 8 warps per SM
  return grid_for(size_t(m), SPMV_THREADS / 32, size_t(num_sms()) * 16);
}

void spmv_device(const macis_b200_csr* A, double alpha, const double* x,
                 double beta, double* y, cudaStream_t s) {
  const int64_t m = A->m;
  if(m == 0) return;
  const unsigned g = spmv_grid(m);
  if(A->val_bytes == 8) {
    if(A->idx_bytes == 4)
      spmv_k<int32_t, double, false><<<g, SPMV_THREADS, 0, s>>>(
          m, A->n, (const int32_t*)A->rowptr, (const int32_t*)A->colind,
          (const double*)A->nzval, A->diag, x, nullptr, alpha, beta, y), note_launch();
    else
      spmv_k<int64_t, double, false><<<g, SPMV_THREADS, 0, s>>>(
          m, A->n, (const int64_t*)A->rowptr, (const int64_t*)A->colind,
          (const double*)A->nzval, A->diag, x, nullptr, alpha, beta, y), note_launch();
  } else {
    Arena W(s);
    float* x32 = W.get<float>(size_t(A->n));
    to_f32_k<<<grid_for(size_t(A->n), 256, 8 * num_sms()), 256, 0, s>>>(
        x, x32, A->n), note_launch();
    if(A->idx_bytes == 4)
      spmv_k<int32_t, float, true><<<g, SPMV_THREADS, 0, s>>>(
          m, A->n, (const int32_t*)A->rowptr, (const int32_t*)A->colind,
          (const float*)A->nzval, A->diag, x, x32, alpha, beta, y), note_launch();
    else
      spmv_k<int64_t, float, true><<<g, SPMV_THREADS, 0, s>>>(
          m, A->n, (const int64_t*)A->rowptr, (const int64_t*)A->colind,
          (const float*)A->nzval, A->diag, x, x32, alpha, beta, y), note_launch();
  }
  MB_CUDA(cudaGetLastError());
}

}  // namespace mb

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
// summed in FP64, plus the FP64 diagonal times the FP64 x. The Davidson
// solver uses the same kernel with the FP64 x (spmv_device_x64).
#include <exception>
#include <mutex>
#include <new>

#include "internal.hpp"
#include "primitives.cuh"

namespace mb {

constexpr int SPMV_THREADS = 256;

// X32: the off-diagonal products use the FP32 copy x32 (the operator of
// macis_b200_spmv on a mixed matrix); otherwise FP32 values multiply the
// FP64 x, so that the product is one fixed linear operator of x (what the
// Davidson residual needs to converge below FP32 resolution).
template <typename CI, typename VT, bool MIXED, bool X32 = MIXED>
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
      if constexpr(X32) {
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
      if constexpr(X32)
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

void spmv_device_x64(const macis_b200_csr* A, double alpha, const double* x,
                     double beta, double* y, cudaStream_t s) {
  if(A->val_bytes == 8) return spmv_device(A, alpha, x, beta, y, s);
  const int64_t m = A->m;
  if(m == 0) return;
  const unsigned g = spmv_grid(m);
  if(A->idx_bytes == 4)
    spmv_k<int32_t, float, true, false><<<g, SPMV_THREADS, 0, s>>>(
        m, A->n, (const int32_t*)A->rowptr, (const int32_t*)A->colind,
        (const float*)A->nzval, A->diag, x, nullptr, alpha, beta, y), note_launch();
  else
    spmv_k<int64_t, float, true, false><<<g, SPMV_THREADS, 0, s>>>(
        m, A->n, (const int64_t*)A->rowptr, (const int64_t*)A->colind,
        (const float*)A->nzval, A->diag, x, nullptr, alpha, beta, y), note_launch();
  MB_CUDA(cudaGetLastError());
}

}  // namespace mb

// ---------------------------------------------------------------------------
// Allocation-free mixed-precision SpMV.
//
// Some callers may not allocate device memory once they are running: a
// service that hands all of HBM to its own pool manager at start-up and
// forbids cudaMalloc afterwards, or a host program whose memory budget is
// fixed when it links this library. For them the FP32 copy of x that the
// mixed-precision product needs lives in the file-scope array below instead
// of a stream-ordered allocation. The array (16 MiB) belongs to this file's
// device module: with CUDA's lazy module loading the module, and with it the
// array and the kernel code, is made resident on a device by the first use
// of this file's code there (any SpMV, or the first allocation-free call),
// and stays until the process exits. That first use may allocate device
// memory; later allocation-free calls allocate nothing.
namespace mb {
namespace {

constexpr int64_t kNoAllocMaxN = int64_t(1) << 22;  // 4,194,304 columns
static __device__ __align__(256) float g_noalloc_x32[kNoAllocMaxN];

// Host code cannot use g_noalloc_x32 as a device address: its name there is
// a host-side stand-in. The device address is looked up once per device with
// that device current.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

float* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  MB_REQUIRE(dev >= 0 && dev < kMaxDevices, MACIS_B200_EINVAL,
             "device ordinal out of range");
  if(!g_noalloc_ptr[dev]) {
    // the caller holds `dev` current (DeviceScope)
    void* p = nullptr;
    MB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_x32));
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  return g_noalloc_ptr[dev];
}

}  // namespace
}  // namespace mb

namespace mb {
namespace {

// Makes `dev` current for the life of the guard and restores the caller's
// device afterwards (the handle's stream and the scratch address belong to
// the matrix's device, whatever device the caller has current).
struct DeviceScope {
  int prev = -1;
  bool switched = false;
  explicit DeviceScope(int dev) {
    MB_CUDA(cudaGetDevice(&prev));
    if(prev != dev) {
      MB_CUDA(cudaSetDevice(dev));
      switched = true;
    }
  }
  ~DeviceScope() {
    if(switched) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace mb

extern "C" int macis_b200_spmv_mixed_noalloc(const macis_b200_csr* A,
                                             double alpha, const double* x,
                                             double beta, double* y) {
  try {
    MB_REQUIRE(A && x && y, MACIS_B200_EINVAL, "null argument");
    MB_REQUIRE(A->val_bytes == 4, MACIS_B200_EINVAL,
               "the allocation-free SpMV needs an FP32-value (mixed) matrix");
    MB_REQUIRE(A->n <= mb::kNoAllocMaxN, MACIS_B200_ECAPACITY,
               "matrix has more columns than the allocation-free scratch "
               "holds (4,194,304)");
    mb::DeviceScope on(A->device);
    float* x32 = mb::noalloc_scratch(A->device);
    const int64_t m = A->m;
    cudaStream_t s = A->stream;
    if(m > 0) {
      // the scratch is fully rewritten before it is read: nothing to clear
      mb::to_f32_k<<<mb::grid_for(size_t(A->n), 256, 8 * mb::num_sms()), 256,
                     0, s>>>(x, x32, A->n), mb::note_launch();
      const unsigned g = mb::spmv_grid(m);
      if(A->idx_bytes == 4)
        mb::spmv_k<int32_t, float, true><<<g, mb::SPMV_THREADS, 0, s>>>(
            m, A->n, (const int32_t*)A->rowptr, (const int32_t*)A->colind,
            (const float*)A->nzval, A->diag, x, x32, alpha, beta, y),
            mb::note_launch();
      else
        mb::spmv_k<int64_t, float, true><<<g, mb::SPMV_THREADS, 0, s>>>(
            m, A->n, (const int64_t*)A->rowptr, (const int64_t*)A->colind,
            (const float*)A->nzval, A->diag, x, x32, alpha, beta, y),
            mb::note_launch();
      MB_CUDA(cudaGetLastError());
    }
    MB_CUDA(cudaStreamSynchronize(s));
    return MACIS_B200_OK;
  } catch(const mb::Error& e) {
    mb::set_error(e.what());
    return e.code;
  } catch(const std::bad_alloc&) {
    mb::set_error("host allocation failed");
    return MACIS_B200_ENOMEM;
  } catch(const std::exception& e) {  // e.g. std::system_error of the mutex
    mb::set_error(e.what());
    return MACIS_B200_EINVAL;
  }
}

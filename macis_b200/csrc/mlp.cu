// Screening network object: FP32 master parameters, Adam state, BF16 operand
// copies, and the training step
//
//   gather minibatch -> forward (mlp_fwd_k, taps) -> loss / dZ2 -> bias and
//   head gradients (row sums) -> dW2 = dZ2^T H1 (tcgen05) -> dZ1 = (dZ2 W2)
//   * GELU'(Z1) (tcgen05, fused epilogue) -> dW1 = dZ1^T X (tcgen05) -> Adam
//   -> repack BF16 operands.
//
// The network has no counterpart in MACIS; the ASCI search uses it to rank
// its work units before exact scoring.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "internal.hpp"
#include "mlp.cuh"
#include "primitives.cuh"

namespace mb {

namespace {

constexpr int GT_M = 128;  // backward GEMM tile
constexpr int GT_N = 64;
constexpr int GT_K = 64;

// C = A B^T for row-major BF16 A [M][K] (lda) and B [N][K] (ldb); M % 128,
// N % 64, K % 64 == 0. MODE 0 stores C (FP32 row-major, ldc). MODE 1 is the
// dZ1 epilogue: v = C[m][n] * GELU'(z1t[n][m]); writes v to of32t[n][m] and
// BF16(v) to obf16t[n][m] (both leading dimension ldo), 0 for m >= mvalid.
struct GemmOut {
  float* c = nullptr;
  int64_t ldc = 0;
  const float* z1t = nullptr;
  float* of32t = nullptr;
  __nv_bfloat16* obf16t = nullptr;
  int64_t ldo = 0;
  int64_t mvalid = 0;
};

template <int MODE>
__global__ void __launch_bounds__(128)
    gemm_tc_k(const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
              int64_t ldb, int64_t K, GemmOut o, int* err, uint64_t limit_ns) {
  constexpr int ABYTES = GT_M * GT_K * 2;  // 16 KB
  constexpr int BBYTES = GT_N * GT_K * 2;  // 8 KB
  constexpr uint32_t A_LBO = GT_M * 16, B_LBO = GT_N * 16;
  constexpr uint32_t IDESC = tc::idesc_bf16(GT_M, GT_N);
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint64_t bar[2];
  __shared__ uint64_t drain;  // used once, by the timeout path only
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = int64_t(blockIdx.y) * GT_M, n0 = int64_t(blockIdx.x) * GT_N;
  if(tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::mbar_init(&drain, 1);
    tc::mbar_init_fence();
  }
  if(warp == 0) tc::tmem_alloc(&tslot, GT_N);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  const int64_t nk = K / GT_K;
  bool fail = false, abort = false;
  for(int64_t c = 0; c < nk; ++c) {
    const int s = int(c & 1);
    uint8_t* as = smem + s * (ABYTES + BBYTES);
    uint8_t* bs = as + ABYTES;
    // the MMAs of chunk c-2 read this stage
    if(c >= 2 &&
       !tc::mbar_wait(&bar[s], uint32_t(((c - 2) >> 1) & 1), limit_ns))
      fail = true;
    if(__syncthreads_or(fail)) {
      abort = true;
      break;
    }
    const int64_t k0 = c * GT_K;
    {
      const uint4* src =
          reinterpret_cast<const uint4*>(A + (m0 + tid) * lda + k0);
#pragma unroll
      for(int i = 0; i < GT_K / 8; ++i)
        *reinterpret_cast<uint4*>(as + i * A_LBO + tid * 16) = __ldg(src + i);
      const int br = tid & (GT_N - 1), half = tid / GT_N;
      const uint4* bsrc =
          reinterpret_cast<const uint4*>(B + (n0 + br) * ldb + k0);
#pragma unroll
      for(int i = 0; i < GT_K / 16; ++i) {
        const int slab = half * (GT_K / 16) + i;
        *reinterpret_cast<uint4*>(bs + slab * B_LBO + br * 16) =
            __ldg(bsrc + slab);
      }
    }
    tc::fence_async_smem();
    __syncthreads();
    if(tid == 0) {
      tc::fence_after_sync();
      const uint32_t aa = tc::smem_addr(as), ba = tc::smem_addr(bs);
#pragma unroll
      for(int ks = 0; ks < GT_K / 16; ++ks)
        tc::mma_bf16(tmem, tc::sdesc(aa + 2 * ks * A_LBO, A_LBO, 128),
                     tc::sdesc(ba + 2 * ks * B_LBO, B_LBO, 128), IDESC,
                     (c | ks) ? 1u : 0u);
      tc::mma_commit(&bar[s]);
    }
  }
  // the last commit covers every MMA of this tile
  if(!abort && nk > 0) {
    const int64_t c = nk - 1;
    if(!tc::mbar_wait(&bar[c & 1], uint32_t((c >> 1) & 1), limit_ns))
      fail = true;
  }
  if(__syncthreads_or(fail)) abort = true;
  if(!abort) {
    tc::fence_after_sync();
    const int r = warp * 32 + lane;
    const int64_t m = m0 + r;
    const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
    for(int c0 = 0; c0 < GT_N; c0 += 16) {
      uint32_t v[16];
      tc::tmem_ld16(trow + uint32_t(c0), v);
      tc::tmem_wait_ld();
      if(MODE == 0) {
        float4* d = reinterpret_cast<float4*>(o.c + m * o.ldc + n0 + c0);
#pragma unroll
        for(int q = 0; q < 4; ++q)
          d[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                             __uint_as_float(v[4 * q + 2]),
                             __uint_as_float(v[4 * q + 3]));
      } else {
        // all 16 pre-activations first: independent loads, one latency
        float z[16];
#pragma unroll
        for(int q = 0; q < 16; ++q)
          z[q] = m < o.mvalid ? __ldg(o.z1t + (n0 + c0 + q) * o.ldo + m) : 0.f;
#pragma unroll
        for(int q = 0; q < 16; ++q) {
          const int64_t n = n0 + c0 + q;
          const float g =
              m < o.mvalid ? __uint_as_float(v[q]) * gelu_grad_f(z[q]) : 0.f;
          o.of32t[n * o.ldo + m] = g;
          o.obf16t[n * o.ldo + m] = __float2bfloat16_rn(g);
        }
      }
    }
  } else if(tid == 0) {
    atomicExch(err, 1);
    // wait (bounded) for every MMA this thread issued before TMEM is freed
    // and the operand tiles are released: a commit on the unused drain
    // barrier completes its phase 0 after all of them
    tc::mma_commit(&drain);
    tc::mbar_wait(&drain, 0u, 100000000ull);
  }
  tc::fence_before_sync();
  __syncthreads();
  if(warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, GT_N);
  }
}

// Loss L = sum_m (y_m - t_m)^2 / (2 nvalid) and its first backward step.
// Thread (j, m), m fastest.
__global__ void mlp_loss_k(const float* y, const float* t, int64_t nvalid,
                           int64_t B, const float* z2t, const float* w3,
                           float* dy, float* dz2t, __nv_bfloat16* dz2t_b,
                           __nv_bfloat16* dz2_b, float* p3t, double* loss) {
  const int64_t total = int64_t(MLP_H) * B;
  for(int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
      idx += int64_t(gridDim.x) * blockDim.x) {
    const int j = int(idx / B);
    const int64_t m = idx % B;
    float g = 0.f, p = 0.f, d = 0.f;
    if(m < nvalid) {
      const float e = y[m] - t[m];
      d = e / float(nvalid);
      const float z = z2t[idx];
      g = d * w3[j] * gelu_grad_f(z);
      p = d * gelu_f(z);
      if(j == 0 && loss) atomicAdd(loss, double(e) * double(e));
    }
    if(j == 0) dy[m] = d;
    dz2t[idx] = g;
    const __nv_bfloat16 gb = __float2bfloat16_rn(g);
    dz2t_b[idx] = gb;
    dz2_b[m * MLP_H + j] = gb;
    p3t[idx] = p;
  }
}

// out[r] = sum_{m < n} in[r * ld + m] in a fixed order (deterministic).
// Rows [0, r1) come from (in, out), rows [r1, r2) from (in2, out2), and so
// on, so that several small reductions share one launch.
struct RowSums {
  const float* in[3];
  float* out[3];
  int rows[3];
};
__global__ void rowsums_k(RowSums R, int64_t ld, int64_t n) {
  __shared__ float sh[256];
  int r = blockIdx.x, g = 0;
  while(g < 2 && r >= R.rows[g]) r -= R.rows[g++];
  const float* row = R.in[g] + int64_t(r) * ld;
  float a = 0.f;
  for(int64_t m = threadIdx.x; m < n; m += blockDim.x) a += row[m];
  sh[threadIdx.x] = a;
  __syncthreads();
  for(int w = blockDim.x / 2; w > 0; w >>= 1) {
    if(int(threadIdx.x) < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if(threadIdx.x == 0) R.out[g][r] = sh[0];
}

__global__ void rowsum_k(const float* in, int64_t ld, int64_t n, float* out) {
  __shared__ float sh[256];
  const float* row = in + int64_t(blockIdx.x) * ld;
  float a = 0.f;
  for(int64_t m = threadIdx.x; m < n; m += blockDim.x) a += row[m];
  sh[threadIdx.x] = a;
  __syncthreads();
  for(int w = blockDim.x / 2; w > 0; w >>= 1) {
    if(int(threadIdx.x) < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if(threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// Minibatch rows idx[0..nvalid) of X [S][din]: xb [B][din], xbt [din][B].
__global__ void mlp_gather_k(const uint16_t* X, const float* t,
                             const int64_t* idx, int64_t nvalid, int64_t B,
                             int din, uint16_t* xb, uint16_t* xbt, float* tb) {
  const int64_t total = int64_t(din) * B;
  for(int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total;
      q += int64_t(gridDim.x) * blockDim.x) {
    const int k = int(q / B);
    const int64_t m = q % B;
    uint16_t v = 0;
    if(m < nvalid) v = X[idx[m] * din + k];
    xbt[q] = v;
    xb[m * din + k] = v;
    if(k == 0) tb[m] = m < nvalid ? t[idx[m]] : 0.f;
  }
}

__global__ void adam_k(float* P, const float* G, float* Mo, float* Ve,
                       int64_t n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += int64_t(gridDim.x) * blockDim.x) {
    const float g = G[i];
    const float m = b1 * Mo[i] + (1.f - b1) * g;
    const float v = b2 * Ve[i] + (1.f - b2) * g * g;
    Mo[i] = m;
    Ve[i] = v;
    P[i] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
  }
}

// BF16 operand copies of W1 [256][din] and W2 [256][256]: the forward's
// slab layout and the row-major transpose W2^T used by the backward.
__global__ void mlp_pack_k(const float* W1, const float* W2, int din,
                           uint16_t* w1t, uint16_t* w2t, uint16_t* w2T) {
  const int64_t n1 = int64_t(MLP_H) * din, n2 = int64_t(MLP_H) * MLP_H;
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n1 + n2;
      i += int64_t(gridDim.x) * blockDim.x) {
    if(i < n1) {
      const int n = int(i / din), k = int(i % din);
      w1t[(int64_t(k / 8) * MLP_H + n) * 8 + (k & 7)] =
          __bfloat16_as_ushort(__float2bfloat16_rn(W1[i]));
    } else {
      const int64_t j = i - n1;
      const int n = int(j / MLP_H), k = int(j % MLP_H);
      const uint16_t b = __bfloat16_as_ushort(__float2bfloat16_rn(W2[j]));
      w2t[(int64_t(k / 8) * MLP_H + n) * 8 + (k & 7)] = b;
      w2T[int64_t(k) * MLP_H + n] = b;
    }
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return double(splitmix(s) >> 11) * 0x1.0p-53; }

template <typename T>
T* dalloc(size_t n) {
  void* p = nullptr;
  MB_CUDA(dev_malloc(&p, std::max<size_t>(n * sizeof(T), 256)));
  return static_cast<T*>(p);
}

void check_err(macis_b200_mlp* m) {
  int e = 0;
  MB_CUDA(cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost,
                          m->stream));
  MB_CUDA(cudaStreamSynchronize(m->stream));
  if(e) {  // cleared, so that the next call starts clean
    MB_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), m->stream));
    MB_CUDA(cudaStreamSynchronize(m->stream));
  }
  MB_REQUIRE(e == 0, MACIS_B200_ETIMEOUT,
             "screening network kernel timed out waiting on a barrier");
}

void repack(macis_b200_mlp* m, cudaStream_t s) {
  mlp_pack_k<<<grid_for(size_t(MLP_H) * (m->din + MLP_H), 256, 4 * num_sms()),
               256, 0, s>>>(m->P + m->off_w1, m->P + m->off_w2, m->din,
                            m->w1t, m->w2t, m->w2T), note_launch();
  MB_CUDA(cudaGetLastError());
}

// Training scratch for a batch of B rows (B % 128 == 0).
void ensure_batch(macis_b200_mlp* m, int64_t B) {
  if(m->B >= B) return;
  for(void* p : m->scratch) cudaFree(p);
  m->scratch.clear();
  auto get = [&](size_t bytes) {
    void* p = nullptr;
    MB_CUDA(dev_malloc(&p, std::max<size_t>(bytes, 256)));
    MB_CUDA(cudaMemset(p, 0, std::max<size_t>(bytes, 256)));
    m->scratch.push_back(p);
    return p;
  };
  const size_t H = MLP_H, din = size_t(m->din);
  m->xb = static_cast<uint16_t*>(get(B * din * 2));
  m->xbt = static_cast<uint16_t*>(get(B * din * 2));
  m->tb = static_cast<float*>(get(B * 4));
  m->yb = static_cast<float*>(get(B * 4));
  m->z1t = static_cast<float*>(get(H * B * 4));
  m->h1t = static_cast<uint16_t*>(get(H * B * 2));
  m->z2t = static_cast<float*>(get(H * B * 4));
  m->dy = static_cast<float*>(get(B * 4));
  m->dz2t = static_cast<float*>(get(H * B * 4));
  m->dz2t_b = static_cast<uint16_t*>(get(H * B * 2));
  m->dz2_b = static_cast<uint16_t*>(get(H * B * 2));
  m->p3t = static_cast<float*>(get(H * B * 4));
  m->dz1t = static_cast<float*>(get(H * B * 4));
  m->dz1t_b = static_cast<uint16_t*>(get(H * B * 2));
  m->idx = static_cast<int64_t*>(get(B * 8));
  m->B = B;
}

MlpWeights weights_of(const macis_b200_mlp* m) {
  return MlpWeights{m->din,
                    reinterpret_cast<const uint4*>(m->w1t),
                    reinterpret_cast<const uint4*>(m->w2t),
                    m->P + m->off_b1,
                    m->P + m->off_b2,
                    m->P + m->off_w3,
                    m->P + m->off_b3};
}

template <class Src, bool TRAIN>
void launch_fwd(const macis_b200_mlp* m, const Src& src, int64_t nrows,
                float* y, MlpTaps taps, cudaStream_t s) {
  if(nrows <= 0) return;
  const size_t smem = mlp_fwd_smem_bytes(m->din);
  auto kern = mlp_fwd_k<Src, TRAIN>;
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(smem)));
  const int64_t tiles = (nrows + MLP_TM - 1) / MLP_TM;
  const unsigned grid = unsigned(std::min<int64_t>(tiles, num_sms()));
  kern<<<grid, MLP_TM, smem, s>>>(weights_of(m), src, nrows, y, taps, m->err,
                                  wait_limit_ns()),
      note_launch();
  MB_CUDA(cudaGetLastError());
}

template <int MODE>
void gemm(const macis_b200_mlp* m, const uint16_t* A, int64_t lda,
          const uint16_t* B, int64_t ldb, int64_t M, int64_t N, int64_t K,
          const GemmOut& o, cudaStream_t s) {
  MB_REQUIRE(M % GT_M == 0 && N % GT_N == 0 && K % GT_K == 0,
             MACIS_B200_EINVAL, "network GEMM shape not tile aligned");
  const int smem = 2 * (GT_M + GT_N) * GT_K * 2;
  auto kern = gemm_tc_k<MODE>;
  MB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem));
  dim3 grid(unsigned(N / GT_N), unsigned(M / GT_M));
  kern<<<grid, 128, smem, s>>>(reinterpret_cast<const __nv_bfloat16*>(A), lda,
                               reinterpret_cast<const __nv_bfloat16*>(B), ldb,
                               K, o, m->err, wait_limit_ns()), note_launch();
  MB_CUDA(cudaGetLastError());
}

// Forward + backward on rows idx[0..nvalid) of (X, t); gradients in m->G.
void fwd_bwd(macis_b200_mlp* m, const uint16_t* X, const float* t,
             const int64_t* idx, int64_t nvalid, int64_t B, double* loss_acc,
             cudaStream_t s) {
  const int din = m->din;
  const int sms = num_sms();
  mlp_gather_k<<<grid_for(size_t(din) * B, 256, 8 * sms), 256, 0, s>>>(
      X, t, idx, nvalid, B, din, m->xb, m->xbt, m->tb), note_launch();
  MlpTaps taps;
  taps.z1t = m->z1t;
  taps.h1t = reinterpret_cast<__nv_bfloat16*>(m->h1t);
  taps.z2t = m->z2t;
  taps.ld = B;
  launch_fwd<DenseRows, true>(
      m, DenseRows{reinterpret_cast<const uint4*>(m->xb), din}, nvalid, m->yb,
      taps, s);
  mlp_loss_k<<<grid_for(size_t(MLP_H) * B, 256, 8 * sms), 256, 0, s>>>(
      m->yb, m->tb, nvalid, B, m->z2t, m->P + m->off_w3, m->dy, m->dz2t,
      reinterpret_cast<__nv_bfloat16*>(m->dz2t_b),
      reinterpret_cast<__nv_bfloat16*>(m->dz2_b), m->p3t, loss_acc), note_launch();
  float* G = m->G;
  RowSums rs{{m->dz2t, m->p3t, m->dy},
             {G + m->off_b2, G + m->off_w3, G + m->off_b3},
             {MLP_H, MLP_H, 1}};
  rowsums_k<<<2 * MLP_H + 1, 256, 0, s>>>(rs, B, B), note_launch();
  // dW2[o][i] = sum_m dZ2[m][o] H1[m][i]
  GemmOut o2;
  o2.c = G + m->off_w2;
  o2.ldc = MLP_H;
  gemm<0>(m, m->dz2t_b, B, m->h1t, B, MLP_H, MLP_H, B, o2, s);
  // dZ1[m][i] = (sum_o dZ2[m][o] W2[o][i]) GELU'(Z1[m][i]), stored transposed
  GemmOut o1;
  o1.z1t = m->z1t;
  o1.of32t = m->dz1t;
  o1.obf16t = reinterpret_cast<__nv_bfloat16*>(m->dz1t_b);
  o1.ldo = B;
  o1.mvalid = nvalid;
  gemm<1>(m, m->dz2_b, MLP_H, m->w2T, MLP_H, B, MLP_H, MLP_H, o1, s);
  rowsum_k<<<MLP_H, 256, 0, s>>>(m->dz1t, B, B, G + m->off_b1), note_launch();
  // dW1[o][k] = sum_m dZ1[m][o] X[m][k]
  GemmOut o3;
  o3.c = G + m->off_w1;
  o3.ldc = din;
  gemm<0>(m, m->dz1t_b, B, m->xbt, B, MLP_H, din, B, o3, s);
}

}  // namespace

// ------------------------------------------------------------------ object
macis_b200_mlp* mlp_create(int din, uint64_t seed) {
  MB_REQUIRE(din > 0 && din % MLP_KC == 0 && din <= 512, MACIS_B200_EINVAL,
             "network input width must be a positive multiple of 64 (<= 512)");
  auto* m = new macis_b200_mlp;
  try {
    m->din = din;
    MB_CUDA(cudaGetDevice(&m->device));
    MB_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->off_w1 = 0;
    m->off_b1 = m->off_w1 + size_t(MLP_H) * din;
    m->off_w2 = m->off_b1 + MLP_H;
    m->off_b2 = m->off_w2 + size_t(MLP_H) * MLP_H;
    m->off_w3 = m->off_b2 + MLP_H;
    m->off_b3 = m->off_w3 + MLP_H;
    m->nparams = m->off_b3 + 1;
    m->P = dalloc<float>(m->nparams);
    m->G = dalloc<float>(m->nparams);
    m->Mo = dalloc<float>(m->nparams);
    m->Ve = dalloc<float>(m->nparams);
    m->w1t = dalloc<uint16_t>(size_t(MLP_H) * din);
    m->w2t = dalloc<uint16_t>(size_t(MLP_H) * MLP_H);
    m->w2T = dalloc<uint16_t>(size_t(MLP_H) * MLP_H);
    m->err = dalloc<int>(1);
    MB_CUDA(cudaMemset(m->err, 0, sizeof(int)));
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
    std::vector<float> h(m->nparams, 0.f);
    uint64_t st = seed;
    const double a1 = 1.0 / std::sqrt(double(din)), a2 = 1.0 / std::sqrt(256.0);
    for(size_t i = 0; i < size_t(MLP_H) * din; ++i)
      h[m->off_w1 + i] = float((2 * uniform01(st) - 1) * a1);
    for(size_t i = 0; i < size_t(MLP_H) * MLP_H; ++i)
      h[m->off_w2 + i] = float((2 * uniform01(st) - 1) * a2);
    for(size_t i = 0; i < size_t(MLP_H); ++i)
      h[m->off_w3 + i] = float((2 * uniform01(st) - 1) * a2);
    mlp_set_params(m, h.data());
  } catch(...) {
    mlp_destroy(m);
    throw;
  }
  return m;
}

void mlp_destroy(macis_b200_mlp* m) {
  if(!m) return;
  if(m->stream) cudaStreamSynchronize(m->stream);
  for(void* p : {static_cast<void*>(m->P), static_cast<void*>(m->G),
                 static_cast<void*>(m->Mo), static_cast<void*>(m->Ve),
                 static_cast<void*>(m->w1t), static_cast<void*>(m->w2t),
                 static_cast<void*>(m->w2T), static_cast<void*>(m->err),
                 static_cast<void*>(m->xs), static_cast<void*>(m->ts)})
    if(p) cudaFree(p);
  for(void* p : m->scratch) cudaFree(p);
  if(m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

void mlp_set_params(macis_b200_mlp* m, const float* host) {
  cudaStream_t s = m->stream;
  MB_CUDA(cudaMemcpyAsync(m->P, host, m->nparams * 4, cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemsetAsync(m->Mo, 0, m->nparams * 4, s));
  MB_CUDA(cudaMemsetAsync(m->Ve, 0, m->nparams * 4, s));
  m->step = 0;
  repack(m, s);
  MB_CUDA(cudaStreamSynchronize(s));
}

void mlp_get_params(const macis_b200_mlp* m, float* host) {
  MB_CUDA(cudaMemcpyAsync(host, m->P, m->nparams * 4, cudaMemcpyDeviceToHost,
                          m->stream));
  MB_CUDA(cudaStreamSynchronize(m->stream));
}

MlpWeights mlp_weights(const macis_b200_mlp* m) { return weights_of(m); }

void mlp_forward_device(macis_b200_mlp* m, const uint16_t* X, int64_t n,
                        float* y, cudaStream_t s) {
  launch_fwd<DenseRows, false>(
      m, DenseRows{reinterpret_cast<const uint4*>(X), m->din}, n, y, MlpTaps{},
      s);
  MB_CUDA(cudaStreamSynchronize(s));
  check_err(m);
}

double mlp_gradients_device(macis_b200_mlp* m, const uint16_t* X,
                            const float* t, int64_t n, float* grad) {
  MB_REQUIRE(n > 0, MACIS_B200_EINVAL, "empty batch");
  cudaStream_t s = m->stream;
  const int64_t B = (n + MLP_TM - 1) / MLP_TM * MLP_TM;
  ensure_batch(m, B);
  std::vector<int64_t> id(n);
  for(int64_t i = 0; i < n; ++i) id[i] = i;
  MB_CUDA(cudaMemcpyAsync(m->idx, id.data(), n * 8, cudaMemcpyHostToDevice, s));
  double* dl = nullptr;
  MB_CUDA(dev_malloc_async(&dl, 8, s));
  MB_CUDA(cudaMemsetAsync(dl, 0, 8, s));
  fwd_bwd(m, X, t, m->idx, n, B, dl, s);
  double l = 0;
  MB_CUDA(cudaMemcpyAsync(&l, dl, 8, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaMemcpyAsync(grad, m->G, m->nparams * 4, cudaMemcpyDeviceToDevice, s));
  MB_CUDA(cudaFreeAsync(dl, s));
  MB_CUDA(cudaStreamSynchronize(s));
  check_err(m);
  return l / (2.0 * double(n));
}

double mlp_train_device(macis_b200_mlp* m, const uint16_t* X, const float* t,
                        int64_t S, int epochs, int batch, double lr,
                        uint64_t seed) {
  MB_REQUIRE(S > 0 && epochs > 0 && batch > 0 && lr > 0, MACIS_B200_EINVAL,
             "invalid training arguments");
  cudaStream_t s = m->stream;
  const int64_t B = (int64_t(batch) + MLP_TM - 1) / MLP_TM * MLP_TM;
  ensure_batch(m, B);
  int64_t* perm = nullptr;
  double* dl = nullptr;
  MB_CUDA(dev_malloc_async(&perm, size_t(S) * 8, s));
  MB_CUDA(dev_malloc_async(&dl, 8, s));
  std::vector<int64_t> p(S);
  for(int64_t i = 0; i < S; ++i) p[i] = i;
  uint64_t st = seed ^ 0x5DEECE66Dull;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double last = 0;
  auto t0 = std::chrono::steady_clock::now();
  for(int e = 0; e < epochs; ++e) {
    for(int64_t i = S - 1; i > 0; --i)  // Fisher-Yates
      std::swap(p[i], p[int64_t(splitmix(st) % uint64_t(i + 1))]);
    MB_CUDA(cudaMemcpyAsync(perm, p.data(), size_t(S) * 8, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemsetAsync(dl, 0, 8, s));
    for(int64_t off = 0; off < S; off += B) {
      const int64_t nb = std::min<int64_t>(B, S - off);
      fwd_bwd(m, X, t, perm + off, nb, B, dl, s);
      ++m->step;
      const float bc1 = float(1.0 - std::pow(double(b1), double(m->step)));
      const float bc2 = float(1.0 - std::pow(double(b2), double(m->step)));
      adam_k<<<grid_for(m->nparams, 256, 4 * num_sms()), 256, 0, s>>>(
          m->P, m->G, m->Mo, m->Ve, int64_t(m->nparams), float(lr), b1, b2, eps,
          bc1, bc2), note_launch();
      repack(m, s);
    }
    MB_CUDA(cudaMemcpyAsync(&last, dl, 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
  }
  MB_CUDA(cudaFreeAsync(perm, s));
  MB_CUDA(cudaFreeAsync(dl, s));
  MB_CUDA(cudaStreamSynchronize(s));
  check_err(m);
  m->train_ms = std::chrono::duration<double, std::milli>(
                    std::chrono::steady_clock::now() - t0)
                    .count();
  m->last_loss = last / (2.0 * double(S));
  return m->last_loss;
}

namespace {
__global__ void clamp_below_k(float* t, size_t n, float lo) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    t[i] = fmaxf(t[i], lo);
}
}  // namespace

float mlp_clamp_samples(macis_b200_mlp* m, double q) {
  MB_REQUIRE(q >= 0 && q <= 1, MACIS_B200_EINVAL, "quantile outside [0, 1]");
  MB_REQUIRE(m->ns > 0, MACIS_B200_EINVAL, "no recorded samples");
  std::vector<float> t(m->ns);
  MB_CUDA(cudaMemcpyAsync(t.data(), m->ts, m->ns * 4, cudaMemcpyDeviceToHost,
                          m->stream));
  MB_CUDA(cudaStreamSynchronize(m->stream));
  const size_t k = std::min(m->ns - 1, size_t(q * double(m->ns - 1) + 0.5));
  std::nth_element(t.begin(), t.begin() + k, t.end());
  const float lo = t[k];
  clamp_below_k<<<grid_for(m->ns, 256, 4 * num_sms()), 256, 0, m->stream>>>(
      m->ts, m->ns, lo), note_launch();
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(m->stream));
  return lo;
}

void mlp_reserve_samples(macis_b200_mlp* m, size_t cap) {
  if(m->cap >= cap) return;
  if(m->xs) cudaFree(m->xs);
  if(m->ts) cudaFree(m->ts);
  m->xs = nullptr;
  m->ts = nullptr;
  m->cap = 0;
  m->ns = 0;
  m->xs = dalloc<uint16_t>(cap * size_t(m->din));
  m->ts = dalloc<float>(cap);
  m->cap = cap;
}

}  // namespace mb

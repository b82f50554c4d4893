// Screening network: din -> 256 -> 256 -> 1, GELU after both hidden layers.
// W1, W2 are BF16 tcgen05 operands with FP32 accumulation in TMEM; biases,
// the 256 -> 1 head and all master weights are FP32.
//
// The forward kernel is a persistent loop over tiles of 128 rows. Per tile:
//   1. a row source writes the 128 x din BF16 input tile into shared memory
//      (either a dense row-major matrix, or features computed on the fly from
//      the ASCI search's units, so that the input never goes through HBM);
//   2. one thread issues the layer-1 MMAs (M = 128, N = 256, K = 16 each)
//      while the weights stream through a 3-stage ring of 32 KB chunks
//      (64 K-columns x 256 rows) loaded with untiled bulk copies;
//   3. the 128 threads read the accumulator rows from TMEM, add the bias,
//      apply GELU and write H1 back into the input tile's shared memory in
//      the MMA operand layout;
//   4. layer 2 runs the same way on H1 with W2, and the epilogue applies bias
//      + GELU and the FP32 dot product with the head.
// The weights are kept in HBM already in the operand layout (tc.cuh), so a
// chunk is one contiguous 32 KB copy.
#pragma once
#include <cuda_bf16.h>

#include "tc.cuh"

namespace mb {

constexpr int MLP_H = 256;                     // hidden width
constexpr int MLP_TM = 128;                    // rows per tile (MMA M)
constexpr int MLP_KC = 64;                     // K columns per weight chunk
constexpr int MLP_WCHUNK = MLP_H * MLP_KC * 2;  // 32 KB
constexpr int MLP_STAGES = 3;
constexpr int MLP_NFEAT = 64;  // feature columns after the occupation bits

struct MlpWeights {
  int din;            // input width, a multiple of 64
  const uint4* w1t;   // operand layout: din/8 slabs x 256 rows x 16 B
  const uint4* w2t;   // 32 slabs x 256 rows x 16 B
  const float* b1;    // 256
  const float* b2;    // 256
  const float* w3;    // 256
  const float* b3;    // 1
};

// Training taps of the forward pass (column-major over rows: [256][ld]).
struct MlpTaps {
  float* z1t = nullptr;
  __nv_bfloat16* h1t = nullptr;
  float* z2t = nullptr;
  int64_t ld = 0;
};

__device__ __forceinline__ float gelu_f(float z) {
  return 0.5f * z * (1.f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad_f(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) +
         z * 0.39894228040143268f * expf(-0.5f * z * z);
}
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

inline size_t mlp_fwd_smem_bytes(int din) {
  const int kx = din > MLP_H ? din : MLP_H;
  return size_t(kx) * MLP_TM * 2 + size_t(MLP_STAGES) * MLP_WCHUNK +
         (2 * MLP_STAGES + 2) * 8 + 3 * MLP_H * 4 + 16;
}

// Dense row source: X row-major [nrows][din] BF16.
struct DenseRows {
  const uint4* x;
  int din;
  __device__ void fill(int64_t row0, int nvalid, uint8_t* xs, int tid) const {
    const int nkc = din / 8;
    for(int q = tid; q < MLP_TM * nkc; q += MLP_TM) {
      const int kc = q / MLP_TM, r = q % MLP_TM;
      uint4 v = make_uint4(0, 0, 0, 0);
      if(r < nvalid) v = __ldg(x + (row0 + r) * nkc + kc);
      *reinterpret_cast<uint4*>(xs + size_t(kc) * (MLP_TM * 16) + r * 16) = v;
    }
  }
};

// Forward over nrows rows; y[row] = network output. TRAIN also writes the
// taps. Every barrier wait gives up after limit_ns nanoseconds; then err
// (device) is set, the CTA waits (at most 100 ms each) for its bulk copies
// and MMAs still in flight, frees its TMEM and returns.
template <class Src, bool TRAIN>
__global__ void __launch_bounds__(MLP_TM, 1)
    mlp_fwd_k(MlpWeights W, Src src, int64_t nrows, float* y, MlpTaps tap,
              int* err, uint64_t limit_ns) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int din = W.din;
  const int nk1 = din / MLP_KC;
  const int cpt = nk1 + MLP_H / MLP_KC;  // weight chunks per tile
  const int kx = din > MLP_H ? din : MLP_H;
  uint8_t* xs = smem;
  uint8_t* ws = smem + size_t(kx) * MLP_TM * 2;
  uint64_t* full = reinterpret_cast<uint64_t*>(ws + MLP_STAGES * MLP_WCHUNK);
  uint64_t* empty = full + MLP_STAGES;
  uint64_t* accb = empty + MLP_STAGES;
  uint64_t* drain = accb + 1;  // used once, by the timeout path only
  float* sb1 = reinterpret_cast<float*>(drain + 1);
  float* sb2 = sb1 + MLP_H;
  float* sw3 = sb2 + MLP_H;

  const int64_t ntiles = (nrows + MLP_TM - 1) / MLP_TM;
  if(int64_t(blockIdx.x) >= ntiles) return;  // uniform; before any TMEM use
  const int64_t my_tiles = (ntiles - 1 - blockIdx.x) / gridDim.x + 1;

  for(int i = tid; i < MLP_H; i += MLP_TM) {
    sb1[i] = W.b1[i];
    sb2[i] = W.b2[i];
    sw3[i] = W.w3[i];
  }
  const float b3 = W.b3[0];
  if(tid == 0) {
    for(int s = 0; s < MLP_STAGES; ++s) {
      tc::mbar_init(full + s, 1);
      tc::mbar_init(empty + s, 1);
    }
    tc::mbar_init(accb, 1);
    tc::mbar_init(drain, 1);
    tc::mbar_init_fence();
  }
  if(warp == 0) tc::tmem_alloc(&tslot, MLP_H);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;

  const int64_t total = my_tiles * cpt;
  int64_t g_load = 0, g_mma = 0;  // meaningful in thread 0 only
  auto issue_load = [&](int64_t g) {
    const int s = int(g % MLP_STAGES);
    const int j = int(g % cpt);
    const uint4* srcp = j < nk1 ? W.w1t + size_t(j) * (MLP_WCHUNK / 16)
                                : W.w2t + size_t(j - nk1) * (MLP_WCHUNK / 16);
    tc::mbar_expect_tx(full + s, MLP_WCHUNK);
    tc::bulk_g2s(ws + size_t(s) * MLP_WCHUNK, srcp, MLP_WCHUNK, full + s);
  };
  if(tid == 0)
    for(; g_load < (total < MLP_STAGES ? total : MLP_STAGES); ++g_load)
      issue_load(g_load);

  constexpr uint32_t IDESC = tc::idesc_bf16(MLP_TM, MLP_H);
  constexpr uint32_t A_LBO = MLP_TM * 16;  // input / H1 slab
  constexpr uint32_t B_LBO = MLP_H * 16;   // weight slab
  uint32_t acc_n = 0;                      // accumulator commits so far
  bool fail = false;                       // this thread saw a timeout
  bool abort = false;                      // some thread did (uniform)
  const int r = warp * 32 + lane;          // tile row of this thread
  const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);

  for(int64_t lt = 0; lt < my_tiles; ++lt) {
    const int64_t row0 = (int64_t(blockIdx.x) + lt * gridDim.x) * MLP_TM;
    const int nvalid =
        int(nrows - row0 < MLP_TM ? nrows - row0 : int64_t(MLP_TM));
    src.fill(row0, nvalid, xs, tid);
    tc::fence_async_smem();
    if(__syncthreads_or(fail)) {
      abort = true;
      break;
    }

    for(int layer = 0; layer < 2; ++layer) {
      if(tid == 0) {
        tc::fence_after_sync();
        const int nch = layer == 0 ? nk1 : MLP_H / MLP_KC;
        const uint32_t xaddr = tc::smem_addr(xs);
        for(int c = 0; c < nch && !fail; ++c, ++g_mma) {
          const int s = int(g_mma % MLP_STAGES);
          if(!tc::mbar_wait(full + s, uint32_t((g_mma / MLP_STAGES) & 1),
                            limit_ns)) {
            fail = true;
            break;
          }
          const uint32_t waddr = tc::smem_addr(ws + size_t(s) * MLP_WCHUNK);
#pragma unroll
          for(int ks = 0; ks < MLP_KC / 16; ++ks) {
            const uint32_t slab = uint32_t(c * (MLP_KC / 8) + 2 * ks);
            const uint64_t da = tc::sdesc(xaddr + slab * A_LBO, A_LBO, 128);
            const uint64_t db =
                tc::sdesc(waddr + uint32_t(2 * ks) * B_LBO, B_LBO, 128);
            tc::mma_bf16(tmem, da, db, IDESC, (c | ks) ? 1u : 0u);
          }
          tc::mma_commit(empty + s);
          // refill the previous chunk's stage once its MMAs completed
          if(g_mma >= 1 && g_load < total) {
            const int64_t gp = g_mma - 1;
            if(!tc::mbar_wait(empty + gp % MLP_STAGES,
                              uint32_t((gp / MLP_STAGES) & 1), limit_ns)) {
              fail = true;
              break;
            }
            issue_load(g_load++);
          }
        }
        tc::mma_commit(accb);
      }
      // every thread: the accumulator of this layer
      if(!fail && !tc::mbar_wait(accb, acc_n & 1, limit_ns)) fail = true;
      ++acc_n;
      if(__syncthreads_or(fail)) {
        abort = true;
        break;
      }
      tc::fence_after_sync();
      const int64_t row = row0 + r;
      if(layer == 0) {
        for(int c0 = 0; c0 < MLP_H; c0 += 16) {
          uint32_t v[16];
          tc::tmem_ld16(trow + uint32_t(c0), v);
          tc::tmem_wait_ld();
          uint32_t pk[8];
#pragma unroll
          for(int q = 0; q < 16; q += 2) {
            const float z0 = __uint_as_float(v[q]) + sb1[c0 + q];
            const float z1 = __uint_as_float(v[q + 1]) + sb1[c0 + q + 1];
            pk[q / 2] = pack_bf16x2(gelu_f(z0), gelu_f(z1));
            if(TRAIN && r < nvalid) {
              tap.z1t[size_t(c0 + q) * tap.ld + row] = z0;
              tap.z1t[size_t(c0 + q + 1) * tap.ld + row] = z1;
              const uint32_t w = pk[q / 2];
              tap.h1t[size_t(c0 + q) * tap.ld + row] =
                  __ushort_as_bfloat16(uint16_t(w & 0xFFFF));
              tap.h1t[size_t(c0 + q + 1) * tap.ld + row] =
                  __ushort_as_bfloat16(uint16_t(w >> 16));
            }
          }
          uint8_t* d = xs + size_t(c0 / 8) * A_LBO + r * 16;
          *reinterpret_cast<uint4*>(d) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          *reinterpret_cast<uint4*>(d + A_LBO) =
              make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        tc::fence_before_sync();
        tc::fence_async_smem();
      } else {
        float acc = 0.f;
        for(int c0 = 0; c0 < MLP_H; c0 += 16) {
          uint32_t v[16];
          tc::tmem_ld16(trow + uint32_t(c0), v);
          tc::tmem_wait_ld();
#pragma unroll
          for(int q = 0; q < 16; ++q) {
            const float z = __uint_as_float(v[q]) + sb2[c0 + q];
            acc = fmaf(gelu_f(z), sw3[c0 + q], acc);
            if(TRAIN && r < nvalid) tap.z2t[size_t(c0 + q) * tap.ld + row] = z;
          }
        }
        if(r < nvalid) y[row] = acc + b3;
        tc::fence_before_sync();
      }
      if(__syncthreads_or(fail)) {
        abort = true;
        break;
      }
    }
    if(abort) break;
  }

  if(abort) {
    if(tid == 0) {
      atomicExch(err, 1);
      // bounded wait for the bulk copies still in flight: at most one per
      // stage is outstanding, and its phase is the stage's current one
      for(int64_t g = g_mma; g < g_load; ++g)
        tc::mbar_wait(full + g % MLP_STAGES, uint32_t((g / MLP_STAGES) & 1),
                      100000000ull);
      // and for every MMA this thread issued: a commit on the unused drain
      // barrier completes its phase 0 only after all of them (a commit on
      // accb could not be waited for unambiguously: its previous phase may
      // still be open)
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0u, 100000000ull);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if(warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, MLP_H);
  }
}

}  // namespace mb

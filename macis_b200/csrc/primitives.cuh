// Device-wide primitives written for this library: a workspace arena, an
// exclusive scan and a stable LSD radix sort over multi-word keys.
//
// The radix sort is the dedup engine of the ASCI search (the reference's
// std::sort by bitset_less, include/macis/asci/determinant_sort.hpp:40-57)
// and the grouping step of the Hamiltonian build. Keys are NW little-endian
// uint64 words stored item-contiguous; word NW-1 is the most significant
// (the bitset_less order, bitset_operations.hpp:289-306). Only 8-bit digits
// in which some key differs from the first key are sorted, so a 24-orbital
// string costs 3 passes whatever its word width. Within a tile each warp
// ranks its items with __match_any_sync, which keeps the sort stable: equal
// keys leave in input order, which fixes the accumulation order of duplicate
// ASCI contributions.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <vector>

#include "common.cuh"

namespace mb {

// ------------------------------------------------------------- workspace
// Stream-ordered allocations from the device's default memory pool; freed on
// destruction. Every buffer is 256-byte aligned.
struct Arena {
  cudaStream_t s;
  std::vector<void*> ptrs;
  explicit Arena(cudaStream_t st) : s(st) {}
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    size_t bytes = n * sizeof(T);
    if(bytes == 0) bytes = 256;
    const cudaError_t e = dev_malloc_async(&p, (bytes + 255) & ~size_t(255), s);
    if(e != cudaSuccess) {
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      throw Error(e == cudaErrorMemoryAllocation ? MACIS_B200_ENOMEM
                                                 : MACIS_B200_ECUDA,
                  "device allocation of " + std::to_string(bytes) +
                      " bytes failed (" + std::to_string(fr) +
                      " bytes free on the device): " + cudaGetErrorString(e));
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  void release(void* p) {
    for(auto& q : ptrs)
      if(q == p) {
        cudaFreeAsync(q, s);
        q = nullptr;
      }
  }
  ~Arena() {
    for(void* p : ptrs)
      if(p) cudaFreeAsync(p, s);
  }
};

// ------------------------------------------------------------------ scan
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_IPT = 8;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_IPT;

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* sh, T* total) {
  // sh: SCAN_THREADS/32 + 1 entries
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for(int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if(lane >= o) x += y;
  }
  if(lane == 31) sh[wid] = x;
  __syncthreads();
  if(wid == 0) {
    T w = lane < (int)(blockDim.x >> 5) ? sh[lane] : T(0);
#pragma unroll
    for(int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if(lane >= o) w += y;
    }
    if(lane < (int)(blockDim.x >> 5)) sh[lane] = w;
  }
  __syncthreads();
  T base = wid ? sh[wid - 1] : T(0);
  if(total) *total = sh[(blockDim.x >> 5) - 1];
  T r = base + x - v;
  __syncthreads();
  return r;
}

template <typename TI, typename TO>
__global__ void scan_reduce_k(const TI* in, size_t n, TO* sums) {
  __shared__ TO sh[SCAN_THREADS / 32 + 1];
  size_t base = size_t(blockIdx.x) * SCAN_CHUNK;
  TO acc = 0;
#pragma unroll
  for(int i = 0; i < SCAN_IPT; ++i) {
    size_t j = base + size_t(threadIdx.x) * SCAN_IPT + i;
    if(j < n) acc += TO(in[j]);
  }
  TO tot;
  block_excl_scan<TO>(acc, sh, &tot);
  if(threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <typename TI, typename TO>
__global__ void scan_apply_k(const TI* in, size_t n, TO* out,
                             const TO* offsets) {
  __shared__ TO sh[SCAN_THREADS / 32 + 1];
  size_t base = size_t(blockIdx.x) * SCAN_CHUNK;
  TO v[SCAN_IPT];
  TO acc = 0;
#pragma unroll
  for(int i = 0; i < SCAN_IPT; ++i) {
    size_t j = base + size_t(threadIdx.x) * SCAN_IPT + i;
    v[i] = j < n ? TO(in[j]) : TO(0);
    acc += v[i];
  }
  TO pre = block_excl_scan<TO>(acc, sh, nullptr);
  pre += offsets ? offsets[blockIdx.x] : TO(0);
#pragma unroll
  for(int i = 0; i < SCAN_IPT; ++i) {
    size_t j = base + size_t(threadIdx.x) * SCAN_IPT + i;
    if(j < n) out[j] = pre;
    pre += v[i];
  }
}

// out[i] = sum_{j<i} in[j]; out may alias in. If total != nullptr the grand
// total is written to *total (device pointer). Returns nothing; sync-free.
template <typename TI, typename TO>
void exclusive_scan(const TI* in, TO* out, size_t n, TO* total, Arena& A) {
  if(n == 0) {
    if(total) MB_CUDA(cudaMemsetAsync(total, 0, sizeof(TO), A.s));
    return;
  }
  size_t nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  if(nb == 1) {
    TO* sums = A.get<TO>(2);
    scan_reduce_k<TI, TO><<<1, SCAN_THREADS, 0, A.s>>>(in, n, sums), note_launch();
    if(total) MB_CUDA(cudaMemcpyAsync(total, sums, sizeof(TO), cudaMemcpyDeviceToDevice, A.s));
    scan_apply_k<TI, TO><<<1, SCAN_THREADS, 0, A.s>>>(in, n, out, nullptr), note_launch();
    return;
  }
  TO* sums = A.get<TO>(nb + 1);
  scan_reduce_k<TI, TO><<<unsigned(nb), SCAN_THREADS, 0, A.s>>>(in, n, sums), note_launch();
  exclusive_scan<TO, TO>(sums, sums, nb, total, A);
  scan_apply_k<TI, TO><<<unsigned(nb), SCAN_THREADS, 0, A.s>>>(in, n, out,
                                                               sums), note_launch();
}

// ------------------------------------------------------------ radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
// 8 items per thread: a 48 KB staging tile and few enough registers for 4
// resident blocks (measured: 16 items, 96 KB tiles and 2 blocks per SM made
// the sort passes latency-bound; 8 items cut the n = 48 ASCI sort by 25 %)
constexpr int RS_IPT = 8;
constexpr int RS_TILE = RS_THREADS * RS_IPT;  // 2048 items per block
constexpr int RS_WARP_ITEMS = RS_TILE / RS_WARPS;

template <int NW>
struct Key {
  uint64_t w[NW];
};

template <int NW>
__device__ __forceinline__ Key<NW> load_key(const uint64_t* k, size_t i) {
  Key<NW> r;
  if constexpr(NW == 2) {
    const ulonglong2 v = reinterpret_cast<const ulonglong2*>(k)[i];
    r.w[0] = v.x;
    r.w[1] = v.y;
  } else if constexpr(NW == 4) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(k) + 2 * i;
    ulonglong2 a = p[0], b = p[1];
    r.w[0] = a.x;
    r.w[1] = a.y;
    r.w[2] = b.x;
    r.w[3] = b.y;
  } else {
#pragma unroll
    for(int j = 0; j < NW; ++j) r.w[j] = k[i * NW + j];
  }
  return r;
}
template <int NW>
__device__ __forceinline__ void store_key(uint64_t* k, size_t i, Key<NW> r) {
  if constexpr(NW == 2) {
    reinterpret_cast<ulonglong2*>(k)[i] = make_ulonglong2(r.w[0], r.w[1]);
  } else if constexpr(NW == 4) {
    ulonglong2* p = reinterpret_cast<ulonglong2*>(k) + 2 * i;
    p[0] = make_ulonglong2(r.w[0], r.w[1]);
    p[1] = make_ulonglong2(r.w[2], r.w[3]);
  } else {
#pragma unroll
    for(int j = 0; j < NW; ++j) k[i * NW + j] = r.w[j];
  }
}
template <int NW>
__device__ __forceinline__ int key_cmp(const Key<NW>& a, const Key<NW>& b) {
#pragma unroll
  for(int j = NW - 1; j >= 0; --j) {
    if(a.w[j] < b.w[j]) return -1;
    if(a.w[j] > b.w[j]) return 1;
  }
  return 0;
}
template <int NW>
__device__ __forceinline__ bool key_eq(const Key<NW>& a, const Key<NW>& b) {
  bool r = true;
#pragma unroll
  for(int j = 0; j < NW; ++j) r &= a.w[j] == b.w[j];
  return r;
}

// OR over all keys of (key ^ key[0]) per word: the bits that vary.
template <int NW>
__global__ void key_vary_k(const uint64_t* keys, size_t n, uint64_t* vary) {
  uint64_t acc[NW];
  Key<NW> k0 = load_key<NW>(keys, 0);
#pragma unroll
  for(int j = 0; j < NW; ++j) acc[j] = 0;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    Key<NW> k = load_key<NW>(keys, i);
#pragma unroll
    for(int j = 0; j < NW; ++j) acc[j] |= k.w[j] ^ k0.w[j];
  }
#pragma unroll
  for(int j = 0; j < NW; ++j) {
    uint64_t v = acc[j];
    for(int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    if((threadIdx.x & 31) == 0 && v) atomicOr((unsigned long long*)&vary[j], v);
  }
}

template <int NW>
__device__ __forceinline__ unsigned digit_of(const Key<NW>& k, int shift) {
  // select the word with predicated moves, not a dynamic index (which
  // would place the key in local memory)
  const int sel = shift >> 6;
  uint64_t w;
  if constexpr(NW == 1) {
    w = k.w[0];
  } else if constexpr(NW == 2) {
    w = sel ? k.w[1] : k.w[0];
  } else {
    const uint64_t lo = (sel & 1) ? k.w[1] : k.w[0];
    const uint64_t hi = (sel & 1) ? k.w[3] : k.w[2];
    w = (sel & 2) ? hi : lo;
  }
  return unsigned(w >> (shift & 63)) & 255u;
}

template <int NW>
__global__ void __launch_bounds__(RS_THREADS)
    radix_hist_k(const uint64_t* keys, size_t n, int shift, uint32_t* counts,
                 unsigned nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = size_t(blockIdx.x) * RS_TILE;
#pragma unroll 4
  for(int r = 0; r < RS_IPT; ++r) {
    size_t i = base + size_t(r) * RS_THREADS + threadIdx.x;
    if(i < n) atomicAdd(&h[digit_of<NW>(load_key<NW>(keys, i), shift)], 1u);
  }
  __syncthreads();
  counts[size_t(threadIdx.x) * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Bytes of shared memory the scatter stages a tile in.
template <int NW, typename P>
constexpr size_t rs_stage_bytes() {
  return size_t(RS_TILE) * (8 * NW + sizeof(P));
}

// One digit pass over one tile of RS_TILE items starting at tile0. Every
// warp ranks its 256 items (__match_any_sync, input order), the block turns
// the per-warp counts into each item's position in a bucket-ordered copy of
// the tile in shared memory, and then consecutive threads write consecutive
// items of a bucket to consecutive addresses, so the stores of a bucket run
// (8 items per bucket on average) coalesce. Stable: within a bucket items
// keep warp, round and lane order, which is the input order. Keys are read
// twice (the second time from L2) so that no per-thread key array is needed.
// `resolve(d, count)` is called by thread d (one per digit) with the tile's
// count of digit d, between two block barriers, and returns the output
// position of the tile's first item with that digit.
template <int NW>
struct ShiftDigit {  // the byte of the key at bit `shift`
  int shift;
  __device__ __forceinline__ unsigned operator()(const Key<NW>& k) const {
    return digit_of<NW>(k, shift);
  }
};

template <int NW, typename P, class Digit, class Resolve>
__device__ __forceinline__ void rs_tile_pass(const uint64_t* keys,
                                             const P* vals, size_t n,
                                             Digit digit, size_t tile0,
                                             uint64_t* keys_out, P* vals_out,
                                             Resolve resolve) {
  extern __shared__ __align__(16) uint8_t rs_smem[];
  uint64_t* skeys = reinterpret_cast<uint64_t*>(rs_smem);
  P* svals = reinterpret_cast<P*>(skeys + size_t(RS_TILE) * NW);
  __shared__ uint32_t wcount[RS_WARPS][256];
  __shared__ uint32_t bstart[256];
  __shared__ uint64_t boff[256];
  __shared__ uint32_t scan_sh[RS_WARPS + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for(int d = threadIdx.x; d < RS_WARPS * 256; d += RS_THREADS)
    (&wcount[0][0])[d] = 0;
  __syncthreads();
  const size_t wbase = tile0 + size_t(wid) * RS_WARP_ITEMS;
  uint32_t rank[RS_IPT];
  unsigned dig[RS_IPT];
  // all loads first (16 in flight per thread), then the dependent ranking
#pragma unroll
  for(int r = 0; r < RS_IPT; ++r) {
    const size_t i = wbase + size_t(r) * 32 + lane;
    dig[r] = i < n ? digit(load_key<NW>(keys, i)) : 256u;
  }
#pragma unroll
  for(int r = 0; r < RS_IPT; ++r) {
    const bool ok = dig[r] < 256u;
    const unsigned peers = __match_any_sync(0xffffffffu, dig[r]);
    const unsigned before = __popc(peers & lanemask_lt());
    const int leader = __ffs(peers) - 1;
    uint32_t c = 0;
    if(ok) c = wcount[wid][dig[r]];
    rank[r] = c + before;
    __syncwarp();
    if(ok && lane == leader) wcount[wid][dig[r]] = c + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    // per digit: exclusive prefix over warps, then over digits (bucket
    // starts inside the tile), and the digit's output position
    const int d = threadIdx.x;
    uint32_t acc = 0;
#pragma unroll
    for(int w = 0; w < RS_WARPS; ++w) {
      const uint32_t c = wcount[w][d];
      wcount[w][d] = acc;
      acc += c;
    }
    bstart[d] = block_excl_scan<uint32_t>(acc, scan_sh, nullptr);
    boff[d] = resolve(d, acc);
  }
  __syncthreads();
#pragma unroll
  for(int r = 0; r < RS_IPT; ++r) {
    if(dig[r] < 256u) {
      const size_t i = wbase + size_t(r) * 32 + lane;
      const uint32_t pos = bstart[dig[r]] + wcount[wid][dig[r]] + rank[r];
      store_key<NW>(skeys, pos, load_key<NW>(keys, i));
      if(vals) svals[pos] = vals[i];
    }
  }
  __syncthreads();
  const int cnt = int(n - tile0 < size_t(RS_TILE) ? n - tile0 : size_t(RS_TILE));
  for(int j = threadIdx.x; j < cnt; j += RS_THREADS) {
    const Key<NW> kk = load_key<NW>(skeys, j);
    const unsigned d = digit(kk);
    const size_t dst = boff[d] + uint32_t(j - bstart[d]);
    store_key<NW>(keys_out, dst, kk);
    if(vals) vals_out[dst] = svals[j];
  }
}

// One digit pass with per-block bucket offsets from radix_hist_k + scan.
template <int NW, typename P>
__global__ void __launch_bounds__(RS_THREADS, 4)
    radix_scatter_k(const uint64_t* keys, const P* vals, size_t n, int shift,
                    const uint64_t* offsets, unsigned nblocks,
                    uint64_t* keys_out, P* vals_out) {
  // issued before the ranking: its latency hides behind the tile loads
  const uint64_t my_off =
      offsets[size_t(threadIdx.x) * nblocks + blockIdx.x];
  rs_tile_pass<NW, P>(keys, vals, n, ShiftDigit<NW>{shift},
                      size_t(blockIdx.x) * RS_TILE, keys_out, vals_out,
                      [&](int, uint32_t) { return my_off; });
}

// ------------------------------------------------------ one-sweep passes
// All digit histograms of the sort in one read of the keys: hist[p][d] =
// number of keys whose digit at shifts[p] is d (shared-memory counts per
// block, then one global add per (p, d)).
constexpr int RS_MAX_PASSES = 32;
// sorts of at least this many keys may use the one-sweep passes
constexpr size_t RS_ONESWEEP_MIN = size_t(1) << 16;
// polls of one look-back wait (each an L2 round trip) before it gives up
constexpr long long RS_SPIN_LIMIT = 1ll << 22;
template <int NW>
__global__ void __launch_bounds__(RS_THREADS)
    rs_hist_all_k(const uint64_t* keys, size_t n, const int* shifts, int np,
                  unsigned long long* hist) {
  __shared__ uint32_t h[RS_MAX_PASSES][256];
  __shared__ int sh_shift[RS_MAX_PASSES];
  for(int i = threadIdx.x; i < np * 256; i += RS_THREADS) (&h[0][0])[i] = 0;
  if(threadIdx.x < np) sh_shift[threadIdx.x] = shifts[threadIdx.x];
  __syncthreads();
  for(size_t i = size_t(blockIdx.x) * RS_THREADS + threadIdx.x; i < n;
      i += size_t(gridDim.x) * RS_THREADS) {
    const Key<NW> k = load_key<NW>(keys, i);
    for(int p = 0; p < np; ++p) atomicAdd(&h[p][digit_of<NW>(k, sh_shift[p])], 1u);
  }
  __syncthreads();
  for(int i = threadIdx.x; i < np * 256; i += RS_THREADS)
    if((&h[0][0])[i]) atomicAdd(hist + i, (unsigned long long)(&h[0][0])[i]);
}

// Status word of (tile, digit) in a one-sweep pass: the tile's count of the
// digit once ranked (AGG) or the inclusive count over tiles 0..tile (PRE).
constexpr uint64_t RS_AGG = 1ull << 62, RS_PRE = 2ull << 62;
constexpr uint64_t RS_VAL = (1ull << 62) - 1;

__device__ __forceinline__ uint64_t rs_ld_status(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void rs_st_status(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One digit pass in one kernel: blocks take tiles in order from a counter,
// publish their per-digit counts, and find the counts of all earlier tiles
// by looking back over the status words (decoupled look-back), so no
// separate histogram or scan of the pass is needed. Every look-back wait is
// bounded by `spin_limit` polls; a block that gives up sets *err and the
// host reruns the pass with radix_hist_k / radix_scatter_k.
template <int NW, typename P, class Digit>
__global__ void __launch_bounds__(RS_THREADS, 4)
    rs_onesweep_k(const uint64_t* keys, const P* vals, size_t n, Digit digit,
                  const unsigned long long* bucket, uint64_t* status,
                  unsigned* tile_counter, int* err, uint64_t* keys_out,
                  P* vals_out, long long spin_limit) {
  __shared__ uint32_t tile_sh;
  if(threadIdx.x == 0) tile_sh = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = tile_sh;
  const uint64_t base_d = bucket[threadIdx.x];
  rs_tile_pass<NW, P>(
      keys, vals, n, digit, size_t(tile) * RS_TILE, keys_out, vals_out,
      [&](int d, uint32_t count) -> uint64_t {
        uint64_t* mine = status + size_t(tile) * 256 + d;
        if(tile == 0) {
          rs_st_status(mine, RS_PRE | count);
          return base_d;
        }
        rs_st_status(mine, RS_AGG | count);
        uint64_t excl = 0;
        long long polls = 0;
        for(int64_t t = int64_t(tile) - 1; t >= 0;) {
          const uint64_t w = rs_ld_status(status + size_t(t) * 256 + d);
          const uint64_t flag = w & ~RS_VAL;
          if(flag == 0) {
            if(++polls > spin_limit) {
              atomicExch(err, 1);
              break;
            }
            continue;
          }
          excl += w & RS_VAL;
          if(flag == RS_PRE) break;
          --t;
        }
        rs_st_status(mine, RS_PRE | (excl + count));
        return base_d + excl;
      });
}

// Stable sort of n keys (NW words each) with optional payload. The sorted
// result ends in (keys, vals); keys_alt/vals_alt are scratch of the same
// size. Returns the number of digit passes run.
template <int NW, typename P>
int radix_sort(uint64_t* keys, P* vals, uint64_t* keys_alt, P* vals_alt,
               size_t n, Arena& A) {
  if(n < 2) return 0;
  uint64_t* d_vary = A.get<uint64_t>(NW);
  MB_CUDA(cudaMemsetAsync(d_vary, 0, NW * 8, A.s));
  key_vary_k<NW><<<grid_for(n, 256, 4 * num_sms()), 256, 0, A.s>>>(keys, n,
                                                                   d_vary), note_launch();
  uint64_t vary[NW];
  MB_CUDA(cudaMemcpyAsync(vary, d_vary, NW * 8, cudaMemcpyDeviceToHost, A.s));
  MB_CUDA(cudaStreamSynchronize(A.s));
  const unsigned nblocks = unsigned((n + RS_TILE - 1) / RS_TILE);
  constexpr size_t stage = rs_stage_bytes<NW, P>();
  MB_CUDA(cudaFuncSetAttribute(radix_scatter_k<NW, P>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(stage)));
  int passes = 0;
  std::vector<int> shifts;
  for(int w = 0; w < NW; ++w)
    for(int sft = 0; sft < 64; sft += 8)
      if((vary[w] >> sft) & 255ull) shifts.push_back(64 * w + sft);
  const int np = int(shifts.size());
  uint64_t *kin = keys, *kout = keys_alt;
  P *vin = vals, *vout = vals_alt;
  uint32_t* counts = nullptr;
  uint64_t* offs = nullptr;
  // classic pass: per-block histogram, scan, scatter
  auto classic_pass = [&](int shift) {
    if(!counts) {
      counts = A.get<uint32_t>(size_t(256) * nblocks);
      offs = A.get<uint64_t>(size_t(256) * nblocks);
    }
    radix_hist_k<NW><<<nblocks, RS_THREADS, 0, A.s>>>(kin, n, shift, counts,
                                                      nblocks), note_launch();
    exclusive_scan<uint32_t, uint64_t>(counts, offs, size_t(256) * nblocks,
                                       nullptr, A);
    radix_scatter_k<NW, P><<<nblocks, RS_THREADS, stage, A.s>>>(
        kin, vin, n, shift, offs, nblocks, kout, vout), note_launch();
  };
  // The one-sweep passes are opt-in (MACIS_B200_SORT_ONESWEEP=1): measured
  // on the n = 48 ASCI searches with bin-grouped ranges, the classic passes
  // were faster (1e5 core dets: 6.9 s against 8.1-11.3 s; 1e4: 0.64 s
  // against 0.67-0.69 s) and steadier
  const char* opt = getenv("MACIS_B200_SORT_ONESWEEP");
  const bool onesweep = n >= RS_ONESWEEP_MIN && np <= RS_MAX_PASSES &&
                        opt && opt[0] == '1';
  if(onesweep) {
    // all digit histograms in one read, bucket starts per pass on the host
    MB_CUDA(cudaFuncSetAttribute(rs_onesweep_k<NW, P, ShiftDigit<NW>>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(stage)));
    int* d_shifts = A.get<int>(size_t(np));
    MB_CUDA(cudaMemcpyAsync(d_shifts, shifts.data(), size_t(np) * sizeof(int),
                            cudaMemcpyHostToDevice, A.s));
    auto* hist = A.get<unsigned long long>(size_t(np) * 256);
    MB_CUDA(cudaMemsetAsync(hist, 0, size_t(np) * 256 * 8, A.s));
    rs_hist_all_k<NW><<<grid_for(n, RS_THREADS, 4 * size_t(num_sms())),
                        RS_THREADS, 0, A.s>>>(keys, n, d_shifts, np, hist),
        note_launch();
    std::vector<unsigned long long> h(size_t(np) * 256);
    MB_CUDA(cudaMemcpyAsync(h.data(), hist, h.size() * 8,
                            cudaMemcpyDeviceToHost, A.s));
    MB_CUDA(cudaStreamSynchronize(A.s));
    for(int p = 0; p < np; ++p) {
      unsigned long long acc = 0;
      for(int d = 0; d < 256; ++d) {
        const unsigned long long c = h[size_t(p) * 256 + d];
        h[size_t(p) * 256 + d] = acc;
        acc += c;
      }
    }
    auto* bucket = A.get<unsigned long long>(h.size());
    MB_CUDA(cudaMemcpyAsync(bucket, h.data(), h.size() * 8,
                            cudaMemcpyHostToDevice, A.s));
    uint64_t* status = A.get<uint64_t>(size_t(nblocks) * 256);
    unsigned* counter = A.get<unsigned>(1);
    int* err = A.get<int>(1);
    MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), A.s));
    for(int p = 0; p < np; ++p) {
      MB_CUDA(cudaMemsetAsync(status, 0, size_t(nblocks) * 256 * 8, A.s));
      MB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), A.s));
      rs_onesweep_k<NW, P><<<nblocks, RS_THREADS, stage, A.s>>>(
          kin, vin, n, ShiftDigit<NW>{shifts[p]}, bucket + size_t(p) * 256,
          status, counter, err, kout, vout, RS_SPIN_LIMIT), note_launch();
      int e = 0;
      MB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost,
                              A.s));
      MB_CUDA(cudaStreamSynchronize(A.s));
      if(e) {  // a look-back gave up: this pass again, the classic way
        MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), A.s));
        classic_pass(shifts[p]);
      }
      std::swap(kin, kout);
      std::swap(vin, vout);
      ++passes;
    }
  } else {
    for(int p = 0; p < np; ++p) {
      classic_pass(shifts[p]);
      std::swap(kin, kout);
      std::swap(vin, vout);
      ++passes;
    }
  }
  if(kin != keys) {
    MB_CUDA(cudaMemcpyAsync(keys, kin, n * NW * 8, cudaMemcpyDeviceToDevice, A.s));
    if(vals)
      MB_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(P), cudaMemcpyDeviceToDevice, A.s));
  }
  return passes;
}

// Counts of each digit value (< nbuckets <= 256) of a functor over the keys.
template <int NW, class Digit>
__global__ void __launch_bounds__(RS_THREADS)
    rs_hist_fn_k(const uint64_t* keys, size_t n, Digit digit,
                 unsigned long long* hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for(size_t i = size_t(blockIdx.x) * RS_THREADS + threadIdx.x; i < n;
      i += size_t(gridDim.x) * RS_THREADS)
    atomicAdd(&h[digit(load_key<NW>(keys, i))], 1u);
  __syncthreads();
  if(h[threadIdx.x])
    atomicAdd(hist + threadIdx.x, (unsigned long long)h[threadIdx.x]);
}

// Stable partition of (keys, vals) into (keys_out, vals_out) by the bucket
// digit(key) < nbuckets <= 256 (one histogram read, one one-sweep pass;
// the classic passes if a look-back gives up). Returns the nbuckets + 1
// bucket offsets.
template <int NW, typename P, class Digit>
std::vector<size_t> stable_partition(const uint64_t* keys, const P* vals,
                                     uint64_t* keys_out, P* vals_out,
                                     size_t n, int nbuckets, Digit digit,
                                     Arena& A) {
  std::vector<size_t> off(size_t(nbuckets) + 1, 0);
  if(n == 0) return off;
  auto* hist = A.get<unsigned long long>(256);
  MB_CUDA(cudaMemsetAsync(hist, 0, 256 * 8, A.s));
  rs_hist_fn_k<NW><<<grid_for(n, RS_THREADS, 4 * size_t(num_sms())),
                     RS_THREADS, 0, A.s>>>(keys, n, digit, hist), note_launch();
  std::vector<unsigned long long> h(256);
  MB_CUDA(cudaMemcpyAsync(h.data(), hist, 256 * 8, cudaMemcpyDeviceToHost,
                          A.s));
  MB_CUDA(cudaStreamSynchronize(A.s));
  unsigned long long acc = 0;
  for(int d = 0; d < 256; ++d) {
    const unsigned long long c = h[d];
    h[d] = acc;
    acc += c;
    if(d < nbuckets) off[size_t(d) + 1] = size_t(acc);
  }
  MB_REQUIRE(acc == n, MACIS_B200_EINVAL, "partition digit out of range");
  auto* bucket = A.get<unsigned long long>(256);
  MB_CUDA(cudaMemcpyAsync(bucket, h.data(), 256 * 8, cudaMemcpyHostToDevice,
                          A.s));
  const unsigned nblocks = unsigned((n + RS_TILE - 1) / RS_TILE);
  constexpr size_t stage = rs_stage_bytes<NW, P>();
  MB_CUDA(cudaFuncSetAttribute(rs_onesweep_k<NW, P, Digit>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(stage)));
  uint64_t* status = A.get<uint64_t>(size_t(nblocks) * 256);
  unsigned* counter = A.get<unsigned>(1);
  int* err = A.get<int>(1);
  MB_CUDA(cudaMemsetAsync(status, 0, size_t(nblocks) * 256 * 8, A.s));
  MB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), A.s));
  MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), A.s));
  rs_onesweep_k<NW, P, Digit><<<nblocks, RS_THREADS, stage, A.s>>>(
      keys, vals, n, digit, bucket, status, counter, err, keys_out, vals_out,
      RS_SPIN_LIMIT), note_launch();
  int e = 0;
  MB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, A.s));
  MB_CUDA(cudaStreamSynchronize(A.s));
  MB_REQUIRE(e == 0, MACIS_B200_ETIMEOUT,
             "partition pass: a look-back wait gave up");
  A.release(status);
  return off;
}

// Device bytes that allocations can still obtain: free memory plus what the
// default stream-ordered pool holds without using it.
inline size_t device_bytes_available() {
  size_t freeb = 0, totb = 0;
  MB_CUDA(cudaMemGetInfo(&freeb, &totb));
  int dev = 0;
  MB_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  if(cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long res = 0, used = 0;  // the attributes are 64-bit
    if(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &res) ==
           cudaSuccess &&
       cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) ==
           cudaSuccess &&
       res > used)
      freeb += size_t(res - used);
  }
  return freeb;
}
// Copy a device value to the host (synchronising the stream).
template <typename T>
T to_host(const T* d, cudaStream_t s) {
  T h;
  MB_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace mb

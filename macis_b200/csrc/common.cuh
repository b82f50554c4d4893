// Shared device/host definitions for the B200 selected-CI kernels.
//
// Determinants are kept in HBM as arrays of little-endian uint64 words, NW =
// NBITS/64 words per determinant, in the std::bitset<NBITS> word layout of
// the reference (include/macis/bitset_operations.hpp:264-286): NBITS=64 packs
// alpha in bits 0..31 and beta in bits 32..63 of one word; NBITS=128 has
// alpha in word 0 and beta in word 1; NBITS=256 has alpha in words 0-1 and
// beta in words 2-3. Spin strings are handled as Spin<NSW> (1 or 2 words).
#pragma once
#include <atomic>
#include <nvtx3/nvToolsExt.h>
#include <climits>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/macis_b200.h"

namespace mb {

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define MB_CUDA(x)                                                         \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if(e_ != cudaSuccess)                                                  \
      throw ::mb::Error(e_ == cudaErrorMemoryAllocation ? MACIS_B200_ENOMEM \
                                                         : MACIS_B200_ECUDA, \
                        std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while(0)

#define MB_REQUIRE(cond, code, msg)                  \
  do {                                               \
    if(!(cond)) throw ::mb::Error((code), (msg));    \
  } while(0)

// ----------------------------------------------------------- spin strings
template <int NSW>
struct Spin {
  uint64_t w[NSW];
};

template <int NSW>
__host__ __device__ __forceinline__ Spin<NSW> sp_zero() {
  Spin<NSW> s;
#pragma unroll
  for(int i = 0; i < NSW; ++i) s.w[i] = 0;
  return s;
}
template <int NSW>
__host__ __device__ __forceinline__ Spin<NSW> operator^(Spin<NSW> a,
                                                        Spin<NSW> b) {
#pragma unroll
  for(int i = 0; i < NSW; ++i) a.w[i] ^= b.w[i];
  return a;
}
template <int NSW>
__host__ __device__ __forceinline__ Spin<NSW> operator&(Spin<NSW> a,
                                                        Spin<NSW> b) {
#pragma unroll
  for(int i = 0; i < NSW; ++i) a.w[i] &= b.w[i];
  return a;
}
template <int NSW>
__host__ __device__ __forceinline__ bool operator==(Spin<NSW> a, Spin<NSW> b) {
  bool r = true;
#pragma unroll
  for(int i = 0; i < NSW; ++i) r &= (a.w[i] == b.w[i]);
  return r;
}
template <int NSW>
__device__ __forceinline__ int sp_popc(Spin<NSW> a) {
  int c = 0;
#pragma unroll
  for(int i = 0; i < NSW; ++i) c += __popcll(a.w[i]);
  return c;
}
// Index of the lowest set bit (ffs - 1 of bitset_operations.hpp:153-172).
template <int NSW>
__device__ __forceinline__ int sp_lowest(Spin<NSW> a) {
#pragma unroll
  for(int i = 0; i < NSW; ++i)
    if(a.w[i]) return 64 * i + __ffsll((long long)a.w[i]) - 1;
  return -1;
}
template <int NSW>
__device__ __forceinline__ Spin<NSW> sp_flip(Spin<NSW> a, int i) {
  a.w[i >> 6] ^= 1ull << (i & 63);
  return a;
}
template <int NSW>
__device__ __forceinline__ int sp_test(Spin<NSW> a, int i) {
  return int((a.w[i >> 6] >> (i & 63)) & 1ull);
}
// Number of set bits of a strictly between orbitals lo and hi (lo < hi).
template <int NSW>
__device__ __forceinline__ int sp_count_between(Spin<NSW> a, int lo, int hi) {
  int c = 0;
#pragma unroll
  for(int w = 0; w < NSW; ++w) {
    // bits (lo, hi) restricted to word w
    const int b0 = 64 * w, b1 = 64 * w + 64;
    int s = lo + 1 > b0 ? lo + 1 : b0;
    int e = hi < b1 ? hi : b1;
    if(s < e) {
      const int ls = s - b0, le = e - b0;  // [ls, le) within the word
      uint64_t m = (le == 64 ? ~0ull : ((1ull << le) - 1)) & ~((1ull << ls) - 1);
      c += __popcll(a.w[w] & m);
    }
  }
  return c;
}

// single_excitation_sign(state, p, q) (sd_operations.hpp:503-513): parity of
// the occupied orbitals of `state` strictly between p and q.
template <int NSW>
__device__ __forceinline__ double ex_sign(Spin<NSW> state, int p, int q) {
  const int lo = p < q ? p : q, hi = p < q ? q : p;
  return (sp_count_between(state, lo, hi) & 1) ? -1. : 1.;
}

// ---------------------------------------------------------- determinants
template <int NBITS>
struct DetTraits {
  static constexpr int NW = NBITS / 64;
  static constexpr int NSW = NBITS == 256 ? 2 : 1;
  using spin = Spin<NSW>;
  __device__ __forceinline__ static spin alpha(const uint64_t* d) {
    spin s;
    if constexpr(NBITS == 64)
      s.w[0] = d[0] & 0xffffffffull;
    else if constexpr(NBITS == 128)
      s.w[0] = d[0];
    else {
      s.w[0] = d[0];
      s.w[1] = d[1];
    }
    return s;
  }
  __device__ __forceinline__ static spin beta(const uint64_t* d) {
    spin s;
    if constexpr(NBITS == 64)
      s.w[0] = d[0] >> 32;
    else if constexpr(NBITS == 128)
      s.w[0] = d[1];
    else {
      s.w[0] = d[2];
      s.w[1] = d[3];
    }
    return s;
  }
  __device__ __forceinline__ static void make(uint64_t* d, spin a, spin b) {
    if constexpr(NBITS == 64)
      d[0] = (a.w[0] & 0xffffffffull) | (b.w[0] << 32);
    else if constexpr(NBITS == 128) {
      d[0] = a.w[0];
      d[1] = b.w[0];
    } else {
      d[0] = a.w[0];
      d[1] = a.w[1];
      d[2] = b.w[0];
      d[3] = b.w[1];
    }
  }
};

// ------------------------------------------------------------- integrals
// Device copies of the integrals and the intermediates of
// HamiltonianGenerator::generate_integral_intermediates
// (hamiltonian_generator/impl.hpp:26-70), all column-major.
struct Ints {
  int n;
  const double* T;       // n^2
  const double* V;       // n^4
  const double* G;       // n^4: V(i,j,k,l) - V(i,l,k,j)
  const double* G_red;   // n^3: G(k,k,i,j) at k + i n + j n^2
  const double* V_red;   // n^3: V(k,k,i,j)
  const double* G2_red;  // n^2: 0.5 G(i,i,j,j)
  const double* V2_red;  // n^2: V(i,i,j,j)
};

__device__ __forceinline__ size_t idx4(int p, int q, int r, int s, int n) {
  return size_t(p) + size_t(n) * (size_t(q) + size_t(n) * (size_t(r) + size_t(n) * size_t(s)));
}

// Packed excitation: o1 | v1 << 7 | o2 << 14 | v2 << 21 | (sign<0) << 28.
__device__ __forceinline__ uint32_t pack_ex(int o1, int v1, int o2, int v2,
                                            double sign) {
  return uint32_t(o1) | (uint32_t(v1) << 7) | (uint32_t(o2) << 14) |
         (uint32_t(v2) << 21) | (sign < 0 ? (1u << 28) : 0u);
}
__device__ __forceinline__ int ex_o1(uint32_t e) { return e & 127; }
__device__ __forceinline__ int ex_v1(uint32_t e) { return (e >> 7) & 127; }
__device__ __forceinline__ int ex_o2(uint32_t e) { return (e >> 14) & 127; }
__device__ __forceinline__ int ex_v2(uint32_t e) { return (e >> 21) & 127; }
__device__ __forceinline__ double ex_sgn(uint32_t e) {
  return (e >> 28) & 1 ? -1. : 1.;
}

// single_excitation_sign_indices (sd_operations.hpp:516-525): o1 is the
// orbital of ket that bra lacks, v1 the orbital of bra that ket lacks.
template <int NSW>
__device__ __forceinline__ uint32_t single_ex(Spin<NSW> bra, Spin<NSW> ket) {
  const Spin<NSW> ex = bra ^ ket;
  const int o1 = sp_lowest(ket & ex), v1 = sp_lowest(bra & ex);
  return pack_ex(o1, v1, 0, 0, ex_sign(ket, v1, o1));
}
// doubles_sign_indices (sd_operations.hpp:528-543).
template <int NSW>
__device__ __forceinline__ uint32_t double_ex(Spin<NSW> bra, Spin<NSW> ket) {
  Spin<NSW> ex = bra ^ ket;
  const int o1 = sp_lowest(ket & ex), v1 = sp_lowest(bra & ex);
  double sign = ex_sign(ket, v1, o1);
  ket = sp_flip(sp_flip(ket, o1), v1);
  ex = sp_flip(sp_flip(ex, o1), v1);
  const int o2 = sp_lowest(ket & ex), v2 = sp_lowest(bra & ex);
  sign *= ex_sign(ket, v2, o2);
  return pack_ex(o1, v1, o2, v2, sign);
}

// matrix_element_2 (matrix_elements.hpp:76-96) from a packed single
// excitation; occ_s/occ_o are the bra's same-spin and other-spin occupied
// orbitals in ascending order, summed in that order.
template <int NSW>
__device__ __forceinline__ double me_single(const Ints& I, uint32_t e,
                                            Spin<NSW> occ_s,
                                            Spin<NSW> occ_o) {
  const int o1 = ex_o1(e), v1 = ex_v1(e), n = I.n;
  double h = __ldg(I.T + v1 + size_t(o1) * n);
  const double* Gov = I.G_red + size_t(v1) * n + size_t(o1) * n * n;
  for(int p; (p = sp_lowest(occ_s)) >= 0; occ_s = sp_flip(occ_s, p))
    h += __ldg(Gov + p);
  const double* Vov = I.V_red + size_t(v1) * n + size_t(o1) * n * n;
  for(int p; (p = sp_lowest(occ_o)) >= 0; occ_o = sp_flip(occ_o, p))
    h += __ldg(Vov + p);
  return ex_sgn(e) * h;
}
// matrix_element_4 (matrix_elements.hpp:55-61).
__device__ __forceinline__ double me_ss_double(const Ints& I, uint32_t e) {
  return ex_sgn(e) *
         __ldg(I.G + idx4(ex_v1(e), ex_o1(e), ex_v2(e), ex_o2(e), I.n));
}
// matrix_element_22 (matrix_elements.hpp:63-74): sign = sign_a * sign_b.
__device__ __forceinline__ double me_os_double(const Ints& I, uint32_t ea,
                                               uint32_t eb) {
  const double sign = ex_sgn(ea) * ex_sgn(eb);
  return sign *
         __ldg(I.V + idx4(ex_v1(ea), ex_o1(ea), ex_v1(eb), ex_o1(eb), I.n));
}
// matrix_element_diag (matrix_elements.hpp:98-125), reference summation
// order.
template <int NSW>
__device__ double me_diag(const Ints& I, Spin<NSW> a, Spin<NSW> b) {
  const int n = I.n;
  double h = 0;
  for(Spin<NSW> s = a; sp_popc(s);) {
    int p = sp_lowest(s);
    h += __ldg(I.T + size_t(p) * (n + 1));
    s = sp_flip(s, p);
  }
  for(Spin<NSW> s = b; sp_popc(s);) {
    int p = sp_lowest(s);
    h += __ldg(I.T + size_t(p) * (n + 1));
    s = sp_flip(s, p);
  }
  for(Spin<NSW> sq = a; sp_popc(sq);) {
    int q = sp_lowest(sq);
    sq = sp_flip(sq, q);
    for(Spin<NSW> sp = a; sp_popc(sp);) {
      int p = sp_lowest(sp);
      sp = sp_flip(sp, p);
      h += __ldg(I.G2_red + p + size_t(q) * n);
    }
  }
  for(Spin<NSW> sq = b; sp_popc(sq);) {
    int q = sp_lowest(sq);
    sq = sp_flip(sq, q);
    for(Spin<NSW> sp = b; sp_popc(sp);) {
      int p = sp_lowest(sp);
      sp = sp_flip(sp, p);
      h += __ldg(I.G2_red + p + size_t(q) * n);
    }
  }
  for(Spin<NSW> sq = b; sp_popc(sq);) {
    int q = sp_lowest(sq);
    sq = sp_flip(sq, q);
    for(Spin<NSW> sp = a; sp_popc(sp);) {
      int p = sp_lowest(sp);
      sp = sp_flip(sp, p);
      h += __ldg(I.V2_red + p + size_t(q) * n);
    }
  }
  return h;
}

// Full matrix_element(bra, ket) dispatch (matrix_elements.hpp:22-53).
template <int NSW>
__device__ double me_generic(const Ints& I, Spin<NSW> ba, Spin<NSW> bb,
                             Spin<NSW> ka, Spin<NSW> kb) {
  const int ca = sp_popc(ba ^ ka), cb = sp_popc(bb ^ kb);
  if(ca + cb > 4) return 0.;
  if(ca == 4) return me_ss_double(I, double_ex(ba, ka));
  if(cb == 4) return me_ss_double(I, double_ex(bb, kb));
  if(ca == 2 && cb == 2) return me_os_double(I, single_ex(ba, ka), single_ex(bb, kb));
  if(ca == 2) return me_single(I, single_ex(ba, ka), ba, bb);
  if(cb == 2) return me_single(I, single_ex(bb, kb), bb, ba);
  return me_diag(I, ba, bb);
}

// --------------------------------------------------------------- helpers
// Number of kernels this library has launched (diagnostics for benchmarks).
inline unsigned long long& launch_counter() {
  static unsigned long long n = 0;
  return n;
}
inline void note_launch() { ++launch_counter(); }

// Named range on a profiler's timeline (NVTX v3, header-only: a no-op unless
// a tool is attached), around the library's phases.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// ------------------------------------------------------- fault injection
// Host-side failures for the tests of the error paths
// (macis_b200_inject_fault): the (k+1)-th next device allocation made by the
// library reports out-of-memory (once), or CSR builds with int32 indices
// accept fewer nonzeros. Nothing is made to fail on the device.
struct FaultInjection {
  std::atomic<int64_t> alloc_countdown{-1};  // -1: off
  std::atomic<int64_t> int32_limit{INT32_MAX};
};
inline FaultInjection& faults() {
  static FaultInjection f;
  return f;
}
inline bool take_injected_alloc_failure() {
  auto& c = faults().alloc_countdown;
  const int64_t v = c.load(std::memory_order_relaxed);
  if(v < 0) return false;
  c.store(v - 1, std::memory_order_relaxed);  // 0 -> -1: fires once
  return v == 0;
}
// Every device allocation of the library goes through these two.
template <typename T>
inline cudaError_t dev_malloc_async(T** p, size_t bytes, cudaStream_t s) {
  if(take_injected_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, s);
}
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  if(take_injected_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}
inline int64_t int32_index_limit() {
  return faults().int32_limit.load(std::memory_order_relaxed);
}

// Time limit of every barrier wait in the tensor-core kernels, nanoseconds
// (macis_b200_set_wait_limit_ns; 2 s by default). A wait that runs out makes
// the kernel record an error, drain its copies and MMAs in flight (fixed
// 100 ms bounds), free its TMEM and return; the call reports ETIMEOUT.
constexpr uint64_t kDefaultWaitLimitNs = 2000000000ull;
inline std::atomic<uint64_t>& wait_limit_slot() {
  static std::atomic<uint64_t> v{kDefaultWaitLimitNs};
  return v;
}
inline uint64_t wait_limit_ns() {
  return wait_limit_slot().load(std::memory_order_relaxed);
}

inline int num_sms() {
  static int n = 0;
  if(!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if(n <= 0) n = 148;
  }
  return n;
}

inline unsigned grid_for(size_t work, int block, size_t max_blocks = 0) {
  size_t g = (work + block - 1) / block;
  if(max_blocks && g > max_blocks) g = max_blocks;
  if(g < 1) g = 1;
  if(g > 0x7fffffffull) g = 0x7fffffff;
  return unsigned(g);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

}  // namespace mb

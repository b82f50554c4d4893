// CSR Hamiltonian build on the GPU -- the B200 replacement of
// DoubleLoopHamiltonianGenerator::make_csr_hamiltonian_block_
// (include/macis/hamiltonian_generator/double_loop.hpp:31-98).
//
// The reference tests every (bra, ket) pair. Here the ket determinants are
// grouped by alpha string and only alpha strings within two excitations of
// the bra alpha are visited ("sorted double loop over unique alpha strings
// and their beta partners"):
//
//  * Direct-product path (CAS / full-CI spaces, the order of
//    generate_hilbert_space, sd_operations.hpp:461-476): det i = (A, B) with
//    A = i / UB, B = i % UB. Per alpha string A the list of A' within two
//    excitations and per beta string B the lists of B' within one and two
//    excitations are precomputed with their packed (hole, particle, sign)
//    data, so a row is emitted as the concatenation over ascending A' of the
//    ascending B' lists: columns come out sorted with no search and no sort,
//    and every entry costs one list read and one integral gather.
//  * General path (selected spaces): kets sorted by (alpha, beta); per row
//    the connected alpha groups are scanned with popcount tests (exact-beta
//    binary search for alpha doubles); candidates are sorted by column in
//    shared memory (rows above 1024 candidates go through the radix sort).
//
// Both paths count candidates first (|h| > thresh applied in the fill), so
// rows are written once at their final position unless some element falls
// below the threshold, in which case a compaction pass closes the gaps.
// Matrix elements follow the reference summation order exactly
// (common.cuh), so values are bit-identical to the reference.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "internal.hpp"
#include "primitives.cuh"

namespace mb {

constexpr int HB_WARPS = 4;
constexpr int HB_THREADS = 32 * HB_WARPS;
constexpr int GEN_CAP = 1024;  // candidates sorted in shared memory per warp

template <int NSW>
__device__ __forceinline__ int sp_cmp(const Spin<NSW>& a, const Spin<NSW>& b) {
#pragma unroll
  for(int j = NSW - 1; j >= 0; --j) {
    if(a.w[j] < b.w[j]) return -1;
    if(a.w[j] > b.w[j]) return 1;
  }
  return 0;
}

template <int NSW>
__device__ __forceinline__ Spin<NSW> ld_spin(const uint64_t* p, size_t i) {
  Spin<NSW> s;
#pragma unroll
  for(int j = 0; j < NSW; ++j) s.w[j] = p[i * NSW + j];
  return s;
}
template <int NSW>
__device__ __forceinline__ void st_spin(uint64_t* p, size_t i, Spin<NSW> s) {
#pragma unroll
  for(int j = 0; j < NSW; ++j) p[i * NSW + j] = s.w[j];
}

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for(int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, v, o);
    if(lane >= o) v += y;
  }
  return v;
}

// ----------------------------------------------------- spin extraction
template <int NBITS>
__global__ void split_spins_k(const uint64_t* dets, size_t n, uint64_t* a,
                              uint64_t* b) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* d = dets + i * D::NW;
    if(a) st_spin<D::NSW>(a, i, D::alpha(d));
    if(b) st_spin<D::NSW>(b, i, D::beta(d));
  }
}

// ------------------------------------------------ direct-product detection
template <int NBITS>
__global__ void first_alpha_change_k(const uint64_t* dets, size_t n,
                                     unsigned long long* first) {
  // block-wide minimum first, one atomic per block
  using D = DetTraits<NBITS>;
  __shared__ unsigned long long wmin[32];
  const auto a0 = D::alpha(dets);
  unsigned long long best = ~0ull;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(!(D::alpha(dets + i * D::NW) == a0)) {
      best = i;
      break;  // later i of this thread are larger
    }
  for(int o = 16; o; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, best, o);
    best = y < best ? y : best;
  }
  if((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
  __syncthreads();
  if(threadIdx.x == 0) {
    for(int w = 1; w < int(blockDim.x >> 5); ++w) best = wmin[w] < best ? wmin[w] : best;
    if(best != ~0ull) atomicMin(first, best);
  }
}

// Flags any determinant that breaks the (A = i/UB, B = i%UB) product layout,
// is zero, or changes the electron count of a spin.
template <int NBITS>
__global__ void dp_check_k(const uint64_t* dets, size_t n, size_t ub,
                           int* bad) {
  using D = DetTraits<NBITS>;
  const auto a0 = D::alpha(dets), b0 = D::beta(dets);
  const int pa = sp_popc(a0), pb = sp_popc(b0);
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* d = dets + i * D::NW;
    const auto a = D::alpha(d), b = D::beta(d);
    const size_t A = i / ub, B = i % ub;
    bool ok = a == D::alpha(dets + A * ub * D::NW) &&
              b == D::beta(dets + B * D::NW) && sp_popc(a) == pa &&
              sp_popc(b) == pb && (pa + pb) > 0;
    if(!ok) atomicOr(bad, 1);
  }
}

template <int NW>
__global__ void adjacent_dup_k(const uint64_t* keys, size_t n, int* dup) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x + 1; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(key_eq<NW>(load_key<NW>(keys, i), load_key<NW>(keys, i - 1)))
      atomicOr(dup, 1);
}

template <int NBITS>
__global__ void gather_block_spins_k(const uint64_t* dets, size_t ua,
                                     size_t ub, uint64_t* alphas,
                                     uint64_t* betas) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
      i < (ua > ub ? ua : ub); i += size_t(gridDim.x) * blockDim.x) {
    if(i < ua) st_spin<D::NSW>(alphas, i, D::alpha(dets + i * ub * D::NW));
    if(i < ub) st_spin<D::NSW>(betas, i, D::beta(dets + i * D::NW));
  }
}

// ----------------------------------------------------- spin connectivity
// For every left string l, the right strings r (ascending) with
// popcount(l ^ r) <= maxp, each with its packed excitation seen from bra=l,
// ket=r and popcount in bits 29..31. Warp per left string; count pass when
// col == nullptr.
template <int NSW>
__global__ void spin_conn_k(const uint64_t* left, size_t nl,
                            const uint64_t* right, size_t nr, int maxp,
                            const int64_t* off, int64_t* cnt, int32_t* col,
                            uint32_t* info) {
  const int lane = threadIdx.x & 31;
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t l = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      l < nl; l += nwarp) {
    const Spin<NSW> L = ld_spin<NSW>(left, l);
    int64_t c = 0;
    const int64_t base = off ? off[l] : 0;
    for(size_t r0 = 0; r0 < nr; r0 += 32) {
      const size_t r = r0 + lane;
      Spin<NSW> R = sp_zero<NSW>();
      int p = 99;
      if(r < nr) {
        R = ld_spin<NSW>(right, r);
        p = sp_popc(L ^ R);
      }
      const bool hit = p <= maxp;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if(col && hit) {
        const int64_t pos = base + c + __popc(m & lanemask_lt());
        uint32_t e = 0;
        if(p == 2)
          e = single_ex(L, R);
        else if(p == 4)
          e = double_ex(L, R);
        col[pos] = int32_t(r);
        info[pos] = e | (uint32_t(p) << 29);
      }
      c += __popc(m);
    }
    if(!col && lane == 0) cnt[l] = c;
  }
}

struct DPData {
  int64_t UA, UB;
  const uint64_t* ua;      // UA spins
  const uint64_t* ub;      // UB spins
  const int64_t* aoff;     // UA+1
  const int32_t* acol;     // A'
  const uint32_t* ainfo;   // packed, pa in bits 29..31
  const int64_t* l2off;    // UB+1
  const int32_t* l2col;
  const uint32_t* l2info;
  const int64_t* l4off;    // UB+1
  const int32_t* l4col;
  const uint32_t* l4info;
  // same-spin parts of the single-excitation elements (dp_pg_k)
  const int64_t* pgaoff;   // UA+1
  const double* pga;
  const int64_t* pgboff;   // UB+1
  const double* pgb;
  // signed G value of every double of the alpha and beta L4 lists (0 for
  // the other entries): the fill reads it with the list entry instead of
  // gathering G
  const double* aval;
  const double* l4val;
};

// Occupied and empty orbitals of a spin string, in ascending order, into
// occ[0..no) and vir[0..n-no) (one orbital per lane).
template <int NSW>
__device__ __forceinline__ void spin_lists(const Spin<NSW>& s, int n, int lane,
                                           uint8_t* occ, uint8_t* vir) {
  for(int i = lane; i < n; i += 32) {
    int below = 0;  // occupied orbitals below i
#pragma unroll
    for(int w = 0; w < NSW; ++w) {
      const int lo = 64 * w;
      if(i > lo)
        below += __popcll(s.w[w] &
                          (i - lo >= 64 ? ~0ull : ((1ull << (i - lo)) - 1)));
    }
    if(sp_test(s, i))
      occ[below] = uint8_t(i);
    else
      vir[i - below] = uint8_t(i);
  }
}

// Singles per spin string: popcount * (n - popcount).
template <int NSW>
__global__ void dp_pgcount_k(const uint64_t* strings, int64_t ns, int n,
                             int64_t* cnt) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < ns;
      i += int64_t(gridDim.x) * blockDim.x) {
    const int no = sp_popc(ld_spin<NSW>(strings, i));
    cnt[i] = int64_t(no) * (n - no);
  }
}

// Same-spin part of every single excitation of every spin string s:
//   pg[off[s] + i nv + j] = T(v,o) + sum_{p in occ(s)} G_red(p,v,o)
// with v the i-th occupied and o the j-th empty orbital of s, summed in the
// order of matrix_element_2 (matrix_elements.hpp:86-104: T, then the
// same-spin G_red terms by ascending p). The element of a determinant adds
// the other-spin V_red terms to this partial sum in the same order, so the
// split is bit-exact. One warp per string.
template <int NSW>
__global__ void dp_pg_k(Ints I, const uint64_t* strings, int64_t ns,
                        const int64_t* off, double* pg) {
  __shared__ uint8_t lists[8][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int n = I.n, n2 = n * n;
  uint8_t* occ = lists[wid];
  uint8_t* vir = occ + 128;
  for(int64_t st = int64_t(blockIdx.x) * 8 + wid; st < ns;
      st += int64_t(gridDim.x) * 8) {
    const Spin<NSW> sp = ld_spin<NSW>(strings, st);
    const int no = sp_popc(sp), nv = n - no;
    __syncwarp();
    spin_lists<NSW>(sp, n, lane, occ, vir);
    __syncwarp();
    double* out = pg + off[st];
    for(int u = lane; u < no * nv; u += 32) {
      const int v = occ[u / nv], o = vir[u % nv];
      double h = __ldg(I.T + v + o * n);
      const double* Gov = I.G_red + v * n + o * n2;
      for(int k = 0; k < no; ++k) h += __ldg(Gov + occ[k]);
      out[u] = h;
    }
  }
}

// Signed G value of each double of an encoded connection list (0 for the
// other entries).
__global__ void dp_dval_k(const uint32_t* info, int64_t m, const double* G,
                          double* val) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
      i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t e = info[i];
    double v = 0.0;
    if(((e >> 29) & 3u) == 2u) {
      const double g = G[e & 0x0FFFFFFFu];
      v = (e >> 31) ? -g : g;
    }
    val[i] = v;
  }
}

// Per alpha string: how many connected A' at popcount 0, 2, 4.
__global__ void dp_acount_k(const int64_t* aoff, const uint32_t* ainfo,
                            int64_t UA, int32_t* na) {
  for(int64_t A = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; A < UA;
      A += int64_t(gridDim.x) * blockDim.x) {
    int c0 = 0, c2 = 0, c4 = 0;
    for(int64_t j = aoff[A]; j < aoff[A + 1]; ++j) {
      const int p = ainfo[j] >> 29;
      c0 += p == 0;
      c2 += p == 2;
      c4 += p == 4;
    }
    na[3 * A] = c0;
    na[3 * A + 1] = c2;
    na[3 * A + 2] = c4;
  }
}

__global__ void dp_rowcount_k(const int32_t* na, const int64_t* l2off,
                              const int64_t* l4off, int64_t r0, int64_t nrows,
                              int64_t UB, int64_t* cnt) {
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nrows;
      i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t A = (r0 + i) / UB, B = (r0 + i) % UB;
    cnt[i] = int64_t(na[3 * A]) * (l4off[B + 1] - l4off[B]) +
             int64_t(na[3 * A + 1]) * (l2off[B + 1] - l2off[B]) +
             int64_t(na[3 * A + 2]);
  }
}

// Diagonal matrix elements of a determinant list (matrix_element_diag).
template <int NBITS>
__global__ void hdiag_k(Ints I, const uint64_t* dets, size_t n, double* out) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* d = dets + i * D::NW;
    out[i] = me_diag(I, D::alpha(d), D::beta(d));
  }
}

template <typename VT>
__device__ __forceinline__ VT store_val(double h, bool is_diag);
template <>
__device__ __forceinline__ double store_val<double>(double h, bool) {
  return h;
}
template <>
__device__ __forceinline__ float store_val<float>(double h, bool is_diag) {
  return is_diag ? 0.0f : float(h);
}

// Direct-product fill. A CTA of DP_WARPS warps takes DP_WARPS rows that
// share one beta string B (rows (A..A+DP_WARPS-1, B)); the beta lists L2(B), L4(B)
// and the signed values of L4's beta doubles are staged once in shared
// memory.
// Each warp first evaluates all Slater-Condon singles of its bra into a
// shared table F[spin][v*n + o] (per-string partial sums plus the other-spin
// terms, reference summation order), then emits the row: entries are produced in ascending column order
// as the concatenation over connected alpha strings A' of the beta lists,
// two 32-entry rounds in flight, threshold compaction by ballot and
// streaming stores (the output must not evict the integrals from L2).
constexpr int DP_WARPS = 12;
// resident CTAs per SM: 24 warps of 80 registers (measured on the
// CAS(12e,12o) fill: 24 warps at 80 registers beat 32 at 64 by 7 %; of the
// 24-warp shapes 12 x 2 is ~1.5 % ahead of 8 x 3 and 6 x 4, since 12 rows
// share each staged beta list)
constexpr int DP_CTAS = 2;
constexpr int DP_THREADS = 32 * DP_WARPS;

struct DPShared {
  int n;
  int64_t l2max, l4max;
  size_t f_off, l2_off, l4_off, l4v_off, occ_off, bytes;
};

__host__ __device__ inline DPShared dp_shared_layout(int n, int64_t l2max,
                                                     int64_t l4max) {
  DPShared L;
  L.n = n;
  L.l2max = l2max;
  L.l4max = l4max;
  size_t o = 0;
  L.f_off = o;
  o += size_t(DP_WARPS) * 2 * n * n * 8;
  L.l2_off = o;
  o += size_t(l2max) * 8;
  L.l4_off = o;
  o += size_t(l4max) * 8;
  L.l4v_off = o;
  o += size_t(l4max) * 8;
  L.occ_off = o;
  o += size_t(DP_WARPS) * 4 * 128;  // occ/vir lists, both spins
  L.bytes = (o + 15) & ~size_t(15);
  return L;
}

// Packed list words of the fill (y of a uint2 whose x is the partner
// string index): bits 0..27 an integral offset, bits 29..30 the excitation
// class (0 none, 1 single, 2 double), bit 31 the fermionic sign.
//   alpha list:  single -> pair index a = v1 + o1 n (row a of VT) in bits
//                0..13, singles-table index v1 n + o1 in bits 14..27
//                double -> G offset of (v1,o1,v2,o2)
//   beta L2:     single -> pair index b = v1 + o1 n (column b of VT)
//   beta L4:     single -> singles-table index n^2 + v1 n + o1
//                double -> G offset
__global__ void dp_encode_k(uint32_t* info, int64_t m, int n, int which) {
  const uint32_t n2 = uint32_t(n) * n;
  for(int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
      i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t e = info[i];
    const int p = int(e >> 29);
    const uint32_t sg = (e >> 28) & 1u;
    uint32_t off = 0, cls = 0;
    const uint32_t o1 = ex_o1(e), v1 = ex_v1(e), o2 = ex_o2(e), v2 = ex_v2(e);
    if(p == 2) {
      cls = 1;
      if(which == 0)  // pair index (row of VT) | singles-table index << 14
        off = (v1 + o1 * n) | ((v1 * n + o1) << 14);
      else if(which == 1)
        off = v1 + o1 * n;  // pair index: column of VT
      else
        off = n2 + v1 * n + o1;
    } else if(p == 4) {
      cls = 2;
      off = v1 + n * (o1 + n * (v2 + n * o2));
    }
    info[i] = off | (cls << 29) | (sg << 31);
  }
}

// VT[a n^2 + b] = V[a + b n^2] for pair indices a, b < n^2
__global__ void v_pair_transpose_k(const double* V, double* VT, int n) {
  const size_t n2 = size_t(n) * n, n4 = n2 * n2;
  for(size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n4;
      x += size_t(gridDim.x) * blockDim.x)
    VT[(x % n2) * n2 + x / n2] = V[x];
}

const double* ham_vt(macis_b200_ham* h) {
  if(!h->VT) {
    const int n = h->norb;
    const size_t n4 = size_t(n) * n * n * n;
    MB_CUDA(dev_malloc(&h->VT, n4 * 8));
    v_pair_transpose_k<<<grid_for(n4, 256, 8 * num_sms()), 256, 0, h->stream>>>(
        h->V, h->VT, n), note_launch();
    MB_CUDA(cudaGetLastError());
  }
  return h->VT;
}

__device__ __forceinline__ double sgnd(uint32_t w, double v) {
  return (w >> 31) ? -v : v;  // == sign * v for sign in {+1, -1}
}

template <int NBITS, typename CI, typename VT>
__global__ void __launch_bounds__(DP_THREADS, DP_CTAS)
    dp_fill_k(Ints I, const double* __restrict__ Vt, DPData d, DPShared L,
              const double* __restrict__ hdiag,
              const int64_t* __restrict__ rowptr, CI* __restrict__ colind,
              VT* __restrict__ nzval, double* __restrict__ diag,
              int64_t* __restrict__ rowcnt, double thresh, int64_t r0,
              int64_t nrows) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  extern __shared__ __align__(16) unsigned char dsm[];
  // alpha-single segments of the current chunk: (row position, column
  // base, VT row offset, sign bit) and the alpha-single value
  __shared__ int4 seg_d[DP_WARPS][32];
  __shared__ double seg_single[DP_WARPS][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int n = L.n;
  const int n2 = n * n;
  double* F = reinterpret_cast<double*>(dsm + L.f_off) + size_t(wid) * 2 * n2;
  const uint2* sl2 = reinterpret_cast<const uint2*>(dsm + L.l2_off);
  const uint2* sl4 = reinterpret_cast<const uint2*>(dsm + L.l4_off);
  const double* sl4v = reinterpret_cast<const double*>(dsm + L.l4v_off);
  uint8_t* occl = dsm + L.occ_off + size_t(wid) * 512;  // occ[2][128]
  uint8_t* virl = occl + 256;                           // vir[2][128]
  const double* __restrict__ gVT = Vt;
  const int32_t UB = int32_t(d.UB);
  const int64_t A_lo = r0 / d.UB, A_hi = (r0 + nrows - 1) / d.UB;
  const int64_t nachunk = (A_hi - A_lo + DP_WARPS) / DP_WARPS;
  const int64_t nitems = nachunk * d.UB;
  for(int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int32_t B = int32_t(item % d.UB);
    const int64_t ac = item / d.UB;
    const int64_t l2b = d.l2off[B], l4b = d.l4off[B];
    const int32_t n2l = int32_t(d.l2off[B + 1] - l2b);
    const int32_t n4l = int32_t(d.l4off[B + 1] - l4b);
    __syncthreads();  // previous item's lists are no longer read
    uint2* wl2 = reinterpret_cast<uint2*>(dsm + L.l2_off);
    uint2* wl4 = reinterpret_cast<uint2*>(dsm + L.l4_off);
    const bool s2 = n2l <= L.l2max, s4 = n4l <= L.l4max;
    if(s2)
      for(int x = threadIdx.x; x < n2l; x += DP_THREADS)
        wl2[x] = make_uint2(uint32_t(d.l2col[l2b + x]), d.l2info[l2b + x]);
    if(s4)
      for(int x = threadIdx.x; x < n4l; x += DP_THREADS) {
        wl4[x] = make_uint2(uint32_t(d.l4col[l4b + x]), d.l4info[l4b + x]);
        reinterpret_cast<double*>(dsm + L.l4v_off)[x] = d.l4val[l4b + x];
      }
    __syncthreads();
    const int64_t A = A_lo + ac * DP_WARPS + wid;
    const int64_t grow = A * d.UB + B;
    if(A > A_hi || grow < r0 || grow >= r0 + nrows) continue;
    const int32_t row = int32_t(grow - r0);
    const Spin<NSW> sp[2] = {ld_spin<NSW>(d.ua, A), ld_spin<NSW>(d.ub, B)};
    // occupied / virtual lists, one orbital per lane
    int no[2], nv[2];
#pragma unroll
    for(int S = 0; S < 2; ++S) {
      no[S] = sp_popc(sp[S]);
      nv[S] = n - no[S];
      spin_lists<NSW>(sp[S], n, lane, occl + S * 128, virl + S * 128);
    }
    __syncwarp();
    // singles table: F[spin][v*n + o] = (T(v,o) + sum_{p in occ_same}
    // G_red(p,v,o)) + sum_{p in occ_other} V_red(p,v,o)
    // (matrix_elements.hpp:86-104 without the sign), v occupied and o empty
    // in the bra. The bracket is the per-string partial sum of dp_pg_k.
    {
      const int nsa = no[0] * nv[0], nsb = no[1] * nv[1];
      const double* __restrict__ pga = d.pga + d.pgaoff[A];
      const double* __restrict__ pgb = d.pgb + d.pgboff[B];
      // i = u / nv by a float product: (u + 0.5) / nv stays >= 0.5 / nv
      // away from an integer, far above the rounding error for u < 2^14
      const float rva = 1.0f / float(nv[0] > 0 ? nv[0] : 1);
      const float rvb = 1.0f / float(nv[1] > 0 ? nv[1] : 1);
      for(int t = lane; t < nsa + nsb; t += 32) {
        // selects instead of no[S] / nv[S]: a dynamic index would put the
        // arrays in local memory
        const int S = t < nsa ? 0 : 1;
        const int u = S ? t - nsa : t;
        const int nvS = S ? nv[1] : nv[0];
        const int noO = S ? no[0] : no[1];
        const int i = int((float(u) + 0.5f) * (S ? rvb : rva));
        const int v = occl[S * 128 + i], o = virl[S * 128 + (u - i * nvS)];
        double h = __ldg((S ? pgb : pga) + u);
        const double* Vov = I.V_red + v * n + o * n2;
        const uint8_t* po = occl + (1 - S) * 128;
#pragma unroll 4
        for(int k = 0; k < noO; ++k) h += __ldg(Vov + po[k]);
        F[S * n2 + v * n + o] = h;
      }
    }
    __syncwarp();
    const double hd = hdiag[row];
    const int64_t out0 = rowptr[row];
    CI* __restrict__ rc = colind + out0;
    VT* __restrict__ rv = nzval + out0;
    int32_t pos = 0, dropped = 0;  // dropped: this lane's count
    uint2 el = make_uint2(0u, 0u);  // this lane's entry of the beta L2 list
    if(lane < n2l)
      el = s2 ? sl2[lane]
              : make_uint2(uint32_t(__ldg(d.l2col + l2b + lane)),
                           __ldg(d.l2info + l2b + lane));
    // beta L2 entries 32..63 (n2l <= 64): each lane also holds entry lane + 32
    // and emits it in the same segment iteration as entry lane
    const bool fold = n2l > 32 && n2l <= 64;
    uint2 el2 = make_uint2(0u, 0u);
    const bool has2 = fold && lane + 32 < n2l;
    if(has2)
      el2 = s2 ? sl2[lane + 32]
               : make_uint2(uint32_t(__ldg(d.l2col + l2b + lane + 32)),
                            __ldg(d.l2info + l2b + lane + 32));
    using CS = typename std::conditional<sizeof(CI) == 4, int, long long>::type;
    CS* __restrict__ rcs = reinterpret_cast<CS*>(rc);
    // entries whose column differs from the row (every phase but the
    // same-alpha segment): no diagonal test
    auto put = [&](bool act, int32_t p, int32_t col, double h) {
      if(act) {
        const bool keep = fabs(h) > thresh;
        dropped += !keep;
        __stcs(rcs + p, CS(keep ? col : -1));
        __stcs(rv + p, store_val<VT>(h, false));
      }
    };
    auto put_d = [&](bool act, int32_t p, int32_t col, double h) {
      if(act) {
        const bool keep = fabs(h) > thresh;
        dropped += !keep;
        const bool isd = keep && col == row;
        __stcs(rcs + p, CS(keep ? col : -1));
        __stcs(rv + p, store_val<VT>(h, isd));
        if(isd) diag[row] = h;
      }
    };
    const int64_t c1 = d.aoff[A + 1];
    // the next chunk of the alpha list is loaded while this one is emitted
    int32_t nx_col = 0;
    uint32_t nx_ai = 0;
    double nx_val = 0.0;
    {
      const int64_t j = d.aoff[A] + lane;
      if(j < c1) {
        nx_col = __ldg(d.acol + j);
        nx_ai = __ldg(d.ainfo + j);
        nx_val = __ldg(d.aval + j);
      }
    }
    for(int64_t c = d.aoff[A]; c < c1; c += 32) {
      const int64_t j = c + lane;
      int32_t colA = 0;
      uint32_t ai = 0;
      double aval = 0.0;
      int cls = 3, cnt = 0;
      if(j < c1) {
        colA = nx_col * UB;
        ai = nx_ai;
        aval = nx_val;
        cls = int((ai >> 29) & 3u);
        cnt = cls == 0 ? n4l : cls == 1 ? n2l : 1;
      }
      if(j + 32 < c1) {
        nx_col = __ldg(d.acol + j + 32);
        nx_ai = __ldg(d.ainfo + j + 32);
        nx_val = __ldg(d.aval + j + 32);
      }
      const int incl = warp_incl_scan(cnt);
      const int32_t spos = pos + incl - cnt;
      pos += __shfl_sync(0xffffffffu, incl, 31);
      // (1) alpha doubles: beta unchanged, one entry each
      {
        put(cls == 2, spos, colA + B, aval);
      }
      // (2) the same-alpha segment: every beta string within two excitations
      unsigned m0 = __ballot_sync(0xffffffffu, cls == 0);
      while(m0) {
        const int L0 = __ffs(m0) - 1;
        m0 &= m0 - 1;
        const int32_t sp0 = __shfl_sync(0xffffffffu, spos, L0);
        const int32_t cA = __shfl_sync(0xffffffffu, colA, L0);
        for(int32_t t = lane; t - lane < n4l; t += 32) {
          const bool act = t < n4l;
          double h = 0;
          int32_t col = 0;
          if(act) {
            const uint2 ent = s4 ? sl4[t]
                                 : make_uint2(uint32_t(__ldg(d.l4col + l4b + t)),
                                              __ldg(d.l4info + l4b + t));
            const uint32_t cb = (ent.y >> 29) & 3u, off = ent.y & 0x0FFFFFFFu;
            // singles from this row's table (shared; offsets < 2 n^2),
            // doubles already signed
            const double vf = F[off < uint32_t(2 * n2) ? off : 0u];
            const double vd = s4 ? sl4v[t] : __ldg(d.l4val + l4b + t);
            col = cA + int32_t(ent.x);
            h = cb == 0 ? hd : cb == 1 ? sgnd(ent.y, vf) : vd;
          }
          put_d(act, sp0 + t, col, h);
        }
      }
      // (3) alpha singles: one segment of n2l entries (beta within one
      // excitation) per connected alpha string. Each lane keeps its beta
      // list entry for the row; the warp sweeps the segments.
      const unsigned m2 = __ballot_sync(0xffffffffu, cls == 1);
      if(cls == 1) {
        const int rk = __popc(m2 & lanemask_lt());
        const uint32_t pa_ = ai & 0x3FFFu;  // v1 + o1 n
        seg_d[wid][rk] = make_int4(spos, colA, int(pa_ * uint32_t(n2)),
                                   int(ai & 0x80000000u));
        seg_single[wid][rk] = sgnd(ai, F[(ai >> 14) & 0x3FFFu]);
      }
      __syncwarp();
      const int k2 = __popc(m2);
      if(fold) {
        const bool bsame = ((el.y >> 29) & 3u) == 0;
        const uint32_t boff = el.y & 0x0FFFFFFFu, bsg = el.y & 0x80000000u;
        const bool bsame2 = ((el2.y >> 29) & 3u) == 0;
        const uint32_t boff2 = el2.y & 0x0FFFFFFFu, bsg2 = el2.y & 0x80000000u;
        CS* __restrict__ rcl = rcs + lane;
        VT* __restrict__ rvl = rv + lane;
        for(int q = 0; q < k2; ++q) {
          const int4 sd = seg_d[wid][q];
          const double sgl = seg_single[wid][q];
          const double v = __ldg(gVT + uint32_t(sd.z + int(boff)));
          const double v2 = has2 ? __ldg(gVT + uint32_t(sd.z + int(boff2))) : 0.0;
          const double hv = __hiloint2double(
              __double2hiint(v) ^ (sd.w ^ int(bsg)), __double2loint(v));
          const double h = bsame ? sgl : hv;
          const bool keep = fabs(h) > thresh;
          dropped += keep ? 0 : 1;
          const uint32_t p = uint32_t(sd.x);
          __stcs(rcl + p, CS(keep ? sd.y + int32_t(el.x) : -1));
          __stcs(rvl + p, store_val<VT>(h, false));
          if(has2) {
            const double hv2 = __hiloint2double(
                __double2hiint(v2) ^ (sd.w ^ int(bsg2)), __double2loint(v2));
            const double h2 = bsame2 ? sgl : hv2;
            const bool keep2 = fabs(h2) > thresh;
            dropped += keep2 ? 0 : 1;
            __stcs(rcl + p + 32, CS(keep2 ? sd.y + int32_t(el2.x) : -1));
            __stcs(rvl + p + 32, store_val<VT>(h2, false));
          }
        }
      } else if(lane < n2l) {
        // branch-free body: the same-beta entry (offset 0) also loads from
        // its VT row and then selects the alpha-single value
        const bool bsame = ((el.y >> 29) & 3u) == 0;
        const uint32_t boff = el.y & 0x0FFFFFFFu, bsg = el.y & 0x80000000u;
        const int32_t elx = int32_t(el.x);
        CS* __restrict__ rcl = rcs + lane;
        VT* __restrict__ rvl = rv + lane;
#pragma unroll 2
        for(int q = 0; q < k2; ++q) {
          const int4 sd = seg_d[wid][q];
          const double sgl = seg_single[wid][q];
          const double v = __ldg(gVT + uint32_t(sd.z + int(boff)));
          // sign of the element: one XOR on the high word
          const double hv = __hiloint2double(
              __double2hiint(v) ^ (sd.w ^ int(bsg)), __double2loint(v));
          const double h = bsame ? sgl : hv;
          const bool keep = fabs(h) > thresh;
          dropped += keep ? 0 : 1;
          const uint32_t p = uint32_t(sd.x);
          __stcs(rcl + p, CS(keep ? sd.y + elx : -1));
          __stcs(rvl + p, store_val<VT>(h, false));
        }
      }
      if(n2l > 64) {  // list entries 32.. of every segment, flattened
        const int32_t w2 = n2l - 32;
        const int32_t tot2 = k2 * w2;
        const float invw = 1.0f / float(w2);
        for(int32_t e = lane; e < tot2; e += 32) {
          int sg = int(float(e) * invw);
          if(sg * w2 > e) --sg;
          if((sg + 1) * w2 <= e) ++sg;
          const int32_t t = 32 + e - sg * w2;
          const uint2 ent = s2 ? sl2[t]
                               : make_uint2(uint32_t(__ldg(d.l2col + l2b + t)),
                                            __ldg(d.l2info + l2b + t));
          const int4 sd = seg_d[wid][sg];
          const double sgl = seg_single[wid][sg];
          const double v = __ldg(gVT + uint32_t(sd.z + int(ent.y & 0x0FFFFFFFu)));
          const double hv = __hiloint2double(
              __double2hiint(v) ^ (sd.w ^ int(ent.y & 0x80000000u)),
              __double2loint(v));
          const double h = ((ent.y >> 29) & 3u) == 0 ? sgl : hv;
          const bool keep = fabs(h) > thresh;
          dropped += keep ? 0 : 1;
          const uint32_t p = uint32_t(sd.x + t);
          __stcs(rcs + p, CS(keep ? sd.y + int32_t(ent.x) : -1));
          __stcs(rv + p, store_val<VT>(h, false));
        }
      }
      __syncwarp();
    }
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
      dropped += __shfl_xor_sync(0xffffffffu, dropped, o);
    if(lane == 0) rowcnt[row] = int64_t(pos) - dropped;
  }
}

// Removes the entries marked with column -1 while packing rows to their
// final offsets (direct-product path with dropped elements).
template <typename CI, typename VT>
__global__ void compact_marked_k(const int64_t* oldptr, const int64_t* newptr,
                                 size_t m, const CI* ci, const VT* nz, CI* ci2,
                                 VT* nz2) {
  const int lane = threadIdx.x & 31;
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t r = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      r < m; r += nwarp) {
    const int64_t s = oldptr[r], e = oldptr[r + 1];
    int64_t o = newptr[r];
    for(int64_t b = s; b < e; b += 32) {
      const int64_t i = b + lane;
      CI c = 0;
      VT v = 0;
      bool keep = false;
      if(i < e) {
        c = ci[i];
        v = nz[i];
        keep = c >= 0;
      }
      const unsigned msk = __ballot_sync(0xffffffffu, keep);
      if(keep) {
        const int64_t p = o + __popc(msk & lanemask_lt());
        ci2[p] = c;
        nz2[p] = v;
      }
      o += __popc(msk);
    }
  }
}

// -------------------------------------------------------- general path
template <int NBITS>
struct GenKey {
  // sort key with the alpha string most significant
  static constexpr int KW = NBITS == 64 ? 1 : (NBITS == 128 ? 2 : 4);
};

template <int NBITS>
__global__ void gen_keys_k(const uint64_t* dets, size_t n, uint64_t* keys,
                           uint32_t* idx) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* d = dets + i * D::NW;
    const auto a = D::alpha(d), b = D::beta(d);
    if constexpr(NBITS == 64) {
      keys[i] = (a.w[0] << 32) | b.w[0];
    } else if constexpr(NBITS == 128) {
      keys[2 * i] = b.w[0];
      keys[2 * i + 1] = a.w[0];
    } else {
      keys[4 * i] = b.w[0];
      keys[4 * i + 1] = b.w[1];
      keys[4 * i + 2] = a.w[0];
      keys[4 * i + 3] = a.w[1];
    }
    idx[i] = uint32_t(i);
  }
}

template <int NBITS>
__device__ __forceinline__ void key_spins(const uint64_t* keys, size_t i,
                                          Spin<DetTraits<NBITS>::NSW>& a,
                                          Spin<DetTraits<NBITS>::NSW>& b) {
  if constexpr(NBITS == 64) {
    a.w[0] = keys[i] >> 32;
    b.w[0] = keys[i] & 0xffffffffull;
  } else if constexpr(NBITS == 128) {
    b.w[0] = keys[2 * i];
    a.w[0] = keys[2 * i + 1];
  } else {
    b.w[0] = keys[4 * i];
    b.w[1] = keys[4 * i + 1];
    a.w[0] = keys[4 * i + 2];
    a.w[1] = keys[4 * i + 3];
  }
}

// flags[i] = 1 at the first nonzero key of each alpha group; zero keys
// (zero determinants, which the reference skips) get 0 and are counted.
template <int NBITS>
__global__ void gen_group_flags_k(const uint64_t* keys, size_t n,
                                  uint32_t* flags,
                                  unsigned long long* nzero) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  constexpr int KW = GenKey<NBITS>::KW;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    Spin<NSW> a, b;
    key_spins<NBITS>(keys, i, a, b);
    const bool zero = sp_popc(a) + sp_popc(b) == 0;
    uint32_t f = 0;
    if(zero)
      atomicAdd(nzero, 1ull);
    else if(i == 0)
      f = 1;
    else {
      Spin<NSW> pa, pb;
      key_spins<NBITS>(keys, i - 1, pa, pb);
      const bool pzero = sp_popc(pa) + sp_popc(pb) == 0;
      f = (pzero || !(pa == a)) ? 1 : 0;
    }
    flags[i] = f;
    (void)KW;
  }
}

// Group tables: goff[g] (first sorted position), galpha[g]; sorted betas;
// per original index its group (or -1 for zero determinants).
template <int NBITS>
__global__ void gen_groups_k(const uint64_t* keys, const uint32_t* idx,
                             const uint32_t* flags, const uint32_t* gid_excl,
                             size_t n, int64_t* goff, uint64_t* galpha,
                             uint64_t* sbeta, int32_t* rowgroup) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    Spin<NSW> a, b;
    key_spins<NBITS>(keys, i, a, b);
    st_spin<NSW>(sbeta, i, b);
    const bool zero = sp_popc(a) + sp_popc(b) == 0;
    const uint32_t g = gid_excl[i] + flags[i] - 1;
    if(flags[i]) {
      goff[g] = int64_t(i);
      st_spin<NSW>(galpha, g, a);
    }
    if(rowgroup) rowgroup[idx[i]] = zero ? -1 : int32_t(g);
  }
}

__global__ void gen_group_end_k(int64_t* goff, uint32_t ng, int64_t end) {
  goff[ng] = end;
}

// ---- beta-major view of the kets: a row's alpha-double connections are the
// kets with its own beta whose alpha is 4 bits away, found by walking the
// kets of that beta when there are fewer of them than alpha-double groups.

// Sort keys with the beta string most significant.
template <int NBITS>
__global__ void gen_bkeys_k(const uint64_t* dets, size_t n, uint64_t* keys,
                            uint32_t* idx) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* d = dets + i * D::NW;
    const auto a = D::alpha(d), b = D::beta(d);
    if constexpr(NBITS == 64) {
      keys[i] = (b.w[0] << 32) | a.w[0];
    } else if constexpr(NBITS == 128) {
      keys[2 * i] = a.w[0];
      keys[2 * i + 1] = b.w[0];
    } else {
      keys[4 * i] = a.w[0];
      keys[4 * i + 1] = a.w[1];
      keys[4 * i + 2] = b.w[0];
      keys[4 * i + 3] = b.w[1];
    }
    idx[i] = uint32_t(i);
  }
}

template <int NBITS>
__device__ __forceinline__ void bkey_spins(const uint64_t* keys, size_t i,
                                           Spin<DetTraits<NBITS>::NSW>& a,
                                           Spin<DetTraits<NBITS>::NSW>& b) {
  if constexpr(NBITS == 64) {
    b.w[0] = keys[i] >> 32;
    a.w[0] = keys[i] & 0xffffffffull;
  } else if constexpr(NBITS == 128) {
    a.w[0] = keys[2 * i];
    b.w[0] = keys[2 * i + 1];
  } else {
    a.w[0] = keys[4 * i];
    a.w[1] = keys[4 * i + 1];
    b.w[0] = keys[4 * i + 2];
    b.w[1] = keys[4 * i + 3];
  }
}

// amaj[idx[m]] = m: original ket index -> alpha-major sorted position.
__global__ void gen_invert_k(const uint32_t* idx, size_t n, uint32_t* amaj) {
  for(size_t m = size_t(blockIdx.x) * blockDim.x + threadIdx.x; m < n;
      m += size_t(gridDim.x) * blockDim.x)
    amaj[idx[m]] = uint32_t(m);
}

// mgroup[m] = alpha group of sorted position m (-1 stays for zero dets).
__global__ void gen_mgroup_k(const int64_t* goff, uint32_t ng,
                             int32_t* mgroup) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for(int64_t gi = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      gi < int64_t(ng); gi += nw)
    for(int64_t m = goff[gi] + lane; m < goff[gi + 1]; m += 32)
      mgroup[m] = int32_t(gi);
}

// Per beta-major position: its alpha string and alpha-major position; flags
// at the first position of every distinct beta.
template <int NBITS>
__global__ void gen_bmajor_k(const uint64_t* bkeys, const uint32_t* bidx,
                             size_t n, const uint32_t* amaj, uint64_t* bm_alpha,
                             uint32_t* bm_m, uint32_t* bflags) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    Spin<NSW> a, b;
    bkey_spins<NBITS>(bkeys, i, a, b);
    st_spin<NSW>(bm_alpha, i, a);
    bm_m[i] = amaj[bidx[i]];
    uint32_t f = 1;
    if(i > 0) {
      Spin<NSW> pa, pb;
      bkey_spins<NBITS>(bkeys, i - 1, pa, pb);
      f = (pb == b) ? 0u : 1u;
    }
    bflags[i] = f;
  }
}

// Distinct betas (sorted) and the start of each in beta-major order.
template <int NBITS>
__global__ void gen_bgroups_k(const uint64_t* bkeys, const uint32_t* bflags,
                              const uint32_t* bgx, size_t n, int64_t* bgoff,
                              uint64_t* bgbeta) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    if(!bflags[i]) continue;
    Spin<NSW> a, b;
    bkey_spins<NBITS>(bkeys, i, a, b);
    bgoff[bgx[i]] = int64_t(i);
    st_spin<NSW>(bgbeta, bgx[i], b);
  }
}

// Alpha connectivity between bra groups and ket groups: (ket group, pa).
// Count pass (col == nullptr): cnt[l] = all connected groups, cnt4[l] =
// those at pa == 4. Fill pass: the pa <= 3 entries of bra group l first, in
// ket-group order, then its pa == 4 entries from off[l] + cnt[l] - cnt4[l].
template <int NSW>
__global__ void gen_aconn_k(const uint64_t* balpha, size_t nb,
                            const uint64_t* kalpha, size_t nk,
                            const int64_t* off, int64_t* cnt, int64_t* cnt4,
                            int32_t* col, uint8_t* pa_out) {
  const int lane = threadIdx.x & 31;
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t l = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      l < nb; l += nwarp) {
    const Spin<NSW> L = ld_spin<NSW>(balpha, l);
    int64_t c = 0, c4 = 0;
    const int64_t base = off ? off[l] : 0;
    const int64_t base4 = col ? base + cnt[l] - cnt4[l] : 0;
    for(size_t r0 = 0; r0 < nk; r0 += 32) {
      const size_t r = r0 + lane;
      int p = 99;
      if(r < nk) p = sp_popc(L ^ ld_spin<NSW>(kalpha, r));
      const bool hit = p <= 3, hit4 = p == 4;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      const unsigned m4 = __ballot_sync(0xffffffffu, hit4);
      if(col && (hit || hit4)) {
        const int64_t pos = hit ? base + c + __popc(m & lanemask_lt())
                                : base4 + c4 + __popc(m4 & lanemask_lt());
        col[pos] = int32_t(r);
        pa_out[pos] = uint8_t(p);
      }
      c += __popc(m);
      c4 += __popc(m4);
    }
    if(!col && lane == 0) {
      cnt[l] = c + c4;
      cnt4[l] = c4;
    }
  }
}

struct GenData {
  const int32_t* rowgroup;  // bra row -> bra group (-1: zero det)
  const int64_t* aoff;      // bra group -> aconn range
  const int32_t* acol;      // ket group
  const uint8_t* apa;
  const int64_t* goff;      // ket group -> sorted range
  const uint64_t* kalpha;   // ket group alpha
  const uint64_t* sbeta;    // sorted ket betas
  const uint32_t* sidx;     // sorted ket -> original index
  // beta hash tables of the large ket groups (gen_hsize_k / gen_hinsert_k)
  const int64_t* hoff;      // ket group -> table range (empty: no table)
  const int32_t* htab;      // sorted position - group start, -1 empty
  const int32_t* gbpop;     // ket group -> common beta popcount (-1: none)
  int n;                    // orbitals
  const int64_t* a4cnt;     // bra group -> its pa == 4 entries (at the end)
  // beta-major view of the kets (gen_bmajor_k / gen_bgroups_k)
  const uint64_t* bgbeta;   // distinct ket betas, sorted
  const int64_t* bgoff;     // their ranges in beta-major order
  int64_t nbgb;             // number of distinct ket betas
  const uint64_t* bm_alpha; // per beta-major position: alpha string
  const uint32_t* bm_m;     // per beta-major position: alpha-major position
  const int32_t* mgroup;    // alpha-major position -> ket group (-1: none)
};

// Ket groups of at least GEN_HASH_MIN members get a hash table of their
// betas so that a bra row connected to them by an alpha single excitation
// can look up its own beta single excitations instead of testing every
// member (a few hundred lookups against up to ~1e5 member tests for the
// large groups of ASCI spaces).
constexpr int64_t GEN_HASH_MIN = 256;

template <int NSW>
__device__ __forceinline__ uint64_t spin_hash(const Spin<NSW>& a) {
  uint64_t x = 0;
#pragma unroll
  for(int w = 0; w < NSW; ++w) x = (x ^ a.w[w]) * 0x9E3779B97F4A7C15ull;
  x ^= x >> 29;
  x *= 0xBF58476D1CE4E5B9ull;
  return x ^ (x >> 32);
}

// Per ket group (one warp each): the table size (a power of two >= 2 G for
// groups of G >= GEN_HASH_MIN members whose betas share one popcount, else
// 0) and that popcount (-1 when the group has no table).
template <int NSW>
__global__ void gen_hsize_k(const int64_t* goff, uint32_t ng,
                            const uint64_t* sbeta, int64_t* hsz,
                            int32_t* gbpop) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for(int64_t gi = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      gi < int64_t(ng); gi += nw) {
    const int64_t m0 = goff[gi], m1 = goff[gi + 1];
    int64_t sz = 0;
    int pc = -1;
    if(m1 - m0 >= GEN_HASH_MIN) {
      pc = sp_popc(ld_spin<NSW>(sbeta, m0));
      bool same = true;
      for(int64_t m = m0 + lane; m < m1; m += 32)
        same = same && sp_popc(ld_spin<NSW>(sbeta, m)) == pc;
      same = __all_sync(0xffffffffu, same);
      if(same) {
        sz = 1;
        while(sz < 2 * (m1 - m0)) sz <<= 1;
      } else {
        pc = -1;
      }
    }
    if(lane == 0) {
      hsz[gi] = sz;
      gbpop[gi] = pc;
    }
  }
}

// Inserts the first sorted position of every distinct beta of a ket group
// into its table (linear probing; the table has at least twice as many
// slots as entries, so every insertion finds a free slot).
template <int NSW>
__global__ void gen_hinsert_k(const int64_t* goff, uint32_t ng,
                              const uint64_t* sbeta, const int64_t* hoff,
                              int32_t* htab) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = int64_t(gridDim.x) * (blockDim.x >> 5);
  for(int64_t gi = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      gi < int64_t(ng); gi += nw) {
    const int64_t h0 = hoff[gi], hs = hoff[gi + 1] - h0;
    if(hs == 0) continue;
    const uint64_t mask = uint64_t(hs) - 1;
    const int64_t m0 = goff[gi], m1 = goff[gi + 1];
    for(int64_t m = m0 + lane; m < m1; m += 32) {
      const Spin<NSW> b = ld_spin<NSW>(sbeta, m);
      if(m > m0 && ld_spin<NSW>(sbeta, m - 1) == b) continue;  // duplicate
      uint64_t slot = spin_hash<NSW>(b) & mask;
      for(int64_t t = 0; t < hs; ++t) {
        if(atomicCAS(htab + h0 + slot, -1, int32_t(m - m0)) == -1) break;
        slot = (slot + 1) & mask;
      }
    }
  }
}

// Enumerates the candidate kets of one bra row warp-synchronously; calls
// emit(active, sorted_pos, ket_group, pa, pb) for chunks of <= 32.
template <int NSW, class F>
__device__ __forceinline__ void gen_enumerate(const GenData& g, int32_t rg,
                                              Spin<NSW> ba, Spin<NSW> bb,
                                              uint8_t* ov, F&& emit) {
  const int lane = threadIdx.x & 31;
  // occupied / empty orbitals of the bra beta (ov[0..128), ov[128..256)),
  // for the hash lookups of its single excitations
  const int nob = sp_popc(bb), nvb = g.n - nob;
  const int nenum = 1 + nob * nvb;  // the beta itself and its singles
  const float rnv = 1.0f / float(nvb > 0 ? nvb : 1);
  __syncwarp();
  spin_lists<NSW>(bb, g.n, lane, ov, ov + 128);
  __syncwarp();
  // the kets with beta bb (beta-major range [b0, b1))
  int64_t b0 = 0, b1 = 0;
  {
    int64_t lo = 0, hi = g.nbgb;
    while(lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if(sp_cmp(ld_spin<NSW>(g.bgbeta, mid), bb) < 0)
        lo = mid + 1;
      else
        hi = mid;
    }
    if(lo < g.nbgb && ld_spin<NSW>(g.bgbeta, lo) == bb) {
      b0 = g.bgoff[lo];
      b1 = g.bgoff[lo + 1];
    }
  }
  const int64_t c1 = g.aoff[rg + 1];
  const int64_t c4 = c1 - g.a4cnt[rg];  // the pa == 4 entries start here
  // alpha doubles through the kets of beta bb when they are fewer than the
  // alpha-double groups (each of which would take a binary search)
  const bool by_beta = b1 - b0 < c1 - c4;
  const int64_t cend = by_beta ? c4 : c1;
  if(by_beta) {
    for(int64_t p0 = b0; p0 < b1; p0 += 32) {
      const int64_t p = p0 + lane;
      bool act = false;
      int64_t m = 0;
      int32_t kg = 0;
      if(p < b1) {
        m = g.bm_m[p];
        kg = g.mgroup[m];
        act = kg >= 0 && sp_popc(ld_spin<NSW>(g.bm_alpha, p) ^ ba) == 4;
      }
      emit(act, m, kg, 4, 0);
    }
  }
  for(int64_t c = g.aoff[rg]; c < cend; c += 32) {
    const int64_t j = c + lane;
    const bool valid = j < cend;
    int32_t kg = 0;
    int pa = 99;
    if(valid) {
      kg = g.acol[j];
      pa = g.apa[j];
    }
    // alpha doubles (pa == 4): only the identical beta can connect
    int64_t lo = 0, hi = 0;
    if(valid && pa == 4) {
      int64_t a = g.goff[kg], b = g.goff[kg + 1];
      while(a < b) {  // lower bound
        const int64_t mid = (a + b) >> 1;
        if(sp_cmp(ld_spin<NSW>(g.sbeta, mid), bb) < 0)
          a = mid + 1;
        else
          b = mid;
      }
      lo = a;
      b = g.goff[kg + 1];
      while(a < b) {  // upper bound
        const int64_t mid = (a + b) >> 1;
        if(sp_cmp(ld_spin<NSW>(g.sbeta, mid), bb) <= 0)
          a = mid + 1;
        else
          b = mid;
      }
      hi = a;
    }
    int rem = int(hi - lo);
    int maxrem = rem;
#pragma unroll
    for(int o = 16; o; o >>= 1)
      maxrem = max(maxrem, __shfl_xor_sync(0xffffffffu, maxrem, o));
    for(int r = 0; r < maxrem; ++r) emit(r < rem, lo + r, kg, 4, 0);
    // pa <= 3: scan the group members
    unsigned scan = __ballot_sync(0xffffffffu, valid && pa <= 3);
    while(scan) {
      const int L = __ffs(scan) - 1;
      scan &= scan - 1;
      const int32_t gg = __shfl_sync(0xffffffffu, kg, L);
      const int ppa = __shfl_sync(0xffffffffu, pa, L);
      const int limit = 4 - ppa;
      const int64_t m0 = g.goff[gg], m1 = g.goff[gg + 1];
      const int64_t h0 = g.hoff[gg], hs = g.hoff[gg + 1] - h0;
      if(ppa == 2 && hs > 0 && g.gbpop[gg] == nob &&
         m1 - m0 > 8 * int64_t(nenum)) {
        // alpha single into a large group: only betas within one
        // excitation of bb connect, and all of them have bb's popcount
        const uint64_t mask = uint64_t(hs) - 1;
        for(int u0 = 0; u0 < nenum; u0 += 32) {
          const int u = u0 + lane;
          int64_t lo = 0, hi = 0;
          int pbv = 0;
          if(u < nenum) {
            Spin<NSW> q = bb;
            if(u > 0) {
              const int i = int((float(u - 1) + 0.5f) * rnv);
              const int j = (u - 1) - i * nvb;
              q = sp_flip(sp_flip(q, ov[i]), ov[128 + j]);
              pbv = 2;
            }
            uint64_t slot = spin_hash<NSW>(q) & mask;
            for(int64_t t = 0; t < hs; ++t) {
              const int32_t r = g.htab[h0 + slot];
              if(r < 0) break;
              if(ld_spin<NSW>(g.sbeta, m0 + r) == q) {
                lo = m0 + r;
                hi = lo + 1;
                while(hi < m1 && ld_spin<NSW>(g.sbeta, hi) == q) ++hi;
                break;
              }
              slot = (slot + 1) & mask;
            }
          }
          const int rem = int(hi - lo);
          int mr = rem;
#pragma unroll
          for(int o = 16; o; o >>= 1)
            mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, o));
          for(int r = 0; r < mr; ++r) emit(r < rem, lo + r, gg, 2, pbv);
        }
        continue;
      }
      for(int64_t base = m0; base < m1; base += 32) {
        const int64_t m = base + lane;
        bool act = m < m1;
        int pb = 99;
        if(act) pb = sp_popc(ld_spin<NSW>(g.sbeta, m) ^ bb);
        act = act && pb <= limit;
        emit(act, m, gg, ppa, pb);
      }
    }
  }
}

template <int NBITS>
__global__ void __launch_bounds__(HB_THREADS)
    gen_count_k(GenData g, const uint64_t* bra, size_t nbra, int64_t* cnt) {
  using D = DetTraits<NBITS>;
  __shared__ uint8_t s_ov[HB_WARPS][256];
  const int64_t nwarp = int64_t(gridDim.x) * HB_WARPS;
  for(int64_t row = int64_t(blockIdx.x) * HB_WARPS + (threadIdx.x >> 5);
      row < int64_t(nbra); row += nwarp) {
    const int32_t rg = g.rowgroup[row];
    int64_t c = 0;
    if(rg >= 0) {
      const auto ba = D::alpha(bra + row * D::NW);
      const auto bb = D::beta(bra + row * D::NW);
      gen_enumerate<D::NSW>(g, rg, ba, bb, s_ov[threadIdx.x >> 5],
                            [&](bool act, int64_t, int32_t, int, int) {
        c += __popc(__ballot_sync(0xffffffffu, act));
      });
    }
    if((threadIdx.x & 31) == 0) cnt[row] = c;
  }
}

// Fill: candidates go to a per-warp shared buffer (col, value), are sorted
// by column with a bitonic network and written with threshold compaction.
// Rows with more than GEN_CAP candidates are written unsorted to the
// long-row scratch (lcol/lval at loff[row]) and finished by the radix sort.
template <int NBITS, typename CI, typename VT>
__global__ void __launch_bounds__(HB_THREADS)
    gen_fill_k(Ints I, GenData g, const uint64_t* bra, int64_t row_a,
               int64_t row_b, const double* __restrict__ hdiag,
               const int64_t* __restrict__ rowptr,
               const int64_t* __restrict__ loff, int64_t lbase0,
               const uint32_t* __restrict__ lidx, uint64_t* lkey,
               double* lval, CI* __restrict__ colind, VT* __restrict__ nzval,
               double* __restrict__ diag, int64_t* __restrict__ rowcnt,
               double thresh) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  __shared__ uint32_t s_col[HB_WARPS][GEN_CAP];
  __shared__ double s_val[HB_WARPS][GEN_CAP];
  // orbital lists of the bra beta, 256 bytes per warp: dynamic, since the
  // candidate buffers take the whole static allowance
  extern __shared__ __align__(16) uint8_t gen_ov[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t* bc = s_col[wid];
  double* bv = s_val[wid];
  const int64_t nwarp = int64_t(gridDim.x) * HB_WARPS;
  for(int64_t row = row_a + int64_t(blockIdx.x) * HB_WARPS + wid; row < row_b;
      row += nwarp) {
    const int32_t rg = g.rowgroup[row];
    const int64_t ncand = rowptr[row + 1] - rowptr[row];
    if(rg < 0 || ncand == 0) {
      if(lane == 0) rowcnt[row] = 0;
      continue;
    }
    const bool lng = ncand > GEN_CAP;
    // long rows: (long-row index, column) sort keys and values into this
    // chunk's scratch
    const int64_t lbase = lng ? loff[row] - lbase0 : 0;
    const uint64_t lhi = lng ? uint64_t(lidx[row]) << 32 : 0;
    const uint64_t* bd = bra + row * D::NW;
    const Spin<NSW> ba = D::alpha(bd), bb = D::beta(bd);
    const double hd = hdiag[row];
    int64_t c = 0;
    gen_enumerate<NSW>(g, rg, ba, bb, gen_ov + wid * 256, [&](bool act, int64_t m,
                                                 int32_t kg, int pa, int pb) {
      double h = 0;
      uint32_t col = 0;
      if(act) {
        const Spin<NSW> ka = ld_spin<NSW>(g.kalpha, kg);
        const Spin<NSW> kb = ld_spin<NSW>(g.sbeta, m);
        if(pa == 0 && pb == 0)
          h = hd;
        else
          h = me_generic(I, ba, bb, ka, kb);
        col = g.sidx[m];
      }
      const unsigned msk = __ballot_sync(0xffffffffu, act);
      if(act) {
        const int64_t pos = c + __popc(msk & lanemask_lt());
        if(lng) {
          lkey[lbase + pos] = lhi | col;
          lval[lbase + pos] = h;
        } else {
          bc[pos] = col;
          bv[pos] = h;
        }
      }
      c += __popc(msk);
    });
    if(lng) {
      if(lane == 0) rowcnt[row] = -1;  // finished by the long-row pass
      continue;
    }
    __syncwarp();
    // bitonic sort of the c entries by column
    int P = 1;
    while(P < c) P <<= 1;
    for(int i = int(c) + lane; i < P; i += 32) bc[i] = 0xffffffffu;
    __syncwarp();
    for(int k = 2; k <= P; k <<= 1)
      for(int jj = k >> 1; jj > 0; jj >>= 1) {
        for(int i = lane; i < P; i += 32) {
          const int ixj = i ^ jj;
          if(ixj > i) {
            const bool up = (i & k) == 0;
            const uint32_t a = bc[i], b = bc[ixj];
            if((a > b) == up) {
              bc[i] = b;
              bc[ixj] = a;
              const double t = bv[i];
              bv[i] = bv[ixj];
              bv[ixj] = t;
            }
          }
        }
        __syncwarp();
      }
    // threshold compaction into the row
    const int64_t out0 = rowptr[row];
    int64_t kept = 0;
    for(int64_t base = 0; base < c; base += 32) {
      const int64_t i = base + lane;
      bool keep = false;
      uint32_t col = 0;
      double h = 0;
      if(i < c) {
        col = bc[i];
        h = bv[i];
        keep = fabs(h) > thresh;
      }
      const unsigned msk = __ballot_sync(0xffffffffu, keep);
      if(keep) {
        const int64_t pos = out0 + kept + __popc(msk & lanemask_lt());
        const bool isd = int64_t(col) == row;
        colind[pos] = CI(col);
        nzval[pos] = store_val<VT>(h, isd);
        if(isd) diag[row] = h;
      }
      kept += __popc(msk);
    }
    if(lane == 0) rowcnt[row] = kept;
    __syncwarp();
  }
}

// Long rows: the keys (row_rank << 32 | col) were radix-sorted with their
// FP64 values; write them back with threshold compaction.
template <typename CI, typename VT>
__global__ void long_rows_write_k(const int64_t* lrows, int64_t nl,
                                  const int64_t* loff_sorted, int64_t base0,
                                  const uint64_t* keys, const double* vals,
                                  const int64_t* rowptr, CI* colind,
                                  VT* nzval, double* diag, int64_t* rowcnt,
                                  double thresh) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = int64_t(gridDim.x) * (blockDim.x >> 5);
  for(int64_t r = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      r < nl; r += nwarp) {
    const int64_t row = lrows[r];
    const int64_t b = loff_sorted[r] - base0, e = loff_sorted[r + 1] - base0;
    const int64_t out0 = rowptr[row];
    int64_t kept = 0;
    for(int64_t base = b; base < e; base += 32) {
      const int64_t i = base + lane;
      bool keep = false;
      uint32_t col = 0;
      double h = 0;
      if(i < e) {
        col = uint32_t(keys[i] & 0xffffffffull);
        h = vals[i];
        keep = fabs(h) > thresh;
      }
      const unsigned msk = __ballot_sync(0xffffffffu, keep);
      if(keep) {
        const int64_t pos = out0 + kept + __popc(msk & lanemask_lt());
        const bool isd = int64_t(col) == row;
        colind[pos] = CI(col);
        nzval[pos] = store_val<VT>(h, isd);
        if(isd) diag[row] = h;
      }
      kept += __popc(msk);
    }
    if(lane == 0) rowcnt[row] = kept;
  }
}

__global__ void long_flags_k(const int64_t* rowptr, size_t n, uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = (rowptr[i + 1] - rowptr[i]) > GEN_CAP ? 1u : 0u;
}

__global__ void long_list_k(const int64_t* rowptr, size_t n,
                            const uint32_t* f, const uint32_t* fpos,
                            int64_t* lrows, int64_t* lcnt, int64_t* loff_row) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(f[i]) {
      lrows[fpos[i]] = int64_t(i);
      lcnt[fpos[i]] = rowptr[i + 1] - rowptr[i];
    }
}

__global__ void long_rowoff_k(const int64_t* lrows, const int64_t* loff,
                              int64_t nl, int64_t* loff_row) {
  for(int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < nl;
      r += int64_t(gridDim.x) * blockDim.x)
    loff_row[lrows[r]] = loff[r];
}

// --------------------------------------------------------- compaction
template <typename CI, typename VT>
__global__ void compact_rows_k(const int64_t* oldptr, const int64_t* newptr,
                               size_t m, const CI* ci, const VT* nz, CI* ci2,
                               VT* nz2) {
  const int lane = threadIdx.x & 31;
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t r = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      r < m; r += nwarp) {
    const int64_t s = oldptr[r], d = newptr[r], n = newptr[r + 1] - d;
    for(int64_t i = lane; i < n; i += 32) {
      ci2[d + i] = ci[s + i];
      nz2[d + i] = nz[s + i];
    }
  }
}

template <typename CI>
__global__ void rowptr_cast_k(const int64_t* in, size_t n, CI* out) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    out[i] = CI(in[i]);
}

// ----------------------------------------------------------- driver
// General-path tables of a (bra, ket) pair: kets sorted by (alpha, beta)
// with their alpha groups, the bra rows' groups, the alpha connectivity of
// bra groups to ket groups (pa <= 3 first, pa == 4 last), beta hash tables
// of the large ket groups and the beta-major view of the kets. Everything
// lives in A; `sub` says that bra is the contiguous block of ket starting
// at row r0.
template <int NBITS>
static GenData gen_plan(macis_b200_ham* h, const uint64_t* bra, size_t nbra,
                        const uint64_t* ket, size_t nket, bool sub, int64_t r0,
                        Arena& A) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  cudaStream_t s = A.s;
  const int sms = num_sms();
  constexpr int KW = GenKey<NBITS>::KW;
  auto sort_side = [&](const uint64_t* dets, size_t n, uint64_t*& keys,
                       uint32_t*& idx, int64_t*& goff, uint64_t*& galpha,
                       uint64_t*& sbeta, int32_t* rowgroup, uint32_t& ng) {
    keys = A.get<uint64_t>(n * KW);
    idx = A.get<uint32_t>(n);
    uint64_t* k2 = A.get<uint64_t>(n * KW);
    uint32_t* i2 = A.get<uint32_t>(n);
    gen_keys_k<NBITS><<<grid_for(n, 256, 8 * sms), 256, 0, s>>>(dets, n,
                                                               keys, idx), note_launch();
    radix_sort<KW, uint32_t>(keys, idx, k2, i2, n, A);
    A.release(k2);
    A.release(i2);
    uint32_t* flags = A.get<uint32_t>(n);
    uint32_t* gx = A.get<uint32_t>(n + 1);
    auto* nz = A.get<unsigned long long>(1);
    MB_CUDA(cudaMemsetAsync(nz, 0, 8, s));
    gen_group_flags_k<NBITS><<<grid_for(n, 256, 8 * sms), 256, 0, s>>>(
        keys, n, flags, nz), note_launch();
    exclusive_scan<uint32_t, uint32_t>(flags, gx, n, gx + n, A);
    ng = to_host(gx + n, s);
    goff = A.get<int64_t>(ng + 1);
    galpha = A.get<uint64_t>((ng + 1) * NSW);
    sbeta = A.get<uint64_t>(n * NSW);
    gen_groups_k<NBITS><<<grid_for(n, 256, 8 * sms), 256, 0, s>>>(
        keys, idx, flags, gx, n, goff, galpha, sbeta, rowgroup), note_launch();
    gen_group_end_k<<<1, 1, 0, s>>>(goff, ng, int64_t(n)), note_launch();
  };
  uint64_t *kkeys, *kalpha, *ksbeta;
  uint32_t *kidx, nkg = 0;
  int64_t* kgoff;
  int32_t* rowgroup = A.get<int32_t>(sub ? nket : nbra);
  sort_side(ket, nket, kkeys, kidx, kgoff, kalpha, ksbeta,
            sub ? rowgroup : nullptr, nkg);
  if(sub) rowgroup += r0;
  const uint64_t* balpha = kalpha;
  uint32_t nbg = nkg;
  if(!sub) {
    uint64_t *bkeys, *bsbeta, *bal;
    uint32_t* bidx;
    int64_t* bgoff;
    sort_side(bra, nbra, bkeys, bidx, bgoff, bal, bsbeta, rowgroup, nbg);
    balpha = bal;
  }
  // alpha connectivity bra groups -> ket groups
  int64_t* acnt = A.get<int64_t>(nbg + 1);
  int64_t* acnt4 = A.get<int64_t>(nbg + 1);
  int64_t* aoff = A.get<int64_t>(nbg + 1);
  const unsigned ga = grid_for(size_t(nbg) * 32, 256, 16 * sms);
  gen_aconn_k<NSW><<<ga, 256, 0, s>>>(balpha, nbg, kalpha, nkg, nullptr,
                                      acnt, acnt4, nullptr, nullptr), note_launch();
  exclusive_scan<int64_t, int64_t>(acnt, aoff, nbg, aoff + nbg, A);
  const int64_t natot = to_host(aoff + nbg, s);
  int32_t* acol = A.get<int32_t>(natot + 1);
  uint8_t* apa = A.get<uint8_t>(natot + 1);
  gen_aconn_k<NSW><<<ga, 256, 0, s>>>(balpha, nbg, kalpha, nkg, aoff, acnt,
                                      acnt4, acol, apa), note_launch();
  // beta hash tables of the large ket groups
  int64_t* hoff = A.get<int64_t>(nkg + 1);
  int32_t* gbpop = A.get<int32_t>(nkg + 1);
  int32_t* htab;
  {
    int64_t* hsz = A.get<int64_t>(nkg + 1);
    const unsigned gh = grid_for(size_t(nkg) * 32, 256, 16 * sms);
    gen_hsize_k<NSW><<<gh, 256, 0, s>>>(kgoff, nkg, ksbeta, hsz, gbpop), note_launch();
    exclusive_scan<int64_t, int64_t>(hsz, hoff, nkg, hoff + nkg, A);
    A.release(hsz);
    const int64_t htot = to_host(hoff + nkg, s);
    htab = A.get<int32_t>(size_t(std::max<int64_t>(htot, 1)));
    MB_CUDA(cudaMemsetAsync(htab, 0xFF, size_t(std::max<int64_t>(htot, 1)) * 4, s));
    if(htot > 0)
      gen_hinsert_k<NSW><<<gh, 256, 0, s>>>(kgoff, nkg, ksbeta, hoff, htab), note_launch();
  }
  // beta-major view of the kets
  uint64_t *bm_alpha, *bgbeta;
  uint32_t* bm_m;
  int32_t* mgroup;
  int64_t* bgoff;
  int64_t nbgb = 0;
  {
    uint64_t* bkeys = A.get<uint64_t>(nket * KW);
    uint32_t* bidx = A.get<uint32_t>(nket);
    uint64_t* k2 = A.get<uint64_t>(nket * KW);
    uint32_t* i2 = A.get<uint32_t>(nket);
    gen_bkeys_k<NBITS><<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(
        ket, nket, bkeys, bidx), note_launch();
    radix_sort<KW, uint32_t>(bkeys, bidx, k2, i2, nket, A);
    A.release(k2);
    A.release(i2);
    uint32_t* amaj = A.get<uint32_t>(nket);
    gen_invert_k<<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(kidx, nket,
                                                             amaj), note_launch();
    mgroup = A.get<int32_t>(nket);
    MB_CUDA(cudaMemsetAsync(mgroup, 0xFF, nket * 4, s));
    gen_mgroup_k<<<grid_for(size_t(nkg) * 32, 256, 16 * sms), 256, 0, s>>>(
        kgoff, nkg, mgroup), note_launch();
    bm_alpha = A.get<uint64_t>(nket * NSW);
    bm_m = A.get<uint32_t>(nket);
    uint32_t* bfl = A.get<uint32_t>(nket);
    uint32_t* bgx = A.get<uint32_t>(nket + 1);
    gen_bmajor_k<NBITS><<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(
        bkeys, bidx, nket, amaj, bm_alpha, bm_m, bfl), note_launch();
    exclusive_scan<uint32_t, uint32_t>(bfl, bgx, nket, bgx + nket, A);
    nbgb = int64_t(to_host(bgx + nket, s));
    bgoff = A.get<int64_t>(size_t(nbgb) + 1);
    bgbeta = A.get<uint64_t>((size_t(nbgb) + 1) * NSW);
    gen_bgroups_k<NBITS><<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(
        bkeys, bfl, bgx, nket, bgoff, bgbeta), note_launch();
    gen_group_end_k<<<1, 1, 0, s>>>(bgoff, uint32_t(nbgb), int64_t(nket)), note_launch();
    A.release(bkeys);
    A.release(bidx);
    A.release(amaj);
    A.release(bfl);
    A.release(bgx);
  }
  GenData gd{rowgroup, aoff, acol, apa, kgoff, kalpha, ksbeta, kidx,
             hoff, htab, gbpop, h->norb, acnt4,
             bgbeta, bgoff, nbgb, bm_alpha, bm_m, mgroup};
  return gd;
}

template <int NBITS, typename CI, typename VT>
static void build_impl(macis_b200_ham* h, const uint64_t* bra, size_t nbra,
                       const uint64_t* ket, size_t nket, double thresh,
                       macis_b200_csr* out) {
  bool general_fill_timed = false;  // the chunked general fill sums its own time
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  cudaStream_t s = h->stream;
  Arena A(s);
  const Ints I = h->ints();
  const int sms = num_sms();
  // bra may be a contiguous row block of the ket list (the row partition of
  // make_dist_csr_hamiltonian, csr_hamiltonian.hpp:49-82)
  const bool sub = bra >= ket && bra + nbra * D::NW <= ket + nket * D::NW &&
                   (bra - ket) % D::NW == 0;
  const int64_t r0 = sub ? int64_t((bra - ket) / D::NW) : 0;

  out->m = int64_t(nbra);
  out->n = int64_t(nket);
  MB_CUDA(dev_malloc_async(&out->diag, std::max<size_t>(nbra, 1) * 8, s));
  MB_CUDA(cudaMemsetAsync(out->diag, 0, std::max<size_t>(nbra, 1) * 8, s));
  int64_t* rowptr64 = A.get<int64_t>(nbra + 1);
  int64_t* rowcnt = A.get<int64_t>(nbra + 1);
  int64_t* nnz_d = A.get<int64_t>(1);
  double* hdiag = A.get<double>(nbra + 1);

  struct Ev {
    cudaEvent_t e[2];
    Ev() { cudaEventCreate(&e[0]); cudaEventCreate(&e[1]); }
    ~Ev() { cudaEventDestroy(e[0]); cudaEventDestroy(e[1]); }
    cudaEvent_t& operator[](int i) { return e[i]; }
  } ev;
  if(nbra == 0 || nket == 0) {
    out->nnz = 0;
    MB_CUDA(dev_malloc_async(&out->rowptr, (nbra + 1) * sizeof(CI), s));
    MB_CUDA(cudaMemsetAsync(out->rowptr, 0, (nbra + 1) * sizeof(CI), s));
    MB_CUDA(dev_malloc_async(&out->colind, 256, s));
    MB_CUDA(dev_malloc_async(&out->nzval, 256, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return;
  }
  MB_REQUIRE(nket < (size_t(1) << 31), MACIS_B200_ECAPACITY,
             "ket list longer than 2^31 determinants");

  hdiag_k<NBITS><<<grid_for(nbra, 256, 8 * sms), 256, 0, s>>>(I, bra, nbra,
                                                              hdiag), note_launch();

  // ---------------------------------------------- direct-product check
  bool direct = false;
  size_t UA = 0, UB = 0;
  uint64_t *ua = nullptr, *ub = nullptr;
  if(sub) {
    auto* first = A.get<unsigned long long>(1);
    const unsigned long long big = ~0ull;
    MB_CUDA(cudaMemcpyAsync(first, &big, 8, cudaMemcpyHostToDevice, s));
    first_alpha_change_k<NBITS><<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(
        ket, nket, first), note_launch();
    unsigned long long f = to_host(first, s);
    UB = f == big ? nket : size_t(f);
    if(UB > 0 && nket % UB == 0) {
      UA = nket / UB;
      int* bad = A.get<int>(2);
      MB_CUDA(cudaMemsetAsync(bad, 0, 8, s));
      dp_check_k<NBITS><<<grid_for(nket, 256, 8 * sms), 256, 0, s>>>(
          ket, nket, UB, bad), note_launch();
      ua = A.get<uint64_t>(UA * NSW);
      ub = A.get<uint64_t>(UB * NSW);
      gather_block_spins_k<NBITS><<<grid_for(std::max(UA, UB), 256, 8 * sms),
                                    256, 0, s>>>(ket, UA, UB, ua, ub), note_launch();
      // uniqueness of block alphas and of the betas of block 0
      uint64_t* sa = A.get<uint64_t>(UA * NSW);
      uint64_t* sb = A.get<uint64_t>(UB * NSW);
      uint64_t* tmp = A.get<uint64_t>(std::max(UA, UB) * NSW);
      MB_CUDA(cudaMemcpyAsync(sa, ua, UA * NSW * 8, cudaMemcpyDeviceToDevice, s));
      MB_CUDA(cudaMemcpyAsync(sb, ub, UB * NSW * 8, cudaMemcpyDeviceToDevice, s));
      radix_sort<NSW, uint32_t>(sa, nullptr, tmp, nullptr, UA, A);
      radix_sort<NSW, uint32_t>(sb, nullptr, tmp, nullptr, UB, A);
      adjacent_dup_k<NSW><<<grid_for(UA, 256, 4 * sms), 256, 0, s>>>(sa, UA, bad + 1), note_launch();
      adjacent_dup_k<NSW><<<grid_for(UB, 256, 4 * sms), 256, 0, s>>>(sb, UB, bad + 1), note_launch();
      int hb[2];
      MB_CUDA(cudaMemcpyAsync(hb, bad, 8, cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      // the fill keeps a singles table of 2 norb^2 doubles per warp in
      // shared memory: spaces whose orbitals make it too large (norb above
      // ~33) take the general path even when they have the product layout
      direct = hb[0] == 0 && hb[1] == 0 && UA < (size_t(1) << 31) &&
               UB < (size_t(1) << 31) && h->norb <= 127 &&
               dp_shared_layout(int(h->norb), 512, 1024).bytes <= 220 * 1024;
    }
  }

  int64_t nnz_ub = 0;
  CI* colind = nullptr;
  VT* nzval = nullptr;
  if(direct) {
    out->direct_product = true;
    // spin connectivity lists
    auto conn = [&](const uint64_t* L, size_t nl, int maxp, int64_t*& off,
                    int32_t*& col, uint32_t*& info) {
      int64_t* cnt = A.get<int64_t>(nl + 1);
      off = A.get<int64_t>(nl + 1);
      const unsigned g = grid_for(nl * 32, 256, 16 * sms);
      spin_conn_k<NSW><<<g, 256, 0, s>>>(L, nl, L, nl, maxp, nullptr, cnt,
                                         nullptr, nullptr), note_launch();
      exclusive_scan<int64_t, int64_t>(cnt, off, nl, off + nl, A);
      const int64_t tot = to_host(off + nl, s);
      col = A.get<int32_t>(tot + 1);
      info = A.get<uint32_t>(tot + 1);
      spin_conn_k<NSW><<<g, 256, 0, s>>>(L, nl, L, nl, maxp, off, cnt, col,
                                         info), note_launch();
    };
    int64_t *aoff, *l2off, *l4off;
    int32_t *acol, *l2col, *l4col;
    uint32_t *ainfo, *l2info, *l4info;
    conn(ua, UA, 4, aoff, acol, ainfo);
    conn(ub, UB, 2, l2off, l2col, l2info);
    conn(ub, UB, 4, l4off, l4col, l4info);
    int32_t* na = A.get<int32_t>(3 * UA);
    dp_acount_k<<<grid_for(UA, 256, 4 * sms), 256, 0, s>>>(aoff, ainfo,
                                                          int64_t(UA), na), note_launch();
    dp_rowcount_k<<<grid_for(nbra, 256, 8 * sms), 256, 0, s>>>(
        na, l2off, l4off, r0, int64_t(nbra), int64_t(UB), rowcnt), note_launch();
    exclusive_scan<int64_t, int64_t>(rowcnt, rowptr64, nbra, rowptr64 + nbra, A);
    nnz_ub = to_host(rowptr64 + nbra, s);
    out->nnz_candidates = nnz_ub;
    MB_CUDA(dev_malloc_async(&colind, std::max<int64_t>(nnz_ub, 1) * sizeof(CI), s));
    MB_CUDA(dev_malloc_async(&nzval, std::max<int64_t>(nnz_ub, 1) * sizeof(VT), s));
    {
      const int nn0 = h->norb;
      const int64_t na_ = to_host(aoff + UA, s), n2_ = to_host(l2off + UB, s),
                    n4_ = to_host(l4off + UB, s);
      dp_encode_k<<<grid_for(size_t(na_), 256, 8 * sms), 256, 0, s>>>(ainfo, na_, nn0, 0), note_launch();
      dp_encode_k<<<grid_for(size_t(n2_), 256, 8 * sms), 256, 0, s>>>(l2info, n2_, nn0, 1), note_launch();
      dp_encode_k<<<grid_for(size_t(n4_), 256, 8 * sms), 256, 0, s>>>(l4info, n4_, nn0, 2), note_launch();
    }
    // orbital lists of the kernels below hold 128 entries per spin
    MB_REQUIRE(nket < (size_t(1) << 31) && h->norb <= 127,
               MACIS_B200_ECAPACITY,
               "direct-product fill needs < 2^31 determinants, norb < 128");
    // same-spin partial sums of the singles, per alpha and per beta string
    auto pg_table = [&](const uint64_t* strs, size_t ns, int64_t*& off,
                        double*& pg) {
      int64_t* cnt = A.get<int64_t>(ns + 1);
      off = A.get<int64_t>(ns + 1);
      dp_pgcount_k<NSW><<<grid_for(ns, 256, 4 * sms), 256, 0, s>>>(
          strs, int64_t(ns), h->norb, cnt), note_launch();
      exclusive_scan<int64_t, int64_t>(cnt, off, ns, off + ns, A);
      const int64_t tot = to_host(off + ns, s);
      pg = A.get<double>(size_t(std::max<int64_t>(tot, 1)));
      dp_pg_k<NSW><<<grid_for(ns * 32, 256, 8 * sms), 256, 0, s>>>(
          I, strs, int64_t(ns), off, pg), note_launch();
    };
    int64_t *pgaoff, *pgboff;
    double *pga, *pgb;
    pg_table(ua, UA, pgaoff, pga);
    pg_table(ub, UB, pgboff, pgb);
    // signed values of the alpha doubles and of the beta L4 doubles
    double *aval, *l4val;
    {
      const int64_t na_ = to_host(aoff + UA, s), n4_ = to_host(l4off + UB, s);
      aval = A.get<double>(size_t(std::max<int64_t>(na_, 1)));
      l4val = A.get<double>(size_t(std::max<int64_t>(n4_, 1)));
      dp_dval_k<<<grid_for(size_t(na_), 256, 8 * sms), 256, 0, s>>>(
          ainfo, na_, I.G, aval), note_launch();
      dp_dval_k<<<grid_for(size_t(n4_), 256, 8 * sms), 256, 0, s>>>(
          l4info, n4_, I.G, l4val), note_launch();
    }
    DPData d{int64_t(UA), int64_t(UB), ua, ub, aoff, acol, ainfo,
             l2off, l2col, l2info, l4off, l4col, l4info,
             pgaoff, pga, pgboff, pgb, aval, l4val};
    // shared-memory plan: integrals for the singles if they fit, the longest
    // beta lists, per-warp singles tables
    int64_t l2max = 0, l4max = 0;
    {
      std::vector<int64_t> h2(UB + 1), h4(UB + 1);
      MB_CUDA(cudaMemcpyAsync(h2.data(), l2off, (UB + 1) * 8, cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaMemcpyAsync(h4.data(), l4off, (UB + 1) * 8, cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      for(size_t b = 0; b < UB; ++b) {
        l2max = std::max(l2max, h2[b + 1] - h2[b]);
        l4max = std::max(l4max, h4[b + 1] - h4[b]);
      }
    }
    const int nn = h->norb;
    // The integrals of the singles are read through L1 rather than staged in
    // shared memory: per-CTA copies would take the L1 capacity that the
    // G / V gathers need (measured: staging made the C2 fill 10% slower).
    l2max = std::min<int64_t>(l2max, 2048);
    l4max = std::min<int64_t>(l4max, 4096);
    DPShared Ls = dp_shared_layout(nn, l2max, l4max);
    if(Ls.bytes > 200 * 1024) {
      Ls = dp_shared_layout(nn, std::min<int64_t>(l2max, 512),
                            std::min<int64_t>(l4max, 1024));
    }
    MB_REQUIRE(Ls.bytes <= 220 * 1024, MACIS_B200_EINVAL,
               "norb too large for the direct-product fill");
    MB_CUDA(cudaFuncSetAttribute(dp_fill_k<NBITS, CI, VT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(Ls.bytes)));
    // shared-memory carveout: the smallest that keeps DP_CTAS CTAs resident
    // (dynamic + static shared memory + the 1 KB the SM reserves per CTA),
    // the rest is L1. The carveout is a preference that the driver maps to
    // one of a few sizes, so it is raised until the occupancy query agrees.
    int per_sm = 0;
    {
      cudaFuncAttributes fa;
      MB_CUDA(cudaFuncGetAttributes(&fa, dp_fill_k<NBITS, CI, VT>));
      const size_t per_cta = Ls.bytes + fa.sharedSizeBytes + 1024;
      int pct = int(std::min<size_t>(
          100, (DP_CTAS * per_cta * 100 + 228 * 1024 - 1) / (228 * 1024)));
      for(;;) {
        MB_CUDA(cudaFuncSetAttribute(
            dp_fill_k<NBITS, CI, VT>,
            cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, dp_fill_k<NBITS, CI, VT>, DP_THREADS, Ls.bytes));
        if(per_sm >= DP_CTAS || pct >= 100) break;
        pct = std::min(100, pct + 5);
      }
    }
    const unsigned g = unsigned(std::max(1, per_sm) * sms);
    ham_vt(h);
    NvtxRange nv_fill("macis_b200: direct-product fill");
    cudaEventRecord(ev[0], s);
    dp_fill_k<NBITS, CI, VT><<<g, DP_THREADS, Ls.bytes, s>>>(
        I, h->VT, d, Ls, hdiag, rowptr64, colind, nzval, out->diag, rowcnt, thresh,
        r0, int64_t(nbra)), note_launch();
    cudaEventRecord(ev[1], s);
    MB_CUDA(cudaGetLastError());
  } else {
    // ------------------------------------------------ general path
    GenData gd = gen_plan<NBITS>(h, bra, nbra, ket, nket, sub, r0, A);
    const unsigned gr = grid_for(nbra, HB_WARPS, size_t(sms) * 16);
    gen_count_k<NBITS><<<gr, HB_THREADS, 0, s>>>(gd, bra, nbra, rowcnt), note_launch();
    exclusive_scan<int64_t, int64_t>(rowcnt, rowptr64, nbra, rowptr64 + nbra, A);
    nnz_ub = to_host(rowptr64 + nbra, s);
    out->nnz_candidates = nnz_ub;
    MB_CUDA(dev_malloc_async(&colind, std::max<int64_t>(nnz_ub, 1) * sizeof(CI), s));
    MB_CUDA(dev_malloc_async(&nzval, std::max<int64_t>(nnz_ub, 1) * sizeof(VT), s));
    // long rows
    uint32_t* lf = A.get<uint32_t>(nbra + 1);
    uint32_t* lpos = A.get<uint32_t>(nbra + 1);
    long_flags_k<<<grid_for(nbra, 256, 8 * sms), 256, 0, s>>>(rowptr64, nbra, lf), note_launch();
    exclusive_scan<uint32_t, uint32_t>(lf, lpos, nbra, lpos + nbra, A);
    const uint32_t nl = to_host(lpos + nbra, s);
    out->long_rows = nl;
    int64_t *lrows = nullptr, *lcnt = nullptr, *loff = nullptr,
            *loff_row = nullptr;
    int64_t ltot = 0;
    std::vector<int64_t> h_lrows, h_loff;
    if(nl) {
      lrows = A.get<int64_t>(nl + 1);
      lcnt = A.get<int64_t>(nl + 1);
      loff = A.get<int64_t>(nl + 1);
      loff_row = A.get<int64_t>(nbra);
      long_list_k<<<grid_for(nbra, 256, 8 * sms), 256, 0, s>>>(
          rowptr64, nbra, lf, lpos, lrows, lcnt, loff_row), note_launch();
      exclusive_scan<int64_t, int64_t>(lcnt, loff, nl, loff + nl, A);
      ltot = to_host(loff + nl, s);
      long_rowoff_k<<<grid_for(nl, 256, 4 * sms), 256, 0, s>>>(lrows, loff, nl,
                                                              loff_row), note_launch();
      h_lrows.resize(nl);
      h_loff.resize(nl + 1);
      MB_CUDA(cudaMemcpyAsync(h_lrows.data(), lrows, nl * 8,
                              cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaMemcpyAsync(h_loff.data(), loff, (nl + 1) * 8,
                              cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
    }
    // Long rows are finished in chunks of consecutive rows whose scratch
    // (key + value, and the sort's second copy: 32 B per entry) fits in
    // what is free; short rows of the chunk are written by the same launch.
    int64_t lchunk = int64_t(0.7 * double(device_bytes_available()) / 32.0);
    lchunk = std::max<int64_t>(lchunk, int64_t(1) << 20);
    constexpr int gen_dyn = HB_WARPS * 256;
    MB_CUDA(cudaFuncSetAttribute(gen_fill_k<NBITS, CI, VT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 gen_dyn));
    float fill_ms_tot = 0.f;
    int64_t la = 0;  // next long row (list index)
    int64_t row_a = 0;
    do {
      int64_t lb = la;  // long rows [la, lb) in this chunk
      while(lb < int64_t(nl) && (lb == la || h_loff[lb + 1] - h_loff[la] <= lchunk))
        ++lb;
      const int64_t row_b = lb < int64_t(nl) ? h_lrows[lb] : int64_t(nbra);
      const int64_t cbase = nl ? h_loff[la] : 0;
      const int64_t centries = nl ? h_loff[lb] - cbase : 0;
      Arena C(s);
      uint64_t* lkey = C.get<uint64_t>(centries + 1);
      double* lval = C.get<double>(centries + 1);
      cudaEventRecord(ev[0], s);
      gen_fill_k<NBITS, CI, VT><<<gr, HB_THREADS, gen_dyn, s>>>(
          I, gd, bra, row_a, row_b, hdiag, rowptr64, loff_row, cbase, lpos,
          lkey, lval, colind, nzval, out->diag, rowcnt, thresh), note_launch();
      cudaEventRecord(ev[1], s);
      MB_CUDA(cudaGetLastError());
      MB_CUDA(cudaEventSynchronize(ev[1]));
      float ms = 0.f;
      MB_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      fill_ms_tot += ms;
      if(lb > la) {
        uint64_t* lk2 = C.get<uint64_t>(centries + 1);
        double* lv2 = C.get<double>(centries + 1);
        radix_sort<1, double>(lkey, lval, lk2, lv2, size_t(centries), C);
        long_rows_write_k<CI, VT><<<grid_for(size_t(lb - la) * 32, 256, 8 * sms),
                                    256, 0, s>>>(
            lrows + la, lb - la, loff + la, cbase, lkey, lval, rowptr64,
            colind, nzval, out->diag, rowcnt, thresh), note_launch();
        MB_CUDA(cudaGetLastError());
      }
      la = lb;
      row_a = row_b;
    } while(row_a < int64_t(nbra));
    out->fill_ms = fill_ms_tot;
    general_fill_timed = true;
  }

  // ------------------------------------------- exact row pointer + compaction
  int64_t* newptr = A.get<int64_t>(nbra + 1);
  exclusive_scan<int64_t, int64_t>(rowcnt, newptr, nbra, newptr + nbra, A);
  const int64_t nnz = to_host(newptr + nbra, s);
  out->nnz = nnz;
  if(sizeof(CI) == 4)
    MB_REQUIRE(nnz <= int32_index_limit(), MACIS_B200_ECAPACITY,
               "nnz exceeds the int32 index range; use 64-bit indices");
  if(nnz != nnz_ub) {
    CI* ci2 = nullptr;
    VT* nz2 = nullptr;
    MB_CUDA(dev_malloc_async(&ci2, std::max<int64_t>(nnz, 1) * sizeof(CI), s));
    MB_CUDA(dev_malloc_async(&nz2, std::max<int64_t>(nnz, 1) * sizeof(VT), s));
    if(direct)
      compact_marked_k<CI, VT><<<grid_for(nbra * 32, 256, 16 * sms), 256, 0, s>>>(
          rowptr64, newptr, nbra, colind, nzval, ci2, nz2), note_launch();
    else
      compact_rows_k<CI, VT><<<grid_for(nbra * 32, 256, 16 * sms), 256, 0, s>>>(
          rowptr64, newptr, nbra, colind, nzval, ci2, nz2), note_launch();
    cudaFreeAsync(colind, s);
    cudaFreeAsync(nzval, s);
    colind = ci2;
    nzval = nz2;
  }
  MB_CUDA(dev_malloc_async(&out->rowptr, (nbra + 1) * sizeof(CI), s));
  rowptr_cast_k<CI><<<grid_for(nbra + 1, 256, 8 * sms), 256, 0, s>>>(
      newptr, nbra + 1, static_cast<CI*>(out->rowptr)), note_launch();
  out->colind = colind;
  out->nzval = nzval;
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(s));
  if(!general_fill_timed) cudaEventElapsedTime(&out->fill_ms, ev[0], ev[1]);
}

macis_b200_csr* build_csr_device(macis_b200_ham* h, const uint64_t* bra,
                                 size_t nbra, const uint64_t* ket, size_t nket,
                                 double thresh, int idx_bytes, int val_bytes) {
  NvtxRange nv("macis_b200: CSR build");
  MB_REQUIRE(idx_bytes == 4 || idx_bytes == 8, MACIS_B200_EINVAL,
             "Unsupported index_t");
  MB_REQUIRE(val_bytes == 4 || val_bytes == 8, MACIS_B200_EINVAL,
             "val_bytes must be 4 or 8");
  auto* out = new macis_b200_csr;
  out->idx_bytes = idx_bytes;
  out->val_bytes = val_bytes;
  out->device = h->device;
  MB_CUDA(cudaStreamCreateWithFlags(&out->stream, cudaStreamNonBlocking));
  out->own_stream = true;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, h->stream);
  try {
#define MB_BUILD(NB)                                                          \
  if(idx_bytes == 4 && val_bytes == 8)                                        \
    build_impl<NB, int32_t, double>(h, bra, nbra, ket, nket, thresh, out);    \
  else if(idx_bytes == 4)                                                     \
    build_impl<NB, int32_t, float>(h, bra, nbra, ket, nket, thresh, out);     \
  else if(val_bytes == 8)                                                     \
    build_impl<NB, int64_t, double>(h, bra, nbra, ket, nket, thresh, out);    \
  else                                                                        \
    build_impl<NB, int64_t, float>(h, bra, nbra, ket, nket, thresh, out);
    if(h->nbits == 64) {
      MB_BUILD(64)
    } else if(h->nbits == 128) {
      MB_BUILD(128)
    } else {
      MB_BUILD(256)
    }
#undef MB_BUILD
  } catch(...) {
    cudaStreamSynchronize(h->stream);
    if(out->rowptr) cudaFreeAsync(out->rowptr, h->stream);
    if(out->colind) cudaFreeAsync(out->colind, h->stream);
    if(out->nzval) cudaFreeAsync(out->nzval, h->stream);
    if(out->diag) cudaFreeAsync(out->diag, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(out->stream);
    delete out;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&out->build_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return out;
}

}  // namespace mb

// ------------------------------------------------ matrix-free H x
// The operator keeps its own stream and a copy of the generator's integral
// pointers: the generator must outlive every product, but destroying the
// operator never touches it.
struct macis_b200_hop {
  mb::Ints I{};
  int nbits = 64;
  cudaStream_t stream = nullptr;
  int64_t n = 0;
  double thresh = 0.0;
  bool mixed = false;
  uint64_t* dets = nullptr;  // device copy of the determinant list
  double* diag = nullptr;    // H_ii
  mb::Arena* A = nullptr;    // owns dets, diag and the enumeration tables
  mb::GenData g{};
};

namespace mb {

// y = alpha H x + beta y, one warp per row: the candidates of the general
// build's enumeration (gen_enumerate), each element evaluated, thresholded
// as in the build and accumulated into the row sum (no storage). mixed:
// off-diagonal elements rounded to FP32 first, as in an FP32-valued CSR.
template <int NBITS>
__global__ void __launch_bounds__(HB_THREADS)
    gen_apply_k(Ints I, GenData g, const uint64_t* dets, int64_t n,
                const double* __restrict__ hdiag, double thresh, int mixed,
                double alpha, const double* __restrict__ x, double beta,
                double* __restrict__ y) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  extern __shared__ __align__(16) uint8_t gen_ov[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t nwarp = int64_t(gridDim.x) * HB_WARPS;
  for(int64_t row = int64_t(blockIdx.x) * HB_WARPS + wid; row < n;
      row += nwarp) {
    const int32_t rg = g.rowgroup[row];
    double acc = 0.0;
    if(rg >= 0) {
      const uint64_t* bd = dets + row * D::NW;
      const Spin<NSW> ba = D::alpha(bd), bb = D::beta(bd);
      const double hd = hdiag[row];
      gen_enumerate<NSW>(g, rg, ba, bb, gen_ov + wid * 256,
                         [&](bool act, int64_t m, int32_t kg, int pa, int pb) {
        if(act) {
          const uint32_t col = g.sidx[m];
          double h;
          if(pa == 0 && pb == 0)
            h = hd;
          else
            h = me_generic(I, ba, bb, ld_spin<NSW>(g.kalpha, kg),
                           ld_spin<NSW>(g.sbeta, m));
          if(fabs(h) > thresh) {
            if(mixed && int64_t(col) != row) h = double(float(h));
            acc += h * x[col];
          }
        }
      });
#pragma unroll
      for(int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    }
    if(lane == 0) y[row] = alpha * acc + (beta != 0.0 ? beta * y[row] : 0.0);
  }
}

macis_b200_hop* hop_create(macis_b200_ham* h, const uint64_t* dets, size_t n,
                           double thresh, bool mixed, bool device_ptrs) {
  MB_REQUIRE(n > 0, MACIS_B200_EINVAL, "empty determinant list");
  MB_REQUIRE(n < (size_t(1) << 31), MACIS_B200_ECAPACITY,
             "matrix-free H needs < 2^31 determinants");
  const size_t nw = size_t(h->nbits / 64);
  const int sms = num_sms();
  const Ints I = h->ints();
  auto* op = new macis_b200_hop;
  op->I = I;
  op->nbits = h->nbits;
  op->n = int64_t(n);
  op->thresh = thresh;
  op->mixed = mixed;
  if(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) !=
     cudaSuccess) {
    delete op;
    MB_REQUIRE(false, MACIS_B200_ECUDA, "stream creation failed");
  }
  cudaStream_t s = op->stream;
  try {
    op->A = new Arena(s);
    op->dets = op->A->get<uint64_t>(n * nw);
    MB_CUDA(cudaMemcpyAsync(op->dets, dets, n * nw * 8,
                            device_ptrs ? cudaMemcpyDeviceToDevice
                                        : cudaMemcpyHostToDevice, s));
    op->diag = op->A->get<double>(n);
#define MB_HOP_PLAN(NB)                                                     \
  hdiag_k<NB><<<grid_for(n, 256, 8 * sms), 256, 0, s>>>(I, op->dets, n,     \
                                                        op->diag),          \
      note_launch();                                                        \
  op->g = gen_plan<NB>(h, op->dets, n, op->dets, n, true, 0, *op->A);
    if(h->nbits == 64) {
      MB_HOP_PLAN(64)
    } else if(h->nbits == 128) {
      MB_HOP_PLAN(128)
    } else {
      MB_HOP_PLAN(256)
    }
#undef MB_HOP_PLAN
    MB_CUDA(cudaStreamSynchronize(s));
  } catch(...) {
    cudaStreamSynchronize(s);
    delete op->A;
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    delete op;
    throw;
  }
  return op;
}

void hop_apply(const macis_b200_hop* op, double alpha, const double* x,
               double beta, double* y) {
  cudaStream_t s = op->stream;
  const unsigned gr = grid_for(size_t(op->n), HB_WARPS, size_t(num_sms()) * 16);
  constexpr int dyn = HB_WARPS * 256;
  const Ints I = op->I;
#define MB_HOP_APPLY(NB)                                                     \
  gen_apply_k<NB><<<gr, HB_THREADS, dyn, s>>>(I, op->g, op->dets, op->n,     \
                                              op->diag, op->thresh,          \
                                              op->mixed ? 1 : 0, alpha, x,   \
                                              beta, y),                      \
      note_launch();
  if(op->nbits == 64) {
    MB_HOP_APPLY(64)
  } else if(op->nbits == 128) {
    MB_HOP_APPLY(128)
  } else {
    MB_HOP_APPLY(256)
  }
#undef MB_HOP_APPLY
  MB_CUDA(cudaGetLastError());
}

void hop_destroy(macis_b200_hop* op) {
  if(!op) return;
  cudaStreamSynchronize(op->stream);
  delete op->A;
  cudaStreamSynchronize(op->stream);
  cudaStreamDestroy(op->stream);
  delete op;
}

int64_t hop_size(const macis_b200_hop* op) { return op->n; }
const double* hop_diag(const macis_b200_hop* op) { return op->diag; }
cudaStream_t hop_stream(const macis_b200_hop* op) { return op->stream; }

}  // namespace mb

// ------------------------------------------------ 1- and 2-RDMs
namespace mb {

__device__ __forceinline__ void rdm_add(double* a, size_t i, double v) {
  atomicAdd(a + i, v);
}

// Contributions of one (bra, ket) pair: rdm_contributions and its parts
// (include/macis/util/rdms.hpp:15-131), dispatched in the same order (the
// two-body branches only when trdm is given). ordm(p,q) = ordm[p + q n],
// trdm(p,q,r,s) = trdm[p + n (q + n (r + n s))].
template <int NSW>
__device__ void rdm_pair(Spin<NSW> ba, Spin<NSW> bb, Spin<NSW> ka,
                         Spin<NSW> kb, double val, int n, double* ordm,
                         double* trdm) {
  const int ca = sp_popc(ba ^ ka), cb = sp_popc(bb ^ kb);
  if(ca + cb > 4) return;
  auto t4 = [&](int p, int q, int r, int s, double v) {
    rdm_add(trdm, size_t(p) + size_t(n) * (q + size_t(n) * (r + size_t(n) * s)),
            v);
  };
  if((ca == 4 || cb == 4) && trdm) {  // rdm_contributions_4, :15-25
    const uint32_t e = ca == 4 ? double_ex(ba, ka) : double_ex(bb, kb);
    const int o1 = ex_o1(e), v1 = ex_v1(e), o2 = ex_o2(e), v2 = ex_v2(e);
    const double v = val * (ex_sgn(e) * 0.5);
    t4(v1, o1, v2, o2, v);
    t4(v2, o1, v1, o2, -v);
    t4(v1, o2, v2, o1, -v);
    t4(v2, o2, v1, o1, v);
  } else if(ca == 2 && cb == 2 && trdm) {  // rdm_contributions_22, :27-41
    const uint32_t ea = single_ex(ba, ka), eb = single_ex(bb, kb);
    const double v = val * (ex_sgn(ea) * ex_sgn(eb) * 0.5);
    t4(ex_v1(ea), ex_o1(ea), ex_v1(eb), ex_o1(eb), v);
    t4(ex_v1(eb), ex_o1(eb), ex_v1(ea), ex_o1(ea), v);
  } else if(ca == 2 || cb == 2) {  // rdm_contributions_2, :43-66
    const bool a = ca == 2;
    const uint32_t e = a ? single_ex(ba, ka) : single_ex(bb, kb);
    const Spin<NSW> occ_s = a ? ba : bb, occ_o = a ? bb : ba;
    const int o1 = ex_o1(e), v1 = ex_v1(e);
    const double sg = ex_sgn(e);
    rdm_add(ordm, size_t(v1) + size_t(n) * o1, sg * val);
    if(trdm) {
      const double v = val * (sg * 0.5);
      for(Spin<NSW> s = occ_s; sp_popc(s);) {
        const int p = sp_lowest(s);
        s = sp_flip(s, p);
        t4(v1, o1, p, p, v);
        t4(p, p, v1, o1, v);
        t4(v1, p, p, o1, -v);
        t4(p, o1, v1, p, -v);
      }
      for(Spin<NSW> s = occ_o; sp_popc(s);) {
        const int p = sp_lowest(s);
        s = sp_flip(s, p);
        t4(v1, o1, p, p, v);
        t4(p, p, v1, o1, v);
      }
    }
  } else {  // rdm_contributions_diag, :68-99
    for(Spin<NSW> s = ba; sp_popc(s);) {
      const int p = sp_lowest(s);
      s = sp_flip(s, p);
      rdm_add(ordm, size_t(p) * (n + 1), val);
    }
    for(Spin<NSW> s = bb; sp_popc(s);) {
      const int p = sp_lowest(s);
      s = sp_flip(s, p);
      rdm_add(ordm, size_t(p) * (n + 1), val);
    }
    if(trdm) {
      const double v = val * 0.5;
      for(int spin = 0; spin < 2; ++spin) {
        const Spin<NSW> o = spin ? bb : ba;
        for(Spin<NSW> sq = o; sp_popc(sq);) {
          const int q = sp_lowest(sq);
          sq = sp_flip(sq, q);
          for(Spin<NSW> sp = o; sp_popc(sp);) {
            const int p = sp_lowest(sp);
            sp = sp_flip(sp, p);
            t4(p, p, q, q, v);
            t4(p, q, p, q, -v);
          }
        }
      }
      for(Spin<NSW> sq = bb; sp_popc(sq);) {
        const int q = sp_lowest(sq);
        sq = sp_flip(sq, q);
        for(Spin<NSW> sp = ba; sp_popc(sp);) {
          const int p = sp_lowest(sp);
          sp = sp_flip(sp, p);
          t4(p, p, q, q, v);
          t4(q, q, p, p, v);
        }
      }
    }
  }
}

// form_rdms (double_loop.hpp:117-165) over one determinant list: every
// (bra, ket) pair within four spin-orbital differences with |C_i C_j| >
// 1e-16 adds its contributions. One warp per bra row; the pairs come from
// the general build's enumeration; sums are atomic (order not fixed).
template <int NBITS>
__global__ void __launch_bounds__(HB_THREADS)
    rdm_k(GenData g, const uint64_t* dets, int64_t n, const double* C,
          int norb, double* ordm, double* trdm) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  extern __shared__ __align__(16) uint8_t gen_ov[];
  const int wid = threadIdx.x >> 5;
  const int64_t nwarp = int64_t(gridDim.x) * HB_WARPS;
  for(int64_t row = int64_t(blockIdx.x) * HB_WARPS + wid; row < n;
      row += nwarp) {
    const int32_t rg = g.rowgroup[row];
    if(rg < 0) continue;
    const uint64_t* bd = dets + row * D::NW;
    const Spin<NSW> ba = D::alpha(bd), bb = D::beta(bd);
    const double ci = C[row];
    gen_enumerate<NSW>(g, rg, ba, bb, gen_ov + wid * 256,
                       [&](bool act, int64_t m, int32_t kg, int, int) {
      if(!act) return;
      const double val = ci * C[g.sidx[m]];
      if(!(fabs(val) > 1e-16)) return;
      rdm_pair<NSW>(ba, bb, ld_spin<NSW>(g.kalpha, kg),
                    ld_spin<NSW>(g.sbeta, m), val, norb, ordm, trdm);
    });
  }
}

// ordm (n^2) and trdm (n^4, may be null) are device arrays the results are
// added to; dets and C device arrays of length n.
void form_rdms_device(macis_b200_ham* h, const uint64_t* dets, size_t n,
                      const double* C, double* ordm, double* trdm) {
  if(n == 0) return;
  MB_REQUIRE(n < (size_t(1) << 31), MACIS_B200_ECAPACITY,
             "RDMs need < 2^31 determinants");
  cudaStream_t s = h->stream;
  Arena A(s);
  const unsigned gr = grid_for(n, HB_WARPS, size_t(num_sms()) * 16);
  constexpr int dyn = HB_WARPS * 256;
#define MB_RDM(NB)                                                          \
  {                                                                         \
    const GenData g = gen_plan<NB>(h, dets, n, dets, n, true, 0, A);        \
    rdm_k<NB><<<gr, HB_THREADS, dyn, s>>>(g, dets, int64_t(n), C, h->norb,  \
                                         ordm, trdm),                       \
        note_launch();                                                      \
  }
  if(h->nbits == 64) {
    MB_RDM(64)
  } else if(h->nbits == 128) {
    MB_RDM(128)
  } else {
    MB_RDM(256)
  }
#undef MB_RDM
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace mb

// ASCI search on the GPU, replacing macis::asci_search at MPI world size 1
// (include/macis/asci/determinant_search.hpp:395-663):
//
//  1. per core det: occupied/virtual lists, orbital energies
//     (single_orbital_ens, fast_diagonals.hpp:34-53) and H_ii
//  2. contributions (determinant_contributions.hpp:26-160) in two passes --
//     a count pass over "units" (singles of a spin, or one (i,a) outer pair
//     of a double loop) and a fill pass writing every (det, rv) record at its
//     exact position -- so the raw list is the reference push_back order
//  3. stable radix sort by determinant and a sequential per-segment sum:
//     duplicates are added in generation order (sort_and_accumulate_asci_pairs,
//     determinant_sort.hpp:40-83)
//  4. drop core dets and zero scores (keep_only_largest_copy_asci_pairs +
//     partition, determinant_sort.hpp:86-120, determinant_search.hpp:528-544)
//  5. top-k by |rv| with an MSD radix select; ties at the k-th score are
//     resolved towards smaller determinants (determinant_search.hpp:622-626
//     leaves them unspecified)
//
// When the raw contributions do not fit in HBM at once, the candidate
// determinants are split into ranges by a hash of the determinant; each
// range is generated, sorted and accumulated on its own (its sums are
// complete) and merged into a running top-k.
#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "internal.hpp"
#include "mlp.cuh"
#include "primitives.cuh"

namespace mb {

constexpr int MAXORB = 128;

struct CoreData {
  int n;
  const uint64_t* dets;  // ncdets x NW
  const double* C;
  size_t ncdets;
  uint8_t* occ;   // ncdets x 2 x MAXORB  (alpha, beta) ascending occupied
  uint8_t* vir;   // ncdets x 2 x MAXORB  ascending virtual (below n)
  uint8_t* cnt;   // ncdets x 4: nocc_a, nocc_b, nvir_a, nvir_b
  double* eps;    // ncdets x 2 x n
  double* hd;     // ncdets
  int64_t* uoff;  // ncdets+1 unit offsets
  int32_t* udet;  // per unit: the core det it belongs to
  const double* pairmax;  // 2 n^2 outer-pair integral bounds (screening)
  const double* VT;       // V with its index pairs swapped (ham_vt): the
                          // opposite-spin elements of one outer pair are a
                          // contiguous row
};

// udet[u] = c for the units u of core det c (one warp per det): one load
// per unit instead of a binary search over uoff.
__global__ void unit_owner_fill_k(const int64_t* uoff, size_t ncdets,
                                  int32_t* udet) {
  const int lane = threadIdx.x & 31;
  const size_t nw = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t c = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      c < ncdets; c += nw)
    for(int64_t u = uoff[c] + lane; u < uoff[c + 1]; u += 32)
      udet[u] = int32_t(c);
}

// Outer-pair integral bounds (macis_b200_ham::pairmax). G rows are
// contiguous (warp per pair); V is read with one thread per pair so that a
// warp's loads are consecutive.
__global__ void pairmax_g_k(const double* G, int n, double* out) {
  const int lane = threadIdx.x & 31;
  const size_t n2 = size_t(n) * n;
  for(size_t p = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      p < n2; p += size_t(gridDim.x) * (blockDim.x >> 5)) {
    double m = 0.0;
    for(size_t q = lane; q < n2; q += 32) m = fmax(m, fabs(G[p * n2 + q]));
    for(int o = 16; o > 0; o >>= 1)
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if(lane == 0) out[p] = m;
  }
}
__global__ void pairmax_v_k(const double* V, int n, double* out) {
  const size_t n2 = size_t(n) * n;
  for(size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n2;
      p += size_t(gridDim.x) * blockDim.x) {
    double m = 0.0;
    for(size_t q = 0; q < n2; ++q) m = fmax(m, fabs(V[p + q * n2]));
    out[p] = m;
  }
}

// Per core det precompute; one warp per det (bitset_to_occ_vir,
// sd_operations.hpp:82-97; single_orbital_ens; matrix_element diag).
template <int NBITS>
__global__ void core_prep_k(Ints I, CoreData cd, int just_singles,
                            int64_t* units) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  const int lane = threadIdx.x & 31;
  const int n = cd.n;
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t c = size_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
      c < cd.ncdets; c += nwarp) {
    const uint64_t* d = cd.dets + c * D::NW;
    const Spin<NSW> sp[2] = {D::alpha(d), D::beta(d)};
    int no[2], nv[2];
    for(int s = 0; s < 2; ++s) {
      // lists: lane 0 writes sequentially (n <= 128)
      if(lane == 0) {
        int a = 0, v = 0;
        for(int i = 0; i < n; ++i) {
          if(sp_test(sp[s], i))
            cd.occ[(c * 2 + s) * MAXORB + a++] = uint8_t(i);
          else
            cd.vir[(c * 2 + s) * MAXORB + v++] = uint8_t(i);
        }
      }
      no[s] = sp_popc(sp[s]);
      nv[s] = n - no[s];
    }
    if(lane == 0) {
      cd.cnt[c * 4 + 0] = uint8_t(no[0]);
      cd.cnt[c * 4 + 1] = uint8_t(no[1]);
      cd.cnt[c * 4 + 2] = uint8_t(nv[0]);
      cd.cnt[c * 4 + 3] = uint8_t(nv[1]);
      cd.hd[c] = me_diag(I, sp[0], sp[1]);
      const int64_t u = just_singles
                            ? 2
                            : 2 + int64_t(no[0]) * nv[0] + int64_t(no[1]) * nv[1] +
                                  int64_t(no[0]) * nv[0];
      units[c] = u;
    }
    // eps_same for spin s: ss = sp[s], os = sp[1-s]
    for(int s = 0; s < 2; ++s)
      for(int i = lane; i < n; i += 32) {
        double e = __ldg(I.T + size_t(i) * (n + 1));
        for(Spin<NSW> q = sp[s]; sp_popc(q);) {
          const int p = sp_lowest(q);
          q = sp_flip(q, p);
          e += __ldg(I.G2_red + i + size_t(p) * n) + __ldg(I.G2_red + p + size_t(i) * n);
        }
        e -= __ldg(I.G2_red + size_t(i) * (n + 1));
        for(Spin<NSW> q = sp[1 - s]; sp_popc(q);) {
          const int p = sp_lowest(q);
          q = sp_flip(q, p);
          e += __ldg(I.V2_red + i + size_t(p) * n);
        }
        cd.eps[(c * 2 + s) * n + i] = e;
      }
  }
}

template <int NBITS>
__device__ __forceinline__ void det_flip(uint64_t* d, int spin, int orb) {
  if constexpr(NBITS == 64) {
    d[0] ^= 1ull << (orb + 32 * spin);
  } else if constexpr(NBITS == 128) {
    d[spin] ^= 1ull << orb;
  } else {
    d[2 * spin + (orb >> 6)] ^= 1ull << (orb & 63);
  }
}

// Candidate ranges of a partitioned search: the alpha string of a candidate
// determinant is hashed to one of ASCI_BINS bins, and a range is an interval
// of bins [blo, bhi) chosen from the measured bin loads. Every contribution
// to one determinant falls into the same range, and the units whose alpha
// string is fixed (beta singles, beta same-spin doubles, opposite-spin
// doubles for one outer alpha pair) fall into one bin as a whole.
constexpr uint32_t ASCI_BINS = 4096;
// Second-level split of one oversized bin: a hash of the beta string.
template <int NSW>
__device__ __forceinline__ uint32_t beta_sub(const Spin<NSW>& b,
                                             uint32_t nsub) {
  uint64_t h = 0xD1B54A32D192ED03ull;
#pragma unroll
  for(int j = 0; j < NSW; ++j) {
    h ^= b.w[j];
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
    h ^= h >> 31;
  }
  return uint32_t((uint64_t(uint32_t(h >> 32)) * nsub) >> 32);
}
template <int NSW>
__device__ __forceinline__ uint32_t alpha_bin(const Spin<NSW>& a) {
  uint64_t h = 0x9E3779B97F4A7C15ull;
#pragma unroll
  for(int j = 0; j < NSW; ++j) {
    h ^= a.w[j];
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
    h ^= h >> 31;
  }
  return uint32_t(h >> 52);  // 12 bits: ASCI_BINS
}

// Sort group of a candidate record of a range: groups are runs of the
// range's alpha-string bins (gtab: bin -> group), so that equal
// determinants share a group.
template <int NBITS>
struct BinGroup {
  const uint8_t* gtab;  // ASCI_BINS entries
  __device__ __forceinline__ unsigned operator()(
      const Key<DetTraits<NBITS>::NW>& k) const {
    using D = DetTraits<NBITS>;
    return gtab[alpha_bin<D::NSW>(D::alpha(k.w))];
  }
};

// Alpha lists of a partitioned search. The bins of the contributions of an
// alpha same-spin double unit (kind 2) depend only on the core det's alpha
// string, and so does their threshold test (|G| against the tolerance):
// for a distinct alpha string u and outer pair k = ii * nvA + aa, the inner
// indices q of the kept contributions are listed once per search, grouped
// by the candidate range their bin falls into (ascending q inside a group).
// A range's count pass then reads each unit's count from the lists instead
// of evaluating the bins of all its contributions, and its fill pass
// generates the listed contributions only. The lists cover the alpha
// strings shared by the most core dets, as many as fit the memory budget
// (lidx >= 0); the alpha doubles of the others keep the per-contribution
// test. The bins of the units with a fixed alpha string (kinds 1, 3, 4) are
// tabulated for every distinct alpha string. Used for the ranges that are
// not split by beta string (group g >= 0).
struct AlphaLists {
  const int32_t* aidx = nullptr;  // per core det: its alpha string
  const int32_t* lidx = nullptr;  // per alpha string: its list block, or -1
  int NK = 0;                     // nA * nvA outer pairs per alpha string
  int G = 0;                      // groups: the unsplit ranges
  const uint16_t* abin = nullptr;  // per alpha string: its bin
  const uint16_t* kbin = nullptr;  // per (u, k): bin after the outer alpha
                                   // excitation (opposite-spin units)
  const int64_t* base = nullptr;   // per (list block, k): first list entry
  const uint16_t* rel = nullptr;   // per (list block, k): G + 1 group starts
  const uint16_t* q = nullptr;     // inner indices, by group
  int g = -1;                      // group of the range, -1: not used
};

// String ranks. The candidate determinants of a search are the core dets'
// alpha strings, their singles and doubles, combined with beta strings of
// the same kinds. With every distinct candidate string of a spin replaced
// by its rank in the sorted list of those strings, a candidate determinant
// is one 64-bit key, (beta rank << bits_a) | alpha rank, that sorts in the
// same order as the determinant's bitset: the digit passes of the candidate
// sort cover bits_a + bits_b bits instead of the 2 x norb varying bits of
// the determinant, over 16-byte instead of 24- or 40-byte records. Per
// distinct core string u of a spin the table R holds the ranks of its
// M = 1 + N1 + N2 candidates: u itself, its N1 singles (index ii * nv + aa,
// occupied ii -> virtual aa) and its N2 doubles (row ii * nv + aa, then the
// inner index q of the double loops of unit_run).
struct SpinRanks {
  const uint32_t* R = nullptr;
  const int32_t* idx = nullptr;  // per core det: its string
  int64_t M = 0, N1 = 0;
};
struct RankTables {
  SpinRanks a, b;
  int bits_a = 0;
  const uint64_t* La = nullptr;  // distinct candidate alpha strings (NSW words)
  const uint64_t* Lb = nullptr;
  const uint16_t* bin_a = nullptr;  // per alpha rank: its bin
};
// First double of row ii * nv + aa among the doubles of a string with ne
// electrons and nv virtuals (rows before it hold (ne-1-ii')(nv-1-aa') each).
__device__ __forceinline__ int64_t double_row_base(int ii, int aa, int ne,
                                                   int nv) {
  const int64_t A = int64_t(ii) * (ne - 1) - int64_t(ii) * (ii - 1) / 2;
  const int64_t T = int64_t(nv) * (nv - 1) / 2;
  const int64_t B = int64_t(aa) * (nv - 1) - int64_t(aa) * (aa - 1) / 2;
  return A * T + int64_t(ne - 1 - ii) * B;
}

// The candidate strings of the distinct core strings, one thread per
// (string, candidate): written with their index, for the rank sort.
template <int NSW>
__global__ void cand_strings_k(const uint64_t* words, const uint8_t* occ,
                               const uint8_t* vir, size_t nu, int ne, int nv,
                               int64_t M, int64_t N1, const int64_t* dbase,
                               int nrows, uint64_t* cand, uint32_t* idx) {
  const size_t tot = nu * size_t(M);
  for(size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < tot;
      e += size_t(gridDim.x) * blockDim.x) {
    const size_t u = e / size_t(M);
    const int64_t r = int64_t(e - u * size_t(M));
    Spin<NSW> st;
#pragma unroll
    for(int j = 0; j < NSW; ++j) st.w[j] = words[u * NSW + j];
    const uint8_t* o = occ + u * MAXORB;
    const uint8_t* v = vir + u * MAXORB;
    if(r >= 1 && r <= N1) {
      const int t = int(r - 1), ii = t / nv, aa = t - ii * nv;
      st = sp_flip(sp_flip(st, int(o[ii])), int(v[aa]));
    } else if(r > N1) {
      const int64_t d = r - 1 - N1;
      int lo = 0, hi = nrows;  // last row whose first double is <= d
      while(hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if(dbase[mid] <= d) lo = mid; else hi = mid;
      }
      const int ii = lo / nv, aa = lo - ii * nv;
      const int span = nv - 1 - aa;
      const int q = int(d - dbase[lo]);
      const int jj = ii + 1 + q / span, bb = aa + 1 + q % span;
      st = sp_flip(sp_flip(sp_flip(sp_flip(st, int(o[ii])), int(o[jj])),
                           int(v[aa])), int(v[bb]));
    }
#pragma unroll
    for(int j = 0; j < NSW; ++j) cand[e * NSW + j] = st.w[j];
    idx[e] = uint32_t(e);
  }
}
// Rank of every candidate (sorted position p holds candidate idx[p]) and
// the distinct strings in rank order.
template <int NSW>
__global__ void rank_scatter_k(const uint64_t* cand, const uint32_t* idx,
                               const uint32_t* f, const uint32_t* fx, size_t n,
                               uint32_t* R, uint64_t* L) {
  for(size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
      p += size_t(gridDim.x) * blockDim.x) {
    const uint32_t r = fx[p] + f[p] - 1;
    R[idx[p]] = r;
    if(f[p]) {
#pragma unroll
      for(int j = 0; j < NSW; ++j) L[size_t(r) * NSW + j] = cand[p * NSW + j];
    }
  }
}
template <int NSW>
__global__ void string_bins_k(const uint64_t* L, size_t n, uint16_t* bin) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    Spin<NSW> st;
#pragma unroll
    for(int j = 0; j < NSW; ++j) st.w[j] = L[i * NSW + j];
    bin[i] = uint16_t(alpha_bin<NSW>(st));
  }
}
// Ranked keys back to determinants.
template <int NBITS>
__global__ void unrank_k(const uint64_t* rk, size_t n, RankTables rt,
                         uint64_t* dets) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  const uint64_t ma = (uint64_t(1) << rt.bits_a) - 1;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t k = rk[i];
    const size_t ra = size_t(k & ma), rb = size_t(k >> rt.bits_a);
    Spin<NSW> a, b;
#pragma unroll
    for(int j = 0; j < NSW; ++j) {
      a.w[j] = rt.La[ra * NSW + j];
      b.w[j] = rt.Lb[rb * NSW + j];
    }
    D::make(dets + i * D::NW, a, b);
  }
}
// Sort group of a ranked key: the group of its alpha string's bin.
struct RankBinGroup {
  const uint8_t* gtab;
  const uint16_t* bin_a;
  uint64_t mask_a;
  __device__ __forceinline__ unsigned operator()(const Key<1>& k) const {
    return gtab[bin_a[k.w[0] & mask_a]];
  }
};

#define G2R(p, q) __ldg(I.G2_red + (p) + size_t(q) * n)
#define V2R(p, q) __ldg(I.V2_red + (p) + size_t(q) * n)

// A unit of core det c: t = 0 / 1 alpha / beta singles; then the (ii, aa)
// outer pairs of the same-spin alpha doubles, of the same-spin beta doubles
// and of the opposite-spin doubles (alpha outer, beta inner).
struct UnitDesc {
  int kind, ii, aa;
  int64_t ninner;
};
__device__ __forceinline__ UnitDesc decode_unit(int nA, int nB, int nvA,
                                                int nvB, int64_t t) {
  UnitDesc d{0, 0, 0, 0};
  if(t == 0) {
    d.kind = 0;
    d.ninner = int64_t(nA) * nvA;
  } else if(t == 1) {
    d.kind = 1;
    d.ninner = int64_t(nB) * nvB;
  } else if(t < 2 + int64_t(nA) * nvA) {
    d.kind = 2;
    d.ii = int((t - 2) / nvA);
    d.aa = int((t - 2) % nvA);
    d.ninner = int64_t(nA - 1 - d.ii) * (nvA - 1 - d.aa);
  } else if(t < 2 + int64_t(nA) * nvA + int64_t(nB) * nvB) {
    d.kind = 3;
    const int64_t u = t - 2 - int64_t(nA) * nvA;
    d.ii = int(u / nvB);
    d.aa = int(u % nvB);
    d.ninner = int64_t(nB - 1 - d.ii) * (nvB - 1 - d.aa);
  } else {
    d.kind = 4;
    const int64_t u = t - 2 - int64_t(nA) * nvA - int64_t(nB) * nvB;
    d.ii = int(u / nvA);
    d.aa = int(u % nvA);
    d.ninner = int64_t(nB) * nvB;
  }
  return d;
}

// One unit of contributions; MODE 0 counts, MODE 1 writes determinants,
// MODE 2 writes ranked keys (RankTables). Warp-synchronous.
// q / d for 0 <= q < 2^14 and 1 <= d <= 128 from a float product with rd =
// 1 / d: (q + 0.5) / d is at least 0.5 / d away from an integer, far above
// the float rounding error (< 2^-22 q / d), so truncation gives the quotient
// without a 64-bit integer division per contribution.
__device__ __forceinline__ int small_div(int64_t q, float rd) {
  return int((float(q) + 0.5f) * rd);
}

template <int NBITS, int MODE>
__device__ void unit_run(const Ints& I, const CoreData& cd, size_t c, int64_t t,
                         double E0, double tol, int64_t* count_out,
                         int64_t out0, uint64_t* keys, double* rv,
                         float* umax, uint32_t blo, uint32_t bhi,
                         uint32_t nsub, uint32_t sub,
                         unsigned long long* hist, const AlphaLists& al,
                         const RankTables& rt) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  const int lane = threadIdx.x & 31;
  const int n = cd.n;
  const int nA = cd.cnt[c * 4], nB = cd.cnt[c * 4 + 1];
  const int nvA = cd.cnt[c * 4 + 2], nvB = cd.cnt[c * 4 + 3];
  const uint8_t* occA = cd.occ + (c * 2) * MAXORB;
  const uint8_t* occB = cd.occ + (c * 2 + 1) * MAXORB;
  const uint8_t* virA = cd.vir + (c * 2) * MAXORB;
  const uint8_t* virB = cd.vir + (c * 2 + 1) * MAXORB;
  const double* epsA = cd.eps + (c * 2) * n;
  const double* epsB = cd.eps + (c * 2 + 1) * n;
  const double coeff = cd.C[c], hii = cd.hd[c];
  const uint64_t* det = cd.dets + c * D::NW;
  const Spin<NSW> sA = D::alpha(det), sB = D::beta(det);

  const UnitDesc ud = decode_unit(nA, nB, nvA, nvB, t);
  const int kind = ud.kind, ii = ud.ii, aa = ud.aa;
  const int64_t ninner = ud.ninner;
  int64_t done = 0;
  float mx = 0.f;  // largest |rv| of this lane (MODE 1)
  // partitioned search: units with a fixed alpha string are in or out of
  // range as a whole; the others test each contribution before evaluating it
  // A range of a split bin also selects one beta-hash class (nsub > 1): the
  // units with a varying alpha string have a fixed beta string (tested once
  // here), the others test each contribution's beta string.
  const bool part = blo > 0 || bhi < ASCI_BINS;
  const bool split = nsub > 1;
  bool chk = part;
  bool chkb = false;
  const bool fixed_alpha = kind == 1 || kind == 3 || kind == 4;
  uint32_t ubin = 0;
  // with alpha lists the caller runs a unit only when it has contributions
  // in the range: no bin test
  // list block of the unit's alpha string (alpha doubles)
  const int32_t lb = (al.g >= 0 && kind == 2) ? al.lidx[al.aidx[c]] : -1;
  const bool listed = al.g >= 0 && kind != 0 && (kind != 2 || lb >= 0);
  if(listed) chk = false;
  if(fixed_alpha && !listed && (part || hist)) {
    Spin<NSW> ua = sA;
    if(kind == 4) ua = sp_flip(sp_flip(sA, int(occA[ii])), int(virA[aa]));
    ubin = alpha_bin<NSW>(ua);
    if(part && (ubin < blo || ubin >= bhi)) {
      if(MODE == 0 && lane == 0) *count_out = 0;
      return;
    }
    chk = false;
    chkb = split;
  }
  if(!fixed_alpha && split && beta_sub<NSW>(sB, nsub) != sub) {
    if(MODE == 0 && lane == 0) *count_out = 0;
    return;
  }
  // ranked keys: the rank of the spin string that is fixed for the unit, and
  // the table of the other spin's ranks indexed by the inner index q
  uint64_t rfix = 0;
  const uint32_t* rvar = nullptr;
  int rshift = 0;
  if constexpr(MODE == 2) {
    const uint32_t* Ra = rt.a.R + size_t(rt.a.idx[c]) * size_t(rt.a.M);
    const uint32_t* Rb = rt.b.R + size_t(rt.b.idx[c]) * size_t(rt.b.M);
    const int ba = rt.bits_a;
    if(kind == 0) {
      rfix = uint64_t(Rb[0]) << ba;
      rvar = Ra + 1;
    } else if(kind == 1) {
      rfix = Ra[0];
      rvar = Rb + 1;
      rshift = ba;
    } else if(kind == 2) {
      rfix = uint64_t(Rb[0]) << ba;
      rvar = Ra + 1 + rt.a.N1 + double_row_base(ii, aa, nA, nvA);
    } else if(kind == 3) {
      rfix = Ra[0];
      rvar = Rb + 1 + rt.b.N1 + double_row_base(ii, aa, nB, nvB);
      rshift = ba;
    } else {
      rfix = Ra[1 + ii * nvA + aa];
      rvar = Rb + 1;
      rshift = ba;
    }
  }
  int64_t nloop = ninner;
  const uint16_t* qlist = nullptr;
  if(listed && kind == 2) {
    const size_t row = size_t(lb) * al.NK + size_t(ii) * nvA + aa;
    const uint16_t* rr = al.rel + row * (al.G + 1);
    const int e0 = rr[al.g];
    qlist = al.q + al.base[row] + e0;
    nloop = int64_t(rr[al.g + 1]) - e0;
  }
  for(int64_t q0 = 0; q0 < nloop; q0 += 32) {
    const int64_t qi = q0 + lane;
    bool keep = false;
    double r = 0;
    uint64_t ex[D::NW];
    uint64_t rkey = 0;
    if(qi < nloop) {
      const int64_t q = qlist ? int64_t(qlist[qi]) : qi;
      if(kind <= 1) {
        // append_singles_asci_contributions (determinant_contributions.hpp:25-66)
        const int S = kind;
        const int nS = S ? nB : nA, nvS = S ? nvB : nvA;
        const uint8_t* occS = S ? occB : occA;
        const uint8_t* virS = S ? virB : virA;
        const int nO = S ? nA : nB;
        const uint8_t* occO = S ? occA : occB;
        const int qd = small_div(q, 1.0f / float(nvS));
        const int i = occS[qd], a = virS[int(q) - qd * nvS];
        uint32_t cbin = 0;
        if(S == 0 && (chk || hist))
          cbin = alpha_bin<NSW>(sp_flip(sp_flip(sA, i), a));
        bool inr = !chk || (cbin >= blo && cbin < bhi);
        if(chkb)  // S == 1
          inr = beta_sub<NSW>(sp_flip(sp_flip(sB, i), a), nsub) == sub;
        double h = 0;
        if(inr) {
          h = __ldg(I.T + a + size_t(i) * n);
          const double* Gov = I.G_red + size_t(a) * n + size_t(i) * n * n;
          const double* Vov = I.V_red + size_t(a) * n + size_t(i) * n * n;
          for(int p = 0; p < nS; ++p) h += __ldg(Gov + occS[p]);
          for(int p = 0; p < nO; ++p) h += __ldg(Vov + occO[p]);
        }
        keep = inr && !(fabs(h) < tol);
        if(MODE == 0 && hist && S == 0 && keep) atomicAdd(hist + cbin, 1ull);
        if(MODE >= 1 && keep) {
          const double* eps = S ? epsB : epsA;
          h *= ex_sign(S ? sB : sA, a, i);
          const double hd = hii + eps[a] - eps[i] - G2R(a, i) - G2R(i, a);
          h /= (E0 - hd);
          r = coeff * h;
          if constexpr(MODE == 1) {
#pragma unroll
            for(int w = 0; w < D::NW; ++w) ex[w] = det[w];
            det_flip<NBITS>(ex, S, i);
            det_flip<NBITS>(ex, S, a);
          }
        }
        (void)nS;
      } else if(kind <= 3) {
        // append_ss_doubles_asci_contributions (determinant_contributions.hpp:68-120)
        const int S = kind - 2;
        const int nvS = S ? nvB : nvA;
        const uint8_t* occS = S ? occB : occA;
        const uint8_t* virS = S ? virB : virA;
        const int span = nvS - 1 - aa;
        const int qd = small_div(q, 1.0f / float(span));
        const int jj = ii + 1 + qd, bb = aa + 1 + (int(q) - qd * span);
        const int i = occS[ii], a = virS[aa], j = occS[jj], b = virS[bb];
        uint32_t cbin = 0;
        if(S == 0 && (chk || hist))
          cbin = alpha_bin<NSW>(
              sp_flip(sp_flip(sp_flip(sp_flip(sA, i), j), a), b));
        bool inr = !chk || (cbin >= blo && cbin < bhi);
        if(chkb)  // S == 1
          inr = beta_sub<NSW>(
                    sp_flip(sp_flip(sp_flip(sp_flip(sB, i), j), a), b), nsub) ==
                sub;
        const double Gv =
            inr ? __ldg(I.G + size_t(a + size_t(i) * n) * n * n + b + size_t(j) * n)
                : 0.0;
        keep = inr && !(fabs(Gv) < tol);
        if(MODE == 0 && hist && S == 0 && keep) atomicAdd(hist + cbin, 1ull);
        if(MODE >= 1 && keep) {
          const Spin<NSW> st = S ? sB : sA;
          Spin<NSW> fx = sp_flip(sp_flip(sp_flip(sp_flip(sp_zero<NSW>(), i), j), a), b);
          const uint32_t e = double_ex(st, st ^ fx);
          double h = ex_sgn(e) * Gv;
          const double* eps = S ? epsB : epsA;
          const double hd = hii + eps[a] + eps[b] - eps[i] - eps[j] + G2R(i, j) +
                            G2R(j, i) + G2R(a, b) + G2R(b, a) - G2R(a, i) -
                            G2R(i, a) - G2R(b, i) - G2R(i, b) - G2R(a, j) -
                            G2R(j, a) - G2R(b, j) - G2R(j, b);
          h /= (E0 - hd);
          r = coeff * h;
          if constexpr(MODE == 1) {
#pragma unroll
            for(int w = 0; w < D::NW; ++w) ex[w] = det[w];
            det_flip<NBITS>(ex, S, i);
            det_flip<NBITS>(ex, S, j);
            det_flip<NBITS>(ex, S, a);
            det_flip<NBITS>(ex, S, b);
          }
        }
      } else {
        // append_os_doubles_asci_contributions (determinant_contributions.hpp:122-160)
        const int i = occA[ii], a = virA[aa];
        const int qd = small_div(q, 1.0f / float(nvB));
        const int j = occB[qd], b = virB[int(q) - qd * nvB];
        const bool inr =
            !chkb || beta_sub<NSW>(sp_flip(sp_flip(sB, j), b), nsub) == sub;
        // V(a,i,b,j) from row (a,i) of the pair-swapped copy: consecutive
        // inner indices read neighbouring addresses
        const double Vv =
            inr ? __ldg(cd.VT + size_t(a + size_t(i) * n) * n * n + b + size_t(j) * n)
                : 0.0;
        keep = inr && !(fabs(Vv) < tol);
        if(MODE >= 1 && keep) {
          const double sign = ex_sign(sA, a, i) * ex_sign(sB, b, j);
          double h = sign * Vv;
          const double hd = hii + epsA[a] + epsB[b] - epsA[i] - epsB[j] +
                            V2R(i, j) + V2R(a, b) - G2R(a, i) - G2R(i, a) -
                            G2R(b, j) - G2R(j, b) - V2R(a, j) - V2R(i, b);
          h /= (E0 - hd);
          r = coeff * h;
          if constexpr(MODE == 1) {
#pragma unroll
            for(int w = 0; w < D::NW; ++w) ex[w] = det[w];
            det_flip<NBITS>(ex, 0, a);
            det_flip<NBITS>(ex, 0, i);
            det_flip<NBITS>(ex, 1, j);
            det_flip<NBITS>(ex, 1, b);
          }
        }
      }
      if constexpr(MODE == 2)
        if(keep) rkey = rfix | (uint64_t(__ldg(rvar + q)) << rshift);
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if(MODE >= 1 && keep) {
      const int64_t pos = out0 + done + __popc(m & lanemask_lt());
      if constexpr(MODE == 1) {
#pragma unroll
        for(int w = 0; w < D::NW; ++w) keys[pos * D::NW + w] = ex[w];
      } else {
        keys[pos] = rkey;
      }
      rv[pos] = r;
      mx = fmaxf(mx, float(fabs(r)));
    }
    done += __popc(m);
  }
  if(MODE == 0 && lane == 0) {
    *count_out = done;
    if(hist && fixed_alpha && done) atomicAdd(hist + ubin, (unsigned long long)done);
  }
  if(MODE >= 1 && umax) {
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if(lane == 0) *umax = fmaxf(*umax, mx);  // running max over ranges
  }
}
#undef G2R
#undef V2R

// Units [u0, u1) of the batch, a warp at a time over runs of 32
// consecutive units: the lanes read the 32 units' masks, counts, owners and
// output offsets at once, and the warp runs the units with work one after
// another (a fill pass skips the units without contributions in its range:
// output positions come from the offsets, not from the order).
template <int NBITS, int MODE>
__global__ void __launch_bounds__(256)
    units_k(Ints I, CoreData cd, int64_t u0, int64_t u1, size_t c0, size_t c1,
            double E0, double tol, int64_t* counts, const int64_t* outoff,
            uint64_t* keys, double* rv, const uint8_t* umask, float* umax,
            uint32_t blo, uint32_t bhi, uint32_t nsub, uint32_t sub,
            unsigned long long* hist, AlphaLists al, RankTables rt) {
  // hist (count pass only): per-block bin counts in shared memory
  // (dynamic, ASCI_BINS x 8 B), added to the global histogram at the end
  extern __shared__ unsigned long long shist[];
  if(hist) {
    for(uint32_t i = threadIdx.x; i < ASCI_BINS; i += blockDim.x) shist[i] = 0;
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = int64_t(gridDim.x) * (blockDim.x >> 5);
  for(int64_t ub = u0 + (int64_t(blockIdx.x) * (blockDim.x >> 5) +
                         (threadIdx.x >> 5)) * 32;
      ub < u1; ub += nwarp * 32) {
    const int64_t ul = ub + lane;
    bool run = ul < u1;
    if(run && umask && !umask[ul]) {  // screened out: no contributions
      if(MODE == 0) counts[ul - u0] = 0;
      run = false;
    }
    int64_t off = 0;
    if(MODE >= 1 && run) {
      run = counts[ul - u0] != 0;
      off = outoff[ul - u0];
    }
    int32_t own = 0;
    int64_t t = 0;
    if(run) {  // core det owning unit ul (in [c0, c1)), and its index there
      own = cd.udet[ul];
      t = ul - cd.uoff[own];
    }
    if(MODE == 0 && al.g >= 0 && run) {
      // count pass of a range with alpha lists (list_rest): only the alpha
      // singles and the alpha doubles of unlisted alpha strings; the others
      // were counted by range_count_k
      const int64_t KA = int64_t(cd.cnt[size_t(own) * 4]) * cd.cnt[size_t(own) * 4 + 2];
      run = t == 0 || (t >= 2 && t < 2 + KA && al.lidx[al.aidx[own]] < 0);
    }
    for(unsigned m = __ballot_sync(0xffffffffu, run); m; m &= m - 1) {
      const int l = __ffs(m) - 1;
      const int64_t u = ub + l;
      const size_t c = size_t(__shfl_sync(0xffffffffu, own, l));
      const int64_t tu = __shfl_sync(0xffffffffu, t, l);
      const int64_t ou = __shfl_sync(0xffffffffu, off, l);
      unit_run<NBITS, MODE>(I, cd, c, tu, E0, tol, counts + (u - u0), ou, keys,
                            rv, umax ? umax + u : nullptr, blo, bhi, nsub, sub,
                            hist ? shist : nullptr, al, rt);
    }
  }
  if(hist) {
    __syncthreads();
    for(uint32_t i = threadIdx.x; i < ASCI_BINS; i += blockDim.x)
      if(shist[i]) atomicAdd(hist + i, shist[i]);
  }
}

// Alpha lists: the bin of every distinct alpha string and, per outer pair,
// of the string after the outer alpha excitation (one thread per pair).
template <int NBITS>
__global__ void alpha_bins_k(CoreData cd, const int32_t* rep, size_t nua,
                             int nvA, int NK, uint16_t* kbin, uint16_t* abin) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  const size_t rows = nua * size_t(NK);
  for(size_t row = size_t(blockIdx.x) * blockDim.x + threadIdx.x; row < rows;
      row += size_t(gridDim.x) * blockDim.x) {
    const size_t u = row / NK;
    const int k = int(row - u * NK);
    const int ii = k / nvA, aa = k - ii * nvA;
    const size_t c = size_t(rep[u]);
    const Spin<NSW> sA = D::alpha(cd.dets + c * D::NW);
    const int i = cd.occ[(c * 2) * MAXORB + ii], a = cd.vir[(c * 2) * MAXORB + aa];
    kbin[row] = uint16_t(alpha_bin<NSW>(sp_flip(sp_flip(sA, i), a)));
    if(k == 0) abin[u] = uint16_t(alpha_bin<NSW>(sA));
  }
}

// Alpha lists, count pass: one warp per (list block, outer pair k) row.
// Writes the row's group starts (prefix of the per-group counts, G + 1
// entries); grp maps a bin to its group (0xFFFF: a split range or outside
// this search's bins). The lists keep the inner indices whose integral
// passes the threshold test of unit_run (kind 2) and whose bin has a group.
// rep: per list block, a core det with its alpha string.
template <int NBITS>
__global__ void __launch_bounds__(256)
    alpha_count_k(Ints I, CoreData cd, const int32_t* rep, size_t nua, int nA,
                  int nvA, double tol, const uint16_t* grp, AlphaLists al,
                  uint16_t* rel, int64_t* tot) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  extern __shared__ int gcnt[];  // per warp: G counters
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int* cnt = gcnt + wib * (al.G + 1);
  const int n = cd.n;
  const size_t rows = nua * size_t(al.NK);
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t row = size_t(blockIdx.x) * (blockDim.x >> 5) + wib; row < rows;
      row += nwarp) {
    const size_t u = row / al.NK;
    const int k = int(row - u * al.NK);
    const int ii = k / nvA, aa = k - ii * nvA;
    const size_t c = size_t(rep[u]);
    const uint8_t* occA = cd.occ + (c * 2) * MAXORB;
    const uint8_t* virA = cd.vir + (c * 2) * MAXORB;
    const Spin<NSW> sA = D::alpha(cd.dets + c * D::NW);
    for(int g = lane; g < al.G; g += 32) cnt[g] = 0;
    __syncwarp();
    const int i = occA[ii], a = virA[aa];
    const int span = nvA - 1 - aa;
    const int64_t ninner = int64_t(nA - 1 - ii) * span;
    for(int64_t q = lane; q < ninner; q += 32) {
      const int qd = small_div(q, 1.0f / float(span));
      const int j = occA[ii + 1 + qd], b = virA[aa + 1 + (int(q) - qd * span)];
      const double Gv =
          __ldg(I.G + size_t(a + size_t(i) * n) * n * n + b + size_t(j) * n);
      if(!(fabs(Gv) < tol)) {
        const unsigned g = grp[alpha_bin<NSW>(
            sp_flip(sp_flip(sp_flip(sp_flip(sA, i), j), a), b))];
        if(g != 0xFFFFu) atomicAdd(cnt + g, 1);
      }
    }
    __syncwarp();
    if(lane == 0) {
      int acc = 0;
      uint16_t* rr = rel + row * (al.G + 1);
      for(int g = 0; g < al.G; ++g) {
        rr[g] = uint16_t(acc);
        acc += cnt[g];
      }
      rr[al.G] = uint16_t(acc);
      tot[row] = acc;
    }
    __syncwarp();
  }
}

// Alpha lists, fill pass: the same rows, inner indices written at their
// group's position in ascending q (lanes with equal groups ranked by
// __match_any_sync).
template <int NBITS>
__global__ void __launch_bounds__(256)
    alpha_fill_k(Ints I, CoreData cd, const int32_t* rep, size_t nua, int nA,
                 int nvA, double tol, const uint16_t* grp, AlphaLists al,
                 uint16_t* qout) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  extern __shared__ int gcnt[];  // per warp: running position per group
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int* run = gcnt + wib * (al.G + 1);
  const int n = cd.n;
  const size_t rows = nua * size_t(al.NK);
  const size_t nwarp = size_t(gridDim.x) * (blockDim.x >> 5);
  for(size_t row = size_t(blockIdx.x) * (blockDim.x >> 5) + wib; row < rows;
      row += nwarp) {
    const size_t u = row / al.NK;
    const int k = int(row - u * al.NK);
    const int ii = k / nvA, aa = k - ii * nvA;
    const size_t c = size_t(rep[u]);
    const uint8_t* occA = cd.occ + (c * 2) * MAXORB;
    const uint8_t* virA = cd.vir + (c * 2) * MAXORB;
    const Spin<NSW> sA = D::alpha(cd.dets + c * D::NW);
    const uint16_t* rr = al.rel + row * (al.G + 1);
    for(int g = lane; g < al.G; g += 32) run[g] = rr[g];
    __syncwarp();
    uint16_t* out = qout + al.base[row];
    const int i = occA[ii], a = virA[aa];
    const int span = nvA - 1 - aa;
    const int64_t ninner = int64_t(nA - 1 - ii) * span;
    for(int64_t q0 = 0; q0 < ninner; q0 += 32) {
      const int64_t q = q0 + lane;
      unsigned g = 0xFFFFu;
      if(q < ninner) {
        const int qd = small_div(q, 1.0f / float(span));
        const int j = occA[ii + 1 + qd],
                  b = virA[aa + 1 + (int(q) - qd * span)];
        const double Gv =
            __ldg(I.G + size_t(a + size_t(i) * n) * n * n + b + size_t(j) * n);
        if(!(fabs(Gv) < tol))
          g = grp[alpha_bin<NSW>(
              sp_flip(sp_flip(sp_flip(sp_flip(sA, i), j), a), b))];
      }
      const unsigned peers = __match_any_sync(0xffffffffu, g);
      if(g != 0xFFFFu) {
        out[run[g] + __popc(peers & lanemask_lt())] = uint16_t(q);
      }
      __syncwarp();
      if(g != 0xFFFFu && (peers & lanemask_lt()) == 0) run[g] += __popc(peers);
      __syncwarp();
    }
  }
}

// Count pass of an unsplit range with alpha lists: one thread per unit.
// Fixed-alpha units (kinds 1, 3, 4) are in the range as a whole, with the
// count of the whole-search pass (ucnt); alpha doubles (kind 2) of listed
// alpha strings read their group's list length. The alpha singles (kind 0,
// whose threshold test depends on the beta string) and the alpha doubles of
// unlisted strings are left to units_k's count pass (list_rest).
__global__ void range_count_k(CoreData cd, AlphaLists al, int64_t U,
                              const int64_t* ucnt, const uint8_t* umask,
                              uint32_t blo, uint32_t bhi, int64_t* rc) {
  for(int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < U;
      u += int64_t(gridDim.x) * blockDim.x) {
    const size_t c = size_t(cd.udet[u]);
    const int64_t t = u - cd.uoff[c];
    if(t == 0) continue;
    int64_t r = 0;
    if(!umask || umask[u]) {
      const int64_t KA = int64_t(cd.cnt[c * 4]) * cd.cnt[c * 4 + 2];
      const int64_t KB = int64_t(cd.cnt[c * 4 + 1]) * cd.cnt[c * 4 + 3];
      const size_t ua = size_t(al.aidx[c]);
      uint32_t bin = ASCI_BINS;
      if(t < 2 + KA && t >= 2) {
        const int32_t lb = al.lidx[ua];
        if(lb < 0) continue;  // counted by units_k
        const uint16_t* rr = al.rel + (size_t(lb) * al.NK + size_t(t - 2)) * (al.G + 1);
        r = int64_t(rr[al.g + 1]) - rr[al.g];
      } else if(t == 1 || t < 2 + KA + KB) {
        bin = al.abin[ua];
      } else {
        bin = al.kbin[ua * al.NK + size_t(t - 2 - KA - KB)];
      }
      if(bin < ASCI_BINS && bin >= blo && bin < bhi) r = ucnt[u];
    }
    rc[u] = r;
  }
}

// ------------------------------------------------------ learned screening
// Network input of a unit (width 2 * 64 NSW + 64):
//   occupation bits of the core det after the unit's outer excitation
//   (alpha orbitals in columns [0, 64 NSW), beta in [64 NSW, 128 NSW)), then
//   64 features: 1, ln|C_c| / 10, one-hot kind (5), eps of the outer hole and
//   particle and their difference, E0 - H_cc, ln(1 + inner count) / 10, the
//   outer orbitals scaled to (0, 1], ln of the outer pair's integral bound
//   (macis_b200_ham::pairmax) / 10, a crude ln score estimate
//   (ln|C| + ln bound - ln|E0 - H_cc - (eps_a - eps_i)|) / 10, and the
//   eps-weighted occupations of orbitals 0..47 of the excited det (eps =
//   the core det's single-orbital energies of the spin).
constexpr int UNIT_EPS_ORBS = 48;

template <int NBITS>
__host__ __device__ constexpr int unit_din() {
  return 2 * 64 * DetTraits<NBITS>::NSW + MLP_NFEAT;
}

__device__ __forceinline__ size_t unit_owner(const CoreData& cd, int64_t u) {
  return size_t(cd.udet[u]);
}

__device__ __forceinline__ uint32_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// put(k, v): 16-byte piece k (columns [8k, 8k+8)) of the unit's row.
template <int NBITS, class Put>
__device__ void unit_features(const CoreData& cd, double E0, int64_t u,
                              Put&& put) {
  using D = DetTraits<NBITS>;
  constexpr int NSW = D::NSW;
  const size_t c = unit_owner(cd, u);
  const int64_t t = u - cd.uoff[c];
  const int n = cd.n;
  const int no[2] = {cd.cnt[c * 4], cd.cnt[c * 4 + 1]};
  const int nv[2] = {cd.cnt[c * 4 + 2], cd.cnt[c * 4 + 3]};
  const UnitDesc ud = decode_unit(no[0], no[1], nv[0], nv[1], t);
  const uint64_t* det = cd.dets + c * D::NW;
  Spin<NSW> sp[2] = {D::alpha(det), D::beta(det)};
  const double* eps[2] = {cd.eps + (c * 2) * n, cd.eps + (c * 2 + 1) * n};
  int S = 0, hole = -1, part = -1;
  if(ud.kind >= 2) {
    S = ud.kind == 3 ? 1 : 0;
    hole = cd.occ[(c * 2 + S) * MAXORB + ud.ii];
    part = cd.vir[(c * 2 + S) * MAXORB + ud.aa];
    sp[S] = sp_flip(sp_flip(sp[S], hole), part);
  }
  // occupation bits, one byte per piece
#pragma unroll
  for(int s = 0; s < 2; ++s)
#pragma unroll
    for(int b = 0; b < NSW * 8; ++b) {
      const uint32_t byte = uint32_t(sp[s].w[b >> 3] >> ((b & 7) * 8)) & 0xFFu;
      uint32_t w[4];
#pragma unroll
      for(int q = 0; q < 4; ++q)
        w[q] = (((byte >> (2 * q)) & 1u) ? 0x3F80u : 0u) |
               (((byte >> (2 * q + 1)) & 1u) ? 0x3F800000u : 0u);
      put(s * NSW * 8 + b, make_uint4(w[0], w[1], w[2], w[3]));
    }
  // scalar features
  const double eh = hole >= 0 ? eps[S][hole] : 0.0;
  const double ep = part >= 0 ? eps[S][part] : 0.0;
  float f[16];
  f[0] = 1.f;
  f[1] = float(log(fabs(cd.C[c]) + 1e-300) / 10.0);
#pragma unroll
  for(int k = 0; k < 5; ++k) f[2 + k] = ud.kind == k ? 1.f : 0.f;
  f[7] = float(eh);
  f[8] = float(ep);
  f[9] = float(ep - eh);
  f[10] = float(E0 - cd.hd[c]);
  f[11] = float(log(1.0 + double(ud.ninner)) / 10.0);
  f[12] = hole >= 0 ? float(hole + 1) / float(n) : 0.f;
  f[13] = part >= 0 ? float(part + 1) / float(n) : 0.f;
  // outer-pair integral bound and a crude log-score estimate
  const double lnc = log(fabs(cd.C[c]) + 1e-300);
  if(ud.kind >= 2) {
    const size_t pr = size_t(part) + size_t(hole) * n;
    const double bound =
        cd.pairmax[(ud.kind == 4 ? size_t(n) * n : 0) + pr];
    const double lb = log(bound + 1e-300);
    f[14] = float(lb / 10.0);
    f[15] = float((lnc + lb - log(fabs(E0 - cd.hd[c] - (ep - eh)) + 1e-3)) /
                  10.0);
  } else {
    f[14] = 0.f;
    f[15] = float((lnc - log(fabs(E0 - cd.hd[c]) + 1e-3)) / 10.0);
  }
  const int base = 2 * NSW * 8;
#pragma unroll
  for(int q = 0; q < 2; ++q) {
    uint32_t w[4];
#pragma unroll
    for(int k = 0; k < 4; ++k)
      w[k] = bf16_bits(f[8 * q + 2 * k]) | (bf16_bits(f[8 * q + 2 * k + 1]) << 16);
    put(base + q, make_uint4(w[0], w[1], w[2], w[3]));
  }
  // eps-weighted occupations
  for(int q = 0; q < UNIT_EPS_ORBS / 8; ++q) {
    uint32_t w[4];
#pragma unroll
    for(int k = 0; k < 4; ++k) {
      float v2[2];
#pragma unroll
      for(int h = 0; h < 2; ++h) {
        const int p = 8 * q + 2 * k + h;
        double e = 0.0;
        if(p < n) {
          if(sp_test(sp[0], p)) e += eps[0][p];
          if(sp_test(sp[1], p)) e += eps[1][p];
        }
        v2[h] = float(e);
      }
      w[k] = bf16_bits(v2[0]) | (bf16_bits(v2[1]) << 16);
    }
    put(base + 2 + q, make_uint4(w[0], w[1], w[2], w[3]));
  }
}

// Row source of the fused forward: tile row r = unit row0 + r.
template <int NBITS>
struct UnitRows {
  CoreData cd;
  double E0;
  __device__ void fill(int64_t row0, int nvalid, uint8_t* xs, int tid) const {
    uint8_t* base = xs + tid * 16;
    if(tid < nvalid) {
      unit_features<NBITS>(cd, E0, row0 + tid, [&](int k, uint4 v) {
        *reinterpret_cast<uint4*>(base + size_t(k) * (MLP_TM * 16)) = v;
      });
    } else {
      for(int k = 0; k < unit_din<NBITS>() / 8; ++k)
        *reinterpret_cast<uint4*>(base + size_t(k) * (MLP_TM * 16)) =
            make_uint4(0, 0, 0, 0);
    }
  }
};

// Rows of the listed units into X [n][din] (row-major BF16), and targets
// t = (ln max(umax, 1e-12) + 20) / 5 when umax is given.
template <int NBITS>
__global__ void unit_rows_k(CoreData cd, double E0, const int64_t* units,
                            int64_t first, size_t n, uint16_t* X,
                            const float* umax, float* t) {
  constexpr int DIN = unit_din<NBITS>();
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const int64_t u = units ? units[i] : first + int64_t(i);
    uint4* row = reinterpret_cast<uint4*>(X + i * DIN);
    unit_features<NBITS>(cd, E0, u, [&](int k, uint4 v) { row[k] = v; });
    if(t) t[i] = (logf(fmaxf(umax[u], 1e-12f)) + 20.f) / 5.f;
  }
}

__device__ __forceinline__ uint32_t pred_key(float x) {
  const uint32_t b = __float_as_uint(x);
  if(x != x) return 0u;  // NaN ranks last
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__global__ void pred_hist_k(const float* y, size_t n, uint32_t prefix,
                            uint32_t mask, int shift,
                            unsigned long long* hist) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t k = pred_key(y[i]);
    if((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  if(h[threadIdx.x])
    atomicAdd(&hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// keep units predicted at or above the threshold key, plus a hashed random
// fraction (explore / 2^64) of the others
__global__ void unit_mask_k(const float* y, size_t n, uint32_t T,
                            uint64_t explore, uint64_t seed, uint8_t* mask,
                            unsigned long long* nkept) {
  unsigned int c = 0;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const bool k = pred_key(y[i]) >= T ||
                   mix64(seed + 0x9E3779B97F4A7C15ull * (i + 1)) < explore;
    mask[i] = k ? 1 : 0;
    c += k;
  }
  for(int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if((threadIdx.x & 31) == 0 && c) atomicAdd(nkept, (unsigned long long)c);
}
// sample flags over the units that ran (mask or all)
__global__ void sample_flags_k(const uint8_t* mask, size_t n, uint64_t p,
                               uint64_t seed, uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = ((!mask || mask[i]) &&
            mix64(seed ^ (0xD1B54A32D192ED03ull * (i + 1))) <= p)
               ? 1u
               : 0u;
}
__global__ void sample_list_k(const uint32_t* f, const uint32_t* fx, size_t n,
                              size_t cap, int64_t* list) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(f[i] && fx[i] < cap) list[fx[i]] = int64_t(i);
}

// --------------------------------------------------- accumulate / merge
template <int NW>
__global__ void seg_flags_k(const uint64_t* keys, size_t n, uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = (i == 0 || !key_eq<NW>(load_key<NW>(keys, i), load_key<NW>(keys, i - 1)))
               ? 1u
               : 0u;
}
template <int NW>
__global__ void seg_starts_k(const uint32_t* f, const uint32_t* fx, size_t n,
                             int64_t* start, const uint64_t* keys,
                             uint64_t* ukeys) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(f[i]) {
      start[fx[i]] = int64_t(i);
      store_key<NW>(ukeys, fx[i], load_key<NW>(keys, i));
    }
}
// Sequential sum of each segment in sorted (= generation) order.
__global__ void seg_sum_k(const int64_t* start, size_t nseg, size_t n,
                          const double* rv, double* out) {
  for(size_t s = size_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nseg;
      s += size_t(gridDim.x) * blockDim.x) {
    const int64_t b = start[s], e = s + 1 < nseg ? start[s + 1] : int64_t(n);
    double a = rv[b];
    for(int64_t j = b + 1; j < e; ++j) a += rv[j];
    out[s] = a;
  }
}

// --------------------------------------------------------- core / top-k
// Candidates of a range that may enter the top-k: nonzero scores whose
// |rv| bits are at least tcut (the running k-th score so far: the final
// threshold is never lower, and ties stay), and not core dets.
template <int NW>
__global__ void keep_flags_k(const uint64_t* keys, const double* rv, size_t n,
                             const uint64_t* core, size_t nc, uint64_t tcut,
                             uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const double a = fabs(rv[i]);
    if(!(-a < 0.0) || uint64_t(__double_as_longlong(a)) < tcut) {
      f[i] = 0u;
      continue;
    }
    const Key<NW> k = load_key<NW>(keys, i);
    size_t lo = 0, hi = nc;
    bool found = false;
    while(lo < hi) {
      const size_t mid = (lo + hi) >> 1;
      const int c = key_cmp<NW>(load_key<NW>(core, mid), k);
      if(c == 0) {
        found = true;
        break;
      }
      if(c < 0)
        lo = mid + 1;
      else
        hi = mid;
    }
    f[i] = found ? 0u : 1u;
  }
}
template <int NW>
__global__ void compact_k(const uint64_t* keys, const double* rv, size_t n,
                          const uint32_t* f, const uint32_t* fx,
                          uint64_t* ok, double* orv) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    if(f[i]) {
      store_key<NW>(ok, fx[i], load_key<NW>(keys, i));
      orv[fx[i]] = rv[i];
    }
}
// Prune: keep |rv| > tol (determinant_search.hpp:122-127).
__global__ void prune_flags_k(const double* rv, size_t n, double tol,
                              uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = fabs(rv[i]) > tol ? 1u : 0u;
}

__global__ void select_hist_k(const double* rv, size_t n, uint64_t prefix,
                              uint64_t mask, int shift,
                              unsigned long long* hist) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t k = uint64_t(__double_as_longlong(fabs(rv[i])));
    if((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255], 1u);
  }
  __syncthreads();
  if(h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}
__global__ void select_flags_k(const double* rv, size_t n, uint64_t T,
                               uint32_t* gt, uint32_t* eq) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t k = uint64_t(__double_as_longlong(fabs(rv[i])));
    gt[i] = k > T;
    eq[i] = k == T;
  }
}
// |rv| at or above the threshold bits T (candidates that stay in the running
// top-k, ties included)
__global__ void ge_flags_k(const double* rv, size_t n, uint64_t T,
                           uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = uint64_t(__double_as_longlong(fabs(rv[i]))) >= T ? 1u : 0u;
}
// final selection: everything above the threshold, and the ties whose
// determinant is not above Kmax (the need-th smallest tied determinant)
template <int NW>
__global__ void tie_select_k(const uint64_t* keys, const uint32_t* gt,
                             const uint32_t* eq, size_t n, Key<NW> Kmax,
                             uint32_t* f) {
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x)
    f[i] = gt[i] || (eq[i] && key_cmp<NW>(load_key<NW>(keys, i), Kmax) <= 0);
}

// ----------------------------------------------------------------- driver
namespace {
struct Pairs {
  uint64_t* keys = nullptr;
  double* rv = nullptr;
  size_t n = 0;
};
double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now() - t)
      .count();
}
}  // namespace

// Core-det precompute and unit offsets; returns the unit count.
template <int NBITS>
static int64_t core_setup(macis_b200_ham* h, Arena& A, const uint64_t* cdets,
                          size_t ncdets, const double* C, int just_singles,
                          CoreData& cd) {
  cudaStream_t s = h->stream;
  const int n = h->norb;
  const int sms = num_sms();
  cd = CoreData{};
  cd.n = n;
  cd.dets = cdets;
  cd.C = C;
  cd.ncdets = ncdets;
  cd.occ = A.get<uint8_t>(ncdets * 2 * MAXORB + 1);
  cd.vir = A.get<uint8_t>(ncdets * 2 * MAXORB + 1);
  cd.cnt = A.get<uint8_t>(ncdets * 4 + 1);
  cd.eps = A.get<double>(ncdets * 2 * n + 1);
  cd.hd = A.get<double>(ncdets + 1);
  int64_t* units = A.get<int64_t>(ncdets + 1);
  cd.uoff = A.get<int64_t>(ncdets + 1);
  if(!h->pairmax) {
    const size_t n2 = size_t(n) * n;
    MB_CUDA(dev_malloc(&h->pairmax, 2 * n2 * sizeof(double)));
    pairmax_g_k<<<grid_for(n2 * 32, 256, 16 * sms), 256, 0, s>>>(
        h->G, n, h->pairmax), note_launch();
    pairmax_v_k<<<grid_for(n2, 128, 4 * sms), 128, 0, s>>>(
        h->V, n, h->pairmax + n2), note_launch();
    MB_CUDA(cudaGetLastError());
  }
  cd.pairmax = h->pairmax;
  cd.VT = ham_vt(h);
  if(ncdets) {
    core_prep_k<NBITS><<<grid_for(ncdets * 32, 256, 16 * sms), 256, 0, s>>>(
        h->ints(), cd, just_singles, units), note_launch();
    MB_CUDA(cudaGetLastError());
  }
  exclusive_scan<int64_t, int64_t>(units, cd.uoff, ncdets, cd.uoff + ncdets, A);
  const int64_t U = ncdets ? to_host(cd.uoff + ncdets, s) : 0;
  MB_REQUIRE(ncdets < (size_t(1) << 31), MACIS_B200_ECAPACITY,
             "ASCI search needs < 2^31 core determinants");
  cd.udet = A.get<int32_t>(size_t(U) + 1);
  if(U > 0)
    unit_owner_fill_k<<<grid_for(ncdets * 32, 256, 16 * sms), 256, 0, s>>>(
        cd.uoff, ncdets, cd.udet), note_launch();
  return U;
}

// Distinct spin strings of the core dets (host, from a copy of the dets):
// per det the index of its string of the spin, per string a representative
// det, its words and its occupied / virtual orbital lists. Empty (nu = 0)
// when the electron counts of the spin differ between dets.
struct SpinPlan {
  std::vector<int32_t> idx, rep;
  std::vector<uint64_t> words;  // nu x NSW
  std::vector<uint8_t> occ, vir;  // nu x MAXORB
  size_t nu = 0;
  int ne = 0, nv = 0;
};
template <int NBITS>
static SpinPlan plan_spin(const std::vector<uint64_t>& hd, size_t ncdets,
                          int n, int spin) {
  constexpr int NW = DetTraits<NBITS>::NW;
  constexpr int NSW = DetTraits<NBITS>::NSW;
  SpinPlan sp;
  if(!ncdets) return sp;
  auto key = [&](size_t c) {
    const uint64_t* d = hd.data() + c * NW;
    if constexpr(NBITS == 64)
      return std::pair<uint64_t, uint64_t>(
          spin ? d[0] >> 32 : d[0] & 0xffffffffull, 0);
    else if constexpr(NBITS == 128)
      return std::pair<uint64_t, uint64_t>(d[spin], 0);
    else
      return std::pair<uint64_t, uint64_t>(d[2 * spin + 1], d[2 * spin]);
  };
  std::vector<uint32_t> ord(ncdets);
  for(size_t c = 0; c < ncdets; ++c) ord[c] = uint32_t(c);
  std::sort(ord.begin(), ord.end(),
            [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
  sp.idx.resize(ncdets);
  for(size_t p = 0; p < ncdets; ++p) {
    if(p == 0 || key(ord[p]) != key(ord[p - 1])) {
      const auto k = key(ord[p]);
      const int ne = __builtin_popcountll(k.first) + __builtin_popcountll(k.second);
      if(p == 0) sp.ne = ne;
      if(ne != sp.ne) return SpinPlan{};
      sp.rep.push_back(int32_t(ord[p]));
      // words in the determinant's order (low word first)
      if constexpr(NSW == 1) {
        sp.words.push_back(k.first);
      } else {
        sp.words.push_back(k.second);
        sp.words.push_back(k.first);
      }
      std::vector<uint8_t> o(MAXORB, 0), v(MAXORB, 0);
      int no = 0, nv = 0;
      for(int i = 0; i < n; ++i) {
        const uint64_t w = i < 64 ? (NSW == 1 ? k.first : k.second) : k.first;
        if((w >> (i & 63)) & 1)
          o[no++] = uint8_t(i);
        else
          v[nv++] = uint8_t(i);
      }
      sp.occ.insert(sp.occ.end(), o.begin(), o.end());
      sp.vir.insert(sp.vir.end(), v.begin(), v.end());
    }
    sp.idx[ord[p]] = int32_t(sp.rep.size() - 1);
  }
  sp.nu = sp.rep.size();
  sp.nv = n - sp.ne;
  return sp;
}

// Candidates per distinct core string of a spin with ne electrons and nv
// virtuals: itself, ne nv singles, C(ne,2) C(nv,2) doubles.
static int64_t spin_candidates(int ne, int nv) {
  return 1 + int64_t(ne) * nv +
         int64_t(ne) * (ne - 1) / 2 * (int64_t(nv) * (nv - 1) / 2);
}

// Rank table of one spin (SpinRanks) and its distinct candidate strings in
// rank order (*L, NSW words each); returns their number. The candidates are
// generated with their index, radix-sorted, and equal neighbours share a
// rank.
template <int NBITS>
static size_t build_spin_ranks(const SpinPlan& sp, Arena& A, cudaStream_t s,
                               SpinRanks& out, uint64_t** L) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  const int ne = sp.ne, nv = sp.nv, nrows = ne * nv;
  const int64_t M = spin_candidates(ne, nv);
  const size_t tot = sp.nu * size_t(M);
  const int sms = num_sms();
  std::vector<int64_t> db(size_t(nrows) + 1, 0);
  for(int k = 0; k < nrows; ++k) {
    const int ii = k / nv, aa = k - ii * nv;
    db[size_t(k) + 1] = db[k] + int64_t(ne - 1 - ii) * (nv - 1 - aa);
  }
  uint32_t* R = A.get<uint32_t>(tot + 1);
  uint64_t* words = A.get<uint64_t>(sp.nu * NSW);
  uint8_t* occ = A.get<uint8_t>(sp.nu * MAXORB);
  uint8_t* vir = A.get<uint8_t>(sp.nu * MAXORB);
  int64_t* dbase = A.get<int64_t>(db.size());
  MB_CUDA(cudaMemcpyAsync(words, sp.words.data(), sp.nu * NSW * 8,
                          cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemcpyAsync(occ, sp.occ.data(), sp.nu * MAXORB,
                          cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemcpyAsync(vir, sp.vir.data(), sp.nu * MAXORB,
                          cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemcpyAsync(dbase, db.data(), db.size() * 8,
                          cudaMemcpyHostToDevice, s));
  uint64_t* cand = A.get<uint64_t>(tot * NSW + NSW);
  uint32_t* idx = A.get<uint32_t>(tot + 1);
  cand_strings_k<NSW><<<grid_for(tot, 256, 16 * sms), 256, 0, s>>>(
      words, occ, vir, sp.nu, ne, nv, M, int64_t(nrows), dbase, nrows, cand,
      idx), note_launch();
  MB_CUDA(cudaGetLastError());
  {
    uint64_t* cand2 = A.get<uint64_t>(tot * NSW + NSW);
    uint32_t* idx2 = A.get<uint32_t>(tot + 1);
    radix_sort<NSW, uint32_t>(cand, idx, cand2, idx2, tot, A);
    A.release(cand2);
    A.release(idx2);
  }
  uint32_t* f = A.get<uint32_t>(tot + 1);
  uint32_t* fx = A.get<uint32_t>(tot + 1);
  seg_flags_k<NSW><<<grid_for(tot, 256, 16 * sms), 256, 0, s>>>(cand, tot, f),
      note_launch();
  exclusive_scan<uint32_t, uint32_t>(f, fx, tot, fx + tot, A);
  const size_t NL = to_host(fx + tot, s);
  uint64_t* Ls = A.get<uint64_t>(NL * NSW + NSW);
  rank_scatter_k<NSW><<<grid_for(tot, 256, 16 * sms), 256, 0, s>>>(
      cand, idx, f, fx, tot, R, Ls), note_launch();
  MB_CUDA(cudaGetLastError());
  for(void* q : {static_cast<void*>(cand), static_cast<void*>(idx),
                 static_cast<void*>(f), static_cast<void*>(fx),
                 static_cast<void*>(words), static_cast<void*>(occ),
                 static_cast<void*>(vir), static_cast<void*>(dbase)})
    A.release(q);
  out.R = R;
  out.M = M;
  out.N1 = int64_t(nrows);
  *L = Ls;
  return NL;
}

static int bits_for(size_t n) {
  return n <= 1 ? 1 : 64 - __builtin_clzll(uint64_t(n - 1));
}

// Rank tables of both spins (RankTables), when they fit: the tables and
// the distinct candidate strings within 10 % of the free device memory,
// the candidate sort within half of it, 32-bit candidate indices and
// bits_a + bits_b <= 64. Returns the key width in bits, 0 when not built.
template <int NBITS>
static int build_ranks(const SpinPlan& pa, const SpinPlan& pb, size_t ncdets,
                       Arena& A, cudaStream_t s, RankTables& rt) {
  constexpr int NSW = DetTraits<NBITS>::NSW;
  const size_t ta = pa.nu * size_t(spin_candidates(pa.ne, pa.nv));
  const size_t tb = pb.nu * size_t(spin_candidates(pb.ne, pb.nv));
  if(ta >= (size_t(1) << 32) - 1 || tb >= (size_t(1) << 32) - 1) return 0;
  // the rank tables (4 B per candidate) first; the distinct candidate
  // strings, far fewer where core strings share candidates, are checked
  // once they are known
  const double avail = double(device_bytes_available());
  const double tables = 4.0 * double(ta + tb) + 8.0 * double(ncdets);
  const double trans = double(std::max(ta, tb)) * (16.0 * NSW + 20.0);
  if(tables > 0.1 * avail || tables + trans > 0.5 * avail) return 0;
  uint64_t *La = nullptr, *Lb = nullptr;
  SpinRanks ra, rb;
  const size_t na = build_spin_ranks<NBITS>(pa, A, s, ra, &La);
  const size_t nb = build_spin_ranks<NBITS>(pb, A, s, rb, &Lb);
  const int ba = bits_for(na), bb = bits_for(nb);
  const double strings = (8.0 * NSW + 2.0) * double(na) + 8.0 * NSW * double(nb);
  if(ba + bb > 64 || tables + strings > 0.15 * avail) {
    for(const void* q : {static_cast<const void*>(ra.R),
                         static_cast<const void*>(rb.R),
                         static_cast<const void*>(La),
                         static_cast<const void*>(Lb)})
      A.release(const_cast<void*>(q));
    return 0;
  }
  uint16_t* bin = A.get<uint16_t>(na + 1);
  string_bins_k<NSW><<<grid_for(na, 256, 4 * num_sms()), 256, 0, s>>>(
      La, na, bin), note_launch();
  int32_t* ai = A.get<int32_t>(ncdets);
  int32_t* bi = A.get<int32_t>(ncdets);
  MB_CUDA(cudaMemcpyAsync(ai, pa.idx.data(), ncdets * 4,
                          cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemcpyAsync(bi, pb.idx.data(), ncdets * 4,
                          cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaGetLastError());
  ra.idx = ai;
  rb.idx = bi;
  rt.a = ra;
  rt.b = rb;
  rt.bits_a = ba;
  rt.La = La;
  rt.Lb = Lb;
  rt.bin_a = bin;
  return ba + bb;
}

static void check_net(const macis_b200_mlp* net, cudaStream_t s) {
  int e = 0;
  MB_CUDA(cudaMemcpyAsync(&e, net->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  if(e) {  // cleared, so that the next call starts clean
    MB_CUDA(cudaMemsetAsync(net->err, 0, sizeof(int), s));
    MB_CUDA(cudaStreamSynchronize(s));
  }
  MB_REQUIRE(e == 0, MACIS_B200_ETIMEOUT,
             "screening network kernel timed out waiting on a barrier");
}

template <int NBITS>
static void asci_impl(macis_b200_ham* h, const macis_b200_asci_settings& st,
                      const macis_b200_asci_screen* scr, size_t ndets_max,
                      const uint64_t* cdets, size_t ncdets, double E0,
                      const double* C, uint64_t* out_dets, size_t* nout,
                      std::vector<uint64_t>* ps, std::vector<double>* pr,
                      bool pairs_only, const AsciPart* part) {
  constexpr int NW = DetTraits<NBITS>::NW;
  cudaStream_t s = h->stream;
  Arena A(s);
  const Ints I = h->ints();
  const int sms = num_sms();
  auto t_all = std::chrono::steady_clock::now();
  macis_b200_asci_stats stats{};
  NvtxRange nv("macis_b200: ASCI search");

  // ------------------------------------------------ core precompute
  CoreData cd{};
  const int64_t U = core_setup<NBITS>(h, A, cdets, ncdets, C, st.just_singles, cd);

  // ------------------------------------------------ learned screening
  macis_b200_mlp* net = scr ? scr->net : nullptr;
  const bool screen = net && scr->use_net && U > 0;
  const bool record = net && scr->max_samples > 0 && U > 0;
  if(net)
    MB_REQUIRE(net->din == unit_din<NBITS>(), MACIS_B200_EINVAL,
               "screening network input width does not match the determinant width");
  stats.units_total = uint64_t(U);
  stats.units_kept = uint64_t(U);
  auto t_scr = std::chrono::steady_clock::now();
  uint8_t* umask = nullptr;
  float* umax = nullptr;
  if(record) {
    umax = A.get<float>(size_t(U));
    MB_CUDA(cudaMemsetAsync(umax, 0, size_t(U) * 4, s));
  }
  if(screen) {
    MB_REQUIRE(scr->keep_frac > 0 && scr->keep_frac <= 1 &&
                   scr->explore_frac >= 0 && scr->explore_frac <= 1,
               MACIS_B200_EINVAL, "keep_frac in (0,1], explore_frac in [0,1]");
    float* pred = A.get<float>(size_t(U));
    const size_t smem = mlp_fwd_smem_bytes(net->din);
    auto kern = mlp_fwd_k<UnitRows<NBITS>, false>;
    MB_CUDA(cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int64_t tiles = (U + MLP_TM - 1) / MLP_TM;
    cudaEvent_t ev[2];
    MB_CUDA(cudaEventCreate(&ev[0]));
    MB_CUDA(cudaEventCreate(&ev[1]));
    MB_CUDA(cudaEventRecord(ev[0], s));
    kern<<<unsigned(std::min<int64_t>(tiles, sms)), MLP_TM, smem, s>>>(
        mlp_weights(net), UnitRows<NBITS>{cd, E0}, U, pred, MlpTaps{},
        net->err, wait_limit_ns()), note_launch();
    MB_CUDA(cudaGetLastError());
    MB_CUDA(cudaEventRecord(ev[1], s));
    MB_CUDA(cudaEventSynchronize(ev[1]));
    float pms = 0.f;
    MB_CUDA(cudaEventElapsedTime(&pms, ev[0], ev[1]));
    stats.predict_ms = pms;
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    // threshold key of the keep-th largest prediction (MSD radix select)
    uint64_t need = uint64_t(std::ceil(scr->keep_frac * double(U)));
    need = std::min<uint64_t>(std::max<uint64_t>(need, 1), uint64_t(U));
    auto* hist = A.get<unsigned long long>(256);
    uint32_t prefix = 0, msk = 0;
    for(int shift = 24; shift >= 0; shift -= 8) {
      MB_CUDA(cudaMemsetAsync(hist, 0, 256 * 8, s));
      pred_hist_k<<<grid_for(size_t(U), 256, 8 * sms), 256, 0, s>>>(
          pred, size_t(U), prefix, msk, shift, hist), note_launch();
      unsigned long long hh[256];
      MB_CUDA(cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      int d = 255;
      for(; d > 0; --d) {
        if(hh[d] >= need) break;
        need -= hh[d];
      }
      prefix |= uint32_t(d) << shift;
      msk |= 255u << shift;
    }
    umask = A.get<uint8_t>(size_t(U));
    auto* nk = A.get<unsigned long long>(1);
    MB_CUDA(cudaMemsetAsync(nk, 0, 8, s));
    const double ex = scr->explore_frac * 18446744073709551616.0;
    const uint64_t explore =
        ex >= 18446744073709551615.0 ? ~uint64_t(0) : uint64_t(ex);
    unit_mask_k<<<grid_for(size_t(U), 256, 8 * sms), 256, 0, s>>>(
        pred, size_t(U), prefix, explore, scr->seed, umask, nk), note_launch();
    stats.units_kept = to_host(nk, s);
    check_net(net, s);
  }
  stats.screen_ms = ms_since(t_scr);

  // unit counts of the whole search (count pass over all units at once)
  int64_t* ucnt = A.get<int64_t>(U + 1);
  auto* dhist = A.get<unsigned long long>(ASCI_BINS);
  MB_CUDA(cudaMemsetAsync(dhist, 0, ASCI_BINS * 8, s));
  if(U) {
    const size_t hbytes = ASCI_BINS * sizeof(unsigned long long);
    MB_CUDA(cudaFuncSetAttribute(units_k<NBITS, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(hbytes)));
    units_k<NBITS, 0><<<grid_for(size_t(U), 256, 32 * sms), 256, hbytes,
                        s>>>(I, cd, 0, U, 0, ncdets, E0, st.h_el_tol, ucnt,
                             nullptr, nullptr, nullptr, umask, nullptr, 0u,
                             ASCI_BINS, 0u, 0u, dhist, AlphaLists{},
                             RankTables{}),
        note_launch();
  }
  int64_t* uout = A.get<int64_t>(U + 1);
  exclusive_scan<int64_t, int64_t>(ucnt, uout, size_t(U), uout + U, A);
  const int64_t Ptot = U ? to_host(uout + U, s) : 0;
  stats.raw_pairs = uint64_t(Ptot);

  // The candidate determinants are split into nr ranges by a hash of the
  // determinant, sized so that one range's raw contributions fit in memory.
  // Every contribution to a determinant lands in its range, so each range's
  // accumulated scores are complete (summed in generation order, as in the
  // unpartitioned search) and the range can go straight into the running
  // top-k: memory stays bounded by one range plus ~ndets_max candidates.
  // ranked candidate keys (RankTables) for searches above 2^22 raw
  // contributions (MACIS_B200_ASCI_RANKS: 0 off, 1 always)
  std::vector<uint64_t> hdets;  // the core dets on the host, for the plans
  auto host_dets = [&]() -> const std::vector<uint64_t>& {
    if(hdets.empty() && ncdets) {
      hdets.resize(ncdets * NW);
      MB_CUDA(cudaMemcpyAsync(hdets.data(), cdets, ncdets * NW * 8,
                              cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
    }
    return hdets;
  };
  SpinPlan pa;
  bool pa_done = false;
  auto alpha_plan = [&]() -> const SpinPlan& {
    if(!pa_done) pa = plan_spin<NBITS>(host_dets(), ncdets, h->norb, 0);
    pa_done = true;
    return pa;
  };
  RankTables rt;
  bool ranked = false;
  if constexpr(NBITS > 64) {
    const char* e = getenv("MACIS_B200_ASCI_RANKS");
    const bool force = e && e[0] == '1', off = e && e[0] == '0';
    if(U && !off && (force || Ptot >= (int64_t(1) << 22))) {
      auto t_rk = std::chrono::steady_clock::now();
      const SpinPlan& a = alpha_plan();
      const SpinPlan b = plan_spin<NBITS>(host_dets(), ncdets, h->norb, 1);
      if(a.nu && b.nu) {
        const int bits = build_ranks<NBITS>(a, b, ncdets, A, s, rt);
        ranked = bits > 0;
        stats.key_bits = uint64_t(bits);
      }
      stats.rank_ms = ms_since(t_rk);
    }
  }
  // bytes of a sorted record, and of a candidate with its determinant
  // (the unique candidates of a range, the survivors)
  const double rs = ranked ? 16.0 : double(NW * 8 + 8);
  const double rf = double(NW * 8 + 8);
  // per raw contribution while a range is processed, whichever phase holds
  // more: record + sort copy, flags and radix tables (sort); or the unique
  // candidates as determinants, their flags and kept copy and the running
  // top-k concatenation (few duplicates: unique ~ raw; 128 B at 256 bits,
  // more than a ranked-key record's sort)
  const double per_pair = std::max(4.0 * rs + 20.0, 3.0 * rf + 8.0);
  const size_t topk = ndets_max - ncdets;   // size_t arithmetic (:547)
  const double keep_reserve =
      6.0 * rf * double(std::min<uint64_t>(topk, uint64_t(Ptot)));
  // MACIS_B200_ASCI_BATCH_PAIRS caps the raw pairs per range (exercises the
  // partitioned path on small problems).
  int64_t cap = 0;
  const char* cap_env = getenv("MACIS_B200_ASCI_BATCH_PAIRS");
  if(const char* e = cap_env) {
    cap = std::max<int64_t>(1, atoll(e));
  } else {
    cap = int64_t((0.8 * double(device_bytes_available()) - keep_reserve) /
                  per_pair);
    cap = std::min<int64_t>(std::max<int64_t>(cap, int64_t(1) << 20),
                            int64_t(1) << 31);
  }
  // records per sort group of a range (MACIS_B200_ASCI_SORT_GROUP). Only
  // determinant keys are grouped by default: with ranked keys (16-byte
  // records) a range sorted whole was measured as fast as or faster than
  // any grouping (n = 48: 1e4 core dets 246 against 276 ms, 1e5 core dets
  // 3.48 s against 3.35-5.9 s for groups of 5e8-1.07e9 records)
  uint64_t sort_group_cap = ranked ? ~uint64_t(0) : uint64_t(4) << 28;
  if(const char* e = getenv("MACIS_B200_ASCI_SORT_GROUP"))
    sort_group_cap = std::max<uint64_t>(1, uint64_t(atoll(e)));
  // ranges: consecutive alpha-string bins packed up to the cap from the
  // measured bin loads (a single bin above the cap is a range of its own)
  // (a bin above the cap is split into beta-hash classes)
  std::vector<uint32_t> rlo, rhi, rns, rsub;
  auto add_range = [&](uint32_t lo, uint32_t hi, uint32_t ns, uint32_t sb) {
    rlo.push_back(lo);
    rhi.push_back(hi);
    rns.push_back(ns);
    rsub.push_back(sb);
  };
  // a part of a split search owns the bins [bin_lo, bin_hi): the cuts fall
  // where the cumulative bin load crosses index / count of the total (the
  // histogram, hence the cut, is the same on every part)
  uint32_t bin_lo = 0, bin_hi = ASCI_BINS;
  std::vector<unsigned long long> hh;
  auto load_hist = [&] {
    if(!hh.empty()) return;
    hh.resize(ASCI_BINS);
    MB_CUDA(cudaMemcpyAsync(hh.data(), dhist, ASCI_BINS * 8,
                            cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
  };
  uint64_t Ppart = uint64_t(Ptot);
  if(part && part->count > 1) {
    load_hist();
    auto cut = [&](uint32_t r) -> uint32_t {
      if(r == 0) return 0;
      if(r >= part->count) return ASCI_BINS;
      // first bin whose preceding load reaches r / count of the total
      const long double want =
          (long double)Ptot * (long double)r / (long double)part->count;
      unsigned long long c = 0;
      for(uint32_t b = 0; b < ASCI_BINS; ++b) {
        if((long double)c >= want) return b;
        c += hh[b];
      }
      return ASCI_BINS;
    };
    bin_lo = cut(part->index);
    bin_hi = std::max(bin_lo, cut(part->index + 1));
    Ppart = 0;
    for(uint32_t b = bin_lo; b < bin_hi; ++b) Ppart += hh[b];
  }
  // alpha lists (AlphaLists) when the ranges need count passes of their own:
  // bin tables for every distinct alpha string, and lists for as many of
  // the strings shared by the most core dets as fit 15 % of the free memory
  // (MACIS_B200_ASCI_ALPHA_LISTS: 0 none, N at most N listed strings); the
  // memory comes off the range size
  SpinPlan ap;
  int g_est = 0;
  size_t nlist = 0;
  const char* al_env = getenv("MACIS_B200_ASCI_ALPHA_LISTS");
  const long long al_max = al_env ? atoll(al_env) : -1;
  if(al_max != 0 && !pairs_only && !st.just_singles && bin_lo < bin_hi &&
     ((part && part->count > 1) || Ppart > uint64_t(cap))) {
    ap = alpha_plan();
    if(ap.nu) {
      g_est = int(std::min<uint64_t>(1024, 2 * ((Ppart + cap - 1) / cap) + 2));
      const double nk = double(ap.ne) * ap.nv;
      const double pairs2 = double(ap.ne) * (ap.ne - 1) / 2 * double(ap.nv) *
                            (ap.nv - 1) / 2;
      const double fixed = 4.0 * double(ncdets + 2 * ap.nu) +
                           2.0 * double(ap.nu) * (nk + 1.0) + 16384.0;
      const double per_list = nk * (18.0 + 2.0 * (g_est + 1)) + 2.0 * pairs2;
      const double budget = 0.15 * double(device_bytes_available()) - fixed;
      if(budget < 0) {
        ap = SpinPlan{};
      } else {
        nlist = std::min<size_t>(ap.nu, size_t(budget / per_list));
        if(al_max > 0) nlist = std::min<size_t>(nlist, size_t(al_max));
        const double bytes = fixed + double(nlist) * per_list;
        if(!cap_env)
          cap = std::max<int64_t>(cap - int64_t(bytes / per_pair), int64_t(1) << 20);
      }
    }
  }
  if(bin_lo == bin_hi) {
    // this part owns no bins: nothing to search
  } else if((Ppart <= uint64_t(cap) || pairs_only) && bin_lo == 0 &&
            bin_hi == ASCI_BINS) {  // pairs_only: the full list is the result
    add_range(0, ASCI_BINS, 0, 0);
  } else if(Ppart <= uint64_t(cap)) {
    add_range(bin_lo, bin_hi, 0, 0);
  } else {
    load_hist();
    uint32_t b0 = bin_lo;
    unsigned long long acc = 0;
    for(uint32_t b = bin_lo; b < bin_hi; ++b) {
      if(hh[b] > uint64_t(cap)) {
        if(acc) add_range(b0, b, 0, 0);
        const uint32_t ns = uint32_t(std::ceil(1.25 * double(hh[b]) / double(cap)));
        for(uint32_t k = 0; k < ns; ++k) add_range(b, b + 1, ns, k);
        b0 = b + 1;
        acc = 0;
        continue;
      }
      if(acc && acc + hh[b] > uint64_t(cap)) {
        add_range(b0, b, 0, 0);
        b0 = b;
        acc = 0;
      }
      acc += hh[b];
    }
    if(b0 < bin_hi) add_range(b0, bin_hi, 0, 0);
  }
  const uint32_t nr = uint32_t(rlo.size());
  stats.batches = nr;
  // groups of the alpha lists: the unsplit ranges
  std::vector<int> rgrp(nr, -1);
  AlphaLists al;
  if(ap.nu) {
    int G = 0;
    for(uint32_t r = 0; r < nr; ++r)
      if(rns[r] == 0) rgrp[r] = G++;
    if(G == 0) {
      std::fill(rgrp.begin(), rgrp.end(), -1);
    } else {
      // lists only where their memory was planned and they pay
      if(G > g_est || (G < 2 && 2 * ap.nu > ncdets)) nlist = 0;
      std::vector<uint16_t> gt(ASCI_BINS, 0xFFFFu);
      for(uint32_t r = 0; r < nr; ++r)
        if(rgrp[r] >= 0)
          for(uint32_t b = rlo[r]; b < rhi[r]; ++b) gt[b] = uint16_t(rgrp[r]);
      // list blocks: the alpha strings of the most core dets first
      std::vector<int32_t> mult(ap.nu, 0), order(ap.nu), lx(ap.nu, -1),
          lrep(nlist + 1, 0);
      for(size_t c = 0; c < ncdets; ++c) ++mult[ap.idx[c]];
      for(size_t u = 0; u < ap.nu; ++u) order[u] = int32_t(u);
      std::stable_sort(order.begin(), order.end(),
                       [&](int32_t x, int32_t y) { return mult[x] > mult[y]; });
      for(size_t b = 0; b < nlist; ++b) {
        lx[order[b]] = int32_t(b);
        lrep[b] = ap.rep[order[b]];
      }
      uint16_t* grp = A.get<uint16_t>(ASCI_BINS);
      MB_CUDA(cudaMemcpyAsync(grp, gt.data(), ASCI_BINS * 2,
                              cudaMemcpyHostToDevice, s));
      int32_t* aidx = A.get<int32_t>(ncdets);
      int32_t* rep = A.get<int32_t>(ap.nu);
      int32_t* lidx = A.get<int32_t>(ap.nu);
      int32_t* lrp = A.get<int32_t>(nlist + 1);
      MB_CUDA(cudaMemcpyAsync(aidx, ap.idx.data(), ncdets * 4,
                              cudaMemcpyHostToDevice, s));
      MB_CUDA(cudaMemcpyAsync(rep, ap.rep.data(), ap.nu * 4,
                              cudaMemcpyHostToDevice, s));
      MB_CUDA(cudaMemcpyAsync(lidx, lx.data(), ap.nu * 4,
                              cudaMemcpyHostToDevice, s));
      MB_CUDA(cudaMemcpyAsync(lrp, lrep.data(), (nlist + 1) * 4,
                              cudaMemcpyHostToDevice, s));
      al.aidx = aidx;
      al.lidx = lidx;
      al.NK = ap.ne * ap.nv;
      al.G = G;
      const size_t brows = ap.nu * size_t(al.NK);
      uint16_t* abin = A.get<uint16_t>(ap.nu);
      uint16_t* kbin = A.get<uint16_t>(brows + 1);
      al.abin = abin;
      al.kbin = kbin;
      if(brows)
        alpha_bins_k<NBITS><<<grid_for(brows, 256, 16 * sms), 256, 0, s>>>(
            cd, rep, ap.nu, ap.nv, al.NK, kbin, abin), note_launch();
      const size_t rows = nlist * size_t(al.NK);
      uint16_t* rel = A.get<uint16_t>(rows * (G + 1) + 1);
      int64_t* base = A.get<int64_t>(rows + 1);
      al.rel = rel;
      al.base = base;
      const size_t smem = 8 * size_t(G + 1) * sizeof(int);
      if(rows) {
        int64_t* tot = A.get<int64_t>(rows + 1);
        alpha_count_k<NBITS><<<grid_for(rows * 32, 256, 16 * sms), 256, smem,
                               s>>>(I, cd, lrp, nlist, ap.ne, ap.nv,
                                    st.h_el_tol, grp, al, rel, tot),
            note_launch();
        MB_CUDA(cudaGetLastError());
        exclusive_scan<int64_t, int64_t>(tot, base, rows, base + rows, A);
        A.release(tot);
      }
      const int64_t E = rows ? to_host(base + rows, s) : 0;
      uint16_t* ql = A.get<uint16_t>(size_t(E) + 1);
      al.q = ql;
      if(E)
        alpha_fill_k<NBITS><<<grid_for(rows * 32, 256, 16 * sms), 256, smem,
                              s>>>(I, cd, lrp, nlist, ap.ne, ap.nv,
                                   st.h_el_tol, grp, al, ql), note_launch();
      MB_CUDA(cudaGetLastError());
      stats.alpha_strings = nlist;
    }
  }
  stats.pairs_ms = ms_since(t_all);

  // sorted core dets (dropped from the candidates)
  uint64_t* core = A.get<uint64_t>(ncdets * NW + NW);
  if(ncdets) {
    uint64_t* ct = A.get<uint64_t>(ncdets * NW + NW);
    MB_CUDA(cudaMemcpyAsync(core, cdets, ncdets * NW * 8,
                            cudaMemcpyDeviceToDevice, s));
    radix_sort<NW, uint32_t>(core, nullptr, ct, nullptr, ncdets, A);
    A.release(ct);
  }

  // MSD radix select on |rv| bits: the bits T of the topk-th largest score
  // and how many entries equal to T still belong to the top-k.
  auto kth_bits = [&](const double* rv, size_t n, uint64_t want,
                      uint64_t* need_out) {
    auto* hist = A.get<unsigned long long>(256);
    uint64_t prefix = 0, mask = 0, need = want;
    for(int shift = 56; shift >= 0; shift -= 8) {
      MB_CUDA(cudaMemsetAsync(hist, 0, 256 * 8, s));
      select_hist_k<<<grid_for(n, 256, 8 * sms), 256, 0, s>>>(
          rv, n, prefix, mask, shift, hist), note_launch();
      unsigned long long hh[256];
      MB_CUDA(cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      int d = 255;
      for(; d > 0; --d) {
        if(hh[d] >= need) break;
        need -= hh[d];
      }
      prefix |= uint64_t(d) << shift;
      mask |= uint64_t(255) << shift;
    }
    A.release(hist);
    *need_out = need;
    return prefix;
  };
  // keep the flagged entries of (keys, rv, n) in new A-owned arrays
  auto compact_to = [&](Arena& W, const uint64_t* keys, const double* rv,
                        size_t n, const uint32_t* f) {
    uint32_t* fx = W.get<uint32_t>(n + 1);
    exclusive_scan<uint32_t, uint32_t>(f, fx, n, fx + n, W);
    Pairs o;
    o.n = to_host(fx + n, s);
    o.keys = A.get<uint64_t>(o.n * NW + NW);
    o.rv = A.get<double>(o.n + 1);
    if(n)
      compact_k<NW><<<grid_for(n, 256, 16 * sms), 256, 0, s>>>(
          keys, rv, n, f, fx, o.keys, o.rv), note_launch();
    W.release(fx);
    return o;
  };

  Pairs surv;  // running top-k candidates (ties at the threshold included)
  uint64_t tcut = 0;  // |rv| bits of its k-th score once it holds k
  uint64_t uniq_total = 0, kept_total = 0;
  double sort_ms = 0, pair_ms = 0, keep_ms = 0;
  for(uint32_t rr = 0; rr < nr; ++rr) {
    auto tb = std::chrono::steady_clock::now();
    NvtxRange nv_range("macis_b200: ASCI candidate range");
    Arena B(s);
    int64_t* rc = ucnt;
    int64_t* off = uout;
    int64_t P = Ptot;
    // the first count pass covered every bin: a range that does not (one of
    // several, or the share of a split search) is counted on its own
    if(nr > 1 || rlo[rr] != 0 || rhi[rr] != ASCI_BINS) {
      rc = B.get<int64_t>(U + 1);
      off = B.get<int64_t>(U + 1);
      if(rgrp[rr] >= 0) {
        AlphaLists alr = al;
        alr.g = rgrp[rr];
        range_count_k<<<grid_for(size_t(U), 256, 16 * sms), 256, 0, s>>>(
            cd, alr, U, ucnt, umask, rlo[rr], rhi[rr], rc), note_launch();
        // alpha singles and the alpha doubles of unlisted strings
        units_k<NBITS, 0><<<grid_for(size_t(U), 256, 32 * sms), 256, 0, s>>>(
            I, cd, 0, U, 0, ncdets, E0, st.h_el_tol, rc, nullptr, nullptr,
            nullptr, umask, nullptr, rlo[rr], rhi[rr], rns[rr], rsub[rr],
            nullptr, alr, RankTables{}), note_launch();
      } else {
        units_k<NBITS, 0><<<grid_for(size_t(U), 256, 32 * sms), 256, 0,
                            s>>>(I, cd, 0, U, 0, ncdets, E0, st.h_el_tol, rc,
                                 nullptr, nullptr, nullptr, umask, nullptr,
                                 rlo[rr], rhi[rr], rns[rr], rsub[rr], nullptr,
                                 AlphaLists{}, RankTables{}), note_launch();
      }
      exclusive_scan<int64_t, int64_t>(rc, off, size_t(U), off + U, B);
      P = to_host(off + U, s);
    }
    const size_t KWr = ranked ? 1 : NW;  // words per record key
    uint64_t* keys = B.get<uint64_t>(size_t(P) * KWr + KWr);
    double* rv = B.get<double>(size_t(P) + 1);
    if(P) {
      AlphaLists alr{};
      if(rgrp[rr] >= 0 && rc != ucnt) {
        alr = al;
        alr.g = rgrp[rr];
      }
      if(ranked)
        units_k<NBITS, 2><<<grid_for(size_t(U), 256, 32 * sms), 256, 0,
                            s>>>(I, cd, 0, U, 0, ncdets, E0, st.h_el_tol, rc,
                                 off, keys, rv, umask, umax, rlo[rr], rhi[rr],
                                 rns[rr], rsub[rr], nullptr, alr, rt),
            note_launch();
      else
        units_k<NBITS, 1><<<grid_for(size_t(U), 256, 32 * sms), 256, 0,
                            s>>>(I, cd, 0, U, 0, ncdets, E0, st.h_el_tol, rc,
                                 off, keys, rv, umask, umax, rlo[rr], rhi[rr],
                                 rns[rr], rsub[rr], nullptr, alr,
                                 RankTables{}), note_launch();
      MB_CUDA(cudaGetLastError());
    }
    MB_CUDA(cudaStreamSynchronize(s));
    pair_ms += ms_since(tb);
    tb = std::chrono::steady_clock::now();
    // sort + accumulate (stable: duplicates summed in generation order)
    Pairs uq;
    uint64_t* k2 = nullptr;
    double* r2 = nullptr;
    // KW key words per record; group(dg) the sort-group functor of a bin ->
    // group table
    auto accumulate = [&](auto kw, auto group) {
      constexpr int KW = decltype(kw)::value;
      k2 = B.get<uint64_t>(size_t(P) * KW + KW);
      r2 = B.get<double>(size_t(P) + 1);
      // a large range is first split by bin into groups that are sorted
      // one at a time: the digit passes of a sort over fewer records run
      // faster (measured: 12 passes over 6e8 records at 1.7x the rate of
      // 1.3e9), and equal determinants share a bin, so each group's sums
      // are complete and in generation order
      std::vector<size_t> goff{0, size_t(P)};
      if(!pairs_only && rns[rr] == 0 && rhi[rr] - rlo[rr] > 1 &&
         uint64_t(P) > sort_group_cap) {
        load_hist();
        std::vector<uint8_t> gt(ASCI_BINS, 0);
        int g = 0;
        unsigned long long acc = 0;
        for(uint32_t b = rlo[rr]; b < rhi[rr]; ++b) {
          if(acc && acc + hh[b] > sort_group_cap && g < 255) {
            ++g;
            acc = 0;
          }
          gt[b] = uint8_t(g);
          acc += hh[b];
        }
        if(g > 0) {
          uint8_t* dg = B.get<uint8_t>(ASCI_BINS);
          MB_CUDA(cudaMemcpyAsync(dg, gt.data(), ASCI_BINS,
                                  cudaMemcpyHostToDevice, s));
          goff = stable_partition<KW, double>(keys, rv, k2, r2, size_t(P),
                                              g + 1, group(dg), B);
          std::swap(keys, k2);
          std::swap(rv, r2);
          stats.sort_pass_items += uint64_t(P);
        }
      }
      for(size_t gi = 0; gi + 1 < goff.size(); ++gi) {
        const size_t a = goff[gi], m = goff[gi + 1] - a;
        stats.sort_pass_items +=
            uint64_t(radix_sort<KW, double>(keys + a * KW, rv + a,
                                            k2 + a * KW, r2 + a, m, B)) *
            uint64_t(m);
      }
      uint32_t* f = B.get<uint32_t>(size_t(P) + 1);
      uint32_t* fx = B.get<uint32_t>(size_t(P) + 1);
      seg_flags_k<KW><<<grid_for(size_t(P), 256, 16 * sms), 256, 0, s>>>(
          keys, size_t(P), f), note_launch();
      exclusive_scan<uint32_t, uint32_t>(f, fx, size_t(P), fx + P, B);
      const uint32_t nu = to_host(fx + P, s);
      int64_t* start = B.get<int64_t>(nu + 1);
      // unique keys into k2, sums into r2
      seg_starts_k<KW><<<grid_for(size_t(P), 256, 16 * sms), 256, 0, s>>>(
          f, fx, size_t(P), start, keys, k2), note_launch();
      seg_sum_k<<<grid_for(nu, 256, 16 * sms), 256, 0, s>>>(
          start, nu, size_t(P), rv, r2), note_launch();
      // the raw records are summed: release them before the keep / top-k
      for(void* q : {static_cast<void*>(f), static_cast<void*>(fx),
                     static_cast<void*>(start), static_cast<void*>(keys),
                     static_cast<void*>(rv)})
        B.release(q);
      return nu;
    };
    if(P) {
      uint32_t nu = 0;
      if(ranked) {
        nu = accumulate(std::integral_constant<int, 1>{},
                        [&](const uint8_t* dg) {
                          return RankBinGroup{
                              dg, rt.bin_a, (uint64_t(1) << rt.bits_a) - 1};
                        });
        // ranked keys back to determinants
        uint64_t* kd = B.get<uint64_t>(size_t(nu) * NW + NW);
        if(nu)
          unrank_k<NBITS><<<grid_for(nu, 256, 16 * sms), 256, 0, s>>>(
              k2, nu, rt, kd), note_launch();
        B.release(k2);
        k2 = kd;
      } else {
        nu = accumulate(std::integral_constant<int, NW>{},
                        [&](const uint8_t* dg) { return BinGroup<NBITS>{dg}; });
      }
      uq.keys = k2;
      uq.rv = r2;
      uq.n = nu;
    }
    uniq_total += uq.n;
    // pruning when the accumulated lists outgrow pair_size_max
    // (determinant_search.hpp:121-137)
    if(uq.n && uniq_total > st.pair_size_max) {
      uint32_t* f = B.get<uint32_t>(uq.n + 1);
      prune_flags_k<<<grid_for(uq.n, 256, 16 * sms), 256, 0, s>>>(
          uq.rv, uq.n, st.rv_prune_tol, f), note_launch();
      Pairs p2 = compact_to(B, uq.keys, uq.rv, uq.n, f);
      uq = p2;  // A-owned now
    }
    MB_CUDA(cudaStreamSynchronize(s));
    sort_ms += ms_since(tb);

    if(pairs_only) {  // nr == 1: the accumulated list is the answer
      ps->resize(uq.n * NW);
      pr->resize(uq.n);
      if(uq.n) {
        MB_CUDA(cudaMemcpyAsync(ps->data(), uq.keys, uq.n * NW * 8,
                                cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(pr->data(), uq.rv, uq.n * 8,
                                cudaMemcpyDeviceToHost, s));
      }
      MB_CUDA(cudaStreamSynchronize(s));
      continue;
    }
    // drop core dets and zero scores (keep_only_largest_copy_asci_pairs +
    // partition, determinant_sort.hpp:86-120, determinant_search.hpp:528-544)
    tb = std::chrono::steady_clock::now();
    Pairs kept;
    if(uq.n) {
      uint32_t* f = B.get<uint32_t>(uq.n + 1);
      keep_flags_k<NW><<<grid_for(uq.n, 256, 16 * sms), 256, 0, s>>>(
          uq.keys, uq.rv, uq.n, core, ncdets, tcut, f), note_launch();
      kept = compact_to(B, uq.keys, uq.rv, uq.n, f);
    }
    kept_total += kept.n;
    // running top-k: survivors + this range, cut at the topk-th score (all
    // entries tied with it stay)
    Pairs cat;
    cat.n = surv.n + kept.n;
    if(surv.n == 0) {  // the first candidates: no copy
      cat = kept;
      kept = Pairs{};
    } else {
      cat.keys = A.get<uint64_t>(cat.n * NW + NW);
      cat.rv = A.get<double>(cat.n + 1);
    }
    if(surv.n) {
      MB_CUDA(cudaMemcpyAsync(cat.keys, surv.keys, surv.n * NW * 8,
                              cudaMemcpyDeviceToDevice, s));
      MB_CUDA(cudaMemcpyAsync(cat.rv, surv.rv, surv.n * 8,
                              cudaMemcpyDeviceToDevice, s));
      A.release(surv.keys);
      A.release(surv.rv);
    }
    if(kept.n) {
      MB_CUDA(cudaMemcpyAsync(cat.keys + surv.n * NW, kept.keys,
                              kept.n * NW * 8, cudaMemcpyDeviceToDevice, s));
      MB_CUDA(cudaMemcpyAsync(cat.rv + surv.n, kept.rv, kept.n * 8,
                              cudaMemcpyDeviceToDevice, s));
      A.release(kept.keys);
      A.release(kept.rv);
    }
    if(uq.keys != k2) {  // pruned copy lives in A
      A.release(uq.keys);
      A.release(uq.rv);
    }
    if(cat.n > topk) {
      uint64_t need = 0;
      const uint64_t T = kth_bits(cat.rv, cat.n, topk, &need);
      tcut = T;
      uint32_t* f = B.get<uint32_t>(cat.n + 1);
      ge_flags_k<<<grid_for(cat.n, 256, 16 * sms), 256, 0, s>>>(
          cat.rv, cat.n, T, f), note_launch();
      surv = compact_to(B, cat.keys, cat.rv, cat.n, f);
      A.release(cat.keys);
      A.release(cat.rv);
    } else {
      surv = cat;
    }
    MB_CUDA(cudaStreamSynchronize(s));
    keep_ms += ms_since(tb);
  }
  stats.unique_pairs = uniq_total;
  stats.kept_pairs = kept_total;
  stats.pairs_ms += pair_ms;
  stats.sort_ms = sort_ms;
  stats.keep_ms = keep_ms;

  // ---------------------------- (unit features, exact log score) samples
  if(record) {
    t_scr = std::chrono::steady_clock::now();
    const size_t rcap = size_t(scr->max_samples);
    const double cand = double(stats.units_kept);
    const double frac = double(rcap) / std::max(cand, 1.0);
    const uint64_t p =
        frac >= 1.0 ? ~uint64_t(0) : uint64_t(frac * 18446744073709551616.0);
    uint32_t* f = A.get<uint32_t>(size_t(U) + 1);
    uint32_t* fx = A.get<uint32_t>(size_t(U) + 1);
    sample_flags_k<<<grid_for(size_t(U), 256, 16 * sms), 256, 0, s>>>(
        umask, size_t(U), p, scr->seed + 1, f), note_launch();
    exclusive_scan<uint32_t, uint32_t>(f, fx, size_t(U), fx + U, A);
    const size_t nrec = std::min<size_t>(to_host(fx + U, s), rcap);
    int64_t* list = A.get<int64_t>(nrec + 1);
    sample_list_k<<<grid_for(size_t(U), 256, 16 * sms), 256, 0, s>>>(
        f, fx, size_t(U), nrec, list), note_launch();
    MB_CUDA(cudaStreamSynchronize(s));
    mlp_reserve_samples(net, rcap);
    if(nrec)
      unit_rows_k<NBITS><<<grid_for(nrec, 128, 16 * sms), 128, 0, s>>>(
          cd, E0, list, 0, nrec, net->xs, umax, net->ts), note_launch();
    MB_CUDA(cudaGetLastError());
    MB_CUDA(cudaStreamSynchronize(s));
    net->ns = nrec;
    stats.samples = nrec;
    stats.screen_ms += ms_since(t_scr);
  }

  if(pairs_only) {
    h->last_asci = stats;
    return;
  }
  if(part) {
    // the part's running top-k, ties at its cut included: the union over
    // the parts holds the whole search's top-k
    h->part_states.resize(surv.n * NW);
    h->part_scores.resize(surv.n);
    if(surv.n) {
      MB_CUDA(cudaMemcpyAsync(h->part_states.data(), surv.keys,
                              surv.n * NW * 8, cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaMemcpyAsync(h->part_scores.data(), surv.rv, surv.n * 8,
                              cudaMemcpyDeviceToHost, s));
    }
    MB_CUDA(cudaStreamSynchronize(s));
    stats.total_ms = ms_since(t_all);
    h->last_asci = stats;
    return;
  }

  // ------------------------------------------------------------- top-k
  // Ties at the topk-th score go to the smaller determinants
  // (determinant_search.hpp:622-626 leaves them unspecified); the result is
  // returned in ascending determinant order.
  auto tt = std::chrono::steady_clock::now();
  Pairs selp = surv;
  if(surv.n > topk) {
    uint64_t need = 0;
    const uint64_t T = kth_bits(surv.rv, surv.n, topk, &need);
    uint32_t* gt = A.get<uint32_t>(surv.n + 1);
    uint32_t* eq = A.get<uint32_t>(surv.n + 1);
    select_flags_k<<<grid_for(surv.n, 256, 16 * sms), 256, 0, s>>>(
        surv.rv, surv.n, T, gt, eq), note_launch();
    // the need-th smallest tied determinant
    uint32_t* eqx = A.get<uint32_t>(surv.n + 1);
    exclusive_scan<uint32_t, uint32_t>(eq, eqx, surv.n, eqx + surv.n, A);
    const uint32_t neq = to_host(eqx + surv.n, s);
    Key<NW> kmax;
    {
      uint64_t* ek = A.get<uint64_t>(size_t(neq) * NW + NW);
      uint64_t* ek2 = A.get<uint64_t>(size_t(neq) * NW + NW);
      double* dummy = A.get<double>(neq + 1);
      compact_k<NW><<<grid_for(surv.n, 256, 16 * sms), 256, 0, s>>>(
          surv.keys, surv.rv, surv.n, eq, eqx, ek, dummy), note_launch();
      radix_sort<NW, uint32_t>(ek, nullptr, ek2, nullptr, neq, A);
      MB_REQUIRE(need >= 1 && need <= neq, MACIS_B200_EINVAL,
                 "internal: tie count out of range in the top-k selection");
      MB_CUDA(cudaMemcpyAsync(kmax.w, ek + (need - 1) * NW, NW * 8,
                              cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
    }
    uint32_t* sel = A.get<uint32_t>(surv.n + 1);
    tie_select_k<NW><<<grid_for(surv.n, 256, 16 * sms), 256, 0, s>>>(
        surv.keys, gt, eq, surv.n, kmax, sel), note_launch();
    selp = compact_to(A, surv.keys, surv.rv, surv.n, sel);
  }
  const size_t nsel = selp.n;
  MB_REQUIRE(nsel <= ndets_max, MACIS_B200_ECAPACITY,
             "ASCI search result exceeds ndets_max + ncdets determinants");
  if(nsel) {
    uint64_t* k2 = A.get<uint64_t>(nsel * NW + NW);
    radix_sort<NW, uint32_t>(selp.keys, nullptr, k2, nullptr, nsel, A);
    MB_CUDA(cudaMemcpyAsync(out_dets, selp.keys, nsel * NW * 8,
                            cudaMemcpyDeviceToDevice, s));
  }
  if(ncdets)
    MB_CUDA(cudaMemcpyAsync(out_dets + nsel * NW, cdets, ncdets * NW * 8,
                            cudaMemcpyDeviceToDevice, s));
  *nout = nsel + ncdets;
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(s));
  stats.topk_ms = ms_since(tt);
  stats.total_ms = ms_since(t_all);
  h->last_asci = stats;
}

void asci_search_device(macis_b200_ham* h, const macis_b200_asci_settings& s,
                        const macis_b200_asci_screen* scr, size_t ndets_max,
                        const uint64_t* cdets, size_t ncdets, double E0,
                        const double* C, uint64_t* out_dets, size_t* nout,
                        std::vector<uint64_t>* ps, std::vector<double>* pr,
                        bool pairs_only, const AsciPart* part) {
  MB_REQUIRE(h->norb <= MAXORB, MACIS_B200_EINVAL, "norb too large for ASCI");
  if(h->nbits == 64)
    asci_impl<64>(h, s, scr, ndets_max, cdets, ncdets, E0, C, out_dets, nout,
                  ps, pr, pairs_only, part);
  else if(h->nbits == 128)
    asci_impl<128>(h, s, scr, ndets_max, cdets, ncdets, E0, C, out_dets, nout,
                   ps, pr, pairs_only, part);
  else
    asci_impl<256>(h, s, scr, ndets_max, cdets, ncdets, E0, C, out_dets, nout,
                   ps, pr, pairs_only, part);
}

template <int NBITS>
static int64_t unit_features_impl(macis_b200_ham* h, const uint64_t* cdets,
                                  size_t ncdets, double E0, const double* C,
                                  size_t first, size_t n, uint16_t* X) {
  Arena A(h->stream);
  CoreData cd{};
  const int64_t U = core_setup<NBITS>(h, A, cdets, ncdets, C, 0, cd);
  if(X && n) {
    MB_REQUIRE(first + n <= size_t(U), MACIS_B200_EINVAL,
               "unit range outside the search's units");
    unit_rows_k<NBITS><<<grid_for(n, 128, 16 * num_sms()), 128, 0, h->stream>>>(
        cd, E0, nullptr, int64_t(first), n, X, nullptr, nullptr), note_launch();
    MB_CUDA(cudaGetLastError());
  }
  MB_CUDA(cudaStreamSynchronize(h->stream));
  return U;
}

int64_t asci_unit_features_device(macis_b200_ham* h, const uint64_t* cdets,
                                  size_t ncdets, double E0, const double* C,
                                  size_t first, size_t n, uint16_t* X) {
  MB_REQUIRE(h->norb <= MAXORB, MACIS_B200_EINVAL, "norb too large for ASCI");
  if(h->nbits == 64)
    return unit_features_impl<64>(h, cdets, ncdets, E0, C, first, n, X);
  if(h->nbits == 128)
    return unit_features_impl<128>(h, cdets, ncdets, E0, C, first, n, X);
  return unit_features_impl<256>(h, cdets, ncdets, E0, C, first, n, X);
}

int asci_unit_din(int nbits) {
  return nbits == 256 ? unit_din<256>() : unit_din<64>();
}

}  // namespace mb

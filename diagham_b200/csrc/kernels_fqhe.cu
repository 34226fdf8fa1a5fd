// Pull-form, atomic-free H.x for spin-polarised fermions on the sphere (sm_100a).
//
// One thread owns one basis row r; the 32 lanes of a warp own 32 consecutive rows, so rows that
// share their high orbitals (most of a warp) walk the same (m1, m2) pairs in lock-step and the
// gathers of moves confined to high orbitals land on consecutive x entries (coalesced).
//
// Per row (FermionOnSphere word s, bit m = orbital m):
//   for every occupied pair m1 > m2 (descending), a = s - m1 - m2, M = m1 + m2:
//     the admissible creations m3 > m4 = M - m3 (both empty in a) are the set bits of
//       e & mirror_M(e) & [m3 > M/2],  e = empty orbitals of a,  mirror_M(e) bit p = e bit (M - p)
//     sign = (-1)^(1 + |s in (m2, m1)| + |a in (m4, m3)|)  -- the AA * AdAd sign of
//            FermionOnSphere::AA (FermionOnSphere.cc:790) and ::AdAd (:949), from popcounts
//     target t = a + m3 + m4, index(t) = high_offset[t >> LB] + low_rank[t & (2^LB - 1)]
//            (or DiagHam's lookup table + binary search, FermionOnSphere.cc:1431)
//     y[r] += sign * factor(m1, m2, m3) * x[index(t)]
// H is real symmetric, so this pull form equals the reference's push form
// (AbstractQHEOnSphereHamiltonian.cc:456-488) up to FP rounding.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"

namespace dh {

namespace {

constexpr int kMatvecThreads = 256;

__device__ __forceinline__ uint64_t between_mask(int lo, int hi) {
  // bits strictly between lo and hi (lo < hi <= 63)
  return ((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull);
}

__device__ __forceinline__ uint64_t mirror_bits(uint64_t e, int M) {
  // bit p of the result = bit (M - p) of e (0 when M - p is outside 0..63)
  uint64_t r = __brevll(e);
  return (M <= 63) ? (r >> (63 - M)) : (r << (M - 63));
}

struct SmemLayout {
  int factor_bytes;
  int pair_bytes;
  int lookup_bytes;
  int total;
};

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }

inline SmemLayout smem_layout(const FqheDevice& f, int elem) {
  SmemLayout s;
  s.factor_bytes = align16(f.nbr_factors * elem);
  s.pair_bytes = align16(f.nbr_pairs * (int)sizeof(int));
  s.lookup_bytes = 0;
  if (f.index_mode == DH_INDEX_RANK && f.kernel_variant == 2) s.lookup_bytes = align16((1 << f.low_bits) * 2);
  if (f.index_mode == DH_INDEX_LOOKUP)
    s.lookup_bytes = align16((f.lz_max + 1) * ((1 << f.lookup_bits) + 1) * (int)sizeof(int)) +
                     align16((f.lz_max + 1) * (int)sizeof(int));
  s.total = s.factor_bytes + s.pair_bytes + s.lookup_bytes;
  return s;
}

template <int MODE>
__device__ __forceinline__ long long target_index(const FqheDevice& f, uint64_t t, const int* slookup,
                                                  const int* sshift) {
  if (MODE == DH_INDEX_RANK) {
    const int lb = f.low_bits;
    return (long long)__ldg(f.high_offset + (t >> lb)) + (long long)__ldg(f.low_rank + (t & ((1ull << lb) - 1ull)));
  } else {
    // FermionOnSphere::FindStateIndex: the highest-bit table brackets a binary search on the
    // descending word array (bracket [t[v + 1], t[v]], FermionOnSphere.cc:1431-1455)
    const int l = 63 - __clzll(t);
    const int width = (1 << f.lookup_bits) + 1;
    const long long v = (long long)(t >> sshift[l]);
    long long lo = slookup[l * width + v + 1];
    long long hi = slookup[l * width + v];
    while (hi - lo > 1) {
      long long mid = (lo + hi) >> 1;
      if (__ldg(f.words + mid) > t)
        lo = mid;
      else
        hi = mid;
    }
    return (__ldg(f.words + lo) == t) ? lo : hi;
  }
}

template <typename T>
__device__ __forceinline__ T load_x(const T* p) {
  return __ldg(p);
}

template <typename TG, int K, int MODE, bool RANGE>
__global__ void __launch_bounds__(kMatvecThreads) fqhe_matvec_kernel(FqheDevice f, MatvecArgs a, SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  int* spair = reinterpret_cast<int*>(smem + lay.factor_bytes);
  int* slookup = reinterpret_cast<int*>(smem + lay.factor_bytes + lay.pair_bytes);
  int* sshift = slookup + ((MODE == DH_INDEX_LOOKUP) ? (f.lz_max + 1) * ((1 << f.lookup_bits) + 1) : 0);

  const TG* gfac = static_cast<const TG*>(f.factors);
  for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
  for (int i = threadIdx.x; i < f.nbr_pairs; i += blockDim.x) spair[i] = f.pair_offset[i];
  if (MODE == DH_INDEX_LOOKUP) {
    const int n = (f.lz_max + 1) * ((1 << f.lookup_bits) + 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) slookup[i] = f.lookup[i];
    for (int i = threadIdx.x; i <= f.lz_max; i += blockDim.x) sshift[i] = f.lookup_shift[i];
  }
  __syncthreads();

  const TG* x = static_cast<const TG*>(a.x);
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : f.dim;
  for (long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    uint64_t rem1 = s;
    while (rem1) {
      const int m1 = 63 - __clzll(rem1);
      rem1 &= ~(1ull << m1);
      uint64_t rem2 = rem1;
      const int pbase = m1 * (m1 - 1) / 2;
      while (rem2) {
        const int m2 = 63 - __clzll(rem2);
        rem2 &= ~(1ull << m2);
        const uint64_t an = s & ~((1ull << m1) | (1ull << m2));
        const int M = m1 + m2;
        const int paa = 1 + __popcll(s & between_mask(m2, m1));
        const uint64_t e = ~an & full;
        uint64_t valid = e & mirror_bits(e, M) & (~0ull << (M / 2 + 1));
        const TG* fp = sfac + (spair[pbase + m2] - (M / 2 + 1));
        while (valid) {
          const int m3 = __ffsll(valid) - 1;
          valid &= valid - 1ull;
          const int m4 = M - m3;
          const uint64_t t = an | (1ull << m3) | (1ull << m4);
          const int par = paa + __popcll(an & between_mask(m4, m3));
          const long long idx = target_index<MODE>(f, t, slookup, sshift);
          if (RANGE && (idx < a.col_first || idx >= a.col_last)) continue;
          TG fct = fp[m3];
          if (par & 1) fct = -fct;
          const TG* xp = x + idx * a.ld;
#pragma unroll
          for (int j = 0; j < K; ++j) acc[j] += fct * load_x(xp + j * a.vstride);
        }
      }
    }
    const bool diag = (r >= a.row_first && r < a.row_last);
    double* y = static_cast<double*>(a.y);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double v = (double)acc[j];
      if (diag && a.shift != 0.0) {
        double xd = a.xdiag ? a.xdiag[r * a.ld + j * a.vstride] : (double)x[r * a.ld + j * a.vstride];
        v += a.shift * xd;
      }
      double* yp = y + r * a.ld_y + j * a.vstride_y;
      *yp = a.accumulate ? (*yp + v) : v;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Rank-mode product, split-word form.  The word is handled as a low half (orbitals 0..LB-1) and a
// high half (LB..lz_max), the two halves of the rank tables: index(t) = HO[t_high] + LR[t_low].
// Per row, HO of the row's own high half is loaded once and LR of its low half is r - HO.  Per
// annihilated pair, whichever half the pair leaves untouched keeps the row's table value, so
//   creations in the low half only  (m4 < m3 < LB):  one LR load,
//   creations in the high half only (LB <= m4 < m3): one HO load,
//   mixed creations (m4 < LB <= m3):                 one LR and one HO load,
// all in 32-bit arithmetic.  Two creations are processed per iteration so that two independent
// table-load -> gather chains are in flight per thread.
__device__ __forceinline__ uint32_t between32(int lo, int hi) {
  // bits strictly between lo and hi, 0 <= lo < hi <= 32
  const uint32_t upto = (hi >= 32) ? 0xffffffffu : ((1u << hi) - 1u);
  return upto & ~((2u << lo) - 1u);
}

// K gathered values of target row idx: interleaved blocks ([row][K], IL) load them as one vector.
// W256: the FP64 block of 4 with 32-byte aligned rows, one 256-bit load per row that bypasses L1
// (the 248 MB block at N=12, 2S=33 does not fit L1 or L2; L1 is left to the rank tables)
template <typename TG, int K, bool IL, bool W256 = false>
__device__ __forceinline__ void load_row(const TG* x, const MatvecArgs& a, int idx, TG (&v)[K]) {
  if constexpr (IL) {
    const TG* p = x + (long long)idx * K;
    if constexpr (W256 && sizeof(TG) == 8 && K == 4) {
      ldg_row32_no_l1(reinterpret_cast<const double*>(p), *reinterpret_cast<double(*)[4]>(&v));
    } else if constexpr (sizeof(TG) == 4 && K == 4) {
      // the FP32 block of 4 (124 MB at N=12, 2S=33) lives in L2: its gathers skip L1, which keeps L1
      // for the rank tables (9.60-9.65 ms per step against 9.68-9.75 ms with cached gathers)
      const float4 q = __ldcg(reinterpret_cast<const float4*>(p));
      v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else if constexpr (sizeof(TG) == 4 && K == 2) {
      const float2 q = __ldg(reinterpret_cast<const float2*>(p));
      v[0] = q.x; v[1] = q.y;
    } else if constexpr (sizeof(TG) == 8 && (K == 2 || K == 4)) {
#pragma unroll
      for (int j = 0; j < K; j += 2) {
        const double2 q = __ldg(reinterpret_cast<const double2*>(p) + j / 2);
        v[j] = q.x;
        v[j + 1] = q.y;
      }
    } else {
#pragma unroll
      for (int j = 0; j < K; ++j) v[j] = __ldg(p + j);
    }
  } else {
    if (K == 1 && a.ld == 1) {
      v[0] = __ldg(x + idx);
      return;
    }
    const TG* p = x + (long long)idx * a.ld;
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = __ldg(p + j * a.vstride);
  }
}

// acc + fa xa + fb xb with the roundings fixed: fb xb, then fused with fa xa, then added to acc
// (left to the compiler, the contraction into FMAs may differ between launch forms)
__device__ __forceinline__ double pair_term(double acc, double fa, double xa, double fb, double xb) {
  return __dadd_rn(acc, __fma_rn(fa, xa, __dmul_rn(fb, xb)));
}
__device__ __forceinline__ float pair_term(float acc, float fa, float xa, float fb, float xb) {
  return __fadd_rn(acc, __fmaf_rn(fa, xa, __fmul_rn(fb, xb)));
}

// The gathers of a row's elements, two targets per call.  PIPE: the two loads of a call are issued
// before the previous call's values are used, so four target rows are in flight per thread; the
// pairs are added in the same order and with the same roundings either way (identical results).
template <typename TG, int K, bool RANGE, bool IL, bool W256, bool PIPE>
struct Gatherer {
  TG pa[K], pb[K];
  TG pfa, pfb;
  __device__ __forceinline__ Gatherer() : pfa(TG(0)), pfb(TG(0)) {
#pragma unroll
    for (int j = 0; j < K; ++j) pa[j] = pb[j] = TG(0);
  }
  __device__ __forceinline__ void add2(TG (&acc)[K], const TG* x, const MatvecArgs& a, int ia, TG fa, int ib, TG fb) {
    if (RANGE) {
      if (ia < a.col_first || ia >= a.col_last) fa = TG(0);
      if (ib < a.col_first || ib >= a.col_last) fb = TG(0);
    }
    TG xa[K], xb[K];
    load_row<TG, K, IL, W256>(x, a, ia, xa);
    load_row<TG, K, IL, W256>(x, a, ib, xb);
    if constexpr (PIPE) {
#pragma unroll
      for (int j = 0; j < K; ++j) acc[j] = pair_term(acc[j], pfa, pa[j], pfb, pb[j]);
#pragma unroll
      for (int j = 0; j < K; ++j) {
        pa[j] = xa[j];
        pb[j] = xb[j];
      }
      pfa = fa;
      pfb = fb;
    } else {
#pragma unroll
      for (int j = 0; j < K; ++j) acc[j] = pair_term(acc[j], fa, xa[j], fb, xb[j]);
    }
  }
  __device__ __forceinline__ void finish(TG (&acc)[K]) {
    if constexpr (PIPE) {
#pragma unroll
      for (int j = 0; j < K; ++j) acc[j] = pair_term(acc[j], pfa, pa[j], pfb, pb[j]);
    }
  }
};

// the rank tables and words of one sector
struct SplitTables {
  const uint64_t* words;
  const int32_t* HO;
  const uint16_t* LR;
  int LB;
  uint64_t full;
};

// Off-diagonal elements of row r accumulated into acc (K vectors) and the sum of its diagonal
// factors into dsum; the caller adds dsum * x[r] and the shift.
template <typename TG, int K, bool RANGE, bool IL, bool W256 = false, bool PIPE = false>
__device__ __forceinline__ void split_row(const SplitTables& t, const TG* sfac, const int* spair, long long r,
                                          const TG* x, const MatvecArgs& a, TG (&acc)[K], TG& dsum) {
  Gatherer<TG, K, RANGE, IL, W256, PIPE> g;
  const int LB = t.LB;
  const uint32_t lmask = (1u << LB) - 1u;
  const int32_t* __restrict__ HO = t.HO;
  const uint16_t* __restrict__ LR = t.LR;
  const uint64_t s = __ldg(t.words + r);
  const uint32_t sl = (uint32_t)s & lmask;
  const uint32_t sh = (uint32_t)(s >> LB);
  const int ho_row = __ldg(HO + sh);
  const int lr_row = (int)(r - ho_row);
  // a non-diagonal creation pair is empty in the row itself, so its admissible m3 for the sum M
  // are E & mirror_M(E) above M/2; the bit reversal of E is taken once per row
  const uint64_t E = ~s & t.full;
  const uint64_t RE = __brevll(E);
  // exclusive prefix parity of s: bit k = parity of the occupied orbitals below k
  uint64_t pp = s;
  pp ^= pp << 1;
  pp ^= pp << 2;
  pp ^= pp << 4;
  pp ^= pp << 8;
  pp ^= pp << 16;
  pp ^= pp << 32;
  pp <<= 1;
  // diagonal elements: (m3, m4) = (m1, m2) is admissible for every occupied pair and its
  // AA * AdAd sign is -1, so they add -sum(factor(m1, m2, m1)) * x[r]
  uint64_t rem1 = s;
  while (rem1) {
    const int m1 = 63 - __clzll(rem1);
    rem1 &= ~(1ull << m1);
    uint64_t rem2 = rem1;
    const int pbase = m1 * (m1 - 1) / 2;
    const int p1 = (int)(pp >> m1) & 1;
    while (rem2) {
      const int m2 = 63 - __clzll(rem2);
      rem2 &= ~(1ull << m2);
      const int M = m1 + m2;
      const TG* fp = sfac + (spair[pbase + m2] - (M / 2 + 1));
      dsum -= fp[m1];
      const uint64_t mir = (M <= 63) ? (RE >> (63 - M)) : (RE << (M - 63));
      const uint64_t valid = E & mir & (~0ull << (M / 2 + 1));
      if (!valid) continue;
      // AA sign parity: 1 + occupied orbitals strictly between m2 and m1
      const int paa = 1 ^ p1 ^ ((int)(pp >> (m2 + 1)) & 1);
      const uint32_t anl = sl & ~((m1 < LB ? (1u << m1) : 0u) | (m2 < LB ? (1u << m2) : 0u));
      const uint32_t anh = sh & ~((m1 >= LB ? (1u << (m1 - LB)) : 0u) | (m2 >= LB ? (1u << (m2 - LB)) : 0u));
      // split the admissible m3 into three 32-bit masks:
      //   vl: m3 < LB (creations in the low half), bit m3
      //   vh: m4 = M - m3 >= LB (creations in the high half), bit m3 - LB
      //   vm: m4 < LB <= m3 (mixed), bit m3 - LB
      uint32_t vl = (uint32_t)valid & lmask;
      const uint64_t hv = valid >> LB;
      const int hcut = M - 2 * LB;  // relative m3 - LB <= M - 2 LB  <=>  m4 >= LB
      const uint64_t hkeep = (hcut < 0) ? 0ull : ((hcut >= 63) ? ~0ull : ((2ull << hcut) - 1ull));
      uint32_t vh = (uint32_t)(hv & hkeep);
      uint32_t vm = (uint32_t)(hv & ~hkeep);
      if (vl) {
        const int base = (m1 < LB) ? ho_row : __ldg(HO + anh);
        while (vl) {
          const int m3a = __ffs(vl) - 1;
          vl &= vl - 1u;
          const bool two = vl != 0u;
          const int m3b = two ? __ffs(vl) - 1 : m3a;
          vl &= vl - 1u;
          const int m4a = M - m3a, m4b = M - m3b;
          const int ia = base + LR[anl | (1u << m3a) | (1u << m4a)];
          const int ib = base + LR[anl | (1u << m3b) | (1u << m4b)];
          TG fa = fp[m3a], fb = two ? fp[m3b] : TG(0);
          if ((paa + __popc(anl & between32(m4a, m3a))) & 1) fa = -fa;
          if ((paa + __popc(anl & between32(m4b, m3b))) & 1) fb = -fb;
          g.add2(acc, x, a, ia, fa, ib, fb);
        }
      }
      if (vh) {
        const int base = (m2 >= LB) ? lr_row : LR[anl];
        const TG* fph = fp + LB;
        const int MH = M - 2 * LB;
        while (vh) {
          const int ha3 = __ffs(vh) - 1;
          vh &= vh - 1u;
          const bool two = vh != 0u;
          const int hb3 = two ? __ffs(vh) - 1 : ha3;
          vh &= vh - 1u;
          const int ha4 = MH - ha3, hb4 = MH - hb3;
          const int ia = base + __ldg(HO + (anh | (1u << ha3) | (1u << ha4)));
          const int ib = base + __ldg(HO + (anh | (1u << hb3) | (1u << hb4)));
          TG fa = fph[ha3], fb = two ? fph[hb3] : TG(0);
          if ((paa + __popc(anh & between32(ha4, ha3))) & 1) fa = -fa;
          if ((paa + __popc(anh & between32(hb4, hb3))) & 1) fb = -fb;
          g.add2(acc, x, a, ia, fa, ib, fb);
        }
      }
      if (vm) {
        // m4 < LB <= m3: the orbitals between them are the low ones above m4 and the high ones below m3
        const TG* fph = fp + LB;
        const int ML = M - LB;
        while (vm) {
          const int ha3 = __ffs(vm) - 1;
          vm &= vm - 1u;
          const bool two = vm != 0u;
          const int hb3 = two ? __ffs(vm) - 1 : ha3;
          vm &= vm - 1u;
          const int m4a = ML - ha3, m4b = ML - hb3;
          const int ia = __ldg(HO + (anh | (1u << ha3))) + LR[anl | (1u << m4a)];
          const int ib = __ldg(HO + (anh | (1u << hb3))) + LR[anl | (1u << m4b)];
          TG fa = fph[ha3], fb = two ? fph[hb3] : TG(0);
          const int pa = __popc(anl & between32(m4a, LB)) + __popc(anh & ((1u << ha3) - 1u));
          const int pb = __popc(anl & between32(m4b, LB)) + __popc(anh & ((1u << hb3) - 1u));
          if ((paa + pa) & 1) fa = -fa;
          if ((paa + pb) & 1) fb = -fb;
          g.add2(acc, x, a, ia, fa, ib, fb);
        }
      }
    }
  }
  g.finish(acc);
}

// four resident blocks of 256 threads per SM: at most 64 registers per thread (a tighter bound of 48
// registers for the FP32 single-vector form measured slower)
constexpr int kSplitMinBlocks = 4;

// Launch forms of the split kernel the autotuner chooses between (threads per block, resident
// blocks per SM, i.e. the register budget, and the gather pipeline depth).
struct SplitForm {
  int threads, min_blocks;
  bool pipe;
};
constexpr SplitForm kSplitForms[kNbrSplitForms] = {
    {256, 4, false}, {256, 3, false}, {256, 3, true}, {256, 2, true},
    {128, 8, false}, {256, 2, false}, {192, 4, false}, {128, 6, false}};

// IL: the K vectors are row-interleaved ([row][K], ld = K, vstride = 1 for x and y); W256: and the
// FP64 rows of 4 are 32-byte aligned (one 256-bit gather per target row); FORM: kSplitForms entry
template <typename TG, int K, bool RANGE, bool LR_SMEM, bool IL, bool W256 = false, int FORM = 0>
__global__ void __launch_bounds__(kSplitForms[FORM].threads, kSplitForms[FORM].min_blocks)
    fqhe_split_kernel(FqheDevice f, MatvecArgs a, SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  int* spair = reinterpret_cast<int*>(smem + lay.factor_bytes);
  const TG* gfac = static_cast<const TG*>(f.factors);
  for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
  for (int i = threadIdx.x; i < f.nbr_pairs; i += blockDim.x) spair[i] = f.pair_offset[i];
  SplitTables t;
  t.words = f.words;
  t.HO = f.high_offset;
  t.LR = f.low_rank;
  t.LB = f.low_bits;
  t.full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  if (LR_SMEM) {
    uint16_t* slr = reinterpret_cast<uint16_t*>(smem + lay.factor_bytes + lay.pair_bytes);
    const uint4* src = reinterpret_cast<const uint4*>(f.low_rank);
    uint4* dst = reinterpret_cast<uint4*>(slr);
    for (int i = threadIdx.x; i < (1 << t.LB) / 8; i += blockDim.x) dst[i] = src[i];
    t.LR = slr;
  }
  __syncthreads();
  const TG* x = static_cast<const TG*>(a.x);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : f.dim;
  for (long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    TG dsum = TG(0);
    split_row<TG, K, RANGE, IL, W256, kSplitForms[FORM].pipe>(t, sfac, spair, r, x, a, acc, dsum);
    if (!RANGE || (r >= a.col_first && r < a.col_last)) {
      TG xr[K];
      load_row<TG, K, IL, W256>(x, a, (int)r, xr);
#pragma unroll
      for (int j = 0; j < K; ++j) acc[j] += dsum * xr[j];
    }
    const bool diag = (r >= a.row_first && r < a.row_last);
    double* y = static_cast<double*>(a.y);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double v = (double)acc[j];
      const long long xo = IL ? r * K + j : r * a.ld + j * a.vstride;
      if (diag && a.shift != 0.0) {
        double xd = a.xdiag ? a.xdiag[xo] : (double)x[xo];
        v += a.shift * xd;
      }
      double* yp = y + (IL ? r * K + j : r * a.ld_y + j * a.vstride_y);
      *yp = a.accumulate ? (*yp + v) : v;
    }
  }
}

// All Lz sectors of one system in one launch: rows of every sector are concatenated (sector s owns
// rows [row_offset[s], row_offset[s+1])), vectors are K-interleaved ([row][K]) over the
// concatenated rows, and the factors (same 2S and V for every sector) are staged once per block.
// A thread finds its sector by a binary search over the offsets kept in shared memory.
template <typename TG, int K>
__global__ void __launch_bounds__(kMatvecThreads) fqhe_sectors_kernel(SectorBatchDevice b, SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  int* spair = reinterpret_cast<int*>(smem + lay.factor_bytes);
  long long* soff = reinterpret_cast<long long*>(smem + lay.factor_bytes + lay.pair_bytes);
  const TG* gfac = static_cast<const TG*>(b.factors);
  for (int i = threadIdx.x; i < b.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
  for (int i = threadIdx.x; i < b.nbr_pairs; i += blockDim.x) spair[i] = b.pair_offset[i];
  for (int i = threadIdx.x; i <= b.nbr_sectors; i += blockDim.x) soff[i] = b.row_offset[i];
  __syncthreads();
  const uint64_t full = (b.lz_max >= 63) ? ~0ull : ((1ull << (b.lz_max + 1)) - 1ull);
  const TG* xall = static_cast<const TG*>(b.x);
  MatvecArgs a = {};
  a.ld = K;
  a.vstride = 1;
  const long long total = soff[b.nbr_sectors];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += stride) {
    int lo = 0, hi = b.nbr_sectors;  // soff[lo] <= g < soff[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (soff[mid] <= g) lo = mid; else hi = mid;
    }
    const long long off = soff[lo];
    const long long r = g - off;
    if (b.active && !b.active[lo]) {  // a finished sector: zero rows, no enumeration
#pragma unroll
      for (int j = 0; j < K; ++j) b.y[g * K + j] = 0.0;
      continue;
    }
    SplitTables t;
    t.words = b.words[lo];
    t.HO = b.high_offset[lo];
    t.LR = b.low_rank;
    t.LB = b.low_bits;
    t.full = full;
    const TG* x = xall + off * K;
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    TG dsum = TG(0);
    split_row<TG, K, false, true>(t, sfac, spair, r, x, a, acc, dsum);
    TG xr[K];
    load_row<TG, K, true>(x, a, (int)r, xr);
    double* y = b.y + g * K;
    const double* xd = b.xdiag ? b.xdiag + g * K : nullptr;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double v = (double)(acc[j] + dsum * xr[j]);
      if (b.shift != 0.0) v += b.shift * (xd ? xd[j] : (double)xr[j]);
      y[j] = v;
    }
  }
}

using MatvecKernel = void (*)(FqheDevice, MatvecArgs, SmemLayout);

// the split-word kernel of one launch form (full column range, tables read through L1)
template <typename TG, int K, bool IL, bool W256>
MatvecKernel split_form_kernel(int form) {
  switch (form) {
    case 1: return fqhe_split_kernel<TG, K, false, false, IL, W256, 1>;
    case 2: return fqhe_split_kernel<TG, K, false, false, IL, W256, 2>;
    case 3: return fqhe_split_kernel<TG, K, false, false, IL, W256, 3>;
    case 4: return fqhe_split_kernel<TG, K, false, false, IL, W256, 4>;
    case 5: return fqhe_split_kernel<TG, K, false, false, IL, W256, 5>;
    case 6: return fqhe_split_kernel<TG, K, false, false, IL, W256, 6>;
    case 7: return fqhe_split_kernel<TG, K, false, false, IL, W256, 7>;
    default: return fqhe_split_kernel<TG, K, false, false, IL, W256, 0>;
  }
}

template <typename TG, int K, int MODE, bool RANGE>
int launch_one(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  SmemLayout lay = smem_layout(f, sizeof(TG));
  MatvecKernel kern = fqhe_matvec_kernel<TG, K, MODE, RANGE>;
  int threads = kMatvecThreads;
  // the split-word form needs both halves of a word in 32 bits; variant 2 stages the low-rank table
  // in shared memory
  if (MODE == DH_INDEX_RANK && f.kernel_variant != 1 && f.low_bits <= 31 && f.lz_max + 1 - f.low_bits <= 31) {
    kern = (f.kernel_variant == 2) ? fqhe_split_kernel<TG, K, RANGE, true, false>
                                   : fqhe_split_kernel<TG, K, RANGE, false, false>;
    if constexpr (!RANGE) {
      if (f.kernel_variant != 2) {
        const int form = (f.split_form >= 0 && f.split_form < kNbrSplitForms) ? f.split_form : 0;
        kern = split_form_kernel<TG, K, false, false>(form);
        if constexpr (K > 1) {
          // row-interleaved blocks (block Lanczos): vector loads of the K values of a target row
          if (a.ld == K && a.vstride == 1 && a.ld_y == K && a.vstride_y == 1 && il_rows_aligned(a, K, sizeof(TG))) {
            kern = split_form_kernel<TG, K, true, false>(form);
            if constexpr (sizeof(TG) == 8 && K == 4)
              if ((reinterpret_cast<uintptr_t>(a.x) & 31) == 0) kern = split_form_kernel<TG, K, true, true>(form);
          }
        } else if (a.ld == 1 && a.ld_y == 1) {
          // one contiguous vector: the same form with the row stride known at compile time
          kern = split_form_kernel<TG, K, true, false>(form);
        }
        threads = kSplitForms[form].threads;
      }
    }
  }
  if (lay.total > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total));
  int dev = 0, sms = 0, per_sm = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, lay.total));
  if (per_sm < 1) {
    set_error("fqhe matvec: %d bytes of shared memory per block do not fit", lay.total);
    return DH_ERR_UNSUPPORTED;
  }
  const long long rows = (a.out_last > 0 ? a.out_last : f.dim) - a.out_first;
  long long need = (rows + threads - 1) / threads;
  long long grid = (long long)sms * per_sm;
  if (need < grid) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, threads, lay.total, s>>>(f, a, lay);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename TG, int K>
int dispatch_mode(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  const bool range = (a.col_first > 0 || a.col_last < f.dim);
  if (f.index_mode == DH_INDEX_LOOKUP)
    return range ? launch_one<TG, K, DH_INDEX_LOOKUP, true>(f, a, s) : launch_one<TG, K, DH_INDEX_LOOKUP, false>(f, a, s);
  return range ? launch_one<TG, K, DH_INDEX_RANK, true>(f, a, s) : launch_one<TG, K, DH_INDEX_RANK, false>(f, a, s);
}

template <typename TG>
int dispatch_k(const FqheDevice& f, MatvecArgs a, cudaStream_t s) {
  // vectors are processed in groups of 4, 2 and 1 sharing one enumeration
  int left = a.nbr_vectors;
  const char* x0 = static_cast<const char*>(a.x);
  char* y0 = static_cast<char*>(a.y);
  const double* xd0 = a.xdiag;
  int done = 0;
  while (left > 0) {
    int k = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    MatvecArgs b = a;
    b.x = x0 + (size_t)done * a.vstride * sizeof(TG);
    b.y = y0 + (size_t)done * a.vstride_y * sizeof(double);
    b.xdiag = xd0 ? xd0 + (size_t)done * a.vstride : nullptr;
    b.nbr_vectors = k;
    int rc = (k == 4) ? dispatch_mode<TG, 4>(f, b, s) : (k == 2 ? dispatch_mode<TG, 2>(f, b, s) : dispatch_mode<TG, 1>(f, b, s));
    if (rc != DH_OK) return rc;
    left -= k;
    done += k;
  }
  return DH_OK;
}

// ------------------------------------------------------------- unranking
// Word of basis index i: orbitals from the top down; with n fermions and orbital-sum s still to
// place, the states occupying orbital p come first (descending order), and there are
// counts[n-1][p][s-p] of them.
__global__ void fqhe_unrank_kernel(int nbr_fermions, int lz_max, int total_sum, long long dim, uint64_t* words,
                                   const int64_t* counts, int so, int ss) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= dim) return;
  long long rest = i;
  int n = nbr_fermions, sum = total_sum;
  uint64_t w = 0;
  for (int p = lz_max; p >= 0 && n > 0; --p) {
    long long c = 0;
    if (sum - p >= 0) c = counts[(size_t)(n - 1) * so + (size_t)p * ss + (sum - p)];
    if (rest < c) {
      w |= 1ull << p;
      --n;
      sum -= p;
    } else {
      rest -= c;
    }
  }
  words[i] = w;
}

// ------------------------------------------------------ per-row dump
// The reference enumeration order of AbstractQHEOnSphereHamiltonian::LowLevelAddMultiply
// (:456-488): pairs m1 ascending then m2 ascending (M1Value/M2Value), m3 ascending (M3Values).
template <int MODE>
__global__ void fqhe_row_kernel(FqheDevice f, long long row, int* targets, int* signs, int* fidx, int cap,
                                int* count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int width = (1 << f.lookup_bits) + 1;
  (void)width;
  const uint64_t s = f.words[row];
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  int n = 0;
  for (int m1 = 1; m1 <= f.lz_max; ++m1) {
    if (!((s >> m1) & 1)) continue;
    for (int m2 = 0; m2 < m1; ++m2) {
      if (!((s >> m2) & 1)) continue;
      const uint64_t an = s & ~((1ull << m1) | (1ull << m2));
      const int M = m1 + m2;
      const int paa = 1 + __popcll(s & between_mask(m2, m1));
      const uint64_t e = ~an & full;
      uint64_t valid = e & mirror_bits(e, M) & (~0ull << (M / 2 + 1));
      const int fb = f.pair_offset[m1 * (m1 - 1) / 2 + m2] - (M / 2 + 1);
      while (valid) {
        const int m3 = __ffsll(valid) - 1;
        valid &= valid - 1ull;
        const int m4 = M - m3;
        const uint64_t t = an | (1ull << m3) | (1ull << m4);
        const int par = paa + __popcll(an & between_mask(m4, m3));
        long long idx;
        if (MODE == DH_INDEX_RANK) {
          idx = (long long)f.high_offset[t >> f.low_bits] + f.low_rank[t & ((1ull << f.low_bits) - 1ull)];
        } else {
          const int l = 63 - __clzll(t);
          const int wdt = (1 << f.lookup_bits) + 1;
          const long long v = (long long)(t >> f.lookup_shift[l]);
          long long lo = f.lookup[l * wdt + v + 1], hi = f.lookup[l * wdt + v];
          while (hi - lo > 1) {
            long long mid = (lo + hi) >> 1;
            if (f.words[mid] > t) lo = mid; else hi = mid;
          }
          idx = (f.words[lo] == t) ? lo : hi;
        }
        if (n < cap) {
          targets[n] = (int)idx;
          signs[n] = (par & 1) ? -1 : 1;
          fidx[n] = fb + m3;
        }
        ++n;
      }
    }
  }
  *count = n;
}

// ----------------------------------------------------- adjoint bins
// bins[f] = sum over rows r and elements (r -> t) of factor f of u[r] * sign * v[t].  Each block
// accumulates into shared-memory bins and writes its partial row of a [blocks][factors] scratch
// array; a second kernel sums the partials in block order (deterministic, no global atomics).
constexpr int kBinThreads = 256;

template <int MODE>
__global__ void __launch_bounds__(kBinThreads) fqhe_bins_kernel(FqheDevice f, const double* u, const double* v,
                                                                double* partial, SmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* sbins = reinterpret_cast<double*>(smem);
  int* spair = reinterpret_cast<int*>(smem + align16(f.nbr_factors * (int)sizeof(double)));
  int* slookup = spair + align16(f.nbr_pairs * (int)sizeof(int)) / (int)sizeof(int);
  int* sshift = slookup + ((MODE == DH_INDEX_LOOKUP) ? (f.lz_max + 1) * ((1 << f.lookup_bits) + 1) : 0);
  for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) sbins[i] = 0.0;
  for (int i = threadIdx.x; i < f.nbr_pairs; i += blockDim.x) spair[i] = f.pair_offset[i];
  if (MODE == DH_INDEX_LOOKUP) {
    const int n = (f.lz_max + 1) * ((1 << f.lookup_bits) + 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) slookup[i] = f.lookup[i];
    for (int i = threadIdx.x; i <= f.lz_max; i += blockDim.x) sshift[i] = f.lookup_shift[i];
  }
  __syncthreads();
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    const double ur = u[r];
    if (ur == 0.0) continue;
    uint64_t rem1 = s;
    while (rem1) {
      const int m1 = 63 - __clzll(rem1);
      rem1 &= ~(1ull << m1);
      uint64_t rem2 = rem1;
      const int pbase = m1 * (m1 - 1) / 2;
      while (rem2) {
        const int m2 = 63 - __clzll(rem2);
        rem2 &= ~(1ull << m2);
        const uint64_t an = s & ~((1ull << m1) | (1ull << m2));
        const int M = m1 + m2;
        const int paa = 1 + __popcll(s & between_mask(m2, m1));
        const uint64_t e = ~an & full;
        uint64_t valid = e & mirror_bits(e, M) & (~0ull << (M / 2 + 1));
        const int fb = spair[pbase + m2] - (M / 2 + 1);
        while (valid) {
          const int m3 = __ffsll(valid) - 1;
          valid &= valid - 1ull;
          const int m4 = M - m3;
          const uint64_t t = an | (1ull << m3) | (1ull << m4);
          const int par = paa + __popcll(an & between_mask(m4, m3));
          const long long idx = target_index<MODE>(f, t, slookup, sshift);
          const double c = ur * __ldg(v + idx);
          atomicAdd(sbins + fb + m3, (par & 1) ? -c : c);
        }
      }
    }
  }
  __syncthreads();
  double* out = partial + (size_t)blockIdx.x * f.nbr_factors;
  for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) out[i] = sbins[i];
}

__global__ void sum_partial_bins(const double* partial, int nblocks, int nbins, double* bins) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbins) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; ++b) acc += partial[(size_t)b * nbins + i];
  bins[i] = acc;
}

// number of generated elements (moves) of all rows, block partials then one atomic per block
__global__ void fqhe_count_kernel(FqheDevice f, unsigned long long* total) {
  __shared__ unsigned long long acc;
  if (threadIdx.x == 0) acc = 0;
  __syncthreads();
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  unsigned long long mine = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = f.words[r];
    uint64_t rem1 = s;
    while (rem1) {
      const int m1 = 63 - __clzll(rem1);
      rem1 &= ~(1ull << m1);
      uint64_t rem2 = rem1;
      while (rem2) {
        const int m2 = 63 - __clzll(rem2);
        rem2 &= ~(1ull << m2);
        const uint64_t an = s & ~((1ull << m1) | (1ull << m2));
        const uint64_t e = ~an & full;
        const int M = m1 + m2;
        mine += __popcll(e & mirror_bits(e, M) & (~0ull << (M / 2 + 1)));
      }
    }
  }
  atomicAdd(&acc, mine);
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(total, acc);
}

template <int MODE>
__global__ void fqhe_find_kernel(FqheDevice f, const uint64_t* words, long long n, long long* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t t = words[i];
  if (MODE == DH_INDEX_RANK) {
    const long long hi = t >> f.low_bits;
    if (hi >= (1ll << (f.lz_max + 1 - f.low_bits))) {
      out[i] = -1;
      return;
    }
    const int off = f.high_offset[hi];
    out[i] = (off < 0) ? -1 : (long long)off + f.low_rank[t & ((1ull << f.low_bits) - 1ull)];
    if (out[i] >= 0 && (out[i] >= f.dim || f.words[out[i]] != t)) out[i] = -1;
  } else {
    if (t == 0 || (63 - __clzll(t)) > f.lz_max) {
      out[i] = -1;
      return;
    }
    const int l = 63 - __clzll(t);
    const int wdt = (1 << f.lookup_bits) + 1;
    const long long v = (long long)(t >> f.lookup_shift[l]);
    long long lo = f.lookup[l * wdt + v + 1], hi = f.lookup[l * wdt + v];
    if (lo < 0 || hi < 0) {
      out[i] = -1;
      return;
    }
    while (hi - lo > 1) {
      long long mid = (lo + hi) >> 1;
      if (f.words[mid] > t) lo = mid; else hi = mid;
    }
    long long r = (f.words[lo] == t) ? lo : hi;
    out[i] = (f.words[r] == t) ? r : -1;
  }
}

}  // namespace

int launch_fqhe_unrank(int nbr_fermions, int lz_max, int total_sum, long long dim, uint64_t* words,
                       const int64_t* counts_dev, int count_stride_o, int count_stride_s, cudaStream_t s) {
  if (dim <= 0) return DH_OK;
  unsigned grid = (unsigned)((dim + 255) / 256);
  fqhe_unrank_kernel<<<grid, 256, 0, s>>>(nbr_fermions, lz_max, total_sum, dim, words, counts_dev,
                                          count_stride_o, count_stride_s);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_matvec(const FqheDevice& f, const MatvecArgs& a, int precision, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  if (precision == DH_PRECISION_FP32) return dispatch_k<float>(f, a, s);
  return dispatch_k<double>(f, a, s);
}

template <typename TG, int K>
static int launch_sectors_typed(const SectorBatchDevice& b, cudaStream_t s) {
  SmemLayout lay;
  lay.factor_bytes = align16(b.nbr_factors * (int)sizeof(TG));
  lay.pair_bytes = align16(b.nbr_pairs * (int)sizeof(int));
  lay.lookup_bytes = align16((b.nbr_sectors + 1) * (int)sizeof(long long));
  lay.total = lay.factor_bytes + lay.pair_bytes + lay.lookup_bytes;
  auto kern = fqhe_sectors_kernel<TG, K>;
  if (lay.total > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total));
  int dev = 0, sms = 0, per_sm = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMatvecThreads, lay.total));
  DH_CHECK(per_sm >= 1, DH_ERR_UNSUPPORTED, "sector kernel: %d bytes of shared memory per block do not fit", lay.total);
  long long need = (b.total_rows + kMatvecThreads - 1) / kMatvecThreads;
  long long grid = (long long)sms * per_sm;
  if (need < grid) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, kMatvecThreads, lay.total, s>>>(b, lay);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_sectors(const SectorBatchDevice& b, int precision, cudaStream_t s) {
  if (b.total_rows <= 0) return DH_OK;
  DH_CHECK(b.low_bits <= 31 && b.lz_max + 1 - b.low_bits <= 31, DH_ERR_UNSUPPORTED, "lz_max too large for the sector kernel");
  if (precision == DH_PRECISION_FP32) {
    switch (b.block) {
      case 1: return launch_sectors_typed<float, 1>(b, s);
      case 2: return launch_sectors_typed<float, 2>(b, s);
      case 4: return launch_sectors_typed<float, 4>(b, s);
    }
  } else {
    switch (b.block) {
      case 1: return launch_sectors_typed<double, 1>(b, s);
      case 2: return launch_sectors_typed<double, 2>(b, s);
      case 4: return launch_sectors_typed<double, 4>(b, s);
    }
  }
  set_error("sector kernel: block size %d not in {1, 2, 4}", b.block);
  return DH_ERR_UNSUPPORTED;
}

int launch_fqhe_row_elements(const FqheDevice& f, long long row, int* targets, int* signs, int* factor_index,
                             int cap, int* count, cudaStream_t s) {
  if (f.index_mode == DH_INDEX_LOOKUP)
    fqhe_row_kernel<DH_INDEX_LOOKUP><<<1, 32, 0, s>>>(f, row, targets, signs, factor_index, cap, count);
  else
    fqhe_row_kernel<DH_INDEX_RANK><<<1, 32, 0, s>>>(f, row, targets, signs, factor_index, cap, count);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_bins(const FqheDevice& f, const double* u, const double* v, double* partial_bins, int nblocks,
                     double* bins, cudaStream_t s) {
  SmemLayout lay = smem_layout(f, sizeof(double));
  if (f.dim > 0) {
    if (f.index_mode == DH_INDEX_LOOKUP) {
      auto kern = fqhe_bins_kernel<DH_INDEX_LOOKUP>;
      if (lay.total > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total));
      kern<<<nblocks, kBinThreads, lay.total, s>>>(f, u, v, partial_bins, lay);
    } else {
      auto kern = fqhe_bins_kernel<DH_INDEX_RANK>;
      if (lay.total > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total));
      kern<<<nblocks, kBinThreads, lay.total, s>>>(f, u, v, partial_bins, lay);
    }
    DH_CUDA(cudaGetLastError());
  }
  sum_partial_bins<<<(f.nbr_factors + 255) / 256, 256, 0, s>>>(partial_bins, f.dim > 0 ? nblocks : 0, f.nbr_factors,
                                                                 bins);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_count(const FqheDevice& f, unsigned long long* total, cudaStream_t s) {
  DH_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), s));
  if (f.dim <= 0) return DH_OK;
  long long g = (f.dim + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  fqhe_count_kernel<<<(unsigned)g, 256, 0, s>>>(f, total);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_find(const FqheDevice& f, const uint64_t* words, long long n, long long* out, cudaStream_t s) {
  if (n <= 0) return DH_OK;
  unsigned grid = (unsigned)((n + 255) / 256);
  if (f.index_mode == DH_INDEX_LOOKUP)
    fqhe_find_kernel<DH_INDEX_LOOKUP><<<grid, 256, 0, s>>>(f, words, n, out);
  else
    fqhe_find_kernel<DH_INDEX_RANK><<<grid, 256, 0, s>>>(f, words, n, out);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

}  // namespace dh

// Spin-polarised fermions on the sphere beyond the split-word rank tables: FermionOnSphere with
// 41 <= lz_max <= 62 and FermionOnSphereLong (FQHE/src/HilbertSpace/FermionOnSphereLong.cc, lz_max up
// to 126, one 128-bit word per state) on sm_100a.
//
// Words are two 64-bit halves (orbital m = bit m of low | high << 64).  States are in the reference's
// order: descending words (FermionOnSphereLong::GenerateStates, .cc:911-943, places the highest
// fermion as high as it can first).
//
// Rank.  With C(n, o, s) the number of ways to put n fermions in orbitals 0..o-1 with orbital sum s
// (the sector's count table), the states below w in that order are, fermion by fermion, those that
// keep every fermion above it and move it (and the ones below) lower with the same sum:
//     index(w) = dim - 1 - sum over fermions i of C(n_i, p_i, s_i),
// p_i the fermion's orbital, n_i the number of fermions at or below p_i and s_i the sum of their
// orbitals.  One table load per fermion.  A move of two fermions m1, m2 -> m3, m4 (same sum) leaves
// n_i and s_i of every fermion below min(m2, m4) and above max(m1, m3) unchanged, so the target's
// index is the row's own index corrected over that orbital range only.  The counts used are numbers
// of states of the sector, so they fit the int32 table (entries that no state uses saturate).
//
// Product.  Pull form, one thread per row, the factor tables of the generic Hamiltonian (pair m1 > m2,
// then the creations m3 > m4 = m1 + m2 - m3) read through the read-only cache (at lz_max = 126 they
// are 1.4 MB), the AA * AdAd sign from popcounts as in the 64-bit kernels (FermionOnSphere::AA
// FermionOnSphere.cc:790, ::AdAd :949; FermionOnSphereLong.cc keeps the same conventions).  H is
// real symmetric, so the pull form equals the reference's push form
// (AbstractQHEOnSphereHamiltonian.cc:456-488).
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"

namespace dh {

namespace {

constexpr int kLongThreads = 256;

struct U128 {
  uint64_t lo, hi;
};

__device__ __forceinline__ U128 u_and(U128 a, U128 b) { return {a.lo & b.lo, a.hi & b.hi}; }
__device__ __forceinline__ U128 u_or(U128 a, U128 b) { return {a.lo | b.lo, a.hi | b.hi}; }
__device__ __forceinline__ U128 u_not(U128 a) { return {~a.lo, ~a.hi}; }
__device__ __forceinline__ bool u_any(U128 a) { return (a.lo | a.hi) != 0ull; }
__device__ __forceinline__ int u_popc(U128 a) { return __popcll(a.lo) + __popcll(a.hi); }
__device__ __forceinline__ U128 u_bit(int q) {
  return q < 64 ? U128{1ull << q, 0ull} : U128{0ull, 1ull << (q - 64)};
}
// bits 0 .. q-1 (0 <= q <= 128)
__device__ __forceinline__ U128 u_below(int q) {
  if (q <= 0) return {0ull, 0ull};
  if (q < 64) return {(1ull << q) - 1ull, 0ull};
  if (q == 64) return {~0ull, 0ull};
  if (q < 128) return {~0ull, (1ull << (q - 64)) - 1ull};
  return {~0ull, ~0ull};
}
// bits strictly between lo and hi (lo < hi)
__device__ __forceinline__ U128 u_between(int lo, int hi) { return u_and(u_below(hi), u_not(u_below(lo + 1))); }
__device__ __forceinline__ int u_lowest(U128 a) { return a.lo ? __ffsll(a.lo) - 1 : 64 + __ffsll(a.hi) - 1; }
__device__ __forceinline__ U128 u_clear_lowest(U128 a) {
  if (a.lo) return {a.lo & (a.lo - 1ull), a.hi};
  return {0ull, a.hi & (a.hi - 1ull)};
}
__device__ __forceinline__ int u_highest(U128 a) { return a.hi ? 127 - __clzll(a.hi) : 63 - __clzll(a.lo); }
__device__ __forceinline__ U128 u_shr(U128 a, int n) {  // 0 <= n < 256
  if (n == 0) return a;
  if (n >= 128) return {0ull, 0ull};
  if (n >= 64) return {a.hi >> (n - 64), 0ull};
  return {(a.lo >> n) | (a.hi << (64 - n)), a.hi >> n};
}
__device__ __forceinline__ U128 u_shl(U128 a, int n) {  // 0 <= n < 256
  if (n == 0) return a;
  if (n >= 128) return {0ull, 0ull};
  if (n >= 64) return {0ull, a.lo << (n - 64)};
  return {a.lo << n, (a.hi << n) | (a.lo >> (64 - n))};
}
// bit p of the result = bit (M - p) of e (0 when M - p is outside 0..127)
__device__ __forceinline__ U128 u_mirror(U128 e, int M) {
  const U128 r = {__brevll(e.hi), __brevll(e.lo)};  // bit p = bit 127 - p of e
  return (M <= 127) ? u_shr(r, 127 - M) : u_shl(r, M - 127);
}
// sum of the positions of the set bits
__device__ __forceinline__ int u_position_sum(U128 a) {
  const uint64_t m0 = 0xaaaaaaaaaaaaaaaaull, m1 = 0xccccccccccccccccull, m2 = 0xf0f0f0f0f0f0f0f0ull,
                 m3 = 0xff00ff00ff00ff00ull, m4 = 0xffff0000ffff0000ull, m5 = 0xffffffff00000000ull;
  return (__popcll(a.lo & m0) + __popcll(a.hi & m0)) + 2 * (__popcll(a.lo & m1) + __popcll(a.hi & m1)) +
         4 * (__popcll(a.lo & m2) + __popcll(a.hi & m2)) + 8 * (__popcll(a.lo & m3) + __popcll(a.hi & m3)) +
         16 * (__popcll(a.lo & m4) + __popcll(a.hi & m4)) + 32 * (__popcll(a.lo & m5) + __popcll(a.hi & m5)) +
         64 * __popcll(a.hi);
}

// the same operations on one 64-bit word (sectors with lz_max <= 63)
__device__ __forceinline__ uint64_t u_and(uint64_t a, uint64_t b) { return a & b; }
__device__ __forceinline__ uint64_t u_or(uint64_t a, uint64_t b) { return a | b; }
__device__ __forceinline__ uint64_t u_not(uint64_t a) { return ~a; }
__device__ __forceinline__ bool u_any(uint64_t a) { return a != 0ull; }
__device__ __forceinline__ int u_popc(uint64_t a) { return __popcll(a); }
__device__ __forceinline__ int u_lowest(uint64_t a) { return __ffsll(a) - 1; }
__device__ __forceinline__ uint64_t u_clear_lowest(uint64_t a) { return a & (a - 1ull); }
__device__ __forceinline__ int u_highest(uint64_t a) { return 63 - __clzll(a); }
__device__ __forceinline__ int u_position_sum(uint64_t a) {
  return __popcll(a & 0xaaaaaaaaaaaaaaaaull) + 2 * __popcll(a & 0xccccccccccccccccull) +
         4 * __popcll(a & 0xf0f0f0f0f0f0f0f0ull) + 8 * __popcll(a & 0xff00ff00ff00ff00ull) +
         16 * __popcll(a & 0xffff0000ffff0000ull) + 32 * __popcll(a & 0xffffffff00000000ull);
}

template <typename W>
struct Word;
template <>
struct Word<U128> {
  __device__ static __forceinline__ U128 bit(int q) { return u_bit(q); }
  __device__ static __forceinline__ U128 below(int q) { return u_below(q); }
  __device__ static __forceinline__ U128 between(int lo, int hi) { return u_between(lo, hi); }
  __device__ static __forceinline__ U128 mirror(U128 e, int M) { return u_mirror(e, M); }
  __device__ static __forceinline__ U128 load(const uint64_t* words, long long i) {
    const ulonglong2 q = __ldg(reinterpret_cast<const ulonglong2*>(words) + i);
    return {q.x, q.y};
  }
};
template <>
struct Word<uint64_t> {
  __device__ static __forceinline__ uint64_t bit(int q) { return 1ull << q; }
  __device__ static __forceinline__ uint64_t below(int q) { return q >= 64 ? ~0ull : ((1ull << q) - 1ull); }
  __device__ static __forceinline__ uint64_t between(int lo, int hi) { return below(hi) & ~below(lo + 1); }
  // bit p of the result = bit (M - p) of e, M <= 125
  __device__ static __forceinline__ uint64_t mirror(uint64_t e, int M) {
    const uint64_t r = __brevll(e);
    return (M <= 63) ? (r >> (63 - M)) : (r << (M - 63));
  }
  // the low half of the stored (low, high) pair: lz_max <= 63 leaves the high half zero
  __device__ static __forceinline__ uint64_t load(const uint64_t* words, long long i) { return __ldg(words + 2 * i); }
};

// C(n, o, s), 1 <= n <= N, 0 <= o <= lz_max + 1, 0 <= s <= total_sum
__device__ __forceinline__ long long count_at(const FqheLongDevice& f, int n, int o, int s) {
  return (long long)__ldg(f.table + (size_t)(n - 1) * f.stride_n + (size_t)o * f.stride_o + s);
}

// sum over the fermions of w in orbitals [lo, hi] of C(n_i, p_i, s_i), given the number and the
// orbital sum of the fermions below lo
template <typename W>
__device__ __forceinline__ long long range_terms(const FqheLongDevice& f, W w, int lo, int hi, int n, int s) {
  W bits = u_and(w, u_and(Word<W>::below(hi + 1), u_not(Word<W>::below(lo))));
  long long acc = 0;
  while (u_any(bits)) {
    const int q = u_lowest(bits);
    bits = u_clear_lowest(bits);
    ++n;
    s += q;
    acc += count_at(f, n, q, s);
  }
  return acc;
}

template <typename TG, int K, bool IL>
__device__ __forceinline__ void gather_row(const TG* x, const MatvecArgs& a, long long idx, TG (&v)[K]) {
  if constexpr (IL) {
    const TG* p = x + idx * K;
    if constexpr (sizeof(TG) == 4 && K == 4) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(p));
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
    const TG* p = x + idx * a.ld;
#pragma unroll
    for (int j = 0; j < K; ++j) v[j] = __ldg(p + j * a.vstride);
  }
}

// Rows of at most kPrefixFermions fermions keep, in shared memory, the prefix sums of their own rank
// terms and orbitals over their fermions in ascending order (term[j] = sum of the j lowest fermions'
// C(n_i, p_i, s_i), osum[j] = sum of their orbitals): the row's share of any orbital range is then two
// popcounts and three shared loads, and only the target's fermions in the range are walked.
constexpr int kPrefixFermions = 20;

template <typename W, typename TG, int K, bool RANGE, bool IL, bool PREFIX>
__global__ void __launch_bounds__(kLongThreads) long_matvec_kernel(FqheLongDevice f, MatvecArgs a) {
  using O = Word<W>;
  extern __shared__ int prefix_smem[];
  // thread-strided: entry j of this thread at [j * blockDim.x + threadIdx.x], N + 1 entries each
  int* term = prefix_smem;
  int* osum = prefix_smem + (f.nbr_fermions + 1) * kLongThreads;
  const int L = f.lz_max;
  const W full = O::below(L + 1);
  const TG* fac = static_cast<const TG*>(f.factors);
  const TG* x = static_cast<const TG*>(a.x);
  double* y = static_cast<double*>(a.y);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : f.dim;
  for (long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    const W s = O::load(f.words, r);
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    if (PREFIX) {
      W bits = s;
      int j = 0, sum = 0, run = 0;
      term[threadIdx.x] = 0;
      osum[threadIdx.x] = 0;
      while (u_any(bits)) {
        const int q = u_lowest(bits);
        bits = u_clear_lowest(bits);
        ++j;
        sum += q;
        run += (int)count_at(f, j, q, sum);
        term[j * kLongThreads + threadIdx.x] = run;
        osum[j * kLongThreads + threadIdx.x] = sum;
      }
    }
    W rem1 = s;
    while (u_any(rem1)) {
      const int m1 = u_highest(rem1);
      rem1 = u_and(rem1, u_not(O::bit(m1)));
      W rem2 = rem1;
      while (u_any(rem2)) {
        const int m2 = u_highest(rem2);
        rem2 = u_and(rem2, u_not(O::bit(m2)));
        const int M = m1 + m2;
        const W an = u_and(s, u_not(u_or(O::bit(m1), O::bit(m2))));
        const W e = u_and(u_not(an), full);
        W valid = u_and(u_and(e, O::mirror(e, M)), u_not(O::below(M / 2 + 1)));
        if (!u_any(valid)) continue;
        const int paa = 1 + u_popc(u_and(s, O::between(m2, m1)));
        const long long fbase = (long long)__ldg(f.pair_offset + m1 * (m1 - 1) / 2 + m2) - (M / 2 + 1);
        while (u_any(valid)) {
          const int m3 = u_lowest(valid);
          valid = u_clear_lowest(valid);
          const int m4 = M - m3;
          const W t = u_or(an, u_or(O::bit(m3), O::bit(m4)));
          const int par = paa + u_popc(u_and(an, O::between(m4, m3)));
          // the target's index: the row's, corrected over the orbitals [lo, hi] the move touches
          const int lo = min(m2, m4), hi = max(m1, m3);
          long long idx;
          if (PREFIX) {
            const int n0 = u_popc(u_and(s, O::below(lo))), n1 = u_popc(u_and(s, O::below(hi + 1)));
            const int s0 = osum[n0 * kLongThreads + threadIdx.x];
            idx = r + (term[n1 * kLongThreads + threadIdx.x] - term[n0 * kLongThreads + threadIdx.x]) -
                  range_terms<W>(f, t, lo, hi, n0, s0);
          } else {
            const W low_part = u_and(s, O::below(lo));
            const int n0 = u_popc(low_part), s0 = u_position_sum(low_part);
            idx = r + range_terms<W>(f, s, lo, hi, n0, s0) - range_terms<W>(f, t, lo, hi, n0, s0);
          }
          if (RANGE && (idx < a.col_first || idx >= a.col_last)) continue;
          TG fct = __ldg(fac + fbase + m3);
          if (par & 1) fct = -fct;
          TG v[K];
          gather_row<TG, K, IL>(x, a, idx, v);
#pragma unroll
          for (int j = 0; j < K; ++j) acc[j] += fct * v[j];
        }
      }
    }
    const bool diag = (r >= a.row_first && r < a.row_last);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double v = (double)acc[j];
      if (diag && a.shift != 0.0) {
        const long long xo = IL ? r * K + j : r * a.ld + j * a.vstride;
        const double xd = a.xdiag ? a.xdiag[xo] : (double)x[xo];
        v += a.shift * xd;
      }
      double* yp = y + (IL ? r * K + j : r * a.ld_y + j * a.vstride_y);
      *yp = a.accumulate ? (*yp + v) : v;
    }
  }
}

// state index -> word: fermion by fermion from the top, the orbital q of the next fermion is the
// lowest one whose block of states (those with that fermion at q or lower) still holds the index
__global__ void long_unrank_kernel(FqheLongDevice f, uint64_t* words) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.dim) return;
  long long r = i;
  int n = f.nbr_fermions, s = f.total_sum, upper = f.lz_max + 1;
  U128 w = {0ull, 0ull};
  while (n > 0) {
    const long long total = count_at(f, n, upper, s);
    const long long need = total - r;  // 1 .. total
    // smallest o in [1, upper] with C(n, o, s) >= need; the fermion sits at o - 1
    int lo = 1, hi = upper;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (count_at(f, n, mid, s) >= need)
        hi = mid;
      else
        lo = mid + 1;
    }
    const int q = lo - 1;
    r -= total - count_at(f, n, lo, s);
    w = u_or(w, u_bit(q));
    s -= q;
    --n;
    upper = q;
  }
  reinterpret_cast<ulonglong2*>(words)[i] = make_ulonglong2(w.lo, w.hi);
}

// FindStateIndex for (low, high) words: the index, or -1 for a word outside the sector
__global__ void long_find_kernel(FqheLongDevice f, const uint64_t* words, long long n, long long* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U128 w = {words[2 * i], words[2 * i + 1]};
  const U128 outside = u_and(w, u_not(u_below(f.lz_max + 1)));
  if (u_any(outside) || u_popc(w) != f.nbr_fermions || u_position_sum(w) != f.total_sum) {
    out[i] = -1;
    return;
  }
  out[i] = f.dim - 1 - range_terms<U128>(f, w, 0, f.lz_max, 0, 0);
}

// elements (moves, the diagonal ones included) that one product generates
template <typename W>
__global__ void __launch_bounds__(kLongThreads) long_count_kernel(FqheLongDevice f, unsigned long long* total) {
  using O = Word<W>;
  const int L = f.lz_max;
  const W full = O::below(L + 1);
  unsigned long long c = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const W s = O::load(f.words, r);
    W rem1 = s;
    while (u_any(rem1)) {
      const int m1 = u_highest(rem1);
      rem1 = u_and(rem1, u_not(O::bit(m1)));
      W rem2 = rem1;
      while (u_any(rem2)) {
        const int m2 = u_highest(rem2);
        rem2 = u_and(rem2, u_not(O::bit(m2)));
        const int M = m1 + m2;
        const W an = u_and(s, u_not(u_or(O::bit(m1), O::bit(m2))));
        const W e = u_and(u_not(an), full);
        c += u_popc(u_and(u_and(e, O::mirror(e, M)), u_not(O::below(M / 2 + 1))));
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(total, c);
}

// ------------------------------------------- moves one at a time: stored elements
// Visits the moves of row r (word s) in the product kernel's order (m1 > m2 descending, m3 ascending);
// visit(target, factor index, negative, diagonal).  Targets from the count-table walk over the
// orbitals the move touches, both sides.
template <typename W, typename Visit>
__device__ __forceinline__ void long_visit_row(const FqheLongDevice& f, long long r, W s, Visit&& visit) {
  using O = Word<W>;
  const W full = O::below(f.lz_max + 1);
  W rem1 = s;
  while (u_any(rem1)) {
    const int m1 = u_highest(rem1);
    rem1 = u_and(rem1, u_not(O::bit(m1)));
    W rem2 = rem1;
    while (u_any(rem2)) {
      const int m2 = u_highest(rem2);
      rem2 = u_and(rem2, u_not(O::bit(m2)));
      const int M = m1 + m2;
      const W an = u_and(s, u_not(u_or(O::bit(m1), O::bit(m2))));
      const W e = u_and(u_not(an), full);
      W valid = u_and(u_and(e, O::mirror(e, M)), u_not(O::below(M / 2 + 1)));
      const int paa = 1 + u_popc(u_and(s, O::between(m2, m1)));
      const int fbase = __ldg(f.pair_offset + m1 * (m1 - 1) / 2 + m2) - (M / 2 + 1);
      while (u_any(valid)) {
        const int m3 = u_lowest(valid);
        valid = u_clear_lowest(valid);
        const int m4 = M - m3;
        const int par = paa + u_popc(u_and(an, O::between(m4, m3)));
        if (m3 == m1) {
          visit(r, fbase + m3, (par & 1) != 0, true);
          continue;
        }
        const W t = u_or(an, u_or(O::bit(m3), O::bit(m4)));
        const int lo = min(m2, m4), hi = max(m1, m3);
        const W low_part = u_and(s, O::below(lo));
        const int n0 = u_popc(low_part), s0 = u_position_sum(low_part);
        const long long idx = r + range_terms<W>(f, s, lo, hi, n0, s0) - range_terms<W>(f, t, lo, hi, n0, s0);
        visit(idx, fbase + m3, (par & 1) != 0, false);
      }
    }
  }
}

// off-diagonal moves per row: every pair's valid creations less its diagonal one (always valid)
template <typename W>
__global__ void long_row_counts_kernel(FqheLongDevice f, int* counts) {
  using O = Word<W>;
  const W full = O::below(f.lz_max + 1);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const W s = O::load(f.words, r);
    int c = 0;
    W rem1 = s;
    while (u_any(rem1)) {
      const int m1 = u_highest(rem1);
      rem1 = u_and(rem1, u_not(O::bit(m1)));
      W rem2 = rem1;
      while (u_any(rem2)) {
        const int m2 = u_highest(rem2);
        rem2 = u_and(rem2, u_not(O::bit(m2)));
        const int M = m1 + m2;
        const W an = u_and(s, u_not(u_or(O::bit(m1), O::bit(m2))));
        const W e = u_and(u_not(an), full);
        c += u_popc(u_and(u_and(e, O::mirror(e, M)), u_not(O::below(M / 2 + 1)))) - 1;
      }
    }
    counts[r] = c;
  }
}

// element payload: factor index | sign << 31; padding: the row itself times the zero factor
// nbr_factors
template <typename W>
__global__ void long_ell_fill_kernel(FqheLongDevice f, int nbr_factors, const long long* slice_ptr,
                                     const int* slice_len, int* cols, uint32_t* coef) {
  using O = Word<W>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const long long base = slice_ptr[r >> 5];
    const int len = slice_len[r >> 5];
    const int lane = (int)(r & 31);
    auto at = [&](int jj) {
      return base + (long long)(jj / kEllGroup) * (32 * kEllGroup) + lane * kEllGroup + (jj % kEllGroup);
    };
    int j = 0;
    long_visit_row<W>(f, r, O::load(f.words, r), [&](long long idx, int fidx, bool neg, bool diag) {
      if (diag) return;
      const long long p = at(j++);
      cols[p] = (int)idx;
      coef[p] = (uint32_t)fidx | (neg ? 0x80000000u : 0u);
    });
    for (; j < len; ++j) {
      const long long p = at(j);
      cols[p] = (int)r;
      coef[p] = (uint32_t)nbr_factors;
    }
  }
}

// diagonal of every row: the moves (m3, m4) = (m1, m2), each with sign -1
template <typename W>
__global__ void long_diag_kernel(FqheLongDevice f, const double* factors, double* diag64, float* diag32) {
  using O = Word<W>;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const W s = O::load(f.words, r);
    double d = 0.0;
    W rem1 = s;
    while (u_any(rem1)) {
      const int m1 = u_highest(rem1);
      rem1 = u_and(rem1, u_not(O::bit(m1)));
      W rem2 = rem1;
      while (u_any(rem2)) {
        const int m2 = u_highest(rem2);
        rem2 = u_and(rem2, u_not(O::bit(m2)));
        const int M = m1 + m2;
        d -= factors[__ldg(f.pair_offset + m1 * (m1 - 1) / 2 + m2) - (M / 2 + 1) + m1];
      }
    }
    diag64[r] = d;
    diag32[r] = (float)d;
  }
}

// adjoint bins: bins[f] = sum over rows r and moves (r -> t) of factor f of u[r] * sign * v[t], every
// move (the diagonal ones included).  SHARED: per-block partial rows of a [blocks][factors] array
// accumulated in shared memory and summed in block order afterwards (tables up to 2S of about 54);
// else atomics straight into the global bins (the tables of 2S up to 126 reach 2.6 MB)
template <typename W, bool SHARED>
__global__ void __launch_bounds__(kLongThreads) long_bins_kernel(FqheLongDevice f, int nbr_factors, const double* u,
                                                                 const double* v, double* out) {
  using O = Word<W>;
  extern __shared__ __align__(16) unsigned char smem_bins[];
  double* bins = SHARED ? reinterpret_cast<double*>(smem_bins) : out;
  if (SHARED) {
    for (int i = threadIdx.x; i < nbr_factors; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const double ur = u[r];
    if (ur == 0.0) continue;
    long_visit_row<W>(f, r, O::load(f.words, r), [&](long long idx, int fidx, bool neg, bool) {
      const double c = ur * __ldg(v + idx);
      atomicAdd(bins + fidx, neg ? -c : c);
    });
  }
  if (SHARED) {
    __syncthreads();
    double* row = out + (size_t)blockIdx.x * nbr_factors;
    for (int i = threadIdx.x; i < nbr_factors; i += blockDim.x) row[i] = bins[i];
  }
}

__global__ void long_sum_partial_bins(const double* partial, int nblocks, int nbins, double* bins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbins) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; ++b) acc += partial[(size_t)b * nbins + i];
  bins[i] = acc;
}

int grid_for(long long rows) {
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long blocks = (rows + kLongThreads - 1) / kLongThreads;
  const long long cap = (long long)sms * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

template <typename W, typename TG, int K, bool PREFIX>
int launch_prefix(const FqheLongDevice& f, const MatvecArgs& a, cudaStream_t s) {
  const bool range = a.col_first > 0 || a.col_last < f.dim;
  // row-interleaved blocks, or one contiguous vector: row strides known at compile time
  const bool il = K == 1 ? (a.ld == 1 && a.ld_y == 1)
                         : (a.ld == K && a.vstride == 1 && a.ld_y == K && a.vstride_y == 1 &&
                            il_rows_aligned(a, K, sizeof(TG)));
  auto kernel = range ? (il ? long_matvec_kernel<W, TG, K, true, true, PREFIX>
                            : long_matvec_kernel<W, TG, K, true, false, PREFIX>)
                      : (il ? long_matvec_kernel<W, TG, K, false, true, PREFIX>
                            : long_matvec_kernel<W, TG, K, false, false, PREFIX>);
  // sized by the sector's fermion count, so that the rest of the SM's shared storage stays L1
  const size_t smem = PREFIX ? 2 * (size_t)(f.nbr_fermions + 1) * kLongThreads * sizeof(int) : 0;
  const long long rows = (a.out_last > 0 ? a.out_last : f.dim) - a.out_first;
  kernel<<<grid_for(rows), kLongThreads, smem, s>>>(f, a);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename W, typename TG, int K>
int launch_word(const FqheLongDevice& f, const MatvecArgs& a, cudaStream_t s) {
  return f.nbr_fermions <= kPrefixFermions ? launch_prefix<W, TG, K, true>(f, a, s)
                                           : launch_prefix<W, TG, K, false>(f, a, s);
}

// one 64-bit word per state when every orbital fits (lz_max <= 63), the 128-bit form above
template <typename TG, int K>
int launch_typed(const FqheLongDevice& f, const MatvecArgs& a, cudaStream_t s) {
  return f.lz_max <= 63 ? launch_word<uint64_t, TG, K>(f, a, s) : launch_word<U128, TG, K>(f, a, s);
}

template <typename TG>
int launch_k(const FqheLongDevice& f, const MatvecArgs& a, cudaStream_t s) {
  // blocks of K vectors per pass; any vector count in passes of 4, 2 and 1
  MatvecArgs b = a;
  int done = 0;
  while (done < a.nbr_vectors) {
    const int left = a.nbr_vectors - done;
    const int k = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    b.x = static_cast<const TG*>(a.x) + (long long)done * a.vstride;
    b.xdiag = a.xdiag ? a.xdiag + (long long)done * a.vstride : nullptr;
    b.y = static_cast<double*>(a.y) + (long long)done * a.vstride_y;
    b.nbr_vectors = k;
    int rc = (k == 4) ? launch_typed<TG, 4>(f, b, s) : (k == 2) ? launch_typed<TG, 2>(f, b, s) : launch_typed<TG, 1>(f, b, s);
    if (rc != DH_OK) return rc;
    done += k;
  }
  return DH_OK;
}

}  // namespace

int launch_long_unrank(const FqheLongDevice& f, uint64_t* words, cudaStream_t s) {
  if (f.dim == 0) return DH_OK;
  long_unrank_kernel<<<(unsigned)((f.dim + 255) / 256), 256, 0, s>>>(f, words);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_find(const FqheLongDevice& f, const uint64_t* words, long long n, long long* out, cudaStream_t s) {
  if (n == 0) return DH_OK;
  long_find_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, words, n, out);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_count(const FqheLongDevice& f, unsigned long long* total, cudaStream_t s) {
  DH_CUDA(cudaMemsetAsync(total, 0, sizeof(unsigned long long), s));
  if (f.dim == 0) return DH_OK;
  if (f.lz_max <= 63)
    long_count_kernel<uint64_t><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, total);
  else
    long_count_kernel<U128><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, total);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_row_counts(const FqheLongDevice& f, int* counts, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  if (f.lz_max <= 63)
    long_row_counts_kernel<uint64_t><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, counts);
  else
    long_row_counts_kernel<U128><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, counts);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_ell_fill(const FqheLongDevice& f, int nbr_factors, const long long* slice_ptr, const int* slice_len,
                         int* cols, uint32_t* coef, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  if (f.lz_max <= 63)
    long_ell_fill_kernel<uint64_t><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, nbr_factors, slice_ptr, slice_len, cols,
                                                                              coef);
  else
    long_ell_fill_kernel<U128><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, nbr_factors, slice_ptr, slice_len, cols, coef);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_diag(const FqheLongDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  if (f.lz_max <= 63)
    long_diag_kernel<uint64_t><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, factors64, diag64, diag32);
  else
    long_diag_kernel<U128><<<grid_for(f.dim), kLongThreads, 0, s>>>(f, factors64, diag64, diag32);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_long_bins(const FqheLongDevice& f, int nbr_factors, const double* u, const double* v, double* partial_bins,
                     int nblocks, double* bins, cudaStream_t s) {
  const int smem = nbr_factors * (int)sizeof(double);
  const bool shared = smem <= 200 * 1024;
  if (!shared) DH_CUDA(cudaMemsetAsync(bins, 0, (size_t)nbr_factors * sizeof(double), s));
  if (f.dim > 0) {
    if (shared) {
      auto kern = (f.lz_max <= 63) ? long_bins_kernel<uint64_t, true> : long_bins_kernel<U128, true>;
      if (smem > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      kern<<<nblocks, kLongThreads, smem, s>>>(f, nbr_factors, u, v, partial_bins);
    } else {
      auto kern = (f.lz_max <= 63) ? long_bins_kernel<uint64_t, false> : long_bins_kernel<U128, false>;
      kern<<<nblocks, kLongThreads, 0, s>>>(f, nbr_factors, u, v, bins);
    }
    DH_CUDA(cudaGetLastError());
  }
  if (shared) {
    long_sum_partial_bins<<<(nbr_factors + 255) / 256, 256, 0, s>>>(partial_bins, f.dim > 0 ? nblocks : 0, nbr_factors,
                                                                    bins);
    DH_CUDA(cudaGetLastError());
  }
  return DH_OK;
}

int launch_long_matvec(const FqheLongDevice& f, const MatvecArgs& a, int precision, cudaStream_t s) {
  DH_CHECK(f.lz_max >= 1 && f.lz_max <= 126, DH_ERR_ARGUMENT, "bad FermionOnSphereLong space");
  if (f.dim == 0) return DH_OK;
  return precision == DH_PRECISION_FP32 ? launch_k<float>(f, a, s) : launch_k<double>(f, a, s);
}

}  // namespace dh

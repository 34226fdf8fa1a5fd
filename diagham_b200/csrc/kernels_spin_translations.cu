// The periodic J1-J2 chain in a momentum sector: Spin1_2ChainWithTranslations (fixed Sz, elementary
// translation of one site) with SpinChainJ1J2RealHamiltonianWithTranslations (sm_100a).
//
// Basis (Spin1_2ChainWithTranslations.cc:167-235): the words of the Sz sector that are their own
// canonical form (the smallest of their L rotations) and whose orbit size o (rotations back to the
// word) satisfies K o = 0 mod L, in ascending order; NbrStateInOrbit = o.
//
// Product (SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192 with SymmetrizeResult,
// Spin1_2ChainWithTranslations.h:419): a flip of an antiparallel bond of representative s gives a
// word w; its canonical form c = rotation n of w (the first smallest), the target is c's index t,
// and the element is J/2 sqrt(o_s / o_t) cos(2 pi K ((L - n) mod L) / L).  The matrix is real
// symmetric for K = 0 and K = L/2, so the pull form y[s] = sum over flips of s of that element times
// x[t] equals the reference's push form.
//
// B200 layout, two forms.  Canonical (default): every flipped word is canonicalised in registers (its
// L rotations by funnel shifts, the first smallest kept with its rotation count n) and found among
// the representatives (75 MB at L = 32, mostly L2-resident) through a lookup table over their top
// bits and a short bisection; the target's orbit size is the representative's.  Map (optional, the
// DH_TRANS_MAP=1 environment at set-up): a table over the whole Sz sector, indexed by the word's plain
// Spin1_2Chain index (computed from the row's own index with step tables), holds for every word the
// index of its representative, n and its orbit size (8 bytes a word, 4.8 GB at L = 32): one step-
// table rank and one random 8-byte load per element instead of the rotations and the search.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"
#include "dh_spin_tables.cuh"

namespace dh {
namespace {

constexpr int kTransThreads = 256;

__device__ __forceinline__ uint32_t rotr1(uint32_t w, int L, uint32_t mask) {
  return ((w >> 1) | (w << (L - 1))) & mask;
}

__device__ __forceinline__ long long binom64(int n, int k) {
  if (k < 0 || k > n) return 0;
  long long c = 1;
  for (int q = 1; q <= k; ++q) c = c * (n - k + q) / q;
  return c;
}

// the word of ascending rank q among the L-bit words with n ones (colex order)
__device__ uint32_t unrank_ascending(long long q, int L, int n) {
  uint32_t w = 0;
  int k = n;
  for (int pos = L - 1; pos >= 0 && k > 0; --pos) {
    const long long c = binom64(pos, k);
    if (q >= c) {
      w |= 1u << pos;
      q -= c;
      --k;
    }
  }
  return w;
}

// canonical form (first smallest rotation), rotations to it and orbit size
__device__ __forceinline__ void canonical(uint32_t w, int L, uint32_t mask, uint32_t& c, int& n, int& orbit) {
  c = w;
  n = 0;
  orbit = L;
  uint32_t t = w;
  for (int k = 1; k < L; ++k) {
    t = rotr1(t, L, mask);
    if (t == w && orbit == L) orbit = k;
    if (t < c) {
      c = t;
      n = k;
    }
  }
}

// pass 1: per chunk of 1024 ascending ranks, the number of representatives
__global__ void rep_count_kernel(long long total, int L, int n_up, int momentum, unsigned int* chunk_count) {
  const uint32_t mask = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const long long base = (long long)blockIdx.x * 1024;
  unsigned int cnt = 0;
  for (int j = threadIdx.x; j < 1024; j += blockDim.x) {
    const long long q = base + j;
    if (q >= total) break;
    const uint32_t w = unrank_ascending(q, L, n_up);
    uint32_t c;
    int nn, o;
    canonical(w, L, mask, c, nn, o);
    if (c == w && ((long long)o * momentum) % L == 0) ++cnt;
  }
  for (int s = 16; s > 0; s >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, s);
  __shared__ unsigned int part[kTransThreads / 32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = 0;
    for (int i = 0; i < kTransThreads / 32; ++i) t += part[i];
    chunk_count[blockIdx.x] = t;
  }
}

// pass 2: the representatives in ascending order (chunk offsets from pass 1), with their orbit sizes;
// 256 threads take 4 consecutive ranks each and place them with a block scan
__global__ void rep_write_kernel(long long total, int L, int n_up, int momentum, const long long* chunk_offset,
                                 uint32_t* reps, uint8_t* orbits) {
  const uint32_t mask = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  __shared__ unsigned int scan[kTransThreads];
  const long long q0 = (long long)blockIdx.x * 1024 + threadIdx.x * 4;
  uint32_t words[4];
  int orb[4];
  unsigned int keep = 0;
  for (int j = 0; j < 4; ++j) {
    const long long q = q0 + j;
    words[j] = 0;
    orb[j] = 0;
    if (q >= total) continue;
    const uint32_t w = unrank_ascending(q, L, n_up);
    uint32_t c;
    int nn, o;
    canonical(w, L, mask, c, nn, o);
    if (c == w && ((long long)o * momentum) % L == 0) {
      words[j] = w;
      orb[j] = o;
      keep |= 1u << j;
    }
  }
  scan[threadIdx.x] = __popc(keep);
  __syncthreads();
  for (int s = 1; s < kTransThreads; s <<= 1) {
    const unsigned int v = (threadIdx.x >= (unsigned)s) ? scan[threadIdx.x - s] : 0u;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  long long pos = chunk_offset[blockIdx.x] + scan[threadIdx.x] - __popc(keep);
  for (int j = 0; j < 4; ++j)
    if ((keep >> j) & 1u) {
      reps[pos] = words[j];
      orbits[pos] = (uint8_t)orb[j];
      ++pos;
    }
}

// lookup table over the representatives: table[v] = first index whose word >> shift is >= v
__global__ void rep_table_kernel(const uint32_t* reps, long long dim, int shift, long long entries, int* table) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < entries; v += stride) {
    const unsigned long long key = (unsigned long long)v << shift;
    long long lo = 0, hi = dim;  // first index with reps[i] >= key
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if ((unsigned long long)reps[mid] >= key)
        hi = mid;
      else
        lo = mid + 1;
    }
    table[v] = (int)lo;
  }
}

// index of representative c, or -1
__device__ __forceinline__ long long rep_find(const TransDevice& d, uint32_t c) {
  const long long v = (long long)(c >> d.table_shift);
  if (v + 1 >= d.table_entries) return -1;
  long long lo = d.table[v], hi = d.table[v + 1];
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (d.reps[mid] >= c)
      hi = mid;
    else
      lo = mid + 1;
  }
  return (lo < d.dim && d.reps[lo] == c) ? lo : -1;
}

// rotation of an L-bit word by s sites towards the low bits (s rotr1 steps), 0 <= s < L
// Rotations within L bits by one funnel shift: with W = w | w << L (2L bits), the low L bits of W >> s
// are w rotated right by s (0 <= s < L).  lo, hi are the low and high 32 bits of W.
struct RotWord {
  uint32_t lo, hi;
};
__device__ __forceinline__ RotWord rot_prep(uint32_t w, int L) {
  const uint64_t W = (uint64_t)w | ((uint64_t)w << L);
  return {(uint32_t)W, (uint32_t)(W >> 32)};
}
__device__ __forceinline__ uint32_t rot_apply(RotWord r, int s, uint32_t mask) {
  return __funnelshift_r(r.lo, r.hi, s) & mask;
}

// The smallest of the L rotations of w (rotr1 steps) and the number n of steps to it, the first (the
// smallest n) when several rotations give it.  The smallest rotation starts with the longest run of
// zeros at its top, so only the rotations that put a longest zero run there are compared: with
// A_t bit p = 1 iff bits p .. p + t - 1 (cyclically) of w are all zero, the longest run length T is
// the last t with A_t != 0, and each run start p in A_T gives the candidate n = p + T (mod L).
__device__ __forceinline__ uint32_t canonical_rotation(uint32_t w, int L, uint32_t mask, int& n) {
  const uint32_t z = ~w & mask;
  n = 0;
  if (z == 0) return w;  // all ones: every rotation is w
  const RotWord zr = rot_prep(z, L);
  uint32_t a = z;
  int t = 1;
  while (t < L) {
    const uint32_t next = a & rot_apply(zr, t, mask);
    if (next == 0) break;
    a = next;
    ++t;
  }
  // candidates in increasing n: n = (p + t) mod L for every set bit p of a
  uint32_t rem = rot_apply(rot_prep(a, L), L - t, mask);  // bit (p + t) mod L for each p
  const RotWord wr = rot_prep(w, L);
  uint32_t c = 0xffffffffu;
  while (rem) {
    const int j = __ffs(rem) - 1;
    rem &= rem - 1u;
    const uint32_t r = rot_apply(wr, j, mask);
    if (r < c) {
      c = r;
      n = j;
    }
  }
  return c;
}

// index of representative c through the read-only path, or -1 (dimensions below 2^31)
__device__ __forceinline__ int rep_find_ro(const TransDevice& d, uint32_t c) {
  const long long v = (long long)(c >> d.table_shift);
  if (v + 1 >= d.table_entries) return -1;
  int lo = __ldg(d.table + v), hi = __ldg(d.table + v + 1);
  while (lo < hi) {
    const int mid = (int)(((unsigned)lo + (unsigned)hi) >> 1);
    if (__ldg(d.reps + mid) >= c)
      hi = mid;
    else
      lo = mid + 1;
  }
  return (lo < (int)d.dim && __ldg(d.reps + lo) == c) ? lo : -1;
}

// the map entry of a flipped word computed in registers: representative index | n << 32 |
// orbit << 40, or 0xffffffff when the word's orbit is not in the sector
__device__ __forceinline__ unsigned long long canonical_entry(const TransDevice& d, uint32_t wf, int L, uint32_t mask) {
  int n = 0;
  const uint32_t c = canonical_rotation(wf, L, mask, n);
  const int t = rep_find_ro(d, c);
  if (t < 0) return 0xffffffffull;
  return (unsigned long long)t | ((unsigned long long)n << 32) | ((unsigned long long)__ldg(d.orbits + t) << 40);
}

// every word of the Sz sector (ascending rank q): its plain chain index, the index of its
// representative (or none), the rotations to it and its orbit size; and each representative's own
// plain chain index
__global__ void __launch_bounds__(kTransThreads) trans_map_kernel(TransDevice d, long long total, int n_up) {
  __shared__ SpinTables tb;
  build_spin_tables(tb, d.length);
  const int L = d.length;
  const uint32_t mask = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
    const uint32_t w = unrank_ascending(q, L, n_up);
    uint32_t c;
    int n, o;
    canonical(w, L, mask, c, n, o);
    const long long t = rep_find(d, c);
    const int r = spin_rank_index(tb, w, L, (int)d.chain_dim);
    unsigned long long e = 0xffffffffull;
    if (t >= 0) e = (unsigned long long)t | ((unsigned long long)n << 32) | ((unsigned long long)o << 40);
    d.map[r] = e;
    if (t >= 0 && c == w) d.rep_rank[t] = r;
  }
}

template <typename TG, int K, bool IL>
__device__ __forceinline__ void trans_gather(const TG* x, const MatvecArgs& a, long long idx, TG (&v)[K]) {
  if constexpr (IL && sizeof(TG) == 4 && K == 4) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(x + idx * 4));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
  } else if constexpr (IL && sizeof(TG) == 4 && K == 2) {
    const float2 q = __ldg(reinterpret_cast<const float2*>(x + idx * 2));
    v[0] = q.x; v[1] = q.y;
  } else if constexpr (IL && sizeof(TG) == 8 && (K == 2 || K == 4)) {
#pragma unroll
    for (int j = 0; j < K; j += 2) {
      const double2 q = __ldg(reinterpret_cast<const double2*>(x + idx * K) + j / 2);
      v[j] = q.x;
      v[j + 1] = q.y;
    }
  } else {
    const TG* p = x + idx * a.ld;
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = __ldg(p + q * a.vstride);
  }
}

// per-block constants; the step tables only where flipped words are ranked (the map form)
struct TransCoefficients {
  double ratio[33 * 33];  // sqrt(o_s / o_t)
  double phase[32];       // cos(2 pi K m / L)
};
template <bool CANON>
struct TransShared : TransCoefficients {
  SpinTables tb;
};
template <>
struct TransShared<true> : TransCoefficients {};

// the antiparallel bonds of a representative, one flip at a time: the flipped word's plain chain
// index (from the row's own index and the step tables) and J / 2 of the bond
struct FlipCursor {
  uint32_t w, f1, f2;
  int r, wraps;  // wraps: bit 0 J1 (L-1, 0), bit 1 J2 (L-2, 0), bit 2 J2 (L-1, 1)
};

__device__ __forceinline__ FlipCursor flip_cursor(uint32_t w, int r, int L) {
  const uint32_t maskL = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const uint32_t d1 = w ^ (((w >> 1) | (w << (L - 1))) & maskL);
  const uint32_t d2 = w ^ (((w >> 2) | (w << (L - 2))) & maskL);
  FlipCursor c;
  c.w = w;
  c.r = r;
  c.f1 = d1 & (maskL >> 1);
  c.f2 = d2 & (maskL >> 2);
  c.wraps = (int)((d1 >> (L - 1)) & 1u) | ((int)((d2 >> (L - 2)) & 1u) << 1) | ((int)((d2 >> (L - 1)) & 1u) << 2);
  return c;
}

template <typename TG>
__device__ __forceinline__ bool next_flip(FlipCursor& c, const SpinTables& tb, int L, int D, TG hj1, TG hj2, int& ci,
                                          TG& hj) {
  const uint32_t w = c.w;
  if (c.f1) {
    const int ja = __ffs(c.f1) - 1;
    c.f1 &= c.f1 - 1u;
    const int da = tb.j1[(ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 2))];
    ci = ((w >> ja) & 1u) ? c.r + da : c.r - da;
    hj = hj1;
    return true;
  }
  if (c.f2) {
    const int ja = __ffs(c.f2) - 1;
    c.f2 &= c.f2 - 1u;
    const int da = tb.j2[(((w >> (ja + 1)) & 1u) << 10) | (ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 3))];
    ci = ((w >> ja) & 1u) ? c.r + da : c.r - da;
    hj = hj2;
    return true;
  }
  if (c.wraps & 1) {
    c.wraps &= ~1;
    ci = spin_rank_index(tb, w ^ (1u | (1u << (L - 1))), L, D);
    hj = hj1;
    return true;
  }
  if (c.wraps & 2) {
    c.wraps &= ~2;
    ci = spin_rank_index(tb, w ^ (1u | (1u << (L - 2))), L, D);
    hj = hj2;
    return true;
  }
  if (c.wraps & 4) {
    c.wraps = 0;
    ci = spin_rank_index(tb, w ^ (2u | (1u << (L - 1))), L, D);
    hj = hj2;
    return true;
  }
  return false;
}

// the same bonds as next_flip, giving the flip's bit mask (the flipped word is w ^ mask)
template <typename TG>
__device__ __forceinline__ bool next_flip_mask(FlipCursor& c, int L, TG hj1, TG hj2, uint32_t& fm, TG& hj) {
  if (c.f1) {
    const int ja = __ffs(c.f1) - 1;
    c.f1 &= c.f1 - 1u;
    fm = 3u << ja;
    hj = hj1;
    return true;
  }
  if (c.f2) {
    const int ja = __ffs(c.f2) - 1;
    c.f2 &= c.f2 - 1u;
    fm = 5u << ja;
    hj = hj2;
    return true;
  }
  if (c.wraps & 1) {
    c.wraps &= ~1;
    fm = 1u | (1u << (L - 1));
    hj = hj1;
    return true;
  }
  if (c.wraps & 2) {
    c.wraps &= ~2;
    fm = 1u | (1u << (L - 2));
    hj = hj2;
    return true;
  }
  if (c.wraps & 4) {
    c.wraps = 0;
    fm = 2u | (1u << (L - 1));
    hj = hj2;
    return true;
  }
  return false;
}

// flips are taken kTransBatch at a time: their map loads are all issued before the first is used,
// then their gathers, so several independent load chains are in flight per thread
constexpr int kTransBatch = 4;

// CANON: targets from canonicalising the flipped words (no whole-sector map)
template <typename TG, int K, bool IL, bool RANGE, bool CANON>
__global__ void __launch_bounds__(kTransThreads) trans_matvec_kernel(TransDevice d, MatvecArgs a) {
  __shared__ TransShared<CANON> sh;
  if constexpr (!CANON) build_spin_tables(sh.tb, d.length);
  for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) {
    const int os = i / 33, ot = i % 33;
    sh.ratio[i] = (os > 0 && ot > 0) ? sqrt((double)os / (double)ot) : 0.0;
  }
  for (int i = threadIdx.x; i < 32; i += blockDim.x) sh.phase[i] = d.phase[i];
  __syncthreads();
  const int L = d.length;
  const int D = (int)d.chain_dim;
  const uint32_t maskL = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const TG hj1 = (TG)(0.5 * d.j1), hj2 = (TG)(0.5 * d.j2);
  const TG* x = static_cast<const TG*>(a.x);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : d.dim;
  for (long long s = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; s < r_end; s += stride) {
    const uint32_t w = __ldg(d.reps + s);
    const int r = CANON ? 0 : __ldg(d.rep_rank + s);
    const int os = d.orbits[s];
    const uint32_t d1 = w ^ (((w >> 1) | (w << (L - 1))) & maskL);
    const uint32_t d2 = w ^ (((w >> 2) | (w << (L - 2))) & maskL);
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    FlipCursor cur = flip_cursor(w, r, L);
    bool more = true;
    while (more) {
      int ci[kTransBatch];
      TG hj[kTransBatch];
      bool have[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        if constexpr (CANON) {
          uint32_t fm = 0;
          have[q] = more && next_flip_mask<TG>(cur, L, hj1, hj2, fm, hj[q]);
          ci[q] = (int)fm;
        } else {
          if constexpr (!CANON) have[q] = more && next_flip<TG>(cur, sh.tb, L, D, hj1, hj2, ci[q], hj[q]);
        }
        more = have[q];
      }
      unsigned long long e[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        if constexpr (CANON)
          e[q] = have[q] ? canonical_entry(d, w ^ (uint32_t)ci[q], L, maskL) : 0xffffffffull;
        else
          e[q] = have[q] ? __ldg(d.map + ci[q]) : 0xffffffffull;
      }
      TG c[kTransBatch];
      unsigned int t[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        t[q] = (unsigned int)(e[q] & 0xffffffffull);
        bool ok = t[q] != 0xffffffffu;  // the flipped word's orbit is not in this momentum sector
        if (RANGE) ok = ok && (long long)t[q] >= a.col_first && (long long)t[q] < a.col_last;
        const int n = (int)((e[q] >> 32) & 0xffull), ot = (int)((e[q] >> 40) & 0xffull);
        c[q] = ok ? hj[q] * (TG)(sh.ratio[os * 33 + ot] * sh.phase[n ? L - n : 0]) : TG(0);
        if (!ok) t[q] = (unsigned int)s;  // a harmless in-range gather with a zero coefficient
      }
      TG v[kTransBatch][K];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) trans_gather<TG, K, IL>(x, a, t[q], v[q]);
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q)
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += c[q] * v[q][j];
    }
    // diagonal: J/4 (L - 2 #antiparallel bonds) per bond type (SzSzContributions), plus the shift
    const double diag = 0.25 * d.j1 * (double)(L - 2 * __popc(d1)) + 0.25 * d.j2 * (double)(L - 2 * __popc(d2)) +
                        a.shift;
    const bool on_diag = (s >= a.row_first && s < a.row_last);
    double* y = static_cast<double*>(a.y);
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double v = (double)acc[q];
      if (on_diag) {
        const long long xo = IL ? s * K + q : s * a.ld + q * a.vstride;
        const double xd = a.xdiag ? a.xdiag[xo] : (double)x[xo];
        v += diag * xd;
      }
      double* yp = y + (IL ? s * K + q : s * a.ld_y + q * a.vstride_y);
      *yp = a.accumulate ? (*yp + v) : v;
    }
  }
}

template <bool CANON>
struct TransSharedComplex {
  double ratio[33 * 33];  // sqrt(o_s / o_t)
  double phase[32];       // cos(2 pi K m / L)
  double sine[32];        // sin(2 pi K m / L)
  SpinTables tb;
};
template <>
struct TransSharedComplex<true> {
  double ratio[33 * 33];
  double phase[32];
  double sine[32];
};

// SpinChainJ1J2HamiltonianWithTranslations (any K) on complex vectors stored as (Re, Im) pairs; the
// row, column and output ranges of the arguments count doubles (twice the complex index).  The
// reference pushes h(s -> t) = J/2 sqrt(o_s / o_t) exp(2 pi i K m / L) x[s] into y[t]
// (SpinChainJ1J2HamiltonianWithTranslations.cc:149-247); H is Hermitian, so the pull form takes the
// conjugate: y[s] += conj(h(s -> t)) x[t].
template <typename TG, bool RANGE, bool CANON>
__global__ void __launch_bounds__(kTransThreads) trans_matvec_complex_kernel(TransDevice d, MatvecArgs a) {
  __shared__ TransSharedComplex<CANON> sh;
  if constexpr (!CANON) build_spin_tables(sh.tb, d.length);
  for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) {
    const int os = i / 33, ot = i % 33;
    sh.ratio[i] = (os > 0 && ot > 0) ? sqrt((double)os / (double)ot) : 0.0;
  }
  for (int i = threadIdx.x; i < 32; i += blockDim.x) {
    sh.phase[i] = d.phase[i];
    sh.sine[i] = d.sine[i];
  }
  __syncthreads();
  const int L = d.length;
  const uint32_t maskL = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const TG* x = static_cast<const TG*>(a.x);
  double* y = static_cast<double*>(a.y);
  const long long c_first = a.col_first / 2, c_last = a.col_last / 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = (a.out_last > 0 ? a.out_last : 2 * d.dim) / 2;
  for (long long s = a.out_first / 2 + (long long)blockIdx.x * blockDim.x + threadIdx.x; s < r_end; s += stride) {
    const uint32_t w = __ldg(d.reps + s);
    const int r = CANON ? 0 : __ldg(d.rep_rank + s);
    const int os = d.orbits[s];
    TG re = TG(0), im = TG(0);
    // flips kTransBatch at a time, their map loads and then their gathers in flight together
    const TG hj1 = (TG)(0.5 * d.j1), hj2 = (TG)(0.5 * d.j2);
    FlipCursor cur = flip_cursor(w, r, L);
    bool more = true;
    while (more) {
      int ci[kTransBatch];
      TG hj[kTransBatch];
      bool have[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        if constexpr (CANON) {
          uint32_t fm = 0;
          have[q] = more && next_flip_mask<TG>(cur, L, hj1, hj2, fm, hj[q]);
          ci[q] = (int)fm;
        } else {
          if constexpr (!CANON) have[q] = more && next_flip<TG>(cur, sh.tb, L, (int)d.chain_dim, hj1, hj2, ci[q], hj[q]);
        }
        more = have[q];
      }
      unsigned long long e[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        if constexpr (CANON)
          e[q] = have[q] ? canonical_entry(d, w ^ (uint32_t)ci[q], L, maskL) : 0xffffffffull;
        else
          e[q] = have[q] ? __ldg(d.map + ci[q]) : 0xffffffffull;
      }
      TG cr[kTransBatch], cim[kTransBatch];
      unsigned int t[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        t[q] = (unsigned int)(e[q] & 0xffffffffull);
        bool ok = t[q] != 0xffffffffu;  // the flipped word's orbit is not in this momentum sector
        if (RANGE) ok = ok && (long long)t[q] >= c_first && (long long)t[q] < c_last;
        const int n = (int)((e[q] >> 32) & 0xffull), ot = (int)((e[q] >> 40) & 0xffull);
        const int m = n ? L - n : 0;
        const double mag = ok ? sh.ratio[os * 33 + ot] : 0.0;
        cr[q] = hj[q] * (TG)(mag * sh.phase[m]);
        cim[q] = -hj[q] * (TG)(mag * sh.sine[m]);
        if (!ok) t[q] = (unsigned int)s;  // a harmless in-range gather with a zero coefficient
      }
      TG xr[kTransBatch], xi[kTransBatch];
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        if constexpr (sizeof(TG) == 8) {
          const double2 v = __ldg(reinterpret_cast<const double2*>(x) + t[q]);
          xr[q] = v.x;
          xi[q] = v.y;
        } else {
          const float2 v = __ldg(reinterpret_cast<const float2*>(x) + t[q]);
          xr[q] = v.x;
          xi[q] = v.y;
        }
      }
#pragma unroll
      for (int q = 0; q < kTransBatch; ++q) {
        re += cr[q] * xr[q] - cim[q] * xi[q];
        im += cr[q] * xi[q] + cim[q] * xr[q];
      }
    }
    const uint32_t d1 = w ^ (((w >> 1) | (w << (L - 1))) & maskL);
    const uint32_t d2 = w ^ (((w >> 2) | (w << (L - 2))) & maskL);
    double vr = (double)re, vi = (double)im;
    if (2 * s >= a.row_first && 2 * s < a.row_last) {
      const double diag = 0.25 * d.j1 * (double)(L - 2 * __popc(d1)) + 0.25 * d.j2 * (double)(L - 2 * __popc(d2)) +
                          a.shift;
      const double xr = a.xdiag ? a.xdiag[2 * s] : (double)x[2 * s];
      const double xi = a.xdiag ? a.xdiag[2 * s + 1] : (double)x[2 * s + 1];
      vr += diag * xr;
      vi += diag * xi;
    }
    if (a.accumulate) {
      vr += y[2 * s];
      vi += y[2 * s + 1];
    }
    reinterpret_cast<double2*>(y)[s] = make_double2(vr, vi);
  }
}

// elements of one product (antiparallel bonds of the representatives, and those in the sector)
template <bool CANON>
__global__ void __launch_bounds__(kTransThreads) trans_count_kernel(TransDevice d, unsigned long long* total) {
  __shared__ SpinTables tb;
  build_spin_tables(tb, d.length);
  const int L = d.length;
  const int D = (int)d.chain_dim;
  const uint32_t maskL = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  unsigned long long bonds = 0, kept = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < d.dim; s += stride) {
    const uint32_t w = d.reps[s];
    const uint32_t d1 = w ^ (((w >> 1) | (w << (L - 1))) & maskL);
    const uint32_t d2 = w ^ (((w >> 2) | (w << (L - 2))) & maskL);
    bonds += __popc(d1) + __popc(d2);
    if constexpr (CANON) {
      FlipCursor cur = flip_cursor(w, 0, L);
      uint32_t fm = 0;
      double hj = 0.0;
      while (next_flip_mask<double>(cur, L, 0.0, 0.0, fm, hj))
        kept += (canonical_entry(d, w ^ fm, L, maskL) & 0xffffffffull) != 0xffffffffull;
      continue;
    }
    const int r = d.rep_rank[s];
    uint32_t f = d1 & (maskL >> 1);
    while (f) {
      const int ja = __ffs(f) - 1;
      f &= f - 1u;
      const int da = tb.j1[(ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 2))];
      kept += (d.map[((w >> ja) & 1u) ? r + da : r - da] & 0xffffffffull) != 0xffffffffull;
    }
    f = d2 & (maskL >> 2);
    while (f) {
      const int ja = __ffs(f) - 1;
      f &= f - 1u;
      const int da = tb.j2[(((w >> (ja + 1)) & 1u) << 10) | (ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 3))];
      kept += (d.map[((w >> ja) & 1u) ? r + da : r - da] & 0xffffffffull) != 0xffffffffull;
    }
    if ((d1 >> (L - 1)) & 1u)
      kept += (d.map[spin_rank_index(tb, w ^ (1u | (1u << (L - 1))), L, D)] & 0xffffffffull) != 0xffffffffull;
    if ((d2 >> (L - 2)) & 1u)
      kept += (d.map[spin_rank_index(tb, w ^ (1u | (1u << (L - 2))), L, D)] & 0xffffffffull) != 0xffffffffull;
    if ((d2 >> (L - 1)) & 1u)
      kept += (d.map[spin_rank_index(tb, w ^ (2u | (1u << (L - 1))), L, D)] & 0xffffffffull) != 0xffffffffull;
  }
  for (int o = 16; o > 0; o >>= 1) {
    bonds += __shfl_down_sync(0xffffffffu, bonds, o);
    kept += __shfl_down_sync(0xffffffffu, kept, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(total, bonds);
    atomicAdd(total + 1, kept);
  }
}

__global__ void trans_find_kernel(TransDevice d, const uint64_t* words, long long n, long long* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t w = words[i];
  out[i] = (w >> 32) ? -1 : rep_find(d, (uint32_t)w);
}

template <typename TG, int K>
int launch_trans_typed(const TransDevice& d, const MatvecArgs& a, cudaStream_t s) {
  const bool range = a.col_first > 0 || a.col_last < d.dim;
  const bool il = (K > 1) && a.ld == K && a.vstride == 1 && a.ld_y == K && a.vstride_y == 1 &&
                  il_rows_aligned(a, K, sizeof(TG));
  auto kern = range ? (il ? trans_matvec_kernel<TG, K, true, true, true> : trans_matvec_kernel<TG, K, false, true, true>)
                    : (il ? trans_matvec_kernel<TG, K, true, false, true> : trans_matvec_kernel<TG, K, false, false, true>);
  if (d.map)
    kern = range ? (il ? trans_matvec_kernel<TG, K, true, true, false> : trans_matvec_kernel<TG, K, false, true, false>)
                 : (il ? trans_matvec_kernel<TG, K, true, false, false> : trans_matvec_kernel<TG, K, false, false, false>);
  int dev = 0, sms = 148, per_sm = 1;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTransThreads, 0));
  const long long rows = (a.out_last > 0 ? a.out_last : d.dim) - a.out_first;
  long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const long long need = (rows + kTransThreads - 1) / kTransThreads;
  if (need < grid) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, kTransThreads, 0, s>>>(d, a);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename TG>
int launch_trans_k(const TransDevice& d, const MatvecArgs& a, cudaStream_t s) {
  MatvecArgs b = a;
  int done = 0;
  while (done < a.nbr_vectors) {
    const int left = a.nbr_vectors - done;
    const int k = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    b.x = static_cast<const TG*>(a.x) + (long long)done * a.vstride;
    b.xdiag = a.xdiag ? a.xdiag + (long long)done * a.vstride : nullptr;
    b.y = static_cast<double*>(a.y) + (long long)done * a.vstride_y;
    b.nbr_vectors = k;
    int rc = (k == 4) ? launch_trans_typed<TG, 4>(d, b, s)
                      : (k == 2) ? launch_trans_typed<TG, 2>(d, b, s) : launch_trans_typed<TG, 1>(d, b, s);
    if (rc != DH_OK) return rc;
    done += k;
  }
  return DH_OK;
}

}  // namespace

int launch_trans_count(long long total, int L, int n_up, int momentum, unsigned int* chunk_count, cudaStream_t s) {
  const long long chunks = (total + 1023) / 1024;
  if (chunks <= 0) return DH_OK;
  rep_count_kernel<<<(unsigned)chunks, kTransThreads, 0, s>>>(total, L, n_up, momentum, chunk_count);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_trans_write(long long total, int L, int n_up, int momentum, const long long* chunk_offset, uint32_t* reps,
                       uint8_t* orbits, cudaStream_t s) {
  const long long chunks = (total + 1023) / 1024;
  if (chunks <= 0) return DH_OK;
  rep_write_kernel<<<(unsigned)chunks, kTransThreads, 0, s>>>(total, L, n_up, momentum, chunk_offset, reps, orbits);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_trans_table(const uint32_t* reps, long long dim, int shift, long long entries, int* table, cudaStream_t s) {
  long long g = (entries + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  rep_table_kernel<<<(unsigned)g, 256, 0, s>>>(reps, dim, shift, entries, table);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_trans_map(const TransDevice& d, long long total, int n_up, cudaStream_t s) {
  long long g = (total + kTransThreads - 1) / kTransThreads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  trans_map_kernel<<<(unsigned)g, kTransThreads, 0, s>>>(d, total, n_up);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename TG>
int launch_trans_complex(const TransDevice& d, const MatvecArgs& a, cudaStream_t s) {
  // vectors one after the other, each 2 dim doubles (or floats) of (Re, Im) pairs
  DH_CHECK(a.nbr_vectors == 1 || a.ld == 1, DH_ERR_UNSUPPORTED, "complex vectors are multiplied one at a time");
  DH_CHECK(((a.out_first | a.out_last | a.col_first | a.col_last | a.row_first | a.row_last) & 1) == 0,
           DH_ERR_ARGUMENT, "complex ranges must cover whole (Re, Im) pairs");
  const bool range = a.col_first > 0 || a.col_last < 2 * d.dim;
  const long long rows = ((a.out_last > 0 ? a.out_last : 2 * d.dim) - a.out_first) / 2;
  long long g = (rows + kTransThreads - 1) / kTransThreads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  for (int v = 0; v < a.nbr_vectors; ++v) {
    MatvecArgs b = a;
    b.x = static_cast<const TG*>(a.x) + (long long)v * a.vstride;
    b.xdiag = a.xdiag ? a.xdiag + (long long)v * a.vstride : nullptr;
    b.y = static_cast<double*>(a.y) + (long long)v * a.vstride_y;
    b.nbr_vectors = 1;
    if (d.map) {
      if (range)
        trans_matvec_complex_kernel<TG, true, false><<<(unsigned)g, kTransThreads, 0, s>>>(d, b);
      else
        trans_matvec_complex_kernel<TG, false, false><<<(unsigned)g, kTransThreads, 0, s>>>(d, b);
    } else {
      if (range)
        trans_matvec_complex_kernel<TG, true, true><<<(unsigned)g, kTransThreads, 0, s>>>(d, b);
      else
        trans_matvec_complex_kernel<TG, false, true><<<(unsigned)g, kTransThreads, 0, s>>>(d, b);
    }
    DH_CUDA(cudaGetLastError());
  }
  return DH_OK;
}

int launch_trans_matvec(const TransDevice& d, const MatvecArgs& a, int precision, cudaStream_t s) {
  if (d.dim <= 0) return DH_OK;
  if (d.complex_phases)
    return precision == DH_PRECISION_FP32 ? launch_trans_complex<float>(d, a, s) : launch_trans_complex<double>(d, a, s);
  return precision == DH_PRECISION_FP32 ? launch_trans_k<float>(d, a, s) : launch_trans_k<double>(d, a, s);
}

int launch_trans_find(const TransDevice& d, const uint64_t* words, long long n, long long* out, cudaStream_t s) {
  if (n <= 0) return DH_OK;
  trans_find_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, words, n, out);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_trans_count_elements(const TransDevice& d, unsigned long long* total, cudaStream_t s) {
  DH_CUDA(cudaMemsetAsync(total, 0, 2 * sizeof(unsigned long long), s));
  if (d.dim <= 0) return DH_OK;
  long long g = (d.dim + kTransThreads - 1) / kTransThreads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  if (d.map)
    trans_count_kernel<false><<<(unsigned)g, kTransThreads, 0, s>>>(d, total);
  else
    trans_count_kernel<true><<<(unsigned)g, kTransThreads, 0, s>>>(d, total);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

}  // namespace dh

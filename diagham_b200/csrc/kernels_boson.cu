// Pull-form, atomic-free H.x for bosons on the sphere in the BosonOnSphereShort representation
// (sm_100a).
//
// A bosonic state with occupations n_0 .. n_L is stored as the fermionic word of N ones in L + N
// bit positions: from bit 0 up, n_0 ones, a zero, n_1 ones, a zero, ... (BosonOnSphereShort::
// BosonToFermion, BosonOnSphereShort.h:1231), so the basis, its order and FindStateIndex are those
// of FermionOnSphere(N, 2Lz, L + N - 1) (BosonOnSphereShort.cc:83-93) and the split rank tables of
// that fermionic space give every target's index.
//
// One thread owns one basis row r.  Per row the occupations n_m and the group starts P_m (bit of the
// first one of orbital m, or of its separator when empty) are decoded once.  The move m3 = m1 of
// every pair returns to the row: its coefficient n_m2 (n_m1 - [m1 = m2]) goes to a per-row sum that
// multiplies x[r] once.  The other moves:  For every pair
// m1 >= m2 that a_m1 a_m2 can empty (BosonOnSphereShort::AA, .cc:353) and every creation pair
// m3 >= m4 = m1 + m2 - m3 (AdAd, .cc:431):
//   coefficient  sqrt(n_m2 (n_m1 - [m1 = m2])) * sqrt((n'_m4 + 1)(n'_m3 + 1 + [m3 = m4])),
//                n' = occupations after the annihilations
//   target word  the row word with one bit deleted at P_m1, then at P_m2 (higher position first),
//                then one bit inserted at P'_m3, then at P'_m4 (P' = group starts after the
//                deletions), index = HO[t >> LB] + LR[t & (2^LB - 1)]
//   y[r] += factor(m1, m2, m3) * coefficient * x[index]
// The bosonic Hamiltonian is real symmetric, so this pull form equals the reference's push form
// (AbstractQHEOnSphereHamiltonian.cc:456-488) up to FP rounding.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"

namespace dh {

namespace {

constexpr int kBosonThreads = 128;

__device__ __forceinline__ uint64_t delete_bit(uint64_t w, int p) {
  const uint64_t low = (1ull << p) - 1ull;
  return (w & low) | ((w >> 1) & ~low);
}

__device__ __forceinline__ uint64_t insert_one(uint64_t w, int p) {
  const uint64_t low = (1ull << p) - 1ull;
  return (w & low) | (1ull << p) | ((w & ~low) << 1);
}

template <typename TG>
__device__ __forceinline__ TG coef_sqrt(int v);
template <>
__device__ __forceinline__ double coef_sqrt<double>(int v) {
  return sqrt((double)v);
}
template <>
__device__ __forceinline__ float coef_sqrt<float>(int v) {
  return sqrtf((float)v);
}

// K gathered values of row idx: a row-interleaved block ([row][K]) as one vector load
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

// Ranks beyond the split-word tables (words of more than 41 bits).  With C(n, o, s) the fermionic
// sector's count table, index(w) = dim - 1 - sum over the ones of w of C(n_i, p_i, s_i) (n_i ones at or
// below bit p_i, s_i the sum of their positions).  A move changes the word only between the lowest
// and the highest bit where row and target differ; outside that range every term is the row's, so the
// target's index is the row's corrected by the terms of the ones inside the range.
constexpr int kBosonPrefixParticles = 20;

__device__ __forceinline__ long long count_at(const FqheDevice& f, int n, int o, int s) {
  return (long long)__ldg(f.count_table + (size_t)(n - 1) * f.count_stride_n + (size_t)o * f.count_stride_o + s);
}

// the terms of the ones of w at bits lo..hi, given the count n and position sum s of its ones below lo
__device__ __forceinline__ long long count_terms(const FqheDevice& f, uint64_t w, int lo, int hi, int n, int s) {
  uint64_t bits = w & (((hi >= 63) ? ~0ull : ((2ull << hi) - 1ull)) & ~((1ull << lo) - 1ull));
  long long acc = 0;
  while (bits) {
    const int q = __ffsll(bits) - 1;
    bits &= bits - 1ull;
    ++n;
    s += q;
    acc += count_at(f, n, q, s);
  }
  return acc;
}

__device__ __forceinline__ int position_sum(uint64_t a) {
  return __popcll(a & 0xaaaaaaaaaaaaaaaaull) + 2 * __popcll(a & 0xccccccccccccccccull) +
         4 * __popcll(a & 0xf0f0f0f0f0f0f0f0ull) + 8 * __popcll(a & 0xff00ff00ff00ff00ull) +
         16 * __popcll(a & 0xffff0000ffff0000ull) + 32 * __popcll(a & 0xffffffff00000000ull);
}

// RM = 0: split-word rank tables, factors staged in shared memory; RM = 1: count-table ranks with the
// row's prefix sums (its terms and position sums over its ones, thread-strided in shared memory),
// factors read through the cache; RM = 2: count-table ranks walking row and target, factors cached
template <typename TG, int K, bool RANGE, bool IL, int RM>
__global__ void __launch_bounds__(kBosonThreads) boson_matvec_kernel(FqheDevice f, MatvecArgs a, int factor_smem) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  int* spair = reinterpret_cast<int*>(smem + factor_smem);
  int* term = spair + ((f.nbr_pairs + 3) & ~3);
  int* osum = term + (f.nbr_particles + 1) * kBosonThreads;
  // square roots of the occupation products 0 .. N (N - 1) (every n_m2 (n_m1 - [m1 = m2]) and
  // (n'_m4 + 1)(n'_m3 + 1 + [m3 = m4]) lies in that range)
  TG* ssq = reinterpret_cast<TG*>(RM == 1 ? osum + (f.nbr_particles + 1) * kBosonThreads : term);
  const TG* gfac = static_cast<const TG*>(f.factors);
  if (RM == 0)
    for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
  const TG* fac = (RM == 0) ? sfac : gfac;
  for (int i = threadIdx.x; i < f.nbr_pairs; i += blockDim.x) spair[i] = f.pair_offset[i];
  for (int i = threadIdx.x; i <= f.nbr_particles * (f.nbr_particles - 1); i += blockDim.x) ssq[i] = coef_sqrt<TG>(i);
  __syncthreads();

  const int L = f.boson_lz_max;
  const int LB = f.low_bits;
  const uint64_t lmask = (1ull << LB) - 1ull;
  const TG* x = static_cast<const TG*>(a.x);
  double* y = static_cast<double*>(a.y);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : f.dim;
  // Each lane walks its rows, their annihilated pairs and the pairs' creations as one flat stream,
  // so the lanes of a warp stay converged on the move body whatever the occupations and the number
  // of moves of their rows: a lane that finishes a row starts its next one at once.
  long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= r_end) return;
  uint64_t s = 0, sh = 0, sl = 0, occ = 0, dbl = 0, rem1 = 0, rem2 = 0, an = 0;
  int ho_row = 0, lr_row = 0;
  uint8_t n[64], P[64];
  TG acc[K];
  TG dsum = TG(0), saa = TG(0);
  int m1 = -1, m2 = 0, m3 = 1, m3hi = 0, m4 = 0, q3 = 0, c3 = 0, q4 = 0, c4 = 0;
  const TG* fp = fac;
  // row r's word, the halves of its rank, occupations, group starts and pair masks
  auto open_row = [&]() {
    s = __ldg(f.words + r);
    if (RM == 0) {
      sh = s >> LB;
      sl = s & lmask;
      ho_row = __ldg(f.high_offset + sh);
      lr_row = (int)(r - ho_row);
    } else if (RM == 1) {
      uint64_t bits = s;
      int j = 0, sum = 0;
      long long run = 0;
      term[threadIdx.x] = 0;
      osum[threadIdx.x] = 0;
      while (bits) {
        const int q = __ffsll(bits) - 1;
        bits &= bits - 1ull;
        ++j;
        sum += q;
        run += count_at(f, j, q, sum);
        term[j * kBosonThreads + threadIdx.x] = (int)run;
        osum[j * kBosonThreads + threadIdx.x] = sum;
      }
    }
    occ = 0;
    dbl = 0;
    int pos = 0;
    for (int m = 0; m <= L; ++m) {
      const int c = __ffsll(~(s >> pos)) - 1;  // length of the run of ones starting at pos
      P[m] = (uint8_t)pos;
      n[m] = (uint8_t)c;
      occ |= (uint64_t)(c > 0) << m;
      dbl |= (uint64_t)(c > 1) << m;
      pos += c + 1;
    }
    rem1 = occ;
    rem2 = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    dsum = TG(0);  // the move m3 = m1 of every pair returns to the row itself
    m3 = 1;
    m3hi = 0;
  };
  open_row();
  while (true) {
    if (m3 > m3hi) {
      // next pair of this row: m1 over the occupied orbitals ascending, m2 over the occupied orbitals
      // below m1, then m2 = m1 when orbital m1 holds two bosons or more
      while (rem2 == 0 && rem1 != 0) {
        m1 = __ffsll(rem1) - 1;
        rem1 &= rem1 - 1ull;
        rem2 = (occ & ((1ull << m1) - 1ull)) | (dbl & (1ull << m1));
      }
      if (rem2 == 0) {
        // the row is done
        if (!RANGE || (r >= a.col_first && r < a.col_last)) {
          TG xr[K];
          gather_row<TG, K, IL>(x, a, r, xr);
#pragma unroll
          for (int j = 0; j < K; ++j) acc[j] += dsum * xr[j];
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
        r += stride;
        if (r >= r_end) break;
        open_row();
        continue;
      }
      m2 = __ffsll(rem2) - 1;
      rem2 &= rem2 - 1ull;
      const int n1 = n[m1], n2 = n[m2];
      const int caa = n2 * (n1 - (m1 == m2 ? 1 : 0));
      saa = ssq[caa];
      an = delete_bit(delete_bit(s, P[m1]), P[m2]);
      const int M = m1 + m2;
      const int m3lo = (M + 1) >> 1;
      m3hi = (M < L) ? M : L;
      fp = fac + (spair[m1 * (m1 + 1) / 2 + m2] - m3lo);
      // diagonal move: a+_m1 a+_m2 a_m1 a_m2 gives back the row with coefficient n_m2 (n_m1 - [m1 = m2])
      dsum += fp[m1] * (TG)caa;
      // group start q and occupation c of orbitals m3 (walking up) and m4 = M - m3 (walking down) in
      // the word after the annihilations
      m3 = m3lo;
      m4 = M - m3lo;
      q3 = P[m3] - (m3 > m1) - (m3 > m2);
      c3 = n[m3] - (m3 == m1) - (m3 == m2);
      q4 = P[m4] - (m4 > m1) - (m4 > m2);
      c4 = n[m4] - (m4 == m1) - (m4 == m2);
    }
    if (m3 != m1) {
      const int cad = (m3 == m4) ? (c4 + 1) * (c4 + 2) : (c4 + 1) * (c3 + 1);
      const uint64_t t = insert_one(insert_one(an, q3), q4);
      long long idx;
      if (RM == 0) {
        const uint64_t th = t >> LB, tl = t & lmask;
        int hoi = ho_row, lri = lr_row;
        if (th != sh) hoi = __ldg(f.high_offset + th);
        if (tl != sl) lri = (int)__ldg(f.low_rank + tl);
        idx = (long long)hoi + (long long)lri;
      } else {
        const uint64_t diff = s ^ t;  // never 0: m3 != m1 changes the occupations
        const int lo = __ffsll(diff) - 1, hi = 63 - __clzll(diff);
        const uint64_t low_part = s & ((1ull << lo) - 1ull);
        const int n0 = __popcll(low_part);
        if (RM == 1) {
          const int n1 = __popcll(s & ((hi >= 63) ? ~0ull : ((2ull << hi) - 1ull)));
          const int s0 = osum[n0 * kBosonThreads + threadIdx.x];
          idx = r + (long long)(term[n1 * kBosonThreads + threadIdx.x] - term[n0 * kBosonThreads + threadIdx.x]) -
                count_terms(f, t, lo, hi, n0, s0);
        } else {
          const int s0 = position_sum(low_part);
          idx = r + count_terms(f, s, lo, hi, n0, s0) - count_terms(f, t, lo, hi, n0, s0);
        }
      }
      if (!RANGE || (idx >= a.col_first && idx < a.col_last)) {
        const TG c = fp[m3] * saa * ssq[cad];
        TG xv[K];
        gather_row<TG, K, IL>(x, a, idx, xv);
#pragma unroll
        for (int j = 0; j < K; ++j) acc[j] += c * xv[j];
      }
    }
    if (m3 < m3hi) {
      // next group up: it starts after this group and its separator
      q3 += c3 + 1;
      c3 = __ffsll(~(an >> q3)) - 1;
      // next group down: it ends below the separator at q4 - 1
      const int sep = q4 - 1;
      const uint64_t below = ~an & ((1ull << sep) - 1ull);
      const int z = below ? 63 - __clzll(below) : -1;
      q4 = z + 1;
      c4 = sep - q4;
      --m4;
    }
    ++m3;
  }
}

template <typename TG, int K, int RM>
int launch_rank(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  const int factor_smem = (RM == 0) ? (int)((f.nbr_factors * sizeof(TG) + 15) & ~(size_t)15) : 0;
  size_t smem = (size_t)factor_smem + (size_t)((f.nbr_pairs + 3) & ~3) * sizeof(int);
  if (RM == 1) smem += 2 * (size_t)(f.nbr_particles + 1) * kBosonThreads * sizeof(int);
  smem += ((size_t)f.nbr_particles * (f.nbr_particles - 1) + 2) * sizeof(TG);  // occupation square roots
  const bool range = a.col_first > 0 || a.col_last < f.dim;
  // row-interleaved blocks, or one contiguous vector: row strides known at compile time
  const bool il = K == 1 ? (a.ld == 1 && a.ld_y == 1)
                         : (a.ld == K && a.vstride == 1 && a.ld_y == K && a.vstride_y == 1 &&
                            il_rows_aligned(a, K, sizeof(TG)));
  auto kernel = range ? (il ? boson_matvec_kernel<TG, K, true, true, RM> : boson_matvec_kernel<TG, K, true, false, RM>)
                      : (il ? boson_matvec_kernel<TG, K, false, true, RM> : boson_matvec_kernel<TG, K, false, false, RM>);
  if (smem > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long rows = (a.out_last > 0 ? a.out_last : f.dim) - a.out_first;
  long long blocks = (rows + kBosonThreads - 1) / kBosonThreads;
  const long long cap = (long long)sms * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  kernel<<<(unsigned)blocks, kBosonThreads, smem, s>>>(f, a, factor_smem);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename TG, int K>
int launch_typed(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  if (!f.count_table) return launch_rank<TG, K, 0>(f, a, s);
  return f.nbr_particles <= kBosonPrefixParticles ? launch_rank<TG, K, 1>(f, a, s) : launch_rank<TG, K, 2>(f, a, s);
}

template <typename TG>
int launch_k(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
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

// number of elements (moves, diagonal ones included) that one product generates, block partials
// then one atomic per block
__global__ void __launch_bounds__(kBosonThreads) boson_count_kernel(FqheDevice f, unsigned long long* total) {
  __shared__ unsigned long long part[2][kBosonThreads / 32];
  const int L = f.boson_lz_max;
  unsigned long long c = 0, d = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    uint8_t n[64];
    int pos = 0;
    for (int m = 0; m <= L; ++m) {
      const int k = __ffsll(~(s >> pos)) - 1;
      n[m] = (uint8_t)k;
      pos += k + 1;
    }
    for (int m1 = 0; m1 <= L; ++m1) {
      if (n[m1] == 0) continue;
      for (int m2 = 0; m2 <= m1; ++m2) {
        if (n[m2] == 0 || (m2 == m1 && n[m1] < 2)) continue;
        const int M = m1 + m2;
        c += (unsigned long long)(((M < L) ? M : L) - ((M + 1) >> 1) + 1);
        ++d;  // one of them (m3 = m1) is diagonal
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    c += __shfl_down_sync(0xffffffffu, c, o);
    d += __shfl_down_sync(0xffffffffu, d, o);
  }
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = c;
    part[1][threadIdx.x >> 5] = d;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    unsigned long long t = 0;
    for (int w = 0; w < kBosonThreads / 32; ++w) t += part[threadIdx.x][w];
    atomicAdd(total + threadIdx.x, t);
  }
}

// ------------------------------------------- moves one at a time: stored elements and the adjoint
// The index of target word t of row r (word s): the split-word rank tables, or the count-table walk
// between the lowest and highest changed bits.
__device__ __forceinline__ long long boson_target(const FqheDevice& f, uint64_t s, long long r, uint64_t t) {
  if (!f.count_table)
    return (long long)__ldg(f.high_offset + (t >> f.low_bits)) +
           (long long)__ldg(f.low_rank + (t & ((1ull << f.low_bits) - 1ull)));
  const uint64_t diff = s ^ t;
  const int lo = __ffsll(diff) - 1, hi = 63 - __clzll(diff);
  const uint64_t low_part = s & ((1ull << lo) - 1ull);
  const int n0 = __popcll(low_part), s0 = position_sum(low_part);
  return r + count_terms(f, s, lo, hi, n0, s0) - count_terms(f, t, lo, hi, n0, s0);
}

// Visits every move of row r (word s) in the product kernel's order: m1 ascending over the occupied
// orbitals, m2 ascending over the occupied orbitals below m1 then m2 = m1 when orbital m1 holds two
// bosons or more, m3 = ceil(M / 2) .. min(M, L) ascending.  visit(target, factor index, caa, cad,
// diagonal): the element is factor * sqrt(caa) * sqrt(cad) for a move to another word, and
// factor * caa for the diagonal move m3 = m1 (target r, cad unused).
template <typename Visit>
__device__ __forceinline__ void boson_visit_row(const FqheDevice& f, long long r, uint64_t s, Visit&& visit) {
  const int L = f.boson_lz_max;
  uint8_t n[64], P[64];
  uint64_t occ = 0, dbl = 0;
  int pos = 0;
  for (int m = 0; m <= L; ++m) {
    const int c = __ffsll(~(s >> pos)) - 1;
    P[m] = (uint8_t)pos;
    n[m] = (uint8_t)c;
    occ |= (uint64_t)(c > 0) << m;
    dbl |= (uint64_t)(c > 1) << m;
    pos += c + 1;
  }
  uint64_t rem1 = occ;
  while (rem1) {
    const int m1 = __ffsll(rem1) - 1;
    rem1 &= rem1 - 1ull;
    uint64_t rem2 = (occ & ((1ull << m1) - 1ull)) | (dbl & (1ull << m1));
    while (rem2) {
      const int m2 = __ffsll(rem2) - 1;
      rem2 &= rem2 - 1ull;
      const int caa = n[m2] * (n[m1] - (m1 == m2 ? 1 : 0));
      const uint64_t an = delete_bit(delete_bit(s, P[m1]), P[m2]);
      const int M = m1 + m2;
      const int m3lo = (M + 1) >> 1, m3hi = (M < L) ? M : L;
      const int fb = __ldg(f.pair_offset + (m1 * (m1 + 1) / 2 + m2)) - m3lo;
      for (int m3 = m3lo; m3 <= m3hi; ++m3) {
        if (m3 == m1) {
          visit(r, fb + m3, caa, 0, true);
          continue;
        }
        const int m4 = M - m3;
        const int q3 = P[m3] - (m3 > m1) - (m3 > m2), c3 = n[m3] - (m3 == m1) - (m3 == m2);
        const int q4 = P[m4] - (m4 > m1) - (m4 > m2), c4 = n[m4] - (m4 == m1) - (m4 == m2);
        const int cad = (m3 == m4) ? (c4 + 1) * (c4 + 2) : (c4 + 1) * (c3 + 1);
        visit(boson_target(f, s, r, insert_one(insert_one(an, q3), q4)), fb + m3, caa, cad, false);
      }
    }
  }
}

// off-diagonal elements per row (the stored form keeps the diagonal moves as one value per row)
__global__ void boson_row_counts_kernel(FqheDevice f, int* counts) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int L = f.boson_lz_max;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    uint8_t n[64];
    int pos = 0;
    for (int m = 0; m <= L; ++m) {
      const int c = __ffsll(~(s >> pos)) - 1;
      n[m] = (uint8_t)c;
      pos += c + 1;
    }
    int cnt = 0;
    for (int m1 = 0; m1 <= L; ++m1) {
      if (n[m1] == 0) continue;
      for (int m2 = 0; m2 <= m1; ++m2) {
        if (n[m2] == 0 || (m2 == m1 && n[m1] < 2)) continue;
        const int M = m1 + m2;
        cnt += ((M < L) ? M : L) - ((M + 1) >> 1);  // the m3 range less its diagonal move
      }
    }
    counts[r] = cnt;
  }
}

// element payload: factor index | caa << 16 | cad << 24; padding: the row itself times the zero
// factor nbr_factors
__global__ void boson_ell_fill_kernel(FqheDevice f, const long long* slice_ptr, const int* slice_len, int* cols,
                                      uint32_t* coef) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const long long base = slice_ptr[r >> 5];
    const int len = slice_len[r >> 5];
    const int lane = (int)(r & 31);
    int j = 0;
    auto at = [&](int jj) {
      return base + (long long)(jj / kEllGroup) * (32 * kEllGroup) + lane * kEllGroup + (jj % kEllGroup);
    };
    boson_visit_row(f, r, __ldg(f.words + r), [&](long long idx, int fidx, int caa, int cad, bool diag) {
      if (diag) return;
      const long long p = at(j++);
      cols[p] = (int)idx;
      coef[p] = (uint32_t)fidx | ((uint32_t)caa << 16) | ((uint32_t)cad << 24);
    });
    for (; j < len; ++j) {
      const long long p = at(j);
      cols[p] = (int)r;
      coef[p] = (uint32_t)f.nbr_factors;
    }
  }
}

// diagonal of every row: sum over the pairs of factor(m1, m2, m1) n_m2 (n_m1 - [m1 = m2])
__global__ void boson_diag_kernel(FqheDevice f, const double* factors, double* diag64, float* diag32) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    double d = 0.0;
    boson_visit_row(f, r, __ldg(f.words + r), [&](long long, int fidx, int caa, int, bool diag) {
      if (diag) d += factors[fidx] * (double)caa;
    });
    diag64[r] = d;
    diag32[r] = (float)d;
  }
}

// bins[f] = sum over rows r and moves (r -> t) of factor f of u[r] * coefficient * v[t].  SHARED:
// per-block partial rows of a [blocks][factors] array accumulated in shared memory, summed in block
// order afterwards; else atomics straight into the global bins (the widest bosonic tables outgrow
// shared memory)
constexpr int kBosonBinThreads = 256;
template <bool SHARED>
__global__ void __launch_bounds__(kBosonBinThreads) boson_bins_kernel(FqheDevice f, const double* u, const double* v,
                                                                      double* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* bins = SHARED ? reinterpret_cast<double*>(smem) : out;
  if (SHARED) {
    for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) bins[i] = 0.0;
    __syncthreads();
  }
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const double ur = u[r];
    if (ur == 0.0) continue;
    boson_visit_row(f, r, __ldg(f.words + r), [&](long long idx, int fidx, int caa, int cad, bool diag) {
      const double c = diag ? (double)caa : sqrt((double)caa) * sqrt((double)cad);
      atomicAdd(bins + fidx, c * ur * __ldg(v + idx));
    });
  }
  if (SHARED) {
    __syncthreads();
    double* row = out + (size_t)blockIdx.x * f.nbr_factors;
    for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) row[i] = bins[i];
  }
}

__global__ void boson_sum_partial_bins(const double* partial, int nblocks, int nbins, double* bins) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbins) return;
  double acc = 0.0;
  for (int b = 0; b < nblocks; ++b) acc += partial[(size_t)b * nbins + i];
  bins[i] = acc;
}

unsigned boson_grid(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace

int launch_boson_row_counts(const FqheDevice& f, int* counts, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  boson_row_counts_kernel<<<boson_grid(f.dim), 256, 0, s>>>(f, counts);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_boson_ell_fill(const FqheDevice& f, const long long* slice_ptr, const int* slice_len, int* cols,
                          uint32_t* coef, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  boson_ell_fill_kernel<<<boson_grid(f.dim), 256, 0, s>>>(f, slice_ptr, slice_len, cols, coef);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_boson_diag(const FqheDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s) {
  if (f.dim <= 0) return DH_OK;
  boson_diag_kernel<<<boson_grid(f.dim), 256, 0, s>>>(f, factors64, diag64, diag32);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_boson_bins(const FqheDevice& f, const double* u, const double* v, double* partial_bins, int nblocks,
                      double* bins, cudaStream_t s) {
  const int smem = f.nbr_factors * (int)sizeof(double);
  const bool shared = smem <= 200 * 1024;
  if (!shared) DH_CUDA(cudaMemsetAsync(bins, 0, (size_t)f.nbr_factors * sizeof(double), s));
  if (f.dim > 0) {
    if (shared) {
      if (smem > 48 * 1024)
        DH_CUDA(cudaFuncSetAttribute(boson_bins_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      boson_bins_kernel<true><<<nblocks, kBosonBinThreads, smem, s>>>(f, u, v, partial_bins);
    } else {
      boson_bins_kernel<false><<<nblocks, kBosonBinThreads, 0, s>>>(f, u, v, bins);
    }
    DH_CUDA(cudaGetLastError());
  }
  if (shared) {
    boson_sum_partial_bins<<<(f.nbr_factors + 255) / 256, 256, 0, s>>>(partial_bins, f.dim > 0 ? nblocks : 0,
                                                                       f.nbr_factors, bins);
    DH_CUDA(cudaGetLastError());
  }
  return DH_OK;
}

int launch_boson_count(const FqheDevice& f, unsigned long long* total, cudaStream_t s) {
  DH_CUDA(cudaMemsetAsync(total, 0, 2 * sizeof(unsigned long long), s));
  if (f.dim == 0) return DH_OK;
  long long blocks = (f.dim + kBosonThreads - 1) / kBosonThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  boson_count_kernel<<<(unsigned)blocks, kBosonThreads, 0, s>>>(f, total);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_boson_matvec(const FqheDevice& f, const MatvecArgs& a, int precision, cudaStream_t s) {
  DH_CHECK(f.boson_lz_max >= 0 && f.boson_lz_max < 64 && f.lz_max <= 63, DH_ERR_ARGUMENT, "bad boson space");
  if (f.dim == 0) return DH_OK;
  return precision == DH_PRECISION_FP32 ? launch_k<float>(f, a, s) : launch_k<double>(f, a, s);
}

}  // namespace dh

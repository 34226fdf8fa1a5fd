// Pull-form H.x for the periodic J1-J2 spin-1/2 chain on a plain Spin1_2Chain basis (sm_100a).
//
// Basis order (Spin1_2Chain::GenerateStates, Spin1_2Chain.cc:331-394): site 0 is the most
// significant position and spin up (bit set) sorts first, i.e. descending order of the
// bit-reversed word.  With p = L - 1 - site and the up spins sorted by ascending p (k = 1..n),
//     index(w) = D - 1 - sum_k C(p_k, k).
// A flip on bond (j, j+1) moves one up spin by one site without passing another, so the target
// index is r +- C(L-2-j, k-1), k-1 = number of up spins at sites > j+1.  A (j, j+2) flip passes at
// most the middle spin; both cases are closed forms in two binomials.  Only the three bonds that
// wrap around the chain need the full rank (n binomials).  No lookup table, no search.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"
#include "dh_spin_tables.cuh"

namespace dh {
namespace {

constexpr int kSpinThreads = 256;

template <typename TG>
__device__ __forceinline__ long long spin_full_index(uint32_t t, int L, long long D, const int* binom) {
  long long rank = 0;
  int k = 1;
  while (t) {
    const int site = 31 - __clz(t);
    t &= ~(1u << site);
    rank += binom[(L - 1 - site) * 33 + k];
    ++k;
  }
  return D - 1 - rank;
}

// the K values of target row idx: one vector load when the block is row-interleaved (IL)
template <typename TG, int K, bool IL>
__device__ __forceinline__ void spin_gather(const TG* x, const MatvecArgs& a, long long idx, TG (&v)[K]) {
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
    const TG* p = x + idx * (IL ? K : a.ld);
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = __ldg(p + q * (IL ? 1 : a.vstride));
  }
}

template <typename TG, int K, bool IL>
__device__ __forceinline__ void spin_add(TG (&acc)[K], TG h, const TG* x, const MatvecArgs& a, long long idx) {
  TG v[K];
  spin_gather<TG, K, IL>(x, a, idx, v);
#pragma unroll
  for (int q = 0; q < K; ++q) acc[q] += h * v[q];
}

// IL: x, y (and xdiag) are row-interleaved [row][K] blocks (ld = K, vstride = 1).  Rows and
// indices are 32-bit (a 32-site chain has at most C(32, 16) < 2^31 states); lanes own consecutive
// rows, which share their low sites and so mostly the same index step for a given bond: the
// gathers of a warp coalesce.  Flips are taken two at a time so that two gathers are in flight.
template <typename TG, int K, bool IL>
__global__ void __launch_bounds__(kSpinThreads) spin_j1j2_kernel(SpinDevice sp, MatvecArgs a) {
  __shared__ SpinTables tb;
  const int L = sp.length;
  build_spin_tables(tb, L);
  const int D = (int)sp.dim;
  const uint32_t maskL = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const TG hj1 = (TG)(0.5 * sp.j1), hj2 = (TG)(0.5 * sp.j2);
  const TG* x = static_cast<const TG*>(a.x);
  const int stride = gridDim.x * blockDim.x;
  const int r_end = a.out_last > 0 ? (int)a.out_last : D;
  for (int r = (int)a.out_first + blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    const uint32_t w = __ldg(sp.words + r);
    const uint32_t rot1 = ((w >> 1) | (w << (L - 1))) & maskL;  // bit j = spin j+1 (mod L)
    const uint32_t rot2 = ((w >> 2) | (w << (L - 2))) & maskL;  // bit j = spin j+2 (mod L)
    const uint32_t d1 = w ^ rot1, d2 = w ^ rot2;
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    // J1 bonds (j, j+1), j = 0 .. L-2: the up spin moves one site; up at j moves the index forward
    uint32_t f = d1 & (maskL >> 1);
    while (f) {
      const int ja = __ffs(f) - 1;
      f &= f - 1u;
      const bool two = f != 0u;
      const int jb = two ? __ffs(f) - 1 : ja;
      f &= f - 1u;
      const int da = tb.j1[(ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 2))];
      const int db = tb.j1[(jb << 5) | __popc(__funnelshift_rc(w, 0u, jb + 2))];
      const int ia = ((w >> ja) & 1u) ? r + da : r - da;
      const int ib = ((w >> jb) & 1u) ? r + db : r - db;
      TG xa[K], xb[K];
      spin_gather<TG, K, IL>(x, a, ia, xa);
      spin_gather<TG, K, IL>(x, a, ib, xb);
      const TG hb = two ? hj1 : TG(0);
#pragma unroll
      for (int q = 0; q < K; ++q) acc[q] += hj1 * xa[q] + hb * xb[q];
    }
    // J2 bonds (j, j+2), j = 0 .. L-3
    f = d2 & (maskL >> 2);
    while (f) {
      const int ja = __ffs(f) - 1;
      f &= f - 1u;
      const bool two = f != 0u;
      const int jb = two ? __ffs(f) - 1 : ja;
      f &= f - 1u;
      const int da = tb.j2[(((w >> (ja + 1)) & 1u) << 10) | (ja << 5) | __popc(__funnelshift_rc(w, 0u, ja + 3))];
      const int db = tb.j2[(((w >> (jb + 1)) & 1u) << 10) | (jb << 5) | __popc(__funnelshift_rc(w, 0u, jb + 3))];
      const int ia = ((w >> ja) & 1u) ? r + da : r - da;
      const int ib = ((w >> jb) & 1u) ? r + db : r - db;
      TG xa[K], xb[K];
      spin_gather<TG, K, IL>(x, a, ia, xa);
      spin_gather<TG, K, IL>(x, a, ib, xb);
      const TG hb = two ? hj2 : TG(0);
#pragma unroll
      for (int q = 0; q < K; ++q) acc[q] += hj2 * xa[q] + hb * xb[q];
    }
    // bonds that wrap: J1 (L-1, 0), J2 (L-2, 0) and (L-1, 1): the moved spin passes the others
    if ((d1 >> (L - 1)) & 1u)
      spin_add<TG, K, IL>(acc, hj1, x, a, spin_rank_index(tb, w ^ (1u | (1u << (L - 1))), L, D));
    if ((d2 >> (L - 2)) & 1u)
      spin_add<TG, K, IL>(acc, hj2, x, a, spin_rank_index(tb, w ^ (1u | (1u << (L - 2))), L, D));
    if ((d2 >> (L - 1)) & 1u)
      spin_add<TG, K, IL>(acc, hj2, x, a, spin_rank_index(tb, w ^ (2u | (1u << (L - 1))), L, D));
    // diagonal: sum over bonds of J Sz_i Sz_j = J/4 (L - 2 * #antiparallel bonds), plus the shift
    const double diag = 0.25 * sp.j1 * (double)(L - 2 * __popc(d1)) + 0.25 * sp.j2 * (double)(L - 2 * __popc(d2)) +
                        a.shift;
    const bool on_diag = (r >= a.row_first && r < a.row_last);
    double* y = static_cast<double*>(a.y);
    double out[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double v = (double)acc[q];
      if (on_diag) {
        const long long xo = IL ? (long long)r * K + q : r * a.ld + q * a.vstride;
        const double xd = a.xdiag ? a.xdiag[xo] : (double)x[xo];
        v += diag * xd;
      }
      out[q] = v;
    }
    if constexpr (IL && K % 2 == 0) {
      double2* yp = reinterpret_cast<double2*>(y + (long long)r * K);
#pragma unroll
      for (int q = 0; q < K; q += 2) {
        double2 o = make_double2(out[q], out[q + 1]);
        if (a.accumulate) {
          const double2 old = yp[q / 2];
          o.x += old.x;
          o.y += old.y;
        }
        yp[q / 2] = o;
      }
    } else {
#pragma unroll
      for (int q = 0; q < K; ++q) {
        double* yp = y + (IL ? (long long)r * K + q : r * a.ld_y + q * a.vstride_y);
        *yp = a.accumulate ? (*yp + out[q]) : out[q];
      }
    }
  }
}

// Range-restricted variant (LowLevelAddMultiply with a column window): same enumeration, targets
// outside [col_first, col_last) are skipped.  Kept separate so the full product has no branch.
template <typename TG>
__global__ void __launch_bounds__(kSpinThreads) spin_j1j2_range_kernel(SpinDevice sp, MatvecArgs a) {
  __shared__ int binom[33 * 33];
  for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) {
    const int n = i / 33, k = i % 33;
    long long c = 1;
    if (k > n) c = 0;
    else
      for (int q = 1; q <= k; ++q) c = c * (n - k + q) / q;
    binom[i] = (int)c;
  }
  __syncthreads();
  const int L = sp.length;
  const long long D = sp.dim;
  const TG* x = static_cast<const TG*>(a.x);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long r_end = a.out_last > 0 ? a.out_last : D;
  for (long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    const uint32_t w = sp.words[r];
    for (int q = 0; q < a.nbr_vectors; ++q) {
      double acc = 0.0, diag = a.shift;
      for (int j = 0; j < L; ++j) {
        const int nb[2] = {(j + 1) % L, (j + 2) % L};
        const double jj[2] = {sp.j1, sp.j2};
        for (int b = 0; b < 2; ++b) {
          const int k = nb[b];
          const uint32_t bj = (w >> j) & 1u, bk = (w >> k) & 1u;
          diag += jj[b] * ((bj == bk) ? 0.25 : -0.25);
          if (bj != bk) {
            const long long idx = spin_full_index<TG>(w ^ ((1u << j) | (1u << k)), L, D, binom);
            if (idx >= a.col_first && idx < a.col_last) acc += 0.5 * jj[b] * (double)x[idx * a.ld + q * a.vstride];
          }
        }
      }
      double v = (double)(TG)acc;
      if (r >= a.row_first && r < a.row_last) {
        const double xd = a.xdiag ? a.xdiag[r * a.ld + q * a.vstride] : (double)x[r * a.ld + q * a.vstride];
        v += diag * xd;
      }
      double* yp = static_cast<double*>(a.y) + r * a.ld_y + q * a.vstride_y;
      *yp = a.accumulate ? (*yp + v) : v;
    }
  }
}

// word of basis index i: sites 0..L-1, spin up first while ups remain (C(L-1-site, ups-1) states)
__global__ void spin_unrank_kernel(int L, int nbr_up, long long dim, uint32_t* words) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= dim) return;
  long long rest = i;
  int ups = nbr_up;
  uint32_t w = 0;
  for (int site = 0; site < L && ups > 0; ++site) {
    // C(L - 1 - site, ups - 1)
    const int n = L - 1 - site, k = ups - 1;
    long long c = 1;
    if (k > n) c = 0;
    else
      for (int q = 1; q <= k; ++q) c = c * (n - k + q) / q;
    if (rest < c) {
      w |= 1u << site;
      --ups;
    } else {
      rest -= c;
    }
  }
  words[i] = w;
}

__global__ void spin_find_kernel(SpinDevice sp, const uint64_t* words, long long n, long long* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int L = sp.length;
  const uint64_t maskL = (L == 32) ? 0xffffffffull : ((1ull << L) - 1ull);
  // the reference keeps bits L..31 set (Spin1_2Chain.cc:137); only the chain bits matter
  const uint64_t w = words[i];
  const uint32_t t = (uint32_t)(w & maskL);
  if (__popc(t) != sp.nbr_up) {
    out[i] = -1;
    return;
  }
  long long rank = 0;
  int k = 1;
  uint32_t u = t;
  while (u) {
    const int site = 31 - __clz(u);
    u &= ~(1u << site);
    const int nn = L - 1 - site;
    long long c = 1;
    if (k > nn) c = 0;
    else
      for (int q = 1; q <= k; ++q) c = c * (nn - k + q) / q;
    rank += c;
    ++k;
  }
  out[i] = sp.dim - 1 - rank;
}

template <typename TG>
int launch_spin_typed(const SpinDevice& sp, MatvecArgs a, cudaStream_t s) {
  int dev = 0, sms = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  long long need = ((a.out_last > 0 ? a.out_last : sp.dim) - a.out_first + kSpinThreads - 1) / kSpinThreads;
  const bool range = (a.col_first > 0 || a.col_last < sp.dim);
  if (range) {
    long long grid = need < (long long)sms * 8 ? need : (long long)sms * 8;
    spin_j1j2_range_kernel<TG><<<(unsigned)grid, kSpinThreads, 0, s>>>(sp, a);
    DH_CUDA(cudaGetLastError());
    return DH_OK;
  }
  const int nv = a.nbr_vectors;
  const bool one = nv == 1 && a.ld == 1 && a.ld_y == 1;
  if (one || ((nv == 2 || nv == 4) && a.ld == nv && a.vstride == 1 && a.ld_y == nv && a.vstride_y == 1 &&
              il_rows_aligned(a, nv, sizeof(TG)))) {
    // row-interleaved block (or one contiguous vector): one launch with the row strides known at
    // compile time, vector gathers and stores
    auto kern = one ? spin_j1j2_kernel<TG, 1, true>
                    : ((nv == 4) ? spin_j1j2_kernel<TG, 4, true> : spin_j1j2_kernel<TG, 2, true>);
    int per_sm = 0;
    DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSpinThreads, 0));
    long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, kSpinThreads, 0, s>>>(sp, a);
    DH_CUDA(cudaGetLastError());
    return DH_OK;
  }
  int left = a.nbr_vectors, done = 0;
  while (left > 0) {
    int k = left >= 2 ? 2 : 1;
    MatvecArgs b = a;
    b.x = static_cast<const TG*>(a.x) + (size_t)done * a.vstride;
    b.y = static_cast<double*>(a.y) + (size_t)done * a.vstride_y;
    b.xdiag = a.xdiag ? a.xdiag + (size_t)done * a.vstride : nullptr;
    b.nbr_vectors = k;
    int per_sm = 0;
    if (k == 2)
      DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spin_j1j2_kernel<TG, 2, false>, kSpinThreads, 0));
    else
      DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spin_j1j2_kernel<TG, 1, false>, kSpinThreads, 0));
    long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
    if (need < grid) grid = need;
    if (grid < 1) grid = 1;
    if (k == 2)
      spin_j1j2_kernel<TG, 2, false><<<(unsigned)grid, kSpinThreads, 0, s>>>(sp, b);
    else
      spin_j1j2_kernel<TG, 1, false><<<(unsigned)grid, kSpinThreads, 0, s>>>(sp, b);
    DH_CUDA(cudaGetLastError());
    left -= k;
    done += k;
  }
  return DH_OK;
}

}  // namespace

int launch_spin_unrank(int length, int nbr_up, long long dim, uint32_t* words, cudaStream_t s) {
  if (dim <= 0) return DH_OK;
  spin_unrank_kernel<<<(unsigned)((dim + 255) / 256), 256, 0, s>>>(length, nbr_up, dim, words);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_spin_matvec(const SpinDevice& sp, const MatvecArgs& a, int precision, cudaStream_t s) {
  if (sp.dim <= 0) return DH_OK;
  if (precision == DH_PRECISION_FP32) return launch_spin_typed<float>(sp, a, s);
  return launch_spin_typed<double>(sp, a, s);
}

int launch_spin_find(const SpinDevice& sp, const uint64_t* words, long long n, long long* out, cudaStream_t s) {
  if (n <= 0) return DH_OK;
  spin_find_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(sp, words, n, out);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

}  // namespace dh

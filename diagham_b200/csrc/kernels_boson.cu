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

template <typename TG, int K, bool RANGE, bool IL>
__global__ void __launch_bounds__(kBosonThreads) boson_matvec_kernel(FqheDevice f, MatvecArgs a, int factor_smem) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  int* spair = reinterpret_cast<int*>(smem + factor_smem);
  const TG* gfac = static_cast<const TG*>(f.factors);
  for (int i = threadIdx.x; i < f.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
  for (int i = threadIdx.x; i < f.nbr_pairs; i += blockDim.x) spair[i] = f.pair_offset[i];
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
  const TG* fp = sfac;
  // row r's word, the halves of its rank, occupations, group starts and pair masks
  auto open_row = [&]() {
    s = __ldg(f.words + r);
    sh = s >> LB;
    sl = s & lmask;
    ho_row = __ldg(f.high_offset + sh);
    lr_row = (int)(r - ho_row);
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
            const double xd = a.xdiag ? a.xdiag[r * a.ld + j * a.vstride] : (double)x[r * a.ld + j * a.vstride];
            v += a.shift * xd;
          }
          double* yp = y + r * a.ld_y + j * a.vstride_y;
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
      saa = coef_sqrt<TG>(caa);
      an = delete_bit(delete_bit(s, P[m1]), P[m2]);
      const int M = m1 + m2;
      const int m3lo = (M + 1) >> 1;
      m3hi = (M < L) ? M : L;
      fp = sfac + (spair[m1 * (m1 + 1) / 2 + m2] - m3lo);
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
      const uint64_t th = t >> LB, tl = t & lmask;
      int hoi = ho_row, lri = lr_row;
      if (th != sh) hoi = __ldg(f.high_offset + th);
      if (tl != sl) lri = (int)__ldg(f.low_rank + tl);
      const long long idx = (long long)hoi + (long long)lri;
      if (!RANGE || (idx >= a.col_first && idx < a.col_last)) {
        const TG c = fp[m3] * saa * coef_sqrt<TG>(cad);
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

template <typename TG, int K>
int launch_typed(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  const int factor_smem = (int)((f.nbr_factors * sizeof(TG) + 15) & ~(size_t)15);
  const size_t smem = (size_t)factor_smem + (size_t)f.nbr_pairs * sizeof(int);
  const bool range = a.col_first > 0 || a.col_last < f.dim;
  const bool il = (K > 1) && a.ld == K && a.vstride == 1;
  auto kernel = range ? (il ? boson_matvec_kernel<TG, K, true, true> : boson_matvec_kernel<TG, K, true, false>)
                      : (il ? boson_matvec_kernel<TG, K, false, true> : boson_matvec_kernel<TG, K, false, false>);
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

}  // namespace

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

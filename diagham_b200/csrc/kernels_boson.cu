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
// first one of orbital m, or of its separator when empty) are decoded once.  For every pair
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

template <typename TG, int K, bool RANGE>
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
  for (long long r = a.out_first + (long long)blockIdx.x * blockDim.x + threadIdx.x; r < r_end; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    // occupations and group starts of the row
    uint8_t n[64], P[64];
    int pos = 0;
    for (int m = 0; m <= L; ++m) {
      const int c = __ffsll(~(s >> pos)) - 1;  // length of the run of ones starting at pos
      P[m] = (uint8_t)pos;
      n[m] = (uint8_t)c;
      pos += c + 1;
    }
    TG acc[K];
#pragma unroll
    for (int j = 0; j < K; ++j) acc[j] = TG(0);
    for (int m1 = 0; m1 <= L; ++m1) {
      const int n1 = n[m1];
      if (n1 == 0) continue;
      const int p1 = P[m1];
      const uint64_t s1 = delete_bit(s, p1);
      for (int m2 = 0; m2 <= m1; ++m2) {
        const int n2 = n[m2];
        if (n2 == 0 || (m2 == m1 && n1 < 2)) continue;
        const int caa = n2 * (n1 - (m1 == m2 ? 1 : 0));
        const uint64_t an = delete_bit(s1, P[m2]);
        const int M = m1 + m2;
        const int m3lo = (M + 1) >> 1;
        const int m3hi = (M < L) ? M : L;
        const TG* fp = sfac + (spair[m1 * (m1 + 1) / 2 + m2] - m3lo);
        for (int m3 = m3lo; m3 <= m3hi; ++m3) {
          const int m4 = M - m3;
          // occupations and group starts after the annihilations
          const int a3 = n[m3] - (m3 == m1) - (m3 == m2);
          const int a4 = n[m4] - (m4 == m1) - (m4 == m2);
          const int q3 = P[m3] - (m3 > m1) - (m3 > m2);
          const int q4 = P[m4] - (m4 > m1) - (m4 > m2);
          const int cad = (m3 == m4) ? (a4 + 1) * (a4 + 2) : (a4 + 1) * (a3 + 1);
          const uint64_t t = insert_one(insert_one(an, q3), q4);
          const long long idx = (long long)__ldg(f.high_offset + (t >> LB)) + (long long)__ldg(f.low_rank + (t & lmask));
          if (RANGE && (idx < a.col_first || idx >= a.col_last)) continue;
          const TG c = fp[m3] * coef_sqrt<TG>(caa) * coef_sqrt<TG>(cad);
          const TG* xp = x + idx * a.ld;
#pragma unroll
          for (int j = 0; j < K; ++j) acc[j] += c * __ldg(xp + j * a.vstride);
        }
      }
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
  }
}

template <typename TG, int K>
int launch_typed(const FqheDevice& f, const MatvecArgs& a, cudaStream_t s) {
  const int factor_smem = (int)((f.nbr_factors * sizeof(TG) + 15) & ~(size_t)15);
  const size_t smem = (size_t)factor_smem + (size_t)f.nbr_pairs * sizeof(int);
  const bool range = a.col_first > 0 || a.col_last < f.dim;
  auto kernel = range ? boson_matvec_kernel<TG, K, true> : boson_matvec_kernel<TG, K, false>;
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

}  // namespace

int launch_boson_matvec(const FqheDevice& f, const MatvecArgs& a, int precision, cudaStream_t s) {
  DH_CHECK(f.boson_lz_max >= 0 && f.boson_lz_max < 64 && f.lz_max <= 63, DH_ERR_ARGUMENT, "bad boson space");
  if (f.dim == 0) return DH_OK;
  return precision == DH_PRECISION_FP32 ? launch_k<float>(f, a, s) : launch_k<double>(f, a, s);
}

}  // namespace dh

// Step and rank tables of the plain Spin1_2Chain index (device code shared by the chain kernels and
// the momentum-sector kernels).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dh {

// Shared tables of the product kernel (every entry an int: C(32, 16) = 601,080,390 < 2^31).
//   j1[(j << 5) | kk]            J1 flip (j, j+1) index step: C(L-2-j, kk), kk = up spins at sites > j+1
//   j2[(mid << 10) | (j << 5) | kk]  J2 flip (j, j+2) step, kk = up spins at sites > j+2, mid = spin j+1:
//                                  mid = 0: C(p-1, kk) + C(p-2, kk); mid = 1: 2 C(p-1, kk+1) - C(p-2, kk+1), p = L-1-j
//   nib[(n * 33 + c) * 16 + v]  rank contribution of nibble n (positions p = 4n..4n+3 of the
//                                  bit-reversed word) holding v, with c up spins at lower positions:
//                                  sum over bits i of v (ascending) of C(4n+i, c + (bits of v below i) + 1)
struct SpinTables {
  int binom[33 * 33];
  int j1[32 * 32];
  int j2[2 * 32 * 32];
  int nib[8 * 33 * 16];
};

__device__ inline void build_spin_tables(SpinTables& t, int L) {
  for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) {
    const int n = i / 33, k = i % 33;
    long long c = 1;
    if (k > n) c = 0;
    else
      for (int q = 1; q <= k; ++q) c = c * (n - k + q) / q;
    t.binom[i] = (int)c;
  }
  __syncthreads();
  auto C = [&](int n, int k) { return (n < 0 || k < 0 || k > n) ? 0 : t.binom[n * 33 + k]; };
  for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) {
    const int j = i >> 5, kk = i & 31;
    t.j1[i] = (j <= L - 2) ? C(L - 2 - j, kk) : 0;
    const int p = L - 1 - j;
    t.j2[i] = (j <= L - 3) ? C(p - 1, kk) + C(p - 2, kk) : 0;
    t.j2[1024 + i] = (j <= L - 3) ? 2 * C(p - 1, kk + 1) - C(p - 2, kk + 1) : 0;
  }
  for (int i = threadIdx.x; i < 8 * 33 * 16; i += blockDim.x) {
    const int v = i & 15, c = (i >> 4) % 33, n = (i >> 4) / 33;
    int sum = 0, below = 0;
    for (int b = 0; b < 4; ++b)
      if ((v >> b) & 1) {
        sum += C(4 * n + b, c + below + 1);
        ++below;
      }
    t.nib[i] = sum;
  }
  __syncthreads();
}

// index of word t (chain bits only): D - 1 - sum_k C(p_k, k) over the up spins at p = L-1-site in
// ascending order, summed nibble by nibble of the bit-reversed word
__device__ __forceinline__ int spin_rank_index(const SpinTables& tb, uint32_t t, int L, int D) {
  const uint32_t tr = __brev(t) >> (32 - L);
  int rank = 0, c = 0;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const uint32_t v = (tr >> (4 * n)) & 15u;
    rank += tb.nib[(n * 33 + c) * 16 + v];
    c += __popc(v);
  }
  return D - 1 - rank;
}


}  // namespace dh

// Stored-element ("fast multiplication") form of the two-body FQHE product on sm_100a.
//
// The reference can precompute, for every row, the list of (target index, interaction-factor
// index) of its matrix elements and multiply from those lists afterwards
// (AbstractQHEOnSphereHamiltonian::EnableFastMultiplication / FastMultiplicationMemory,
// AbstractQHEOnSphereHamiltonian.cc:3625,3814; QHEParticlePrecalculationOperation.cc:95).  Here the
// lists are kept in device memory as sliced ELL: rows are grouped in slices of 32 consecutive rows
// (one warp), every row of a slice is padded to the slice's longest row rounded up to a multiple of
// kEllPad, and the slice is stored in groups of kEllGroup elements per row: element j of lane l
// sits at slice_ptr + (j / G) * 32 G + l G + j % G, so one 16-byte load gives a lane G targets and
// a warp reads 512 contiguous bytes per load.  Each element is an int32 target and a uint16 factor
// index with the fermionic sign in bit 15; the structure does not depend on the pseudopotentials.
// Diagonal moves are summed per row into a separate diagonal array, recomputed when the
// pseudopotentials change.  Bosonic elements (BosonOnSphereShort) carry their occupation factors: a
// uint32 of factor index | caa << 16 | cad << 24 for the element factor * sqrt(caa) * sqrt(cad), the
// square roots read from a 256-entry table in shared memory.  Fermions of the count-table engine
// (FermionOnSphereLong, FermionOnSphere beyond 40 orbitals) have factor tables too large for 15-bit
// indices and for shared memory: a uint32 of factor index | sign << 31, factors read through the
// cache.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "dh_internal.h"

namespace dh {
namespace {

constexpr int kFastThreads = 256;

__device__ __forceinline__ long long ell_pos(long long slice_base, int lane, int j) {
  return slice_base + (long long)(j / kEllGroup) * (32 * kEllGroup) + lane * kEllGroup + (j % kEllGroup);
}

__device__ __forceinline__ uint64_t bits_between(int lo, int hi) {
  // bits strictly between lo and hi (lo < hi <= 63)
  return ((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull);
}

__device__ __forceinline__ uint64_t mirror_of(uint64_t e, int M) {
  // bit p of the result = bit (M - p) of e (0 when M - p is outside 0..63)
  const uint64_t r = __brevll(e);
  return (M <= 63) ? (r >> (63 - M)) : (r << (M - 63));
}

// Visits the off-diagonal elements of row word s (moves whose two created orbitals are both empty
// in s): pairs m1 > m2 occupied, descending, then m3 ascending over E & mirror_M(E) above M/2.
// visit(target, factor index, negative) is called for each; rank-table target indices.
template <typename Visit>
__device__ __forceinline__ void visit_row(const FqheDevice& f, uint64_t s, Visit&& visit) {
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  const uint64_t E = ~s & full;
  const uint64_t lmask = (1ull << f.low_bits) - 1ull;
  uint64_t rem1 = s;
  while (rem1) {
    const int m1 = 63 - __clzll(rem1);
    rem1 &= ~(1ull << m1);
    uint64_t rem2 = rem1;
    while (rem2) {
      const int m2 = 63 - __clzll(rem2);
      rem2 &= ~(1ull << m2);
      const int M = m1 + m2;
      uint64_t valid = E & mirror_of(E, M) & (~0ull << (M / 2 + 1));
      if (!valid) continue;
      const uint64_t an = s & ~((1ull << m1) | (1ull << m2));
      const int paa = 1 + __popcll(s & bits_between(m2, m1));
      const int fbase = __ldg(f.pair_offset + (m1 * (m1 - 1) / 2 + m2)) - (M / 2 + 1);
      while (valid) {
        const int m3 = __ffsll(valid) - 1;
        valid &= valid - 1ull;
        const int m4 = M - m3;
        const uint64_t t = an | (1ull << m3) | (1ull << m4);
        const int idx = __ldg(f.high_offset + (t >> f.low_bits)) + (int)__ldg(f.low_rank + (t & lmask));
        const bool neg = (paa + __popcll(an & bits_between(m4, m3))) & 1;
        visit(idx, fbase + m3, neg);
      }
    }
  }
}

// row_offset: the space's rows are rows row_offset .. row_offset + dim - 1 of a larger structure (the
// concatenated sectors of the batched solver), their targets shifted by it
__global__ void row_counts_kernel(FqheDevice f, int* counts, long long row_offset) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const uint64_t full = (f.lz_max >= 63) ? ~0ull : ((1ull << (f.lz_max + 1)) - 1ull);
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    const uint64_t E = ~s & full;
    int n = 0;
    uint64_t rem1 = s;
    while (rem1) {
      const int m1 = 63 - __clzll(rem1);
      rem1 &= ~(1ull << m1);
      uint64_t rem2 = rem1;
      while (rem2) {
        const int m2 = 63 - __clzll(rem2);
        rem2 &= ~(1ull << m2);
        const int M = m1 + m2;
        n += __popcll(E & mirror_of(E, M) & (~0ull << (M / 2 + 1)));
      }
    }
    counts[row_offset + r] = n;
  }
}

__global__ void ell_fill_kernel(FqheDevice f, const long long* slice_ptr, const int* slice_len, int* cols,
                                uint16_t* coef, long long row_offset) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const long long g = row_offset + r;
    const long long sl = g >> 5;
    const long long base = slice_ptr[sl];
    const int len = slice_len[sl];
    const int lane = (int)(g & 31);
    int j = 0;
    visit_row(f, __ldg(f.words + r), [&](int idx, int fidx, bool neg) {
      const long long p = ell_pos(base, lane, j);
      cols[p] = (int)(row_offset + idx);
      coef[p] = (uint16_t)(fidx | (neg ? 0x8000 : 0));
      ++j;
    });
    for (; j < len; ++j) {  // padding: the row itself times a zero factor
      const long long p = ell_pos(base, lane, j);
      cols[p] = (int)g;
      coef[p] = (uint16_t)f.nbr_factors;
    }
  }
}

// diagonal of every row: the (m3, m4) = (m1, m2) moves have sign -1, so d = -sum factor(m1, m2, m1)
__global__ void diag_kernel(FqheDevice f, const double* factors, double* diag64, float* diag32, long long row_offset) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < f.dim; r += stride) {
    const uint64_t s = __ldg(f.words + r);
    double d = 0.0;
    uint64_t rem1 = s;
    while (rem1) {
      const int m1 = 63 - __clzll(rem1);
      rem1 &= ~(1ull << m1);
      uint64_t rem2 = rem1;
      while (rem2) {
        const int m2 = 63 - __clzll(rem2);
        rem2 &= ~(1ull << m2);
        const int M = m1 + m2;
        d -= factors[__ldg(f.pair_offset + (m1 * (m1 - 1) / 2 + m2)) - (M / 2 + 1) + m1];
      }
    }
    diag64[row_offset + r] = d;
    diag32[row_offset + r] = (float)d;
  }
}

// sector of concatenated row r (row_offset ascending, nbr_sectors + 1 entries)
__device__ __forceinline__ int ell_sector_of(const long long* row_offset, int nbr_sectors, long long r) {
  int lo = 0, hi = nbr_sectors - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(row_offset + mid) <= r) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename TG, int K, bool IL, bool W256 = false>
__device__ __forceinline__ void gather(const TG* x, const MatvecArgs& a, long long idx, TG (&v)[K]) {
  if constexpr (W256 && IL && sizeof(TG) == 8 && K == 4) {
    ldg_row32_no_l1(reinterpret_cast<const double*>(x + idx * 4), *reinterpret_cast<double(*)[4]>(&v));
  } else if constexpr (IL && sizeof(TG) == 4 && K == 4) {
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

// y = H x from the stored elements: lanes own the 32 rows of a slice.  The element stream is read
// CH elements ahead of the gathers (CH / 4 16-byte target loads and as many 8-byte index loads per
// lane per chunk, issued before the chunk in hand is gathered), so every warp keeps a chunk of the
// stream and a chunk of gathers in flight.  The stream, the diagonal and y go through L2 with
// streaming (evict-first) accesses so that the gathered x keeps the cache.
// W256: FP64 rows of 4 that are 32-byte aligned, gathered with one 256-bit load each
// PK (payload kind): 0 uint16 index | sign << 15, factors in shared memory; 1 (bosons) uint32 payloads
// (16-byte groups of 4, like the targets) with the occupation square roots; 2 uint32 index | sign << 31,
// factors read through the cache
// The element stream is read once: evict-first in L2 and not allocated in L1, which both keep the
// gathered x.
__device__ __forceinline__ uint64_t stream_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ int4 ld_stream(const int4* a, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint4 ld_stream(const uint4* a, uint64_t pol) {
  uint4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint2 ld_stream(const uint2* a, uint64_t pol) {
  uint2 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;"
               : "=r"(v.x), "=r"(v.y)
               : "l"(a), "l"(pol));
  return v;
}

template <typename TG>
__device__ __forceinline__ TG occupation_sqrt(int v);
template <>
__device__ __forceinline__ double occupation_sqrt<double>(int v) {
  return sqrt((double)v);
}
template <>
__device__ __forceinline__ float occupation_sqrt<float>(int v) {
  return sqrtf((float)v);
}

template <typename TG, int K, bool IL, bool W256, int CH, int PK>
__global__ void __launch_bounds__(kFastThreads) ell_product_kernel(EllDevice e, MatvecArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  TG* sfac = reinterpret_cast<TG*>(smem);
  TG* ssq = sfac + e.nbr_factors + 1;
  const TG* gfac = static_cast<const TG*>(e.factors);
  if (PK != 2) {
    for (int i = threadIdx.x; i < e.nbr_factors; i += blockDim.x) sfac[i] = gfac[i];
    if (threadIdx.x == 0) sfac[e.nbr_factors] = TG(0);
  }
  if (PK == 1)
    for (int i = threadIdx.x; i < 256; i += blockDim.x) ssq[i] = occupation_sqrt<TG>(i);
  __syncthreads();
  using KT = std::conditional_t<PK == 0, uint2, uint4>;
  const TG* x = static_cast<const TG*>(a.x);
  const TG* diag = static_cast<const TG*>(e.diag);
  const int lane = threadIdx.x & 31;
  const uint64_t pol = stream_policy();
  static_assert(kEllPad % CH == 0 && CH % kEllGroup == 0, "chunks must tile the padded rows");
  constexpr int NG = CH / kEllGroup;  // 16-byte target groups per chunk
  // a row range starts on a slice boundary (callers split at multiples of 32 rows)
  const long long r_end = a.out_last > 0 ? a.out_last : e.dim;
  const long long nslices = (r_end + 31) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long sl = (a.out_first >> 5) + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); sl < nslices;
       sl += nwarps) {
    const long long r = sl * 32 + lane;
    if (r >= r_end) continue;  // the last slice's lanes beyond the space hold no elements
    int len = e.slice_len[sl];
    // concatenated sectors: the rows of an inactive (converged) sector get y = 0 and no elements
    const bool live = !e.active || __ldg(e.active + ell_sector_of(e.sector_offset, e.nbr_sectors, r)) != 0;
    if (!__any_sync(__activemask(), live)) len = 0;
    const int4* cg = reinterpret_cast<const int4*>(e.cols + e.slice_ptr[sl]) + lane;
    const KT* kg;
    if constexpr (PK != 0) kg = reinterpret_cast<const uint4*>(e.coef32 + e.slice_ptr[sl]) + lane;
    else kg = reinterpret_cast<const uint2*>(e.coef + e.slice_ptr[sl]) + lane;
    TG acc[K];
#pragma unroll
    for (int q = 0; q < K; ++q) acc[q] = TG(0);
    int4 c[NG];
    KT k[NG];
    if (len > 0) {
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        c[g] = ld_stream(cg + g * 32, pol);
        k[g] = ld_stream(kg + g * 32, pol);
      }
    }
    for (int j = 0; j < len; j += CH) {
      int4 cn[NG];
      KT kn[NG];
      const bool more = j + CH < len;
      if (more) {
        const int gn = (j + CH) / kEllGroup;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
          cn[g] = ld_stream(cg + (gn + g) * 32, pol);
          kn[g] = ld_stream(kg + (gn + g) * 32, pol);
        }
      }
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const int cols[4] = {c[g].x, c[g].y, c[g].z, c[g].w};
        unsigned ks[4];
        if constexpr (PK != 0) {
          ks[0] = k[g].x; ks[1] = k[g].y; ks[2] = k[g].z; ks[3] = k[g].w;
        } else {
          ks[0] = k[g].x & 0xffffu; ks[1] = k[g].x >> 16; ks[2] = k[g].y & 0xffffu; ks[3] = k[g].y >> 16;
        }
        TG xv[4][K];
#pragma unroll
        for (int u = 0; u < 4; ++u) gather<TG, K, IL, W256>(x, a, cols[u], xv[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          TG fu;
          if constexpr (PK == 1) {
            fu = sfac[ks[u] & 0xffffu] * ssq[(ks[u] >> 16) & 0xffu] * ssq[ks[u] >> 24];
          } else if constexpr (PK == 2) {
            const unsigned fi = ks[u] & 0x7fffffffu;
            fu = (fi < (unsigned)e.nbr_factors) ? __ldg(gfac + fi) : TG(0);
            if (ks[u] & 0x80000000u) fu = -fu;
          } else {
            fu = sfac[ks[u] & 0x7fffu];
            if (ks[u] & 0x8000u) fu = -fu;
          }
#pragma unroll
          for (int q = 0; q < K; ++q) acc[q] += fu * xv[u][q];
        }
      }
      if (more) {
#pragma unroll
        for (int g = 0; g < NG; ++g) {
          c[g] = cn[g];
          k[g] = kn[g];
        }
      }
    }
    TG xr[K];
    gather<TG, K, IL, W256>(x, a, r, xr);
    const TG d = __ldcs(diag + r);
#pragma unroll
    for (int q = 0; q < K; ++q) acc[q] += d * xr[q];
    const bool on_diag = (r >= a.row_first && r < a.row_last);
    double* y = static_cast<double*>(a.y);
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double v = (double)acc[q];
      const long long xo = IL ? r * K + q : r * a.ld + q * a.vstride;
      if (on_diag && a.shift != 0.0) v += a.shift * (a.xdiag ? a.xdiag[xo] : (double)x[xo]);
      if (!live) v = 0.0;
      double* yp = y + (IL ? r * K + q : r * a.ld_y + q * a.vstride_y);
      __stcs(yp, a.accumulate ? (__ldcs(yp) + v) : v);
    }
  }
}

unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (unsigned)g;
}

template <typename TG, int K, bool IL, int PK>
int launch_ell_payload(const EllDevice& e, const MatvecArgs& a, cudaStream_t s) {
  const bool deep = e.chunk == 16;
  auto kern = deep ? ell_product_kernel<TG, K, IL, false, 16, PK> : ell_product_kernel<TG, K, IL, false, 8, PK>;
  if constexpr (IL && sizeof(TG) == 8 && K == 4)
    if ((reinterpret_cast<uintptr_t>(a.x) & 31) == 0)
      kern = deep ? ell_product_kernel<TG, K, IL, true, 16, PK> : ell_product_kernel<TG, K, IL, true, 8, PK>;
  const int smem = (PK == 2) ? 0 : (e.nbr_factors + 1 + (PK == 1 ? 256 : 0)) * (int)sizeof(TG);
  if (smem > 48 * 1024) DH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int dev = 0, sms = 0, per_sm = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFastThreads, smem));
  DH_CHECK(per_sm >= 1, DH_ERR_UNSUPPORTED, "stored-element product: %d bytes of shared memory do not fit", smem);
  const long long r_end = a.out_last > 0 ? a.out_last : e.dim;
  long long need = ((r_end + 31) / 32 * 32 - (a.out_first & ~31ll) + kFastThreads - 1) / kFastThreads;
  long long grid = (long long)sms * per_sm;
  if (need < grid) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, kFastThreads, smem, s>>>(e, a);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

template <typename TG, int K, bool IL>
int launch_ell_typed(const EllDevice& e, const MatvecArgs& a, cudaStream_t s) {
  if (e.payload == 1) return launch_ell_payload<TG, K, IL, 1>(e, a, s);
  if (e.payload == 2) return launch_ell_payload<TG, K, IL, 2>(e, a, s);
  return launch_ell_payload<TG, K, IL, 0>(e, a, s);
}

template <typename TG>
int launch_ell_k(const EllDevice& e, MatvecArgs a, cudaStream_t s) {
  const int nv = a.nbr_vectors;
  if ((nv == 2 || nv == 4) && a.ld == nv && a.vstride == 1 && a.ld_y == nv && a.vstride_y == 1 &&
      il_rows_aligned(a, nv, sizeof(TG)))
    return nv == 4 ? launch_ell_typed<TG, 4, true>(e, a, s) : launch_ell_typed<TG, 2, true>(e, a, s);
  // one contiguous vector of 128-bit-engine elements: row strides known at compile time (FP64 at
  // N = 6, 2S = 63: 0.409 ms against 0.479 ms; the 16-bit payloads gain nothing from it, and FP32 at
  // N = 11, 2S = 30 takes 0.448 ms against 0.443 ms, so they keep the strided form)
  if (nv == 1 && a.ld == 1 && a.ld_y == 1 && e.payload == 2) return launch_ell_typed<TG, 1, true>(e, a, s);
  // separate or strided vectors: groups of 4, 2 and 1 sharing one pass over the elements
  int left = nv, done = 0;
  while (left > 0) {
    const int k = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    MatvecArgs b = a;
    b.x = static_cast<const TG*>(a.x) + (size_t)done * a.vstride;
    b.y = static_cast<double*>(a.y) + (size_t)done * a.vstride_y;
    b.xdiag = a.xdiag ? a.xdiag + (size_t)done * a.vstride : nullptr;
    b.nbr_vectors = k;
    const int rc = (k == 4) ? launch_ell_typed<TG, 4, false>(e, b, s)
                            : (k == 2 ? launch_ell_typed<TG, 2, false>(e, b, s) : launch_ell_typed<TG, 1, false>(e, b, s));
    if (rc != DH_OK) return rc;
    left -= k;
    done += k;
  }
  return DH_OK;
}

}  // namespace

int launch_fqhe_row_counts(const FqheDevice& f, int* counts, cudaStream_t s, long long row_offset) {
  if (f.dim <= 0) return DH_OK;
  row_counts_kernel<<<grid_for(f.dim), 256, 0, s>>>(f, counts, row_offset);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_ell_fill(const FqheDevice& f, const long long* slice_ptr, const int* slice_len, int* cols,
                         uint16_t* coef, cudaStream_t s, long long row_offset) {
  if (f.dim <= 0) return DH_OK;
  ell_fill_kernel<<<grid_for(f.dim), 256, 0, s>>>(f, slice_ptr, slice_len, cols, coef, row_offset);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_fqhe_diag(const FqheDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s,
                     long long row_offset) {
  if (f.dim <= 0) return DH_OK;
  diag_kernel<<<grid_for(f.dim), 256, 0, s>>>(f, factors64, diag64, diag32, row_offset);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_ell_product(const EllDevice& e, const MatvecArgs& a, int precision, cudaStream_t s) {
  if (e.dim <= 0) return DH_OK;
  if (precision == DH_PRECISION_FP32) return launch_ell_k<float>(e, a, s);
  return launch_ell_k<double>(e, a, s);
}

}  // namespace dh

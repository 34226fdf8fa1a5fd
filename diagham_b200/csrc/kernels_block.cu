// Block (k-vector) kernels of the batched block Lanczos: every sector's block is a tall-skinny
// [rows][k] FP64 array inside one concatenated vector, and every kernel works sector by sector
// through a tile list (tile = up to kTileRows rows of one sector), so all sectors advance in one
// launch.  The small k x k matrices (Gram, recurrence and QR coefficients) are per sector.
// Reductions are two-level and deterministic: tile partials, then a per-sector sum in tile order.
// This is the device side of BasicBlockLanczosAlgorithm's MultipleRealScalarProductOperation /
// AddRealLinearCombinationOperation / ReorthogonalizeVectors (BasicBlockLanczosAlgorithm.cc:524-799).
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"

namespace dh {
namespace {

constexpr int kThreads = 256;

template <int W>
__device__ __forceinline__ void block_sum(double (&acc)[W], double (&out)[W]) {
  __shared__ double red[W][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][warp] = v;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) v += red[j][w];
    out[j] = v;
  }
}

// partial[tile][p * K + q] = sum over the tile's rows of a[r][p] * b[r][q]
template <int K>
__global__ void __launch_bounds__(kThreads) seg_gram_kernel(const double* a, const double* b, TileSetDevice t,
                                                            double* partial) {
  const int tile = blockIdx.x;
  const long long r0 = t.tile_begin[tile], r1 = t.tile_end[tile];
  double acc[K * K];
#pragma unroll
  for (int j = 0; j < K * K; ++j) acc[j] = 0.0;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double av[K], bv[K];
#pragma unroll
    for (int p = 0; p < K; ++p) av[p] = a[r * K + p];
#pragma unroll
    for (int q = 0; q < K; ++q) bv[q] = b[r * K + q];
#pragma unroll
    for (int p = 0; p < K; ++p)
#pragma unroll
      for (int q = 0; q < K; ++q) acc[p * K + q] += av[p] * bv[q];
  }
  double tot[K * K];
  block_sum<K * K>(acc, tot);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K * K; ++j) partial[(size_t)tile * K * K + j] = tot[j];
  }
}

// g[s][j] = sum over the tiles of sector s (in tile order) of partial[tile][j]
template <int K>
__global__ void seg_gram_reduce_kernel(const double* partial, TileSetDevice t, double* g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.nbr_sectors * K * K) return;
  const int s = i / (K * K), j = i % (K * K);
  double acc = 0.0;
  for (int tile = t.sector_tile_first[s]; tile < t.sector_tile_first[s + 1]; ++tile) acc += partial[(size_t)tile * K * K + j];
  g[i] = acc;
}

// w[r] -= v[r] * A_s + vp[r] * Bt_s   (A, Bt: [sector][K][K] row-major; vp / Bt may be null)
template <int K>
__global__ void __launch_bounds__(kThreads) seg_update_kernel(double* w, const double* v, const double* A,
                                                              const double* vp, const double* Bt, TileSetDevice t) {
  const int tile = blockIdx.x;
  const int s = t.tile_sector[tile];
  __shared__ double sA[K * K], sB[K * K];
  if (threadIdx.x < K * K) {
    sA[threadIdx.x] = A[(size_t)s * K * K + threadIdx.x];
    sB[threadIdx.x] = (vp && Bt) ? Bt[(size_t)s * K * K + threadIdx.x] : 0.0;
  }
  __syncthreads();
  const long long r0 = t.tile_begin[tile], r1 = t.tile_end[tile];
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double vr[K], pr[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      vr[j] = v[r * K + j];
      pr[j] = vp ? vp[r * K + j] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < K; ++c) {
      double acc = w[r * K + c];
#pragma unroll
      for (int j = 0; j < K; ++j) acc -= vr[j] * sA[j * K + c] + pr[j] * sB[j * K + c];
      w[r * K + c] = acc;
    }
  }
}

// w[r] = w[r] * M_s in place (M: [sector][K][K] row-major), optional FP32 copy of the result
template <int K>
__global__ void __launch_bounds__(kThreads) seg_rmul_kernel(double* w, const double* M, TileSetDevice t, float* w32) {
  const int tile = blockIdx.x;
  const int s = t.tile_sector[tile];
  __shared__ double sM[K * K];
  if (threadIdx.x < K * K) sM[threadIdx.x] = M[(size_t)s * K * K + threadIdx.x];
  __syncthreads();
  const long long r0 = t.tile_begin[tile], r1 = t.tile_end[tile];
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double in[K];
#pragma unroll
    for (int j = 0; j < K; ++j) in[j] = w[r * K + j];
#pragma unroll
    for (int c = 0; c < K; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < K; ++j) acc += in[j] * sM[j * K + c];
      w[r * K + c] = acc;
      if (w32) w32[r * K + c] = (float)acc;
    }
  }
}

// out[r] (+)= sum_b blocks[b][r] * C_s[b] (Ritz vectors: nb stored blocks of K vectors, C per sector
// [nb * K][K]); writes the K Ritz vectors of every sector
template <int K>
__global__ void __launch_bounds__(kThreads) seg_combine_blocks_kernel(const double* blocks, int nb, long long stride,
                                                                      const double* C, int cstride, TileSetDevice t,
                                                                      double* out) {
  const int tile = blockIdx.x;
  const int s = t.tile_sector[tile];
  const double* Cs = C + (size_t)s * cstride;
  const long long r0 = t.tile_begin[tile], r1 = t.tile_end[tile];
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    double acc[K];
#pragma unroll
    for (int c = 0; c < K; ++c) acc[c] = 0.0;
    for (int b = 0; b < nb; ++b) {
      const double* vb = blocks + (size_t)b * stride + r * K;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const double x = vb[j];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] += x * Cs[(b * K + j) * K + c];
      }
    }
#pragma unroll
    for (int c = 0; c < K; ++c) out[r * K + c] = acc[c];
  }
}

// ------------------------------------------------------------ per-sector k x k step math
// One thread per sector (k <= 4): the small matrices of a block step stay on the device, so a step
// needs no host round trip.  Layout of every matrix: [sector][k][k] row-major.

// A = (G + G^T) / 2 and scale[s] = |A|_F^2 + |Bt|_F^2 (the step's Gram V^T W and B_i^T)
__global__ void step_sym_kernel(const double* G, const double* Bt, int k, int nsec, double* A, double* scale) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsec) return;
  const int kk = k * k;
  const double* g = G + (size_t)s * kk;
  double* a = A + (size_t)s * kk;
  double sc = 0.0;
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      const double v = (i == j) ? g[i * k + i] : 0.5 * (g[i * k + j] + g[j * k + i]);
      a[i * k + j] = v;
      const double b = Bt ? Bt[(size_t)s * kk + i * k + j] : 0.0;
      sc += v * v + b * b;
    }
  scale[s] = sc;
}

// One CholQR pass: G = R^T R (R upper) and Rinv = R^-1.  flags[s] bit 0: the block broke down (a
// pivot below pivot_tol trace(G)), bit 1: it vanished (pass 0 only: trace(G) <= vanish_tol scale[s]).
// A broken sector gets R = Rinv = 0, which zeroes its block.  Pass 0 resets the flags.
__global__ void step_chol_kernel(const double* G, int k, int nsec, int pass, double vanish_tol, double pivot_tol,
                                 const double* scale, double* R, double* Rinv, int* flags) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsec) return;
  const int kk = k * k;
  const double* g = G + (size_t)s * kk;
  double* r = R + (size_t)s * kk;
  double* ri = Rinv + (size_t)s * kk;
  int f = pass == 0 ? 0 : flags[s];
  double trace = 0.0;
  for (int i = 0; i < k; ++i) trace += fabs(g[i * k + i]);
  if (pass == 0 && scale && !(trace > vanish_tol * scale[s])) f |= 3;
  for (int i = 0; i < kk; ++i) r[i] = ri[i] = 0.0;
  bool ok = (f & 1) == 0;
  for (int j = 0; j < k && ok; ++j) {
    double d = g[j * k + j];
    for (int p = 0; p < j; ++p) d -= r[p * k + j] * r[p * k + j];
    if (!(d > pivot_tol * fmax(trace, 1e-300))) {
      ok = false;
      break;
    }
    const double rjj = sqrt(d);
    r[j * k + j] = rjj;
    for (int c = j + 1; c < k; ++c) {
      double v = 0.5 * (g[j * k + c] + g[c * k + j]);
      for (int p = 0; p < j; ++p) v -= r[p * k + j] * r[p * k + c];
      r[j * k + c] = v / rjj;
    }
  }
  if (ok) {
    for (int c = 0; c < k; ++c)  // R Rinv = I, column by column (back substitution)
      for (int i = c; i >= 0; --i) {
        double v = (i == c) ? 1.0 : 0.0;
        for (int p = i + 1; p <= c; ++p) v -= r[i * k + p] * ri[p * k + c];
        ri[i * k + c] = v / r[i * k + i];
      }
  } else {
    f |= 1;
    for (int i = 0; i < kk; ++i) r[i] = ri[i] = 0.0;
  }
  flags[s] = f;
}

// B = R2 R1 (the new block's coefficient, upper; zero for a broken sector) and Bt_next = B^T
__global__ void step_b_kernel(const double* R1, const double* R2, const int* flags, int k, int nsec, double* B,
                              double* Bt_next) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsec) return;
  const int kk = k * k;
  const double* a = R2 + (size_t)s * kk;
  const double* b = R1 + (size_t)s * kk;
  const bool broke = flags[s] & 1;
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) {
      double v = 0.0;
      if (!broke)
        for (int p = 0; p < k; ++p) v += a[i * k + p] * b[p * k + j];
      B[(size_t)s * kk + i * k + j] = v;
      Bt_next[(size_t)s * kk + j * k + i] = v;
    }
}

__global__ void random_block_kernel(double* x, long long rows, int k, int first_col, const long long* row_sector_base,
                                    TileSetDevice t, uint64_t seed) {
  const int tile = blockIdx.x;
  const int s = t.tile_sector[tile];
  const long long base = row_sector_base[s];
  const long long r0 = t.tile_begin[tile], r1 = t.tile_end[tile];
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    for (int j = first_col; j < k; ++j) {
      // vector j of sector s: component i = (i+1)-th splitmix64 output of seed + j
      const uint64_t i = (uint64_t)(r - base);
      uint64_t z = seed + (uint64_t)j + (i + 1) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z = z ^ (z >> 31);
      x[r * k + j] = (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
  }
  (void)rows;
}

// column col of a [n][k] block from / to a contiguous vector (scaled on the way out)
__global__ void put_column_kernel(const double* v, long long n, int k, int col, double* x) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i * k + col] = v[i];
}

__global__ void get_column_kernel(const double* x, long long n, int k, int col, double scale, double* v) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) v[i] = scale * x[i * k + col];
}

__global__ void f32_copy_kernel(const double* x, float* y, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) y[i] = (float)x[i];
}

}  // namespace

int launch_seg_gram(const double* a, const double* b, int k, const TileSetDevice& t, double* partial, double* g,
                    cudaStream_t s) {
  if (t.nbr_tiles <= 0) return DH_OK;
  const int n = t.nbr_sectors * k * k;
  switch (k) {
    case 1:
      seg_gram_kernel<1><<<t.nbr_tiles, kThreads, 0, s>>>(a, b, t, partial);
      seg_gram_reduce_kernel<1><<<(n + 255) / 256, 256, 0, s>>>(partial, t, g);
      break;
    case 2:
      seg_gram_kernel<2><<<t.nbr_tiles, kThreads, 0, s>>>(a, b, t, partial);
      seg_gram_reduce_kernel<2><<<(n + 255) / 256, 256, 0, s>>>(partial, t, g);
      break;
    case 4:
      seg_gram_kernel<4><<<t.nbr_tiles, kThreads, 0, s>>>(a, b, t, partial);
      seg_gram_reduce_kernel<4><<<(n + 255) / 256, 256, 0, s>>>(partial, t, g);
      break;
    default:
      set_error("block size %d not in {1, 2, 4}", k);
      return DH_ERR_UNSUPPORTED;
  }
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_seg_update(double* w, const double* v, const double* A, const double* vp, const double* Bt, int k,
                      const TileSetDevice& t, cudaStream_t s) {
  if (t.nbr_tiles <= 0) return DH_OK;
  switch (k) {
    case 1: seg_update_kernel<1><<<t.nbr_tiles, kThreads, 0, s>>>(w, v, A, vp, Bt, t); break;
    case 2: seg_update_kernel<2><<<t.nbr_tiles, kThreads, 0, s>>>(w, v, A, vp, Bt, t); break;
    case 4: seg_update_kernel<4><<<t.nbr_tiles, kThreads, 0, s>>>(w, v, A, vp, Bt, t); break;
    default: set_error("block size %d not in {1, 2, 4}", k); return DH_ERR_UNSUPPORTED;
  }
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_seg_rmul(double* w, const double* M, int k, const TileSetDevice& t, float* w32, cudaStream_t s) {
  if (t.nbr_tiles <= 0) return DH_OK;
  switch (k) {
    case 1: seg_rmul_kernel<1><<<t.nbr_tiles, kThreads, 0, s>>>(w, M, t, w32); break;
    case 2: seg_rmul_kernel<2><<<t.nbr_tiles, kThreads, 0, s>>>(w, M, t, w32); break;
    case 4: seg_rmul_kernel<4><<<t.nbr_tiles, kThreads, 0, s>>>(w, M, t, w32); break;
    default: set_error("block size %d not in {1, 2, 4}", k); return DH_ERR_UNSUPPORTED;
  }
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_seg_combine_blocks(const double* blocks, int nb, long long stride, const double* C, int cstride, int k,
                              const TileSetDevice& t, double* out, cudaStream_t s) {
  if (t.nbr_tiles <= 0) return DH_OK;
  switch (k) {
    case 1: seg_combine_blocks_kernel<1><<<t.nbr_tiles, kThreads, 0, s>>>(blocks, nb, stride, C, cstride, t, out); break;
    case 2: seg_combine_blocks_kernel<2><<<t.nbr_tiles, kThreads, 0, s>>>(blocks, nb, stride, C, cstride, t, out); break;
    case 4: seg_combine_blocks_kernel<4><<<t.nbr_tiles, kThreads, 0, s>>>(blocks, nb, stride, C, cstride, t, out); break;
    default: set_error("block size %d not in {1, 2, 4}", k); return DH_ERR_UNSUPPORTED;
  }
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_step_sym(const double* G, const double* Bt, int k, int nsec, double* A, double* scale, cudaStream_t s) {
  if (nsec <= 0) return DH_OK;
  step_sym_kernel<<<(nsec + 127) / 128, 128, 0, s>>>(G, Bt, k, nsec, A, scale);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_step_chol(const double* G, int k, int nsec, int pass, double vanish_tol, double pivot_tol, const double* scale,
                     double* R, double* Rinv, int* flags, cudaStream_t s) {
  if (nsec <= 0) return DH_OK;
  step_chol_kernel<<<(nsec + 127) / 128, 128, 0, s>>>(G, k, nsec, pass, vanish_tol, pivot_tol, scale, R, Rinv, flags);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_step_b(const double* R1, const double* R2, const int* flags, int k, int nsec, double* B, double* Bt_next,
                  cudaStream_t s) {
  if (nsec <= 0) return DH_OK;
  step_b_kernel<<<(nsec + 127) / 128, 128, 0, s>>>(R1, R2, flags, k, nsec, B, Bt_next);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_random_block(double* x, long long rows, int k, const long long* row_sector_base, const TileSetDevice& t,
                        uint64_t seed, cudaStream_t s, int first_col) {
  if (t.nbr_tiles <= 0 || first_col >= k) return DH_OK;
  random_block_kernel<<<t.nbr_tiles, kThreads, 0, s>>>(x, rows, k, first_col, row_sector_base, t, seed);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

static unsigned stream_grid(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}

int launch_put_column(const double* v, long long n, int k, int col, double* x, cudaStream_t s) {
  if (n <= 0) return DH_OK;
  put_column_kernel<<<stream_grid(n), 256, 0, s>>>(v, n, k, col, x);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_get_column(const double* x, long long n, int k, int col, double scale, double* v, cudaStream_t s) {
  if (n <= 0) return DH_OK;
  get_column_kernel<<<stream_grid(n), 256, 0, s>>>(x, n, k, col, scale, v);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_f32_copy(const double* x, float* y, long long n, cudaStream_t s) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  f32_copy_kernel<<<(unsigned)g, 256, 0, s>>>(x, y, n);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

}  // namespace dh

// FP64 vector kernels of the Lanczos recurrence (the roles of RealVector::operator* (dot),
// AddLinearCombination and Norm, src/Vector/RealVector.cc:909,1083,3381, and of
// MultipleRealScalarProductOperation / AddRealLinearCombinationOperation).
//
// Every scalar the recurrence needs (alpha, beta, norms) stays in device memory, so a Lanczos step
// is a fixed sequence of launches with no host round trip and can be captured in a CUDA graph.
// Reductions are two-level and deterministic: each block writes its partial sums to a scratch row,
// the last block to finish (ticket counter) adds the rows in block order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "dh_internal.h"

namespace dh {
namespace {

constexpr int kVecThreads = 256;
constexpr int kMaxDots = 8;

struct Ptrs {
  const double* p[kMaxDots];
};

template <int W>
__device__ __forceinline__ void block_reduce_store(double (&acc)[W], double* partial) {
  __shared__ double red[W][kVecThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < W) {
    double v = 0.0;
    for (int w = 0; w < kVecThreads / 32; ++w) v += red[threadIdx.x][w];
    partial[(size_t)blockIdx.x * W + threadIdx.x] = v;
  }
}

// the last block sums the partial rows in block order; returns true in that block
template <int W>
__device__ __forceinline__ bool last_block_sum(const double* partial, unsigned int* ticket, double (&tot)[W]) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  __shared__ double red[W][kVecThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += ((volatile const double*)partial)[(size_t)b * W + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][warp] = v;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double v = 0.0;
    for (int w = 0; w < kVecThreads / 32; ++w) v += red[j][w];
    tot[j] = v;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

template <int W>
__global__ void __launch_bounds__(kVecThreads) multi_dot_kernel(Ptrs vs, const double* __restrict__ y, long long n,
                                                                 double* partial, unsigned int* ticket, double* out) {
  double acc[W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[j] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double yi = y[i];
#pragma unroll
    for (int j = 0; j < W; ++j) acc[j] += vs.p[j][i] * yi;
  }
  block_reduce_store<W>(acc, partial);
  double tot[W];
  if (last_block_sum<W>(partial, ticket, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < W; ++j) out[j] = tot[j];
  }
}

// w = y - ca * a - cb * b (ca, cb device scalars, either vector may be null); norm_out = |w|
__global__ void __launch_bounds__(kVecThreads) lanczos_update_kernel(double* w, const double* y, const double* a,
                                                                      const double* b, const double* ca,
                                                                      const double* cb, long long n, double* partial,
                                                                      unsigned int* ticket, double* norm_out) {
  const double fa = a ? *ca : 0.0, fb = b ? *cb : 0.0;
  double acc[1] = {0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = y[i];
    if (a) v -= fa * a[i];
    if (b) v -= fb * b[i];
    w[i] = v;
    acc[0] += v * v;
  }
  block_reduce_store<1>(acc, partial);
  double tot[1];
  if (last_block_sum<1>(partial, ticket, tot) && threadIdx.x == 0) *norm_out = sqrt(tot[0]);
}

__global__ void scale_convert_kernel(double* v, float* v32, const double* norm, long long n) {
  const double inv = 1.0 / *norm;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double x = v[i] * inv;
    v[i] = x;
    if (v32) v32[i] = (float)x;
  }
}

__global__ void convert_f32_kernel(const double* v, float* v32, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) v32[i] = (float)v[i];
}

__global__ void axpy_scalar_kernel(double* y, const double* x, double a, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) y[i] += a * x[i];
}

// component i: (i+1)-th splitmix64 output of `seed`, mapped to [-1, 1)
__global__ void random_vector_kernel(double* x, long long n, uint64_t seed) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    x[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  }
}

// out[i * m + c] (+)= sum_j v[i * k + j] * coef[j * m + c]   (tall-skinny times small, row-major)
__global__ void gemm_tall_kernel(const double* v, long long n, int k, const double* coef, int m, double* out,
                                 int accumulate) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    for (int c = 0; c < m; ++c) {
      double acc = accumulate ? out[i * m + c] : 0.0;
      for (int j = 0; j < k; ++j) acc += v[i * k + j] * coef[j * m + c];
      out[i * m + c] = acc;
    }
  }
}

// out[p * kb + q] = sum_i a[i * ka + p] * b[i * kb + q]  (ka * kb <= 16)
template <int KA, int KB>
__global__ void __launch_bounds__(kVecThreads) gram_kernel(const double* a, const double* b, long long n,
                                                           double* partial, unsigned int* ticket, double* out) {
  double acc[KA * KB];
#pragma unroll
  for (int j = 0; j < KA * KB; ++j) acc[j] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double av[KA], bv[KB];
#pragma unroll
    for (int p = 0; p < KA; ++p) av[p] = a[i * KA + p];
#pragma unroll
    for (int q = 0; q < KB; ++q) bv[q] = b[i * KB + q];
#pragma unroll
    for (int p = 0; p < KA; ++p)
#pragma unroll
      for (int q = 0; q < KB; ++q) acc[p * KB + q] += av[p] * bv[q];
  }
  block_reduce_store<KA * KB>(acc, partial);
  double tot[KA * KB];
  if (last_block_sum<KA * KB>(partial, ticket, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < KA * KB; ++j) out[j] = tot[j];
  }
}

// ------------------------------------------------------------------ Lanczos steps
// Three rotating vectors: v_i lives in slot i % 3.  Iteration i turns H v_i (in slot (i+1) % 3)
// into v_{i+1} = (H v_i - beta_{i-1} v_{i-1} - alpha_i v_i) / norm, then H v_{i+1} goes to slot
// (i+2) % 3 and beta_i = <v_i|H v_{i+1}>, alpha_{i+1} = <v_{i+1}|H v_{i+1}> (BasicLanczosAlgorithm.cc:
// 170-190).  i is read from cursor[0] on the device and advanced by the dot kernel, so a run of
// iterations needs no host round trip.
__global__ void __launch_bounds__(kVecThreads) lz_update_kernel(LanczosDev st, int phase) {
  const int i = *st.cursor;
  double* w = st.vec + (size_t)((phase + 1) % 3) * st.dim;
  const double* vm = st.vec + (size_t)((phase + 2) % 3) * st.dim;  // v_{i-1}
  const double* v0 = st.vec + (size_t)phase * st.dim;              // v_i
  const double b = (i > 0) ? st.beta[i - 1] : 0.0;
  const double a = st.alpha[i];
  double acc[1] = {0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < st.dim; k += stride) {
    double x = w[k] - a * v0[k];
    if (i > 0) x -= b * vm[k];
    w[k] = x;
    acc[0] += x * x;
  }
  block_reduce_store<1>(acc, st.partial);
  double tot[1];
  if (last_block_sum<1>(st.partial, st.ticket, tot) && threadIdx.x == 0) st.norm[i + 1] = sqrt(tot[0]);
}

// v_{i+1} /= norm, FP32 copy for the FP32 product, optional copy into the Krylov store
__global__ void lz_scale_kernel(LanczosDev st, int phase) {
  const int i = *st.cursor;
  double* w = st.vec + (size_t)((phase + 1) % 3) * st.dim;
  const double inv = 1.0 / st.norm[i + 1];
  double* kv = st.krylov ? st.krylov + (size_t)(i + 1) * st.dim : nullptr;
  if (st.krylov && i + 1 >= st.krylov_cap) kv = nullptr;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < st.dim; k += stride) {
    const double x = w[k] * inv;
    w[k] = x;
    if (st.x32) st.x32[k] = (float)x;
    if (kv) kv[k] = x;
  }
}

// beta_i = <v_i|y>, alpha_{i+1} = <v_{i+1}|y> (y = H v_{i+1}); advances the cursor
__global__ void __launch_bounds__(kVecThreads) lz_dots_kernel(LanczosDev st, int phase) {
  const int i = *st.cursor;
  const double* v0 = st.vec + (size_t)phase * st.dim;
  const double* v1 = st.vec + (size_t)((phase + 1) % 3) * st.dim;
  const double* y = st.vec + (size_t)((phase + 2) % 3) * st.dim;
  double acc[2] = {0.0, 0.0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < st.dim; k += stride) {
    const double yk = y[k];
    acc[0] += v0[k] * yk;
    acc[1] += v1[k] * yk;
  }
  block_reduce_store<2>(acc, st.partial);
  double tot[2];
  if (last_block_sum<2>(st.partial, st.ticket, tot) && threadIdx.x == 0) {
    st.beta[i] = tot[0];
    st.alpha[i + 1] = tot[1];
    *st.cursor = i + 1;
  }
}

// out[k] = (accumulate ? out[k] : 0) + sign * sum_j coef[j] * vs[j * ld + k]   (coef on the device)
__global__ void combine_kernel(const double* vs, int m, long long ld, const double* coef, double sign, double* out,
                               int accumulate, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    double acc = 0.0;
    for (int j = 0; j < m; ++j) acc += coef[j] * vs[(size_t)j * ld + k];
    out[k] = (accumulate ? out[k] : 0.0) + sign * acc;
  }
}

// coef[j] = <vs[j]|y> for m vectors of a strided store (classical Gram-Schmidt projections)
template <int W>
__global__ void __launch_bounds__(kVecThreads) strided_dots_kernel(const double* vs, long long ld, const double* y,
                                                                    long long n, double* partial,
                                                                    unsigned int* ticket, double* out) {
  double acc[W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[j] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const double yk = y[k];
#pragma unroll
    for (int j = 0; j < W; ++j) acc[j] += vs[(size_t)j * ld + k] * yk;
  }
  block_reduce_store<W>(acc, partial);
  double tot[W];
  if (last_block_sum<W>(partial, ticket, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < W; ++j) out[j] = tot[j];
  }
}

__global__ void sqrt_inplace_kernel(double* x) { *x = sqrt(*x); }

inline unsigned grid_for(long long n, int cap) {
  long long g = (n + kVecThreads - 1) / kVecThreads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace

int reducer_init(Reducer& r, DevBuf& storage, int width) {
  int dev = 0, sms = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  r.nblocks = sms * 4;
  r.width = width;
  size_t bytes = (size_t)r.nblocks * width * sizeof(double) + 256;
  int rc = storage.alloc(bytes);
  if (rc != DH_OK) return rc;
  r.partial = storage.as<double>();
  r.ticket = reinterpret_cast<unsigned int*>(static_cast<char*>(storage.ptr) + (size_t)r.nblocks * width * sizeof(double));
  DH_CUDA(cudaMemset(r.ticket, 0, sizeof(unsigned int)));
  return DH_OK;
}

int launch_multi_dot(const double* const* vs, int m, const double* y, long long n, double* out, Reducer& r,
                     cudaStream_t s) {
  if (m < 1 || m > kMaxDots || m > r.width) {
    set_error("multi_dot: %d vectors (at most %d)", m, r.width < kMaxDots ? r.width : kMaxDots);
    return DH_ERR_ARGUMENT;
  }
  Ptrs p = {};
  for (int j = 0; j < m; ++j) p.p[j] = vs[j];
  unsigned g = grid_for(n, r.nblocks);
  switch (m) {
    case 1: multi_dot_kernel<1><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 2: multi_dot_kernel<2><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 3: multi_dot_kernel<3><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 4: multi_dot_kernel<4><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 5: multi_dot_kernel<5><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 6: multi_dot_kernel<6><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    case 7: multi_dot_kernel<7><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
    default: multi_dot_kernel<8><<<g, kVecThreads, 0, s>>>(p, y, n, r.partial, r.ticket, out); break;
  }
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_lanczos_update(double* w, const double* y, const double* a, const double* b, const double* ca,
                          const double* cb, long long n, double* norm_out, Reducer& r, cudaStream_t s) {
  unsigned g = grid_for(n, r.nblocks);
  lanczos_update_kernel<<<g, kVecThreads, 0, s>>>(w, y, a, b, ca, cb, n, r.partial, r.ticket, norm_out);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_scale_convert(double* v, float* v32, const double* norm, long long n, cudaStream_t s) {
  scale_convert_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(v, v32, norm, n);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_convert_f32(const double* v, float* v32, long long n, cudaStream_t s) {
  convert_f32_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(v, v32, n);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_axpy_scalar(double* y, const double* x, double a, long long n, cudaStream_t s) {
  axpy_scalar_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(y, x, a, n);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_random_vector(double* x, long long n, uint64_t seed, cudaStream_t s) {
  random_vector_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(x, n, seed);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_gemm_tall(const double* v, long long n, int k, const double* c, int m, double* out, int accumulate,
                     cudaStream_t s) {
  gemm_tall_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(v, n, k, c, m, out, accumulate);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_gram(const double* a, int ka, const double* b, int kb, long long n, double* out, Reducer& r,
                cudaStream_t s) {
  if (ka * kb > r.width) {
    set_error("gram: %d x %d exceeds the reducer width %d", ka, kb, r.width);
    return DH_ERR_ARGUMENT;
  }
  unsigned g = grid_for(n, r.nblocks);
#define DH_GRAM(A, B)                                                                      \
  if (ka == A && kb == B) {                                                                \
    gram_kernel<A, B><<<g, kVecThreads, 0, s>>>(a, b, n, r.partial, r.ticket, out);        \
    DH_CUDA(cudaGetLastError());                                                           \
    return DH_OK;                                                                          \
  }
  DH_GRAM(1, 1) DH_GRAM(2, 2) DH_GRAM(3, 3) DH_GRAM(4, 4) DH_GRAM(2, 1) DH_GRAM(4, 1) DH_GRAM(1, 2) DH_GRAM(1, 4)
#undef DH_GRAM
  set_error("gram: unsupported block shape %d x %d", ka, kb);
  return DH_ERR_UNSUPPORTED;
}

int launch_lz_update(const LanczosDev& st, int phase, cudaStream_t s) {
  lz_update_kernel<<<st.nblocks, kVecThreads, 0, s>>>(st, phase);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_lz_scale(const LanczosDev& st, int phase, cudaStream_t s) {
  lz_scale_kernel<<<grid_for(st.dim, 148 * 8), kVecThreads, 0, s>>>(st, phase);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_lz_dots(const LanczosDev& st, int phase, cudaStream_t s) {
  lz_dots_kernel<<<st.nblocks, kVecThreads, 0, s>>>(st, phase);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_combine(const double* vs, int m, long long ld, const double* coef, double sign, double* out, int accumulate,
                   long long n, cudaStream_t s) {
  combine_kernel<<<grid_for(n, 148 * 8), kVecThreads, 0, s>>>(vs, m, ld, coef, sign, out, accumulate, n);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

int launch_strided_dots(const double* vs, int m, long long ld, const double* y, long long n, double* out, Reducer& r,
                        cudaStream_t s) {
  unsigned g = grid_for(n, r.nblocks);
  for (int j0 = 0; j0 < m; j0 += 8) {
    const int w = (m - j0 >= 8) ? 8 : m - j0;
    DH_CHECK(w <= r.width, DH_ERR_ARGUMENT, "strided_dots: reducer too narrow");
    const double* base = vs + (size_t)j0 * ld;
    switch (w) {
      case 1: strided_dots_kernel<1><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 2: strided_dots_kernel<2><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 3: strided_dots_kernel<3><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 4: strided_dots_kernel<4><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 5: strided_dots_kernel<5><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 6: strided_dots_kernel<6><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      case 7: strided_dots_kernel<7><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
      default: strided_dots_kernel<8><<<g, kVecThreads, 0, s>>>(base, ld, y, n, r.partial, r.ticket, out + j0); break;
    }
    DH_CUDA(cudaGetLastError());
  }
  return DH_OK;
}

int launch_sqrt_inplace(double* x, cudaStream_t s) {
  sqrt_inplace_kernel<<<1, 1, 0, s>>>(x);
  DH_CUDA(cudaGetLastError());
  return DH_OK;
}

}  // namespace dh

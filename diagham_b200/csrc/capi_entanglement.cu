// C ABI: orbital-cut entanglement of a FermionOnSphere vector on the GPU
// (FermionOnSphere::EvaluatePartialEntanglementMatrix, FermionOnSphere.cc:2474, and
// EvaluatePartialDensityMatrix, :2070).
//
// Subsystem A = orbitals 0..l-1, B = orbitals l..2S.  In the sector (N_A, 2Lz_A) every basis state
// whose A part holds N_A fermions with the sector's orbital sum splits into an A word (its low l bits)
// and a B word (its high bits shifted down by l); M[a][b] = psi(state), rows in the order of
// FermionOnSphere(N_A, 2Lz_A, l - 1), columns in the order of FermionOnSphere(N_B, 2Lz_B, 2S - l),
// and the density matrix is rho_A = M M^T.  On the device: one pass over the basis compacts the
// sector's states (A word, B word, component), the FindStateIndex kernels of the two subsystem
// spaces give their row and column, a scatter fills M and a tiled FP64 kernel forms M M^T.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "dh_internal.h"
#include "dh_objects.h"

using namespace dh;

namespace {

constexpr int kCutThreads = 256;

// words of state i at words[i * wstride]: wstride 2 for the (low, high) pairs of the 128-bit engine,
// whose high halves are zero up to lz_max = 62
__global__ void cut_split_kernel(const uint64_t* words, int wstride, long long dim, const double* psi, int l, int na,
                                 int sum_a, uint64_t* aw, uint64_t* bw, double* val, unsigned long long* count) {
  const uint64_t amask = (l >= 64) ? ~0ull : ((1ull << l) - 1ull);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    const uint64_t w = words[i * wstride];
    const uint64_t a = w & amask;
    if (__popcll(a) != na) continue;
    int s = 0;
    for (uint64_t t = a; t; t &= t - 1ull) s += __ffsll(t) - 1;
    if (s != sum_a) continue;
    const unsigned long long k = atomicAdd(count, 1ull);
    aw[k] = a;
    bw[k] = (l >= 64) ? 0ull : (w >> l);
    val[k] = psi[i];
  }
}

// sum of psi^2 over the states whose A part (low l bits) is key
__global__ void cut_weight_kernel(const uint64_t* words, int wstride, long long dim, const double* psi, int l,
                                  uint64_t key, double* total) {
  const uint64_t amask = (l >= 64) ? ~0ull : ((1ull << l) - 1ull);
  double acc = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride)
    if ((words[i * wstride] & amask) == key) acc += psi[i] * psi[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(total, acc);
}

__global__ void cut_scatter_kernel(const long long* ia, const long long* ib, const double* val, long long n,
                                   double* m, long long cols) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const long long r = ia ? ia[k] : 0, c = ib ? ib[k] : 0;
    m[r * cols + c] = val[k];
  }
}

// rho = M M^T for a row-major rows x cols M: 32 x 32 output tiles, the shared dimension in slices of
// 32 staged in shared memory; each thread accumulates 4 outputs
constexpr int kTile = 32;
__global__ void __launch_bounds__(256) gram_kernel(const double* m, long long rows, long long cols, double* rho) {
  __shared__ double ta[kTile][kTile + 1];
  __shared__ double tb[kTile][kTile + 1];
  const long long i0 = (long long)blockIdx.y * kTile, j0 = (long long)blockIdx.x * kTile;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long k0 = 0; k0 < cols; k0 += kTile) {
    for (int q = 0; q < 4; ++q) {
      const int rr = ty + 8 * q;
      const long long kk = k0 + tx;
      ta[rr][tx] = (i0 + rr < rows && kk < cols) ? m[(i0 + rr) * cols + kk] : 0.0;
      tb[rr][tx] = (j0 + rr < rows && kk < cols) ? m[(j0 + rr) * cols + kk] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kTile; ++kk) {
      const double b = tb[tx][kk];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += ta[ty + 8 * q][kk] * b;
    }
    __syncthreads();
  }
  for (int q = 0; q < 4; ++q) {
    const long long i = i0 + ty + 8 * q, j = j0 + tx;
    if (i < rows && j < rows) rho[i * rows + j] = acc[q];
  }
}

unsigned grid_of(long long n) {
  long long g = (n + kCutThreads - 1) / kCutThreads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}

struct SpaceGuard {
  dh_space_t s = nullptr;
  ~SpaceGuard() {
    if (s) dh_space_destroy(s);
  }
};

// the cut's M on the device (rows x cols, row-major); rows = cols = 0 for an empty sector
int cut_matrix(dh_space_s* sp, const double* state_dev, int l, int na, int lza, bool density, DevBuf& m,
               int64_t* rows, int64_t* cols, bool* nonzero) {
  *rows = *cols = 0;
  *nonzero = false;
  const int N = sp->nbr_fermions, L = sp->lz_max;
  const int nb = N - na;
  if (na < 0 || nb < 0 || na > l || nb > L + 1 - l) return DH_OK;
  // orbital-index sum of A: the reference floors (2 Lz_A + N_A (l - 1)) / 2 (FermionOnSphere.cc:2095), so
  // an odd value selects the sector below it
  const int twice_a = lza + na * (l - 1);
  const int sum_a = (twice_a >= 0) ? twice_a / 2 : -((1 - twice_a) / 2);
  lza = 2 * sum_a - na * (l - 1);
  const int sum_b = sp->total_sum - sum_a;  // of B, absolute orbital indices
  if (sum_a < na * (na - 1) / 2 || sum_a > na * (l - 1) - na * (na - 1) / 2) return DH_OK;
  const bool b_ok = sum_b >= l * nb + nb * (nb - 1) / 2 && sum_b <= nb * L - nb * (nb - 1) / 2;
  if (!b_ok) return DH_OK;  // an empty complementary sector gives an empty result
  (void)density;
  SpaceGuard a_space, b_space;
  int rc;
  int64_t dim_a = 1, dim_b = 1;
  if (na > 0) {
    if ((rc = dh_fermion_on_sphere_create(na, lza, l - 1, 0, &a_space.s)) != DH_OK) return rc;
    dim_a = a_space.s->dim;
  }
  if (nb > 0 && b_ok) {
    const int lz_b = 2 * (sum_b - nb * l) - nb * (L - l);
    if ((rc = dh_fermion_on_sphere_create(nb, lz_b, L - l, 0, &b_space.s)) != DH_OK) return rc;
    dim_b = b_space.s->dim;
  }
  *rows = dim_a;
  *cols = dim_b;
  if ((rc = m.alloc((size_t)std::max<int64_t>(dim_a * dim_b, 1) * sizeof(double))) != DH_OK) return rc;
  DH_CUDA(cudaMemset(m.ptr, 0, (size_t)std::max<int64_t>(dim_a * dim_b, 1) * sizeof(double)));
  if (dim_b == 0) return DH_OK;
  // compact the sector's states
  const long long dim = sp->dim;
  DevBuf aw, bw, val, cnt, ia, ib;
  if ((rc = aw.alloc(dim * sizeof(uint64_t))) != DH_OK || (rc = bw.alloc(dim * sizeof(uint64_t))) != DH_OK ||
      (rc = val.alloc(dim * sizeof(double))) != DH_OK || (rc = cnt.alloc(sizeof(unsigned long long))) != DH_OK)
    return rc;
  DH_CUDA(cudaMemset(cnt.ptr, 0, sizeof(unsigned long long)));
  cut_split_kernel<<<grid_of(dim), kCutThreads>>>(sp->words.as<uint64_t>(), sp->kind == SPACE_FERMION_LONG ? 2 : 1,
                                                 dim, state_dev, l, na, sum_a,
                                                 aw.as<uint64_t>(), bw.as<uint64_t>(), val.as<double>(),
                                                 cnt.as<unsigned long long>());
  DH_CUDA(cudaGetLastError());
  unsigned long long n = 0;
  DH_CUDA(cudaMemcpy(&n, cnt.ptr, sizeof(n), cudaMemcpyDeviceToHost));
  if (n == 0) return DH_OK;
  *nonzero = true;
  if (na > 0) {
    if ((rc = ia.alloc(n * sizeof(long long))) != DH_OK) return rc;
    // the subsystem spaces may be of either engine: the C entry point picks the right search
    if ((rc = dh_space_find_state_index(a_space.s, aw.as<uint64_t>(), (int64_t)n, ia.as<int64_t>())) != DH_OK)
      return rc;
  }
  if (nb > 0) {
    if ((rc = ib.alloc(n * sizeof(long long))) != DH_OK) return rc;
    if ((rc = dh_space_find_state_index(b_space.s, bw.as<uint64_t>(), (int64_t)n, ib.as<int64_t>())) != DH_OK)
      return rc;
  }
  cut_scatter_kernel<<<grid_of((long long)n), kCutThreads>>>(na > 0 ? ia.as<long long>() : nullptr,
                                                             nb > 0 ? ib.as<long long>() : nullptr, val.as<double>(),
                                                             (long long)n, m.as<double>(), dim_b);
  DH_CUDA(cudaGetLastError());
  DH_CUDA(cudaDeviceSynchronize());
  return DH_OK;
}

int copy_out(double* out, const double* dev, int64_t n) {
  if (n <= 0) return DH_OK;
  const cudaMemcpyKind kind = is_device_pointer(out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  DH_CUDA(cudaMemcpy(out, dev, (size_t)n * sizeof(double), kind));
  return DH_OK;
}

int entanglement_common(dh_space_t sp, const double* state, int l, int na, int lza, bool density, double* out,
                        int64_t capacity, int64_t* rows, int64_t* cols) {
  DH_CHECK(sp && state && rows && cols, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(sp->kind == SPACE_FERMION || (sp->kind == SPACE_FERMION_LONG && sp->lz_max <= 62), DH_ERR_UNSUPPORTED,
           "orbital cuts are implemented for FermionOnSphere (lz_max <= 62)");
  *rows = *cols = 0;
  const int64_t dim = sp->dim;
  int rc;
  // l <= 0: A is empty, a 1 x 1 [1] in its trivial sector (FermionOnSphere.cc:2072-2082, :2476-2487)
  if (l <= 0) {
    if (lza == 0 && na == 0) {
      *rows = *cols = 1;
      if (out && capacity >= 1) {
        const double one = 1.0;
        const cudaMemcpyKind kind = is_device_pointer(out) ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
        DH_CUDA(cudaMemcpy(out, &one, sizeof(double), kind));
      }
    }
    return DH_OK;
  }
  // the state on the device
  DevBuf staged;
  const double* psi = state;
  if (!is_device_pointer(state)) {
    if ((rc = staged.alloc((size_t)dim * sizeof(double))) != DH_OK) return rc;
    DH_CUDA(cudaMemcpy(staged.ptr, state, (size_t)dim * sizeof(double), cudaMemcpyHostToDevice));
    psi = staged.as<double>();
  }
  // l > 2S: A is the whole system, M = psi as one column (:2490-2504) and rho = psi psi^T
  if (l > sp->lz_max) {
    if (lza != sp->total_lz || na != sp->nbr_fermions) return DH_OK;
    if (!density) {
      *rows = dim;
      *cols = 1;
      if (out && capacity >= dim) return copy_out(out, psi, dim);
      return DH_OK;
    }
    *rows = *cols = dim;
    if (!out || capacity < dim * dim) return DH_OK;
    DevBuf rho;
    if ((rc = rho.alloc((size_t)dim * dim * sizeof(double))) != DH_OK) return rc;
    dim3 grid((unsigned)((dim + kTile - 1) / kTile), (unsigned)((dim + kTile - 1) / kTile));
    gram_kernel<<<grid, 256>>>(psi, dim, 1, rho.as<double>());
    DH_CUDA(cudaGetLastError());
    return copy_out(out, rho.as<double>(), dim * dim);
  }
  // N_A <= 1: the reference's density matrix is the 1 x 1 weight of the states whose A part is empty
  // (N_A = 0, whatever the sector's Lz) or the one orbital (2Lz_A + l - 1) / 2 (N_A = 1), zero when
  // there is none (FermionOnSphere.cc:2139-2155)
  if (density && na <= 1) {
    const int orbital = (lza + l - 1) >> 1;
    const uint64_t key = (na == 0) ? 0ull : ((orbital >= 0 && orbital < l) ? (1ull << orbital) : ~0ull);
    DevBuf t;
    if ((rc = t.alloc(sizeof(double))) != DH_OK) return rc;
    DH_CUDA(cudaMemset(t.ptr, 0, sizeof(double)));
    if (key != ~0ull) {
      cut_weight_kernel<<<grid_of(dim), kCutThreads>>>(sp->words.as<uint64_t>(), sp->kind == SPACE_FERMION_LONG ? 2 : 1,
                                                      dim, psi, l, key, t.as<double>());
      DH_CUDA(cudaGetLastError());
    }
    *rows = *cols = 1;
    if (out && capacity >= 1) return copy_out(out, t.as<double>(), 1);
    return DH_OK;
  }
  DevBuf m;
  bool nonzero = false;
  int64_t r = 0, c = 0;
  if ((rc = cut_matrix(sp, psi, l, na, lza, density, m, &r, &c, &nonzero)) != DH_OK) return rc;
  if (!density) {
    if (r == 0 || c == 0) return DH_OK;
    *rows = r;
    *cols = c;
    if (out && capacity >= r * c) return copy_out(out, m.as<double>(), r * c);
    return DH_OK;
  }
  // a density matrix with no contributing state is empty (:2262-2268)
  if (r == 0 || c == 0 || !nonzero) return DH_OK;
  *rows = *cols = r;
  if (!out || capacity < r * r) return DH_OK;
  DevBuf rho;
  if ((rc = rho.alloc((size_t)r * r * sizeof(double))) != DH_OK) return rc;
  dim3 grid((unsigned)((r + kTile - 1) / kTile), (unsigned)((r + kTile - 1) / kTile));
  gram_kernel<<<grid, 256>>>(m.as<double>(), r, c, rho.as<double>());
  DH_CUDA(cudaGetLastError());
  return copy_out(out, rho.as<double>(), r * r);
}

}  // namespace

extern "C" {

int dh_fermion_on_sphere_partial_entanglement_matrix(dh_space_t space, const double* state, int subsystem_size,
                                                     int nbr_fermion_sector, int lz_sector, double* matrix,
                                                     int64_t capacity, int64_t* rows, int64_t* cols) {
  return entanglement_common(space, state, subsystem_size, nbr_fermion_sector, lz_sector, false, matrix, capacity, rows,
                             cols);
}

int dh_fermion_on_sphere_partial_density_matrix(dh_space_t space, const double* state, int subsystem_size,
                                                int nbr_fermion_sector, int lz_sector, double* matrix, int64_t capacity,
                                                int64_t* dim) {
  int64_t cols = 0;
  DH_CHECK(dim, DH_ERR_ARGUMENT, "null argument");
  return entanglement_common(space, state, subsystem_size, nbr_fermion_sector, lz_sector, true, matrix, capacity, dim,
                             &cols);
}

}  // extern "C"

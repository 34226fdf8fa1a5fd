// Block Lanczos on the GPU, for one Hamiltonian or for all Lz sectors of a system in lockstep.
//
// Recurrence (the block form of BasicBlockLanczosAlgorithm.cc:524-697, k = block size):
//     W = H V_i;  A_i = V_i^T W;  W -= V_i A_i + V_{i-1} B_i^T;  W = V_{i+1} B_{i+1}  (QR)
// with every block stored k-interleaved ([row][k], FP64) so that one product enumerates each row's
// elements once for the k vectors.  The QR is CholQR2 (Gram matrix, Cholesky, triangular solve,
// twice), the role of ReorthogonalizeVectors (:771-799).  The band matrix of the A_i and B_i is
// diagonalised on the host after every step (band -> tridiagonal -> QL, the reference's
// RealBandDiagonalSymmetricMatrix::Tridiagonalize + Diagonalize), and each sector follows the
// reference's convergence bookkeeping (:683-697, TestConvergence :731).  A sector whose block
// Krylov space is exhausted stops: its band matrix is exact when the whole new block vanished with
// FP64 products; when the block only lost rank (dimension not a multiple of k) or the products were
// FP32, the space is small (at most the vectors built so far) and is diagonalised densely in FP64.
// Sectors of dimension at most full_diag_limit are diagonalised densely from the start, as
// QHEOnSphereMainTask does below --full-diag (:397).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "dh_internal.h"
#include "dh_objects.h"

using namespace dh;

namespace dh {

constexpr long long kTileRows = 4096;
constexpr int EngineRing = 8;  // BlockEngine::kRing
// largest exhausted space diagonalised densely on the host when its band matrix is not exact
constexpr long long kDenseFallbackLimit = 2048;

struct BlockSector {
  long long dim = 0;
  bool active = true;     // still iterating
  bool converged = false;
  bool exhausted = false; // Krylov space exhausted: the band matrix is exact ...
  bool partial = false;   // ... unless the last block only lost rank (dimension not a multiple of k)
  int blocks = 0;         // A blocks recorded
  std::vector<double> A, B;  // A_j (k x k) for j < blocks, B_j (k x k) for 1 <= j <= blocks (B[0] unused)
  double prev_last = 0.0;
  std::vector<double> ritz;
  int count = 0;          // the reference driver's iteration counter (in vectors)
  int steps = 0;
};

// coefficients of one block step for every sector, enough to replay it exactly (every kernel is
// deterministic): the symmetrised A, the B^T used by the update, and the two CholQR inverses
struct StepRecord {
  std::vector<double> A, Bt, inv1, inv2;
  std::vector<double> lock;  // start-block projection coefficients (empty when not locked)
  bool have_prev = false;
};

struct BlockEngine {
  int k = 4, nsec = 0, nev = 1, precision = DH_PRECISION_FP64;
  double eig_precision = 1e-14;
  // > 0: converge on the lowest Ritz vector's residual instead, |r|^2 < residual_target |lambda|
  // (|r| = |B_m s_last| from the band matrix), used by the mixed-precision restarts whose Ritz
  // values move at the FP32 rounding level long after the vector is accurate enough
  double residual_target = 0.0;
  // with residual_target: also stop a sector whose lowest Ritz value no longer moves (1e-13)
  bool stop_on_stagnation = false;
  int max_iter = 400;  // in vectors, as the reference's --iter-max
  long long total = 0;
  std::vector<long long> off;
  cudaStream_t stream = 0;
  DevBuf tiles_buf, vec, x32, partial, small, offs_dev;
  TileSetDevice tiles = {};
  const long long* row_offset_dev = nullptr;  // [nsec + 1] concatenated row offsets on the device
  int slot_cur = 0;
  double* slot[3] = {nullptr, nullptr, nullptr};
  bool have_prev = false;
  std::vector<BlockSector> sec;
  std::function<int(const double*, const float*, double*)> product;
  // the per-step bookkeeping needs only the lowest nev + 1 Ritz values (the batched sectors): for
  // k = 1 they come from bisection on the tridiagonal matrix instead of all of its eigenvalues
  bool lowest_only = false;
  double product_ms = 0.0;
  long long products = 0;
  long long fp64_products = 0;
  std::vector<StepRecord> history;
  // mixed-precision restart from a Ritz block: the start block's product in FP64, the following
  // ones in the engine's precision, every new block projected against the start block
  bool fp64_first_product = false;
  bool lock_start = false;
  DevBuf start_block;    // the orthonormal start block, for replays and the projection
  DevBuf store;          // every block when keep_blocks (store_cap blocks of total * k)
  int store_cap = 0;
  int store_max = 0;     // the store grows (doubling) up to this many blocks while memory allows
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Device-resident steps (engine_step_async): the per-sector k x k matrices of a step live on the
  // device; each step's coefficients and flags go back to a pinned record slot asynchronously, and
  // the host's bookkeeping (engine_process_step) follows the device by a few steps.
  static const int kRing = 8;                    // record slots (steps in flight at most kRing)
  DevBuf stepbuf;                                // G, A, Bt[2], R1, R2, inv1, inv2, B, lock, scale, flags, active
  double *dG = nullptr, *dA = nullptr, *dBt[2] = {nullptr, nullptr}, *dR1 = nullptr, *dR2 = nullptr;
  double *dInv1 = nullptr, *dInv2 = nullptr, *dB = nullptr, *dLock = nullptr, *dScale = nullptr;
  int *dFlags = nullptr, *dActive = nullptr;
  double* rec_host = nullptr;                    // pinned [kRing][6][nsec][k][k]
  int* rec_flags = nullptr;                      // pinned [kRing][nsec]
  int* mask_host = nullptr;                      // pinned [kRing][nsec] active masks being uploaded
  bool rec_locked[kRing] = {}, rec_have_prev[kRing] = {};
  cudaEvent_t ev_rec[kRing] = {}, ev_p0[kRing] = {}, ev_p1[kRing] = {};
  long long issued = 0;                          // steps issued; history.size() = steps processed
  std::vector<int> mask_sent;                    // the active mask the device has (or will have)
  ~BlockEngine() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (int i = 0; i < kRing; ++i) {
      if (ev_rec[i]) cudaEventDestroy(ev_rec[i]);
      if (ev_p0[i]) cudaEventDestroy(ev_p0[i]);
      if (ev_p1[i]) cudaEventDestroy(ev_p1[i]);
    }
    // the owner has waited for the stream (every record's event is waited on by the bookkeeping) and
    // may already have destroyed it: nothing here touches the stream
    if (rec_host) cudaFreeHost(rec_host);
    if (rec_flags) cudaFreeHost(rec_flags);
    if (mask_host) cudaFreeHost(mask_host);
    cudaGetLastError();  // leave no error of this clean-up for a later call to read
  }
};

namespace {

int engine_setup(BlockEngine& e, const std::vector<long long>& dims) {
  e.nsec = (int)dims.size();
  e.off.assign(e.nsec + 1, 0);
  e.sec.assign(e.nsec, BlockSector());
  for (int s = 0; s < e.nsec; ++s) {
    e.off[s + 1] = e.off[s] + dims[s];
    e.sec[s].dim = dims[s];
  }
  e.total = e.off[e.nsec];
  std::vector<int> tsec, first(e.nsec + 1, 0);
  std::vector<long long> tb, te;
  for (int s = 0; s < e.nsec; ++s) {
    first[s] = (int)tsec.size();
    for (long long r = e.off[s]; r < e.off[s + 1]; r += kTileRows) {
      tsec.push_back(s);
      tb.push_back(r);
      te.push_back(std::min(r + kTileRows, e.off[s + 1]));
    }
  }
  first[e.nsec] = (int)tsec.size();
  const int nt = (int)tsec.size();
  const size_t bytes = nt * (sizeof(int) + 2 * sizeof(long long)) + (e.nsec + 1) * (sizeof(int) + sizeof(long long)) + 64;
  int rc;
  if ((rc = e.tiles_buf.alloc(bytes)) != DH_OK) return rc;
  char* p = e.tiles_buf.as<char>();
  long long* d_tb = reinterpret_cast<long long*>(p);
  long long* d_te = d_tb + nt;
  long long* d_off = d_te + nt;
  int* d_ts = reinterpret_cast<int*>(d_off + e.nsec + 1);
  int* d_first = d_ts + nt;
  DH_CUDA(cudaMemcpy(d_tb, tb.data(), nt * sizeof(long long), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(d_te, te.data(), nt * sizeof(long long), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(d_off, e.off.data(), (e.nsec + 1) * sizeof(long long), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(d_ts, tsec.data(), nt * sizeof(int), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(d_first, first.data(), (e.nsec + 1) * sizeof(int), cudaMemcpyHostToDevice));
  e.tiles.tile_sector = d_ts;
  e.tiles.tile_begin = d_tb;
  e.tiles.tile_end = d_te;
  e.tiles.sector_tile_first = d_first;
  e.tiles.nbr_tiles = nt;
  e.tiles.nbr_sectors = e.nsec;
  e.row_offset_dev = d_off;
  const size_t vb = (size_t)e.total * e.k * sizeof(double);
  if ((rc = e.vec.alloc(3 * vb)) != DH_OK) return rc;
  if (e.precision == DH_PRECISION_FP32 && (rc = e.x32.alloc((size_t)e.total * e.k * sizeof(float))) != DH_OK) return rc;
  if ((rc = e.partial.alloc((size_t)std::max(nt, 1) * e.k * e.k * sizeof(double))) != DH_OK) return rc;
  if ((rc = e.small.alloc((size_t)e.nsec * e.k * e.k * 4 * sizeof(double) + 64)) != DH_OK) return rc;
  DH_CUDA(cudaMemset(e.vec.ptr, 0, 3 * vb));
  for (int q = 0; q < 3; ++q) e.slot[q] = e.vec.as<double>() + (size_t)q * e.total * e.k;
  if (!e.ev0) {
    DH_CUDA(cudaEventCreate(&e.ev0));
    DH_CUDA(cudaEventCreate(&e.ev1));
  }
  // device-resident step state and the pinned record ring
  const size_t nk = (size_t)e.nsec * e.k * e.k;
  if ((rc = e.stepbuf.alloc((10 * nk + e.nsec) * sizeof(double) + 2 * (size_t)e.nsec * sizeof(int))) != DH_OK) return rc;
  double* d = e.stepbuf.as<double>();
  e.dG = d;
  e.dA = d + nk;
  e.dBt[0] = d + 2 * nk;
  e.dBt[1] = d + 3 * nk;
  e.dR1 = d + 4 * nk;
  e.dR2 = d + 5 * nk;
  e.dInv1 = d + 6 * nk;
  e.dInv2 = d + 7 * nk;
  e.dB = d + 8 * nk;
  e.dLock = d + 9 * nk;
  e.dScale = d + 10 * nk;
  e.dFlags = reinterpret_cast<int*>(e.dScale + e.nsec);
  e.dActive = e.dFlags + e.nsec;
  DH_CUDA(cudaMemset(e.stepbuf.ptr, 0, e.stepbuf.bytes));
  if (e.rec_host) {
    cudaFreeHost(e.rec_host);
    cudaFreeHost(e.rec_flags);
    cudaFreeHost(e.mask_host);
    e.rec_host = nullptr;
    e.rec_flags = e.mask_host = nullptr;
  }
  DH_CUDA(cudaMallocHost(&e.rec_host, (size_t)EngineRing * 6 * nk * sizeof(double)));
  DH_CUDA(cudaMallocHost(&e.rec_flags, (size_t)EngineRing * e.nsec * sizeof(int)));
  DH_CUDA(cudaMallocHost(&e.mask_host, (size_t)EngineRing * e.nsec * sizeof(int)));
  if (!e.ev_rec[0]) {
    for (int i = 0; i < EngineRing; ++i) {
      DH_CUDA(cudaEventCreateWithFlags(&e.ev_rec[i], cudaEventDisableTiming));
      DH_CUDA(cudaEventCreate(&e.ev_p0[i]));
      DH_CUDA(cudaEventCreate(&e.ev_p1[i]));
    }
  }
  e.mask_sent.assign(e.nsec, -1);
  return DH_OK;
}

// G[s] = X_s^T Y_s for every sector, copied to the host
int engine_gram(BlockEngine& e, const double* x, const double* y, std::vector<double>& g) {
  const int kk = e.k * e.k;
  double* dg = e.small.as<double>();
  int rc = launch_seg_gram(x, y, e.k, e.tiles, e.partial.as<double>(), dg, e.stream);
  if (rc != DH_OK) return rc;
  g.resize((size_t)e.nsec * kk);
  DH_CUDA(cudaMemcpyAsync(g.data(), dg, g.size() * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaStreamSynchronize(e.stream));
  return DH_OK;
}

// Cholesky G = R^T R (R upper); returns false on breakdown (a pivot below tol trace(G)).
// Rinv = R^{-1} (upper).
bool cholesky_inverse(int k, const double* G, double* R, double* Rinv, double tol) {
  double trace = 0.0;
  for (int i = 0; i < k; ++i) trace += fabs(G[i * k + i]);
  for (int i = 0; i < k * k; ++i) R[i] = Rinv[i] = 0.0;
  for (int j = 0; j < k; ++j) {
    double d = G[j * k + j];
    for (int p = 0; p < j; ++p) d -= R[p * k + j] * R[p * k + j];
    if (!(d > tol * std::max(trace, 1e-300))) return false;
    const double rjj = sqrt(d);
    R[j * k + j] = rjj;
    for (int c = j + 1; c < k; ++c) {
      double v = 0.5 * (G[j * k + c] + G[c * k + j]);
      for (int p = 0; p < j; ++p) v -= R[p * k + j] * R[p * k + c];
      R[j * k + c] = v / rjj;
    }
  }
  for (int c = 0; c < k; ++c) {  // R Rinv = I, column by column (back substitution)
    for (int i = c; i >= 0; --i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int p = i + 1; p <= c; ++p) v -= R[i * k + p] * Rinv[p * k + c];
      Rinv[i * k + c] = v / R[i * k + i];
    }
  }
  return true;
}

// X = X Q with X = V B (CholQR2): writes B (k x k per sector, upper) and leaves X orthonormal.
// A sector whose block is numerically zero against its scale (|X|_F^2 < tol scale[s], scale =
// |A|^2 + |B|^2 of the step, tol = 1e-24 with FP64 products and 4e-12, about (32 u_FP32)^2, with
// FP32 ones: the block Krylov space is complete) or whose Gram matrix breaks down gets a zero
// block and is marked exhausted.
int engine_qr(BlockEngine& e, double* x, std::vector<double>& B, float* x32, const std::vector<double>* scale,
              std::vector<double>* inv1 = nullptr, std::vector<double>* inv2 = nullptr) {
  const int k = e.k, kk = k * k;
  std::vector<double> g, R1((size_t)e.nsec * kk), R2((size_t)e.nsec * kk), inv((size_t)e.nsec * kk);
  std::vector<char> broke(e.nsec, 0), vanished(e.nsec, 0);
  double* dM = e.small.as<double>() + (size_t)e.nsec * kk;
  int rc;
  for (int pass = 0; pass < 2; ++pass) {
    if ((rc = engine_gram(e, x, x, g)) != DH_OK) return rc;
    std::vector<double>& R = pass ? R2 : R1;
    // with FP32 products an exhausted Krylov space leaves FP32 rounding noise, not zero: the
    // vanishing and pivot thresholds are about (32 u)^2 of the product's precision
    const bool f32 = e.precision == DH_PRECISION_FP32;
    const double pivot_tol = f32 ? 4e-12 : 1e-26;
    if (pass == 0 && scale) {
      const double tol = f32 ? 4e-12 : 1e-24;
      for (int s = 0; s < e.nsec; ++s) {
        double tr = 0.0;
        for (int i = 0; i < k; ++i) tr += g[(size_t)s * kk + i * k + i];
        if (!(tr > tol * (*scale)[s])) broke[s] = vanished[s] = 1;
      }
    }
    for (int s = 0; s < e.nsec; ++s) {
      if (broke[s] || !cholesky_inverse(k, &g[(size_t)s * kk], &R[(size_t)s * kk], &inv[(size_t)s * kk], pivot_tol)) {
        broke[s] = 1;
        std::fill(&R[(size_t)s * kk], &R[(size_t)s * kk] + kk, 0.0);
        std::fill(&inv[(size_t)s * kk], &inv[(size_t)s * kk] + kk, 0.0);
      }
    }
    DH_CUDA(cudaMemcpyAsync(dM, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    if ((rc = launch_seg_rmul(x, dM, k, e.tiles, pass ? x32 : nullptr, e.stream)) != DH_OK) return rc;
    if (pass == 0 && inv1) *inv1 = inv;
    if (pass == 1 && inv2) *inv2 = inv;
    DH_CUDA(cudaStreamSynchronize(e.stream));  // inv is reused by the next pass
  }
  B.assign((size_t)e.nsec * kk, 0.0);
  for (int s = 0; s < e.nsec; ++s) {
    if (broke[s]) {
      if (!e.sec[s].exhausted) e.sec[s].partial = !vanished[s];
      e.sec[s].exhausted = true;
      continue;
    }
    const double* a = &R2[(size_t)s * kk];
    const double* b = &R1[(size_t)s * kk];
    for (int i = 0; i < k; ++i)
      for (int j = 0; j < k; ++j) {
        double v = 0.0;
        for (int p = 0; p < k; ++p) v += a[i * k + p] * b[p * k + j];
        B[(size_t)s * kk + i * k + j] = v;
      }
  }
  return DH_OK;
}

// y = H x; step = the block step the product belongs to (-1: outside the recurrence)
int engine_product(BlockEngine& e, const double* x, double* y, int step = -1) {
  const int saved = e.precision;
  if (step == 0 && e.fp64_first_product) e.precision = DH_PRECISION_FP64;
  const float* x32 = e.precision == DH_PRECISION_FP32 ? e.x32.as<float>() : nullptr;
  if (e.precision == DH_PRECISION_FP64) ++e.fp64_products;
  DH_CUDA(cudaEventRecord(e.ev0, e.stream));
  int rc = e.product(x, x32, y);
  e.precision = saved;
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaEventRecord(e.ev1, e.stream));
  DH_CUDA(cudaEventSynchronize(e.ev1));
  float ms = 0.0f;
  DH_CUDA(cudaEventElapsedTime(&ms, e.ev0, e.ev1));
  e.product_ms += ms;
  ++e.products;
  return DH_OK;
}

// orthonormalise the start block (slot 0) and prepare its FP32 copy

// the block store doubles (up to store_max blocks) when the next block would not fit; when the new
// size does not fit in half of the free memory, storing stops there and the Ritz vectors are rebuilt
// by replaying the recurrence instead
constexpr int kStoreBlocks = 32;  // blocks stored before the first growth

void store_grow(BlockEngine& e) {
  const int cap = std::min(e.store_max, std::max(2 * e.store_cap, e.store_cap + 1));
  const size_t block = (size_t)e.total * e.k * sizeof(double);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  DevBuf bigger;
  if ((size_t)cap * block >= free_b / 2 || bigger.alloc((size_t)cap * block) != DH_OK) {
    cudaGetLastError();
    e.store_max = e.store_cap;
    return;
  }
  if (cudaMemcpyAsync(bigger.ptr, e.store.ptr, (size_t)e.store_cap * block, cudaMemcpyDeviceToDevice, e.stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(e.stream) != cudaSuccess) {
    cudaGetLastError();
    e.store_max = e.store_cap;
    return;
  }
  std::swap(e.store.ptr, bigger.ptr);
  std::swap(e.store.bytes, bigger.bytes);
  e.store_cap = cap;
}
int engine_start(BlockEngine& e) {
  std::vector<double> B;
  e.slot_cur = 0;
  e.have_prev = false;
  e.issued = 0;
  if (e.dBt[0]) DH_CUDA(cudaMemsetAsync(e.dBt[0], 0, 2 * (size_t)e.nsec * e.k * e.k * sizeof(double), e.stream));
  int rc = engine_qr(e, e.slot[0], B, e.x32.as<float>(), nullptr);
  if (rc != DH_OK) return rc;
  const size_t vb = (size_t)e.total * e.k * sizeof(double);
  if ((rc = ensure_buffer(e.start_block, vb)) != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(e.start_block.ptr, e.slot[0], vb, cudaMemcpyDeviceToDevice, e.stream));
  if (e.store_cap > 0) DH_CUDA(cudaMemcpyAsync(e.store.ptr, e.slot[0], vb, cudaMemcpyDeviceToDevice, e.stream));
  e.history.clear();
  for (int s = 0; s < e.nsec; ++s) {
    BlockSector& b = e.sec[s];
    b.blocks = 0;
    b.steps = 0;
    b.A.clear();
    b.B.assign((size_t)e.k * e.k, 0.0);
    b.prev_last = 0.0;
    b.ritz.clear();
    b.converged = false;
    b.active = !b.exhausted;
  }
  return DH_OK;
}

// FP64 check of a block X holding each sector's Ritz vectors: Y = H X with FP64 products,
// E[s] = <x0|H x0> / <x0|x0> and r2[s] = |H x0 - E x0|^2 / |x0|^2 for the lowest vector x0 of every
// sector.  Y is left holding the residual block.
int engine_mask_all_active(BlockEngine& e);

int engine_fp64_check(BlockEngine& e, const double* X, double* Y, std::vector<double>& E, std::vector<double>& r2) {
  const int k = e.k, kk = k * k;
  int rc0 = engine_mask_all_active(e);
  if (rc0 != DH_OK) return rc0;
  const int saved = e.precision;
  e.precision = DH_PRECISION_FP64;
  int rc = engine_product(e, X, Y);
  e.precision = saved;
  if (rc != DH_OK) return rc;
  std::vector<double> g, a, rr;
  if ((rc = engine_gram(e, X, X, g)) != DH_OK) return rc;
  if ((rc = engine_gram(e, X, Y, a)) != DH_OK) return rc;
  std::vector<double> d((size_t)e.nsec * kk, 0.0);
  for (int s = 0; s < e.nsec; ++s)
    for (int c = 0; c < k; ++c)
      d[(size_t)s * kk + c * k + c] = a[(size_t)s * kk + c * k + c] / std::max(g[(size_t)s * kk + c * k + c], 1e-300);
  double* dA = e.small.as<double>() + 2 * (size_t)e.nsec * kk;
  DH_CUDA(cudaMemcpyAsync(dA, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
  if ((rc = launch_seg_update(Y, X, dA, nullptr, nullptr, k, e.tiles, e.stream)) != DH_OK) return rc;
  if ((rc = engine_gram(e, Y, Y, rr)) != DH_OK) return rc;
  E.assign(e.nsec, 0.0);
  r2.assign(e.nsec, 0.0);
  for (int s = 0; s < e.nsec; ++s) {
    E[s] = d[(size_t)s * kk];
    r2[s] = std::max(rr[(size_t)s * kk], 0.0) / std::max(g[(size_t)s * kk], 1e-300);
  }
  return DH_OK;
}

// Mixed-precision restart: the engine's start block becomes (lowest Ritz vector, fresh random
// vectors) per sector (already copied into slot 0 by the caller); its product is FP64, the
// following ones FP32, and every new block is projected against it.  The Krylov space is the one
// an FP64 restart would build; the FP32 products only touch directions whose coefficients in the
// refined ground state are of the order of the Ritz vector's residual.
// fp64: every product of the restart in FP64 (the last resort of the batched refinement)
int engine_mixed_restart(BlockEngine& e, uint64_t seed, bool fp64 = false) {
  int rc;
  if ((rc = launch_random_block(e.slot[0], e.total, e.k, e.row_offset_dev, e.tiles, seed, e.stream, 1)) != DH_OK)
    return rc;
  e.precision = fp64 ? DH_PRECISION_FP64 : DH_PRECISION_FP32;
  e.fp64_first_product = !fp64;
  e.lock_start = true;
  for (auto& b : e.sec) b.exhausted = b.partial = false;
  return engine_start(e);
}

// the residual target of a mixed restart aiming at |r|^2 <= precision |E| after the FP64 check
inline double restart_residual_target(double precision) { return 0.1 * precision; }

// the FP32 phase converges on the Ritz vector's residual too, down to the FP32 rounding floor of the
// products (|r| of a few 1e-6 relative): when the target lies above it, the FP64 check that follows
// passes without a restart
inline double fp32_phase_residual_target(double precision) { return std::max(0.1 * precision, 1e-11); }

// The device's active mask follows the sectors' active flags (finished sectors' product rows are
// zeroed instead of enumerated); uploaded from a pinned ring slot when it changes.
int engine_sync_active(BlockEngine& e) {
  if (!e.dActive) return DH_OK;
  bool changed = false;
  for (int s = 0; s < e.nsec; ++s) changed |= (e.mask_sent[s] != (e.sec[s].active ? 1 : 0));
  if (!changed) return DH_OK;
  int* m = e.mask_host + (size_t)(e.issued % EngineRing) * e.nsec;
  for (int s = 0; s < e.nsec; ++s) m[s] = e.mask_sent[s] = e.sec[s].active ? 1 : 0;
  DH_CUDA(cudaMemcpyAsync(e.dActive, m, (size_t)e.nsec * sizeof(int), cudaMemcpyHostToDevice, e.stream));
  return DH_OK;
}

// Products outside the recurrence (the FP64 check of Ritz blocks, the replay of recorded steps) cover
// every sector: the device mask is set to all active (and re-sent from the sectors' flags at the next
// issued step).
int engine_mask_all_active(BlockEngine& e) {
  if (!e.dActive) return DH_OK;
  bool all = true;
  for (int s = 0; s < e.nsec; ++s) all &= (e.mask_sent[s] == 1);
  if (all) return DH_OK;
  int* m = e.mask_host + (size_t)(e.issued % EngineRing) * e.nsec;
  for (int s = 0; s < e.nsec; ++s) m[s] = e.mask_sent[s] = 1;
  DH_CUDA(cudaMemcpyAsync(e.dActive, m, (size_t)e.nsec * sizeof(int), cudaMemcpyHostToDevice, e.stream));
  // the slot may be reused by the next issued step's mask: wait for this copy to have read it
  DH_CUDA(cudaStreamSynchronize(e.stream));
  return DH_OK;
}

// One block step for every sector, issued on the stream with no host synchronisation:
//   W = H V;  A = sym(V^T W);  W -= V A + V_prev B^T;  [W -= S (S^T W)];  CholQR2(W) -> B
// The per-sector matrices stay on the device; the step's coefficients and flags are copied to the
// record slot (step mod kRing) and an event marks them complete.  At most kRing - 1 steps may be in
// flight ahead of engine_process_step.
int engine_step_async(BlockEngine& e) {
  const int k = e.k;
  const long long step = e.issued;
  DH_CHECK(step - (long long)e.history.size() < EngineRing - 1, DH_ERR_STATE, "too many block steps in flight");
  const int slot = (int)(step % EngineRing);
  double* V = e.slot[e.slot_cur];
  double* W = e.slot[(e.slot_cur + 1) % 3];
  double* Vp = e.slot[(e.slot_cur + 2) % 3];
  const double* Bt = e.dBt[step & 1];
  double* Bt_next = e.dBt[(step + 1) & 1];
  int rc;
  if ((rc = engine_sync_active(e)) != DH_OK) return rc;
  // the product (FP64 for the start block of a mixed restart), timed by events read at processing
  const int saved = e.precision;
  if (step == 0 && e.fp64_first_product) e.precision = DH_PRECISION_FP64;
  const float* x32 = e.precision == DH_PRECISION_FP32 ? e.x32.as<float>() : nullptr;
  if (e.precision == DH_PRECISION_FP64) ++e.fp64_products;
  DH_CUDA(cudaEventRecord(e.ev_p0[slot], e.stream));
  rc = e.product(V, x32, W);
  e.precision = saved;
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaEventRecord(e.ev_p1[slot], e.stream));
  ++e.products;
  // A = sym(V^T W) and the step's scale |A|^2 + |B|^2; W -= V A + V_prev B^T
  if ((rc = launch_seg_gram(V, W, k, e.tiles, e.partial.as<double>(), e.dG, e.stream)) != DH_OK) return rc;
  if ((rc = launch_step_sym(e.dG, Bt, k, e.nsec, e.dA, e.dScale, e.stream)) != DH_OK) return rc;
  if ((rc = launch_seg_update(W, V, e.dA, e.have_prev ? Vp : nullptr, e.have_prev ? Bt : nullptr, k, e.tiles,
                              e.stream)) != DH_OK)
    return rc;
  // W -= S (S^T W) with S the start block: the FP32 products of the later blocks leave components
  // along S of the order of their rounding, which the recurrence alone would keep
  const bool locked = e.lock_start && step >= 1;
  if (locked) {
    if ((rc = launch_seg_gram(e.start_block.as<double>(), W, k, e.tiles, e.partial.as<double>(), e.dLock, e.stream)) !=
        DH_OK)
      return rc;
    if ((rc = launch_seg_update(W, e.start_block.as<double>(), e.dLock, nullptr, nullptr, k, e.tiles, e.stream)) != DH_OK)
      return rc;
  }
  // CholQR2: X = V B.  With FP32 products an exhausted Krylov space leaves FP32 rounding noise, not
  // zero: the vanishing and pivot thresholds are about (32 u)^2 of the product's precision.  A
  // sector whose block is numerically zero against its step's scale (the Krylov space is complete)
  // or whose Gram matrix breaks down gets a zero block and is flagged.
  const bool f32 = e.precision == DH_PRECISION_FP32;
  const double vanish_tol = f32 ? 4e-12 : 1e-24, pivot_tol = f32 ? 4e-12 : 1e-26;
  if ((rc = launch_seg_gram(W, W, k, e.tiles, e.partial.as<double>(), e.dG, e.stream)) != DH_OK) return rc;
  if ((rc = launch_step_chol(e.dG, k, e.nsec, 0, vanish_tol, pivot_tol, e.dScale, e.dR1, e.dInv1, e.dFlags, e.stream)) !=
      DH_OK)
    return rc;
  if ((rc = launch_seg_rmul(W, e.dInv1, k, e.tiles, nullptr, e.stream)) != DH_OK) return rc;
  if ((rc = launch_seg_gram(W, W, k, e.tiles, e.partial.as<double>(), e.dG, e.stream)) != DH_OK) return rc;
  if ((rc = launch_step_chol(e.dG, k, e.nsec, 1, vanish_tol, pivot_tol, nullptr, e.dR2, e.dInv2, e.dFlags, e.stream)) !=
      DH_OK)
    return rc;
  if ((rc = launch_seg_rmul(W, e.dInv2, k, e.tiles, e.x32.as<float>(), e.stream)) != DH_OK) return rc;
  if ((rc = launch_step_b(e.dR1, e.dR2, e.dFlags, k, e.nsec, e.dB, Bt_next, e.stream)) != DH_OK) return rc;
  // the step's record: A, the B^T it used, the two CholQR inverses, the lock coefficients, B, flags
  const size_t nk = (size_t)e.nsec * k * k, nb_ = nk * sizeof(double);
  double* rec = e.rec_host + (size_t)slot * 6 * nk;
  DH_CUDA(cudaMemcpyAsync(rec, e.dA, nb_, cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaMemcpyAsync(rec + nk, Bt, nb_, cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaMemcpyAsync(rec + 2 * nk, e.dInv1, nb_, cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaMemcpyAsync(rec + 3 * nk, e.dInv2, nb_, cudaMemcpyDeviceToHost, e.stream));
  if (locked) DH_CUDA(cudaMemcpyAsync(rec + 4 * nk, e.dLock, nb_, cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaMemcpyAsync(rec + 5 * nk, e.dB, nb_, cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaMemcpyAsync(e.rec_flags + (size_t)slot * e.nsec, e.dFlags, (size_t)e.nsec * sizeof(int),
                          cudaMemcpyDeviceToHost, e.stream));
  DH_CUDA(cudaEventRecord(e.ev_rec[slot], e.stream));
  e.rec_locked[slot] = locked;
  e.rec_have_prev[slot] = e.have_prev;
  // the block store (W is block step + 1)
  const long long nbk = step + 1;
  if (nbk >= e.store_cap && e.store_cap > 0 && e.store_cap < e.store_max) store_grow(e);
  if (nbk < e.store_cap)
    DH_CUDA(cudaMemcpyAsync(e.store.as<double>() + (size_t)nbk * e.total * e.k, W, (size_t)e.total * e.k * sizeof(double),
                            cudaMemcpyDeviceToDevice, e.stream));
  e.have_prev = true;
  e.slot_cur = (e.slot_cur + 1) % 3;
  ++e.issued;
  return DH_OK;
}

// The host's bookkeeping of the oldest issued step not yet processed: waits for its record, keeps
// its coefficients for replays, and appends A and B to every active sector (exhaustion from the
// device's flags and the counting rule).
int engine_process_step(BlockEngine& e) {
  const int k = e.k, kk = k * k;
  const long long step = (long long)e.history.size();
  DH_CHECK(step < e.issued, DH_ERR_STATE, "no block step in flight");
  const int slot = (int)(step % EngineRing);
  DH_CUDA(cudaEventSynchronize(e.ev_rec[slot]));
  float ms = 0.0f;
  DH_CUDA(cudaEventElapsedTime(&ms, e.ev_p0[slot], e.ev_p1[slot]));
  e.product_ms += ms;
  const size_t nk = (size_t)e.nsec * kk;
  const double* rec = e.rec_host + (size_t)slot * 6 * nk;
  const int* flags = e.rec_flags + (size_t)slot * e.nsec;
  StepRecord r;
  r.A.assign(rec, rec + nk);
  r.Bt.assign(rec + nk, rec + 2 * nk);
  r.inv1.assign(rec + 2 * nk, rec + 3 * nk);
  r.inv2.assign(rec + 3 * nk, rec + 4 * nk);
  if (e.rec_locked[slot]) r.lock.assign(rec + 4 * nk, rec + 5 * nk);
  r.have_prev = e.rec_have_prev[slot];
  e.history.push_back(std::move(r));
  const double* B = rec + 5 * nk;
  const double* A = e.history.back().A.data();
  for (int s = 0; s < e.nsec; ++s) {
    BlockSector& b = e.sec[s];
    if (!b.active) continue;
    const bool was_exhausted = b.exhausted;
    if (flags[s] & 1) {
      if (!b.exhausted) b.partial = !(flags[s] & 2);
      b.exhausted = true;
    }
    b.A.insert(b.A.end(), A + (size_t)s * kk, A + (size_t)(s + 1) * kk);
    b.B.insert(b.B.end(), B + (size_t)s * kk, B + (size_t)(s + 1) * kk);
    ++b.blocks;
    ++b.steps;
    // counting rule: once the blocks would outnumber the dimension the Krylov space is complete
    // (exact band matrix) or the new block has lost rank, whatever the rounding noise says
    if (!b.exhausted && (long long)(b.blocks + 1) * k > b.dim) {
      b.exhausted = true;
      b.partial = (long long)b.blocks * k < b.dim;
    }
    if (b.exhausted && !was_exhausted) b.converged = true;  // the Krylov space is complete
  }
  return DH_OK;
}

// one block step for every sector, its bookkeeping done before returning
int engine_step(BlockEngine& e) {
  int rc = engine_step_async(e);
  if (rc != DH_OK) return rc;
  return engine_process_step(e);
}

// the band matrix of sector s (blocks A_0..A_{m-1} on the diagonal, B_1..B_{m-1} below), dense
void sector_band_matrix(const BlockEngine& e, const BlockSector& b, std::vector<double>& t) {
  const int k = e.k, kk = k * k, m = b.blocks, n = m * k;
  t.assign((size_t)n * n, 0.0);
  for (int j = 0; j < m; ++j) {
    for (int p = 0; p < k; ++p)
      for (int q = 0; q < k; ++q) t[(size_t)(j * k + p) * n + j * k + q] = b.A[(size_t)j * kk + p * k + q];
    if (j + 1 < m)
      for (int p = 0; p < k; ++p)
        for (int q = 0; q < k; ++q) {
          const double v = b.B[(size_t)(j + 1) * kk + p * k + q];
          t[(size_t)((j + 1) * k + p) * n + j * k + q] = v;
          t[(size_t)(j * k + q) * n + (j + 1) * k + p] = v;
        }
  }
}

// eigenvalues of the band matrix of sector s (blocks A_0..A_{m-1}, B_1..B_{m-1})
int sector_eigenvalues(const BlockEngine& e, const BlockSector& b, std::vector<double>& eig) {
  const int k = e.k, kk = k * k, m = b.blocks, n = m * k;
  std::vector<double> t((size_t)n * n, 0.0);
  for (int j = 0; j < m; ++j) {
    for (int p = 0; p < k; ++p)
      for (int q = 0; q < k; ++q) t[(size_t)(j * k + p) * n + j * k + q] = b.A[(size_t)j * kk + p * k + q];
    if (j + 1 < m)
      for (int p = 0; p < k; ++p)
        for (int q = 0; q < k; ++q) {
          const double v = b.B[(size_t)(j + 1) * kk + p * k + q];
          t[(size_t)((j + 1) * k + p) * n + j * k + q] = v;
          t[(size_t)(j * k + q) * n + (j + 1) * k + p] = v;
        }
  }
  eig.assign(n, 0.0);
  return band_eigenvalues(n, std::max(1, 2 * k - 1), t.data(), eig.data());
}

// the nvec lowest eigenpairs of sector s's band matrix; C[(b * k + j) * nvec + c] = component
// (b k + j) of eigenvector c (the coefficients of the Ritz vectors in the Lanczos blocks)
int sector_ritz_coefficients(const BlockEngine& e, const BlockSector& b, int nvec, std::vector<double>& C,
                             std::vector<double>& vals) {
  const int k = e.k, kk = k * k, m = b.blocks, n = m * k;
  std::vector<double> t((size_t)n * n, 0.0);
  for (int j = 0; j < m; ++j) {
    for (int p = 0; p < k; ++p)
      for (int q = 0; q < k; ++q) t[(size_t)(j * k + p) * n + j * k + q] = b.A[(size_t)j * kk + p * k + q];
    if (j + 1 < m)
      for (int p = 0; p < k; ++p)
        for (int q = 0; q < k; ++q) {
          const double v = b.B[(size_t)(j + 1) * kk + p * k + q];
          t[(size_t)((j + 1) * k + p) * n + j * k + q] = v;
          t[(size_t)(j * k + q) * n + (j + 1) * k + p] = v;
        }
  }
  std::vector<double> z((size_t)n * n);
  vals.assign(n, 0.0);
  int rc = symmetric_eigen(n, t.data(), vals.data(), z.data());
  if (rc != DH_OK) return rc;
  C.assign((size_t)n * nvec, 0.0);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < nvec && c < n; ++c) C[(size_t)r * nvec + c] = z[(size_t)r * n + c];
  return DH_OK;
}

// The nvec lowest eigenvectors of a sector's band matrix as coefficients over its blocks
// (C[r * nvec + c]): the band's eigenvalues (Givens reduction and QL, O(n b^2)), then inverse iteration
// at each, orthogonalised against the lower ones and checked against T v = lambda v.  A failed check
// (a nearly degenerate cluster) falls back to the dense eigensolve.
int sector_lowest_vectors(const BlockEngine& e, const BlockSector& b, int nvec, std::vector<double>& C) {
  const int n = b.blocks * e.k;
  const int bw = std::max(1, 2 * e.k - 1);
  std::vector<double> t;
  sector_band_matrix(e, b, t);
  std::vector<double> work(t), eig(n), v(n);
  bool ok = band_eigenvalues(n, bw, work.data(), eig.data()) == DH_OK;
  C.assign((size_t)n * nvec, 0.0);
  for (int c = 0; ok && c < std::min(nvec, n); ++c) {
    if (band_inverse_iteration(n, bw, t.data(), eig[c], v.data()) != DH_OK) {
      ok = false;
      break;
    }
    for (int p = 0; p < c; ++p) {
      double d = 0.0;
      for (int i = 0; i < n; ++i) d += v[i] * C[(size_t)i * nvec + p];
      for (int i = 0; i < n; ++i) v[i] -= d * C[(size_t)i * nvec + p];
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += v[i] * v[i];
    nrm = sqrt(nrm);
    if (!(nrm > 1e-8)) {
      ok = false;
      break;
    }
    double res = 0.0;
    for (int i = 0; i < n; ++i) {
      v[i] /= nrm;
    }
    for (int i = 0; i < n; ++i) {
      double r = -eig[c] * v[i];
      for (int j = std::max(0, i - bw); j <= std::min(n - 1, i + bw); ++j) r += t[(size_t)i * n + j] * v[j];
      res += r * r;
    }
    if (!(res <= 1e-20 * std::max(1.0, eig[c] * eig[c]))) {
      ok = false;
      break;
    }
    for (int i = 0; i < n; ++i) C[(size_t)i * nvec + c] = v[i];
  }
  if (ok) return DH_OK;
  std::vector<double> vals;
  return sector_ritz_coefficients(e, b, nvec, C, vals);
}

// out = the k lowest Ritz vectors of every sector (k-interleaved like the blocks): from the stored
// blocks when they were kept, otherwise by replaying the recorded steps from the start block.
// After a replay the engine's work vectors hold the replayed state.
int engine_ritz(BlockEngine& e, double* out) {
  const int k = e.k, kk = k * k;
  int nb = 0;
  for (auto& b : e.sec) nb = std::max(nb, b.blocks);
  DH_CHECK(nb >= 1, DH_ERR_STATE, "no block step has been run");
  // per-sector coefficient matrices, padded to nb blocks: Cs[(b * k + j) * k + c]
  std::vector<double> C((size_t)e.nsec * nb * kk, 0.0);
  for (int s = 0; s < e.nsec; ++s) {
    const BlockSector& b = e.sec[s];
    if (b.blocks == 0) continue;
    std::vector<double> cs;
    int rc = sector_lowest_vectors(e, b, k, cs);
    if (rc != DH_OK) return rc;
    std::copy(cs.begin(), cs.end(), C.begin() + (size_t)s * nb * kk);
  }
  DevBuf dC;
  int rc;
  if ((rc = dC.alloc(C.size() * sizeof(double))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(dC.ptr, C.data(), C.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
  const long long stride = e.total * k;
  if (nb <= e.store_cap) {
    rc = launch_seg_combine_blocks(e.store.as<double>(), nb, stride, dC.as<double>(), nb * kk, k, e.tiles, out, e.stream);
    if (rc != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(e.stream));
    return DH_OK;
  }
  // replay: V_0 = start block; V_{j+1} = (H V_j - V_j A_j - V_{j-1} B_j^T) inv1_j inv2_j, every sector
  // enumerated (a sector's needed blocks came from steps where it was active)
  if ((rc = engine_mask_all_active(e)) != DH_OK) return rc;
  DH_CUDA(cudaMemsetAsync(out, 0, (size_t)stride * sizeof(double), e.stream));
  double* V = e.slot[0];
  double* W = e.slot[1];
  double* Vp = e.slot[2];
  DH_CUDA(cudaMemcpyAsync(V, e.start_block.ptr, (size_t)stride * sizeof(double), cudaMemcpyDeviceToDevice, e.stream));
  if (e.precision == DH_PRECISION_FP32 && (rc = launch_f32_copy(V, e.x32.as<float>(), stride, e.stream)) != DH_OK)
    return rc;
  DevBuf dm;
  if ((rc = dm.alloc((size_t)e.nsec * kk * 4 * sizeof(double))) != DH_OK) return rc;
  double* dNegC = dm.as<double>();
  double* dA = dNegC + (size_t)e.nsec * kk;
  double* dBt = dA + (size_t)e.nsec * kk;
  double* dInv = dBt + (size_t)e.nsec * kk;
  std::vector<double> negc((size_t)e.nsec * kk);
  for (int j = 0; j < nb; ++j) {
    // out += V_j C_j   (seg_update subtracts V * M, so M = -C_j)
    for (int s = 0; s < e.nsec; ++s)
      for (int i = 0; i < kk; ++i) negc[(size_t)s * kk + i] = -C[(size_t)s * nb * kk + (size_t)j * kk + i];
    DH_CUDA(cudaMemcpyAsync(dNegC, negc.data(), negc.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    if ((rc = launch_seg_update(out, V, dNegC, nullptr, nullptr, k, e.tiles, e.stream)) != DH_OK) return rc;
    if (j + 1 == nb) break;
    const StepRecord& h = e.history[j];
    if ((rc = engine_product(e, V, W, j)) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(dA, h.A.data(), h.A.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    DH_CUDA(cudaMemcpyAsync(dBt, h.Bt.data(), h.Bt.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    if ((rc = launch_seg_update(W, V, dA, h.have_prev ? Vp : nullptr, h.have_prev ? dBt : nullptr, k, e.tiles,
                                e.stream)) != DH_OK)
      return rc;
    if (!h.lock.empty()) {
      DH_CUDA(cudaStreamSynchronize(e.stream));
      DH_CUDA(cudaMemcpyAsync(dA, h.lock.data(), h.lock.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
      if ((rc = launch_seg_update(W, e.start_block.as<double>(), dA, nullptr, nullptr, k, e.tiles, e.stream)) != DH_OK)
        return rc;
    }
    DH_CUDA(cudaMemcpyAsync(dInv, h.inv1.data(), h.inv1.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    if ((rc = launch_seg_rmul(W, dInv, k, e.tiles, nullptr, e.stream)) != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(e.stream));
    DH_CUDA(cudaMemcpyAsync(dInv, h.inv2.data(), h.inv2.size() * sizeof(double), cudaMemcpyHostToDevice, e.stream));
    if ((rc = launch_seg_rmul(W, dInv, k, e.tiles, e.x32.as<float>(), e.stream)) != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(e.stream));
    double* t = Vp;
    Vp = V;
    V = W;
    W = t;
  }
  DH_CUDA(cudaStreamSynchronize(e.stream));
  return DH_OK;
}

// the reference's per-call bookkeeping (BasicBlockLanczosAlgorithm.cc:683-697) and TestConvergence
// (:731): first evaluation sets previous = 2 * lambda, later ones the previous lambda
int sector_evaluate(const BlockEngine& e, BlockSector& b) {
  std::vector<double> eig;
  int rc;
  if (e.lowest_only && e.k == 1) {
    // the lowest Ritz value only: Newton from the previous one (an upper bound by interlacing), or
    // bisection the first time
    const int m = b.blocks;
    std::vector<double> off(std::max(m - 1, 0));
    for (int j = 0; j + 1 < m; ++j) off[j] = b.B[j + 1];
    eig.assign(1, 0.0);
    rc = b.ritz.empty() ? tridiagonal_lowest(m, b.A.data(), off.data(), 1, eig.data())
                        : tridiagonal_lowest_below(m, b.A.data(), off.data(), b.ritz[0], eig.data());
  } else {
    rc = sector_eigenvalues(e, b, eig);
  }
  if (rc != DH_OK) return rc;
  const int nev = std::min(e.nev, (int)eig.size());
  if (b.prev_last != 0.0 && !b.ritz.empty())
    b.prev_last = b.ritz[std::min(nev, (int)b.ritz.size()) - 1];
  else
    b.prev_last = 2.0 * eig[nev - 1];
  b.ritz.swap(eig);
  if (e.residual_target > 0.0 && e.nev == 1) {
    // the residual needs the band matrix's eigenvector (a dense eigensolve on the host): only once
    // the Ritz value has settled to 1e-7, which any residual small enough to pass implies anyway
    const double l0 = b.ritz[0];
    if (!(fabs(l0 - b.prev_last) < 1e-7 * fabs(l0))) return DH_OK;
    // the lowest eigenvector of the band matrix by inverse iteration at the known l0
    std::vector<double> t, C((size_t)b.blocks * e.k);
    sector_band_matrix(e, b, t);
    const int n = b.blocks * e.k;
    rc = band_inverse_iteration(n, std::max(1, 2 * e.k - 1), t.data(), l0, C.data());
    // a nearly degenerate lowest pair (or a failed solve) leaves a mixed vector: check T s = l0 s,
    // else take the dense eigensolve's vector
    double res = 0.0, nrm = 0.0;
    if (rc == DH_OK)
      for (int i = 0; i < n; ++i) {
        double v = -l0 * C[i];
        for (int j = std::max(0, i - 2 * e.k); j <= std::min(n - 1, i + 2 * e.k); ++j) v += t[(size_t)i * n + j] * C[j];
        res += v * v;
        nrm += C[i] * C[i];
      }
    if (rc != DH_OK || !(res <= 1e-20 * std::max(1.0, l0 * l0) * nrm)) {
      std::vector<double> vals;
      if ((rc = sector_ritz_coefficients(e, b, 1, C, vals)) != DH_OK) return rc;
    }
    const int k = e.k, m = b.blocks;
    const double* Bm = &b.B[(size_t)m * k * k];  // X_m = V_m B_m: the block after the last A
    double r2 = 0.0;
    for (int i = 0; i < k; ++i) {
      double v = 0.0;
      for (int j = 0; j < k; ++j) v += Bm[i * k + j] * C[(size_t)((m - 1) * k + j)];
      r2 += v * v;
    }
    if (r2 < e.residual_target * fabs(b.ritz[0])) b.converged = true;
    // (FP32 phase) a Ritz value that no longer moves at all: the products' rounding floor is reached
    if (e.stop_on_stagnation && fabs(l0 - b.prev_last) < 1e-13 * fabs(l0)) b.converged = true;
    return DH_OK;
  }
  // the test needs more Ritz values than wanted ones (rows beyond nev); the lowest-only form keeps
  // just the wanted one and counts the rows instead
  if ((e.lowest_only && e.k == 1) ? b.blocks > e.nev : (int)b.ritz.size() > e.nev) {
    const double l = b.ritz[e.nev - 1];
    if (fabs(l - b.prev_last) < e.eig_precision * fabs(l)) b.converged = true;
  }
  return DH_OK;
}

// Run every active sector until converged, exhausted or at the iteration limit; the driver loop of
// QHEOnSphereMainTask.cc:732-753 per sector (first call nev + 2 block steps, counter (nev + 3) k).
// The device runs kStepLag steps ahead of the host: while step i's band matrices are diagonalised
// on the host (convergence), step i + 1 runs on the GPU.  A sector found finished at step i stops
// being enumerated from the next issued step on (its rows are zeroed); the steps issued past the
// last sector's stop are processed for the replay record and otherwise unused.
constexpr int kStepLag = 2;

int engine_solve(BlockEngine& e) {
  const int first = e.nev + 2;
  int rc;
  for (;;) {
    bool any = false;
    for (auto& b : e.sec) any |= b.active;
    if (!any) break;
    while (e.issued - (long long)e.history.size() < kStepLag)
      if ((rc = engine_step_async(e)) != DH_OK) return rc;
    if ((rc = engine_process_step(e)) != DH_OK) return rc;
    std::vector<int> eval;
    for (int s = 0; s < e.nsec; ++s) {
      BlockSector& b = e.sec[s];
      if (!b.active) continue;
      if (b.steps == first) {
        b.count = (e.nev + 3) * e.k;
        eval.push_back(s);
      } else if (b.steps > first || b.exhausted) {
        b.count += e.k;
        eval.push_back(s);
      }
    }
    // band eigenvalues of the sectors due, spread over host threads (a few microseconds per sector
    // with the lowest-only Newton steps of k = 1: then on this thread)
    std::vector<int> status(eval.size(), DH_OK);
    const int nthreads = (e.lowest_only && e.k == 1)
                             ? 1
                             : std::max(1, std::min((int)eval.size(), (int)std::thread::hardware_concurrency()));
    if (nthreads == 1) {
      for (size_t i = 0; i < eval.size(); ++i) status[i] = sector_evaluate(e, e.sec[eval[i]]);
    } else {
      std::vector<std::thread> pool;
      for (int t = 0; t < nthreads; ++t)
        pool.emplace_back([&, t] {
          for (size_t i = t; i < eval.size(); i += nthreads) status[i] = sector_evaluate(e, e.sec[eval[i]]);
        });
      for (auto& th : pool) th.join();
    }
    for (size_t i = 0; i < eval.size(); ++i) {
      if (status[i] != DH_OK) return status[i];
      BlockSector& b = e.sec[eval[i]];
      if (b.converged || b.exhausted || b.count >= e.max_iter) b.active = false;
    }
  }
  while ((long long)e.history.size() < e.issued)
    if ((rc = engine_process_step(e)) != DH_OK) return rc;
  return DH_OK;
}

}  // namespace

// ------------------------------------------------------------------ batched FQHE sectors

struct SectorBatchHost {
  std::vector<dh_space_s*> spaces;
  DevBuf ptrs;  // words and HO pointer arrays + row offsets
  DevBuf pair_offset, f64, f32;
  InteractionTables tabs;
  ~SectorBatchHost() {
    for (auto* s : spaces) delete s;
  }
};

// Dense FP64 spectrum of a small d x d Hamiltonian: H on the unit vectors, four columns per
// product (product4: y = H x on [d][4] device blocks), then a dense symmetric eigensolve on the
// host.  vals: all eigenvalues ascending; vecs (optional): the lowest nvec eigenvectors, [d][nvec].
int dense_spectrum(long long d, const std::function<int(const double*, double*)>& product4, int nvec,
                   std::vector<double>& vals, std::vector<double>* vecs, cudaStream_t stream) {
  const int k = 4;
  DevBuf x, y;
  int rc;
  if ((rc = x.alloc((size_t)d * k * sizeof(double))) != DH_OK || (rc = y.alloc((size_t)d * k * sizeof(double))) != DH_OK)
    return rc;
  std::vector<double> H((size_t)d * d), xin((size_t)d * k), yout((size_t)d * k);
  for (long long c0 = 0; c0 < d; c0 += k) {
    std::fill(xin.begin(), xin.end(), 0.0);
    for (int j = 0; j < k && c0 + j < d; ++j) xin[(size_t)(c0 + j) * k + j] = 1.0;
    DH_CUDA(cudaMemcpyAsync(x.ptr, xin.data(), xin.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    if ((rc = product4(x.as<double>(), y.as<double>())) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(yout.data(), y.ptr, yout.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    DH_CUDA(cudaStreamSynchronize(stream));
    for (int j = 0; j < k && c0 + j < d; ++j)
      for (long long r = 0; r < d; ++r) H[(size_t)r * d + c0 + j] = yout[(size_t)r * k + j];
  }
  for (long long r = 0; r < d; ++r)  // symmetrise the rounding of the two triangles
    for (long long c = r + 1; c < d; ++c) H[(size_t)r * d + c] = H[(size_t)c * d + r] = 0.5 * (H[(size_t)r * d + c] + H[(size_t)c * d + r]);
  vals.assign(d, 0.0);
  std::vector<double> z;
  if (vecs) z.resize((size_t)d * d);
  if ((rc = symmetric_eigen((int)d, H.data(), vals.data(), vecs ? z.data() : nullptr)) != DH_OK) return rc;
  if (vecs) {
    vecs->assign((size_t)d * nvec, 0.0);
    for (long long r = 0; r < d; ++r)
      for (int c = 0; c < nvec && c < d; ++c) (*vecs)[(size_t)r * nvec + c] = z[(size_t)r * d + c];
  }
  return DH_OK;
}

// the one-sector FP64 product of a batch's space, for dense_spectrum
int dense_lowest(dh_space_s* sp, const SectorBatchHost& hb, int nev, std::vector<double>& out, cudaStream_t stream) {
  const long long d = sp->dim;
  DevBuf ptrs;
  int rc;
  if ((rc = ptrs.alloc(2 * sizeof(void*) + 2 * sizeof(long long))) != DH_OK) return rc;
  const void* hp[2] = {sp->words.ptr, sp->high_offset.ptr};
  long long ho[2] = {0, d};
  DH_CUDA(cudaMemcpy(ptrs.ptr, hp, 2 * sizeof(void*), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(ptrs.as<char>() + 2 * sizeof(void*), ho, 2 * sizeof(long long), cudaMemcpyHostToDevice));
  SectorBatchDevice b = {};
  b.words = reinterpret_cast<const uint64_t* const*>(ptrs.ptr);
  b.high_offset = reinterpret_cast<const int32_t* const*>(ptrs.as<char>() + sizeof(void*));
  b.row_offset = reinterpret_cast<const long long*>(ptrs.as<char>() + 2 * sizeof(void*));
  b.low_rank = sp->low_rank.as<uint16_t>();
  b.pair_offset = hb.pair_offset.as<int32_t>();
  b.factors = hb.f64.ptr;
  b.total_rows = d;
  b.nbr_sectors = 1;
  b.block = 4;
  b.lz_max = sp->lz_max;
  b.low_bits = sp->rank.low_bits;
  b.nbr_pairs = hb.tabs.nbr_pairs;
  b.nbr_factors = hb.tabs.nbr_factors;
  auto product4 = [&b, stream](const double* x, double* y) {
    SectorBatchDevice c = b;
    c.x = x;
    c.y = y;
    return launch_fqhe_sectors(c, DH_PRECISION_FP64, stream);
  };
  std::vector<double> vals;
  if ((rc = dense_spectrum(d, product4, 0, vals, nullptr, stream)) != DH_OK) return rc;
  out.assign(vals.begin(), vals.begin() + std::min<long long>(d, std::max(nev, 1)));
  return DH_OK;
}

// ------------------------------------------------------------------ one Hamiltonian

// BasicBlockLanczosAlgorithm on one Hamiltonian: the engine with a single sector spanning the
// whole space, products through the Hamiltonian's own kernels on [dim][k] blocks.
struct BlockLanczos {
  dh_hamiltonian_s* h = nullptr;
  BlockEngine e;
  int nev = 1, k = 1, max_iter = 0;
  bool initialized = false;
  bool keep = true;        // keep every block on the device when they fit
  bool ritz_valid = false;
  DevBuf ritz;             // the k lowest Ritz vectors, [dim][k]
  DevBuf stage;            // one vector, for host input and output
  ~BlockLanczos() {
    if (e.stream) {
      cudaStreamSynchronize(e.stream);
      cudaStreamDestroy(e.stream);
    }
  }
};

namespace {

int bl_ensure_x32(BlockLanczos* b) {
  BlockEngine& e = b->e;
  return ensure_buffer(e.x32, (size_t)e.total * e.k * sizeof(float));
}

int bl_allocate_store(BlockLanczos* b) {
  BlockEngine& e = b->e;
  e.store.release();
  e.store_cap = 0;
  if (!b->keep) return DH_OK;
  const int cap_max = b->max_iter / b->k + 3;
  const int cap = std::min(cap_max, kStoreBlocks);
  const size_t bytes = (size_t)cap * e.total * e.k * sizeof(double);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  if (bytes < free_b / 2) {
    if (e.store.alloc(bytes) == DH_OK) {
      e.store_cap = cap;
      e.store_max = cap_max;
    } else {
      cudaGetLastError();
    }
  }
  return DH_OK;
}

// the reference's TestConvergence (BasicBlockLanczosAlgorithm.cc:731), or an exhausted Krylov space
bool bl_converged(const BlockLanczos* b) {
  const BlockSector& s = b->e.sec[0];
  if (s.exhausted && s.blocks > 0) return true;
  if (b->e.residual_target > 0.0) return s.converged;  // residual test of sector_evaluate
  if ((int)s.ritz.size() <= b->nev) return false;
  const double l = s.ritz[b->nev - 1];
  return fabs(l - s.prev_last) < b->e.eig_precision * fabs(l);
}

int bl_ritz_block(BlockLanczos* b) {
  if (b->ritz_valid) return DH_OK;
  BlockEngine& e = b->e;
  int rc;
  if ((rc = ensure_buffer(b->ritz, (size_t)e.total * e.k * sizeof(double))) != DH_OK) return rc;
  const bool replay = e.sec[0].blocks > e.store_cap;
  if ((rc = engine_ritz(e, b->ritz.as<double>())) != DH_OK) return rc;
  if (replay) b->initialized = false;  // the replay overwrote the work blocks
  b->ritz_valid = true;
  return DH_OK;
}

}  // namespace

int block_lanczos_create(dh_hamiltonian_s* h, int nev, int k, int max_iter, BlockLanczos** out) {
  *out = nullptr;
  DH_CHECK(k == 1 || k == 2 || k == 4, DH_ERR_UNSUPPORTED, "block size %d not in {1, 2, 4}", k);
  DH_CHECK(k == 1 || !h->complex_phases, DH_ERR_UNSUPPORTED, "complex vectors are multiplied one at a time");
  BlockLanczos* b = new (std::nothrow) BlockLanczos();
  DH_CHECK(b, DH_ERR_MEMORY, "out of host memory");
  b->h = h;
  b->nev = nev;
  b->k = k;
  b->max_iter = max_iter;
  BlockEngine& e = b->e;
  e.k = k;
  e.nev = nev;
  e.max_iter = max_iter;
  e.precision = h->precision;
  int rc = DH_OK;
  if (cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking) != cudaSuccess) {
    e.stream = 0;
    rc = cuda_fail(cudaGetLastError(), "cudaStreamCreate", __FILE__, __LINE__);
  }
  if (rc == DH_OK) rc = engine_setup(e, std::vector<long long>{(long long)hamiltonian_dim(h)});
  if (rc == DH_OK) rc = bl_allocate_store(b);
  if (rc != DH_OK) {
    delete b;
    return rc;
  }
  e.product = [b](const double* x64, const float* x32, double* y) {
    return hamiltonian_apply_block(b->h, x64, x32, y, b->k, b->e.precision, b->e.stream);
  };
  *out = b;
  return DH_OK;
}

void block_lanczos_destroy(BlockLanczos* b) { delete b; }

int block_lanczos_set_storage(BlockLanczos* b, int keep) {
  b->keep = keep != 0;
  b->initialized = false;
  b->ritz_valid = false;
  return bl_allocate_store(b);
}

void block_lanczos_set_precision(BlockLanczos* b, double precision) { b->e.eig_precision = precision; }

int block_lanczos_initialize(BlockLanczos* b, const double* vectors, int nbr_vectors, uint64_t seed) {
  BlockEngine& e = b->e;
  const long long dim = e.total;
  int rc;
  e.precision = b->h->precision;
  if (e.precision == DH_PRECISION_FP32 && (rc = bl_ensure_x32(b)) != DH_OK) return rc;
  if ((rc = launch_random_block(e.slot[0], dim, e.k, e.row_offset_dev, e.tiles, seed, e.stream)) != DH_OK) return rc;
  const int given = vectors ? std::min(nbr_vectors, e.k) : 0;
  for (int j = 0; j < given; ++j) {
    const double* src = vectors + (size_t)j * dim;
    if (!is_device_pointer(vectors)) {
      if ((rc = ensure_buffer(b->stage, (size_t)dim * sizeof(double))) != DH_OK) return rc;
      DH_CUDA(cudaMemcpyAsync(b->stage.ptr, src, (size_t)dim * sizeof(double), cudaMemcpyHostToDevice, e.stream));
      src = b->stage.as<double>();
    }
    if ((rc = launch_put_column(src, dim, e.k, j, e.slot[0], e.stream)) != DH_OK) return rc;
  }
  e.sec[0].exhausted = e.sec[0].partial = false;
  if ((rc = engine_start(e)) != DH_OK) return rc;
  DH_CHECK(!e.sec[0].exhausted, DH_ERR_ARGUMENT, "the start block is linearly dependent");
  b->initialized = true;
  b->ritz_valid = false;
  return DH_OK;
}

// RunLanczosAlgorithm(nbrIter) (BasicBlockLanczosAlgorithm.cc:524-697): nbrIter block steps, at least
// two on the first call, then the band matrix is diagonalised with the reference's bookkeeping
int block_lanczos_run(BlockLanczos* b, int nbr_iter) {
  DH_CHECK(b->initialized, DH_ERR_STATE, "RunLanczosAlgorithm before InitializeLanczosAlgorithm");
  BlockEngine& e = b->e;
  BlockSector& s = e.sec[0];
  DH_CHECK(!(s.exhausted && s.blocks > 0), DH_ERR_STATE, "the block Krylov space is exhausted (the result is exact)");
  if (e.precision == DH_PRECISION_FP32) DH_CHECK(e.x32.ptr, DH_ERR_STATE, "FP32 copy missing");
  int n = s.blocks == 0 ? std::max(nbr_iter, 2) : nbr_iter;
  int rc;
  for (int i = 0; i < n; ++i) {
    if ((rc = engine_step(e)) != DH_OK) return rc;
    if (s.exhausted) {
      s.active = false;
      break;
    }
  }
  b->ritz_valid = false;
  if ((rc = sector_evaluate(e, s)) != DH_OK) return rc;
  // an exhausted space is at most (blocks + 1) k vectors: when its band matrix is not exact (the
  // last block only lost rank, or the products were FP32) diagonalise H densely in FP64
  if (s.exhausted && (s.partial || e.precision == DH_PRECISION_FP32) && e.total <= kDenseFallbackLimit) {
    dh_hamiltonian_s* h = b->h;
    cudaStream_t st = e.stream;
    auto product4 = [h, st](const double* x, double* y) {
      return hamiltonian_apply_block(h, x, nullptr, y, 4, DH_PRECISION_FP64, st);
    };
    std::vector<double> vals, vecs;
    if ((rc = dense_spectrum(e.total, product4, e.k, vals, &vecs, st)) != DH_OK) return rc;
    if ((rc = ensure_buffer(b->ritz, (size_t)e.total * e.k * sizeof(double))) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(b->ritz.ptr, vecs.data(), vecs.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    DH_CUDA(cudaStreamSynchronize(st));
    b->ritz_valid = true;
    s.prev_last = s.ritz.empty() ? 0.0 : s.ritz[std::min(b->nev, (int)s.ritz.size()) - 1];
    s.ritz = vals;
    s.converged = true;
  }
  return DH_OK;
}

bool block_lanczos_converged(const BlockLanczos* b) { return bl_converged(b); }

const std::vector<double>& block_lanczos_ritz(const BlockLanczos* b) { return b->e.sec[0].ritz; }

int block_lanczos_eigenstates(BlockLanczos* b, int n, double* out) {
  BlockEngine& e = b->e;
  DH_CHECK(n >= 1 && n <= e.k, DH_ERR_ARGUMENT, "%d eigenstates asked of a block of %d", n, e.k);
  DH_CHECK(e.sec[0].blocks >= 1, DH_ERR_STATE, "no Lanczos iteration has been run");
  int rc;
  if ((rc = bl_ritz_block(b)) != DH_OK) return rc;
  std::vector<double> g;
  if ((rc = engine_gram(e, b->ritz.as<double>(), b->ritz.as<double>(), g)) != DH_OK) return rc;
  const long long dim = e.total;
  const bool dev = is_device_pointer(out);
  if (!dev && (rc = ensure_buffer(b->stage, (size_t)dim * sizeof(double))) != DH_OK) return rc;
  for (int c = 0; c < n; ++c) {
    const double nrm = sqrt(g[(size_t)c * e.k + c]);
    DH_CHECK(nrm > 0.0, DH_ERR_STATE, "Ritz vector %d vanishes", c);
    double* dst = dev ? out + (size_t)c * dim : b->stage.as<double>();
    if ((rc = launch_get_column(b->ritz.as<double>(), dim, e.k, c, 1.0 / nrm, dst, e.stream)) != DH_OK) return rc;
    if (!dev)
      DH_CUDA(cudaMemcpyAsync(out + (size_t)c * dim, dst, (size_t)dim * sizeof(double), cudaMemcpyDeviceToHost, e.stream));
    DH_CUDA(cudaStreamSynchronize(e.stream));
  }
  return DH_OK;
}

void block_lanczos_counters(const BlockLanczos* b, int64_t* products, int* rows) {
  if (products) *products = b->e.products * b->k;
  if (rows) *rows = b->e.sec[0].blocks * b->k;
}

// the driver loop of QHEOnSphereMainTask.cc:732-753 with a block algorithm: RunLanczosAlgorithm
// (nev + 2), counter (nev + 3) k, then RunLanczosAlgorithm(1) and k more until converged
int block_lanczos_solve(BlockLanczos* b, int max_iter, double* eigenvalues, int* iterations, int* converged) {
  DH_CHECK(b->initialized, DH_ERR_STATE, "solve before InitializeLanczosAlgorithm");
  if (max_iter > b->max_iter) max_iter = b->max_iter;
  int rc = block_lanczos_run(b, b->nev + 2);
  if (rc != DH_OK) return rc;
  int count = (b->nev + 3) * b->k;
  while (!bl_converged(b) && count < max_iter) {
    count += b->k;
    if ((rc = block_lanczos_run(b, 1)) != DH_OK) return rc;
  }
  const std::vector<double>& r = b->e.sec[0].ritz;
  for (int i = 0; i < b->nev; ++i) eigenvalues[i] = i < (int)r.size() ? r[i] : NAN;
  *iterations = count;
  *converged = bl_converged(b) ? 1 : 0;
  return DH_OK;
}

// FP32 products with the FP64 block recurrence to the FP32 resolution of the Ritz values, then the
// Ritz block's FP64 Rayleigh quotients and residuals; while |r_0|^2 > precision |E_0| an FP64 block
// Lanczos restarted from the Ritz block polishes the energy.
int block_lanczos_solve_refined(BlockLanczos* b, int max_iter, double precision, double* out) {
  BlockEngine& e = b->e;
  DH_CHECK(b->initialized && e.sec[0].blocks == 0, DH_ERR_STATE, "refined solve needs a freshly initialised algorithm");
  const double saved_precision = e.eig_precision;
  const long long dim = e.total;
  const int k = e.k;
  int rc;
  if ((rc = bl_ensure_x32(b)) != DH_OK) return rc;
  e.precision = DH_PRECISION_FP32;
  e.fp64_first_product = e.lock_start = false;
  const long long products0 = e.products, fp64_0 = e.fp64_products;
  if ((rc = launch_f32_copy(e.slot[e.slot_cur], e.x32.as<float>(), dim * k, e.stream)) != DH_OK) return rc;
  e.eig_precision = std::max(precision, 1e-9);
  e.residual_target = fp32_phase_residual_target(precision);
  std::vector<double> eig(b->nev);
  int iters = 0, conv = 0;
  rc = block_lanczos_solve(b, max_iter, eig.data(), &iters, &conv);
  e.residual_target = 0.0;
  const double e32 = eig[0];
  if (rc == DH_OK) rc = bl_ritz_block(b);
  double energy = e32, rnorm = 0.0;
  std::vector<double> E, r2;
  for (int round = 0; rc == DH_OK; ++round) {
    // FP64 Rayleigh quotient and residual of the lowest Ritz vector
    if ((rc = engine_fp64_check(e, b->ritz.as<double>(), e.slot[(e.slot_cur + 1) % 3], E, r2)) != DH_OK) break;
    energy = E[0];
    rnorm = sqrt(r2[0]);
    if (r2[0] <= precision * std::max(fabs(energy), 1e-300) || round == 3) break;
    DH_CUDA(cudaMemcpyAsync(e.slot[0], b->ritz.ptr, (size_t)dim * k * sizeof(double), cudaMemcpyDeviceToDevice, e.stream));
    if ((rc = engine_mixed_restart(e, 1000 + round)) != DH_OK) break;
    b->initialized = true;
    b->ritz_valid = false;
    e.eig_precision = precision;
    e.residual_target = restart_residual_target(precision);
    if ((rc = block_lanczos_solve(b, std::min(max_iter, 100 * k), eig.data(), &iters, &conv)) != DH_OK) break;
    rc = bl_ritz_block(b);
  }
  e.fp64_first_product = e.lock_start = false;
  e.residual_target = 0.0;
  e.precision = b->h->precision;
  e.eig_precision = saved_precision;
  if (rc != DH_OK) return rc;
  out[0] = energy;
  out[1] = e32;
  out[2] = rnorm;
  out[3] = (double)((e.products - products0 - (e.fp64_products - fp64_0)) * k);
  out[4] = (double)((e.fp64_products - fp64_0) * k);
  return DH_OK;
}


// The one-launch product over a list of sectors of hb (their rows concatenated in list order); the
// factor table follows the engine's current precision.
struct SectorProduct {
  DevBuf ptrs;
  SectorBatchDevice b = {};
};

int bind_sector_product(SectorBatchHost& hb, const std::vector<int>& sectors, BlockEngine& e, SectorProduct& sp) {
  const int ns = (int)sectors.size();
  int rc;
  if ((rc = sp.ptrs.alloc(2 * ns * sizeof(void*))) != DH_OK) return rc;
  std::vector<const void*> hp(2 * ns);
  for (int i = 0; i < ns; ++i) {
    hp[i] = hb.spaces[sectors[i]]->words.ptr;
    hp[ns + i] = hb.spaces[sectors[i]]->high_offset.ptr;
  }
  DH_CUDA(cudaMemcpy(sp.ptrs.ptr, hp.data(), hp.size() * sizeof(void*), cudaMemcpyHostToDevice));
  SectorBatchDevice& b = sp.b;
  b.words = reinterpret_cast<const uint64_t* const*>(sp.ptrs.ptr);
  b.high_offset = reinterpret_cast<const int32_t* const*>(sp.ptrs.as<char>() + ns * sizeof(void*));
  b.row_offset = e.row_offset_dev;
  b.low_rank = hb.spaces[sectors[0]]->low_rank.as<uint16_t>();
  b.pair_offset = hb.pair_offset.as<int32_t>();
  b.total_rows = e.total;
  b.nbr_sectors = ns;
  b.block = e.k;
  b.lz_max = hb.spaces[sectors[0]]->lz_max;
  b.low_bits = hb.spaces[sectors[0]]->rank.low_bits;
  b.nbr_pairs = hb.tabs.nbr_pairs;
  b.nbr_factors = hb.tabs.nbr_factors;
  SectorBatchDevice* bp = &sp.b;
  SectorBatchHost* hbp = &hb;
  BlockEngine* ep = &e;
  e.product = [bp, hbp, ep](const double* x64, const float* x32, double* y) {
    SectorBatchDevice c = *bp;
    const bool f32 = ep->precision == DH_PRECISION_FP32;
    c.factors = f32 ? hbp->f32.ptr : hbp->f64.ptr;
    c.x = f32 ? static_cast<const void*>(x32) : static_cast<const void*>(x64);
    c.xdiag = f32 ? x64 : nullptr;
    c.y = y;
    c.active = ep->dActive;
    return launch_fqhe_sectors(c, ep->precision, ep->stream);
  };
  return DH_OK;
}

// Stored elements over the concatenated rows of the batched sectors (the batch's
// EnableFastMultiplication, AbstractQHEOnSphereHamiltonian.cc:3625,3814): one sliced ELL in the
// engine's row order, every sector's targets shifted by its row offset, the factor indices of the
// shared interaction and one diagonal per row.  Products then stream it instead of enumerating the
// moves; the rows of converged sectors are skipped as in the on-the-fly kernel.
struct SectorEll {
  DevBuf slice_ptr, slice_len, cols, coef, diag64, diag32;
  size_t bytes = 0;
  int chunk = 16;
};

// built when it needs at most allowed_memory bytes (< 0: no budget) and fits in nine tenths of the
// free device memory; *bytes_needed = its size either way
int build_sector_ell(SectorBatchHost& hb, const std::vector<int>& sectors, const BlockEngine& e, int64_t allowed_memory,
                     SectorEll& ell, bool* built, size_t* bytes_needed) {
  *built = false;
  *bytes_needed = 0;
  const long long total = e.total;
  const int ns = (int)sectors.size();
  DH_CHECK(total < (1ll << 31), DH_ERR_UNSUPPORTED, "stored elements hold int32 targets");
  DH_CHECK(hb.tabs.nbr_factors < 0x8000, DH_ERR_UNSUPPORTED, "%d interaction factors do not fit 15-bit indices",
           hb.tabs.nbr_factors);
  auto device_of = [&](int i) {
    FqheDevice f = fqhe_device(hb.spaces[sectors[i]], nullptr, DH_PRECISION_FP64);
    f.pair_offset = hb.pair_offset.as<int32_t>();
    f.factors = hb.f64.ptr;
    f.nbr_pairs = hb.tabs.nbr_pairs;
    f.nbr_factors = hb.tabs.nbr_factors;
    return f;
  };
  int rc;
  std::vector<int> counts(total);
  {
    DevBuf dcounts;
    if ((rc = dcounts.alloc((size_t)total * sizeof(int))) != DH_OK) return rc;
    for (int i = 0; i < ns; ++i)
      if ((rc = launch_fqhe_row_counts(device_of(i), dcounts.as<int>(), e.stream, e.off[i])) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(counts.data(), dcounts.ptr, (size_t)total * sizeof(int), cudaMemcpyDeviceToHost, e.stream));
    DH_CUDA(cudaStreamSynchronize(e.stream));
  }
  const long long nslices = (total + 31) / 32;
  std::vector<long long> slice_ptr(nslices);
  std::vector<int> slice_len(nslices);
  long long elems = 0;
  for (long long sl = 0; sl < nslices; ++sl) {
    int mx = 0;
    for (long long r = sl * 32; r < std::min(total, sl * 32 + 32); ++r) mx = std::max(mx, counts[r]);
    mx = (mx + kEllPad - 1) / kEllPad * kEllPad;
    slice_ptr[sl] = elems;
    slice_len[sl] = mx;
    elems += 32ll * mx;
  }
  const size_t need = (size_t)elems * (sizeof(int) + sizeof(uint16_t)) + (size_t)nslices * (sizeof(long long) + sizeof(int)) +
                      (size_t)total * (sizeof(double) + sizeof(float));
  *bytes_needed = need;
  if (allowed_memory >= 0 && need > (size_t)allowed_memory) return DH_OK;
  size_t free_b = 0, total_b = 0;
  DH_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (need > free_b / 10 * 9) return DH_OK;
  if ((rc = ell.slice_ptr.alloc((size_t)nslices * sizeof(long long))) != DH_OK ||
      (rc = ell.slice_len.alloc((size_t)nslices * sizeof(int))) != DH_OK ||
      (rc = ell.cols.alloc((size_t)elems * sizeof(int))) != DH_OK ||
      (rc = ell.coef.alloc((size_t)elems * sizeof(uint16_t))) != DH_OK ||
      (rc = ell.diag64.alloc((size_t)total * sizeof(double))) != DH_OK ||
      (rc = ell.diag32.alloc((size_t)total * sizeof(float))) != DH_OK)
    return rc;
  DH_CUDA(cudaMemcpyAsync(ell.slice_ptr.ptr, slice_ptr.data(), nslices * sizeof(long long), cudaMemcpyHostToDevice,
                          e.stream));
  DH_CUDA(cudaMemcpyAsync(ell.slice_len.ptr, slice_len.data(), nslices * sizeof(int), cudaMemcpyHostToDevice, e.stream));
  for (int i = 0; i < ns; ++i) {
    const FqheDevice f = device_of(i);
    if ((rc = launch_fqhe_ell_fill(f, ell.slice_ptr.as<long long>(), ell.slice_len.as<int>(), ell.cols.as<int>(),
                                   ell.coef.as<uint16_t>(), e.stream, e.off[i])) != DH_OK ||
        (rc = launch_fqhe_diag(f, hb.f64.as<double>(), ell.diag64.as<double>(), ell.diag32.as<float>(), e.stream,
                               e.off[i])) != DH_OK)
      return rc;
  }
  DH_CUDA(cudaStreamSynchronize(e.stream));
  ell.bytes = need;
  *built = true;
  return DH_OK;
}

// the engine's products from the stored elements
void bind_sector_ell(SectorBatchHost& hb, SectorEll& ell, BlockEngine& e) {
  SectorBatchHost* hbp = &hb;
  SectorEll* lp = &ell;
  BlockEngine* ep = &e;
  e.product = [hbp, lp, ep](const double* x64, const float* x32, double* y) {
    const bool f32 = ep->precision == DH_PRECISION_FP32;
    EllDevice d = {};
    d.slice_ptr = lp->slice_ptr.as<long long>();
    d.slice_len = lp->slice_len.as<int>();
    d.cols = lp->cols.as<int>();
    d.coef = lp->coef.as<uint16_t>();
    d.payload = 0;
    d.diag = f32 ? lp->diag32.ptr : lp->diag64.ptr;
    d.factors = f32 ? hbp->f32.ptr : hbp->f64.ptr;
    d.dim = ep->total;
    d.nbr_factors = hbp->tabs.nbr_factors;
    d.chunk = lp->chunk;
    d.active = ep->dActive;
    d.sector_offset = ep->row_offset_dev;
    d.nbr_sectors = ep->nsec;
    MatvecArgs a = {};
    a.x = f32 ? static_cast<const void*>(x32) : static_cast<const void*>(x64);
    a.xdiag = f32 ? x64 : nullptr;
    a.y = y;
    a.ld = ep->k;
    a.vstride = 1;
    a.ld_y = ep->k;
    a.vstride_y = 1;
    a.nbr_vectors = ep->k;
    a.col_first = 0;
    a.col_last = ep->total;
    a.row_first = 0;
    a.row_last = ep->total;
    return launch_ell_product(d, a, ep->precision, ep->stream);
  };
}

// keep every block on the device when the store fits in half of the free memory
// the first kStoreBlocks blocks (or all of max_iter / k + 3, when fewer) in half of the free memory;
// the store then grows with the run
void engine_store_if_fits(BlockEngine& e) {
  const int cap_max = e.max_iter / e.k + 3;
  const int cap = std::min(cap_max, kStoreBlocks);
  const size_t bytes = (size_t)cap * e.total * e.k * sizeof(double);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  if (bytes < free_b / 2) {
    if (e.store.alloc(bytes) == DH_OK) {
      e.store_cap = cap;
      e.store_max = cap_max;
    } else {
      cudaGetLastError();
    }
  }
}

}  // namespace dh

extern "C" int dh_fqhe_sectors_block_lanczos(int nbr_fermions, int lz_max, const int* total_lz, int nbr_sectors,
                                             const double* pseudopotentials, int block_size, int max_iter,
                                             double precision_target, int precision, int full_diag_limit,
                                             int64_t allowed_memory, uint64_t seed, double* energies,
                                             int* iterations, double* stats) {
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  DH_CHECK(total_lz && pseudopotentials && energies && iterations && nbr_sectors >= 1, DH_ERR_ARGUMENT, "bad argument");
  DH_CHECK(block_size == 1 || block_size == 2 || block_size == 4, DH_ERR_UNSUPPORTED, "block size must be 1, 2 or 4");
  DH_CHECK(precision == DH_PRECISION_FP64 || precision == DH_PRECISION_FP32, DH_ERR_ARGUMENT, "unknown precision");
  SectorBatchHost hb;
  BlockEngine e;
  SectorEll ell;  // stored elements of the batch (allowed_memory != 0), destroyed before the engine
  size_t ell_bytes = 0;
  double ell_seconds = 0.0;
  e.k = block_size;
  e.nev = 1;
  e.lowest_only = true;
  e.precision = precision;
  e.eig_precision = precision_target > 0.0 ? precision_target : 1e-14;
  e.max_iter = max_iter;
  int rc;
  // spaces (each builds its words and rank tables on the device)
  std::vector<int> lanczos_sectors, dense_sectors;
  std::vector<long long> dims;
  for (int s = 0; s < nbr_sectors; ++s) {
    dh_space_t sp = nullptr;
    rc = dh_fermion_on_sphere_create(nbr_fermions, total_lz[s], lz_max, 9ul << 20, &sp);
    if (rc != DH_OK) return rc;
    hb.spaces.push_back(sp);
    DH_CHECK(sp->kind == SPACE_FERMION, DH_ERR_UNSUPPORTED,
             "batched sectors use the split-word rank tables (lz_max <= 40), not lz_max = %d", lz_max);
    DH_CHECK(sp->rank.low_bits == hb.spaces[0]->rank.low_bits, DH_ERR_STATE, "sectors disagree on the table split");
    if (sp->dim <= full_diag_limit || sp->dim <= 2 * block_size)
      dense_sectors.push_back(s);
    else {
      lanczos_sectors.push_back(s);
      dims.push_back(sp->dim);
    }
  }
  hb.tabs.build(lz_max);
  std::vector<double> v(pseudopotentials, pseudopotentials + lz_max + 1);
  hb.tabs.set_pseudopotentials(v.data());
  std::vector<float> f32(hb.tabs.nbr_factors);
  for (int i = 0; i < hb.tabs.nbr_factors; ++i) f32[i] = (float)hb.tabs.factors[i];
  if ((rc = hb.pair_offset.alloc(hb.tabs.pair_offset.size() * sizeof(int32_t))) != DH_OK ||
      (rc = hb.f64.alloc(hb.tabs.nbr_factors * sizeof(double))) != DH_OK ||
      (rc = hb.f32.alloc(hb.tabs.nbr_factors * sizeof(float))) != DH_OK)
    return rc;
  DH_CUDA(cudaMemcpy(hb.pair_offset.ptr, hb.tabs.pair_offset.data(), hb.tabs.pair_offset.size() * sizeof(int32_t),
                     cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(hb.f64.ptr, hb.tabs.factors.data(), hb.tabs.nbr_factors * sizeof(double), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(hb.f32.ptr, f32.data(), hb.tabs.nbr_factors * sizeof(float), cudaMemcpyHostToDevice));
  DH_CUDA(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      if (s) cudaStreamDestroy(s);
    }
  } guard{e.stream};
  const auto t1 = clk::now();
  // dense sectors
  for (int s : dense_sectors) {
    std::vector<double> ev;
    if ((rc = dense_lowest(hb.spaces[s], hb, 1, ev, e.stream)) != DH_OK) return rc;
    energies[s] = ev[0];
    iterations[s] = 0;
  }
  double fp32_seconds = 0.0, refine_seconds = 0.0, max_shift = 0.0, dense_seconds = 0.0;
  int refined = 0, dense_fallback = 0;
  long long products = 0;
  double product_ms = 0.0;
  if (!lanczos_sectors.empty()) {
    const auto ta = clk::now();
    e.eig_precision = precision == DH_PRECISION_FP32 ? std::max(e.eig_precision, 1e-9) : e.eig_precision;
    // the FP32 phase stops on each sector's Ritz residual (from its band matrix) rather than on the
    // Ritz value's change, so that the FP64 check after it passes without a restart
    if (precision == DH_PRECISION_FP32) {
      e.residual_target = fp32_phase_residual_target(precision_target > 0.0 ? precision_target : 1e-14);
      e.stop_on_stagnation = true;
    }
    if ((rc = engine_setup(e, dims)) != DH_OK) return rc;
    if (precision == DH_PRECISION_FP32) engine_store_if_fits(e);
    SectorProduct prod;
    if ((rc = bind_sector_product(hb, lanczos_sectors, e, prod)) != DH_OK) return rc;
    if (allowed_memory != 0) {
      const auto ts = clk::now();
      bool built = false;
      size_t need = 0;
      if ((rc = build_sector_ell(hb, lanczos_sectors, e, allowed_memory, ell, &built, &need)) != DH_OK) return rc;
      if (built) {
        bind_sector_ell(hb, ell, e);
        ell_bytes = ell.bytes;
      }
      ell_seconds = std::chrono::duration<double>(clk::now() - ts).count();
    }
    const int ns = (int)lanczos_sectors.size();
    // start block: splitmix64 vectors per sector (seed + j for vector j)
    if ((rc = launch_random_block(e.slot[0], e.total, e.k, e.row_offset_dev, e.tiles, seed, e.stream)) != DH_OK)
      return rc;
    if ((rc = engine_start(e)) != DH_OK) return rc;
    if ((rc = engine_solve(e)) != DH_OK) return rc;
    for (int i = 0; i < ns; ++i) {
      const BlockSector& bs = e.sec[i];
      energies[lanczos_sectors[i]] = bs.ritz.empty() ? NAN : bs.ritz[0];
      iterations[lanczos_sectors[i]] = bs.count;
    }
    products += e.products;
    product_ms += e.product_ms;
    // exhausted sectors whose band matrix is not exact (rank lost in the last block) are small: with
    // FP64 products they are diagonalised densely in FP64 at the end; with FP32 products the FP64
    // check of the refinement decides, and only a sector it cannot certify goes dense
    std::vector<char> need_dense(ns, 0);
    for (int i = 0; i < ns; ++i)
      need_dense[i] = precision == DH_PRECISION_FP64 && e.sec[i].exhausted && e.sec[i].partial &&
                      e.sec[i].dim <= kDenseFallbackLimit;
    const auto tb = clk::now();
    fp32_seconds = precision == DH_PRECISION_FP32 ? std::chrono::duration<double>(tb - ta).count() : 0.0;
    if (precision == DH_PRECISION_FP32) {
      // refinement rounds: FP64 Rayleigh quotient and residual of every pending sector's lowest
      // Ritz vector; the sectors above the target restart (mixed precision) from it, in lockstep
      const int k = e.k;
      products = e.products;
      product_ms = e.product_ms;
      std::vector<int> pending;  // positions in lanczos_sectors
      for (int i = 0; i < ns; ++i)
        if (!need_dense[i]) pending.push_back(i);
      BlockEngine* src = &e;            // engine holding the pending sectors' Ritz blocks
      std::vector<int> src_pos(ns, -1);  // position of a lanczos sector inside src
      for (int i = 0; i < ns; ++i) src_pos[i] = i;
      std::unique_ptr<BlockEngine> cur;
      std::unique_ptr<SectorProduct> cur_prod;
      std::unique_ptr<SectorEll> cur_ell;  // the restarted sectors' stored elements (a stored batch)
      DevBuf R;
      for (int round = 0; !pending.empty(); ++round) {
        if ((rc = ensure_buffer(R, (size_t)src->total * k * sizeof(double))) != DH_OK) return rc;
        if ((rc = engine_ritz(*src, R.as<double>())) != DH_OK) return rc;
        std::vector<double> E, r2;
        if ((rc = engine_fp64_check(*src, R.as<double>(), src->slot[0], E, r2)) != DH_OK) return rc;
        std::vector<int> redo;
        for (int i : pending) {
          const int p = src_pos[i];
          const int s = lanczos_sectors[i];
          max_shift = std::max(max_shift, fabs(E[p] - energies[s]));
          energies[s] = E[p];
          if (r2[p] > precision_target * std::max(fabs(E[p]), 1e-300)) redo.push_back(i);
        }
        if (src != &e) {
          products += src->products;
          product_ms += src->product_ms;
        } else {
          products = e.products;
          product_ms = e.product_ms;
        }
        if (round == 0) refined = (int)redo.size();
        if (redo.empty()) break;
        if (round == 4) {
          // not certified after the FP64 restart either: small sectors are diagonalised densely
          for (int i : redo)
            if (e.sec[i].dim <= kDenseFallbackLimit) need_dense[i] = 1;
          break;
        }
        // rounds 0-2 restart with FP32 products after an FP64 first one; a sector still above the
        // target after them restarts with FP64 products throughout
        const bool fp64_round = round == 3;
        auto f = std::make_unique<BlockEngine>();
        f->k = k;
        f->nev = 1;
        f->lowest_only = true;
        f->precision = fp64_round ? DH_PRECISION_FP64 : DH_PRECISION_FP32;
        f->eig_precision = precision_target > 0.0 ? precision_target : 1e-14;
        f->residual_target = restart_residual_target(f->eig_precision);
        f->max_iter = std::min(max_iter, 100 * k);
        f->stream = e.stream;
        std::vector<long long> rdims;
        std::vector<int> rsec;
        for (int i : redo) {
          rdims.push_back(e.sec[i].dim);
          rsec.push_back(lanczos_sectors[i]);
        }
        if ((rc = engine_setup(*f, rdims)) != DH_OK) return rc;
        engine_store_if_fits(*f);
        for (size_t jj = 0; jj < redo.size(); ++jj)
          DH_CUDA(cudaMemcpyAsync(f->slot[0] + (size_t)f->off[jj] * k, R.as<double>() + (size_t)src->off[src_pos[redo[jj]]] * k,
                                  (size_t)rdims[jj] * k * sizeof(double), cudaMemcpyDeviceToDevice, f->stream));
        auto fprod = std::make_unique<SectorProduct>();
        if ((rc = bind_sector_product(hb, rsec, *f, *fprod)) != DH_OK) return rc;
        std::unique_ptr<SectorEll> fell;
        if (ell_bytes > 0) {
          // a stored batch stores the restarted sectors too (their rows at the restart's offsets)
          fell = std::make_unique<SectorEll>();
          bool built = false;
          size_t need = 0;
          if ((rc = build_sector_ell(hb, rsec, *f, allowed_memory, *fell, &built, &need)) != DH_OK) return rc;
          if (built) bind_sector_ell(hb, *fell, *f);
        }
        if ((rc = engine_mixed_restart(*f, seed + 1000 + round, fp64_round)) != DH_OK) return rc;
        if ((rc = engine_solve(*f)) != DH_OK) return rc;
        for (size_t jj = 0; jj < redo.size(); ++jj) {
          const BlockSector& bs = f->sec[jj];
          iterations[rsec[jj]] += bs.count;
          src_pos[redo[jj]] = (int)jj;
        }
        pending.clear();
        for (int i : redo)
          if (!need_dense[i]) pending.push_back(i);
        cur = nullptr;  // the previous round's engine goes before the bindings it used
        cur_prod = std::move(fprod);  // the product binding must outlive the engine using it
        cur_ell = std::move(fell);
        cur = std::move(f);
        src = cur.get();
      }
      refine_seconds = std::chrono::duration<double>(clk::now() - tb).count();
    }
    const auto td = clk::now();
    for (int i = 0; i < ns; ++i) {
      if (!need_dense[i]) continue;
      const int s = lanczos_sectors[i];
      std::vector<double> ev;
      if ((rc = dense_lowest(hb.spaces[s], hb, 1, ev, e.stream)) != DH_OK) return rc;
      if (precision == DH_PRECISION_FP32) max_shift = std::max(max_shift, fabs(ev[0] - energies[s]));
      energies[s] = ev[0];
      ++dense_fallback;
    }
    dense_seconds = std::chrono::duration<double>(clk::now() - td).count();
  }
  const auto t2 = clk::now();
  if (stats) {
    stats[0] = std::chrono::duration<double>(t1 - t0).count();
    stats[1] = std::chrono::duration<double>(t2 - t1).count();
    stats[2] = product_ms / 1000.0;
    stats[3] = (double)products;
    stats[4] = fp32_seconds;
    stats[5] = refine_seconds;
    stats[6] = (double)refined;
    stats[7] = max_shift;
    stats[8] = (double)dense_fallback;
    stats[9] = dense_seconds;
    stats[10] = (double)ell_bytes;
    stats[11] = ell_seconds;
  }
  return DH_OK;
}

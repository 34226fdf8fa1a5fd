// C ABI: Lanczos algorithms on the GPU (see include/diagham_b200.h for the contract).
//
// Vectors stay in device memory in FP64.  The recurrence is the reference's
// (BasicLanczosAlgorithm.cc:148-216): alpha_i = <v_i|H v_i>, beta_i = <v_{i-1}|H v_i>, the new
// vector normalised explicitly.  Its scalars live on the device and are only copied to the host to
// diagonalise the tridiagonal matrix, as AbstractLanczosAlgorithm::Diagonalize does after every
// RunLanczosAlgorithm call (AbstractLanczosAlgorithm.cc:136).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "dh_disk.h"
#include "dh_internal.h"
#include "dh_objects.h"

using namespace dh;

namespace {

// Writes checkpoint files on a background thread: the vectors wait in pinned host memory while the
// GPU carries on with the next iterations.  One job at a time; wait() joins it and re-raises its
// error on the calling thread.
struct DiskWriter {
  double* staging = nullptr;  // pinned host copies of the vectors of the job in flight
  size_t staging_doubles = 0;
  std::thread worker;
  int status = DH_OK;
  std::string message;
  DiskWriter() = default;
  DiskWriter(const DiskWriter&) = delete;
  DiskWriter& operator=(const DiskWriter&) = delete;
  ~DiskWriter() {
    if (worker.joinable()) worker.join();
    if (staging) cudaFreeHost(staging);
  }
  int wait() {
    if (worker.joinable()) worker.join();
    const int rc = status;
    status = DH_OK;
    if (rc != DH_OK) set_error("%s", message.c_str());
    return rc;
  }
  int reserve(size_t doubles) {
    if (staging_doubles >= doubles) return DH_OK;
    if (staging) cudaFreeHost(staging);
    staging = nullptr;
    staging_doubles = 0;
    DH_CUDA(cudaMallocHost(&staging, doubles * sizeof(double)));
    staging_doubles = doubles;
    return DH_OK;
  }
  // job: the vectors staging[q * dim] to paths[q], then (if state_path is not empty) the state file
  void start(std::vector<std::string> paths, int64_t dim, std::string state_path, int algorithm,
             LanczosDiskState state) {
    worker = std::thread([this, paths, dim, state_path, algorithm, state]() {
      int rc = DH_OK;
      for (size_t q = 0; q < paths.size() && rc == DH_OK; ++q)
        rc = vector_file_write(paths[q], staging + q * dim, dim);
      if (rc == DH_OK && !state_path.empty()) rc = lanczos_state_write(state_path, algorithm, state);
      if (rc != DH_OK) message = dh_last_error();
      status = rc;
    });
  }
};

}  // namespace

struct dh_lanczos_s {
  dh_hamiltonian_s* h = nullptr;
  int algorithm = DH_LANCZOS_BASIC;
  int nev = 1;
  int block = 1;
  int max_iter = 0;
  double precision = 1e-14;  // MACHINE_PRECISION (src/config.h:49)
  int64_t dim = 0;
  cudaStream_t stream = 0;
  int cap = 0;  // capacity of the scalar arrays (tridiagonal rows)
  DevBuf vec, x32, scal, red_storage, krylov, initial, coef, ground;
  Reducer red;
  LanczosDev st = {};
  int krylov_cap = 0;
  bool krylov_keep = false;  // the Krylov store grows with the run (up to cap vectors)
  bool initialized = false;
  bool ground_valid = false;
  int index = 0;   // reference "Index": the newest vector is v_{index + 1}
  int rows = 0;    // tridiagonal rows
  double prev_last = 0.0;
  std::vector<double> prev_wanted;
  std::vector<double> alpha, beta, ritz;
  int64_t matvecs = 0;
  int64_t fp64_matvecs = 0;
  // mixed-precision restart: the start vector's product in FP64, the following ones in the
  // Hamiltonian's precision, every new vector projected against the start vector
  bool fp64_first = false;
  bool lock_v0 = false;
  // > 0: converged when the lowest Ritz vector's residual estimate beta |s_last| (of the matrix one
  // row short, whose next beta is known) satisfies |r|^2 < residual_target |lambda|
  double residual_target = 0.0;
  cudaGraphExec_t graph3 = nullptr;  // three iterations starting at phase 0
  dh::BlockLanczos* blk = nullptr;   // DH_LANCZOS_BLOCK: everything runs in the block engine
  // disk storage in the reference's disk-storage formats
  bool disk = false;
  std::string disk_dir;
  int disk_interval = 1;
  int disk_rows = -1;        // rows of the checkpoint on disk (-1: none yet)
  int disk_set = 1;          // basic format: name set of the last checkpoint (0: vector1-3, 1: vector4-6)
  int pending = 0;           // rows a resumed mid-call state owes the next run call
  bool resumed = false;      // the next solve continues the driver loop without its first call
  bool start_known = true;   // `initial` holds the start vector
  bool krylov_valid = true;  // the Krylov store holds v_0, v_1, ... (not after a resume)
  DiskWriter writer;
  ~dh_lanczos_s() {
    if (graph3) cudaGraphExecDestroy(graph3);
    if (blk) dh::block_lanczos_destroy(blk);
  }
};

namespace {

// The Krylov store grows with the run instead of holding max_iter vectors from the start: the first
// kKrylovFirst vectors, then doubling (one device-to-device copy per growth), each growth only while
// it takes less than half of the free device memory.  When it cannot grow the store stops where it
// is (the ground state is then replayed from the start vector), except under full
// re-orthogonalisation, which needs every vector.  A growth drops the captured iterations (their
// kernels hold the store's address).
constexpr int kKrylovFirst = 64;

int lz_reserve_krylov(dh_lanczos_s* l, int rows) {
  rows = std::min(rows, l->cap);
  if (!l->krylov_keep || rows <= l->krylov_cap) return DH_OK;
  const size_t vb = (size_t)l->dim * sizeof(double);
  const int want = std::min(l->cap, std::max(rows, std::max(kKrylovFirst, 2 * l->krylov_cap)));
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  DevBuf grown;
  const bool fits = l->algorithm == DH_LANCZOS_FULL_REORTHOGONALIZED || (size_t)want * vb < free_b / 2;
  if (!fits || grown.alloc((size_t)want * vb) != DH_OK) {
    cudaGetLastError();
    DH_CHECK(l->algorithm != DH_LANCZOS_FULL_REORTHOGONALIZED, DH_ERR_MEMORY,
             "full re-orthogonalisation needs %zu bytes for its vectors", (size_t)want * vb);
    l->krylov_keep = false;
    return DH_OK;
  }
  if (l->krylov_cap > 0) {
    DH_CUDA(cudaMemcpyAsync(grown.ptr, l->krylov.ptr, (size_t)l->krylov_cap * vb, cudaMemcpyDeviceToDevice, l->stream));
    DH_CUDA(cudaStreamSynchronize(l->stream));
  }
  l->krylov.release();
  l->krylov.ptr = grown.ptr;
  l->krylov.bytes = grown.bytes;
  grown.ptr = nullptr;
  grown.bytes = 0;
  l->krylov_cap = want;
  l->st.krylov = l->krylov.as<double>();
  l->st.krylov_cap = want;
  if (l->graph3) {
    cudaGraphExecDestroy(l->graph3);
    l->graph3 = nullptr;
  }
  return DH_OK;
}

int lz_matvec(dh_lanczos_s* l, int src_slot, int dst_slot) {
  double* x = l->st.vec + (size_t)src_slot * l->dim;
  double* y = l->st.vec + (size_t)dst_slot * l->dim;
  ++l->matvecs;
  if (l->h->precision == DH_PRECISION_FP64) ++l->fp64_matvecs;
  return hamiltonian_apply(l->h, x, y, 1, 0, l->dim, 0, l->h->precision == DH_PRECISION_FP32 ? l->st.x32 : nullptr,
                           l->stream);
}

// one iteration: v_{i+1} from H v_i, then H v_{i+1} and the two new scalars (i = index)
int lz_iteration(dh_lanczos_s* l, int i) {
  const int phase = i % 3;
  int rc;
  if ((rc = launch_lz_update(l->st, phase, l->stream)) != DH_OK) return rc;
  if (l->algorithm == DH_LANCZOS_FULL_REORTHOGONALIZED && i + 1 >= 3) {
    // FullReorthogonalizedLanczosAlgorithm.cc:230-243: classical Gram-Schmidt of the new vector
    // against v_0 .. v_{i-2} (v_{i-1}, v_i are handled by the recurrence), before normalisation
    double* w = l->st.vec + (size_t)((phase + 1) % 3) * l->dim;
    const int m = i - 1;
    if ((rc = launch_strided_dots(l->st.krylov, m, l->dim, w, l->dim, l->coef.as<double>(), l->red, l->stream)) != DH_OK)
      return rc;
    if ((rc = launch_combine(l->st.krylov, m, l->dim, l->coef.as<double>(), -1.0, w, 1, l->dim, l->stream)) != DH_OK)
      return rc;
    // the norm of the re-orthogonalised vector
    const double* vs[1] = {w};
    if ((rc = launch_multi_dot(vs, 1, w, l->dim, l->st.norm + i + 1, l->red, l->stream)) != DH_OK) return rc;
    if ((rc = launch_sqrt_inplace(l->st.norm + i + 1, l->stream)) != DH_OK) return rc;
  }
  if (l->lock_v0 && i + 1 >= 2) {
    // project the new vector against the start vector (the FP32 products leave components along it
    // of the order of their rounding), then take its norm again
    double* w = l->st.vec + (size_t)((phase + 1) % 3) * l->dim;
    const double* v0 = l->initial.as<double>();
    double* c = l->coef.as<double>() + l->cap + 4;
    const double* vs[1] = {v0};
    if ((rc = launch_multi_dot(vs, 1, w, l->dim, c, l->red, l->stream)) != DH_OK) return rc;
    if ((rc = launch_combine(v0, 1, l->dim, c, -1.0, w, 1, l->dim, l->stream)) != DH_OK) return rc;
    const double* ws[1] = {w};
    if ((rc = launch_multi_dot(ws, 1, w, l->dim, l->st.norm + i + 1, l->red, l->stream)) != DH_OK) return rc;
    if ((rc = launch_sqrt_inplace(l->st.norm + i + 1, l->stream)) != DH_OK) return rc;
  }
  if ((rc = launch_lz_scale(l->st, phase, l->stream)) != DH_OK) return rc;
  if ((rc = lz_matvec(l, (phase + 1) % 3, (phase + 2) % 3)) != DH_OK) return rc;
  return launch_lz_dots(l->st, phase, l->stream);
}

int lz_first_steps(dh_lanczos_s* l) {
  // v_0 in slot 0 (normalised by initialize); H v_0 -> slot 1; alpha_0 = <v_0|H v_0>
  int rc;
  if (l->st.x32 && (rc = launch_convert_f32(l->st.vec, l->st.x32, l->dim, l->stream)) != DH_OK) return rc;
  if (l->st.krylov)
    DH_CUDA(cudaMemcpyAsync(l->st.krylov, l->st.vec, l->dim * sizeof(double), cudaMemcpyDeviceToDevice, l->stream));
  const int saved = l->h->precision;
  if (l->fp64_first) l->h->precision = DH_PRECISION_FP64;
  rc = lz_matvec(l, 0, 1);
  l->h->precision = saved;
  if (rc != DH_OK) return rc;
  const double* vs[1] = {l->st.vec};
  if ((rc = launch_multi_dot(vs, 1, l->st.vec + l->dim, l->dim, l->st.alpha, l->red, l->stream)) != DH_OK) return rc;
  DH_CUDA(cudaMemsetAsync(l->st.cursor, 0, sizeof(int), l->stream));
  return lz_iteration(l, 0);
}

// copy the scalars, diagonalise the tridiagonal matrix, update the previous-eigenvalue bookkeeping
// exactly as BasicLanczosAlgorithm.cc:200-214 does after each RunLanczosAlgorithm call
int lz_finish_call(dh_lanczos_s* l) {
  l->alpha.resize(l->rows);
  l->beta.resize(std::max(l->rows - 1, 0));
  DH_CUDA(cudaMemcpyAsync(l->alpha.data(), l->st.alpha, l->rows * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
  if (l->rows > 1)
    DH_CUDA(cudaMemcpyAsync(l->beta.data(), l->st.beta, (l->rows - 1) * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  const int nev = std::min(l->nev, l->rows);
  std::vector<double> eig;
  // one wanted value: the lowest from the previous call's (that of a leading block, an upper bound)
  // by Newton steps, O(rows) where QL of the whole matrix is O(rows^2) per call
  auto diagonalise = [&]() -> int {
    if (l->nev == 1 && !l->ritz.empty()) {
      eig.assign(1, 0.0);
      return lanczos_lowest_ritz(l->rows, l->alpha.data(), l->beta.data(), &l->ritz[0], eig.data());
    }
    eig.assign(l->rows, 0.0);
    return tridiagonal_eigen(l->rows, l->alpha.data(), l->beta.data(), eig.data(), nullptr);
  };
  if (l->prev_last != 0.0) {
    l->prev_last = l->ritz[nev - 1];
    for (int i = 0; i < nev; ++i) l->prev_wanted[i] = l->ritz[i];
    int rc = diagonalise();
    if (rc != DH_OK) return rc;
  } else {
    int rc = diagonalise();
    if (rc != DH_OK) return rc;
    l->prev_last = 2.0 * eig[nev - 1];
    for (int i = 0; i < nev; ++i) l->prev_wanted[i] = 2.0 * eig[i];
  }
  l->ritz.swap(eig);
  l->ground_valid = false;
  return DH_OK;
}

// The lowest Ritz pair of the matrix one row short (whose next beta is known): its eigenvalue
// (implicit QL without vectors) and its vector's residual estimate beta |s_last|, the last component
// by inverse iteration on that tridiagonal matrix (O(n) per step instead of accumulating all n
// eigenvectors).  False when there are not yet rows enough.
bool lz_lowest_residual(const dh_lanczos_s* l, double* lambda, double* r) {
  const int n = l->rows - 1;
  if (n < 2 || (int)l->beta.size() < n || l->ritz.empty()) return false;
  std::vector<double> eig(n), t((size_t)n * n, 0.0), z(n);
  if (tridiagonal_eigen(n, l->alpha.data(), l->beta.data(), eig.data(), nullptr) != DH_OK) return false;
  for (int i = 0; i < n; ++i) {
    t[(size_t)i * n + i] = l->alpha[i];
    if (i + 1 < n) t[(size_t)i * n + i + 1] = t[(size_t)(i + 1) * n + i] = l->beta[i];
  }
  if (band_inverse_iteration(n, 1, t.data(), eig[0], z.data()) != DH_OK) return false;
  *lambda = eig[0];
  *r = l->beta[n - 1] * z[n - 1];
  return true;
}

// BasicLanczosAlgorithm::TestConvergence (:220): |lambda_{nev-1} - previous| < precision |lambda_{nev-1}|
bool lz_converged(const dh_lanczos_s* l) {
  if (l->residual_target > 0.0) {
    if (l->ritz.empty()) return false;
    // the residual only once the Ritz value has settled: near the residual target its changes are
    // orders of magnitude below this
    if (fabs(l->ritz[0] - l->prev_last) > 1e-7 * fabs(l->ritz[0])) return false;
    double lambda = 0.0, r = 0.0;
    if (!lz_lowest_residual(l, &lambda, &r)) return false;
    return r * r < l->residual_target * fabs(lambda);
  }
  if ((int)l->ritz.size() < l->nev) return false;
  const double e = l->ritz[l->nev - 1];
  return fabs(e - l->prev_last) < l->precision * fabs(e);
}

// The quantity lz_converged tests over its threshold at the current row (the test passes below 1,
// the residual test's settling condition aside), or a negative value when it cannot be evaluated.
double lz_convergence_ratio(const dh_lanczos_s* l) {
  if (l->residual_target > 0.0) {
    double lambda = 0.0, r = 0.0;
    if (!lz_lowest_residual(l, &lambda, &r)) return -1.0;
    const double den = l->residual_target * fabs(lambda);
    return den > 0.0 ? r * r / den : -1.0;
  }
  if ((int)l->ritz.size() < l->nev) return -1.0;
  const double e = l->ritz[l->nev - 1];
  const double den = l->precision * fabs(e);
  return den > 0.0 ? fabs(e - l->prev_last) / den : -1.0;
}

// ------------------------------------------------------------------ disk storage
// Files of the state after a RunLanczosAlgorithm call: v_index (slot index % 3), v_{index+1} and
// H v_{index+1} (the next two slots), with lanczos.dat in the format of the algorithm's disk-storage
// class.  The copies to pinned memory are ordered on the stream; a background thread writes them.
int lz_checkpoint(dh_lanczos_s* l) {
  int rc = l->writer.wait();
  if (rc != DH_OK) return rc;
  DH_CHECK(l->initialized && l->rows >= 2, DH_ERR_STATE,
           "no Lanczos state to write (not run yet, or its vectors were used to rebuild the ground state)");
  const int64_t dim = l->dim;
  if ((rc = l->writer.reserve((size_t)3 * dim)) != DH_OK) return rc;
  for (int q = 0; q < 3; ++q)
    DH_CUDA(cudaMemcpyAsync(l->writer.staging + (size_t)q * dim, l->st.vec + (size_t)((l->index + q) % 3) * dim,
                            dim * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  LanczosDiskState s;
  s.index = l->index;
  s.prev_last = l->prev_last;
  s.precision = l->precision;
  s.nbr_eigenvalue = l->nev;
  s.nbr_row = l->rows;
  s.diag.assign(l->alpha.begin(), l->alpha.begin() + l->rows);
  s.upper.assign(l->beta.begin(), l->beta.begin() + (l->rows - 1));
  std::vector<std::string> paths;
  if (l->algorithm == DH_LANCZOS_BASIC) {
    // the other name set than the checkpoint on disk, which stays whole until lanczos.dat moves on
    const int set = 1 - l->disk_set;
    for (int q = 0; q < 3; ++q) {
      snprintf(s.names[q], sizeof(s.names[q]), "vector%d", 3 * set + q + 1);
      paths.push_back(join_path(l->disk_dir, s.names[q]));
    }
    l->disk_set = set;
  } else {
    for (int q = 0; q < 3; ++q) {
      char name[16];
      snprintf(name, sizeof(name), "vector.%d", q + 1);
      paths.push_back(join_path(l->disk_dir, name));
    }
  }
  l->writer.start(paths, dim, join_path(l->disk_dir, "lanczos.dat"), l->algorithm, s);
  l->disk_rows = l->rows;
  return DH_OK;
}

// vector.0 of the ground-state format: the (normalised) start vector
int lz_write_start_vector(dh_lanczos_s* l) {
  if (!l->disk || l->algorithm != DH_LANCZOS_WITH_GROUND_STATE) return DH_OK;
  int rc = l->writer.wait();
  if (rc != DH_OK) return rc;
  if ((rc = l->writer.reserve((size_t)l->dim)) != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(l->writer.staging, l->initial.ptr, l->dim * sizeof(double), cudaMemcpyDeviceToHost,
                          l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  l->writer.start({join_path(l->disk_dir, "vector.0")}, l->dim, std::string(), l->algorithm, LanczosDiskState());
  return DH_OK;
}

int lz_run(dh_lanczos_s* l, int nbr_iter) {
  DH_CHECK(l->initialized, DH_ERR_STATE, "RunLanczosAlgorithm before InitializeLanczosAlgorithm");
  int target;
  int rc;
  if (l->rows == 0) {
    target = std::max(nbr_iter, 2);
    DH_CHECK(target <= l->cap, DH_ERR_ARGUMENT, "more Lanczos rows (%d) than max_iter allows (%d)", target, l->cap);
    if ((rc = lz_reserve_krylov(l, target)) != DH_OK) return rc;
    if ((rc = lz_first_steps(l)) != DH_OK) return rc;
    l->index = 0;
    l->rows = 2;
  } else {
    // a state resumed from the middle of a call first completes that call's rows
    target = l->rows + l->pending + nbr_iter;
    DH_CHECK(target <= l->cap, DH_ERR_ARGUMENT, "more Lanczos rows (%d) than max_iter allows (%d)", target, l->cap);
  }
  l->pending = 0;
  if ((rc = lz_reserve_krylov(l, target)) != DH_OK) return rc;
  while (l->rows < target) {
    if ((rc = lz_iteration(l, l->index + 1)) != DH_OK) return rc;
    ++l->index;
    ++l->rows;
  }
  if ((rc = lz_finish_call(l)) != DH_OK) return rc;
  if (l->disk && l->rows - l->disk_rows >= l->disk_interval) return lz_checkpoint(l);
  return DH_OK;
}

// Ritz vector of the lowest Ritz value: from the Krylov store when kept, otherwise by replaying the
// recurrence from the start vector (BasicLanczosAlgorithmWithGroundState.cc:256-335)
int lz_ground_state(dh_lanczos_s* l) {
  if (l->ground_valid) return DH_OK;
  DH_CHECK(l->rows >= 2, DH_ERR_STATE, "no Lanczos iteration has been run");
  const int n = l->rows;
  std::vector<double> eig(n), z((size_t)n * n);
  int rc = tridiagonal_eigen(n, l->alpha.data(), l->beta.data(), eig.data(), z.data());
  if (rc != DH_OK) return rc;
  std::vector<double> c(z.begin(), z.begin() + n);  // column 0 (column-major)
  if ((rc = ensure_buffer(l->ground, l->dim * sizeof(double))) != DH_OK) return rc;
  if ((rc = ensure_buffer(l->coef, (size_t)std::max(n, l->cap + 8) * sizeof(double))) != DH_OK) return rc;
  double* g = l->ground.as<double>();
  if (l->st.krylov && l->krylov_valid && n <= l->krylov_cap) {
    DH_CUDA(cudaMemcpyAsync(l->coef.ptr, c.data(), n * sizeof(double), cudaMemcpyHostToDevice, l->stream));
    if ((rc = launch_combine(l->st.krylov, n, l->dim, l->coef.as<double>(), 1.0, g, 0, l->dim, l->stream)) != DH_OK)
      return rc;
  } else {
    // replay: v_0 = start vector, v_{j+1} = (H v_j - alpha_j v_j - beta_{j-1} v_{j-1}) / |.|
    DH_CHECK(l->start_known, DH_ERR_STATE,
             "the start vector is unknown (a state resumed from the basic disk format does not store it)");
    double* v[3] = {l->st.vec, l->st.vec + l->dim, l->st.vec + 2 * l->dim};
    DH_CUDA(cudaMemcpyAsync(v[0], l->initial.ptr, l->dim * sizeof(double), cudaMemcpyDeviceToDevice, l->stream));
    DH_CUDA(cudaMemsetAsync(g, 0, l->dim * sizeof(double), l->stream));
    if ((rc = launch_axpy_scalar(g, v[0], c[0], l->dim, l->stream)) != DH_OK) return rc;
    double* nrm = l->coef.as<double>();
    for (int j = 0; j + 1 < n; ++j) {
      double* cur = v[j % 3];
      double* prev = v[(j + 2) % 3];
      double* next = v[(j + 1) % 3];
      if ((rc = hamiltonian_apply(l->h, cur, next, 1, 0, l->dim, 0, nullptr, l->stream)) != DH_OK) return rc;
      ++l->matvecs;
      if ((rc = launch_lanczos_update(next, next, cur, j > 0 ? prev : nullptr, l->st.alpha + j,
                                      j > 0 ? l->st.beta + j - 1 : nullptr, l->dim, nrm, l->red, l->stream)) != DH_OK)
        return rc;
      if ((rc = launch_scale_convert(next, nullptr, nrm, l->dim, l->stream)) != DH_OK) return rc;
      if ((rc = launch_axpy_scalar(g, next, c[j + 1], l->dim, l->stream)) != DH_OK) return rc;
    }
    // the three work vectors were overwritten: the algorithm cannot continue from here
    l->initialized = false;
  }
  // normalise
  const double* vs[1] = {g};
  double* nrm = l->coef.as<double>();
  if ((rc = launch_multi_dot(vs, 1, g, l->dim, nrm, l->red, l->stream)) != DH_OK) return rc;
  if ((rc = launch_sqrt_inplace(nrm, l->stream)) != DH_OK) return rc;
  if ((rc = launch_scale_convert(g, nullptr, nrm, l->dim, l->stream)) != DH_OK) return rc;
  DH_CUDA(cudaStreamSynchronize(l->stream));
  l->ground_valid = true;
  return DH_OK;
}

int lz_initialize_device(dh_lanczos_s* l) {
  // normalise slot 0 and keep a copy of the start vector for a replay
  const double* vs[1] = {l->st.vec};
  int rc;
  if ((rc = launch_multi_dot(vs, 1, l->st.vec, l->dim, l->st.norm, l->red, l->stream)) != DH_OK) return rc;
  if ((rc = launch_sqrt_inplace(l->st.norm, l->stream)) != DH_OK) return rc;
  if ((rc = launch_scale_convert(l->st.vec, nullptr, l->st.norm, l->dim, l->stream)) != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(l->initial.ptr, l->st.vec, l->dim * sizeof(double), cudaMemcpyDeviceToDevice, l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  l->initialized = true;
  l->ground_valid = false;
  l->rows = 0;
  l->index = 0;
  l->prev_last = 0.0;
  std::fill(l->prev_wanted.begin(), l->prev_wanted.end(), 0.0);
  l->ritz.clear();
  l->pending = 0;
  l->resumed = false;
  l->start_known = true;
  l->krylov_valid = true;
  l->disk_rows = -1;
  return lz_write_start_vector(l);
}

// Three consecutive iterations (phases 0, 1, 2) captured once as a CUDA graph; the device cursor
// selects the scalars, so the same graph serves every batch that starts at a multiple of three.
int lz_graph3(dh_lanczos_s* l) {
  if (l->graph3) return DH_OK;
  DH_CHECK(l->stream != 0, DH_ERR_STATE, "graph capture needs a non-default stream");
  cudaGraph_t g;
  DH_CUDA(cudaStreamBeginCapture(l->stream, cudaStreamCaptureModeThreadLocal));
  int rc = DH_OK;
  int64_t saved = l->matvecs;
  for (int p = 0; p < 3 && rc == DH_OK; ++p) rc = lz_iteration(l, 3 + p);
  l->matvecs = saved;
  cudaError_t e = cudaStreamEndCapture(l->stream, &g);
  if (rc != DH_OK) return rc;
  DH_CUDA(e);
  e = cudaGraphInstantiate(&l->graph3, g, 0);
  cudaGraphDestroy(g);
  DH_CUDA(e);
  return DH_OK;
}

}  // namespace

extern "C" {

int dh_lanczos_create(dh_hamiltonian_t h, int algorithm, int nbr_eigenvalue, int block_size, int max_iter,
                      dh_lanczos_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  DH_CHECK(algorithm == DH_LANCZOS_BASIC || algorithm == DH_LANCZOS_FULL_REORTHOGONALIZED ||
               algorithm == DH_LANCZOS_WITH_GROUND_STATE || algorithm == DH_LANCZOS_BLOCK,
           DH_ERR_UNSUPPORTED, "unknown algorithm %d", algorithm);
  DH_CHECK(nbr_eigenvalue >= 1, DH_ERR_ARGUMENT, "nbr_eigenvalue must be >= 1");
  DH_CHECK(max_iter >= nbr_eigenvalue + 3, DH_ERR_ARGUMENT, "max_iter must be >= nbr_eigenvalue + 3");
  dh_lanczos_s* l = new (std::nothrow) dh_lanczos_s();
  DH_CHECK(l, DH_ERR_MEMORY, "out of host memory");
  if (algorithm == DH_LANCZOS_BLOCK) {
    l->h = h;
    l->algorithm = algorithm;
    l->nev = nbr_eigenvalue;
    l->block = block_size;
    l->max_iter = max_iter;
    l->dim = hamiltonian_dim(h);
    int rc = block_lanczos_create(h, nbr_eigenvalue, block_size, max_iter, &l->blk);
    if (rc != DH_OK) {
      delete l;
      return rc;
    }
    *out = l;
    return DH_OK;
  }
  l->h = h;
  l->algorithm = algorithm;
  l->nev = nbr_eigenvalue;
  l->max_iter = max_iter;
  l->dim = hamiltonian_dim(h);
  l->cap = max_iter + 2;
  l->prev_wanted.assign(nbr_eigenvalue, 0.0);
  int rc;
  const size_t vb = (size_t)l->dim * sizeof(double);
  if ((rc = l->vec.alloc(3 * vb)) != DH_OK || (rc = l->initial.alloc(vb)) != DH_OK ||
      (rc = l->scal.alloc((size_t)3 * (l->cap + 2) * sizeof(double) + 64)) != DH_OK ||
      (rc = l->coef.alloc((size_t)(l->cap + 8) * sizeof(double))) != DH_OK ||
      (rc = reducer_init(l->red, l->red_storage, 16)) != DH_OK) {
    delete l;
    return rc;
  }
  if (h->precision == DH_PRECISION_FP32 && (rc = l->x32.alloc((size_t)l->dim * sizeof(float))) != DH_OK) {
    delete l;
    return rc;
  }
  // keep the Krylov basis on the device (needed by the full re-orthogonalisation; spares the
  // ground-state replay otherwise): its first vectors now, the rest as the run grows
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t kb = (size_t)l->cap * vb;
  DH_CHECK(algorithm != DH_LANCZOS_FULL_REORTHOGONALIZED || kb < free_b, DH_ERR_MEMORY,
           "full re-orthogonalisation needs %zu bytes for its vectors", kb);
  l->krylov_keep = true;
  if ((rc = lz_reserve_krylov(l, kKrylovFirst)) != DH_OK) {
    delete l;
    return rc;
  }
  if (cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete l;
    return cuda_fail(cudaGetLastError(), "cudaStreamCreate", __FILE__, __LINE__);
  }
  double* sc = l->scal.as<double>();
  l->st.vec = l->vec.as<double>();
  l->st.dim = l->dim;
  l->st.x32 = l->x32.as<float>();
  l->st.krylov = l->krylov.as<double>();
  l->st.krylov_cap = l->krylov_cap;
  l->st.alpha = sc;
  l->st.beta = sc + (l->cap + 2);
  l->st.norm = sc + 2 * (l->cap + 2);
  l->st.cursor = reinterpret_cast<int*>(sc + 3 * (l->cap + 2));
  l->st.partial = l->red.partial;
  l->st.ticket = l->red.ticket;
  l->st.nblocks = l->red.nblocks;
  *out = l;
  return DH_OK;
}

int dh_lanczos_destroy(dh_lanczos_t l) {
  if (l) {
    if (l->stream) cudaStreamSynchronize(l->stream);
    cudaStream_t s = l->stream;
    delete l;
    if (s) cudaStreamDestroy(s);
  }
  return DH_OK;
}

int dh_lanczos_set_vector_storage(dh_lanczos_t l, int keep) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  if (l->blk) return block_lanczos_set_storage(l->blk, keep);
  DH_CHECK(l->algorithm != DH_LANCZOS_FULL_REORTHOGONALIZED || keep, DH_ERR_ARGUMENT,
           "full re-orthogonalisation needs its vectors");
  if (!keep) {
    l->krylov.release();
    l->krylov_cap = 0;
    l->krylov_keep = false;
  } else if (!l->krylov.ptr) {
    l->krylov_keep = true;
    int rc = lz_reserve_krylov(l, kKrylovFirst);
    if (rc != DH_OK) return rc;
  }
  l->st.krylov = l->krylov.as<double>();
  l->st.krylov_cap = l->krylov_cap;
  if (l->graph3) {
    cudaGraphExecDestroy(l->graph3);
    l->graph3 = nullptr;
  }
  l->initialized = false;
  return DH_OK;
}

int dh_lanczos_set_eigenvalue_precision(dh_lanczos_t l, double precision) {
  DH_CHECK(l && precision > 0.0, DH_ERR_ARGUMENT, "bad argument");
  l->precision = precision;
  if (l->blk) block_lanczos_set_precision(l->blk, precision);
  return DH_OK;
}

int dh_lanczos_initialize(dh_lanczos_t l, const double* vectors, int nbr_vectors) {
  DH_CHECK(l && vectors && nbr_vectors >= 1, DH_ERR_ARGUMENT, "bad argument");
  if (l->blk) return block_lanczos_initialize(l->blk, vectors, nbr_vectors, 0);
  const cudaMemcpyKind kind = is_device_pointer(vectors) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  DH_CUDA(cudaMemcpyAsync(l->st.vec, vectors, l->dim * sizeof(double), kind, l->stream));
  return lz_initialize_device(l);
}

int dh_lanczos_initialize_random(dh_lanczos_t l, uint64_t seed) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  if (l->blk) return block_lanczos_initialize(l->blk, nullptr, 0, seed);
  int rc = launch_random_vector(l->st.vec, l->dim, seed, l->stream);
  if (rc != DH_OK) return rc;
  return lz_initialize_device(l);
}

int dh_lanczos_run(dh_lanczos_t l, int nbr_iter) {
  DH_CHECK(l && nbr_iter >= 1, DH_ERR_ARGUMENT, "bad argument");
  if (l->blk) return block_lanczos_run(l->blk, nbr_iter);
  return lz_run(l, nbr_iter);
}

int dh_lanczos_test_convergence(dh_lanczos_t l, int* converged) {
  DH_CHECK(l && converged, DH_ERR_ARGUMENT, "null argument");
  *converged = (l->blk ? block_lanczos_converged(l->blk) : lz_converged(l)) ? 1 : 0;
  return DH_OK;
}

int dh_lanczos_get_eigenvalues(dh_lanczos_t l, double* eigenvalues, int n) {
  DH_CHECK(l && eigenvalues, DH_ERR_ARGUMENT, "null argument");
  if (!l->blk && n > (int)l->ritz.size() && n <= l->rows && (int)l->alpha.size() >= l->rows &&
      (int)l->beta.size() >= l->rows - 1) {
    // a run that wants one value keeps only the lowest: the others by QL of the current matrix
    std::vector<double> eig(l->rows);
    int rc = tridiagonal_eigen(l->rows, l->alpha.data(), l->beta.data(), eig.data(), nullptr);
    if (rc != DH_OK) return rc;
    for (int i = 0; i < n; ++i) eigenvalues[i] = eig[i];
    return DH_OK;
  }
  const std::vector<double>& ritz = l->blk ? block_lanczos_ritz(l->blk) : l->ritz;
  DH_CHECK(n >= 0 && n <= (int)ritz.size(), DH_ERR_ARGUMENT, "only %d Ritz values", (int)ritz.size());
  for (int i = 0; i < n; ++i) eigenvalues[i] = ritz[i];
  return DH_OK;
}

int dh_lanczos_get_ground_state_energy(dh_lanczos_t l, double* energy) {
  DH_CHECK(l && energy, DH_ERR_ARGUMENT, "null argument");
  const std::vector<double>& ritz = l->blk ? block_lanczos_ritz(l->blk) : l->ritz;
  DH_CHECK(!ritz.empty(), DH_ERR_STATE, "no Lanczos iteration has been run");
  *energy = ritz[0];
  return DH_OK;
}

int dh_lanczos_get_ground_state(dh_lanczos_t l, double* vec) {
  DH_CHECK(l && vec, DH_ERR_ARGUMENT, "null argument");
  if (l->blk) return block_lanczos_eigenstates(l->blk, 1, vec);
  int rc = lz_ground_state(l);
  if (rc != DH_OK) return rc;
  const cudaMemcpyKind kind = is_device_pointer(vec) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  DH_CUDA(cudaMemcpyAsync(vec, l->ground.ptr, l->dim * sizeof(double), kind, l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  return DH_OK;
}

int dh_lanczos_get_eigenstates(dh_lanczos_t l, int n, double* vecs) {
  DH_CHECK(l && vecs, DH_ERR_ARGUMENT, "null argument");
  if (l->blk) return block_lanczos_eigenstates(l->blk, n, vecs);
  DH_CHECK(n >= 1 && n <= l->rows, DH_ERR_ARGUMENT, "%d eigenstates asked of %d Lanczos rows", n, l->rows);
  if (n == 1) return dh_lanczos_get_ground_state(l, vecs);
  DH_CHECK(l->st.krylov && l->krylov_valid && l->rows <= l->krylov_cap, DH_ERR_UNSUPPORTED,
           "more than one eigenstate needs the stored Krylov vectors (of a run that was not resumed)");
  const int m = l->rows;
  std::vector<double> eig(m), z((size_t)m * m);
  int rc = tridiagonal_eigen(m, l->alpha.data(), l->beta.data(), eig.data(), z.data());
  if (rc != DH_OK) return rc;
  if ((rc = ensure_buffer(l->ground, l->dim * sizeof(double))) != DH_OK) return rc;
  if ((rc = ensure_buffer(l->coef, (size_t)std::max(m, l->cap + 8) * sizeof(double))) != DH_OK) return rc;
  const bool dev = is_device_pointer(vecs);
  double* g = l->ground.as<double>();
  for (int c = 0; c < n; ++c) {
    double* dst = dev ? vecs + (size_t)c * l->dim : g;
    DH_CUDA(cudaMemcpyAsync(l->coef.ptr, z.data() + (size_t)c * m, m * sizeof(double), cudaMemcpyHostToDevice, l->stream));
    if ((rc = launch_combine(l->st.krylov, m, l->dim, l->coef.as<double>(), 1.0, dst, 0, l->dim, l->stream)) != DH_OK)
      return rc;
    const double* vs[1] = {dst};
    double* nrm = l->coef.as<double>() + m;
    if ((rc = launch_multi_dot(vs, 1, dst, l->dim, nrm, l->red, l->stream)) != DH_OK) return rc;
    if ((rc = launch_sqrt_inplace(nrm, l->stream)) != DH_OK) return rc;
    if ((rc = launch_scale_convert(dst, nullptr, nrm, l->dim, l->stream)) != DH_OK) return rc;
    if (!dev)
      DH_CUDA(cudaMemcpyAsync(vecs + (size_t)c * l->dim, dst, l->dim * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
    DH_CUDA(cudaStreamSynchronize(l->stream));
  }
  l->ground_valid = false;  // the ground-state buffer now holds the last vector
  return DH_OK;
}

int dh_lanczos_get_counters(dh_lanczos_t l, int64_t* matvecs, int* rows) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  if (l->blk) {
    block_lanczos_counters(l->blk, matvecs, rows);
    return DH_OK;
  }
  if (matvecs) *matvecs = l->matvecs;
  if (rows) *rows = l->rows;
  return DH_OK;
}

int dh_lanczos_solve(dh_lanczos_t l, int max_iter, int graph_batch, double* eigenvalues, int* iterations,
                     int* converged) {
  DH_CHECK(l && eigenvalues && iterations && converged, DH_ERR_ARGUMENT, "null argument");
  if (l->blk) return block_lanczos_solve(l->blk, max_iter, eigenvalues, iterations, converged);
  DH_CHECK(l->initialized, DH_ERR_STATE, "solve before InitializeLanczosAlgorithm");
  if (max_iter > l->max_iter) max_iter = l->max_iter;
  int rc;
  // QHEOnSphereMainTask.cc:732-753: RunLanczosAlgorithm(nev + 2), counter = nev + 3; a resumed run
  // (--resume, :730) skips that call and counts from 0
  int count = 0;
  if (!l->resumed) {
    if ((rc = lz_run(l, l->nev + 2)) != DH_OK) return rc;
    count = l->nev + 3;
  }
  l->resumed = false;
  // the start-vector projection indexes its norm from the host, and checkpoints need the state of
  // every call on the device: no graph batches with either
  const bool use_graph =
      graph_batch > 1 && l->algorithm != DH_LANCZOS_FULL_REORTHOGONALIZED && !l->lock_v0 && !l->disk;
  // The iterations of a batch past the converged row are discarded, so a batch is cut short where
  // the convergence test is predicted to pass (lanczos_batch_prediction): the test's ratio to its
  // threshold falls about geometrically once the lowest Ritz value converges, at a rate taken over
  // the last kLanczosRateSpan rows (the ratio is sampled at each batch's end and kLanczosRateSpan
  // rows before it).  A batch that ends short of convergence costs a host round trip, far less than
  // an unneeded product.  (Replayed on the reference's Lanczos runs of seven FQHE sectors at four
  // precisions, the products past convergence fall from 235 to 42 against batches of 16, for 140
  // round trips instead of 121.)
  // Under the residual test (the FP32 phase of the refined solve) the batches stay whole: there the
  // prediction saved no product (67 FP32 products either way at N = 12, 2S = 33, 1e-10).
  const bool adaptive = l->residual_target <= 0.0;
  std::vector<int> sample_rows;
  std::vector<double> sample_logs;
  int batch = graph_batch;
  while (!lz_converged(l) && count < max_iter) {
    if (!use_graph) {
      ++count;
      if ((rc = lz_run(l, 1)) != DH_OK) return rc;
      continue;
    }
    // issue iterations on the device without a host round trip until the next multiple of three,
    // then whole captured triples, then replay the per-iteration convergence test on the host
    int todo = std::min(batch, max_iter - count);
    todo = std::min(todo, l->cap - l->rows);
    if (todo <= 0) break;
    if ((rc = lz_reserve_krylov(l, l->rows + todo)) != DH_OK) return rc;
    const int start_rows = l->rows;
    int issued = 0;
    while (issued < todo && ((l->index + 1) % 3) != 0) {
      if ((rc = lz_iteration(l, l->index + 1)) != DH_OK) break;
      ++l->index;
      ++l->rows;
      ++issued;
    }
    if (rc == DH_OK && todo - issued >= 3 && (rc = lz_graph3(l)) == DH_OK) {
      while (todo - issued >= 3) {
        cudaError_t e = cudaGraphLaunch(l->graph3, l->stream);
        if (e != cudaSuccess) {
          rc = cuda_fail(e, "cudaGraphLaunch", __FILE__, __LINE__);
          break;
        }
        l->index += 3;
        l->rows += 3;
        l->matvecs += 3;
        issued += 3;
      }
    }
    while (rc == DH_OK && issued < todo) {
      if ((rc = lz_iteration(l, l->index + 1)) != DH_OK) break;
      ++l->index;
      ++l->rows;
      ++issued;
    }
    if (rc != DH_OK) return rc;
    // host side: one RunLanczosAlgorithm(1) bookkeeping step per issued iteration
    const int end_rows = l->rows;
    std::vector<double> a(end_rows), b(end_rows);
    DH_CUDA(cudaMemcpyAsync(a.data(), l->st.alpha, end_rows * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
    DH_CUDA(cudaMemcpyAsync(b.data(), l->st.beta, (end_rows - 1) * sizeof(double), cudaMemcpyDeviceToHost, l->stream));
    DH_CUDA(cudaStreamSynchronize(l->stream));
    for (int r = start_rows + 1; r <= end_rows; ++r) {
      ++count;
      l->rows = r;
      if ((rc = lz_finish_call(l)) != DH_OK) return rc;
      if (lz_converged(l) || count >= max_iter) break;
      if (adaptive && (r == end_rows - kLanczosRateSpan || r == end_rows)) {
        const double ratio = lz_convergence_ratio(l);
        if (ratio > 0.0) {
          sample_rows.push_back(r);
          sample_logs.push_back(log(ratio));
        }
      }
    }
    if (l->rows < end_rows) {
      // converged before the end of the batch: the extra iterations are discarded; the Krylov
      // vectors beyond l->rows are unused, so the algorithm cannot be continued
      l->index = l->rows - 2;
      l->initialized = false;
    } else {
      batch = graph_batch;
      if (!sample_rows.empty() && sample_rows.back() == end_rows)
        batch = lanczos_batch_prediction((int)sample_rows.size(), sample_rows.data(), sample_logs.data(), graph_batch);
    }
  }
  if (l->disk) {
    // the final state is on disk when the solve returns
    if (l->rows != l->disk_rows && (rc = lz_checkpoint(l)) != DH_OK) return rc;
    if ((rc = l->writer.wait()) != DH_OK) return rc;
  }
  *iterations = count;
  *converged = lz_converged(l) ? 1 : 0;
  for (int i = 0; i < l->nev && i < (int)l->ritz.size(); ++i) eigenvalues[i] = l->ritz[i];
  return DH_OK;
}

int dh_lanczos_set_disk_storage(dh_lanczos_t l, const char* directory, int interval) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  DH_CHECK(!l->blk && (l->algorithm == DH_LANCZOS_BASIC || l->algorithm == DH_LANCZOS_WITH_GROUND_STATE),
           DH_ERR_UNSUPPORTED, "disk storage is implemented for the basic and with-ground-state algorithms");
  // the files are the real classes' formats; the complex classes (ComplexBasicLanczosAlgorithmWith-
  // DiskStorage) keep complex vectors, which these files would not be
  DH_CHECK(!l->h->complex_phases, DH_ERR_UNSUPPORTED,
           "disk storage of the complex Lanczos classes is not implemented (real formats only)");
  int rc = l->writer.wait();
  if (rc != DH_OK) return rc;
  if (!directory) {
    l->disk = false;
    l->disk_dir.clear();
    return DH_OK;
  }
  DH_CHECK(interval >= 1, DH_ERR_ARGUMENT, "checkpoint interval must be >= 1");
  l->disk = true;
  l->disk_dir = directory;
  l->disk_interval = interval;
  l->disk_rows = -1;
  // a start vector set before disk storage was switched on
  if (l->initialized && l->start_known && l->rows == 0) return lz_write_start_vector(l);
  return DH_OK;
}

int dh_lanczos_write_state(dh_lanczos_t l) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  DH_CHECK(l->disk, DH_ERR_STATE, "WriteState needs disk storage (dh_lanczos_set_disk_storage)");
  int rc = lz_checkpoint(l);
  if (rc != DH_OK) return rc;
  return l->writer.wait();
}

int dh_lanczos_resume(dh_lanczos_t l) {
  DH_CHECK(l, DH_ERR_ARGUMENT, "null lanczos");
  DH_CHECK(l->disk, DH_ERR_STATE, "ResumeLanczosAlgorithm needs disk storage (dh_lanczos_set_disk_storage)");
  int rc = l->writer.wait();
  if (rc != DH_OK) return rc;
  LanczosDiskState s;
  if ((rc = lanczos_state_read(join_path(l->disk_dir, "lanczos.dat"), l->algorithm, &s)) != DH_OK) return rc;
  const bool ground = l->algorithm == DH_LANCZOS_WITH_GROUND_STATE;
  // GroundStateEvaluationFlag 1: the run had finished and its ground state was being assembled
  // (Index then counts assembly steps); every row of the matrix is valid
  const bool finished = ground && s.ground_flag == 1;
  const int rows = finished ? s.nbr_row : s.index + 2;
  DH_CHECK(rows + (finished ? 0 : 1) <= l->cap, DH_ERR_ARGUMENT,
           "the stored state has %d rows; this handle holds %d (max_iter + 2)", rows, l->cap);
  const int64_t dim = l->dim;
  if ((rc = l->writer.reserve((size_t)4 * dim)) != DH_OK) return rc;
  double* host = l->writer.staging;
  if (!finished) {
    for (int q = 0; q < 3; ++q) {
      char name[16];
      if (ground) snprintf(name, sizeof(name), "vector.%d", q + 1);
      const std::string path = join_path(l->disk_dir, ground ? name : s.names[q]);
      if ((rc = vector_file_read(path, host + (size_t)q * dim, dim)) != DH_OK) return rc;
    }
  }
  if (ground && (rc = vector_file_read(join_path(l->disk_dir, "vector.0"), host + (size_t)3 * dim, dim)) != DH_OK)
    return rc;
  std::vector<double> eig(rows);
  if ((rc = tridiagonal_eigen(rows, s.diag.data(), s.upper.data(), eig.data(), nullptr)) != DH_OK) return rc;
  // the device state: the three vectors in their slots, the scalars, the iteration cursor
  if (!finished)
    for (int q = 0; q < 3; ++q)
      DH_CUDA(cudaMemcpyAsync(l->st.vec + (size_t)((s.index + q) % 3) * dim, host + (size_t)q * dim,
                              dim * sizeof(double), cudaMemcpyHostToDevice, l->stream));
  if (ground)
    DH_CUDA(cudaMemcpyAsync(l->initial.ptr, host + (size_t)3 * dim, dim * sizeof(double), cudaMemcpyHostToDevice,
                            l->stream));
  DH_CUDA(cudaMemcpyAsync(l->st.alpha, s.diag.data(), rows * sizeof(double), cudaMemcpyHostToDevice, l->stream));
  DH_CUDA(cudaMemcpyAsync(l->st.beta, s.upper.data(), (rows - 1) * sizeof(double), cudaMemcpyHostToDevice, l->stream));
  const int cursor = rows - 1;
  DH_CUDA(cudaMemcpyAsync(l->st.cursor, &cursor, sizeof(int), cudaMemcpyHostToDevice, l->stream));
  DH_CUDA(cudaStreamSynchronize(l->stream));
  l->alpha.assign(s.diag.begin(), s.diag.begin() + rows);
  l->beta.assign(s.upper.begin(), s.upper.begin() + (rows - 1));
  l->index = rows - 2;
  l->rows = rows;
  l->prev_last = s.prev_last;
  l->precision = s.precision;
  l->ritz.swap(eig);
  l->pending = finished ? 0 : s.nbr_row - rows;
  l->resumed = !finished;
  l->initialized = !finished;
  l->ground_valid = false;
  l->start_known = ground;
  l->krylov_valid = false;
  l->disk_rows = rows;
  l->disk_set = (!ground && s.names[0][6] >= '4') ? 1 : 0;
  return DH_OK;
}

int dh_lanczos_solve_refined(dh_lanczos_t l, int max_iter, double precision, double* out) {
  DH_CHECK(l && out, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(precision > 0.0, DH_ERR_ARGUMENT, "precision must be > 0");
  if (l->blk) return block_lanczos_solve_refined(l->blk, max_iter, precision, out);
  DH_CHECK(l->initialized, DH_ERR_STATE, "solve before InitializeLanczosAlgorithm");
  DH_CHECK(!l->disk, DH_ERR_UNSUPPORTED, "the refined solve restarts its Lanczos runs: switch disk storage off");
  dh_hamiltonian_s* h = l->h;
  const int saved_precision = h->precision;
  const double saved_lz_precision = l->precision;
  const int64_t matvecs0 = l->matvecs, fp64_0 = l->fp64_matvecs;
  int rc;
  auto drop_graph = [&]() {
    if (l->graph3) {
      cudaGraphExecDestroy(l->graph3);
      l->graph3 = nullptr;
    }
  };
  if (!l->st.x32) {
    if ((rc = l->x32.alloc((size_t)l->dim * sizeof(float))) != DH_OK) return rc;
    l->st.x32 = l->x32.as<float>();
    drop_graph();
  }
  l->fp64_first = l->lock_v0 = false;
  // phase 1: FP32 products, FP64 recurrence, converged to the FP32 resolution of the Ritz value
  // (converged on the Ritz vector's residual down to the FP32 rounding floor of the products: when
  // the target lies above it the FP64 check that follows passes without a restart)
  h->precision = DH_PRECISION_FP32;
  l->precision = std::max(precision, 1e-9);
  l->residual_target = std::max(0.1 * precision, 1e-11);
  double e32 = 0.0;
  int iters = 0, conv = 0;
  rc = dh_lanczos_solve(l, max_iter, 16, &e32, &iters, &conv);
  l->residual_target = 0.0;
  if (rc == DH_OK) rc = lz_ground_state(l);
  double energy = e32, rnorm = 0.0;
  double* sc = l->coef.as<double>();
  // FP64 Rayleigh quotient and residual of the Ritz vector
  auto fp64_check = [&]() -> int {
    double* psi = l->ground.as<double>();
    double* hpsi = l->st.vec;
    double* res = l->st.vec + l->dim;
    const int saved = h->precision;
    h->precision = DH_PRECISION_FP64;
    int r = hamiltonian_apply(h, psi, hpsi, 1, 0, l->dim, 0, nullptr, l->stream);
    h->precision = saved;
    ++l->matvecs;
    ++l->fp64_matvecs;
    const double* vs[1] = {psi};
    if (r == DH_OK) r = launch_multi_dot(vs, 1, hpsi, l->dim, sc, l->red, l->stream);
    if (r == DH_OK) r = launch_lanczos_update(res, hpsi, psi, nullptr, sc, nullptr, l->dim, sc + 1, l->red, l->stream);
    double host[2] = {0.0, 0.0};
    if (r == DH_OK && cudaMemcpyAsync(host, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, l->stream) != cudaSuccess)
      r = cuda_fail(cudaGetLastError(), "copy", __FILE__, __LINE__);
    if (r == DH_OK && cudaStreamSynchronize(l->stream) != cudaSuccess)
      r = cuda_fail(cudaGetLastError(), "sync", __FILE__, __LINE__);
    energy = host[0];
    rnorm = host[1];
    return r;
  };
  // the Rayleigh-quotient error is bounded by |r|^2 / gap: while that may exceed the target, restart
  // from the Ritz vector.  With the Krylov vectors stored the restart is mixed precision (the Ritz
  // vector's product in FP64, the correction directions' products in FP32); otherwise it is FP64.
  for (int round = 0; rc == DH_OK; ++round) {
    if ((rc = fp64_check()) != DH_OK) break;
    if (rnorm * rnorm <= precision * std::max(fabs(energy), 1e-300) || round == 3) break;
    DH_CUDA(cudaMemcpyAsync(l->st.vec, l->ground.ptr, l->dim * sizeof(double), cudaMemcpyDeviceToDevice, l->stream));
    drop_graph();
    const bool mixed = l->krylov_cap > 0;
    float* keep32 = l->st.x32;
    if (mixed) {
      l->fp64_first = l->lock_v0 = true;
      l->residual_target = 0.1 * precision;
      h->precision = DH_PRECISION_FP32;
    } else {
      l->st.x32 = nullptr;
      h->precision = DH_PRECISION_FP64;
    }
    rc = lz_initialize_device(l);
    l->precision = precision;
    double e2 = 0.0;
    if (rc == DH_OK) rc = dh_lanczos_solve(l, std::min(max_iter, 200), mixed ? 16 : 1, &e2, &iters, &conv);
    if (rc == DH_OK) rc = lz_ground_state(l);
    l->st.x32 = keep32;
    l->fp64_first = l->lock_v0 = false;
    l->residual_target = 0.0;
    drop_graph();
  }
  h->precision = saved_precision;
  l->precision = saved_lz_precision;
  if (rc != DH_OK) return rc;
  out[0] = energy;
  out[1] = e32;
  out[2] = rnorm;
  out[3] = (double)((l->matvecs - matvecs0) - (l->fp64_matvecs - fp64_0));
  out[4] = (double)(l->fp64_matvecs - fp64_0);
  return DH_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ block-size tuner

extern "C" int dh_hamiltonian_tune_block_size(dh_hamiltonian_t h, int max_iter, double precision, int refined,
                                              int* best_k, double* seconds) {
  DH_CHECK(h && best_k, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(precision > 0.0, DH_ERR_ARGUMENT, "precision must be > 0");
  const int saved_precision = h->precision;
  const int ks[3] = {1, 2, 4};
  double best = 1e300;
  *best_k = 1;
  for (int i = 0; i < 3; ++i) {
    const int k = ks[i];
    if (seconds) seconds[i] = 0.0;
    if (k > 1 && h->complex_phases) continue;  // complex vectors go one at a time
    if ((long long)4 * k > hamiltonian_dim(h)) continue;
    h->precision = refined ? DH_PRECISION_FP32 : DH_PRECISION_FP64;
    dh_lanczos_t l = nullptr;
    int rc = dh_lanczos_create(h, k == 1 ? DH_LANCZOS_BASIC : DH_LANCZOS_BLOCK, 1, k, max_iter, &l);
    if (rc != DH_OK) {
      h->precision = saved_precision;
      return rc;
    }
    struct Guard {
      dh_lanczos_t l;
      ~Guard() { dh_lanczos_destroy(l); }
    } guard{l};
    DH_CUDA(cudaDeviceSynchronize());
    const auto t0 = std::chrono::steady_clock::now();
    if ((rc = dh_lanczos_set_eigenvalue_precision(l, precision)) == DH_OK &&
        (rc = dh_lanczos_initialize_random(l, 0)) == DH_OK) {
      if (refined) {
        double out[5];
        rc = dh_lanczos_solve_refined(l, max_iter, precision, out);
      } else {
        double e = 0.0;
        int it = 0, conv = 0;
        rc = dh_lanczos_solve(l, max_iter, 16, &e, &it, &conv);
      }
    }
    h->precision = saved_precision;
    if (rc != DH_OK) return rc;
    DH_CUDA(cudaDeviceSynchronize());
    const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (seconds) seconds[i] = t;
    if (t < best) {
      best = t;
      *best_k = k;
    }
  }
  return DH_OK;
}

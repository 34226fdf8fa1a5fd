// Handle structures behind the opaque C ABI types.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "dh_internal.h"

// Largest DiagHam lookup table staged in shared memory by the DH_INDEX_LOOKUP kernels.
#define DH_LOOKUP_SMEM_BYTES (96 * 1024)

// The device current when a handle is created; its device memory lives there (-1 without a device).
inline int dh_current_device() {
  int d = -1;
  return cudaGetDevice(&d) == cudaSuccess ? d : -1;
}

struct dh_space_s {
  int kind = 0;
  int device = dh_current_device();
  int64_t dim = 0;
  int index_mode = DH_INDEX_RANK;
  int kernel_variant = 0;  // product kernel of the rank mode (0 split-word, 1 generic, 2 split + smem table)
  int split_form = 0;      // launch form of the split-word kernel (the autotuner's choice)
  int requested_low_bits = 0;
  std::vector<int64_t> counts;  // [n][o][s]: n fermions in orbitals 0..o-1 with orbital-index sum s
  dh::DevBuf words;  // uint64 FermionOnSphere words, uint32 spin words (chain bits only)
  // FermionOnSphere
  int nbr_fermions = 0, lz_max = 0, total_lz = 0, total_sum = 0;
  // BosonOnSphereShort: N bosons in orbitals 0..boson_lz_max, stored as the FermionOnSphere words of
  // N fermions in boson_lz_max + N orbitals (nbr_fermions = N, lz_max = boson_lz_max + N - 1)
  int boson_lz_max = -1;
  unsigned long memory = 0;
  // SPACE_FERMION_LONG: words are (low, high) pairs; the int32 count table; api_halves = 1 when the
  // space was created as FermionOnSphere (its words are 64-bit for dh_space_get_states)
  dh::DevBuf long_table;
  int api_halves = 2;
  // BosonOnSphereShort beyond the split-word tables: uint64 words, ranks from long_table
  bool count_rank = false;
  dh::FermionRankTables rank;
  dh::DevBuf low_rank, high_offset;
  dh::DevBuf lookup, lookup_shift;
  int lookup_bits = 0;
  // Spin1_2Chain
  int length = 0, sz = 0, nbr_up = 0;
  // Spin1_2ChainWithTranslations: representatives in words (uint32, ascending), their orbit sizes
  // and plain chain indices, the table over the whole Sz sector and the lookup over representatives
  int momentum = 0;
  long long chain_dim = 0;
  dh::DevBuf rep_orbit, rep_rank, trans_map, trans_table;
  int table_shift = 0;
  long long table_entries = 0;
};

struct dh_hamiltonian_s {
  dh_space_s* space = nullptr;
  int kind = 0;
  int precision = DH_PRECISION_FP64;
  double shift = 0.0;        // user shift + shift_base
  double shift_base = 0.0;   // constant part of the operator itself (l2 factor x (Lz^2 + Lz))
  bool l2_only = false;      // ParticleOnSphereL2Hamiltonian: no pseudopotentials
  cudaStream_t stream = 0;
  // FQHE
  dh::InteractionTables tabs;
  std::vector<double> v;
  dh::DevBuf pair_offset, factors64, factors32;
  // J1-J2 chain; complex_phases: SpinChainJ1J2HamiltonianWithTranslations at any momentum, acting on
  // complex vectors stored as (Re, Im) pairs, i.e. a real symmetric operator of dimension 2 D
  double j1 = 0.0, j2 = 0.0;
  bool complex_phases = false;
  // stored elements (fast multiplication): built by dh_hamiltonian_enable_fast_multiplication
  bool fast = false;
  bool fast_use = true;  // products read the stored elements (the autotuner may prefer the on-the-fly form)
  int ell_chunk = 16;    // stored elements read ahead of the gathers per lane: 8 or 16
  long long fast_elements = 0;  // stored elements, padding included
  size_t fast_bytes = 0;
  dh::DevBuf ell_slice_ptr, ell_slice_len, ell_cols, ell_coef, ell_coef32, diag64, diag32;  // ell_coef32: bosons
  // staging / scratch
  dh::DevBuf stage_x, stage_y, stage_v, x32, bins_partial, bins;
  dh::Reducer red;
  dh::DevBuf red_storage;
  // products into host memory: a second stream carries finished row chunks back while the next
  // chunks are computed (created on first use)
  static const int kCopyChunks = 8;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t chunk_done[kCopyChunks] = {};
  ~dh_hamiltonian_s() {
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);
      cudaStreamDestroy(copy_stream);
    }
    for (cudaEvent_t e : chunk_done)
      if (e) cudaEventDestroy(e);
  }
};

namespace dh {
// the length of the (real) vectors the Hamiltonian acts on: the space's dimension, twice that for
// complex vectors stored as (Re, Im) pairs
inline int64_t hamiltonian_dim(const dh_hamiltonian_s* h) {
  return h->complex_phases ? 2 * h->space->dim : h->space->dim;
}
bool is_device_pointer(const void* p);
int ensure_buffer(DevBuf& b, size_t bytes);
int build_lookup(dh_space_s* sp);
FqheDevice fqhe_device(const dh_space_s* sp, const dh_hamiltonian_s* h, int precision);
// the product restricted to output rows [out_first, out_last) (out_last = 0: every row)
int hamiltonian_apply_rows(dh_hamiltonian_s* h, const double* x, double* y, int nvec, int64_t first, int64_t nbr,
                           int accumulate, const float* x32_ready, cudaStream_t stream, int64_t out_first,
                           int64_t out_last);
int hamiltonian_apply_block_rows(dh_hamiltonian_s* h, const double* x64, const float* x32, double* y, int k,
                                 int precision, cudaStream_t stream, int64_t out_first, int64_t out_last);
SpinDevice spin_device(const dh_space_s* sp, const dh_hamiltonian_s* h);
TransDevice trans_device(const dh_space_s* sp, const dh_hamiltonian_s* h);
FqheLongDevice fqhe_long_device(const dh_space_s* sp, const dh_hamiltonian_s* h, int precision);
int upload_factors(dh_hamiltonian_s* h);
// (re)build the split-word rank tables of a FermionOnSphere space for a split of low_bits (0: the
// default, or the space's requested split) and upload them
int build_rank_tables(dh_space_s* sp, int low_bits);
// the stored-element view of an FQHE Hamiltonian whose fast multiplication is enabled
EllDevice ell_device(const dh_hamiltonian_s* h, int precision);
// recompute the stored diagonal after the factors changed
int refresh_fast_diagonal(dh_hamiltonian_s* h);
// y (+)= H x for nvec vectors stored one after the other; x32_ready: FP32 copy of x if already made
int hamiltonian_apply(dh_hamiltonian_s* h, const double* x, double* y, int nvec, int64_t first, int64_t nbr,
                      int accumulate, const float* x32_ready, cudaStream_t stream);
// y = H x for a [dim][k] block (x64 FP64; x32 its FP32 copy, used when precision is FP32)
int hamiltonian_apply_block(dh_hamiltonian_s* h, const double* x64, const float* x32, double* y, int k, int precision,
                            cudaStream_t stream);

// block Lanczos on one Hamiltonian (the engine of the batched sectors with a single sector)
struct BlockLanczos;
int block_lanczos_create(dh_hamiltonian_s* h, int nev, int k, int max_iter, BlockLanczos** out);
void block_lanczos_destroy(BlockLanczos* b);
int block_lanczos_set_storage(BlockLanczos* b, int keep);
void block_lanczos_set_precision(BlockLanczos* b, double precision);
// vectors: nbr_vectors vectors one after the other (host or device), the rest of the block random
// from seed; vectors == nullptr: the whole block random
int block_lanczos_initialize(BlockLanczos* b, const double* vectors, int nbr_vectors, uint64_t seed);
int block_lanczos_run(BlockLanczos* b, int nbr_iter);
bool block_lanczos_converged(const BlockLanczos* b);
const std::vector<double>& block_lanczos_ritz(const BlockLanczos* b);
// the n lowest Ritz vectors (n <= k), normalised, one after the other (host or device)
int block_lanczos_eigenstates(BlockLanczos* b, int n, double* out);
void block_lanczos_counters(const BlockLanczos* b, int64_t* products, int* rows);
int block_lanczos_solve(BlockLanczos* b, int max_iter, double* eigenvalues, int* iterations, int* converged);
int block_lanczos_solve_refined(BlockLanczos* b, int max_iter, double precision, double* out);
}  // namespace dh

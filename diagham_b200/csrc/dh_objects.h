// Handle structures behind the opaque C ABI types.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "dh_internal.h"

// Largest DiagHam lookup table staged in shared memory by the DH_INDEX_LOOKUP kernels.
#define DH_LOOKUP_SMEM_BYTES (96 * 1024)

struct dh_space_s {
  int kind = 0;
  int64_t dim = 0;
  int index_mode = DH_INDEX_RANK;
  int kernel_variant = 0;  // product kernel of the rank mode (0 split-word, 1 generic, 2 split + smem table)
  int requested_low_bits = 0;
  dh::DevBuf words;  // uint64 FermionOnSphere words, uint32 spin words (chain bits only)
  // FermionOnSphere
  int nbr_fermions = 0, lz_max = 0, total_lz = 0, total_sum = 0;
  unsigned long memory = 0;
  dh::FermionRankTables rank;
  dh::DevBuf low_rank, high_offset;
  dh::DevBuf lookup, lookup_shift;
  int lookup_bits = 0;
  // Spin1_2Chain
  int length = 0, sz = 0, nbr_up = 0;
};

struct dh_hamiltonian_s {
  dh_space_s* space = nullptr;
  int kind = 0;
  int precision = DH_PRECISION_FP64;
  double shift = 0.0;
  cudaStream_t stream = 0;
  // FQHE
  dh::InteractionTables tabs;
  std::vector<double> v;
  dh::DevBuf pair_offset, factors64, factors32;
  // J1-J2 chain
  double j1 = 0.0, j2 = 0.0;
  // staging / scratch
  dh::DevBuf stage_x, stage_y, stage_v, x32, bins_partial, bins;
  dh::Reducer red;
  dh::DevBuf red_storage;
};

namespace dh {
bool is_device_pointer(const void* p);
int ensure_buffer(DevBuf& b, size_t bytes);
int build_lookup(dh_space_s* sp);
FqheDevice fqhe_device(const dh_space_s* sp, const dh_hamiltonian_s* h, int precision);
SpinDevice spin_device(const dh_space_s* sp, const dh_hamiltonian_s* h);
int upload_factors(dh_hamiltonian_s* h);
// y (+)= H x for nvec vectors stored one after the other; x32_ready: FP32 copy of x if already made
int hamiltonian_apply(dh_hamiltonian_s* h, const double* x, double* y, int nvec, int64_t first, int64_t nbr,
                      int accumulate, const float* x32_ready, cudaStream_t stream);
}  // namespace dh

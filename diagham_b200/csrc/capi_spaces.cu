// C ABI: Hilbert spaces and Hamiltonians (see include/diagham_b200.h for the contract).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <math.h>

#include <algorithm>
#include <memory>
#include <new>
#include <vector>

#include "dh_internal.h"
#include "dh_objects.h"

using namespace dh;

namespace dh {

const char* last_error();

bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// FermionOnSphere set-up: orbital-sum counts, the two rank tables and the basis words
int build_rank_tables(dh_space_s* sp, int low_bits) {
  const int N = sp->nbr_fermions, L = sp->lz_max, K = sp->total_sum;
  const int O = L + 2;
  auto C = [&](int n, int o, int s) -> int64_t { return sp->counts[((size_t)n * O + o) * (K + 1) + s]; };
  // rank tables: index(w) = high_offset[w >> LB] + low_rank[w & (2^LB - 1)]
  FermionRankTables& t = sp->rank;
  t.low_bits = (L + 2) / 2;
  if (sp->requested_low_bits > 0) t.low_bits = sp->requested_low_bits;
  if (low_bits > 0) t.low_bits = low_bits;
  if (sp->kernel_variant == 2 && t.low_bits > 15) t.low_bits = 15;
  if (t.low_bits < 3) t.low_bits = 3;
  if (t.low_bits > L) t.low_bits = L;
  if (L + 1 - t.low_bits > 26) t.low_bits = L + 1 - 26;
  t.high_bits = L + 1 - t.low_bits;
  const int LB = t.low_bits, HB = t.high_bits;
  const int maxsum = LB * (LB - 1) / 2;
  std::vector<int> counter((size_t)(LB + 1) * (maxsum + 1), 0);
  t.low_rank.assign((size_t)1 << LB, 0);
  for (int64_t l = ((int64_t)1 << LB) - 1; l >= 0; --l) {
    int pc = __builtin_popcountll((unsigned long long)l), ws = 0;
    for (int b = 0; b < LB; ++b)
      if ((l >> b) & 1) ws += b;
    int& c = counter[(size_t)pc * (maxsum + 1) + ws];
    DH_CHECK(c < 65535, DH_ERR_UNSUPPORTED, "FermionOnSphere: rank class too large for 16-bit ranks");
    t.low_rank[l] = (uint16_t)c++;
  }
  t.high_offset.assign((size_t)1 << HB, -1);
  int64_t running = 0;
  for (int64_t h = ((int64_t)1 << HB) - 1; h >= 0; --h) {
    int nh = __builtin_popcountll((unsigned long long)h), sh = 0;
    for (int b = 0; b < HB; ++b)
      if ((h >> b) & 1) sh += b + LB;
    int nl = N - nh, sl = K - sh;
    if (nl < 0 || nl > LB || sl < 0 || sl > maxsum) continue;
    int64_t c = C(nl, LB, sl);
    if (c == 0) continue;
    t.high_offset[h] = (int32_t)running;
    running += c;
  }
  DH_CHECK(running == sp->dim, DH_ERR_STATE, "FermionOnSphere: rank tables cover %lld of %lld states",
           (long long)running, (long long)sp->dim);
  int rc;
  sp->low_rank.release();
  sp->high_offset.release();
  if ((rc = sp->low_rank.alloc(t.low_rank.size() * sizeof(uint16_t))) != DH_OK) return rc;
  if ((rc = sp->high_offset.alloc(t.high_offset.size() * sizeof(int32_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy(sp->low_rank.ptr, t.low_rank.data(), t.low_rank.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(sp->high_offset.ptr, t.high_offset.data(), t.high_offset.size() * sizeof(int32_t),
                     cudaMemcpyHostToDevice));
  return DH_OK;
}

// counts[n][o][s]: n fermions in orbitals 0..o-1 with orbital-index sum s (o = 0 .. lz_max + 1), and
// the sector's dimension
static int fermion_counts(dh_space_s* sp) {
  const int N = sp->nbr_fermions, L = sp->lz_max, K = sp->total_sum;
  const int O = L + 2;
  DH_CHECK((double)(N + 1) * O * (K + 1) <= 64.0 * 1024 * 1024, DH_ERR_UNSUPPORTED,
           "FermionOnSphere(%d, %d, %d): the count table would exceed 64M entries", N, sp->total_lz, L);
  sp->counts.assign((size_t)(N + 1) * O * (K + 1), 0);
  auto C = [&](int n, int o, int s) -> int64_t& { return sp->counts[((size_t)n * O + o) * (K + 1) + s]; };
  for (int o = 0; o < O; ++o) C(0, o, 0) = 1;
  for (int n = 1; n <= N; ++n)
    for (int o = 1; o < O; ++o)
      for (int s = 0; s <= K; ++s) {
        int64_t v = C(n, o - 1, s);
        if (s - (o - 1) >= 0) v += C(n - 1, o - 1, s - (o - 1));
        // saturate: only counts of states of the sector (at most its dimension) are ever used
        C(n, o, s) = std::min<int64_t>(v, (int64_t)1 << 62);
      }
  const int64_t dim = C(N, L + 1, K);
  DH_CHECK(dim > 0, DH_ERR_ARGUMENT, "FermionOnSphere(%d, %d, %d): empty sector", N, sp->total_lz, L);
  DH_CHECK(dim < (1ll << 31), DH_ERR_UNSUPPORTED, "FermionOnSphere: dimension %lld >= 2^31", (long long)dim);
  sp->dim = dim;
  return DH_OK;
}

// FermionOnSphereLong (and FermionOnSphere beyond lz_max = 40): the int32 count table and the words,
// unranked on the device in the reference's order
static int build_long_fermion_space(dh_space_s* sp) {
  int rc = fermion_counts(sp);
  if (rc != DH_OK) return rc;
  const int N = sp->nbr_fermions, L = sp->lz_max, K = sp->total_sum;
  const size_t per_n = (size_t)(L + 2) * (K + 1);
  std::vector<int32_t> table((size_t)N * per_n);
  for (int n = 1; n <= N; ++n)
    for (size_t i = 0; i < per_n; ++i)
      table[(size_t)(n - 1) * per_n + i] = (int32_t)std::min<int64_t>(sp->counts[(size_t)n * per_n + i], INT32_MAX);
  if ((rc = sp->long_table.alloc(table.size() * sizeof(int32_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy(sp->long_table.ptr, table.data(), table.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  if ((rc = sp->words.alloc((size_t)sp->dim * 2 * sizeof(uint64_t))) != DH_OK) return rc;
  if ((rc = launch_long_unrank(fqhe_long_device(sp, nullptr, 0), sp->words.as<uint64_t>(), 0)) != DH_OK) return rc;
  DH_CUDA(cudaDeviceSynchronize());
  return DH_OK;
}

// a space of 64-bit words beyond the split-word tables (BosonOnSphereShort up to lz_max + N - 1 = 62):
// the count table and the words of the 128-bit engine, kept as plain uint64 words
static int build_count_rank_space(dh_space_s* sp) {
  int rc = build_long_fermion_space(sp);
  if (rc != DH_OK) return rc;
  DevBuf pairs;
  std::swap(pairs.ptr, sp->words.ptr);
  std::swap(pairs.bytes, sp->words.bytes);
  if ((rc = sp->words.alloc((size_t)sp->dim * sizeof(uint64_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy2D(sp->words.ptr, sizeof(uint64_t), pairs.ptr, 2 * sizeof(uint64_t), sizeof(uint64_t), sp->dim,
                       cudaMemcpyDeviceToDevice));
  DH_CUDA(cudaDeviceSynchronize());
  sp->count_rank = true;
  return DH_OK;
}

static int build_fermion_space(dh_space_s* sp) {
  const int N = sp->nbr_fermions, L = sp->lz_max, K = sp->total_sum;
  const int O = L + 2;  // orbital counts 0 .. L+1
  // counts[n][o][s]: n fermions in orbitals 0..o-1 with orbital-index sum s
  sp->counts.assign((size_t)(N + 1) * O * (K + 1), 0);
  auto C = [&](int n, int o, int s) -> int64_t& { return sp->counts[((size_t)n * O + o) * (K + 1) + s]; };
  for (int o = 0; o < O; ++o) C(0, o, 0) = 1;
  for (int n = 1; n <= N; ++n)
    for (int o = 1; o < O; ++o)
      for (int s = 0; s <= K; ++s) {
        int64_t v = C(n, o - 1, s);
        if (s - (o - 1) >= 0) v += C(n - 1, o - 1, s - (o - 1));
        C(n, o, s) = v;
      }
  const int64_t dim = C(N, L + 1, K);
  DH_CHECK(dim > 0, DH_ERR_ARGUMENT, "FermionOnSphere(%d, %d, %d): empty sector", N, sp->total_lz, L);
  DH_CHECK(dim < (1ll << 31), DH_ERR_UNSUPPORTED, "FermionOnSphere: dimension %lld >= 2^31", (long long)dim);
  sp->dim = dim;
  int rc = build_rank_tables(sp, 0);
  if (rc != DH_OK) return rc;
  DevBuf dcounts;
  if ((rc = dcounts.alloc(sp->counts.size() * sizeof(int64_t))) != DH_OK) return rc;
  if ((rc = sp->words.alloc((size_t)dim * sizeof(uint64_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy(dcounts.ptr, sp->counts.data(), sp->counts.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  rc = launch_fqhe_unrank(N, L, K, dim, sp->words.as<uint64_t>(), dcounts.as<int64_t>(), O * (K + 1), K + 1, 0);
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaDeviceSynchronize());
  return DH_OK;
}

// DiagHam's highest-bit lookup table (FermionOnSphere::GenerateLookUpTable, FermionOnSphere.cc:1659):
// for each highest orbital l, table[l][v] = first index of the block of states with highest orbital l
// whose prefix (word >> shift[l]) is below v, the block start for v above every prefix and the block
// end (next block start, dim - 1 for the last block) for v at or below every prefix.
int build_lookup(dh_space_s* sp) {
  if (sp->lookup.ptr) return DH_OK;
  const int L = sp->lz_max;
  // DiagHam's width from the memory budget, capped to what stays in shared memory
  unsigned long mem = sp->memory / (sizeof(int*) * (unsigned long)(L + 1));
  int bits = 1;
  while (mem > 0) {
    mem >>= 1;
    ++bits;
  }
  if (bits > L + 1) bits = L + 1;
  while (bits > 1 && (size_t)(L + 1) * (((size_t)1 << bits) + 1) * sizeof(int) > (size_t)DH_LOOKUP_SMEM_BYTES) --bits;
  sp->lookup_bits = bits;
  const int64_t dim = sp->dim;
  std::vector<uint64_t> w(dim);
  DH_CUDA(cudaMemcpy(w.data(), sp->words.ptr, dim * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  const int64_t width = ((int64_t)1 << bits) + 1;
  std::vector<int32_t> table((size_t)(L + 1) * width, -1), shift(L + 1);
  for (int l = 0; l <= L; ++l) shift[l] = (l < bits) ? 0 : l + 1 - bits;
  int64_t start = 0;
  while (start < dim) {
    const int l = 63 - __builtin_clzll(w[start] | 1ull);
    int64_t end = start;
    while (end < dim && (63 - __builtin_clzll(w[end] | 1ull)) == l) ++end;
    const int64_t block_end = (end < dim) ? end : dim - 1;
    int64_t idx = start;
    for (int64_t v = width - 1; v >= 0; --v) {
      while (idx < end && (int64_t)(w[idx] >> shift[l]) >= v) ++idx;
      table[(size_t)l * width + v] = (int32_t)((idx < end) ? idx : block_end);
    }
    start = end;
  }
  int rc;
  if ((rc = sp->lookup.alloc(table.size() * sizeof(int32_t))) != DH_OK) return rc;
  if ((rc = sp->lookup_shift.alloc(shift.size() * sizeof(int32_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy(sp->lookup.ptr, table.data(), table.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  DH_CUDA(cudaMemcpy(sp->lookup_shift.ptr, shift.data(), shift.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  return DH_OK;
}

FqheDevice fqhe_device(const dh_space_s* sp, const dh_hamiltonian_s* h, int precision) {
  FqheDevice f = {};
  f.words = sp->words.as<uint64_t>();
  f.low_rank = sp->low_rank.as<uint16_t>();
  f.high_offset = sp->high_offset.as<int32_t>();
  f.lookup = sp->lookup.as<int32_t>();
  f.lookup_shift = sp->lookup_shift.as<int32_t>();
  f.dim = sp->dim;
  f.lz_max = sp->lz_max;
  f.low_bits = sp->rank.low_bits;
  f.lookup_bits = sp->lookup_bits;
  f.index_mode = sp->index_mode;
  f.kernel_variant = sp->kernel_variant;
  f.split_form = sp->split_form;
  f.boson_lz_max = sp->boson_lz_max;
  f.nbr_bosons = (sp->kind == SPACE_BOSON) ? sp->nbr_fermions : 0;
  f.nbr_particles = sp->nbr_fermions;
  if (sp->count_rank) {
    f.count_table = sp->long_table.as<int32_t>();
    f.count_stride_o = sp->total_sum + 1;
    f.count_stride_n = (long long)(sp->lz_max + 2) * (sp->total_sum + 1);
  }
  if (h) {
    f.pair_offset = h->pair_offset.as<int32_t>();
    f.factors = (precision == DH_PRECISION_FP32) ? h->factors32.ptr : h->factors64.ptr;
    f.nbr_pairs = h->tabs.nbr_pairs;
    f.nbr_factors = h->tabs.nbr_factors;
  }
  return f;
}

FqheLongDevice fqhe_long_device(const dh_space_s* sp, const dh_hamiltonian_s* h, int precision) {
  FqheLongDevice f = {};
  f.words = sp->words.as<uint64_t>();
  f.table = sp->long_table.as<int32_t>();
  f.dim = sp->dim;
  f.nbr_fermions = sp->nbr_fermions;
  f.lz_max = sp->lz_max;
  f.total_sum = sp->total_sum;
  f.stride_o = sp->total_sum + 1;
  f.stride_n = (long long)(sp->lz_max + 2) * (sp->total_sum + 1);
  if (h) {
    f.pair_offset = h->pair_offset.as<int32_t>();
    f.factors = (precision == DH_PRECISION_FP32) ? h->factors32.ptr : h->factors64.ptr;
  }
  return f;
}

TransDevice trans_device(const dh_space_s* sp, const dh_hamiltonian_s* h) {
  TransDevice d = {};
  d.reps = sp->words.as<uint32_t>();
  d.rep_rank = sp->rep_rank.as<int32_t>();
  d.orbits = sp->rep_orbit.as<uint8_t>();
  d.map = sp->trans_map.as<unsigned long long>();
  d.table = sp->trans_table.as<int>();
  d.table_entries = sp->table_entries;
  d.table_shift = sp->table_shift;
  d.dim = sp->dim;
  d.chain_dim = sp->chain_dim;
  d.length = sp->length;
  d.momentum = sp->momentum;
  // ExponentialTable of the real Hamiltonian: cos(2 pi K m / L) (SpinChainRealHamiltonianWithTranslations.cc:204)
  const double coef = 2.0 * M_PI / (double)sp->length * (double)sp->momentum;
  for (int m = 0; m < 32; ++m) d.phase[m] = (m < sp->length) ? cos(coef * (double)m) : 0.0;
  // ExponentialTable of the complex Hamiltonian: exp(2 pi i K m / L) (SpinChainJ1J2HamiltonianWithTranslations.cc:390-397)
  for (int m = 0; m < 32; ++m) d.sine[m] = (m < sp->length) ? sin(coef * (double)m) : 0.0;
  if (h) {
    d.j1 = h->j1;
    d.j2 = h->j2;
    d.complex_phases = h->complex_phases ? 1 : 0;
  }
  return d;
}

SpinDevice spin_device(const dh_space_s* sp, const dh_hamiltonian_s* h) {
  SpinDevice s = {};
  s.words = sp->words.as<uint32_t>();
  s.dim = sp->dim;
  s.length = sp->length;
  s.nbr_up = sp->nbr_up;
  if (h) {
    s.j1 = h->j1;
    s.j2 = h->j2;
  }
  return s;
}

int upload_factors(dh_hamiltonian_s* h) {
  const InteractionTables& t = h->tabs;
  std::vector<float> f32(t.nbr_factors);
  for (int i = 0; i < t.nbr_factors; ++i) f32[i] = (float)t.factors[i];
  DH_CUDA(cudaMemcpyAsync(h->factors64.ptr, t.factors.data(), t.nbr_factors * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
  DH_CUDA(cudaMemcpyAsync(h->factors32.ptr, f32.data(), t.nbr_factors * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  return DH_OK;
}

int ensure_buffer(DevBuf& b, size_t bytes) {
  if (b.ptr && b.bytes >= bytes) return DH_OK;
  return b.alloc(bytes);
}

EllDevice ell_device(const dh_hamiltonian_s* h, int precision) {
  EllDevice e = {};
  e.slice_ptr = h->ell_slice_ptr.as<long long>();
  e.slice_len = h->ell_slice_len.as<int>();
  e.cols = h->ell_cols.as<int>();
  e.coef = h->ell_coef.as<uint16_t>();
  e.coef32 = h->ell_coef32.as<uint32_t>();
  e.payload = (h->kind == SPACE_BOSON) ? 1 : (h->kind == SPACE_FERMION_LONG ? 2 : 0);
  e.diag = precision == DH_PRECISION_FP32 ? h->diag32.ptr : h->diag64.ptr;
  e.factors = precision == DH_PRECISION_FP32 ? h->factors32.ptr : h->factors64.ptr;
  e.dim = h->space->dim;
  e.nbr_factors = h->tabs.nbr_factors;
  e.chunk = h->ell_chunk;
  return e;
}

int refresh_fast_diagonal(dh_hamiltonian_s* h) {
  if (!h->fast) return DH_OK;
  int rc;
  if (h->kind == SPACE_FERMION_LONG) {
    rc = launch_long_diag(fqhe_long_device(h->space, h, DH_PRECISION_FP64), h->factors64.as<double>(),
                          h->diag64.as<double>(), h->diag32.as<float>(), h->stream);
  } else {
    const FqheDevice f = fqhe_device(h->space, h, DH_PRECISION_FP64);
    rc = (h->kind == SPACE_BOSON)
             ? launch_boson_diag(f, h->factors64.as<double>(), h->diag64.as<double>(), h->diag32.as<float>(), h->stream)
             : launch_fqhe_diag(f, h->factors64.as<double>(), h->diag64.as<double>(), h->diag32.as<float>(), h->stream);
  }
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaStreamSynchronize(h->stream));
  return DH_OK;
}

// y (+)= H x for nvec vectors stored one after the other (stride dim); x, y device pointers.
// In FP32 mode x is converted to FP32 first and the diagonal (shift) term uses the FP64 x.
int hamiltonian_apply(dh_hamiltonian_s* h, const double* x, double* y, int nvec, int64_t first, int64_t nbr,
                      int accumulate, const float* x32_ready, cudaStream_t stream) {
  return hamiltonian_apply_rows(h, x, y, nvec, first, nbr, accumulate, x32_ready, stream, 0, 0);
}

int hamiltonian_apply_rows(dh_hamiltonian_s* h, const double* x, double* y, int nvec, int64_t first, int64_t nbr,
                           int accumulate, const float* x32_ready, cudaStream_t stream, int64_t out_first,
                           int64_t out_last) {
  dh_space_s* sp = h->space;
  const int64_t dim = hamiltonian_dim(h);
  MatvecArgs a = {};
  a.out_first = out_first;
  a.out_last = out_last;
  a.y = y;
  a.ld = 1;
  a.vstride = dim;
  a.ld_y = 1;
  a.vstride_y = dim;
  a.nbr_vectors = nvec;
  a.shift = h->shift;
  a.col_first = first;
  a.col_last = first + nbr;
  a.row_first = first;
  a.row_last = first + nbr;
  a.accumulate = accumulate;
  int rc;
  if (h->precision == DH_PRECISION_FP32) {
    const float* x32 = x32_ready;
    if (!x32) {
      if ((rc = ensure_buffer(h->x32, (size_t)dim * nvec * sizeof(float))) != DH_OK) return rc;
      if ((rc = launch_convert_f32(x, h->x32.as<float>(), dim * nvec, stream)) != DH_OK) return rc;
      x32 = h->x32.as<float>();
    }
    a.x = x32;
    a.xdiag = x;
  } else {
    a.x = x;
    a.xdiag = nullptr;
  }
  if (sp->kind == SPACE_BOSON) {
    if (h->fast && h->fast_use && first == 0 && nbr == dim) return launch_ell_product(ell_device(h, h->precision), a, h->precision, stream);
    return launch_boson_matvec(fqhe_device(sp, h, h->precision), a, h->precision, stream);
  }
  if (sp->kind == SPACE_SPIN12_TRANSLATIONS) return launch_trans_matvec(trans_device(sp, h), a, h->precision, stream);
  if (sp->kind == SPACE_FERMION_LONG) {
    if (h->fast && h->fast_use && first == 0 && nbr == dim) return launch_ell_product(ell_device(h, h->precision), a, h->precision, stream);
    return launch_long_matvec(fqhe_long_device(sp, h, h->precision), a, h->precision, stream);
  }
  if (sp->kind == SPACE_FERMION) {
    if (h->fast && h->fast_use && first == 0 && nbr == dim) return launch_ell_product(ell_device(h, h->precision), a, h->precision, stream);
    if (sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
    return launch_fqhe_matvec(fqhe_device(sp, h, h->precision), a, h->precision, stream);
  }
  return launch_spin_matvec(spin_device(sp, h), a, h->precision, stream);
}

int hamiltonian_apply_block(dh_hamiltonian_s* h, const double* x64, const float* x32, double* y, int k, int precision,
                            cudaStream_t stream) {
  return hamiltonian_apply_block_rows(h, x64, x32, y, k, precision, stream, 0, 0);
}

int hamiltonian_apply_block_rows(dh_hamiltonian_s* h, const double* x64, const float* x32, double* y, int k,
                                 int precision, cudaStream_t stream, int64_t out_first, int64_t out_last) {
  dh_space_s* sp = h->space;
  MatvecArgs a = {};
  a.out_first = out_first;
  a.out_last = out_last;
  a.y = y;
  a.ld = k;
  a.vstride = 1;
  a.ld_y = k;
  a.vstride_y = 1;
  a.nbr_vectors = k;
  a.shift = h->shift;
  a.col_first = 0;
  a.col_last = hamiltonian_dim(h);
  a.row_first = 0;
  a.row_last = hamiltonian_dim(h);
  a.accumulate = 0;
  if (precision == DH_PRECISION_FP32) {
    DH_CHECK(x32, DH_ERR_STATE, "FP32 product without an FP32 copy of the block");
    a.x = x32;
    a.xdiag = x64;
  } else {
    a.x = x64;
    a.xdiag = nullptr;
  }
  int rc;
  if (sp->kind == SPACE_BOSON) {
    if (h->fast && h->fast_use) return launch_ell_product(ell_device(h, precision), a, precision, stream);
    return launch_boson_matvec(fqhe_device(sp, h, precision), a, precision, stream);
  }
  if (sp->kind == SPACE_SPIN12_TRANSLATIONS) return launch_trans_matvec(trans_device(sp, h), a, precision, stream);
  if (sp->kind == SPACE_FERMION_LONG) {
    if (h->fast && h->fast_use) return launch_ell_product(ell_device(h, precision), a, precision, stream);
    return launch_long_matvec(fqhe_long_device(sp, h, precision), a, precision, stream);
  }
  if (sp->kind == SPACE_FERMION) {
    if (h->fast && h->fast_use) return launch_ell_product(ell_device(h, precision), a, precision, stream);
    if (sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
    return launch_fqhe_matvec(fqhe_device(sp, h, precision), a, precision, stream);
  }
  return launch_spin_matvec(spin_device(sp, h), a, precision, stream);
}

}  // namespace dh

// ===================================================================== C ABI

extern "C" {

const char* dh_last_error(void) { return dh::last_error(); }

const char* dh_version(void) { return "diagham_b200 0.1 (sm_100a)"; }

int dh_device_count(int* count) {
  DH_CHECK(count, DH_ERR_ARGUMENT, "null count");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return DH_OK;
}

int dh_fermion_on_sphere_create(int nbr_fermions, int total_lz, int lz_max, unsigned long memory, dh_space_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(nbr_fermions >= 1, DH_ERR_ARGUMENT, "FermionOnSphere: nbr_fermions must be >= 1");
  DH_CHECK(lz_max >= nbr_fermions - 1, DH_ERR_ARGUMENT, "FermionOnSphere: %d fermions do not fit in %d orbitals",
           nbr_fermions, lz_max + 1);
  DH_CHECK(lz_max <= 62, DH_ERR_UNSUPPORTED,
           "FermionOnSphere: lz_max = %d > 62 does not fit 64-bit words (FermionOnSphereLong takes up to 126)", lz_max);
  const int twice = total_lz + nbr_fermions * lz_max;
  DH_CHECK(twice >= 0 && (twice & 1) == 0, DH_ERR_ARGUMENT,
           "FermionOnSphere: total_lz = %d is not reachable by %d fermions with lz_max = %d", total_lz, nbr_fermions,
           lz_max);
  dh_space_s* sp = new (std::nothrow) dh_space_s();
  DH_CHECK(sp, DH_ERR_MEMORY, "out of host memory");
  sp->kind = SPACE_FERMION;
  sp->nbr_fermions = nbr_fermions;
  sp->lz_max = lz_max;
  sp->total_lz = total_lz;
  sp->total_sum = twice / 2;
  sp->memory = memory;
  sp->index_mode = DH_INDEX_RANK;
  if (lz_max > 40) {
    // beyond the split-word tables: the per-fermion ranks of the 128-bit engine, 64-bit words outside
    sp->kind = SPACE_FERMION_LONG;
    sp->api_halves = 1;
    int rc = build_long_fermion_space(sp);
    if (rc != DH_OK) {
      delete sp;
      return rc;
    }
    *out = sp;
    return DH_OK;
  }
  // product kernel of the rank mode: split-word (default) or the generic one (DH_FQHE_KERNEL=generic)
  // DH_FQHE_LOW_BITS sets the split of the rank tables; "smem" stages the low-rank table in shared
  // memory (the split is then lowered until the table fits in 64 KiB)
  const char* kv = getenv("DH_FQHE_KERNEL");
  sp->kernel_variant = 0;
  if (kv && strcmp(kv, "generic") == 0) sp->kernel_variant = 1;
  if (kv && strcmp(kv, "smem") == 0) sp->kernel_variant = 2;
  const char* lb = getenv("DH_FQHE_LOW_BITS");
  sp->requested_low_bits = lb ? atoi(lb) : 0;
  // DH_FQHE_SPLIT_FORM: launch form of the split-word kernel (as dh_space_set_split_form)
  const char* sf = getenv("DH_FQHE_SPLIT_FORM");
  if (sf && atoi(sf) >= 0 && atoi(sf) < kNbrSplitForms) sp->split_form = atoi(sf);
  int rc = build_fermion_space(sp);
  if (rc != DH_OK) {
    delete sp;
    return rc;
  }
  *out = sp;
  return DH_OK;
}

int dh_fermion_on_sphere_long_create(int nbr_fermions, int total_lz, int lz_max, unsigned long memory,
                                     dh_space_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(nbr_fermions >= 1, DH_ERR_ARGUMENT, "FermionOnSphereLong: nbr_fermions must be >= 1");
  DH_CHECK(lz_max >= nbr_fermions - 1, DH_ERR_ARGUMENT, "FermionOnSphereLong: %d fermions do not fit in %d orbitals",
           nbr_fermions, lz_max + 1);
  DH_CHECK(lz_max >= 1 && lz_max <= 126, DH_ERR_UNSUPPORTED, "FermionOnSphereLong: lz_max = %d not in 1..126", lz_max);
  const int twice = total_lz + nbr_fermions * lz_max;
  DH_CHECK(twice >= 0 && (twice & 1) == 0, DH_ERR_ARGUMENT,
           "FermionOnSphereLong: total_lz = %d is not reachable by %d fermions with lz_max = %d", total_lz,
           nbr_fermions, lz_max);
  dh_space_s* sp = new (std::nothrow) dh_space_s();
  DH_CHECK(sp, DH_ERR_MEMORY, "out of host memory");
  std::unique_ptr<dh_space_s> guard(sp);
  sp->kind = SPACE_FERMION_LONG;
  sp->api_halves = 2;
  sp->nbr_fermions = nbr_fermions;
  sp->lz_max = lz_max;
  sp->total_lz = total_lz;
  sp->total_sum = twice / 2;
  sp->memory = memory;
  sp->index_mode = DH_INDEX_RANK;
  int rc = build_long_fermion_space(sp);
  if (rc != DH_OK) return rc;
  *out = guard.release();
  return DH_OK;
}

int dh_boson_on_sphere_create(int nbr_bosons, int total_lz, int lz_max, unsigned long memory, dh_space_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(nbr_bosons >= 1, DH_ERR_ARGUMENT, "BosonOnSphereShort: nbr_bosons must be >= 1");
  DH_CHECK(lz_max >= 0, DH_ERR_ARGUMENT, "BosonOnSphereShort: lz_max must be >= 0");
  // the reference's BosonOnSphereShort range (BosonOnSphere from lz_max + N - 1 = 63 on,
  // ParticleOnSphereManager.cc:487)
  DH_CHECK(lz_max + nbr_bosons - 1 <= 62, DH_ERR_UNSUPPORTED,
           "BosonOnSphereShort: lz_max + N - 1 = %d > 62 needs the reference's BosonOnSphere", lz_max + nbr_bosons - 1);
  const int twice = total_lz + nbr_bosons * lz_max;
  DH_CHECK(twice >= 0 && (twice & 1) == 0 && twice <= 2 * nbr_bosons * lz_max, DH_ERR_ARGUMENT,
           "BosonOnSphereShort: total_lz = %d is not reachable by %d bosons with lz_max = %d", total_lz, nbr_bosons,
           lz_max);
  dh_space_s* sp = new (std::nothrow) dh_space_s();
  DH_CHECK(sp, DH_ERR_MEMORY, "out of host memory");
  // BosonOnSphereShort.cc:83-93: the basis is FermionOnSphere(N, totalLz, lzMax + N - 1)
  sp->kind = SPACE_BOSON;
  sp->nbr_fermions = nbr_bosons;
  sp->lz_max = lz_max + nbr_bosons - 1;
  sp->boson_lz_max = lz_max;
  sp->total_lz = total_lz;
  sp->total_sum = (total_lz + nbr_bosons * sp->lz_max) / 2;
  sp->memory = memory;
  sp->index_mode = DH_INDEX_RANK;
  sp->kernel_variant = 1;
  const char* lb = getenv("DH_FQHE_LOW_BITS");
  sp->requested_low_bits = lb ? atoi(lb) : 0;
  // up to 40 bits the split-word rank tables; beyond, ranks from the sector's count table
  int rc = (sp->lz_max <= 40) ? build_fermion_space(sp) : build_count_rank_space(sp);
  if (rc != DH_OK) {
    delete sp;
    return rc;
  }
  *out = sp;
  return DH_OK;
}

int dh_spin12_chain_translations_create(int chain_length, int momentum, int sz, int memory, dh_space_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  (void)memory;
  DH_CHECK(chain_length >= 3 && chain_length <= 32, DH_ERR_UNSUPPORTED,
           "Spin1_2ChainWithTranslations: chain length %d not in 3..32", chain_length);
  DH_CHECK(((chain_length + sz) & 1) == 0 && sz >= -chain_length && sz <= chain_length, DH_ERR_ARGUMENT,
           "Spin1_2ChainWithTranslations: sz = %d is not reachable with %d spins", sz, chain_length);
  DH_CHECK(momentum >= 0 && momentum < chain_length, DH_ERR_ARGUMENT, "momentum %d not in 0..%d", momentum,
           chain_length - 1);
  dh_space_s* sp = new (std::nothrow) dh_space_s();
  DH_CHECK(sp, DH_ERR_MEMORY, "out of host memory");
  std::unique_ptr<dh_space_s> guard(sp);
  sp->kind = SPACE_SPIN12_TRANSLATIONS;
  sp->length = chain_length;
  sp->sz = sz;
  sp->nbr_up = (chain_length + sz) / 2;
  sp->momentum = momentum;
  sp->index_mode = DH_INDEX_RANK;
  long long total = 1;
  for (int q = 1; q <= sp->nbr_up; ++q) total = total * (chain_length - sp->nbr_up + q) / q;
  sp->chain_dim = total;
  // representatives in ascending order: per chunk of 1024 words a count, a scan of the counts, then
  // each chunk writes its representatives at its offset (Spin1_2ChainWithTranslations.cc:167-235)
  const long long chunks = (total + 1023) / 1024;
  DevBuf counts, offsets;
  int rc;
  if ((rc = counts.alloc(chunks * sizeof(unsigned int))) != DH_OK) return rc;
  if ((rc = launch_trans_count(total, chain_length, sp->nbr_up, momentum, counts.as<unsigned int>(), 0)) != DH_OK)
    return rc;
  std::vector<unsigned int> hc(chunks);
  DH_CUDA(cudaMemcpy(hc.data(), counts.ptr, chunks * sizeof(unsigned int), cudaMemcpyDeviceToHost));
  std::vector<long long> ho(chunks);
  long long dim = 0;
  for (long long c = 0; c < chunks; ++c) {
    ho[c] = dim;
    dim += hc[c];
  }
  sp->dim = dim;
  if (dim > 0) {
    // the whole-sector map (DH_TRANS_MAP=1) or, by default, flipped words canonicalised in the kernels
    const char* tm = getenv("DH_TRANS_MAP");
    const bool with_map = tm && atoi(tm) != 0;
    if ((rc = offsets.alloc(chunks * sizeof(long long))) != DH_OK ||
        (rc = sp->words.alloc(dim * sizeof(uint32_t))) != DH_OK || (rc = sp->rep_orbit.alloc(dim)) != DH_OK)
      return rc;
    if (with_map && ((rc = sp->rep_rank.alloc(dim * sizeof(int32_t))) != DH_OK ||
                     (rc = sp->trans_map.alloc(total * sizeof(unsigned long long))) != DH_OK))
      return rc;
    DH_CUDA(cudaMemcpy(offsets.ptr, ho.data(), chunks * sizeof(long long), cudaMemcpyHostToDevice));
    if ((rc = launch_trans_write(total, chain_length, sp->nbr_up, momentum, offsets.as<long long>(),
                                 sp->words.as<uint32_t>(), sp->rep_orbit.as<uint8_t>(), 0)) != DH_OK)
      return rc;
    // lookup over the representatives: at most 2^24 + 2 entries of the top bits
    uint32_t last = 0;
    DH_CUDA(cudaMemcpy(&last, sp->words.as<uint32_t>() + (dim - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost));
    const int bits = last ? 32 - __builtin_clz(last) : 1;
    sp->table_shift = bits > 24 ? bits - 24 : 0;
    sp->table_entries = (long long)(last >> sp->table_shift) + 2;
    if ((rc = sp->trans_table.alloc(sp->table_entries * sizeof(int))) != DH_OK) return rc;
    if ((rc = launch_trans_table(sp->words.as<uint32_t>(), dim, sp->table_shift, sp->table_entries,
                                 sp->trans_table.as<int>(), 0)) != DH_OK)
      return rc;
    if (with_map && (rc = launch_trans_map(trans_device(sp, nullptr), total, sp->nbr_up, 0)) != DH_OK) return rc;
    DH_CUDA(cudaDeviceSynchronize());
  }
  *out = guard.release();
  return DH_OK;
}

int dh_spin12_chain_create(int chain_length, int sz, int memory, dh_space_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  (void)memory;
  DH_CHECK(chain_length >= 1 && chain_length <= 32, DH_ERR_UNSUPPORTED, "Spin1_2Chain: chain length %d not in 1..32",
           chain_length);
  DH_CHECK(((chain_length + sz) & 1) == 0 && sz >= -chain_length && sz <= chain_length, DH_ERR_ARGUMENT,
           "Spin1_2Chain: sz = %d is not reachable with %d spins", sz, chain_length);
  dh_space_s* sp = new (std::nothrow) dh_space_s();
  DH_CHECK(sp, DH_ERR_MEMORY, "out of host memory");
  sp->kind = SPACE_SPIN12;
  sp->length = chain_length;
  sp->sz = sz;
  sp->nbr_up = (chain_length + sz) / 2;
  long long c = 1;
  for (int q = 1; q <= sp->nbr_up; ++q) c = c * (chain_length - sp->nbr_up + q) / q;
  sp->dim = c;
  sp->index_mode = DH_INDEX_RANK;
  int rc = sp->words.alloc((size_t)sp->dim * sizeof(uint32_t));
  if (rc == DH_OK) rc = launch_spin_unrank(chain_length, sp->nbr_up, sp->dim, sp->words.as<uint32_t>(), 0);
  if (rc == DH_OK && cudaDeviceSynchronize() != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "unrank", __FILE__, __LINE__);
  if (rc != DH_OK) {
    delete sp;
    return rc;
  }
  *out = sp;
  return DH_OK;
}

int dh_space_destroy(dh_space_t space) {
  delete space;
  return DH_OK;
}

int dh_space_get_dimension(dh_space_t space, int64_t* dim) {
  DH_CHECK(space && dim, DH_ERR_ARGUMENT, "null argument");
  *dim = space->dim;
  return DH_OK;
}

int dh_space_get_states(dh_space_t sp, uint64_t* words, int* lz_max, int64_t first, int64_t n) {
  DH_CHECK(sp && words, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(first >= 0 && n >= 0 && first + n <= sp->dim, DH_ERR_ARGUMENT, "state range out of bounds");
  if (n == 0) return DH_OK;
  if (sp->kind == SPACE_FERMION || sp->kind == SPACE_BOSON) {
    DH_CUDA(cudaMemcpy(words, sp->words.as<uint64_t>() + first, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    if (lz_max)
      for (int64_t i = 0; i < n; ++i) lz_max[i] = words[i] ? 63 - __builtin_clzll(words[i]) : 0;
  } else if (sp->kind == SPACE_FERMION_LONG) {
    DH_CHECK(sp->lz_max <= 63, DH_ERR_UNSUPPORTED,
             "lz_max = %d: the states are 128-bit words (dh_space_get_states_long)", sp->lz_max);
    // the low halves of the (low, high) pairs
    DH_CUDA(cudaMemcpy2D(words, sizeof(uint64_t), sp->words.as<uint64_t>() + 2 * first, 2 * sizeof(uint64_t),
                         sizeof(uint64_t), n, cudaMemcpyDeviceToHost));
    if (lz_max)
      for (int64_t i = 0; i < n; ++i) lz_max[i] = words[i] ? 63 - __builtin_clzll(words[i]) : 0;
  } else if (sp->kind == SPACE_SPIN12_TRANSLATIONS) {
    std::vector<uint32_t> w(n);
    DH_CUDA(cudaMemcpy(w.data(), sp->words.as<uint32_t>() + first, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) words[i] = w[i];
    if (lz_max)
      for (int64_t i = 0; i < n; ++i) lz_max[i] = 0;
  } else {
    std::vector<uint32_t> w(n);
    DH_CUDA(cudaMemcpy(w.data(), sp->words.as<uint32_t>() + first, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // the reference starts from 0xffffffff, so sites L..31 stay set (Spin1_2Chain.cc:137-138)
    const uint64_t high = (sp->length < 32) ? (0xffffffffull & ~((1ull << sp->length) - 1ull)) : 0ull;
    for (int64_t i = 0; i < n; ++i) words[i] = (uint64_t)w[i] | high;
    if (lz_max)
      for (int64_t i = 0; i < n; ++i) lz_max[i] = 0;
  }
  return DH_OK;
}

int dh_space_get_states_long(dh_space_t sp, uint64_t* words, int* lz_max, int64_t first, int64_t n) {
  DH_CHECK(sp && words, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(sp->kind == SPACE_FERMION || sp->kind == SPACE_FERMION_LONG, DH_ERR_UNSUPPORTED,
           "128-bit words exist for fermion spaces");
  DH_CHECK(first >= 0 && n >= 0 && first + n <= sp->dim, DH_ERR_ARGUMENT, "state range out of bounds");
  if (n == 0) return DH_OK;
  if (sp->kind == SPACE_FERMION) {
    DH_CUDA(cudaMemcpy2D(words, 2 * sizeof(uint64_t), sp->words.as<uint64_t>() + first, sizeof(uint64_t),
                         sizeof(uint64_t), n, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; ++i) words[2 * i + 1] = 0;
  } else {
    DH_CUDA(cudaMemcpy(words, sp->words.as<uint64_t>() + 2 * first, n * 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  }
  if (lz_max)
    for (int64_t i = 0; i < n; ++i) {
      const uint64_t lo = words[2 * i], hi = words[2 * i + 1];
      lz_max[i] = hi ? 127 - __builtin_clzll(hi) : (lo ? 63 - __builtin_clzll(lo) : 0);
    }
  return DH_OK;
}

int dh_space_find_state_index_long(dh_space_t sp, const uint64_t* words, int64_t n, int64_t* indices) {
  DH_CHECK(sp && words && indices, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(sp->kind == SPACE_FERMION || sp->kind == SPACE_FERMION_LONG, DH_ERR_UNSUPPORTED,
           "128-bit words exist for fermion spaces");
  if (n <= 0) return DH_OK;
  std::vector<uint64_t> host;
  const uint64_t* src = words;
  if (is_device_pointer(words)) {
    host.resize(2 * n);
    DH_CUDA(cudaMemcpy(host.data(), words, 2 * n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    src = host.data();
  }
  if (sp->kind == SPACE_FERMION) {
    // words with high bits are not states of a 64-bit space
    std::vector<uint64_t> low(n);
    std::vector<int64_t> idx(n);
    for (int64_t i = 0; i < n; ++i) low[i] = src[2 * i];
    int rc = dh_space_find_state_index(sp, low.data(), n, idx.data());
    if (rc != DH_OK) return rc;
    for (int64_t i = 0; i < n; ++i)
      if (src[2 * i + 1]) idx[i] = -1;
    if (is_device_pointer(indices))
      DH_CUDA(cudaMemcpy(indices, idx.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    else
      memcpy(indices, idx.data(), n * sizeof(int64_t));
    return DH_OK;
  }
  DevBuf dw, di;
  int rc;
  if ((rc = dw.alloc(2 * n * sizeof(uint64_t))) != DH_OK || (rc = di.alloc(n * sizeof(int64_t))) != DH_OK) return rc;
  DH_CUDA(cudaMemcpy(dw.ptr, src, 2 * n * sizeof(uint64_t), cudaMemcpyHostToDevice));
  if ((rc = launch_long_find(fqhe_long_device(sp, nullptr, 0), dw.as<uint64_t>(), n, di.as<long long>(), 0)) != DH_OK)
    return rc;
  DH_CUDA(cudaDeviceSynchronize());
  DH_CUDA(cudaMemcpy(indices, di.ptr, n * sizeof(int64_t),
                     is_device_pointer(indices) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  return DH_OK;
}

int dh_space_set_index_mode(dh_space_t sp, int mode) {
  DH_CHECK(sp, DH_ERR_ARGUMENT, "null space");
  DH_CHECK(mode == DH_INDEX_RANK || mode == DH_INDEX_LOOKUP, DH_ERR_ARGUMENT, "unknown index mode %d", mode);
  DH_CHECK(sp->kind == SPACE_FERMION || mode == DH_INDEX_RANK, DH_ERR_UNSUPPORTED,
           "the spin chain and the boson space use their rank tables only");
  if (mode == DH_INDEX_LOOKUP) {
    int rc = build_lookup(sp);
    if (rc != DH_OK) return rc;
  }
  sp->index_mode = mode;
  return DH_OK;
}

int dh_space_set_split_form(dh_space_t sp, int form) {
  DH_CHECK(sp, DH_ERR_ARGUMENT, "null space");
  DH_CHECK(form >= 0 && form < kNbrSplitForms && kNbrSplitForms == DH_SPLIT_FORMS, DH_ERR_ARGUMENT,
           "launch form %d not in 0..%d", form, kNbrSplitForms - 1);
  sp->split_form = form;
  return DH_OK;
}

int dh_space_find_state_index(dh_space_t sp, const uint64_t* words, int64_t n, int64_t* indices) {
  DH_CHECK(sp && words && indices, DH_ERR_ARGUMENT, "null argument");
  if (n <= 0) return DH_OK;
  DevBuf dw, di;
  const uint64_t* w = words;
  int64_t* out = indices;
  const bool in_dev = is_device_pointer(words), out_dev = is_device_pointer(indices);
  int rc;
  if (!in_dev) {
    if ((rc = dw.alloc(n * sizeof(uint64_t))) != DH_OK) return rc;
    DH_CUDA(cudaMemcpy(dw.ptr, words, n * sizeof(uint64_t), cudaMemcpyHostToDevice));
    w = dw.as<uint64_t>();
  }
  if (!out_dev) {
    if ((rc = di.alloc(n * sizeof(int64_t))) != DH_OK) return rc;
    out = di.as<int64_t>();
  }
  if ((sp->kind == SPACE_FERMION || sp->kind == SPACE_BOSON) && !sp->count_rank) {
    if (sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
    rc = launch_fqhe_find(fqhe_device(sp, nullptr, 0), w, n, reinterpret_cast<long long*>(out), 0);
  } else if (sp->kind == SPACE_FERMION_LONG || sp->count_rank) {
    // 64-bit words as (word, 0) pairs
    DevBuf pairs;
    if ((rc = pairs.alloc(2 * n * sizeof(uint64_t))) != DH_OK) return rc;
    DH_CUDA(cudaMemset(pairs.ptr, 0, 2 * n * sizeof(uint64_t)));
    DH_CUDA(cudaMemcpy2D(pairs.ptr, 2 * sizeof(uint64_t), w, sizeof(uint64_t), sizeof(uint64_t), n,
                         cudaMemcpyDeviceToDevice));
    rc = launch_long_find(fqhe_long_device(sp, nullptr, 0), pairs.as<uint64_t>(), n, reinterpret_cast<long long*>(out), 0);
    if (rc == DH_OK) DH_CUDA(cudaDeviceSynchronize());
  } else if (sp->kind == SPACE_SPIN12_TRANSLATIONS) {
    rc = launch_trans_find(trans_device(sp, nullptr), w, n, reinterpret_cast<long long*>(out), 0);
  } else {
    rc = launch_spin_find(spin_device(sp, nullptr), w, n, reinterpret_cast<long long*>(out), 0);
  }
  if (rc != DH_OK) return rc;
  DH_CUDA(cudaDeviceSynchronize());
  if (!out_dev) DH_CUDA(cudaMemcpy(indices, out, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
  return DH_OK;
}

// ----------------------------------------------------------- Hamiltonians

int dh_particle_on_sphere_generic_hamiltonian_create(dh_space_t sp, int nbr_particles, int lz_max,
                                                     const double* pseudopotentials, double l2_factor,
                                                     dh_hamiltonian_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(sp && pseudopotentials, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(sp->kind == SPACE_FERMION || sp->kind == SPACE_FERMION_LONG || sp->kind == SPACE_BOSON, DH_ERR_ARGUMENT,
           "ParticleOnSphereGenericHamiltonian needs a FermionOnSphere(Long) or BosonOnSphereShort space");
  const bool bosons = sp->kind == SPACE_BOSON;
  const int space_lz_max = bosons ? sp->boson_lz_max : sp->lz_max;
  DH_CHECK(nbr_particles == sp->nbr_fermions && lz_max == space_lz_max, DH_ERR_ARGUMENT,
           "Hamiltonian (N = %d, lz_max = %d) does not match its space (N = %d, lz_max = %d)", nbr_particles, lz_max,
           sp->nbr_fermions, space_lz_max);
  DH_CHECK(l2_factor == 0.0 || nbr_particles >= 2, DH_ERR_UNSUPPORTED, "an L^2 term needs at least two particles");
  dh_hamiltonian_s* h = new (std::nothrow) dh_hamiltonian_s();
  DH_CHECK(h, DH_ERR_MEMORY, "out of host memory");
  h->space = sp;
  h->kind = sp->kind;
  // the particle statistics of the space select the factors, as Particles->GetParticleStatistic()
  // does in EvaluateInteractionFactors (ParticleOnSphereGenericHamiltonian.cc:514)
  if (bosons)
    h->tabs.build_bosons(lz_max);
  else
    h->tabs.build(lz_max);
  if (l2_factor != 0.0) {
    // ParticleOnSphereGenericHamiltonian adds l2Factor L^2 (its L2Operator): a two-body table on top
    // of the interaction's, and the constant l2Factor (Lz^2 + Lz) in the shift
    h->tabs.build_l2(nbr_particles);
    h->tabs.l2_factor = l2_factor;
    h->shift_base = l2_factor * l2_constant(sp->total_lz);
    h->shift = h->shift_base;
  }
  h->v.assign(pseudopotentials, pseudopotentials + lz_max + 1);
  h->tabs.set_pseudopotentials(h->v.data());
  int rc;
  if ((rc = h->pair_offset.alloc(h->tabs.pair_offset.size() * sizeof(int32_t))) != DH_OK ||
      (rc = h->factors64.alloc(h->tabs.nbr_factors * sizeof(double))) != DH_OK ||
      (rc = h->factors32.alloc(h->tabs.nbr_factors * sizeof(float))) != DH_OK ||
      (rc = reducer_init(h->red, h->red_storage, 16)) != DH_OK) {
    delete h;
    return rc;
  }
  if (cudaMemcpy(h->pair_offset.ptr, h->tabs.pair_offset.data(), h->tabs.pair_offset.size() * sizeof(int32_t),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    delete h;
    return cuda_fail(cudaGetLastError(), "upload pair offsets", __FILE__, __LINE__);
  }
  if ((rc = upload_factors(h)) != DH_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return DH_OK;
}

int dh_particle_on_sphere_l2_hamiltonian_create(dh_space_t sp, int nbr_particles, int lz_max, int total_lz,
                                                double l2_factor, dh_hamiltonian_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(sp && (sp->kind == SPACE_FERMION || sp->kind == SPACE_FERMION_LONG || sp->kind == SPACE_BOSON),
           DH_ERR_ARGUMENT, "ParticleOnSphereL2Hamiltonian needs a FermionOnSphere(Long) or BosonOnSphereShort space");
  DH_CHECK(total_lz == sp->total_lz, DH_ERR_ARGUMENT, "total_lz %d does not match the space's %d", total_lz, sp->total_lz);
  DH_CHECK(l2_factor != 0.0, DH_ERR_ARGUMENT, "l2_factor must not be 0");
  std::vector<double> zero(lz_max + 1, 0.0);
  int rc = dh_particle_on_sphere_generic_hamiltonian_create(sp, nbr_particles, lz_max, zero.data(), l2_factor, out);
  if (rc != DH_OK) return rc;
  (*out)->l2_only = true;
  return DH_OK;
}

static int j1j2_create(dh_space_t sp, double j1, double j2, bool complex_phases, dh_hamiltonian_t* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  DH_CHECK(sp && (sp->kind == SPACE_SPIN12 || sp->kind == SPACE_SPIN12_TRANSLATIONS), DH_ERR_ARGUMENT,
           "the J1-J2 chain needs a Spin1_2Chain or Spin1_2ChainWithTranslations space");
  DH_CHECK(!complex_phases || sp->kind == SPACE_SPIN12_TRANSLATIONS, DH_ERR_ARGUMENT,
           "the complex J1-J2 Hamiltonian needs a Spin1_2ChainWithTranslations space");
  DH_CHECK(sp->length >= 3, DH_ERR_UNSUPPORTED, "the periodic J1-J2 chain needs at least 3 sites");
  // the real Hamiltonian of a momentum sector (SpinChainJ1J2RealHamiltonianWithTranslations) is the
  // Hamiltonian only where the phases are real: K = 0 and K = L / 2
  DH_CHECK(complex_phases || sp->kind != SPACE_SPIN12_TRANSLATIONS || sp->momentum == 0 || 2 * sp->momentum == sp->length,
           DH_ERR_UNSUPPORTED, "momentum %d of %d sites needs complex arithmetic (K = 0 or L / 2 only)", sp->momentum,
           sp->length);
  dh_hamiltonian_s* h = new (std::nothrow) dh_hamiltonian_s();
  DH_CHECK(h, DH_ERR_MEMORY, "out of host memory");
  h->space = sp;
  h->kind = sp->kind;
  h->j1 = j1;
  h->j2 = j2;
  h->complex_phases = complex_phases;
  int rc = reducer_init(h->red, h->red_storage, 16);
  if (rc != DH_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return DH_OK;
}

int dh_spin_chain_j1j2_hamiltonian_create(dh_space_t sp, double j1, double j2, dh_hamiltonian_t* out) {
  return j1j2_create(sp, j1, j2, false, out);
}

int dh_spin_chain_j1j2_complex_hamiltonian_create(dh_space_t sp, double j1, double j2, dh_hamiltonian_t* out) {
  return j1j2_create(sp, j1, j2, true, out);
}

int dh_hamiltonian_destroy(dh_hamiltonian_t h) {
  delete h;
  return DH_OK;
}

int dh_hamiltonian_get_dimension(dh_hamiltonian_t h, int64_t* dim) {
  DH_CHECK(h && dim, DH_ERR_ARGUMENT, "null argument");
  *dim = hamiltonian_dim(h);
  return DH_OK;
}

int dh_hamiltonian_shift(dh_hamiltonian_t h, double shift) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  h->shift = shift + h->shift_base;
  return DH_OK;
}

int dh_hamiltonian_set_precision(dh_hamiltonian_t h, int precision) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  DH_CHECK(precision == DH_PRECISION_FP64 || precision == DH_PRECISION_FP32, DH_ERR_ARGUMENT, "unknown precision %d",
           precision);
  h->precision = precision;
  return DH_OK;
}

int dh_hamiltonian_set_pseudopotentials(dh_hamiltonian_t h, const double* v) {
  DH_CHECK(h && v, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK((h->kind == SPACE_FERMION || h->kind == SPACE_FERMION_LONG || h->kind == SPACE_BOSON) && !h->l2_only,
           DH_ERR_ARGUMENT, "pseudopotentials only apply to FQHE interaction Hamiltonians");
  h->v.assign(v, v + h->tabs.lz_max + 1);
  h->tabs.set_pseudopotentials(h->v.data());
  int rc = upload_factors(h);
  if (rc != DH_OK) return rc;
  return refresh_fast_diagonal(h);  // the stored elements hold factor indices: only the diagonal changes
}

int dh_hamiltonian_enable_fast_multiplication(dh_hamiltonian_t h, int64_t allowed_memory, int* enabled,
                                              int64_t* bytes) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  if (enabled) *enabled = 0;
  if (bytes) *bytes = 0;
  DH_CHECK(h->kind == SPACE_FERMION || h->kind == SPACE_BOSON || h->kind == SPACE_FERMION_LONG, DH_ERR_UNSUPPORTED,
           "stored elements are available for FermionOnSphere(Long) and BosonOnSphereShort Hamiltonians");
  const bool bosons = h->kind == SPACE_BOSON;
  const bool wide = h->kind == SPACE_FERMION_LONG;  // uint32 index | sign payloads
  DH_CHECK(h->tabs.nbr_factors < (wide ? 0x7fffffff : bosons ? 0x10000 : 0x8000), DH_ERR_UNSUPPORTED,
           "%d interaction factors do not fit %d-bit indices", h->tabs.nbr_factors, wide ? 31 : bosons ? 16 : 15);
  DH_CHECK(h->space->dim < (1ll << 31), DH_ERR_UNSUPPORTED, "stored elements hold int32 targets");
  // a bosonic element keeps n_m2 (n_m1 - [m1 = m2]) <= N (N - 1) and its creation product in 8 bits each
  DH_CHECK(!bosons || h->space->nbr_fermions <= 16, DH_ERR_UNSUPPORTED,
           "stored bosonic elements hold occupation products of at most 16 bosons (N = %d)", h->space->nbr_fermions);
  if (h->fast) {
    if (enabled) *enabled = 1;
    if (bytes) *bytes = (int64_t)h->fast_bytes;
    return DH_OK;
  }
  dh_space_s* sp = h->space;
  const long long dim = sp->dim;
  const FqheDevice f = fqhe_device(sp, h, DH_PRECISION_FP64);
  int rc;
  // per-row element counts, then the slices (32 rows, padded to the longest) and their offsets
  std::vector<int> counts(dim);
  {
    DevBuf dcounts;
    if ((rc = dcounts.alloc((size_t)dim * sizeof(int))) != DH_OK) return rc;
    if ((rc = wide     ? launch_long_row_counts(fqhe_long_device(sp, h, DH_PRECISION_FP64), dcounts.as<int>(), h->stream)
              : bosons ? launch_boson_row_counts(f, dcounts.as<int>(), h->stream)
                       : launch_fqhe_row_counts(f, dcounts.as<int>(), h->stream)) != DH_OK)
      return rc;
    DH_CUDA(cudaMemcpyAsync(counts.data(), dcounts.ptr, (size_t)dim * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    DH_CUDA(cudaStreamSynchronize(h->stream));
  }
  const long long nslices = (dim + 31) / 32;
  std::vector<long long> slice_ptr(nslices);
  std::vector<int> slice_len(nslices);
  long long total = 0;
  for (long long sl = 0; sl < nslices; ++sl) {
    int mx = 0;
    for (long long r = sl * 32; r < std::min(dim, sl * 32 + 32); ++r) mx = std::max(mx, counts[r]);
    mx = (mx + kEllPad - 1) / kEllPad * kEllPad;  // the product reads whole chunks
    slice_ptr[sl] = total;
    slice_len[sl] = mx;
    total += 32ll * mx;
  }
  const size_t payload = (bosons || wide) ? sizeof(uint32_t) : sizeof(uint16_t);
  const size_t need = (size_t)total * (sizeof(int) + payload) + (size_t)nslices * (sizeof(long long) + sizeof(int)) +
                      (size_t)dim * (sizeof(double) + sizeof(float));
  if (bytes) *bytes = (int64_t)need;
  if (allowed_memory >= 0 && need > (size_t)allowed_memory) return DH_OK;  // the caller's memory budget
  size_t free_b = 0, total_b = 0;
  DH_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (need > free_b / 10 * 9) return DH_OK;
  if ((rc = h->ell_slice_ptr.alloc((size_t)nslices * sizeof(long long))) != DH_OK ||
      (rc = h->ell_slice_len.alloc((size_t)nslices * sizeof(int))) != DH_OK ||
      (rc = h->ell_cols.alloc((size_t)total * sizeof(int))) != DH_OK ||
      (rc = ((bosons || wide) ? h->ell_coef32 : h->ell_coef).alloc((size_t)total * payload)) != DH_OK ||
      (rc = h->diag64.alloc((size_t)dim * sizeof(double))) != DH_OK ||
      (rc = h->diag32.alloc((size_t)dim * sizeof(float))) != DH_OK)
    return rc;
  DH_CUDA(cudaMemcpyAsync(h->ell_slice_ptr.ptr, slice_ptr.data(), slice_ptr.size() * sizeof(long long),
                          cudaMemcpyHostToDevice, h->stream));
  DH_CUDA(cudaMemcpyAsync(h->ell_slice_len.ptr, slice_len.data(), slice_len.size() * sizeof(int), cudaMemcpyHostToDevice,
                          h->stream));
  if ((rc = wide ? launch_long_ell_fill(fqhe_long_device(sp, h, DH_PRECISION_FP64), h->tabs.nbr_factors,
                                        h->ell_slice_ptr.as<long long>(), h->ell_slice_len.as<int>(),
                                        h->ell_cols.as<int>(), h->ell_coef32.as<uint32_t>(), h->stream)
              : bosons ? launch_boson_ell_fill(f, h->ell_slice_ptr.as<long long>(), h->ell_slice_len.as<int>(),
                                               h->ell_cols.as<int>(), h->ell_coef32.as<uint32_t>(), h->stream)
                       : launch_fqhe_ell_fill(f, h->ell_slice_ptr.as<long long>(), h->ell_slice_len.as<int>(),
                                              h->ell_cols.as<int>(), h->ell_coef.as<uint16_t>(), h->stream)) != DH_OK)
    return rc;
  h->fast = true;
  h->fast_use = true;
  h->fast_elements = total;
  h->fast_bytes = need;
  if ((rc = refresh_fast_diagonal(h)) != DH_OK) return rc;
  if (enabled) *enabled = 1;
  return DH_OK;
}

int dh_hamiltonian_disable_fast_multiplication(dh_hamiltonian_t h) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->fast = false;
  h->fast_elements = 0;
  h->fast_bytes = 0;
  h->ell_slice_ptr.release();
  h->ell_slice_len.release();
  h->ell_cols.release();
  h->ell_coef.release();
  h->ell_coef32.release();
  h->diag64.release();
  h->diag32.release();
  return DH_OK;
}

int dh_hamiltonian_set_stream(dh_hamiltonian_t h, void* stream) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  h->stream = static_cast<cudaStream_t>(stream);
  return DH_OK;
}

// A product whose result goes to host memory: the rows are computed in up to kCopyChunks chunks on
// the handle's stream, and each chunk's rows are copied to the host on a second stream as soon as
// they are done, so the copy of all but the last chunk overlaps the product.  run(r0, r1) enqueues
// the product of rows [r0, r1) on h->stream; copy(r0, r1, s) enqueues their device-to-host copy on s.
extern "C++" {
template <typename Run, typename Copy>
static int product_to_host(dh_hamiltonian_s* h, int64_t dim, Run run, Copy copy) {
  // chunks of at least 2^18 rows, boundaries on multiples of 256 rows (slices of the stored form)
  int chunks = (int)std::min<int64_t>(dh_hamiltonian_s::kCopyChunks, std::max<int64_t>(1, dim >> 18));
  if (chunks > 1 && !h->copy_stream) {
    if (cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      h->copy_stream = nullptr;
    }
    for (int c = 0; h->copy_stream && c < dh_hamiltonian_s::kCopyChunks; ++c)
      DH_CUDA(cudaEventCreateWithFlags(&h->chunk_done[c], cudaEventDisableTiming));
  }
  if (!h->copy_stream) chunks = 1;
  int rc;
  if (chunks == 1) {
    if ((rc = run(0, dim)) != DH_OK) return rc;
    if ((rc = copy(0, dim, h->stream)) != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(h->stream));
    return DH_OK;
  }
  const int64_t step = ((dim + chunks - 1) / chunks + 255) & ~(int64_t)255;
  for (int c = 0; c < chunks; ++c) {
    const int64_t r0 = (int64_t)c * step, r1 = std::min(dim, r0 + step);
    if (r0 >= r1) break;
    if ((rc = run(r0, r1)) != DH_OK) return rc;
    DH_CUDA(cudaEventRecord(h->chunk_done[c], h->stream));
    DH_CUDA(cudaStreamWaitEvent(h->copy_stream, h->chunk_done[c], 0));
    if ((rc = copy(r0, r1, h->copy_stream)) != DH_OK) return rc;
  }
  DH_CUDA(cudaStreamSynchronize(h->copy_stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  return DH_OK;
}
}  // extern "C++"

static int multiply_common(dh_hamiltonian_t h, const double* src, double* dst, int nvec, int64_t first, int64_t nbr,
                           int accumulate) {
  DH_CHECK(h && src && dst, DH_ERR_ARGUMENT, "null argument");
  const int64_t dim = hamiltonian_dim(h);
  if (nbr < 0) nbr = dim - first;
  DH_CHECK(!h->complex_phases || ((first | nbr) & 1) == 0, DH_ERR_ARGUMENT,
           "complex components come in (Re, Im) pairs: first and nbr must be even");
  DH_CHECK(first >= 0 && first + nbr <= dim, DH_ERR_ARGUMENT, "component range [%lld, %lld) outside [0, %lld)",
           (long long)first, (long long)(first + nbr), (long long)dim);
  DH_CHECK(nvec >= 1, DH_ERR_ARGUMENT, "nbr_vectors must be >= 1");
  const size_t bytes = (size_t)dim * nvec * sizeof(double);
  const bool src_dev = is_device_pointer(src), dst_dev = is_device_pointer(dst);
  const double* x = src;
  double* y = dst;
  int rc;
  if (!src_dev) {
    if ((rc = ensure_buffer(h->stage_x, bytes)) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(h->stage_x.ptr, src, bytes, cudaMemcpyHostToDevice, h->stream));
    x = h->stage_x.as<double>();
  }
  if (!dst_dev) {
    if ((rc = ensure_buffer(h->stage_y, bytes)) != DH_OK) return rc;
    if (accumulate) DH_CUDA(cudaMemcpyAsync(h->stage_y.ptr, dst, bytes, cudaMemcpyHostToDevice, h->stream));
    y = h->stage_y.as<double>();
  }
  // LowLevelMultiply clears the destination, then adds (AbstractHamiltonian.cc:475-476); the pull
  // kernels write every row, so "clear then add" is a plain store (accumulate = 0)
  if (dst_dev) {
    if ((rc = hamiltonian_apply(h, x, y, nvec, first, nbr, accumulate, nullptr, h->stream)) != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(h->stream));
    return DH_OK;
  }
  const float* x32 = nullptr;
  if (h->precision == DH_PRECISION_FP32) {
    if ((rc = ensure_buffer(h->x32, (size_t)dim * nvec * sizeof(float))) != DH_OK) return rc;
    if ((rc = launch_convert_f32(x, h->x32.as<float>(), dim * nvec, h->stream)) != DH_OK) return rc;
    x32 = h->x32.as<float>();
  }
  return product_to_host(
      h, dim,
      [&](int64_t r0, int64_t r1) {
        return hamiltonian_apply_rows(h, x, y, nvec, first, nbr, accumulate, x32, h->stream, r0, r1);
      },
      [&](int64_t r0, int64_t r1, cudaStream_t cs) -> int {
        // vector j of the result occupies [j dim, (j + 1) dim)
        for (int j = 0; j < nvec; ++j)
          DH_CUDA(cudaMemcpyAsync(dst + (size_t)j * dim + r0, y + (size_t)j * dim + r0, (size_t)(r1 - r0) * sizeof(double),
                                  cudaMemcpyDeviceToHost, cs));
        return DH_OK;
      });
}

int dh_hamiltonian_block_multiply(dh_hamiltonian_t h, const double* x, double* y, int k) {
  DH_CHECK(h && x && y, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(k >= 1, DH_ERR_ARGUMENT, "k must be >= 1");
  DH_CHECK(k == 1 || !h->complex_phases, DH_ERR_UNSUPPORTED, "complex vectors are multiplied one at a time");
  const int64_t dim = hamiltonian_dim(h);
  const size_t bytes = (size_t)dim * k * sizeof(double);
  const bool src_dev = is_device_pointer(x), dst_dev = is_device_pointer(y);
  const double* xd = x;
  double* yd = y;
  int rc;
  if (!src_dev) {
    if ((rc = ensure_buffer(h->stage_x, bytes)) != DH_OK) return rc;
    DH_CUDA(cudaMemcpyAsync(h->stage_x.ptr, x, bytes, cudaMemcpyHostToDevice, h->stream));
    xd = h->stage_x.as<double>();
  }
  if (!dst_dev) {
    if ((rc = ensure_buffer(h->stage_y, bytes)) != DH_OK) return rc;
    yd = h->stage_y.as<double>();
  }
  const float* x32 = nullptr;
  if (h->precision == DH_PRECISION_FP32) {
    if ((rc = ensure_buffer(h->x32, (size_t)dim * k * sizeof(float))) != DH_OK) return rc;
    if ((rc = launch_convert_f32(xd, h->x32.as<float>(), dim * k, h->stream)) != DH_OK) return rc;
    x32 = h->x32.as<float>();
  }
  if (dst_dev) {
    if ((rc = hamiltonian_apply_block(h, xd, x32, yd, k, h->precision, h->stream)) != DH_OK) return rc;
    DH_CUDA(cudaStreamSynchronize(h->stream));
    return DH_OK;
  }
  return product_to_host(
      h, dim,
      [&](int64_t r0, int64_t r1) {
        return hamiltonian_apply_block_rows(h, xd, x32, yd, k, h->precision, h->stream, r0, r1);
      },
      [&](int64_t r0, int64_t r1, cudaStream_t cs) -> int {
        // rows are k-interleaved: rows [r0, r1) are one contiguous range
        DH_CUDA(cudaMemcpyAsync(y + (size_t)r0 * k, yd + (size_t)r0 * k, (size_t)(r1 - r0) * k * sizeof(double),
                                cudaMemcpyDeviceToHost, cs));
        return DH_OK;
      });
}

int dh_hamiltonian_autotune(dh_hamiltonian_t h, int block_size, int repeats, double* out) {
  DH_CHECK(h, DH_ERR_ARGUMENT, "null hamiltonian");
  DH_CHECK(block_size == 1 || block_size == 2 || block_size == 4, DH_ERR_ARGUMENT, "block size %d not in {1, 2, 4}",
           block_size);
  if (repeats < 1) repeats = 3;
  DH_CHECK(!h->complex_phases, DH_ERR_UNSUPPORTED, "the complex chain has a single product form");
  dh_space_s* sp = h->space;
  const int64_t dim = sp->dim;
  const int kmax = 4;
  DevBuf x, x32, y;
  int rc;
  if ((rc = x.alloc((size_t)dim * kmax * sizeof(double))) != DH_OK ||
      (rc = x32.alloc((size_t)dim * kmax * sizeof(float))) != DH_OK ||
      (rc = y.alloc((size_t)dim * kmax * sizeof(double))) != DH_OK)
    return rc;
  cudaStream_t st = h->stream;
  if ((rc = launch_random_vector(x.as<double>(), dim * kmax, 12345, st)) != DH_OK) return rc;
  if ((rc = launch_convert_f32(x.as<double>(), x32.as<float>(), dim * kmax, st)) != DH_OK) return rc;
  if (sp->kind == SPACE_FERMION && sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
  cudaEvent_t e0, e1;
  DH_CUDA(cudaEventCreate(&e0));
  DH_CUDA(cudaEventCreate(&e1));
  struct Events {
    cudaEvent_t a, b;
    ~Events() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } guard{e0, e1};
  // median device time of one product of a k-vector block (one untimed call first)
  auto time_one = [&](int k, double* ms_out) -> int {
    int r = hamiltonian_apply_block(h, x.as<double>(), x32.as<float>(), y.as<double>(), k, h->precision, st);
    if (r != DH_OK) return r;
    std::vector<float> ms(repeats);
    for (int i = 0; i < repeats; ++i) {
      DH_CUDA(cudaEventRecord(e0, st));
      if ((r = hamiltonian_apply_block(h, x.as<double>(), x32.as<float>(), y.as<double>(), k, h->precision, st)) != DH_OK)
        return r;
      DH_CUDA(cudaEventRecord(e1, st));
      DH_CUDA(cudaEventSynchronize(e1));
      DH_CUDA(cudaEventElapsedTime(&ms[i], e0, e1));
    }
    std::sort(ms.begin(), ms.end());
    *ms_out = ms[repeats / 2];
    return DH_OK;
  };
  double best = 1e300;
  int best_variant = sp->kernel_variant, best_lb = sp->rank.low_bits, tried = 0;
  h->fast_use = false;  // the on-the-fly forms first
  sp->split_form = 0;
  if (sp->kind == SPACE_FERMION && sp->index_mode == DH_INDEX_RANK) {
    const int L = sp->lz_max;
    const int lb0 = (L + 2) / 2;
    for (int variant : {0, 2, 1}) {
      for (int lb = lb0 - 2; lb <= lb0 + 2; ++lb) {
        if (variant == 1 && lb != lb0) continue;  // the generic kernel does not read the tables' split
        if (lb < 3 || lb > L || L + 1 - lb > 24) continue;
        if (variant == 2 && lb > 15) continue;    // the staged low-rank table must fit in 64 KiB
        sp->kernel_variant = variant;
        if ((rc = build_rank_tables(sp, lb)) != DH_OK) return rc;
        double ms = 0.0;
        if ((rc = time_one(block_size, &ms)) != DH_OK) return rc;
        ++tried;
        if (ms < best) {
          best = ms;
          best_variant = variant;
          best_lb = sp->rank.low_bits;
        }
      }
    }
    sp->kernel_variant = best_variant;
    if ((rc = build_rank_tables(sp, best_lb)) != DH_OK) return rc;
    // launch forms of the split-word kernel (threads per block, register budget, gather pipeline)
    // at the chosen split
    if (best_variant == 0) {
      int best_form = 0;
      for (int form = 1; form < kNbrSplitForms; ++form) {
        sp->split_form = form;
        double ms = 0.0;
        if ((rc = time_one(block_size, &ms)) != DH_OK) return rc;
        ++tried;
        if (ms < best) {
          best = ms;
          best_form = form;
        }
      }
      sp->split_form = best_form;
    }
  } else {
    if ((rc = time_one(block_size, &best)) != DH_OK) return rc;
    tried = 1;
  }
  // stored elements, when built, at both read-ahead depths: kept in use only if they beat the best
  // on-the-fly form
  double stored_ms = 0.0;
  if (h->fast) {
    h->fast_use = true;
    stored_ms = 1e300;
    int best_chunk = 8;
    for (int chunk : {8, 16}) {
      h->ell_chunk = chunk;
      double ms = 0.0;
      if ((rc = time_one(block_size, &ms)) != DH_OK) return rc;
      ++tried;
      if (ms < stored_ms) {
        stored_ms = ms;
        best_chunk = chunk;
      }
    }
    h->ell_chunk = best_chunk;
    if (stored_ms < best) best = stored_ms;
    else h->fast_use = false;
  }
  double per_k[3] = {0.0, 0.0, 0.0};
  const int ks[3] = {1, 2, 4};
  for (int i = 0; i < 3; ++i)
    if ((rc = time_one(ks[i], &per_k[i])) != DH_OK) return rc;
  if (out) {
    out[7] = stored_ms;
    out[8] = (h->fast && h->fast_use) ? 1.0 : 0.0;
    out[0] = best;
    out[1] = sp->kind == SPACE_FERMION ? sp->kernel_variant : 0;
    out[2] = sp->kind == SPACE_FERMION ? sp->rank.low_bits : 0;
    out[3] = per_k[0];
    out[4] = per_k[1];
    out[5] = per_k[2];
    out[6] = tried;
    out[9] = sp->kind == SPACE_FERMION ? sp->split_form : 0;
    out[10] = h->fast ? h->ell_chunk : 0;
  }
  return DH_OK;
}

int dh_hamiltonian_low_level_add_multiply(dh_hamiltonian_t h, const double* src, double* dst, int64_t first,
                                          int64_t nbr) {
  return multiply_common(h, src, dst, 1, first, nbr, 1);
}

int dh_hamiltonian_low_level_multiply(dh_hamiltonian_t h, const double* src, double* dst, int64_t first, int64_t nbr) {
  return multiply_common(h, src, dst, 1, first, nbr, 0);
}

int dh_hamiltonian_low_level_multiple_add_multiply(dh_hamiltonian_t h, const double* srcs, double* dsts,
                                                   int nbr_vectors, int64_t first, int64_t nbr) {
  return multiply_common(h, srcs, dsts, nbr_vectors, first, nbr, 1);
}

int dh_hamiltonian_matrix_element(dh_hamiltonian_t h, const double* v1, const double* v2, double* out) {
  DH_CHECK(h && v1 && v2 && out, DH_ERR_ARGUMENT, "null argument");
  const int64_t dim = hamiltonian_dim(h);
  const size_t bytes = (size_t)dim * sizeof(double);
  int rc;
  if ((rc = ensure_buffer(h->stage_y, bytes)) != DH_OK) return rc;
  if ((rc = ensure_buffer(h->stage_v, 2 * bytes + 64)) != DH_OK) return rc;
  const double* a = v1;
  const double* b = v2;
  double* tmp_a = h->stage_v.as<double>();
  double* tmp_b = tmp_a + dim;
  if (!is_device_pointer(v1)) {
    DH_CUDA(cudaMemcpyAsync(tmp_a, v1, bytes, cudaMemcpyHostToDevice, h->stream));
    a = tmp_a;
  }
  if (!is_device_pointer(v2)) {
    DH_CUDA(cudaMemcpyAsync(tmp_b, v2, bytes, cudaMemcpyHostToDevice, h->stream));
    b = tmp_b;
  }
  double* y = h->stage_y.as<double>();
  if ((rc = hamiltonian_apply(h, b, y, 1, 0, dim, 0, nullptr, h->stream)) != DH_OK) return rc;
  double* res = reinterpret_cast<double*>(h->stage_v.as<char>() + 2 * bytes);
  const double* vs[1] = {a};
  if ((rc = launch_multi_dot(vs, 1, y, dim, res, h->red, h->stream)) != DH_OK) return rc;
  DH_CUDA(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  return DH_OK;
}

int dh_hamiltonian_row_elements(dh_hamiltonian_t h, int64_t row, int* targets, int* signs, int* factor_index, int cap,
                                int* count) {
  DH_CHECK(h && count && (cap == 0 || (targets && signs && factor_index)), DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(h->kind == SPACE_FERMION, DH_ERR_UNSUPPORTED, "row elements are only available for FQHE Hamiltonians");
  DH_CHECK(row >= 0 && row < h->space->dim, DH_ERR_ARGUMENT, "row %lld out of range", (long long)row);
  dh_space_s* sp = h->space;
  int rc;
  if (sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
  DevBuf buf;
  const int c = cap > 0 ? cap : 1;
  if ((rc = buf.alloc((size_t)3 * c * sizeof(int) + 16)) != DH_OK) return rc;
  int* dt = buf.as<int>();
  int* ds = dt + c;
  int* df = ds + c;
  int* dc = df + c;
  if ((rc = launch_fqhe_row_elements(fqhe_device(sp, h, DH_PRECISION_FP64), row, dt, ds, df, cap, dc, h->stream)) != DH_OK)
    return rc;
  DH_CUDA(cudaStreamSynchronize(h->stream));
  DH_CUDA(cudaMemcpy(count, dc, sizeof(int), cudaMemcpyDeviceToHost));
  const int n = std::min(*count, cap);
  if (n > 0) {
    DH_CUDA(cudaMemcpy(targets, dt, n * sizeof(int), cudaMemcpyDeviceToHost));
    DH_CUDA(cudaMemcpy(signs, ds, n * sizeof(int), cudaMemcpyDeviceToHost));
    DH_CUDA(cudaMemcpy(factor_index, df, n * sizeof(int), cudaMemcpyDeviceToHost));
  }
  return DH_OK;
}

int dh_hamiltonian_get_interaction_factors(dh_hamiltonian_t h, double* factors, int cap, int* count) {
  DH_CHECK(h && count, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK(h->kind == SPACE_FERMION || h->kind == SPACE_FERMION_LONG || h->kind == SPACE_BOSON, DH_ERR_UNSUPPORTED,
           "interaction factors only exist for FQHE Hamiltonians");
  *count = h->tabs.nbr_factors;
  const int n = std::min(cap, h->tabs.nbr_factors);
  if (factors && n > 0) memcpy(factors, h->tabs.factors.data(), n * sizeof(double));
  return DH_OK;
}

int dh_hamiltonian_pseudopotential_adjoint(dh_hamiltonian_t h, const double* u, const double* v, double* out) {
  DH_CHECK(h && u && v && out, DH_ERR_ARGUMENT, "null argument");
  DH_CHECK((h->kind == SPACE_FERMION || h->kind == SPACE_FERMION_LONG || h->kind == SPACE_BOSON) && !h->l2_only,
           DH_ERR_UNSUPPORTED,
           "the pseudopotential adjoint needs a FermionOnSphere(Long) or BosonOnSphereShort interaction Hamiltonian");
  dh_space_s* sp = h->space;
  const int64_t dim = sp->dim;
  const size_t bytes = (size_t)dim * sizeof(double);
  int rc;
  if (sp->index_mode == DH_INDEX_LOOKUP && (rc = build_lookup(sp)) != DH_OK) return rc;
  if ((rc = ensure_buffer(h->stage_v, 2 * bytes + 64)) != DH_OK) return rc;
  const double* du = u;
  const double* dv = v;
  if (!is_device_pointer(u)) {
    DH_CUDA(cudaMemcpyAsync(h->stage_v.ptr, u, bytes, cudaMemcpyHostToDevice, h->stream));
    du = h->stage_v.as<double>();
  }
  if (!is_device_pointer(v)) {
    DH_CUDA(cudaMemcpyAsync(h->stage_v.as<double>() + dim, v, bytes, cudaMemcpyHostToDevice, h->stream));
    dv = h->stage_v.as<double>() + dim;
  }
  int dev = 0, sms = 0;
  DH_CUDA(cudaGetDevice(&dev));
  DH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int nblocks = sms * 2;
  const int nf = h->tabs.nbr_factors;
  // per-block partial bins, except for the large tables of the 128-bit engine and the widest bosonic
  // sectors (atomics into the bins)
  const bool partial =
      !((h->kind == SPACE_FERMION_LONG || h->kind == SPACE_BOSON) && (size_t)nf * sizeof(double) > 200 * 1024);
  if (partial && (rc = ensure_buffer(h->bins_partial, (size_t)nblocks * nf * sizeof(double))) != DH_OK) return rc;
  if ((rc = ensure_buffer(h->bins, (size_t)nf * sizeof(double))) != DH_OK) return rc;
  const FqheDevice fd = fqhe_device(sp, h, DH_PRECISION_FP64);
  if ((rc = (h->kind == SPACE_FERMION_LONG)
                ? launch_long_bins(fqhe_long_device(sp, h, DH_PRECISION_FP64), nf, du, dv, h->bins_partial.as<double>(),
                                   nblocks, h->bins.as<double>(), h->stream)
            : (h->kind == SPACE_BOSON)
                ? launch_boson_bins(fd, du, dv, h->bins_partial.as<double>(), nblocks, h->bins.as<double>(), h->stream)
                : launch_fqhe_bins(fd, du, dv, h->bins_partial.as<double>(), nblocks, h->bins.as<double>(), h->stream)) !=
      DH_OK)
    return rc;
  std::vector<double> bins(nf);
  DH_CUDA(cudaMemcpyAsync(bins.data(), h->bins.ptr, nf * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  const int nlz = h->tabs.lz_max + 1;
  for (int m = 0; m < nlz; ++m) {
    double acc = 0.0;
    for (int f = 0; f < nf; ++f) acc += bins[f] * h->tabs.dfactor[(size_t)f * nlz + m];
    out[m] = acc;
  }
  return DH_OK;
}

int dh_hamiltonian_count_elements(dh_hamiltonian_t h, int64_t* total) {
  DH_CHECK(h && total, DH_ERR_ARGUMENT, "null argument");
  dh_space_s* sp = h->space;
  if (h->kind == SPACE_FERMION_LONG) {
    DevBuf t;
    int rc;
    if ((rc = t.alloc(sizeof(unsigned long long))) != DH_OK) return rc;
    if ((rc = launch_long_count(fqhe_long_device(sp, h, DH_PRECISION_FP64), t.as<unsigned long long>(), h->stream)) !=
        DH_OK)
      return rc;
    unsigned long long v = 0;
    DH_CUDA(cudaMemcpyAsync(&v, t.ptr, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    DH_CUDA(cudaStreamSynchronize(h->stream));
    *total = (int64_t)v;
    return DH_OK;
  }
  if (h->kind == SPACE_SPIN12_TRANSLATIONS) {
    // the flips whose word lies in the momentum sector (the others are dropped, as the reference's
    // SymmetrizeResult returns no index for them)
    DevBuf t;
    int rc;
    if ((rc = t.alloc(2 * sizeof(unsigned long long))) != DH_OK) return rc;
    if ((rc = launch_trans_count_elements(trans_device(sp, h), t.as<unsigned long long>(), h->stream)) != DH_OK)
      return rc;
    unsigned long long v[2] = {0, 0};
    DH_CUDA(cudaMemcpyAsync(v, t.ptr, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    DH_CUDA(cudaStreamSynchronize(h->stream));
    *total = (int64_t)v[1];
    return DH_OK;
  }
  if (h->kind == SPACE_SPIN12) {
    // every antiparallel bond is one flip: sum over the basis of #antiparallel bonds equals
    // (#bonds) * (fraction of states in which a given bond is antiparallel) * dim
    const long long L = sp->length, n = sp->nbr_up;
    const double frac = (L >= 2) ? 2.0 * (double)n * (double)(L - n) / ((double)L * (double)(L - 1)) : 0.0;
    *total = (int64_t)llround(2.0 * (double)L * frac * (double)sp->dim);
    return DH_OK;
  }
  DevBuf t;
  int rc;
  if ((rc = t.alloc(2 * sizeof(unsigned long long))) != DH_OK) return rc;
  if (h->kind == SPACE_BOSON)
    rc = launch_boson_count(fqhe_device(sp, h, DH_PRECISION_FP64), t.as<unsigned long long>(), h->stream);
  else
    rc = launch_fqhe_count(fqhe_device(sp, h, DH_PRECISION_FP64), t.as<unsigned long long>(), h->stream);
  if (rc != DH_OK) return rc;
  unsigned long long v = 0;
  DH_CUDA(cudaMemcpyAsync(&v, t.ptr, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  *total = (int64_t)v;
  return DH_OK;
}

int dh_hamiltonian_count_diagonal_elements(dh_hamiltonian_t h, int64_t* total) {
  DH_CHECK(h && total, DH_ERR_ARGUMENT, "null argument");
  dh_space_s* sp = h->space;
  if (h->kind == SPACE_SPIN12 || h->kind == SPACE_SPIN12_TRANSLATIONS) {
    *total = 0;  // the chain's elements are its flips; the Sz Sz part is computed per row
    return DH_OK;
  }
  if (h->kind == SPACE_FERMION || h->kind == SPACE_FERMION_LONG) {
    // every occupied pair m1 > m2 has one move back to its row (m3 = m1, m4 = m2)
    const long long n = sp->nbr_fermions;
    *total = (int64_t)(n * (n - 1) / 2) * sp->dim;
    return DH_OK;
  }
  DevBuf t;
  int rc;
  if ((rc = t.alloc(2 * sizeof(unsigned long long))) != DH_OK) return rc;
  if ((rc = launch_boson_count(fqhe_device(sp, h, DH_PRECISION_FP64), t.as<unsigned long long>(), h->stream)) != DH_OK)
    return rc;
  unsigned long long v[2] = {0, 0};
  DH_CUDA(cudaMemcpyAsync(v, t.ptr, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  DH_CUDA(cudaStreamSynchronize(h->stream));
  *total = (int64_t)v[1];
  return DH_OK;
}

int dh_coulomb_pseudopotentials(int nbr_flux, double* v) {
  DH_CHECK(v && nbr_flux >= 1 && nbr_flux <= 126, DH_ERR_ARGUMENT, "nbr_flux must be in 1..126");
  coulomb_pseudopotentials(nbr_flux, v);
  return DH_OK;
}

int dh_clebsch_gordan(int j1, int m1, int j2, int m2, int j, double* out) {
  DH_CHECK(out, DH_ERR_ARGUMENT, "null output");
  DH_CHECK(j1 >= 0 && j2 >= 0 && j >= 0 && j1 + j2 + j <= 1196, DH_ERR_ARGUMENT, "angular momenta out of range");
  *out = clebsch_gordan(j1, m1, j2, m2, j);
  return DH_OK;
}

}  // extern "C"

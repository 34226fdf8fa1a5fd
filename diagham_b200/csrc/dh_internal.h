// Internal declarations of the diagham_b200 library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/diagham_b200.h"

namespace dh {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define DH_CUDA(expr)                                                   \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) return ::dh::cuda_fail(_e, #expr, __FILE__, __LINE__); \
  } while (0)

#define DH_CHECK(cond, code, ...)      \
  do {                                 \
    if (!(cond)) {                     \
      ::dh::set_error(__VA_ARGS__);    \
      return (code);                   \
    }                                  \
  } while (0)

// ------------------------------------------------------- device buffers
// A device allocation owned by a handle.  Freed in the destructor.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int alloc(size_t n);
  void release();
  template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// ------------------------------------------------------ host-side maths
// Clebsch-Gordan <j1/2 m1/2; j2/2 m2/2 | j/2 (m1+m2)/2>, every argument doubled.
double clebsch_gordan(int j1, int m1, int j2, int m2, int j);
// LLL Coulomb pseudopotentials V_0..V_nbrFlux on the sphere (FP64).
void coulomb_pseudopotentials(int nbr_flux, double* v);

// Interaction tables of the two-body Hamiltonian on lz_max+1 orbitals.
struct InteractionTables {
  int lz_max = 0;
  int nbr_pairs = 0;                // (m1 > m2) pairs, m1 ascending then m2 ascending
  int nbr_factors = 0;              // (pair, m3) entries with 2 m3 > m1 + m2
  std::vector<int> pair_offset;     // first factor of each pair
  std::vector<double> dfactor;      // [factor][m]: d factor / d V_m (factors are linear in V)
  std::vector<double> factors;      // current factors for the current V (+ l2_factor * l2_part)
  std::vector<double> l2_part;      // [factor]: the two-body table of L^2 (empty: no L^2 term)
  double l2_factor = 0.0;
  bool bosonic = false;             // pair layout of build_bosons (m1 >= m2)
  void build(int lz_max);
  // ParticleOnSphereGenericHamiltonian's bosonic factors (ParticleOnSphereGenericHamiltonian.cc:
  // 620-806): pairs m1 >= m2 (pair m1 (m1 + 1) / 2 + m2), creations m3 >= m4, even relative momentum
  void build_bosons(int lz_max);
  // L^2 of nbr_particles fermions as a two-body table (L^2 = L-L+ + Lz^2 + Lz; the constant part
  // is returned by l2_constant)
  void build_l2(int nbr_particles);
  void set_pseudopotentials(const double* v);
};
// Lz^2 + Lz of the sector 2 Lz = total_lz: the constant part of L^2
double l2_constant(int total_lz);

// Symmetric tridiagonal eigenvalues (ascending) by implicit QL; optional eigenvectors
// (column-major n x n) when z != nullptr.
int tridiagonal_eigen(int n, const double* diag, const double* off, double* eig, double* z);
// the m lowest eigenvalues (ascending) of the same tridiagonal matrix by bisection on Sturm counts
// (O(n) per count, about 60 counts per eigenvalue)
int tridiagonal_lowest(int n, const double* diag, const double* off, int m, double* eig);
// the lowest eigenvalue of the same matrix when an upper bound is known (the previous lowest Ritz
// value of a growing Lanczos matrix): safeguarded Newton on the pivots, a few O(n) passes
int tridiagonal_lowest_below(int n, const double* diag, const double* off, double above, double* eig0);
// Dense symmetric eigen-decomposition (row-major a, destroyed), eigenvalues ascending, optional
// eigenvectors (columns of z, row-major n x n).
int symmetric_eigen(int n, double* a, double* eig, double* z);

// ------------------------------------------------------------- spaces
enum SpaceKind {
  SPACE_FERMION = 1,
  SPACE_SPIN12 = 2,
  SPACE_BOSON = 3,
  SPACE_SPIN12_TRANSLATIONS = 4,
  // FermionOnSphere with 41 <= lz_max <= 62 and FermionOnSphereLong: 128-bit words, per-fermion ranks
  SPACE_FERMION_LONG = 5
};

struct FermionRankTables {
  int low_bits = 0;                 // LB: rank = high_offset[w >> LB] + low_rank[w & (2^LB - 1)]
  int high_bits = 0;
  std::vector<uint16_t> low_rank;   // rank among LB-bit words with equal popcount and weighted sum
  std::vector<int32_t> high_offset; // first index of the block of states sharing the high part, -1 if none
};

// ------------------------------------------------------ kernel launchers
// Launch forms of the split-word FQHE product kernel (threads per block, register budget, gather
// pipeline depth), chosen per space by dh_hamiltonian_autotune.
constexpr int kNbrSplitForms = 8;

struct FqheDevice {
  const uint64_t* words;
  const uint16_t* low_rank;
  const int32_t* high_offset;
  const int32_t* lookup;       // [lz_max+1][2^lookup_shift + 1] (lookup-table search mode)
  const int32_t* lookup_shift; // per highest orbital
  const int32_t* pair_offset;  // [nbr_pairs]
  const void* factors;         // FP64 or FP32 [nbr_factors]
  long long dim;
  int lz_max;
  int low_bits;
  int lookup_bits;
  int nbr_pairs;
  int nbr_factors;
  int index_mode;              // DH_INDEX_RANK or DH_INDEX_LOOKUP
  int kernel_variant;          // 0: split-word rank kernel, 1: generic kernel (rank mode)
  int split_form;              // launch form of the split-word kernel (0 .. kNbrSplitForms - 1)
  int boson_lz_max;            // BosonOnSphereShort: orbitals 0..boson_lz_max (words of lz_max + 1 bits)
  int nbr_bosons;
  // words beyond the split-word tables (BosonOnSphereShort with lz_max + N - 1 > 40): ranks from the
  // fermionic sector's count table C(n, o, s) at (n - 1) * count_stride_n + o * count_stride_o + s
  const int32_t* count_table;
  long long count_stride_n;
  int count_stride_o;
  int nbr_particles;           // N (fermions of the word)
};

// Fermions with 128-bit words (FermionOnSphereLong, and FermionOnSphere beyond the split-word tables)
struct FqheLongDevice {
  const uint64_t* words;        // [dim][2]: low and high 64 bits of each state, descending
  const int32_t* table;         // C(n, o, s) at (n - 1) * stride_n + o * stride_o + s (saturated at 2^31 - 1)
  const int32_t* pair_offset;   // [nbr_pairs]
  const void* factors;          // FP64 or FP32 [nbr_factors]
  long long dim;
  long long stride_n;           // (lz_max + 2) * (total_sum + 1)
  int stride_o;                 // total_sum + 1
  int nbr_fermions, lz_max, total_sum;
};

#ifdef __CUDACC__
// One 32-byte row (four doubles) in a single 256-bit load (sm_100 vector width), through the
// read-only path without allocating in L1.  p must be 32-byte aligned.
__device__ __forceinline__ void ldg_row32_no_l1(const double* p, double (&v)[4]) {
  asm("ld.global.nc.L1::no_allocate.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(p));
}
#endif

struct MatvecArgs {
  const void* x;       // gather source: element (i, j) at x[i * ld + j * vstride]
  void* y;             // output: element (i, j) at y[i * ld_y + j * vstride_y]
  const double* xdiag; // optional FP64 source for the diagonal (shift) term (same layout as x); null = x
  long long ld, vstride, ld_y, vstride_y;
  int nbr_vectors;
  double shift;
  long long col_first, col_last; // only columns (targets) in [col_first, col_last) contribute
  long long row_first, row_last; // rows that receive the diagonal (shift) contribution
  int accumulate;                // y += H x (1) or y = H x (0)
  long long out_first, out_last; // rows computed: [out_first, out_last); out_last = 0: every row
};

// The row-interleaved kernels read a row's K values (and may write its K outputs) with one vector
// access: the x, y and xdiag pointers must be aligned to that access (at most 16 bytes), else the
// strided kernels are used.  elem = sizeof(TG) of the gathered x.
inline bool il_rows_aligned(const MatvecArgs& a, int k, int elem) {
  const uintptr_t ax = (uintptr_t)(k * elem < 16 ? k * elem : 16);
  const uintptr_t ay = (uintptr_t)(k * 8 < 16 ? k * 8 : 16);
  return ((uintptr_t)a.x % ax) == 0 && ((uintptr_t)a.y % ay) == 0 && ((uintptr_t)a.xdiag % ay) == 0;
}

// Every Lz sector of one system in one launch (rows concatenated, vectors K-interleaved).
struct SectorBatchDevice {
  const uint64_t* const* words;       // [nbr_sectors] device pointers (array in device memory)
  const int32_t* const* high_offset;  // [nbr_sectors] device pointers (array in device memory)
  const long long* row_offset;        // [nbr_sectors + 1] in device memory
  const uint16_t* low_rank;           // shared: depends on the split only
  const int32_t* pair_offset;
  const void* factors;                // FP64 or FP32
  const void* x;                      // [total_rows][block]
  const double* xdiag;                // optional FP64 copy of x for the shift term
  double* y;                          // [total_rows][block]
  const int* active;                  // optional [nbr_sectors]: 0 = the sector's rows get y = 0
  long long total_rows;
  double shift;
  int nbr_sectors, block, lz_max, low_bits, nbr_pairs, nbr_factors;
};
int launch_fqhe_sectors(const SectorBatchDevice& b, int precision, cudaStream_t s);

// Tiles of the concatenated rows of several sectors (a tile never straddles two sectors).
struct TileSetDevice {
  const int* tile_sector;        // [nbr_tiles]
  const long long* tile_begin;   // [nbr_tiles] first concatenated row
  const long long* tile_end;     // [nbr_tiles] one past the last
  const int* sector_tile_first;  // [nbr_sectors + 1]
  int nbr_tiles;
  int nbr_sectors;
};
int launch_seg_gram(const double* a, const double* b, int k, const TileSetDevice& t, double* partial, double* g,
                    cudaStream_t s);
int launch_seg_update(double* w, const double* v, const double* A, const double* vp, const double* Bt, int k,
                      const TileSetDevice& t, cudaStream_t s);
int launch_seg_rmul(double* w, const double* M, int k, const TileSetDevice& t, float* w32, cudaStream_t s);
int launch_seg_combine_blocks(const double* blocks, int nb, long long stride, const double* C, int cstride, int k,
                              const TileSetDevice& t, double* out, cudaStream_t s);
// vectors first_col .. k-1 of every sector's [rows][k] block: component i of vector j is the
// (i+1)-th splitmix64 output of seed + j, mapped to [-1, 1)
int launch_random_block(double* x, long long rows, int k, const long long* row_sector_base, const TileSetDevice& t,
                        uint64_t seed, cudaStream_t s, int first_col = 0);
int launch_f32_copy(const double* x, float* y, long long n, cudaStream_t s);
// per-sector k x k math of a block step on the device (one thread per sector): A = sym(G) with
// scale = |A|^2 + |Bt|^2; a CholQR pass (R, R^-1, breakdown / vanishing flags); B = R2 R1, Bt = B^T
int launch_step_sym(const double* G, const double* Bt, int k, int nsec, double* A, double* scale, cudaStream_t s);
int launch_step_chol(const double* G, int k, int nsec, int pass, double vanish_tol, double pivot_tol, const double* scale,
                     double* R, double* Rinv, int* flags, cudaStream_t s);
int launch_step_b(const double* R1, const double* R2, const int* flags, int k, int nsec, double* B, double* Bt_next,
                  cudaStream_t s);
// x[i][col] = v[i] and v[i] = scale * x[i][col] for a [n][k] block x
int launch_put_column(const double* v, long long n, int k, int col, double* x, cudaStream_t s);
int launch_get_column(const double* x, long long n, int k, int col, double scale, double* v, cudaStream_t s);
// eigenvalues (ascending) of a symmetric band matrix of half-bandwidth b stored densely (row-major,
// destroyed): Givens reduction to tridiagonal form touching only the band, then implicit QL
int band_eigenvalues(int n, int b, double* a, double* eig);
// eigenvector of the symmetric band matrix a (dense storage, unchanged) for its eigenvalue lambda, by
// inverse iteration with a banded LU (O(n b^2))
int band_inverse_iteration(int n, int b, const double* a, double lambda, double* vec);
// The lowest Ritz value of a Lanczos tridiagonal matrix of n rows: from the previous lowest value (of
// a leading block, an upper bound by interlacing) by safeguarded Newton steps, O(n); by implicit QL
// when there is none, or when Newton returns the bound unchanged.
int lanczos_lowest_ritz(int n, const double* diag, const double* off, const double* previous, double* lowest);
// The next graph batch of the single-vector Lanczos solve, from the convergence test's ratio to its
// threshold sampled as logarithms at rows rows[0..n) (the last at the newest replayed row): the
// ratio decays about geometrically, the rate is taken over the last kLanczosRateSpan rows (or the
// longest span sampled), and the batch aims at 0.85 of the rows predicted until the ratio reaches
// 1, between 2 and graph_batch; graph_batch when nothing can be predicted.
constexpr int kLanczosRateSpan = 6;
int lanczos_batch_prediction(int n, const int* rows, const double* log_ratio, int graph_batch);

int launch_fqhe_unrank(int nbr_fermions, int lz_max, int total_sum, long long dim, uint64_t* words,
                       const int64_t* counts_dev, int count_stride_o, int count_stride_s, cudaStream_t s);
int launch_fqhe_matvec(const FqheDevice& f, const MatvecArgs& a, int precision, cudaStream_t s);
// BosonOnSphereShort product (kernels_boson.cu), any vector layout, K = 1, 2, 4 (else in passes)
int launch_boson_matvec(const FqheDevice& f, const MatvecArgs& a, int precision, cudaStream_t s);
int launch_long_unrank(const FqheLongDevice& f, uint64_t* words, cudaStream_t s);
int launch_long_find(const FqheLongDevice& f, const uint64_t* words, long long n, long long* out, cudaStream_t s);
int launch_long_count(const FqheLongDevice& f, unsigned long long* total, cudaStream_t s);
int launch_long_matvec(const FqheLongDevice& f, const MatvecArgs& a, int precision, cudaStream_t s);
// total[0] = generated elements, total[1] = those that return to their row (one per annihilated pair)
int launch_boson_count(const FqheDevice& f, unsigned long long* total, cudaStream_t s);
int launch_fqhe_row_elements(const FqheDevice& f, long long row, int* targets, int* signs, int* factor_index,
                             int cap, int* count, cudaStream_t s);
int launch_fqhe_bins(const FqheDevice& f, const double* u, const double* v, double* partial_bins, int nblocks,
                     double* bins, cudaStream_t s);
int launch_fqhe_count(const FqheDevice& f, unsigned long long* total, cudaStream_t s);
int launch_fqhe_find(const FqheDevice& f, const uint64_t* words, long long n, long long* out, cudaStream_t s);

// Stored elements of an FQHE Hamiltonian (sliced ELL, 32-row slices; see kernels_fast.cu)
// Stored elements: per-row lengths of a slice are padded to a multiple of kEllPad; within a slice a
// row's elements come in groups of kEllGroup (one 16-byte load of targets per lane); the product
// reads chunks of 8 or 16 elements ahead of its gathers (EllDevice::chunk, chosen by the autotuner).
constexpr int kEllPad = 16;
constexpr int kEllGroup = 4;
struct EllDevice {
  const long long* slice_ptr;  // [nslices] first element of each slice (a multiple of 32 * kEllPad)
  const int* slice_len;        // [nslices] elements per row of the slice (padded to a multiple of kEllPad)
  const int* cols;             // target index of each element
  const uint16_t* coef;        // factor index | sign << 15; padding holds nbr_factors (a zero factor)
  // payload 1, bosons (BosonOnSphereShort): factor index | caa << 16 | cad << 24, the element being
  // factor * sqrt(caa) * sqrt(cad); payload 2, fermions of the count-table engine (FermionOnSphereLong,
  // FermionOnSphere beyond 40 orbitals): factor index | sign << 31, factors read through the cache
  const uint32_t* coef32;
  int payload;                 // 0: coef (uint16), 1 or 2: coef32 as above
  // optional, the batched sectors: rows of sector i are sector_offset[i] .. sector_offset[i + 1] - 1,
  // and the rows of a sector whose active[i] is 0 get y = 0 without their elements
  const int* active;
  const long long* sector_offset;
  int nbr_sectors;
  const void* diag;            // [dim] diagonal, FP64 or FP32 like the factors
  const void* factors;         // [nbr_factors] FP64 or FP32
  long long dim;
  int nbr_factors;
  int chunk;                   // elements read ahead of the gathers: 8 or 16
};
// row_offset: the space's rows sit at row_offset .. row_offset + dim - 1 of a concatenated structure
// (targets shifted alike)
int launch_fqhe_row_counts(const FqheDevice& f, int* counts, cudaStream_t s, long long row_offset = 0);
int launch_fqhe_ell_fill(const FqheDevice& f, const long long* slice_ptr, const int* slice_len, int* cols,
                         uint16_t* coef, cudaStream_t s, long long row_offset = 0);
int launch_fqhe_diag(const FqheDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s,
                     long long row_offset = 0);
int launch_ell_product(const EllDevice& e, const MatvecArgs& a, int precision, cudaStream_t s);
int launch_long_row_counts(const FqheLongDevice& f, int* counts, cudaStream_t s);
int launch_long_ell_fill(const FqheLongDevice& f, int nbr_factors, const long long* slice_ptr, const int* slice_len,
                         int* cols, uint32_t* coef, cudaStream_t s);
int launch_long_diag(const FqheLongDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s);
int launch_long_bins(const FqheLongDevice& f, int nbr_factors, const double* u, const double* v, double* partial_bins,
                     int nblocks, double* bins, cudaStream_t s);
int launch_boson_row_counts(const FqheDevice& f, int* counts, cudaStream_t s);
int launch_boson_ell_fill(const FqheDevice& f, const long long* slice_ptr, const int* slice_len, int* cols,
                          uint32_t* coef, cudaStream_t s);
int launch_boson_diag(const FqheDevice& f, const double* factors64, double* diag64, float* diag32, cudaStream_t s);
int launch_boson_bins(const FqheDevice& f, const double* u, const double* v, double* partial_bins, int nblocks,
                      double* bins, cudaStream_t s);

struct SpinDevice {
  const uint32_t* words;
  long long dim;
  int length;
  int nbr_up;
  double j1, j2;
};
// Spin1_2ChainWithTranslations with the real J1-J2 Hamiltonian (kernels_spin_translations.cu)
struct TransDevice {
  const uint32_t* reps;      // representatives, ascending
  int32_t* rep_rank;         // their plain Spin1_2Chain index
  const uint8_t* orbits;     // their orbit sizes
  unsigned long long* map;   // per plain chain index: representative | rotations << 32 | orbit << 40
  const int* table;          // lookup over the representatives (first index per word >> table_shift)
  long long table_entries;
  int table_shift;
  long long dim;             // representatives
  long long chain_dim;       // C(L, n_up)
  int length, momentum;
  double j1, j2;
  double phase[32];          // cos(2 pi K m / L)
  double sine[32];           // sin(2 pi K m / L)
  int complex_phases;        // SpinChainJ1J2HamiltonianWithTranslations: (Re, Im) interleaved vectors
};
int launch_trans_count(long long total, int L, int n_up, int momentum, unsigned int* chunk_count, cudaStream_t s);
int launch_trans_write(long long total, int L, int n_up, int momentum, const long long* chunk_offset, uint32_t* reps,
                       uint8_t* orbits, cudaStream_t s);
int launch_trans_table(const uint32_t* reps, long long dim, int shift, long long entries, int* table, cudaStream_t s);
int launch_trans_map(const TransDevice& d, long long total, int n_up, cudaStream_t s);
int launch_trans_matvec(const TransDevice& d, const MatvecArgs& a, int precision, cudaStream_t s);
int launch_trans_find(const TransDevice& d, const uint64_t* words, long long n, long long* out, cudaStream_t s);
// elements of one product: antiparallel bonds of every representative (total[0]) and those whose
// flipped word lies in the momentum sector (total[1])
int launch_trans_count_elements(const TransDevice& d, unsigned long long* total, cudaStream_t s);
int launch_spin_unrank(int length, int nbr_up, long long dim, uint32_t* words, cudaStream_t s);
int launch_spin_matvec(const SpinDevice& sp, const MatvecArgs& a, int precision, cudaStream_t s);
int launch_spin_find(const SpinDevice& sp, const uint64_t* words, long long n, long long* out, cudaStream_t s);

// BLAS-1 style kernels on FP64 vectors (device-resident scalars)
struct Reducer {
  double* partial = nullptr;   // [nblocks * width]
  unsigned int* ticket = nullptr;
  int nblocks = 0;
  int width = 0;
};
int reducer_init(Reducer& r, DevBuf& storage, int width);
int launch_multi_dot(const double* const* vs, int m, const double* y, long long n, double* out, Reducer& r,
                     cudaStream_t s);
int launch_lanczos_update(double* w, const double* y, const double* a, const double* b, const double* ca,
                          const double* cb, long long n, double* norm_out, Reducer& r, cudaStream_t s);
int launch_scale_convert(double* v, float* v32, const double* norm, long long n, cudaStream_t s);
int launch_axpy_scalar(double* y, const double* x, double a, long long n, cudaStream_t s);
int launch_random_vector(double* x, long long n, uint64_t seed, cudaStream_t s);
int launch_convert_f32(const double* v, float* v32, long long n, cudaStream_t s);
int launch_gemm_tall(const double* v, long long n, int k, const double* c, int m, double* out, int accumulate,
                     cudaStream_t s);
int launch_gram(const double* a, int ka, const double* b, int kb, long long n, double* out, Reducer& r,
                cudaStream_t s);

// Device view of a Lanczos run (three rotating FP64 vectors, device scalars, optional store).
struct LanczosDev {
  double* vec;        // 3 * dim, slot q at vec + q * dim
  long long dim;
  float* x32;         // FP32 copy of the newest vector (null in FP64 mode)
  double* krylov;     // Krylov store (null if not kept); vector j at krylov + j * dim
  int krylov_cap;
  double* alpha;
  double* beta;
  double* norm;
  int* cursor;
  double* partial;
  unsigned int* ticket;
  int nblocks;
};
int launch_sqrt_inplace(double* x, cudaStream_t s);
int launch_lz_update(const LanczosDev& st, int phase, cudaStream_t s);
int launch_lz_scale(const LanczosDev& st, int phase, cudaStream_t s);
int launch_lz_dots(const LanczosDev& st, int phase, cudaStream_t s);
int launch_combine(const double* vs, int m, long long ld, const double* coef, double sign, double* out, int accumulate,
                   long long n, cudaStream_t s);
int launch_strided_dots(const double* vs, int m, long long ld, const double* y, long long n, double* out, Reducer& r,
                        cudaStream_t s);

}  // namespace dh

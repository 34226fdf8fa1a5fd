/* diagham_b200.h -- C ABI of the B200 engine for DiagHam's on-the-fly H.v + Lanczos path.
 *
 * Plain C: opaque handles, pointers and sizes, int status codes (0 = success, < 0 = error,
 * message from dh_last_error()).  No function aborts the process or throws.
 *
 * Vectors are FP64 arrays of the Hilbert-space dimension, exactly like DiagHam's RealVector
 * components (src/Vector/RealVector.h:108).  Every vector argument may be a host pointer (the
 * call copies it to and from the GPU) or a device pointer on the library's device (used in
 * place); the kind is detected per pointer.  Calls are ordered on the handle's CUDA stream
 * (default: the legacy default stream, see dh_hamiltonian_set_stream) and return once their
 * results are complete.
 *
 * Handles are not thread-safe: use one handle per host thread, as DiagHam clones Hilbert spaces
 * per thread (FQHE/src/Hamiltonian/AbstractQHEOnSphereHamiltonian.cc:425).
 */
#ifndef DIAGHAM_B200_H
#define DIAGHAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define DH_OK 0
#define DH_ERR_ARGUMENT -1
#define DH_ERR_CUDA -2
#define DH_ERR_MEMORY -3
#define DH_ERR_UNSUPPORTED -4
#define DH_ERR_NOT_CONVERGED -5
#define DH_ERR_STATE -6
#define DH_ERR_IO -7 /* a file could not be read or written, or does not hold what its format says */

/* index search modes of the target-index lookup inside the matvec kernels */
#define DH_INDEX_RANK 0   /* two-table combinatorial rank (default) */
#define DH_INDEX_LOOKUP 1 /* DiagHam's highest-bit lookup table + binary search */

/* arithmetic of the matrix-element generation and gather */
#define DH_PRECISION_FP64 0
#define DH_PRECISION_FP32 1 /* FP32 elements and FP32 per-row accumulation, FP64 output */

/* Lanczos algorithms (src/LanczosAlgorithm/) */
#define DH_LANCZOS_BASIC 0              /* BasicLanczosAlgorithm.cc */
#define DH_LANCZOS_FULL_REORTHOGONALIZED 1 /* FullReorthogonalizedLanczosAlgorithm.cc */
#define DH_LANCZOS_BLOCK 2              /* BasicBlockLanczosAlgorithm.cc */
#define DH_LANCZOS_WITH_GROUND_STATE 3  /* BasicLanczosAlgorithmWithGroundState.cc */

typedef struct dh_space_s* dh_space_t;
typedef struct dh_hamiltonian_s* dh_hamiltonian_t;
typedef struct dh_lanczos_s* dh_lanczos_t;

/* Last error message of the calling thread ("" if none). */
const char* dh_last_error(void);
/* Library version string. */
const char* dh_version(void);
/* Number of CUDA devices visible (0 if none, never an error). */
int dh_device_count(int* count);

/* ================================================================ Hilbert spaces */

/* FermionOnSphere(nbrFermions, totalLz, lzMax, memory):
 * FQHE/src/HilbertSpace/FermionOnSphere.cc:75-130.  total_lz is twice the total Lz, lz_max is 2S.
 * memory sizes DiagHam's lookup table (FermionOnSphere.cc:1659); it only matters for the
 * DH_INDEX_LOOKUP search mode, which stages a table of at most DH_LOOKUP_SMEM_BYTES in shared
 * memory.  lz_max <= 40 uses the split-word rank tables (every index mode, stored elements, the
 * adjoint, batched sectors, orbital cuts); 41 <= lz_max <= 62 (the reference's FermionOnSphere range,
 * ParticleOnSphereManager.cc:282) uses the engine of dh_fermion_on_sphere_long_create, with 64-bit
 * words at this interface and the products, counts, L^2 and Lanczos only.  Rejects lz_max > 62 and
 * sectors of odd (total_lz + nbr_fermions * lz_max). */
int dh_fermion_on_sphere_create(int nbr_fermions, int total_lz, int lz_max, unsigned long memory, dh_space_t* out);

/* FermionOnSphereLong(nbrFermions, totalLz, lzMax, memory):
 * FQHE/src/HilbertSpace/FermionOnSphereLong.cc:67-107, the space the reference selects for
 * 63 <= lz_max <= 126 (ParticleOnSphereManager.cc:307-313): one 128-bit word per state, states in
 * descending order (GenerateStates, .cc:911-943).  Words cross this interface as (low, high) pairs
 * of uint64 (dh_space_get_states_long, dh_space_find_state_index_long).  The index of a word is
 * computed from the sector's count table, one lookup per fermion; no search.  Generic Hamiltonian,
 * L^2, products, counts and Lanczos; memory is accepted for the signature and unused.  Rejects
 * lz_max > 126 and sectors whose count table ((N + 1)(lz_max + 2)(sum + 1) entries) exceeds 64M. */
int dh_fermion_on_sphere_long_create(int nbr_fermions, int total_lz, int lz_max, unsigned long memory,
                                     dh_space_t* out);

/* BosonOnSphereShort(nbrBosons, totalLz, lzMax): FQHE/src/HilbertSpace/BosonOnSphereShort.cc:81-110.
 * The states are stored, ordered and found as the FermionOnSphere(N, totalLz, lzMax + N - 1) words
 * of their occupations (n_0 ones, a zero, n_1 ones, ...; BosonOnSphereShort.h:1231), so
 * dh_space_get_states and dh_space_find_state_index take those words.  Rank index mode only:
 * split-word rank tables up to lz_max + N - 1 = 40, beyond that (to 62, the class's own range: the
 * reference switches to BosonOnSphere from lz_max + N - 1 = 63, ParticleOnSphereManager.cc:487) ranks
 * from the fermionic sector's count table.  Rejects lz_max + N - 1 > 62.  memory is accepted for the
 * signature and unused. */
int dh_boson_on_sphere_create(int nbr_bosons, int total_lz, int lz_max, unsigned long memory, dh_space_t* out);

/* Spin1_2Chain(chainLength, sz, memorySize): Spin/src/HilbertSpace/Spin1_2Chain.cc:113-142.
 * sz is twice the total Sz.  chain_length <= 32. */
int dh_spin12_chain_create(int chain_length, int sz, int memory, dh_space_t* out);

/* Spin1_2ChainWithTranslations(chainLength, momentum, translationStep = 1, sz, memory, memorySlice)
 * (Spin/src/HilbertSpace/Spin1_2ChainWithTranslations.cc:167-235): the momentum-K sector of the
 * periodic chain at fixed 2Sz = sz.  A state is an orbit of the L translations, represented by its
 * smallest word; orbits of size o with K o != 0 mod L are not in the sector; states in ascending order
 * of their representative (dh_space_get_states gives the representatives, dh_space_find_state_index
 * takes them).  Set-up builds, for every word of the Sz sector, its representative's index, the
 * translations to it and its orbit size: C(L, N_up) x 8 bytes of device memory (4.8 GB at L = 32).
 * 3 <= L <= 32; memory is accepted for the signature and unused. */
int dh_spin12_chain_translations_create(int chain_length, int momentum, int sz, int memory, dh_space_t* out);

int dh_space_destroy(dh_space_t space);

/* AbstractHilbertSpace::GetHilbertSpaceDimension (src/HilbertSpace/AbstractHilbertSpace.h:81). */
int dh_space_get_dimension(dh_space_t space, int64_t* dim);

/* StateDescription[first .. first+n) and, for fermions, StateLzMax (FermionOnSphere.h:166-168,
 * Spin1_2Chain.h:64) copied to host arrays, in the reference's own order and bit layout.
 * lz_max may be NULL. */
int dh_space_get_states(dh_space_t space, uint64_t* words, int* lz_max, int64_t first, int64_t n);

/* FindStateIndex for n words (FermionOnSphere.cc:1431, Spin1_2Chain.cc:1002), computed on the GPU
 * with the space's current index mode; host or device arrays. */
int dh_space_find_state_index(dh_space_t space, const uint64_t* words, int64_t n, int64_t* indices);

/* StateDescription of FermionOnSphereLong (FermionOnSphereLong.h:111, ULONGLONG words) as (low, high)
 * uint64 pairs, words[2 i] and words[2 i + 1] for state first + i, with the highest occupied orbital
 * (StateLzMax, .h:113) when lz_max is not NULL; a FermionOnSphere space gives (word, 0). */
int dh_space_get_states_long(dh_space_t space, uint64_t* words, int* lz_max, int64_t first, int64_t n);

/* FermionOnSphereLong::FindStateIndex (FermionOnSphereLong.cc:790, lookup table + bisection in the
 * reference) for n (low, high) word pairs; -1 for a word outside the sector.  Host or device arrays. */
int dh_space_find_state_index_long(dh_space_t space, const uint64_t* words, int64_t n, int64_t* indices);

/* Selects DH_INDEX_RANK or DH_INDEX_LOOKUP for every kernel that uses this space.  No reference
 * counterpart: the lookup mode is FindStateIndex's own search (FermionOnSphere.cc:1431). */
int dh_space_set_index_mode(dh_space_t space, int mode);

/* Launch form (0 .. DH_SPLIT_FORMS - 1) of the split-word product kernel for this space, the choice
 * dh_hamiltonian_autotune makes by timing (see there); every form gives bit-identical products.
 * No reference counterpart. */
#define DH_SPLIT_FORMS 8
int dh_space_set_split_form(dh_space_t space, int form);

/* FermionOnSphere::EvaluatePartialEntanglementMatrix(subsytemSize, nbrFermionSector, lzSector, state)
 * (FermionOnSphere.cc:2474): the orbital cut A = orbitals 0..subsystem_size-1 of state (host or device,
 * the space's dimension), M[a][b] = component of the basis state a (x) b in the sector of N_A =
 * nbr_fermion_sector fermions and 2 Lz_A = lz_sector in A, rows in the order of FermionOnSphere(N_A,
 * lz_sector, subsystem_size - 1), columns in that of the complement's FermionOnSphere(N - N_A, .,
 * 2S - subsystem_size).  *rows x *cols (0 x 0 for an empty sector); the matrix is written row-major
 * into matrix (host or device) when it is not NULL and capacity >= rows * cols, so a first call with
 * matrix = NULL gives the size.  subsystem_size <= 0 and > 2S follow the reference (1 x 1 [1]; the state
 * as one column).  Any FermionOnSphere space (2S <= 62, either word engine); FermionOnSphereLong spaces
 * answer DH_ERR_UNSUPPORTED. */
int dh_fermion_on_sphere_partial_entanglement_matrix(dh_space_t space, const double* state, int subsystem_size,
                                                     int nbr_fermion_sector, int lz_sector, double* matrix,
                                                     int64_t capacity, int64_t* rows, int64_t* cols);

/* FermionOnSphere::EvaluatePartialDensityMatrix (FermionOnSphere.cc:2070): rho_A = M M^T of the same
 * cut, *dim x *dim row-major (empty when no basis state lies in the sector).  As in the reference,
 * N_A <= 1 gives the 1 x 1 weight of the states whose A part is empty (N_A = 0) or the single orbital
 * (lz_sector + subsystem_size - 1) / 2 (N_A = 1). */
int dh_fermion_on_sphere_partial_density_matrix(dh_space_t space, const double* state, int subsystem_size,
                                                int nbr_fermion_sector, int lz_sector, double* matrix, int64_t capacity,
                                                int64_t* dim);

/* ================================================================ Hamiltonians */

/* ParticleOnSphereGenericHamiltonian(particles, nbrParticles, lzmax, pseudoPotential, l2Factor, ...):
 * FQHE/src/Hamiltonian/ParticleOnSphereGenericHamiltonian.cc:66-140, interaction factors
 * :493-612, on-the-fly multiplication (memory = 0).  pseudopotentials = V_0..V_lzmax, V_0 being
 * the delta interaction.  l2_factor != 0 adds l2_factor L^2 (the reference's L2Operator,
 * AbstractQHEOnSphereHamiltonian.cc:541-542), as a second two-body table plus the constant
 * l2_factor (Lz^2 + Lz) in the shift (N >= 2).  The Hamiltonian does not own the space
 * (FQHESphereFermionsTwoBodyGeneric.cc:395-396).  On a BosonOnSphereShort space the factors are the
 * reference's bosonic ones (:620-806: pairs m1 >= m2, even relative angular momenta, weights 4, 2 and
 * 1) and the product applies AA / AdAd with their occupation square roots (BosonOnSphereShort.cc:
 * 353, 431).  Bosonic Hamiltonians take the L^2 term (the operator's bosonic branch,
 * ParticleOnSphereL2Hamiltonian.cc:256-368), stored elements (N <= 16) and the pseudopotential
 * adjoint like fermionic ones. */
int dh_particle_on_sphere_generic_hamiltonian_create(dh_space_t space, int nbr_particles, int lz_max,
                                                     const double* pseudopotentials, double l2_factor,
                                                     dh_hamiltonian_t* out);

/* ParticleOnSphereL2Hamiltonian(particles, nbrParticles, lzmax, totalLz, architecture, l2Factor, memory,
 * fixedLz = true, ...) (FQHE/src/Hamiltonian/ParticleOnSphereL2Hamiltonian.cc:73-133, operator
 * :240-368): l2_factor L^2 on the sector, with L^2 = L-L+ + Lz^2 + Lz written as a two-body table
 * (the one-body part folded into the diagonal pairs at fixed N >= 2) and the constant in the shift,
 * so every product form (on the fly, stored elements, blocks) applies it.  <psi|L^2|psi> =
 * L (L + 1) identifies the total angular momentum of a state.  total_lz must be the space's. */
int dh_particle_on_sphere_l2_hamiltonian_create(dh_space_t space, int nbr_particles, int lz_max, int total_lz,
                                                double l2_factor, dh_hamiltonian_t* out);

/* Periodic J1-J2 spin-1/2 chain on a plain Spin1_2Chain: the element pattern of
 * Spin/src/Hamiltonian/SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192 (flips J/2) and
 * :335-352 (diagonal J Sz_i Sz_j) behind the SpinChainHamiltonian API (SpinChainHamiltonian.cc:257).
 * On a Spin1_2ChainWithTranslations space: SpinChainJ1J2RealHamiltonianWithTranslations(chain,
 * nbrSpin, j1, j2) itself, each flip's word taken to its representative with the factor
 * sqrt(o_from / o_to) cos(2 pi K n / L) (SymmetrizeResult, Spin1_2ChainWithTranslations.h:419); only
 * the real sectors K = 0 and K = L / 2 (DH_ERR_UNSUPPORTED otherwise). */
int dh_spin_chain_j1j2_hamiltonian_create(dh_space_t space, double j1, double j2, dh_hamiltonian_t* out);

/* SpinChainJ1J2HamiltonianWithTranslations(chain, nbrSpin, j1, j2)
 * (Spin/src/Hamiltonian/SpinChainJ1J2HamiltonianWithTranslations.cc:62, product :149-247): the complex
 * J1-J2 Hamiltonian of a momentum sector, any K, with the flip element J/2 sqrt(o_from / o_to)
 * exp(2 pi i K m / L) (ExponentialTable, .cc:390).  Its vectors are the reference's ComplexVector
 * storage, (Re, Im) pairs of doubles: every product, matrix-element and Lanczos entry point given this
 * Hamiltonian takes 2 D doubles per vector (dh_hamiltonian_get_dimension returns 2 D), and component
 * ranges count doubles and must be even.  On (Re, Im) pairs the Hermitian H is a real symmetric
 * operator of dimension 2 D whose eigenvalues are H's, each twice, so the Lanczos entry points find
 * H's spectrum and return complex ground states in this layout; the matrix element is Re <v1|H|v2>.
 * One vector per product (row-interleaved blocks, block Lanczos and the autotuner answer
 * DH_ERR_UNSUPPORTED).  Requires a Spin1_2ChainWithTranslations space. */
int dh_spin_chain_j1j2_complex_hamiltonian_create(dh_space_t space, double j1, double j2, dh_hamiltonian_t* out);

int dh_hamiltonian_destroy(dh_hamiltonian_t h);

/* AbstractHamiltonian::GetHilbertSpaceDimension (src/Hamiltonian/AbstractHamiltonian.h:96). */
int dh_hamiltonian_get_dimension(dh_hamiltonian_t h, int64_t* dim);

/* AbstractQHEOnSphereHamiltonian::ShiftHamiltonian (AbstractQHEOnSphereHamiltonian.cc:144):
 * H + shift * 1 in every product. */
int dh_hamiltonian_shift(dh_hamiltonian_t h, double shift);

/* DH_PRECISION_FP64 (default) or DH_PRECISION_FP32 for every following product.  No reference
 * counterpart: the reference's products are FP64. */
int dh_hamiltonian_set_precision(dh_hamiltonian_t h, int precision);

/* Replaces V_0..V_lzmax and rebuilds the interaction factors as EvaluateInteractionFactors does
 * (ParticleOnSphereGenericHamiltonian.cc:493); FQHE Hamiltonians only. */
int dh_hamiltonian_set_pseudopotentials(dh_hamiltonian_t h, const double* pseudopotentials);

/* CUDA stream (a cudaStream_t passed as void*) the handle's work is ordered on.  No reference
 * counterpart. */
int dh_hamiltonian_set_stream(dh_hamiltonian_t h, void* stream);

/* AbstractHamiltonian::LowLevelAddMultiply(vSource, vDestination, firstComponent, nbrComponent)
 * (src/Hamiltonian/AbstractHamiltonian.h:265, FQHE implementation
 * AbstractQHEOnSphereHamiltonian.cc:410): dst += H[:, first:first+nbr] src[first:first+nbr], i.e.
 * the reference's push-form semantics (columns first..first+nbr-1, destination accumulated),
 * computed in pull form with no atomics.  nbr < 0 means "to the end". */
int dh_hamiltonian_low_level_add_multiply(dh_hamiltonian_t h, const double* src, double* dst, int64_t first,
                                          int64_t nbr);

/* AbstractHamiltonian::LowLevelMultiply (AbstractHamiltonian.cc:448-476): clear dst then add. */
int dh_hamiltonian_low_level_multiply(dh_hamiltonian_t h, const double* src, double* dst, int64_t first,
                                      int64_t nbr);

/* AbstractHamiltonian::LowLevelMultipleAddMultiply(vSources, vDestinations, nbrVectors, first, nbr)
 * (AbstractHamiltonian.h:344, AbstractQHEOnSphereHamiltonian.cc:1217): srcs and dsts hold
 * nbr_vectors vectors of the full dimension one after the other (the RealVector array). */
int dh_hamiltonian_low_level_multiple_add_multiply(dh_hamiltonian_t h, const double* srcs, double* dsts,
                                                   int nbr_vectors, int64_t first, int64_t nbr);

/* y = H x for a block of k vectors stored row-interleaved (x[i * k + j] = component i of vector j,
 * a row-major (dim, k) array), host or device pointers.  One enumeration of each row's matrix
 * elements serves the whole block, with vector loads for k = 2 and 4.  No reference counterpart:
 * LowLevelMultipleAddMultiply (AbstractHamiltonian.h) takes k separate vectors; this is its form
 * for blocks kept interleaved, as the block Lanczos and (dim, k) torch tensors keep them. */
int dh_hamiltonian_block_multiply(dh_hamiltonian_t h, const double* x, double* y, int k);

/* EnableFastMultiplication / FastMultiplicationMemory (AbstractQHEOnSphereHamiltonian.cc:3625,3814):
 * precompute every row's matrix elements (target index, interaction-factor index and sign; the
 * diagonal moves summed per row) in device memory, as sliced ELL (32-row slices padded to their
 * longest row), when they take at most allowed_memory bytes (< 0: no budget) and fit in the free
 * device memory; every later full product of this Hamiltonian then reads them instead of
 * enumerating the moves.  *bytes = the memory the structure needs (set even when it is not built),
 * *enabled = 1 if it was built.  The elements do not depend on the pseudopotentials: setting new
 * ones only recomputes the diagonal.  FermionOnSphere, FermionOnSphereLong and BosonOnSphereShort
 * Hamiltonians; a bosonic element stores, beside its target, the factor index and the two occupation
 * products under its square roots in 8 bits each (N <= 16, else DH_ERR_UNSUPPORTED); an element of the
 * 128-bit engine (FermionOnSphereLong, FermionOnSphere above 40 orbitals) a 31-bit factor index and its
 * sign.  Partial column ranges stay on the fly. */
int dh_hamiltonian_enable_fast_multiplication(dh_hamiltonian_t h, int64_t allowed_memory, int* enabled,
                                              int64_t* bytes);
/* Frees the stored elements: products go back to the on-the-fly kernels.  No reference counterpart
 * (the reference frees them with the Hamiltonian, AbstractQHEOnSphereHamiltonian.cc:3625 allocates). */
int dh_hamiltonian_disable_fast_multiplication(dh_hamiltonian_t h);

/* Autotuner of the product (no reference counterpart): times this Hamiltonian's product on random
 * blocks of block_size vectors (1, 2 or 4; the precision currently set), median of `repeats`
 * CUDA-event timings per candidate, and keeps the fastest FQHE kernel form: split-word rank tables
 * read through L1, split-word with the low-rank table staged in shared memory, or the generic
 * kernel, over rank-table splits LB = default - 2 .. default + 2.  Every candidate computes the
 * same product (the rank function does not depend on the split).  Spin chains have one form.
 * When stored elements exist (dh_hamiltonian_enable_fast_multiplication) their product is timed too
 * and stays in use only if it is the fastest.
 * For the split-word kernel it then times its launch forms at the chosen split (threads per block
 * 256, 192 or 128, resident blocks per SM, i.e. the register budget per thread, and a gather pipeline
 * that keeps four target rows in flight per thread instead of two) and keeps the fastest.
 * out (optional, DH_TUNE_RESULTS doubles): best ms per product, kernel variant (0 split-word,
 * 1 generic, 2 staged table), LB, ms per product of blocks of 1, 2 and 4 vectors with the chosen
 * form, number of candidates timed, ms of the stored-element product (0: none), 1 if the stored
 * elements are in use, launch form of the split-word kernel (0 .. 7: 256 threads x 4 resident
 * blocks, 256 x 3, 256 x 3 pipelined, 256 x 2 pipelined, 128 x 8, 256 x 2, 192 x 4, 128 x 6), the
 * stored-element product's read-ahead depth per lane (8 or 16 elements; 0 without stored elements),
 * which is timed at both depths. */
#define DH_TUNE_RESULTS 11
int dh_hamiltonian_autotune(dh_hamiltonian_t h, int block_size, int repeats, double* out);

/* AbstractHamiltonian::MatrixElement(V1, V2) (AbstractQHEOnSphereHamiltonian.cc:380): <v1|H|v2>. */
int dh_hamiltonian_matrix_element(dh_hamiltonian_t h, const double* v1, const double* v2, double* out);

/* Per-row element list of the on-the-fly product, the contract of
 * AbstractQHEOnSphereHamiltonian::EvaluateMNTwoBodyFastMultiplicationComponent (.h:531):
 * target index, sign (+1/-1) of AA*AdAd and interaction-factor index for every generated element
 * of `row`, in the reference enumeration order.  *count receives the total; at most cap entries
 * are written.  FermionOnSphere Hamiltonians (up to 40 orbitals) only. */
int dh_hamiltonian_row_elements(dh_hamiltonian_t h, int64_t row, int* targets, int* signs, int* factor_index,
                                int cap, int* count);

/* Adjoint of the pseudopotentials (Hellmann-Feynman / bilinear VJP): out[m] = <u| dH/dV_m |v> for
 * m = 0..lz_max.  With u = v = normalised ground state this is dE0/dV_m; with u = upstream gradient
 * and v = x it is the V part of the vector-Jacobian product of H(V) x.  FermionOnSphere(Long) and
 * BosonOnSphereShort interaction Hamiltonians (the 128-bit engine accumulates into the global bins with
 * atomics once its factor table outgrows shared memory, 2S above about 54).  No reference counterpart;
 * its oracle is MatrixElement (AbstractQHEOnSphereHamiltonian.cc:380) of the Hamiltonian with V = e_m. */
int dh_hamiltonian_pseudopotential_adjoint(dh_hamiltonian_t h, const double* u, const double* v, double* out);

/* Number of elements (a+a+aa moves, diagonal ones included; spin flips for the chain) that one
 * product generates over all rows, counted on the GPU: the total of the per-row counting pass of
 * FastMultiplicationMemory (AbstractQHEOnSphereHamiltonian.cc:3625). */
int dh_hamiltonian_count_elements(dh_hamiltonian_t h, int64_t* total);

/* Of those, the elements whose target is their own row (one per annihilated pair for FQHE spaces:
 * C(N, 2) per row for fermions, the number of pairs a_m1 a_m2 can empty for bosons; 0 for the chain,
 * whose elements are its flips).  count_elements - this = the off-diagonal elements, the gathers
 * of distinct targets in the algorithmic byte count.  No reference counterpart. */
int dh_hamiltonian_count_diagonal_elements(dh_hamiltonian_t h, int64_t* total);

/* Same result as dh_hamiltonian_pseudopotential_adjoint, for callers that cannot allocate device
 * memory: applications whose framework owns all device memory through its own allocator or a
 * fixed arena, where a cudaMalloc made by a library fails or breaks the framework's accounting.
 * No counterpart in the reference.
 * It allocates nothing (no cudaMalloc / cudaFree, no staging): u and v must be device pointers;
 * out (lz_max + 1 values) may be host or device memory.  Its per-block scratch is a static device
 * array sized for DH_STATIC_ADJOINT_BLOCKS x DH_STATIC_ADJOINT_MAX_FACTORS doubles (about 7.6 MB,
 * held by every GPU that loads the library until the process exits); Hamiltonians with more
 * interaction factors (lz_max > 33) are rejected with DH_ERR_UNSUPPORTED.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress with that device current).
 * The device that was current when the Hamiltonian's space was created must be current for the
 * call (DH_ERR_STATE otherwise).  The call is synchronous: it waits on the handle's stream and
 * returns with the result written to out.  All calls of a process share its one array; a
 * process-wide mutex serialises them (on every GPU), so calls never overlap on it, and every
 * process has an array of its own.  Each call overwrites what it uses, so the contents left by a
 * previous call do not matter. */
#define DH_STATIC_ADJOINT_BLOCKS 148
#define DH_STATIC_ADJOINT_MAX_FACTORS 6400
int dh_hamiltonian_pseudopotential_adjoint_static(dh_hamiltonian_t h, const double* u, const double* v, double* out);

/* Interaction factors of the current V (flattened in the reference order,
 * ParticleOnSphereGenericHamiltonian.cc:566-606) and their count. */
int dh_hamiltonian_get_interaction_factors(dh_hamiltonian_t h, double* factors, int cap, int* count);

/* ================================================================ Lanczos */

/* Creates one of the reference's Lanczos algorithms on the GPU: AbstractLanczosAlgorithm
 * (src/LanczosAlgorithm/AbstractLanczosAlgorithm.h:45-120) with the recurrence of
 * BasicLanczosAlgorithm.cc:148-216, FullReorthogonalizedLanczosAlgorithm.cc:209-323,
 * BasicBlockLanczosAlgorithm.cc:524-697 or BasicLanczosAlgorithmWithGroundState.cc:256-335.
 * Lanczos vectors stay in FP64 in device memory.  block_size (1, 2 or 4) is used by
 * DH_LANCZOS_BLOCK only: the block is stored row-interleaved and one product enumerates each row's
 * matrix elements once for the whole block; max_iter counts vectors, as the reference's --iter-max,
 * and RunLanczosAlgorithm counts block steps.  The block algorithm keeps every block when they fit
 * in half of the free device memory, otherwise it rebuilds Ritz vectors by replaying its recorded
 * steps. */
int dh_lanczos_create(dh_hamiltonian_t h, int algorithm, int nbr_eigenvalue, int block_size, int max_iter,
                      dh_lanczos_t* out);
int dh_lanczos_destroy(dh_lanczos_t l);

/* Keep every Lanczos vector in device memory (keep = 1, default when it fits in half of the free
 * memory) or only three and rebuild the ground state by a second pass (keep = 0), the store-or-
 * recompute choice of BasicLanczosAlgorithmWithGroundState (DiskFlag, .cc:256-335).  Call before
 * dh_lanczos_initialize. */
int dh_lanczos_set_vector_storage(dh_lanczos_t l, int keep);

/* SetEigenvaluePrecision (AbstractLanczosAlgorithm.h:147); default 1e-14 = MACHINE_PRECISION. */
int dh_lanczos_set_eigenvalue_precision(dh_lanczos_t l, double precision);

/* InitializeLanczosAlgorithm(vector) / (vectors, nbrVectors) (AbstractLanczosAlgorithm.h:83, :89): nbr_vectors
 * vectors one after the other (host or device).  Block algorithms orthonormalise the block; others use
 * vectors[0]. */
int dh_lanczos_initialize(dh_lanczos_t l, const double* vectors, int nbr_vectors);

/* InitializeLanczosAlgorithm() (AbstractLanczosAlgorithm.h:78) with a reproducible start: component i of vector b is the
 * (i+1)-th splitmix64 output of seed + b mapped to [-1, 1), then normalised. */
int dh_lanczos_initialize_random(dh_lanczos_t l, uint64_t seed);

/* RunLanczosAlgorithm(nbrIter) (BasicLanczosAlgorithm.cc:148). */
int dh_lanczos_run(dh_lanczos_t l, int nbr_iter);

/* TestConvergence (BasicLanczosAlgorithm.cc:220, BasicBlockLanczosAlgorithm.cc:731). */
int dh_lanczos_test_convergence(dh_lanczos_t l, int* converged);

/* Lowest n Ritz values, ascending: GetEigenvalues (AbstractLanczosAlgorithm.h:121), i.e. GetDiagonalizedMatrix
 * (:137) + SortMatrixUpOrder. */
int dh_lanczos_get_eigenvalues(dh_lanczos_t l, double* eigenvalues, int n);

/* GetGroundStateEnergy (AbstractLanczosAlgorithm.cc:136-150). */
int dh_lanczos_get_ground_state_energy(dh_lanczos_t l, double* energy);

/* GetGroundState (BasicLanczosAlgorithmWithGroundState.cc:256-335): normalised Ritz vector of the
 * lowest Ritz value, written to vec (host or device). */
int dh_lanczos_get_ground_state(dh_lanczos_t l, double* vec);

/* GetEigenstates(nbrEigenstates) (BasicBlockLanczosAlgorithm.cc:380-500,
 * BasicLanczosAlgorithmWithGroundState.cc:256-335): the n lowest normalised Ritz vectors, one after
 * the other in vecs (host or device).  Block algorithms give up to block_size of them; the others
 * need the stored Krylov vectors for n > 1. */
int dh_lanczos_get_eigenstates(dh_lanczos_t l, int n, double* vecs);

/* Number of matrix-vector products and tridiagonal rows so far.  No reference counterpart (the
 * driver loop counts its own iterations, QHEOnSphereMainTask.cc:732-753). */
int dh_lanczos_get_counters(dh_lanczos_t l, int64_t* matvecs, int* rows);

/* Whole driver loop of QHEOnSphereMainTask.cc:732-753: RunLanczosAlgorithm(nbrEigenvalue + 2), then
 * RunLanczosAlgorithm(1) until TestConvergence() or max_iter iterations, issued as CUDA-graph
 * batches of at most `graph_batch` iterations (>= 1) whose extra iterations past convergence are
 * discarded from the reported result.  Under the eigenvalue test a batch is cut short where the
 * test is predicted to pass (its ratio to the threshold decays about geometrically), so fewer
 * products are issued past convergence; the iterations, and so the results, are those of
 * graph_batch = 1.  *iterations follows the reference's iteration counter (in vectors:
 * (nbrEigenvalue + 3) block_size after the first call, + block_size per step for DH_LANCZOS_BLOCK,
 * whose steps are never graph-batched). */
int dh_lanczos_solve(dh_lanczos_t l, int max_iter, int graph_batch, double* eigenvalues, int* iterations,
                     int* converged);

/* FP32-matvec Lanczos with FP64 recurrence followed by FP64 refinement of the ground state:
 * the Ritz vector is rebuilt from the stored Krylov basis, its FP64 Rayleigh quotient and residual
 * are taken with an FP64 product, and, while the residual bound exceeds `precision` * |E|, a short
 * FP64 Lanczos restarted from it polishes the energy.  out[0] = refined E0, out[1] = FP32-phase E0,
 * out[2] = residual norm, out[3] = FP32 matvecs, out[4] = FP64 matvecs.  With DH_LANCZOS_BLOCK the
 * whole block of Ritz vectors is refined and the FP64 restart is a block Lanczos from it; the
 * algorithm must be freshly initialised.  No reference counterpart: the reference's Lanczos runs its
 * products in FP64 throughout (BasicLanczosAlgorithm.cc:148-216). */
int dh_lanczos_solve_refined(dh_lanczos_t l, int max_iter, double precision, double* out);

/* Block-size tuner: solves H's ground energy to `precision` with k = 1 (DH_LANCZOS_BASIC), 2 and 4
 * (DH_LANCZOS_BLOCK) from the same seeded start, FP32 products + FP64 refinement when refined != 0
 * (dh_lanczos_solve_refined), else FP64 products (dh_lanczos_solve), and returns in *best_k the block
 * size with the shortest wall time to the converged energy (the time per converged Ritz value: a
 * larger block costs more per step and needs fewer steps).  seconds (optional, 3 doubles): the time
 * of each k (0 where a k does not apply).  The Hamiltonian's precision is left as it was.  No
 * reference counterpart: the reference's block size is the --block-size option. */
int dh_hamiltonian_tune_block_size(dh_hamiltonian_t h, int max_iter, double precision, int refined, int* best_k,
                                   double* seconds);

/* Disk storage of the Lanczos state, in the files of the reference's disk-storage classes, so that an
 * interrupted run resumes (here or in the reference) where it stopped:
 *   DH_LANCZOS_BASIC             BasicLanczosAlgorithmWithDiskStorage (src/LanczosAlgorithm/
 *                                BasicLanczosAlgorithmWithDiskStorage.cc:286-335): lanczos.dat and three
 *                                vector files v_Index, v_Index+1, H v_Index+1 named in it;
 *   DH_LANCZOS_WITH_GROUND_STATE BasicLanczosAlgorithmWithGroundStateDiskStorage (...WithGroundState
 *                                DiskStorage.cc:399-453): lanczos.dat, vector.0 (the start vector,
 *                                written by dh_lanczos_initialize*) and vector.1-3 (the same three).
 * The files live in `directory` (the reference uses the working directory).  A checkpoint is written
 * at the end of every RunLanczosAlgorithm call that has added `interval` (>= 1) or more rows since the
 * last one, and at the end of dh_lanczos_solve; interval 1 is the reference's behaviour.  The vectors
 * are copied to pinned host memory on the handle's stream and written by a background thread while
 * the next iterations run; each file goes to a temporary name and is renamed into place, lanczos.dat
 * last.  The basic format alternates between the names vector1-3 and vector4-6 (lanczos.dat names
 * them), so the previous checkpoint stays whole until the new lanczos.dat replaces it.  directory =
 * NULL switches disk storage off.  Other algorithms: DH_ERR_UNSUPPORTED.  Solves with disk storage
 * run without CUDA-graph batches; dh_lanczos_solve_refined rejects it. */
int dh_lanczos_set_disk_storage(dh_lanczos_t l, const char* directory, int interval);

/* WriteState (BasicLanczosAlgorithmWithDiskStorage.cc:286, BasicLanczosAlgorithmWithGroundStateDiskStorage.cc:399):
 * a checkpoint of the current state now; returns once every file is written. */
int dh_lanczos_write_state(dh_lanczos_t l);

/* ResumeLanczosAlgorithm (BasicLanczosAlgorithmWithDiskStorage.cc:161,
 * BasicLanczosAlgorithmWithGroundStateDiskStorage.cc:175): the state in the disk-storage directory
 * replaces dh_lanczos_initialize*.  EigenvaluePrecision and PreviousLastWantedEigenvalue come from the
 * file.  A state written in the middle of a reference RunLanczosAlgorithm call (NbrRow above Index +
 * 2) owes its remaining rows to the next run call, which adds them before its own, as the reference
 * does.  dh_lanczos_solve after a resume continues the driver loop without its first call and counts
 * iterations from 0 (QHEOnSphereMainTask.cc:730-736 with --resume).  A ground-state-format state
 * written during the reference's ground-state evaluation (GroundStateEvaluationFlag 1) holds a
 * finished run: it resumes for dh_lanczos_get_ground_state only (rebuilt from vector.0 and the
 * tridiagonal matrix).  The basic format does not store the start vector, so its resumed runs give
 * eigenvalues but no ground state. */
int dh_lanczos_resume(dh_lanczos_t l);

/* ================================================================ vector files */

/* RealVector::WriteVector (src/Vector/RealVector.cc:3669): little-endian int32 dimension (int32 -1
 * and an int64 dimension from 2^31 on), then the components as little-endian doubles.  vec is a host
 * or device pointer; the file is written under a temporary name and renamed into place.  Eigenstate
 * files are named <prefix>.<index>.vec, prefix = statistics_interaction_n_N_2s_2S_lz_2Lz
 * (FQHE/docs/DataFormat/FermionOnSphere.xml:9-16, QHEOnSphereMainTask.cc:891). */
int dh_vector_write(const char* file_name, const double* vec, int64_t dim);

/* The dimension of the vector stored in file_name: RealVector::ReadVectorDimension (RealVector.cc:3914). */
int dh_vector_file_dimension(const char* file_name, int64_t* dim);

/* RealVector::ReadVector (src/Vector/RealVector.cc:3798) into vec (host or device) of dim doubles:
 * the stored dimension must be dim and the file length must match it exactly (DH_ERR_IO otherwise). */
int dh_vector_read(const char* file_name, double* vec, int64_t dim);

/* ComplexVector::WriteVector (src/Vector/ComplexVector.cc:2606): the same header with the number of
 * complex components dim, then dim (Re, Im) pairs of little-endian doubles; pairs holds 2 dim doubles
 * (host or device), the storage of a complex vector of the complex momentum-sector Hamiltonian. */
int dh_complex_vector_write(const char* file_name, const double* pairs, int64_t dim);

/* The number of complex components of the vector stored in file_name: ComplexVector::ReadVectorDimension
 * (ComplexVector.cc:2854). */
int dh_complex_vector_file_dimension(const char* file_name, int64_t* dim);

/* ComplexVector::ReadVector (src/Vector/ComplexVector.cc:2722) into pairs (host or device, 2 dim doubles);
 * the stored dimension and the file length must match dim (DH_ERR_IO otherwise). */
int dh_complex_vector_read(const char* file_name, double* pairs, int64_t dim);

/* ================================================================ batched sectors */

/* All requested Lz sectors of N fermions in 2S+1 orbitals with one two-body interaction, solved by
 * block Lanczos (block_size vectors per sector, BasicBlockLanczosAlgorithm.cc:524-697) in lockstep:
 * each block product is one launch over every sector, and the block recurrence runs on every
 * sector at once.  Each sector follows the reference's driver loop and convergence test
 * (QHEOnSphereMainTask.cc:732-753, precision_target = the Lanczos precision, max_iter in vectors).
 * Sectors of dimension <= full_diag_limit (or <= 2 block_size) are diagonalised densely, as
 * QHEOnSphereMainTask does below --full-diag (:397); so are sectors whose block Krylov space runs
 * out with a band matrix that is not exact (a last block that only lost rank, or FP32 products).
 * precision == DH_PRECISION_FP32: FP32 products with the FP64 recurrence until each sector's Ritz
 * residual (from its band matrix) falls below max(0.1 precision_target, 1e-11) |E| or its lowest Ritz
 * value stops moving; then every sector's lowest Ritz vector gets an FP64
 * Rayleigh quotient and residual, and the sectors whose |r|^2 > precision_target |E| are polished
 * by an FP64 block Lanczos restarted from their Ritz blocks, all of them in lockstep.
 * energies[s] = lowest eigenvalue of sector s, iterations[s] = the driver's counter (both phases;
 * 0 for dense sectors); stats (optional, DH_SECTOR_STATS values): set-up seconds, solve seconds,
 * device time of the block products, number of block products, FP32-phase seconds, refinement
 * seconds, number of sectors restarted in FP64, largest |E_refined - E_FP32| over the sectors,
 * number of sectors diagonalised densely after an exhausted Krylov space, seconds spent on them,
 * bytes of the stored elements (0: products on the fly), seconds spent building them.
 * allowed_memory: the reference's --memory (FastMultiplicationMemory / EnableFastMultiplication,
 * AbstractQHEOnSphereHamiltonian.cc:3625,3814) for the whole batch: 0 computes every product on the
 * fly; otherwise the Lanczos sectors' elements are stored once as one sliced ELL over their
 * concatenated rows when they take at most allowed_memory bytes (< 0: no budget) and fit in the free
 * device memory, and the first phase's products (and the FP64 checks) stream them; the rows of
 * converged sectors are skipped either way.  The sectors share the split-word rank tables:
 * lz_max <= 40 (DH_ERR_UNSUPPORTED above).  The Krylov blocks the refinement needs are kept in
 * device memory as far as half of the free memory allows (growing with the run), else rebuilt by
 * replaying the recurrence. */
#define DH_SECTOR_STATS 12
int dh_fqhe_sectors_block_lanczos(int nbr_fermions, int lz_max, const int* total_lz, int nbr_sectors,
                                  const double* pseudopotentials, int block_size, int max_iter,
                                  double precision_target, int precision, int full_diag_limit,
                                  int64_t allowed_memory, uint64_t seed, double* energies, int* iterations,
                                  double* stats);

/* ================================================================ setup helpers */

/* EvaluatePseudopotentials(nbrFlux, 0, 0.0) (FQHE/src/Tools/FQHESpectrum/PseudoPotentials.cc:35):
 * lowest-Landau-level Coulomb V_0..V_nbrFlux on the sphere, FP64 on the host. */
int dh_coulomb_pseudopotentials(int nbr_flux, double* v);

/* ClebschGordanCoefficients::GetCoefficient (src/MathTools/ClebschGordanCoefficients.cc:136),
 * every argument doubled. */
int dh_clebsch_gordan(int j1, int m1, int j2, int m2, int j, double* out);

#ifdef __cplusplus
}
#endif
#endif

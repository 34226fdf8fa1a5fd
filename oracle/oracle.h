/* oracle.h -- CPU restatement of DiagHam's on-the-fly H.v + Lanczos path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load liboracle.so, and only as the checker.
 * The product (diagham_b200) never links or calls it.
 *
 * Pinning: every function below is checked against golden vectors produced by
 * the reference itself (oracle/_ref/ref_tool, built from the reference sources
 * by oracle/Makefile) and committed under tests/golden/, and against the
 * documented basis order of FQHE/docs/DataFormat/FermionOnSphere.xml:19-40.
 *
 * Conventions (all in the reference's own units):
 *   lz_max   = 2S (orbitals 0..lz_max, orbital m has Lz = m - S)
 *   total_lz = twice the total Lz
 *   words    = occupation bitstrings, bit m = orbital m (FermionOnSphere) or
 *              site i (Spin1_2Chain, bit set = spin up)
 */
#ifndef DIAGHAM_ORACLE_H
#define DIAGHAM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- fermions on the sphere (FQHE/src/HilbertSpace/FermionOnSphere.cc) ---- */
long orc_fermion_dimension(int nbr_fermions, int total_lz, int lz_max);
long orc_fermion_basis(int nbr_fermions, int total_lz, int lz_max, uint64_t* words, int* state_lz_max);
int orc_lookup_shift_from_memory(int lz_max, unsigned long memory);
void orc_fermion_lookup_table(const uint64_t* words, const int* state_lz_max, long dim, int lz_max,
                              int max_shift, int* table, int* table_shift);
long orc_fermion_find_state_index(const uint64_t* words, long dim, const int* table, const int* table_shift,
                                  int max_shift, uint64_t word, int lzmax);
double orc_fermion_aa(uint64_t state, int n1, int n2, uint64_t* out);
double orc_fermion_adad(uint64_t state, int m1, int m2, uint64_t* out);

/* ---- interaction (ParticleOnSphereGenericHamiltonian.cc:493-612) ---- */
double orc_clebsch_gordan(int j1, int m1, int j2, int m2, int j);
int orc_nbr_pairs(int lz_max);
int orc_interaction_tables(int lz_max, const double* pseudopotentials, int* m1v, int* m2v, int* nbr_m3,
                           int* m3_offset, int* m3v, double* factors);
int orc_interaction_derivatives(int lz_max, double* dfactors);
void orc_coulomb_pseudopotentials(int nbr_flux, double* v);

/* ---- matvec (AbstractQHEOnSphereHamiltonian.cc:410-552) ---- */
typedef struct
{
  int nbr_fermions, lz_max, total_lz;
  long dim;
  const uint64_t* words;
  const int* state_lz_max;
  const int* table;
  const int* table_shift;
  int max_shift;
  int nbr_pairs;
  const int* m1v;
  const int* m2v;
  const int* nbr_m3;
  const int* m3_offset;
  const int* m3v;
  const double* factors;
  double shift;
} orc_fqhe_t;

void orc_fqhe_push_add_multiply(const orc_fqhe_t* h, const double* x, double* y, long first, long nbr);
void orc_fqhe_pull_multiply(const orc_fqhe_t* h, const double* x, double* y);
long orc_fqhe_row_elements(const orc_fqhe_t* h, long row, int* target, int* sign, int* factor_index, long cap);
void orc_fqhe_expectation_bins(const orc_fqhe_t* h, const double* u, const double* v, double* bins);

/* BosonOnSphereShort: occupations <-> fermionic words, AA / AdAd, the bosonic factors and the product
 * (h holds the FermionOnSphere(N, 2Lz, lz_max + N - 1) words and the bosonic tables) */
void orc_boson_unpack(uint64_t w, int lz_max, int* n);
uint64_t orc_boson_pack(const int* n, int lz_max);
double orc_boson_aa(const int* occ, int lz_max, int n1, int n2, int* out);
double orc_boson_adad(const int* occ, int lz_max, int m1, int m2, uint64_t* out);
int orc_boson_nbr_pairs(int lz_max);
int orc_boson_interaction_tables(int lz_max, const double* v, int* m1v, int* m2v, int* nbr_m3, int* m3_offset,
                                 int* m3v, double* factors);
void orc_boson_push_add_multiply(const orc_fqhe_t* h, const double* x, double* y, long first, long nbr);
void orc_boson_pull_multiply(const orc_fqhe_t* h, const double* x, double* y);
void orc_boson_matvec_cb(void* ctx, const double* x, double* y);

/* ---- spin-1/2 chain (Spin/src/HilbertSpace/Spin1_2Chain.cc) ---- */
long orc_spin_dimension(int length, int sz);
long orc_spin_basis(int length, int sz, uint64_t* words);
long orc_spin_find_state_index(int length, int sz, uint64_t word);
void orc_spin_j1j2_multiply(int length, int sz, const uint64_t* words, long dim, double j1, double j2,
                            double shift, const double* x, double* y);

/* ---- deterministic start vectors (shared with the product and the tests) ---- */
void orc_random_vector(uint64_t seed, long dim, double* x);

/* ---- Lanczos (src/LanczosAlgorithm/BasicLanczosAlgorithm.cc:98-228) ---- */
typedef void (*orc_matvec_fn)(void* ctx, const double* x, double* y);
int orc_tridiagonal_eigenvalues(int n, const double* diag, const double* off, double* eig);
int orc_symmetric_eigen(int n, double* a, double* eig, double* vecs);
int orc_basic_lanczos(orc_matvec_fn mv, void* ctx, long dim, const double* v0, int nev, int max_iter,
                      double precision, double* eigenvalues, int* iterations, double* alpha, double* beta);
void orc_fqhe_matvec_cb(void* ctx, const double* x, double* y);

#ifdef __cplusplus
}
#endif
#endif

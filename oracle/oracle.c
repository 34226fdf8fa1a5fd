/* oracle.c -- CPU restatement of DiagHam's on-the-fly H.v + Lanczos path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Plain C, FP64, single thread.
 * Each function cites the reference file:line whose behaviour it restates.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ===================================================================== */
/* fermions on the sphere                                                 */
/* ===================================================================== */

/* number of ways to put n fermions in orbitals 0..o-1 with orbital-index sum s */
static long count_subsets(int n, int o, int s)
{
  if (n == 0)
    return s == 0 ? 1 : 0;
  if (o < n || s < 0)
    return 0;
  long lo = (long) n * (n - 1) / 2;
  long hi = (long) n * (2 * o - n - 1) / 2;
  if (s < lo || s > hi)
    return 0;
  /* either orbital o-1 is occupied or it is not */
  return count_subsets(n - 1, o - 1, s - (o - 1)) + count_subsets(n, o - 1, s);
}

/* FermionOnSphere::EvaluateHilbertSpaceDimension, FermionOnSphere.cc:1794-1826 */
long orc_fermion_dimension(int nbr_fermions, int total_lz, int lz_max)
{
  if (nbr_fermions == 0)
    return 1;
  int twice = total_lz + nbr_fermions * lz_max;
  if (twice < 0 || (twice & 1))
    return 0;
  return count_subsets(nbr_fermions, lz_max + 1, twice / 2);
}

typedef struct
{
  uint64_t* words;
  int* lzmax;
  long pos;
} gen_ctx;

/* places the highest remaining fermion first, highest orbital first: this yields the basis
 * sorted in descending uint64 order, which is the order of FermionOnSphere::GenerateStates
 * (FermionOnSphere.cc:1621-1653; documented in FQHE/docs/DataFormat/FermionOnSphere.xml:19-40) */
static void gen_fermions(gen_ctx* c, int n, int top, int s, uint64_t prefix)
{
  if (n == 0)
    {
      if (s == 0)
        {
          if (c->words)
            c->words[c->pos] = prefix;
          if (c->lzmax)
            c->lzmax[c->pos] = prefix ? 63 - __builtin_clzll(prefix) : 0;
          c->pos++;
        }
      return;
    }
  for (int p = top; p >= n - 1; --p)
    {
      int rem = s - p;
      long lo = (long) (n - 1) * (n - 2) / 2;
      long hi = (long) (n - 1) * (2 * p - n) / 2; /* n-1 fermions in orbitals 0..p-1 */
      if (rem < lo)
        continue;
      if (rem > hi)
        break; /* lower p only lowers the reachable maximum */
      gen_fermions(c, n - 1, p - 1, rem, prefix | (1ull << p));
    }
}

long orc_fermion_basis(int nbr_fermions, int total_lz, int lz_max, uint64_t* words, int* state_lz_max)
{
  if (nbr_fermions == 0)
    {
      if (words)
        words[0] = 0;
      if (state_lz_max)
        state_lz_max[0] = 0;
      return 1;
    }
  int twice = total_lz + nbr_fermions * lz_max;
  if (twice < 0 || (twice & 1))
    return 0;
  gen_ctx c = {words, state_lz_max, 0};
  gen_fermions(&c, nbr_fermions, lz_max, twice / 2, 0);
  return c.pos;
}

/* FermionOnSphere::GenerateLookUpTable, FermionOnSphere.cc:1659-1668: the table width is derived
 * from the memory budget divided by (pointer size x number of orbitals) */
int orc_lookup_shift_from_memory(int lz_max, unsigned long memory)
{
  memory /= (sizeof(int*) * (unsigned long) (lz_max + 1));
  int shift = 1;
  while (memory > 0)
    {
      memory >>= 1;
      ++shift;
    }
  if (shift > lz_max + 1)
    shift = lz_max + 1;
  return shift;
}

/* Lookup-table semantics of FermionOnSphere.cc:1659-1743.  For every highest-occupied orbital l,
 * table[l][v] (v = 0 .. 2^max_shift) is the first basis index, within the block of states whose
 * highest bit is l, at which (word >> table_shift[l]) drops below v; v above the block's largest
 * prefix gives the block start and v at or below its smallest prefix gives the block end (the
 * next block's first index, or dim - 1 for the last block).  Tables of absent l are left as -1. */
void orc_fermion_lookup_table(const uint64_t* words, const int* state_lz_max, long dim, int lz_max,
                              int max_shift, int* table, int* table_shift)
{
  long width = (1l << max_shift) + 1;
  for (long i = 0; i < (long) (lz_max + 1) * width; ++i)
    table[i] = -1;
  for (int l = 0; l <= lz_max; ++l)
    table_shift[l] = (l < max_shift) ? 0 : l + 1 - max_shift;
  long start = 0;
  while (start < dim)
    {
      int l = state_lz_max[start];
      long end = start;
      while (end < dim && state_lz_max[end] == l)
        ++end;
      int* t = table + (long) l * width;
      int sh = table_shift[l];
      long block_end = (end < dim) ? end : dim - 1;
      /* walk v downward; idx advances to the first state whose prefix is < v */
      long idx = start;
      for (long v = width - 1; v >= 0; --v)
        {
          while (idx < end && (long) (words[idx] >> sh) >= v)
            ++idx;
          t[v] = (int) ((idx < end) ? idx : block_end);
        }
      start = end;
    }
}

/* FermionOnSphere::FindStateIndex, FermionOnSphere.cc:1431-1455: binary search on the
 * descending word array inside the bracket given by the lookup table */
long orc_fermion_find_state_index(const uint64_t* words, long dim, const int* table, const int* table_shift,
                                  int max_shift, uint64_t word, int lzmax)
{
  (void) dim;
  long width = (1l << max_shift) + 1;
  const int* t = table + (long) lzmax * width;
  long v = (long) (word >> table_shift[lzmax]);
  long hi_state = t[v + 1]; /* smaller index end: larger words */
  long lo_state = t[v];     /* larger index end */
  long a = hi_state, b = lo_state;
  while (b - a > 1)
    {
      long mid = (a + b) >> 1;
      if (words[mid] > word)
        a = mid;
      else
        b = mid;
    }
  if (words[a] == word)
    return a;
  return b;
}

static inline double parity_sign(uint64_t x)
{
  return (__builtin_popcountll(x) & 1) ? -1.0 : 1.0;
}

/* FermionOnSphere::AA, FermionOnSphere.cc:790-825 (annihilate n2 then n1; each sign is the
 * parity of the occupied orbitals at and above the annihilated one) */
double orc_fermion_aa(uint64_t state, int n1, int n2, uint64_t* out)
{
  if (n1 == n2 || !((state >> n1) & 1) || !((state >> n2) & 1))
    return 0.0;
  double c = parity_sign(state >> n2);
  state &= ~(1ull << n2);
  c *= parity_sign(state >> n1);
  state &= ~(1ull << n1);
  *out = state;
  return c;
}

/* FermionOnSphere::AdAd, FermionOnSphere.cc:949-995 (create m2 then m1; each sign is the parity
 * of the occupied orbitals above the created one) */
double orc_fermion_adad(uint64_t state, int m1, int m2, uint64_t* out)
{
  if ((state >> m2) & 1)
    return 0.0;
  double c = parity_sign(state >> m2);
  state |= 1ull << m2;
  if ((state >> m1) & 1)
    return 0.0;
  c *= parity_sign(state >> m1);
  state |= 1ull << m1;
  *out = state;
  return c;
}

/* ===================================================================== */
/* Clebsch-Gordan coefficients: Racah's closed formula evaluated in        */
/* double-double arithmetic (about 32 significant digits), so the          */
/* alternating sum keeps full double precision after cancellation.        */
/* ===================================================================== */

typedef struct
{
  double hi, lo;
} dd;

static inline dd dd_from(double a)
{
  dd r = {a, 0.0};
  return r;
}
static inline dd two_sum(double a, double b)
{
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  dd r = {s, e};
  return r;
}
static inline dd dd_add(dd a, dd b)
{
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return two_sum(s.hi, s.lo);
}
static inline dd dd_neg(dd a)
{
  dd r = {-a.hi, -a.lo};
  return r;
}
static inline dd dd_mul(dd a, dd b)
{
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return two_sum(p, e);
}
static inline dd dd_div(dd a, dd b)
{
  double q1 = a.hi / b.hi;
  dd r = dd_add(a, dd_neg(dd_mul(dd_from(q1), b)));
  double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul(dd_from(q2), b)));
  double q3 = r.hi / b.hi;
  return dd_add(two_sum(q1, q2), dd_from(q3));
}
static inline dd dd_sqrt(dd a)
{
  if (a.hi <= 0.0)
    return dd_from(0.0);
  double x = sqrt(a.hi);
  dd xx = dd_mul(dd_from(x), dd_from(x));
  dd r = dd_add(a, dd_neg(xx));
  double corr = r.hi / (2.0 * x);
  return two_sum(x, corr);
}

/* a double-double mantissa with a binary exponent (value = m 2^e, |m.hi| in [0.5, 1)), so that
 * factorials up to ORC_MAX_FACT and products of six of them stay representable; scaling by powers
 * of two is exact, so the digits are those of plain double-double arithmetic */
typedef struct
{
  dd m;
  int e;
} xd;

static inline xd xd_norm(dd m, int e)
{
  xd r;
  if (m.hi == 0.0)
    {
      r.m = dd_from(0.0);
      r.e = 0;
      return r;
    }
  int k;
  frexp(m.hi, &k);
  r.m.hi = ldexp(m.hi, -k);
  r.m.lo = ldexp(m.lo, -k);
  r.e = e + k;
  return r;
}
static inline xd xd_from(double a)
{
  return xd_norm(dd_from(a), 0);
}
static inline xd xd_mul(xd a, xd b)
{
  return xd_norm(dd_mul(a.m, b.m), a.e + b.e);
}
static inline xd xd_div(xd a, xd b)
{
  return xd_norm(dd_div(a.m, b.m), a.e - b.e);
}
static inline xd xd_add(xd a, xd b)
{
  if (a.m.hi == 0.0)
    return b;
  if (b.m.hi == 0.0)
    return a;
  if (a.e < b.e)
    {
      xd t = a;
      a = b;
      b = t;
    }
  int d = a.e - b.e;
  if (d > 240)
    return a;
  dd bs = {ldexp(b.m.hi, -d), ldexp(b.m.lo, -d)};
  return xd_norm(dd_add(a.m, bs), a.e);
}
static inline xd xd_sqrt(xd a)
{
  if (a.m.hi <= 0.0)
    return xd_from(0.0);
  if (a.e & 1)
    {
      a.m = dd_mul(a.m, dd_from(2.0));
      a.e -= 1;
    }
  return xd_norm(dd_sqrt(a.m), a.e / 2);
}

#define ORC_MAX_FACT 600
static xd fact_table[ORC_MAX_FACT + 1];
static int fact_ready = 0;

static void init_factorials(void)
{
  if (fact_ready)
    return;
  fact_table[0] = xd_from(1.0);
  for (int n = 1; n <= ORC_MAX_FACT; ++n)
    fact_table[n] = xd_mul(fact_table[n - 1], xd_from((double) n));
  fact_ready = 1;
}

/* <j1/2 m1/2 ; j2/2 m2/2 | j/2 (m1+m2)/2> with every argument doubled (Condon-Shortley phase) */
double orc_clebsch_gordan(int j1, int m1, int j2, int m2, int j)
{
  init_factorials();
  int m = m1 + m2;
  if (abs(m1) > j1 || abs(m2) > j2 || abs(m) > j)
    return 0.0;
  if (((j1 + m1) & 1) || ((j2 + m2) & 1) || ((j + m) & 1) || ((j1 + j2 + j) & 1))
    return 0.0;
  if (j < abs(j1 - j2) || j > j1 + j2)
    return 0.0;
  int a = (j1 + j2 - j) / 2, b = (j1 - j2 + j) / 2, c = (-j1 + j2 + j) / 2, d = (j1 + j2 + j) / 2 + 1;
  int jm1 = (j1 - m1) / 2, jp1 = (j1 + m1) / 2, jm2 = (j2 - m2) / 2, jp2 = (j2 + m2) / 2;
  int Jm = (j - m) / 2, Jp = (j + m) / 2;
  if (d > ORC_MAX_FACT)
    return NAN;
  xd pre = xd_mul(xd_from((double) (j + 1)), xd_mul(fact_table[a], xd_mul(fact_table[b], fact_table[c])));
  pre = xd_div(pre, fact_table[d]);
  xd pre2 = xd_mul(xd_mul(fact_table[Jp], fact_table[Jm]),
                   xd_mul(xd_mul(fact_table[jm1], fact_table[jp1]), xd_mul(fact_table[jm2], fact_table[jp2])));
  xd sum = xd_from(0.0);
  /* k runs over all values keeping every factorial argument non-negative */
  int e1 = (j - j2 + m1) / 2; /* J - j2 + m1 */
  int e2 = (j - j1 - m2) / 2; /* J - j1 - m2 */
  int kmin = 0;
  if (-e1 > kmin)
    kmin = -e1;
  if (-e2 > kmin)
    kmin = -e2;
  int kmax = a;
  if (jm1 < kmax)
    kmax = jm1;
  if (jp2 < kmax)
    kmax = jp2;
  /* the first term with its exponent, then every term relative to it through the ratio of
   * consecutive terms, -(a-k)(jm1-k)(jp2-k) / ((k+1)(e1+k+1)(e2+k+1)), integers below 2^53 */
  xd den0 = xd_mul(xd_mul(fact_table[kmin], fact_table[a - kmin]),
                   xd_mul(xd_mul(fact_table[jm1 - kmin], fact_table[jp2 - kmin]),
                          xd_mul(fact_table[e1 + kmin], fact_table[e2 + kmin])));
  xd first = xd_div(xd_from((kmin & 1) ? -1.0 : 1.0), den0);
  dd term = dd_from(1.0), rel = dd_from(1.0);
  int scale = 0; /* rel and term are held times 2^-scale */
  for (int k = kmin; k < kmax; ++k)
    {
      double num = (double) (a - k) * (double) (jm1 - k) * (double) (jp2 - k);
      double dnm = (double) (k + 1) * (double) (e1 + k + 1) * (double) (e2 + k + 1);
      term = dd_div(dd_mul(term, dd_from(-num)), dd_from(dnm));
      rel = dd_add(rel, term);
      if (fabs(term.hi) > 0x1p400)
        {
          term.hi = ldexp(term.hi, -400);
          term.lo = ldexp(term.lo, -400);
          rel.hi = ldexp(rel.hi, -400);
          rel.lo = ldexp(rel.lo, -400);
          scale += 400;
        }
    }
  sum = xd_mul(first, xd_norm(rel, scale));
  xd r = xd_mul(xd_sqrt(xd_mul(pre, pre2)), sum);
  return ldexp(r.m.hi, r.e) + ldexp(r.m.lo, r.e);
}

/* ===================================================================== */
/* interaction factors, ParticleOnSphereGenericHamiltonian.cc:493-612    */
/* ===================================================================== */

int orc_nbr_pairs(int lz_max)
{
  return (lz_max + 1) * lz_max / 2;
}

/* pair order: m1 ascending, m2 < m1 ascending; per pair the m3 values (2 m3 > m1 + m2, m4 = m1 + m2 - m3
 * a valid orbital) ascending.  Returns the number of factors.  m3_offset[p] = first factor of pair p. */
static int interaction_core(int lz_max, const double* v, int* m1v, int* m2v, int* nbr_m3, int* m3_offset,
                            int* m3v, double* factors, double* dfactors)
{
  int nlz = lz_max + 1;
  int sign = (lz_max & 1) ? 0 : 1; /* keeps odd relative angular momentum only (fermions) */
  int pair = 0, nf = 0;
  /* <S m_a; S m_b | J/2 (m_a + m_b)/2> of the pairs, evaluated once each: cache[(a nlz + b) nlz + J/2]
   * with NaN for "not yet" */
  size_t ncache = (size_t) nlz * nlz * nlz;
  double* cache = (double*) malloc(sizeof(double) * ncache);
  for (size_t i = 0; i < ncache; ++i)
    cache[i] = NAN;
#define PAIR_CG(ia, ib, J)                                                                             \
  (isnan(cache[((size_t) (ia) * nlz + (ib)) * nlz + (J) / 2])                                          \
       ? (cache[((size_t) (ia) * nlz + (ib)) * nlz + (J) / 2] =                                        \
              orc_clebsch_gordan(lz_max, 2 * (ia) - lz_max, lz_max, 2 * (ib) - lz_max, (J)))          \
       : cache[((size_t) (ia) * nlz + (ib)) * nlz + (J) / 2])
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 < m1; ++m2)
      {
        int lim = m1 + m2 > lz_max ? lz_max : m1 + m2;
        int mn = m1 + m2 - lz_max < 0 ? 0 : m1 + m2 - lz_max;
        if (m1v)
          {
            m1v[pair] = m1;
            m2v[pair] = m2;
            m3_offset[pair] = nf;
          }
        int cnt = 0;
        int d1 = 2 * m1 - lz_max, d2 = 2 * m2 - lz_max;
        for (int m3 = mn; m3 <= lim; ++m3)
          {
            if (2 * m3 <= m1 + m2)
              continue;
            int m4 = m1 + m2 - m3;
            if (m3v)
              m3v[nf] = m3;
            int jmin = abs(d1 + d2);
            double acc = 0.0;
            for (int J = jmin; J <= 2 * lz_max; J += 2)
              {
                if (((J >> 1) & 1) != sign)
                  continue;
                double c12 = PAIR_CG(m1, m2, J);
                double c34 = PAIR_CG(m3, m4, J);
                int mrel = lz_max - (J >> 1);
                if (v)
                  acc += v[mrel] * c12 * c34;
                if (dfactors)
                  dfactors[(long) nf * nlz + mrel] += -4.0 * c12 * c34;
              }
            if (factors)
              factors[nf] = -4.0 * acc;
            ++nf;
            ++cnt;
          }
        if (nbr_m3)
          nbr_m3[pair] = cnt;
        ++pair;
      }
#undef PAIR_CG
  free(cache);
  return nf;
}

int orc_interaction_tables(int lz_max, const double* pseudopotentials, int* m1v, int* m2v, int* nbr_m3,
                           int* m3_offset, int* m3v, double* factors)
{
  return interaction_core(lz_max, pseudopotentials, m1v, m2v, nbr_m3, m3_offset, m3v, factors, NULL);
}

/* d factor_f / d V_m, row-major [factor][m]; the factors are linear in V */
int orc_interaction_derivatives(int lz_max, double* dfactors)
{
  int nf = interaction_core(lz_max, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL);
  memset(dfactors, 0, sizeof(double) * (size_t) nf * (lz_max + 1));
  return interaction_core(lz_max, NULL, NULL, NULL, NULL, NULL, NULL, NULL, dfactors);
}

/* EvaluatePseudopotentials(nbrFlux, landauLevel = 0, layerSeparation = 0), PseudoPotentials.cc:35-85:
 * lowest-Landau-level Coulomb pseudopotentials V_0..V_nbrFlux on the sphere */
void orc_coulomb_pseudopotentials(int nbr_flux, double* v)
{
  int mm = nbr_flux;
  int n = mm + 1;
  /* main[l][i] = <S m ; S -m | l 0>, m = 2i - mm (doubled) */
  double* cg_main = (double*) malloc(sizeof(double) * n * n);
  /* cg_j[j][i1][i2] = <S m1 ; j (m2 - m1) | S m2> */
  double* cg_j = (double*) malloc(sizeof(double) * n * n * n);
  double* cg_top = (double*) malloc(sizeof(double) * n);
  for (int l = 0; l < n; ++l)
    for (int i = 0; i < n; ++i)
      {
        int m = 2 * i - mm;
        cg_main[l * n + i] = orc_clebsch_gordan(mm, m, mm, -m, 2 * l);
      }
  for (int j = 0; j < n; ++j)
    {
      cg_top[j] = orc_clebsch_gordan(mm, mm, 2 * j, 0, mm);
      for (int i1 = 0; i1 < n; ++i1)
        for (int i2 = 0; i2 < n; ++i2)
          {
            int m1 = 2 * i1 - mm, m2 = 2 * i2 - mm;
            cg_j[((long) j * n + i1) * n + i2] = orc_clebsch_gordan(mm, m1, 2 * j, m2 - m1, mm);
          }
    }
  for (int l = 0; l < n; ++l)
    {
      double total = 0.0;
      for (int i1 = 0; i1 < n; ++i1)
        for (int i2 = 0; i2 < n; ++i2)
          {
            int m1 = 2 * i1 - mm, m2 = 2 * i2 - mm;
            int jmin = abs(m1 - m2) >> 1;
            double acc = 0.0, sgn = 1.0;
            for (int j = jmin; j <= mm; ++j)
              {
                double t = cg_j[((long) j * n + i1) * n + i2] * cg_top[j];
                acc += sgn * t * t;
                sgn = -sgn;
              }
            total += cg_main[l * n + i1] * cg_main[l * n + i2] * acc;
          }
      v[mm - l] = total / sqrt(0.5 * nbr_flux);
    }
  free(cg_main);
  free(cg_j);
  free(cg_top);
}

/* ===================================================================== */
/* matvec                                                                 */
/* ===================================================================== */

static long fqhe_index(const orc_fqhe_t* h, uint64_t w)
{
  int l = w ? 63 - __builtin_clzll(w) : 0;
  return orc_fermion_find_state_index(h->words, h->dim, h->table, h->table_shift, h->max_shift, w, l);
}

/* AbstractQHEOnSphereHamiltonian::LowLevelAddMultiply, on-the-fly branch with NbrM12Indices != 0
 * (:456-488): push form, dst[target] += AA * x[i] * factor * AdAd, then dst[i] += shift * x[i] */
void orc_fqhe_push_add_multiply(const orc_fqhe_t* h, const double* x, double* y, long first, long nbr)
{
  long last = first + nbr;
  for (long i = first; i < last; ++i)
    {
      uint64_t s = h->words[i];
      for (int p = 0; p < h->nbr_pairs; ++p)
        {
          uint64_t a;
          double c = orc_fermion_aa(s, h->m1v[p], h->m2v[p], &a);
          if (c == 0.0)
            continue;
          c *= x[i];
          int sum = h->m1v[p] + h->m2v[p];
          for (int q = 0; q < h->nbr_m3[p]; ++q)
            {
              int m3 = h->m3v[h->m3_offset[p] + q];
              uint64_t t;
              double c2 = orc_fermion_adad(a, m3, sum - m3, &t);
              if (c2 == 0.0)
                continue;
              long idx = fqhe_index(h, t);
              y[idx] += c * h->factors[h->m3_offset[p] + q] * c2;
            }
        }
    }
  for (long i = first; i < last; ++i)
    y[i] += h->shift * x[i];
}

/* pull form of the same product (H is real symmetric): y[i] = shift x[i] + sum_moves h(i->t) x[t] */
void orc_fqhe_pull_multiply(const orc_fqhe_t* h, const double* x, double* y)
{
  for (long i = 0; i < h->dim; ++i)
    {
      uint64_t s = h->words[i];
      double acc = 0.0;
      for (int p = 0; p < h->nbr_pairs; ++p)
        {
          uint64_t a;
          double c = orc_fermion_aa(s, h->m1v[p], h->m2v[p], &a);
          if (c == 0.0)
            continue;
          int sum = h->m1v[p] + h->m2v[p];
          for (int q = 0; q < h->nbr_m3[p]; ++q)
            {
              int m3 = h->m3v[h->m3_offset[p] + q];
              uint64_t t;
              double c2 = orc_fermion_adad(a, m3, sum - m3, &t);
              if (c2 == 0.0)
                continue;
              acc += c * c2 * h->factors[h->m3_offset[p] + q] * x[fqhe_index(h, t)];
            }
        }
      y[i] = acc + h->shift * x[i];
    }
}

/* one (target, sign, factor index) triple per generated element of row, in reference order */
long orc_fqhe_row_elements(const orc_fqhe_t* h, long row, int* target, int* sign, int* factor_index, long cap)
{
  uint64_t s = h->words[row];
  long n = 0;
  for (int p = 0; p < h->nbr_pairs; ++p)
    {
      uint64_t a;
      double c = orc_fermion_aa(s, h->m1v[p], h->m2v[p], &a);
      if (c == 0.0)
        continue;
      int sum = h->m1v[p] + h->m2v[p];
      for (int q = 0; q < h->nbr_m3[p]; ++q)
        {
          int m3 = h->m3v[h->m3_offset[p] + q];
          uint64_t t;
          double c2 = orc_fermion_adad(a, m3, sum - m3, &t);
          if (c2 == 0.0)
            continue;
          if (n < cap)
            {
              target[n] = (int) fqhe_index(h, t);
              sign[n] = (c * c2 > 0.0) ? 1 : -1;
              factor_index[n] = h->m3_offset[p] + q;
            }
          ++n;
        }
    }
  return n;
}

/* bins[f] = sum over rows i and elements (i -> t) of factor f of u[i] * sign * v[t]; contracting
 * with d factor / d V_m gives <u|dH/dV_m|v> (the pseudopotentials enter H linearly) */
void orc_fqhe_expectation_bins(const orc_fqhe_t* h, const double* u, const double* v, double* bins)
{
  for (long i = 0; i < h->dim; ++i)
    {
      uint64_t s = h->words[i];
      for (int p = 0; p < h->nbr_pairs; ++p)
        {
          uint64_t a;
          double c = orc_fermion_aa(s, h->m1v[p], h->m2v[p], &a);
          if (c == 0.0)
            continue;
          int sum = h->m1v[p] + h->m2v[p];
          for (int q = 0; q < h->nbr_m3[p]; ++q)
            {
              int m3 = h->m3v[h->m3_offset[p] + q];
              uint64_t t;
              double c2 = orc_fermion_adad(a, m3, sum - m3, &t);
              if (c2 == 0.0)
                continue;
              bins[h->m3_offset[p] + q] += u[i] * c * c2 * v[fqhe_index(h, t)];
            }
        }
    }
}

void orc_fqhe_matvec_cb(void* ctx, const double* x, double* y)
{
  orc_fqhe_pull_multiply((const orc_fqhe_t*) ctx, x, y);
}

/* ===================================================================== */
/* spin-1/2 chain                                                         */
/* ===================================================================== */

static long binom(int n, int k)
{
  if (k < 0 || k > n)
    return 0;
  long r = 1;
  for (int i = 1; i <= k; ++i)
    r = r * (n - k + i) / i;
  return r;
}

/* Spin1_2Chain::EvaluateHilbertSpaceDimension: C(L, nbr up), sz = 2 Sz = 2 nbr_up - L */
long orc_spin_dimension(int length, int sz)
{
  if (((length + sz) & 1) || abs(sz) > length)
    return 0;
  return binom(length, (length + sz) / 2);
}

typedef struct
{
  int length;
  uint64_t high; /* bits length..31 stay set, as in Spin1_2Chain.cc:137-138 */
  uint64_t* words;
  long pos;
} spin_gen;

/* Spin1_2Chain::GenerateStates, Spin1_2Chain.cc:331-394: site 0 first, spin up (bit set) before
 * spin down, so the basis is sorted in descending order of the bit-reversed word */
static void gen_spin(spin_gen* c, int site, int ups, uint64_t bits)
{
  int left = c->length - site;
  if (ups < 0 || ups > left)
    return;
  if (site == c->length)
    {
      if (c->words)
        c->words[c->pos] = bits | c->high;
      c->pos++;
      return;
    }
  gen_spin(c, site + 1, ups - 1, bits | (1ull << site));
  gen_spin(c, site + 1, ups, bits);
}

long orc_spin_basis(int length, int sz, uint64_t* words)
{
  if (((length + sz) & 1) || abs(sz) > length)
    return 0;
  spin_gen c;
  c.length = length;
  c.high = (length < 32) ? (0xffffffffull & ~((1ull << length) - 1)) : 0;
  c.words = words;
  c.pos = 0;
  gen_spin(&c, 0, (length + sz) / 2, 0);
  return c.pos;
}

/* index of a word in that order: count the basis states that sort before it.  Walking sites
 * 0..L-1, every site where the word has spin down while a spin up would still fit contributes the
 * number of completions with that site up. */
long orc_spin_find_state_index(int length, int sz, uint64_t word)
{
  int ups = (length + sz) / 2;
  long idx = 0;
  for (int site = 0; site < length && ups > 0; ++site)
    {
      if ((word >> site) & 1)
        --ups;
      else
        idx += binom(length - site - 1, ups - 1);
    }
  return idx;
}

/* J1-J2 periodic chain: pattern of SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192 (flips
 * with J/2) and :335-352 (diagonal J Sz_i Sz_j), applied on a plain Spin1_2Chain through the API
 * model of SpinChainHamiltonian.cc:257-298; pull form */
void orc_spin_j1j2_multiply(int length, int sz, const uint64_t* words, long dim, double j1, double j2,
                            double shift, const double* x, double* y)
{
  for (long i = 0; i < dim; ++i)
    {
      uint64_t w = words[i];
      double diag = 0.0, acc = 0.0;
      for (int j = 0; j < length; ++j)
        {
          int nb[2] = {(j + 1) % length, (j + 2) % length};
          double jj[2] = {j1, j2};
          for (int b = 0; b < 2; ++b)
            {
              int k = nb[b];
              int bj = (w >> j) & 1, bk = (w >> k) & 1;
              diag += jj[b] * ((bj == bk) ? 0.25 : -0.25);
              if (bj != bk)
                {
                  uint64_t t = w ^ ((1ull << j) | (1ull << k));
                  acc += 0.5 * jj[b] * x[orc_spin_find_state_index(length, sz, t)];
                }
            }
        }
      y[i] = (diag + shift) * x[i] + acc;
    }
}

/* ===================================================================== */
/* deterministic start vectors                                            */
/* ===================================================================== */

/* component i is the (i+1)-th output of splitmix64 seeded with seed, mapped to [-1, 1), then the
 * whole vector is normalised */
void orc_random_vector(uint64_t seed, long dim, double* x)
{
  double norm = 0.0;
  for (long i = 0; i < dim; ++i)
    {
      uint64_t z = seed + (uint64_t) (i + 1) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z = z ^ (z >> 31);
      x[i] = (double) (z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
      norm += x[i] * x[i];
    }
  norm = sqrt(norm);
  for (long i = 0; i < dim; ++i)
    x[i] /= norm;
}

/* ===================================================================== */
/* Lanczos                                                                */
/* ===================================================================== */

/* eigenvalues of the symmetric tridiagonal matrix (diag[0..n-1], off[0..n-2]) by implicit-shift QL
 * iterations with Wilkinson shifts, sorted ascending (the role of
 * RealTriDiagonalSymmetricMatrix::Diagonalize + SortMatrixUpOrder, RealTriDiagonalSymmetricMatrix.cc:687,1611) */
static int cmp_double(const void* a, const void* b)
{
  double x = *(const double*) a, y = *(const double*) b;
  return (x < y) ? -1 : (x > y);
}

int orc_tridiagonal_eigenvalues(int n, const double* diag, const double* off, double* eig)
{
  double* d = eig;
  double* e = (double*) calloc((size_t) n + 1, sizeof(double));
  for (int i = 0; i < n; ++i)
    d[i] = diag[i];
  for (int i = 0; i + 1 < n; ++i)
    e[i] = off[i];
  for (int l = 0; l < n; ++l)
    {
      int iter = 0;
      for (;;)
        {
          int m;
          for (m = l; m + 1 < n; ++m)
            {
              double dd2 = fabs(d[m]) + fabs(d[m + 1]);
              if (fabs(e[m]) <= 1e-300 || fabs(e[m]) <= 2.220446049250313e-16 * dd2)
                break;
            }
          if (m == l)
            break;
          if (++iter > 200)
            {
              free(e);
              return -1;
            }
          /* Wilkinson shift from the leading 2x2 block */
          double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
          double r = hypot(g, 1.0);
          g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
          double s = 1.0, c = 1.0, p = 0.0;
          int i;
          for (i = m - 1; i >= l; --i)
            {
              double f = s * e[i], b = c * e[i];
              r = hypot(f, g);
              e[i + 1] = r;
              if (r == 0.0)
                {
                  d[i + 1] -= p;
                  e[m] = 0.0;
                  break;
                }
              s = f / r;
              c = g / r;
              g = d[i + 1] - p;
              r = (d[i] - g) * s + 2.0 * c * b;
              p = s * r;
              d[i + 1] = g + p;
              g = c * r - b;
            }
          if (r == 0.0 && i >= l)
            continue;
          d[l] -= p;
          e[l] = g;
          e[m] = 0.0;
        }
    }
  free(e);
  qsort(eig, (size_t) n, sizeof(double), cmp_double);
  return 0;
}

/* cyclic Jacobi eigen-decomposition of a dense symmetric n x n matrix (row-major, destroyed);
 * eigenvalues ascending, eigenvectors as columns of vecs (may be NULL) */
int orc_symmetric_eigen(int n, double* a, double* eig, double* vecs)
{
  double* v = vecs ? vecs : (double*) malloc(sizeof(double) * (size_t) n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      v[i * n + j] = (i == j);
  for (int sweep = 0; sweep < 100; ++sweep)
    {
      double off = 0.0;
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
          off += a[i * n + j] * a[i * n + j];
      if (off < 1e-300)
        break;
      for (int p = 0; p < n; ++p)
        for (int q = p + 1; q < n; ++q)
          {
            double apq = a[p * n + q];
            if (fabs(apq) < 1e-300)
              continue;
            double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
            for (int k = 0; k < n; ++k)
              {
                double akp = a[k * n + p], akq = a[k * n + q];
                a[k * n + p] = c * akp - s * akq;
                a[k * n + q] = s * akp + c * akq;
              }
            for (int k = 0; k < n; ++k)
              {
                double apk = a[p * n + k], aqk = a[q * n + k];
                a[p * n + k] = c * apk - s * aqk;
                a[q * n + k] = s * apk + c * aqk;
              }
            for (int k = 0; k < n; ++k)
              {
                double vkp = v[k * n + p], vkq = v[k * n + q];
                v[k * n + p] = c * vkp - s * vkq;
                v[k * n + q] = s * vkp + c * vkq;
              }
          }
    }
  /* sort ascending, permuting eigenvector columns */
  for (int i = 0; i < n; ++i)
    eig[i] = a[i * n + i];
  for (int i = 0; i < n; ++i)
    {
      int k = i;
      for (int j = i + 1; j < n; ++j)
        if (eig[j] < eig[k])
          k = j;
      if (k != i)
        {
          double t = eig[i];
          eig[i] = eig[k];
          eig[k] = t;
          for (int r = 0; r < n; ++r)
            {
              double x = v[r * n + i];
              v[r * n + i] = v[r * n + k];
              v[r * n + k] = x;
            }
        }
    }
  if (!vecs)
    free(v);
  return 0;
}

static double dot(long n, const double* a, const double* b)
{
  double s = 0.0;
  for (long i = 0; i < n; ++i)
    s += a[i] * b[i];
  return s;
}

/* BasicLanczosAlgorithm::RunLanczosAlgorithm (BasicLanczosAlgorithm.cc:148-216) driven by the loop
 * of QHEOnSphereMainTask.cc:732-753: first call with nev + 2 steps, then one step per call until
 * BasicLanczosAlgorithm::TestConvergence (:220) holds or max_iter is reached.  The recurrence takes
 * alpha_i = <v_i|H v_i> and beta_i = <v_{i-1}|H v_i> exactly as the reference does.
 * Returns 1 if converged. */
int orc_basic_lanczos(orc_matvec_fn mv, void* ctx, long dim, const double* v0, int nev, int max_iter,
                      double precision, double* eigenvalues, int* iterations, double* alpha, double* beta)
{
  double* v1 = (double*) malloc(sizeof(double) * dim);
  double* v2 = (double*) malloc(sizeof(double) * dim);
  double* v3 = (double*) malloc(sizeof(double) * dim);
  double* eig = (double*) malloc(sizeof(double) * (size_t) (max_iter + 4));
  memcpy(v1, v0, sizeof(double) * dim);
  int n = 0; /* rows of the tridiagonal matrix */
  double prev = 0.0;
  int steps = nev + 2;
  if (steps < 2)
    steps = 2;
  /* first two vectors (:152-166) */
  mv(ctx, v1, v2);
  alpha[0] = dot(dim, v1, v2);
  for (long i = 0; i < dim; ++i)
    v2[i] -= alpha[0] * v1[i];
  double nrm = sqrt(dot(dim, v2, v2));
  for (long i = 0; i < dim; ++i)
    v2[i] /= nrm;
  mv(ctx, v2, v3);
  beta[0] = dot(dim, v1, v3);
  alpha[1] = dot(dim, v2, v3);
  n = 2;
  int count = nev + 3; /* iteration counter of the driver loop */
  int converged = 0;
  int target_rows = steps;
  for (;;)
    {
      while (n < target_rows)
        {
          for (long i = 0; i < dim; ++i)
            v3[i] -= beta[n - 2] * v1[i] + alpha[n - 1] * v2[i];
          nrm = sqrt(dot(dim, v3, v3));
          for (long i = 0; i < dim; ++i)
            v3[i] /= nrm;
          double* t = v1;
          v1 = v2;
          v2 = v3;
          v3 = t;
          mv(ctx, v2, v3);
          beta[n - 1] = dot(dim, v1, v3);
          alpha[n] = dot(dim, v2, v3);
          ++n;
        }
      /* :200-214: a stored previous value of zero means "first call" */
      if (prev != 0.0)
        {
          prev = eig[nev - 1];
          orc_tridiagonal_eigenvalues(n, alpha, beta, eig);
        }
      else
        {
          orc_tridiagonal_eigenvalues(n, alpha, beta, eig);
          prev = 2.0 * eig[nev - 1];
        }
      converged = fabs(eig[nev - 1] - prev) < precision * fabs(eig[nev - 1]);
      if (converged || count >= max_iter)
        break;
      ++count;
      target_rows = n + 1;
    }
  for (int i = 0; i < nev; ++i)
    eigenvalues[i] = eig[i];
  *iterations = count;
  free(v1);
  free(v2);
  free(v3);
  free(eig);
  return converged;
}

/* ===================================================================== */
/* bosons: BosonOnSphereShort (FQHE/src/HilbertSpace/BosonOnSphereShort) */
/* ===================================================================== */

/* FermionToBoson / BosonToFermion (BosonOnSphereShort.h:1231-1290): occupations n_0..n_lzmax <->
 * the fermionic word with, from bit 0 up, n_0 ones, a zero, n_1 ones, a zero, ... */
void orc_boson_unpack(uint64_t w, int lz_max, int* n)
{
  for (int m = 0; m <= lz_max; ++m)
    {
      int c = 0;
      while (w & 1ull)
        {
          ++c;
          w >>= 1;
        }
      n[m] = c;
      w >>= 1;
    }
}

uint64_t orc_boson_pack(const int* n, int lz_max)
{
  uint64_t w = 0;
  int shift = 0;
  for (int m = 0; m <= lz_max; ++m)
    {
      w |= ((1ull << n[m]) - 1ull) << shift;
      shift += n[m] + 1;
    }
  return w;
}

/* AA (BosonOnSphereShort.cc:353-375): annihilate n2 then n1 on a copy of the occupations, coefficient
 * sqrt(n_n2 (n_n1 after the first)); 0 when either orbital is empty */
double orc_boson_aa(const int* occ, int lz_max, int n1, int n2, int* out)
{
  for (int m = 0; m <= lz_max; ++m)
    out[m] = occ[m];
  if (out[n2] == 0)
    return 0.0;
  double c = out[n2];
  --out[n2];
  if (out[n1] == 0)
    return 0.0;
  c *= out[n1];
  --out[n1];
  return sqrt(c);
}

/* AdAd (BosonOnSphereShort.cc:431-451): create m2 then m1, coefficient sqrt((n_m2 + 1)(n_m1 + 1 after)) */
double orc_boson_adad(const int* occ, int lz_max, int m1, int m2, uint64_t* out)
{
  int t[64];
  for (int m = 0; m <= lz_max; ++m)
    t[m] = occ[m];
  ++t[m2];
  double c = t[m2];
  ++t[m1];
  c *= t[m1];
  *out = orc_boson_pack(t, lz_max);
  return sqrt(c);
}

int orc_boson_nbr_pairs(int lz_max)
{
  return (lz_max + 1) * (lz_max + 2) / 2;
}

/* the bosonic branch of ParticleOnSphereGenericHamiltonian::EvaluateInteractionFactors (:620-806):
 * pairs m1 ascending, m2 = 0..m1 (m2 = m1 last); per pair the m3 with 2 m3 >= m1 + m2 and m4 a valid
 * orbital, ascending; factor = w sum_J V CG(m1 m2; J) CG(m3 m4; J) over the J with (J / 2) of the
 * parity opposite to the fermionic one, w = 4, halved for m1 = m2 and again for m3 = m4 */
int orc_boson_interaction_tables(int lz_max, const double* v, int* m1v, int* m2v, int* nbr_m3, int* m3_offset,
                                 int* m3v, double* factors)
{
  int nlz = lz_max + 1;
  int sign = (lz_max & 1) ? 0 : 1;
  int pair = 0, nf = 0;
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 <= m1; ++m2)
      {
        int lim = m1 + m2 > lz_max ? lz_max : m1 + m2;
        int mn = m1 + m2 - lz_max < 0 ? 0 : m1 + m2 - lz_max;
        if (m1v)
          {
            m1v[pair] = m1;
            m2v[pair] = m2;
            m3_offset[pair] = nf;
          }
        int cnt = 0;
        int d1 = 2 * m1 - lz_max, d2 = 2 * m2 - lz_max;
        for (int m3 = mn; m3 <= lim; ++m3)
          {
            if (2 * m3 < m1 + m2)
              continue;
            int m4 = m1 + m2 - m3;
            int d3 = 2 * m3 - lz_max, d4 = 2 * m4 - lz_max;
            if (m3v)
              m3v[nf] = m3;
            double acc = 0.0;
            for (int J = abs(d1 + d2); J <= 2 * lz_max; J += 2)
              {
                if (((J >> 1) & 1) == sign)
                  continue;
                acc += v[lz_max - (J >> 1)] * orc_clebsch_gordan(lz_max, d1, lz_max, d2, J) *
                       orc_clebsch_gordan(lz_max, d3, lz_max, d4, J);
              }
            double w = 4.0;
            if (m1 == m2)
              w *= 0.5;
            if (m3 == m4)
              w *= 0.5;
            if (factors)
              factors[nf] = w * acc;
            ++nf;
            ++cnt;
          }
        if (nbr_m3)
          nbr_m3[pair] = cnt;
        ++pair;
      }
  return nf;
}

/* the boson product through the same on-the-fly loop (AbstractQHEOnSphereHamiltonian.cc:456-488,
 * push form; and its pull form, H being real symmetric); h holds the fermionic words of the
 * BosonOnSphereShort basis (h->lz_max = lz_max + N - 1) and the bosonic tables */
void orc_boson_push_add_multiply(const orc_fqhe_t* h, const double* x, double* y, long first, long nbr)
{
  int lz_max = h->lz_max - h->nbr_fermions + 1;
  int occ[64], a[64];
  for (long i = first; i < first + nbr; ++i)
    {
      orc_boson_unpack(h->words[i], lz_max, occ);
      for (int p = 0; p < h->nbr_pairs; ++p)
        {
          double c = orc_boson_aa(occ, lz_max, h->m1v[p], h->m2v[p], a);
          if (c == 0.0)
            continue;
          c *= x[i];
          int sum = h->m1v[p] + h->m2v[p];
          for (int q = 0; q < h->nbr_m3[p]; ++q)
            {
              int m3 = h->m3v[h->m3_offset[p] + q];
              uint64_t t;
              double c2 = orc_boson_adad(a, lz_max, m3, sum - m3, &t);
              y[fqhe_index(h, t)] += c * h->factors[h->m3_offset[p] + q] * c2;
            }
        }
    }
  for (long i = first; i < first + nbr; ++i)
    y[i] += h->shift * x[i];
}

void orc_boson_pull_multiply(const orc_fqhe_t* h, const double* x, double* y)
{
  int lz_max = h->lz_max - h->nbr_fermions + 1;
  int occ[64], a[64];
  for (long i = 0; i < h->dim; ++i)
    {
      orc_boson_unpack(h->words[i], lz_max, occ);
      double acc = 0.0;
      for (int p = 0; p < h->nbr_pairs; ++p)
        {
          double c = orc_boson_aa(occ, lz_max, h->m1v[p], h->m2v[p], a);
          if (c == 0.0)
            continue;
          int sum = h->m1v[p] + h->m2v[p];
          for (int q = 0; q < h->nbr_m3[p]; ++q)
            {
              int m3 = h->m3v[h->m3_offset[p] + q];
              uint64_t t;
              double c2 = orc_boson_adad(a, lz_max, m3, sum - m3, &t);
              acc += c * c2 * h->factors[h->m3_offset[p] + q] * x[fqhe_index(h, t)];
            }
        }
      y[i] = acc + h->shift * x[i];
    }
}

void orc_boson_matvec_cb(void* ctx, const double* x, double* y)
{
  orc_boson_pull_multiply((const orc_fqhe_t*) ctx, x, y);
}

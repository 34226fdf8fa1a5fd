// Host-side set-up maths of the engine: Clebsch-Gordan coefficients, Coulomb pseudopotentials,
// the interaction-factor tables of ParticleOnSphereGenericHamiltonian, and the small FP64
// eigensolvers used on the Lanczos tridiagonal / band matrices.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <limits>
#include <cmath>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "dh_internal.h"

namespace dh {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
  return e == cudaErrorMemoryAllocation ? DH_ERR_MEMORY : DH_ERR_CUDA;
}

int DevBuf::alloc(size_t n) {
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  bytes = n;
  return DH_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

// ---------------------------------------------- double-double arithmetic
// Two doubles hi + lo carry ~32 significant digits; Racah's alternating sum for the
// Clebsch-Gordan coefficients cancels up to ~10 digits at 2S = 33, so it is summed in this format.
namespace {
struct DD {
  double hi, lo;
};
inline DD dd(double a) { return {a, 0.0}; }
inline DD quick_two_sum(double a, double b) {
  double s = a + b;
  return {s, b - (s - a)};
}
inline DD two_sum(double a, double b) {
  double s = a + b, v = s - a;
  return {s, (a - (s - v)) + (b - v)};
}
inline DD operator+(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
inline DD operator-(DD a) { return {-a.hi, -a.lo}; }
inline DD operator*(DD a, DD b) {
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
  return quick_two_sum(p, e);
}
inline DD operator/(DD a, DD b) {
  double q1 = a.hi / b.hi;
  DD r = a + (-(dd(q1) * b));
  double q2 = r.hi / b.hi;
  r = r + (-(dd(q2) * b));
  double q3 = r.hi / b.hi;
  return quick_two_sum(q1, q2) + dd(q3);
}
inline DD dd_sqrt(DD a) {
  if (a.hi <= 0.0) return dd(0.0);
  double x = sqrt(a.hi);
  DD r = a + (-(dd(x) * dd(x)));
  return quick_two_sum(x, r.hi / (2.0 * x));
}

// A double-double mantissa with a binary exponent (value = m * 2^e, |m.hi| in [0.5, 1)): factorials
// up to kMaxFactorial and Racah's products of six of them stay representable, and because scaling by
// powers of two is exact the digits are those of plain double-double arithmetic.
struct XD {
  DD m;
  int e;
};
inline XD xnorm(DD m, int e) {
  if (m.hi == 0.0) return {dd(0.0), 0};
  int k;
  frexp(m.hi, &k);
  return {{ldexp(m.hi, -k), ldexp(m.lo, -k)}, e + k};
}
inline XD xd(double a) { return xnorm(dd(a), 0); }
inline XD operator*(XD a, XD b) { return xnorm(a.m * b.m, a.e + b.e); }
inline XD operator/(XD a, XD b) { return xnorm(a.m / b.m, a.e - b.e); }
inline XD operator-(XD a) { return {-a.m, a.e}; }
inline XD operator+(XD a, XD b) {
  if (a.m.hi == 0.0) return b;
  if (b.m.hi == 0.0) return a;
  if (a.e < b.e) std::swap(a, b);
  const int d = a.e - b.e;
  if (d > 240) return a;
  return xnorm(a.m + DD{ldexp(b.m.hi, -d), ldexp(b.m.lo, -d)}, a.e);
}
inline XD xsqrt(XD a) {
  if (a.m.hi <= 0.0) return {dd(0.0), 0};
  if (a.e & 1) {
    a.m = a.m * dd(2.0);
    a.e -= 1;
  }
  return xnorm(dd_sqrt(a.m), a.e / 2);
}
inline double xvalue(XD a) { return ldexp(a.m.hi, a.e) + ldexp(a.m.lo, a.e); }

constexpr int kMaxFactorial = 600;
const std::vector<XD>& factorials() {
  static std::vector<XD> f;
  static std::once_flag once;
  std::call_once(once, [] {
    f.resize(kMaxFactorial + 1);
    f[0] = xd(1.0);
    for (int n = 1; n <= kMaxFactorial; ++n) f[n] = f[n - 1] * xd((double)n);
  });
  return f;
}
}  // namespace

// Racah's formula for <j1 m1; j2 m2 | j m1+m2>, Condon-Shortley phase; doubled arguments.
double clebsch_gordan(int j1, int m1, int j2, int m2, int j) {
  const std::vector<XD>& F = factorials();
  int m = m1 + m2;
  if (abs(m1) > j1 || abs(m2) > j2 || abs(m) > j) return 0.0;
  if (((j1 + m1) | (j2 + m2) | (j + m) | (j1 + j2 + j)) & 1) return 0.0;
  if (j < abs(j1 - j2) || j > j1 + j2) return 0.0;
  if ((j1 + j2 + j) / 2 + 1 > kMaxFactorial) return NAN;
  const int a = (j1 + j2 - j) / 2, b = (j1 - j2 + j) / 2, c = (j2 - j1 + j) / 2, d = (j1 + j2 + j) / 2 + 1;
  const int jm1 = (j1 - m1) / 2, jp1 = (j1 + m1) / 2, jm2 = (j2 - m2) / 2, jp2 = (j2 + m2) / 2;
  const int Jm = (j - m) / 2, Jp = (j + m) / 2;
  const int e1 = (j - j2 + m1) / 2, e2 = (j - j1 - m2) / 2;
  XD norm2 = xd((double)(j + 1)) * F[a] * F[b] * F[c] / F[d];
  norm2 = norm2 * (F[Jp] * F[Jm] * F[jm1] * F[jp1] * F[jm2] * F[jp2]);
  int kmin = std::max(0, std::max(-e1, -e2));
  int kmax = std::min(a, std::min(jm1, jp2));
  // sum over k of (-1)^k / (k! (a-k)! (jm1-k)! (jp2-k)! (e1+k)! (e2+k)!): the first term with its
  // exponent, then the terms relative to it by their ratio, a ratio of integers below 2^53
  // -(a-k)(jm1-k)(jp2-k) / ((k+1)(e1+k+1)(e2+k+1)), in double-double
  XD first = xd((kmin & 1) ? -1.0 : 1.0) /
             (F[kmin] * F[a - kmin] * F[jm1 - kmin] * F[jp2 - kmin] * F[e1 + kmin] * F[e2 + kmin]);
  DD term = dd(1.0), sum = dd(1.0);
  int scale = 0;  // sum and term are held times 2^-scale
  for (int k = kmin; k < kmax; ++k) {
    const double num = (double)(a - k) * (double)(jm1 - k) * (double)(jp2 - k);
    const double den = (double)(k + 1) * (double)(e1 + k + 1) * (double)(e2 + k + 1);
    term = term * dd(-num) / dd(den);
    sum = sum + term;
    if (fabs(term.hi) > 0x1p400) {
      term = {ldexp(term.hi, -400), ldexp(term.lo, -400)};
      sum = {ldexp(sum.hi, -400), ldexp(sum.lo, -400)};
      scale += 400;
    }
  }
  return xvalue(xsqrt(norm2) * first * xnorm(sum, scale));
}

// Lowest-Landau-level Coulomb pseudopotentials on the sphere: the multipole expansion of
// PseudoPotentials.cc:35-85 (landau level 0, zero layer separation, so all form factors are 1).
void coulomb_pseudopotentials(int nbr_flux, double* v) {
  const int mm = nbr_flux, n = nbr_flux + 1;
  std::vector<double> cg_pair(n * n), cg_j((size_t)n * n * n), cg_top(n);
  for (int l = 0; l < n; ++l)
    for (int i = 0; i < n; ++i) cg_pair[l * n + i] = clebsch_gordan(mm, 2 * i - mm, mm, mm - 2 * i, 2 * l);
  for (int j = 0; j < n; ++j) {
    cg_top[j] = clebsch_gordan(mm, mm, 2 * j, 0, mm);
    for (int i1 = 0; i1 < n; ++i1)
      for (int i2 = 0; i2 < n; ++i2)
        cg_j[((size_t)j * n + i1) * n + i2] = clebsch_gordan(mm, 2 * i1 - mm, 2 * j, 2 * (i2 - i1), mm);
  }
  // inner[i1][i2] = sum_{j >= |m1 - m2|} (-1)^(j - jmin) (<S m1; j m2-m1|S m2> <S S; j 0|S S>)^2
  std::vector<double> inner((size_t)n * n);
  for (int i1 = 0; i1 < n; ++i1)
    for (int i2 = 0; i2 < n; ++i2) {
      double acc = 0.0, sgn = 1.0;
      for (int j = abs(i1 - i2); j <= mm; ++j) {
        double t = cg_j[((size_t)j * n + i1) * n + i2] * cg_top[j];
        acc += sgn * t * t;
        sgn = -sgn;
      }
      inner[(size_t)i1 * n + i2] = acc;
    }
  for (int l = 0; l < n; ++l) {
    double total = 0.0;
    for (int i1 = 0; i1 < n; ++i1)
      for (int i2 = 0; i2 < n; ++i2) total += cg_pair[l * n + i1] * cg_pair[l * n + i2] * inner[(size_t)i1 * n + i2];
    v[mm - l] = total / sqrt(0.5 * nbr_flux);
  }
}

// ------------------------------------------------------ interaction tables
// Pair (m1 > m2) order: m1 ascending, then m2 ascending (pair index m1 (m1 - 1) / 2 + m2); per pair the
// m3 with 2 m3 > m1 + m2 and m4 = m1 + m2 - m3 >= 0 ascending (m3 = floor(M / 2) + 1 .. min(M, lzmax)).
// The factor of (m1, m2, m3) is -4 sum_J V_{lzmax - J/2} <m1 m2|J> <m3 m4|J> over odd relative
// angular momentum (ParticleOnSphereGenericHamiltonian.cc:509-606); it is linear in V, so the
// table stores d factor / d V_m and the factors of any V are one contraction away.
void InteractionTables::build(int lzmax) {
  lz_max = lzmax;
  const int nlz = lzmax + 1;
  const int parity = (lzmax & 1) ? 0 : 1;
  nbr_pairs = nlz * lzmax / 2;
  pair_offset.assign(nbr_pairs + 1, 0);
  int nf = 0;
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 < m1; ++m2) {
      int p = m1 * (m1 - 1) / 2 + m2;
      pair_offset[p] = nf;
      int M = m1 + m2;
      nf += std::min(M, lzmax) - (M / 2 + 1) + 1;
    }
  pair_offset[nbr_pairs] = nf;
  nbr_factors = nf;
  dfactor.assign((size_t)nf * nlz, 0.0);
  // CG table over the pair's doubled projections: cg[(i1 * nlz + i2) * nlz + J/2], for the ordered
  // pairs i1 > i2 that the factors use (m1 > m2 and m3 > m4)
  std::vector<double> cg((size_t)nlz * nlz * nlz, 0.0);
  for (int i1 = 0; i1 < nlz; ++i1)
    for (int i2 = 0; i2 < i1; ++i2)
      for (int J = 0; J <= 2 * lzmax; J += 2)
        cg[((size_t)i1 * nlz + i2) * nlz + J / 2] = clebsch_gordan(lzmax, 2 * i1 - lzmax, lzmax, 2 * i2 - lzmax, J);
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 < m1; ++m2) {
      int M = m1 + m2;
      int f = pair_offset[m1 * (m1 - 1) / 2 + m2];
      for (int m3 = M / 2 + 1; m3 <= std::min(M, lzmax); ++m3, ++f) {
        int m4 = M - m3;
        for (int J = abs(2 * M - 2 * lzmax); J <= 2 * lzmax; J += 2) {
          if (((J >> 1) & 1) != parity) continue;
          double c12 = cg[((size_t)m1 * nlz + m2) * nlz + J / 2];
          double c34 = cg[((size_t)m3 * nlz + m4) * nlz + J / 2];
          dfactor[(size_t)f * nlz + (lzmax - J / 2)] = -4.0 * c12 * c34;
        }
      }
    }
  factors.assign(nf, 0.0);
}

void InteractionTables::build_bosons(int lzmax) {
  lz_max = lzmax;
  bosonic = true;
  const int nlz = lzmax + 1;
  // the reference keeps the pseudopotentials whose J / 2 has the parity opposite to the fermionic one
  const int parity = (lzmax & 1) ? 0 : 1;
  nbr_pairs = nlz * (nlz + 1) / 2;
  pair_offset.assign(nbr_pairs + 1, 0);
  int nf = 0;
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 <= m1; ++m2) {
      const int M = m1 + m2;
      pair_offset[m1 * (m1 + 1) / 2 + m2] = nf;
      nf += std::min(M, lzmax) - (M + 1) / 2 + 1;  // m3 = ceil(M / 2) .. min(M, lz_max)
    }
  pair_offset[nbr_pairs] = nf;
  nbr_factors = nf;
  dfactor.assign((size_t)nf * nlz, 0.0);
  std::vector<double> cg((size_t)nlz * nlz * nlz, 0.0);
  for (int i1 = 0; i1 < nlz; ++i1)
    for (int i2 = 0; i2 < nlz; ++i2)
      for (int J = 0; J <= 2 * lzmax; J += 2)
        cg[((size_t)i1 * nlz + i2) * nlz + J / 2] = clebsch_gordan(lzmax, 2 * i1 - lzmax, lzmax, 2 * i2 - lzmax, J);
  for (int m1 = 0; m1 < nlz; ++m1)
    for (int m2 = 0; m2 <= m1; ++m2) {
      const int M = m1 + m2;
      int f = pair_offset[m1 * (m1 + 1) / 2 + m2];
      for (int m3 = (M + 1) / 2; m3 <= std::min(M, lzmax); ++m3, ++f) {
        const int m4 = M - m3;
        // 4 for distinct pairs, halved for each pair of equal orbitals (the reference's weights)
        const double w = 4.0 * ((m1 == m2) ? 0.5 : 1.0) * ((m3 == m4) ? 0.5 : 1.0);
        for (int J = abs(2 * M - 2 * lzmax); J <= 2 * lzmax; J += 2) {
          if (((J >> 1) & 1) == parity) continue;
          const double c12 = cg[((size_t)m1 * nlz + m2) * nlz + J / 2];
          const double c34 = cg[((size_t)m3 * nlz + m4) * nlz + J / 2];
          dfactor[(size_t)f * nlz + (lzmax - J / 2)] = w * c12 * c34;
        }
      }
    }
  factors.assign(nf, 0.0);
}

void InteractionTables::set_pseudopotentials(const double* v) {
  const int nlz = lz_max + 1;
  // J ascending (m descending), as the reference accumulates its Clebsch-Gordan sum
  for (int f = 0; f < nbr_factors; ++f) {
    double acc = 0.0;
    for (int m = lz_max; m >= 0; --m) acc += v[m] * dfactor[(size_t)f * nlz + m];
    factors[f] = acc;
  }
  if (!l2_part.empty() && l2_factor != 0.0)
    for (int f = 0; f < nbr_factors; ++f) factors[f] += l2_factor * l2_part[f];
}

// L^2 = L-L+ + Lz^2 + Lz, the operator of ParticleOnSphereL2Hamiltonian (ParticleOnSphereL2Hamiltonian.cc:
// 240-368), written in this table's form: the element of move (m1, m2) -> (m3, m4) is
// F(m1, m2, m3) <t| a+_m3 a+_m4 a_m1 a_m2 |s>.  With L+ = sum_m lam_m a+_{m+1} a_m,
//   L-L+ = sum_m lam_m^2 n_m - sum_{m, m'} lam_m lam_m' a+_m' a+_{m+1} a_{m'+1} a_m,
// each two-body term is reordered to (m3 > m4, m1 > m2) with its fermionic sign, and the one-body
// part is folded into the diagonal pair factors: at fixed N, sum_m w_m n_m =
// sum_{a > b} (w_a + w_b) / (N - 1) n_a n_b, and a diagonal factor F contributes -F n_a n_b.
void InteractionTables::build_l2(int nbr_particles) {
  const int S2 = lz_max;
  std::vector<double> lam(S2 + 1, 0.0);
  for (int m = 0; m <= S2; ++m) lam[m] = 0.5 * sqrt((double)(S2 * (S2 + 2) - (2 * m - S2) * (2 * m - S2 + 2)));
  l2_part.assign(nbr_factors, 0.0);
  if (bosonic) {
    // Bosons commute: a_{m'+1} a+_{m+1} = a+_{m+1} a_{m'+1} + [m = m'], so
    //   L-L+ = sum_m lam_m^2 n_m + sum_{m, m'} lam_m lam_m' a+_m' a+_{m+1} a_{m'+1} a_m,
    // and every two-body term is already the table's operator a+_m3 a+_m4 a_m1 a_m2 with m1 = max(m'+1, m),
    // m2 = min(m'+1, m), m3 = max(m', m+1), no sign.  The one-body part goes into the diagonal factors:
    // at fixed N, sum_m w_m n_m = sum_{a > b} (w_a + w_b) / (N - 1) n_a n_b + sum_a w_a / (N - 1) n_a (n_a - 1),
    // and the diagonal move (a, b) -> (a, b) has the element n_a n_b (a > b) or n_a (n_a - 1) (a = b).
    auto bslot = [&](int m1, int m2, int m3) -> double& {
      const int M = m1 + m2;
      return l2_part[pair_offset[m1 * (m1 + 1) / 2 + m2] + (m3 - (M + 1) / 2)];
    };
    for (int m = 0; m < S2; ++m)
      for (int mp = 0; mp < S2; ++mp)
        bslot(std::max(mp + 1, m), std::min(mp + 1, m), std::max(mp, m + 1)) += lam[m] * lam[mp];
    for (int a = 0; a <= S2; ++a) {
      for (int b = 0; b < a; ++b) bslot(a, b, a) += (lam[a] * lam[a] + lam[b] * lam[b]) / (nbr_particles - 1);
      bslot(a, a, a) += lam[a] * lam[a] / (nbr_particles - 1);
    }
    return;
  }
  auto slot = [&](int m1, int m2, int m3) -> double& {
    const int M = m1 + m2;
    return l2_part[pair_offset[m1 * (m1 - 1) / 2 + m2] + (m3 - (M / 2 + 1))];
  };
  for (int m = 0; m < S2; ++m)
    for (int mp = 0; mp < S2; ++mp) {
      if (mp == m + 1 || mp + 1 == m) continue;
      int a, b, c, d;
      double s = -lam[m] * lam[mp];
      if (mp > m + 1) {
        a = mp;
        b = m + 1;
      } else {
        a = m + 1;
        b = mp;
        s = -s;
      }
      if (mp + 1 > m) {
        c = mp + 1;
        d = m;
      } else {
        c = m;
        d = mp + 1;
        s = -s;
      }
      (void)b;
      slot(c, d, a) += s;
    }
  for (int a = 0; a <= S2; ++a)
    for (int b = 0; b < a; ++b) slot(a, b, a) -= (lam[a] * lam[a] + lam[b] * lam[b]) / (nbr_particles - 1);
}

double l2_constant(int total_lz) {
  const double lz = 0.5 * total_lz;
  return lz * lz + lz;
}

// ------------------------------------------------------------ eigensolvers
// Implicit QL with Wilkinson shifts on a symmetric tridiagonal matrix; eigenvectors are the
// accumulated rotations (z column-major n x n, columns = eigenvectors), sorted ascending.
int tridiagonal_eigen(int n, const double* diag, const double* off, double* eig, double* z) {
  std::vector<double> d(diag, diag + n), e(n + 1, 0.0);
  for (int i = 0; i + 1 < n; ++i) e[i] = off[i];
  if (z) {
    std::fill(z, z + (size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) z[(size_t)i * n + i] = 1.0;
  }
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m + 1 < n; ++m) {
        double s = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= 2.220446049250313e-16 * s || fabs(e[m]) < 1e-300) break;
      }
      if (m == l) break;
      if (++iter > 300) {
        set_error("tridiagonal QL did not converge");
        return DH_ERR_NOT_CONVERGED;
      }
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        double f = s * e[i], b = c * e[i];
        r = hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        if (z) {
          double* zi = z + (size_t)i * n;
          double* zi1 = z + (size_t)(i + 1) * n;
          for (int k = 0; k < n; ++k) {
            double t = zi1[k];
            zi1[k] = s * zi[k] + c * t;
            zi[k] = c * zi[k] - s * t;
          }
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
  for (int i = 0; i < n; ++i) eig[i] = d[order[i]];
  if (z) {
    std::vector<double> tmp((size_t)n * n);
    for (int i = 0; i < n; ++i) memcpy(&tmp[(size_t)i * n], z + (size_t)order[i] * n, sizeof(double) * n);
    memcpy(z, tmp.data(), sizeof(double) * n * n);
  }
  return DH_OK;
}

// Bisection on the Sturm sequence: the number of eigenvalues below x is the number of negative
// pivots of the LDL^T factorisation of T - x (q_0 = d_0 - x, q_i = d_i - x - e_{i-1}^2 / q_{i-1}),
// started from the Gershgorin interval and halved until it is a few ulps wide.
int tridiagonal_lowest(int n, const double* diag, const double* off, int m, double* eig) {
  if (n <= 0 || m <= 0) return DH_OK;
  m = std::min(m, n);
  double lo = diag[0], hi = diag[0], scale = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(off[i - 1]) : 0.0) + (i + 1 < n ? fabs(off[i]) : 0.0);
    lo = std::min(lo, diag[i] - r);
    hi = std::max(hi, diag[i] + r);
    scale = std::max(scale, fabs(diag[i]) + r);
  }
  const double tiny = std::numeric_limits<double>::min() / std::numeric_limits<double>::epsilon();
  auto below = [&](double x) {
    int c = 0;
    double q = diag[0] - x;
    if (q < 0.0) ++c;
    for (int i = 1; i < n; ++i) {
      if (fabs(q) < tiny) q = (q < 0.0) ? -tiny : tiny;
      q = diag[i] - x - off[i - 1] * off[i - 1] / q;
      if (q < 0.0) ++c;
    }
    return c;
  };
  const double tol = 4.0 * std::numeric_limits<double>::epsilon() * std::max(scale, tiny);
  double left = lo - tol;
  for (int j = 0; j < m; ++j) {
    double a = left, b = hi + tol;
    // eigenvalue j: the smallest x with more than j eigenvalues below it
    for (int it = 0; it < 200 && b - a > tol; ++it) {
      const double mid = 0.5 * (a + b);
      if (below(mid) > j)
        b = mid;
      else
        a = mid;
    }
    eig[j] = 0.5 * (a + b);
    left = a;  // the next eigenvalue is not below this one
  }
  return DH_OK;
}

// The lowest eigenvalue of the tridiagonal matrix given an upper bound `above` (the lowest eigenvalue
// of its leading (n - 1) x (n - 1) block: by interlacing the new one is not above it).  Newton steps on
// det(T - x) from the pivots q_k of T - x (q_0 = d_0 - x, q_k = d_k - x - e_{k-1}^2 / q_{k-1}; the
// logarithmic derivative is sum_k q_k' / q_k), kept inside a bracket that the Sturm counts (the
// number of negative pivots = eigenvalues below x) shrink; a step that leaves the bracket bisects.
int tridiagonal_lowest_below(int n, const double* diag, const double* off, double above, double* eig0) {
  if (n <= 0) return DH_OK;
  double lo = diag[0], scale = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? fabs(off[i - 1]) : 0.0) + (i + 1 < n ? fabs(off[i]) : 0.0);
    lo = std::min(lo, diag[i] - r);
    scale = std::max(scale, fabs(diag[i]) + r);
  }
  const double tiny = std::numeric_limits<double>::min() / std::numeric_limits<double>::epsilon();
  const double tol = 4.0 * std::numeric_limits<double>::epsilon() * std::max(scale, tiny);
  // pivots at x: the Sturm count and the Newton step -det / det'
  auto eval = [&](double x, int& below, double& step) {
    below = 0;
    double q = diag[0] - x, dq = -1.0, sum = 0.0;
    for (int i = 0;; ++i) {
      if (fabs(q) < tiny) q = (q < 0.0) ? -tiny : tiny;
      if (q < 0.0) ++below;
      sum += dq / q;
      if (i + 1 == n) break;
      const double e2 = off[i] * off[i];
      const double qn = diag[i + 1] - x - e2 / q;
      dq = -1.0 + e2 * dq / (q * q);
      q = qn;
    }
    step = (sum != 0.0) ? -1.0 / sum : 0.0;
  };
  double hi = std::max(above, lo) + tol;
  int c = 0;
  double step = 0.0;
  eval(hi, c, step);
  if (c == 0) {  // nothing below the bound: the eigenvalue is the bound (to rounding)
    *eig0 = above;
    return DH_OK;
  }
  lo -= tol;
  double x = hi;
  for (int it = 0; it < 200 && hi - lo > tol; ++it) {
    double nx = x + step;
    if (!(nx > lo && nx < hi)) nx = 0.5 * (lo + hi);
    x = nx;
    eval(x, c, step);
    if (c >= 1)
      hi = x;
    else
      lo = x;
    if (fabs(step) <= tol) {
      // a root: the lowest one only if nothing lies below it (Newton may have found the next one,
      // which can sit at the top of the bracket), else the bracket drops below it and bisects on
      const double root = x + step;
      int below = 0;
      double unused = 0.0;
      eval(root - tol, below, unused);
      if (below == 0) {
        *eig0 = root;
        return DH_OK;
      }
      hi = std::min(hi, root - tol);
      step = hi - lo;  // outside the bracket: the next point is its midpoint
    }
  }
  *eig0 = 0.5 * (lo + hi);
  return DH_OK;
}

// Householder reduction of a dense symmetric matrix to tridiagonal form, then implicit QL.
// a (row-major n x n) is overwritten; z (row-major, columns = eigenvectors) optional.
int symmetric_eigen(int n, double* a, double* eig, double* z) {
  if (n == 0) return DH_OK;
  std::vector<double> hv((size_t)n * n, 0.0), hnorm(n, 0.0), v(n), p(n);
  for (int k = 0; k + 2 < n; ++k) {
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += a[(size_t)i * n + k] * a[(size_t)i * n + k];
    alpha = sqrt(alpha);
    if (alpha == 0.0) continue;
    double x0 = a[(size_t)(k + 1) * n + k];
    if (x0 > 0) alpha = -alpha;
    std::fill(v.begin(), v.end(), 0.0);
    v[k + 1] = x0 - alpha;
    for (int i = k + 2; i < n; ++i) v[i] = a[(size_t)i * n + k];
    double vn2 = 0.0;
    for (int i = k + 1; i < n; ++i) vn2 += v[i] * v[i];
    if (vn2 == 0.0) continue;
    // A <- H A H, H = I - 2 v v^T / |v|^2, as A - v w^T - w v^T
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += a[(size_t)i * n + j] * v[j];
      p[i] = 2.0 * s / vn2;
    }
    double K = 0.0;
    for (int i = k + 1; i < n; ++i) K += v[i] * p[i];
    K /= vn2;
    for (int i = 0; i < n; ++i) p[i] -= K * v[i];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) a[(size_t)i * n + j] -= v[i] * p[j] + p[i] * v[j];
    memcpy(&hv[(size_t)k * n], v.data(), sizeof(double) * n);
    hnorm[k] = vn2;
  }
  std::vector<double> d(n), off(n > 1 ? n - 1 : 1, 0.0);
  for (int k = 0; k < n; ++k) d[k] = a[(size_t)k * n + k];
  for (int k = 0; k + 1 < n; ++k) off[k] = a[(size_t)(k + 1) * n + k];
  std::vector<double> zt;
  if (z) zt.resize((size_t)n * n);
  int rc = tridiagonal_eigen(n, d.data(), off.data(), eig, z ? zt.data() : nullptr);
  if (rc != DH_OK || !z) return rc;
  // eigenvectors of A = H_0 H_1 ... H_{n-3} (eigenvectors of T)
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) z[(size_t)r * n + c] = zt[(size_t)c * n + r];
  for (int k = n - 3; k >= 0; --k) {
    if (hnorm[k] == 0.0) continue;
    const double* hk = &hv[(size_t)k * n];
    for (int c = 0; c < n; ++c) {
      double s = 0.0;
      for (int i = k + 1; i < n; ++i) s += hk[i] * z[(size_t)i * n + c];
      s = 2.0 * s / hnorm[k];
      for (int i = k + 1; i < n; ++i) z[(size_t)i * n + c] -= s * hk[i];
    }
  }
  return DH_OK;
}

// Symmetric band matrix (half-bandwidth b, dense row-major storage) to tridiagonal form by Givens
// rotations with bulge chasing (Schwarz's algorithm; the role of
// RealBandDiagonalSymmetricMatrix::Tridiagonalize, RealBandDiagonalSymmetricMatrix.cc:847), then the
// implicit QL of tridiagonal_eigen.  Each rotation touches O(b) entries: O(n^2 b) work overall.
namespace {
void band_rotate(double* a, int n, int b, int p, int q, double c, double s) {
  const int lo = std::max(0, p - b - 2), hi = std::min(n - 1, q + b + 1);
  for (int col = lo; col <= hi; ++col) {
    if (col == p || col == q) continue;
    const double x = a[(size_t)p * n + col], y = a[(size_t)q * n + col];
    const double xp = c * x + s * y, yq = -s * x + c * y;
    a[(size_t)p * n + col] = xp;
    a[(size_t)col * n + p] = xp;
    a[(size_t)q * n + col] = yq;
    a[(size_t)col * n + q] = yq;
  }
  const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q], apq = a[(size_t)p * n + q];
  a[(size_t)p * n + p] = c * c * app + 2.0 * c * s * apq + s * s * aqq;
  a[(size_t)q * n + q] = s * s * app - 2.0 * c * s * apq + c * c * aqq;
  const double off = (c * c - s * s) * apq + c * s * (aqq - app);
  a[(size_t)p * n + q] = off;
  a[(size_t)q * n + p] = off;
}

// zero a[q][j] against a[p][j] (j < p = q - 1) with a rotation in the (p, q) plane
void band_annihilate(double* a, int n, int b, int p, int q, int j) {
  const double x = a[(size_t)p * n + j], y = a[(size_t)q * n + j];
  if (y == 0.0) return;
  const double r = hypot(x, y);
  band_rotate(a, n, b, p, q, x / r, y / r);
  a[(size_t)q * n + j] = 0.0;
  a[(size_t)j * n + q] = 0.0;
}
}  // namespace

int band_eigenvalues(int n, int b, double* a, double* eig) {
  if (n <= 0) return DH_OK;
  for (int j = 0; j + 2 < n; ++j) {
    for (int i = std::min(j + b, n - 1); i >= j + 2; --i) {
      band_annihilate(a, n, b, i - 1, i, j);
      // the rotation leaves a bulge at (i + b, i - 1); chase it down the band
      for (int k = i; k + b < n; k += b) band_annihilate(a, n, b, k + b - 1, k + b, k - 1);
    }
  }
  std::vector<double> d(n), e(n > 1 ? n - 1 : 1, 0.0);
  for (int i = 0; i < n; ++i) d[i] = a[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = a[(size_t)(i + 1) * n + i];
  return tridiagonal_eigen(n, d.data(), e.data(), eig, nullptr);
}

// Eigenvector of the symmetric band matrix a (dense row-major, half-bandwidth b, not modified) for
// the eigenvalue lambda, by inverse iteration: (a - sigma) y = x solved with a banded LU with partial
// pivoting (fill-in up to 2 b above the diagonal), sigma just below lambda, three iterations from a
// constant start.  O(n b^2) per iteration against O(n^3) for a dense eigensolve.
int band_inverse_iteration(int n, int b, const double* a, double lambda, double* vec) {
  if (n <= 0) return DH_OK;
  const int w = 3 * b + 1;  // columns kept per row of the factor: j - b .. j + 2 b
  double scale = 0.0;
  for (int i = 0; i < n; ++i) scale = std::max(scale, fabs(a[(size_t)i * n + i]));
  const double sigma = lambda - 1e-12 * std::max(scale, 1.0);
  // u[i][c] holds column i - b + c of row i
  std::vector<double> u((size_t)n * w, 0.0);
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i)
    for (int j = std::max(0, i - b); j <= std::min(n - 1, i + b); ++j)
      u[(size_t)i * w + (j - i + b)] = a[(size_t)i * n + j] - (i == j ? sigma : 0.0);
  auto at = [&](int i, int j) -> double& { return u[(size_t)i * w + (j - i + b)]; };
  // row-interchange LU restricted to the band window
  std::vector<double> rowbuf(w);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(at(k, k));
    for (int i = k + 1; i <= std::min(n - 1, k + b); ++i)
      if (fabs(at(i, k)) > best) {
        best = fabs(at(i, k));
        p = i;
      }
    piv[k] = p;
    if (p != k) {
      // swap rows k and p over columns k .. k + 2b (their common window)
      for (int j = k; j <= std::min(n - 1, k + 2 * b); ++j) {
        const bool pk = (j - k + b) < w, pp = (j - p + b) >= 0 && (j - p + b) < w;
        double vk = pk ? at(k, j) : 0.0, vp = pp ? at(p, j) : 0.0;
        if (pk) at(k, j) = vp;
        if (pp) at(p, j) = vk;
      }
    }
    double d = at(k, k);
    if (d == 0.0) d = at(k, k) = 1e-300;
    for (int i = k + 1; i <= std::min(n - 1, k + b); ++i) {
      const double l = at(i, k) / d;
      at(i, k) = l;
      for (int j = k + 1; j <= std::min(n - 1, k + 2 * b); ++j)
        if (j - i + b < w) at(i, j) -= l * at(k, j);
    }
  }
  std::vector<double> y(n, 1.0 / sqrt((double)n));
  for (int it = 0; it < 3; ++it) {
    // forward: L z = P y
    for (int k = 0; k < n; ++k) {
      if (piv[k] != k) std::swap(y[k], y[piv[k]]);
      for (int i = k + 1; i <= std::min(n - 1, k + b); ++i) y[i] -= at(i, k) * y[k];
    }
    // backward: U v = z
    for (int i = n - 1; i >= 0; --i) {
      double v = y[i];
      for (int j = i + 1; j <= std::min(n - 1, i + 2 * b); ++j) v -= at(i, j) * y[j];
      y[i] = v / at(i, i);
    }
    double nrm = 0.0;
    for (double v : y) nrm += v * v;
    nrm = sqrt(nrm);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) return DH_ERR_STATE;
    for (double& v : y) v /= nrm;
  }
  std::copy(y.begin(), y.end(), vec);
  return DH_OK;
}

// ------------------------------------------------------------ Lanczos Ritz value per row
int lanczos_lowest_ritz(int n, const double* diag, const double* off, const double* previous, double* lowest) {
  if (previous) {
    int rc = tridiagonal_lowest_below(n, diag, off, *previous, lowest);
    if (rc != DH_OK) return rc;
    if (*lowest != *previous) return DH_OK;
    // the bound came back unchanged (the value moved by less than the Newton tolerance): the QL
    // value, whose change the convergence test compares at full resolution
  }
  std::vector<double> eig(n);
  int rc = tridiagonal_eigen(n, diag, off, eig.data(), nullptr);
  if (rc != DH_OK) return rc;
  *lowest = eig[0];
  return DH_OK;
}

// ------------------------------------------------------------ Lanczos batch sizes
int lanczos_batch_prediction(int n, const int* rows, const double* log_ratio, int graph_batch) {
  constexpr int kMinBatch = 2;
  constexpr double kAim = 0.85;
  if (n < 2 || graph_batch <= kMinBatch) return graph_batch;
  const int end = rows[n - 1];
  const double lr = log_ratio[n - 1];
  if (!(lr > 0.0)) return graph_batch;  // passing already, or not a number
  int ref = n - 2;
  while (ref > 0 && end - rows[ref] < kLanczosRateSpan) --ref;
  if (rows[ref] >= end) return graph_batch;
  const double rate = (log_ratio[ref] - lr) / (double)(end - rows[ref]);  // log decrease per row
  if (!(rate > 0.0)) return graph_batch;
  const double rows_left = ceil(kAim * lr / rate);
  return (int)std::max((double)kMinBatch, std::min((double)graph_batch, rows_left));
}

}  // namespace dh

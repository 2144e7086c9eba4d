// harmonic_tables.h -- coefficients of the real harmonics of degree 1..8 and
// the weights of the three-body invariants q_L, computed from their
// mathematical definition.
//
// The descriptor's harmonic of degree L and order m at the unit vector u is
//   Y_Lm(u) = Z_Lm(u_z) * {Re, Im} (u_x + i u_y)^m,
// Z_Lm the primitive integer polynomial (content divided out, positive
// leading coefficient) proportional to d^m P_L / dz^m, P_L the Legendre
// polynomial: d^m P_L / dz^m = kappa_Lm Z_Lm.  The invariant
//   q_L = sum_m |sum_j g(r_ij) Ylm_normalised(u_ij)|^2
// of the reference (find_q_one, nep_utilities.cuh; C3B table at :51) is then
//   q_L = C_L0 s_L0^2 + 2 sum_{m>0} C_Lm (s_Lm,re^2 + s_Lm,im^2),
//   C_Lm = (2L + 1) / (4 pi) * (L - m)! / (L + m)! * kappa_Lm^2,
// with s the moments of the Z_Lm-based harmonics.  Component order per L:
// m = 0, then (re, im) for m = 1..L, starting at L^2 - 1.
#pragma once

#include <cstdlib>

namespace nepx {

constexpr int kHarmonicLMax = 8;

struct HarmonicTables {
  double z[kHarmonicLMax + 1][kHarmonicLMax + 1][kHarmonicLMax + 1];   // [L][m][power of z]
  double c3b[(kHarmonicLMax + 1) * (kHarmonicLMax + 1) - 1];           // weight per component
};

inline long long gcd_ll(long long a, long long b)
{
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

inline HarmonicTables make_harmonic_tables()
{
  HarmonicTables t{};
  const double pi = 3.14159265358979323846;
  for (int L = 1; L <= kHarmonicLMax; ++L) {
    // 2^L P_L(z) = sum_k (-1)^k C(L, k) C(2L - 2k, L) z^(L - 2k)
    long long p[kHarmonicLMax + 1] = {0};
    for (int k = 0; 2 * k <= L; ++k) {
      long long c1 = 1, c2 = 1;
      for (int r = 1; r <= k; ++r) c1 = c1 * (L - r + 1) / r;
      for (int r = 1; r <= L; ++r) c2 = c2 * (2 * L - 2 * k - r + 1) / r;
      p[L - 2 * k] = (k % 2 ? -1 : 1) * c1 * c2;
    }
    for (int m = 0; m <= L; ++m) {
      // m-th derivative of 2^L P_L
      long long d[kHarmonicLMax + 1] = {0};
      for (int k = 0; k + m <= L; ++k) {
        long long f = 1;
        for (int r = k + 1; r <= k + m; ++r) f *= r;
        d[k] = p[k + m] * f;
      }
      long long g = 0;
      for (int k = 0; k + m <= L; ++k) g = gcd_ll(g, d[k]);
      if (d[L - m] < 0) g = -g;
      for (int k = 0; k + m <= L; ++k) t.z[L][m][k] = static_cast<double>(d[k] / g);
      const double kappa = static_cast<double>(g) / static_cast<double>(1LL << L);
      double ratio = 1.0;   // (L - m)! / (L + m)!
      for (int r = L - m + 1; r <= L + m; ++r) ratio /= r;
      const double c = (2 * L + 1) / (4.0 * pi) * ratio * kappa * kappa;
      const int st = L * L - 1;
      if (m == 0) {
        t.c3b[st] = c;
      } else {
        t.c3b[st + 2 * m - 1] = c;
        t.c3b[st + 2 * m] = c;
      }
    }
  }
  return t;
}

}  // namespace nepx

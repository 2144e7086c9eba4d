// nhc.h -- Nose-Hoover chain half step, shared by the device thermostat and
// the host known-answer test.
//
// Martyna-Tuckerman-Klein chain of length kChainLength integrated with a
// 7-point Suzuki-Yoshida factorisation and 4 multiple-time-step substeps
// (Tuckerman, "Statistical Mechanics: Theory and Molecular Simulation", the
// scheme of the reference's thermostat_nhc.cpp:47-116).  Returns the velocity
// scale of this half step; ek2 is twice the kinetic energy, dN the number of
// degrees of freedom, kT the target temperature in eV.
#pragma once

#include <cmath>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#endif
#endif

namespace nepx {

constexpr int kChainLength = 4;

__host__ __device__ inline double nhc_half_step(double* pos, double* mom, const double* mass,
                                                double ek2, double kT, double dN, double dt_half)
{
  const double w[7] = {0.784513610477560,  0.235573213359357, -1.17767998417887,
                       1.31518632068391,  -1.17767998417887,  0.235573213359357,
                       0.784513610477560};
  const int M = kChainLength;
  double factor = 1.0;
  for (int a = 0; a < 7; ++a) {
    const double dt2 = dt_half * w[a] / 4;
    const double dt4 = dt2 * 0.5;
    const double dt8 = dt4 * 0.5;
    for (int b = 0; b < 4; ++b) {
      double G = mom[M - 2] * mom[M - 2] / mass[M - 2] - kT;
      mom[M - 1] += dt4 * G;
      for (int m = M - 2; m >= 0; --m) {
        const double t = exp(-dt8 * mom[m + 1] / mass[m + 1]);
        G = m == 0 ? ek2 - dN * kT : mom[m - 1] * mom[m - 1] / mass[m - 1] - kT;
        mom[m] = t * (t * mom[m] + dt4 * G);
      }
      for (int m = M - 1; m >= 0; --m) pos[m] += dt2 * mom[m] / mass[m];
      const double f = exp(-dt2 * mom[0] / mass[0]);
      ek2 *= f * f;
      factor *= f;
      for (int m = 0; m < M - 1; ++m) {
        const double t = exp(-dt8 * mom[m + 1] / mass[m + 1]);
        G = m == 0 ? ek2 - dN * kT : mom[m - 1] * mom[m - 1] / mass[m - 1] - kT;
        mom[m] = t * (t * mom[m] + dt4 * G);
      }
      G = mom[M - 2] * mom[M - 2] / mass[M - 2] - kT;
      mom[M - 1] += dt4 * G;
    }
  }
  return factor;
}

}  // namespace nepx

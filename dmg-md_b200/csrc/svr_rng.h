// svr_rng.h -- host random stream of the stochastic thermostat and barostat.
//
// The reference draws on the host from std::mt19937 with
// std::uniform_real_distribution<double>(0, 1)
// (src/gpumd_compat/thermostat_svr.cpp:20-126): a Marsaglia polar Gaussian
// that caches its second value, the Numerical Recipes gamma deviate, and
// Bussi's sum of squared Gaussian noises (Bussi, Donadio, Parrinello,
// J. Chem. Phys. 126, 014101 (2007)).  None of these draws depends on the
// kinetic energy, so the engine generates every step's draws ahead of a run
// and the device combines them with the kinetic energy it reduced itself:
// the device step never waits on the host, and the sequence matches the
// reference draw for draw (tests/golden/thermostats/svr.json).
#pragma once

#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>

#ifndef __CUDACC__
#define __host__
#define __device__
#endif

namespace nepx {

struct SvrRng {
  std::mt19937 rng;
  int iset = 0;
  double gset = 0.0;

  explicit SvrRng(uint32_t seed) : rng(seed) {}

  double uniform()
  {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    return u(rng);
  }

  // Marsaglia polar method; the second deviate is kept for the next call.
  double gasdev()
  {
    if (iset == 0) {
      double v1, v2, rsq;
      do {
        v1 = 2.0 * uniform() - 1.0;
        v2 = 2.0 * uniform() - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while (rsq >= 1.0 || rsq == 0.0);
      const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
      gset = v1 * fac;
      iset = 1;
      return v2 * fac;
    }
    iset = 0;
    return gset;
  }

  // Gamma deviate of integer order ia: product of uniforms below 6, else the
  // rejection method with a Lorentzian comparison function.
  double gamdev(int ia)
  {
    if (ia < 1) throw std::invalid_argument("gamma deviate needs order >= 1");
    double x;
    if (ia < 6) {
      x = 1.0;
      for (int j = 1; j <= ia; ++j) x *= uniform();
      return -std::log(x);
    }
    double e, y, am, s, v1, v2;
    do {
      do {
        do {
          v1 = uniform();
          v2 = 2.0 * uniform() - 1.0;
        } while (v1 * v1 + v2 * v2 > 1.0);
        y = v2 / v1;
        am = ia - 1;
        s = std::sqrt(2.0 * am + 1.0);
        x = s * y + am;
      } while (x <= 0.0);
      e = (1.0 + y * y) * std::exp(am * std::log(x / am) - s * y);
    } while (uniform() > e);
    return x;
  }

  // Sum of nn squared unit Gaussians.
  double sumnoises(int nn)
  {
    if (nn == 0) return 0.0;
    if (nn == 1) {
      const double r = gasdev();
      return r * r;
    }
    if (nn % 2 == 0) return 2.0 * gamdev(nn / 2);
    const double r = gasdev();
    return 2.0 * gamdev((nn - 1) / 2) + r * r;
  }
};

// Bussi's kinetic-energy resampling given its two random inputs:
// rr (one Gaussian, drawn first) and sum (sumnoises(ndeg - 1)).
// factor = exp(-1/taut) for taut > 0.1, else 0.
__host__ __device__ inline double resample_kinetic(double kk, double sigma, int ndeg,
                                                    double factor, double rr, double sum)
{
  return kk + (1.0 - factor) * (sigma * (sum + rr * rr) / ndeg - kk) +
         2.0 * rr * sqrt(kk * sigma / ndeg * (1.0 - factor) * factor);
}

}  // namespace nepx

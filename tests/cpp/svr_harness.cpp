// Test harness: exposes the engine's host random stream (svr_rng.h) and its
// kinetic-energy resampling to ctypes, so the thermostat known-answer tests
// run on the CPU.  Compiled by tests/test_thermostat_kat.py.
#include <cmath>
#include <cstdint>

#include "../../dmg-md_b200/csrc/svr_rng.h"

extern "C" {

// The reference fixture protocol (tests/thermostats/fixtures/generate_svr.py):
// fresh stream, 6 Gaussians, sumnoises for nn in nn_list, then `steps`
// resamplings of (kk, sigma, ndeg, taut).
void svr_fixture(uint32_t seed, int ndeg, double taut, double kk, double sigma, const int* nn_list,
                 int n_nn, int steps, double* gauss6, double* sums, double* resampled)
{
  nepx::SvrRng r(seed);
  for (int k = 0; k < 6; ++k) gauss6[k] = r.gasdev();
  for (int k = 0; k < n_nn; ++k) sums[k] = r.sumnoises(nn_list[k]);
  const double factor = taut > 0.1 ? std::exp(-1.0 / taut) : 0.0;
  for (int k = 0; k < steps; ++k) {
    const double rr = r.gasdev();
    const double sum = r.sumnoises(ndeg - 1);
    resampled[k] = nepx::resample_kinetic(kk, sigma, ndeg, factor, rr, sum);
  }
}

// The per-step draws nepx_md_run generates: {rr, sumnoises(ndeg-1), barostat gaussian}.
void svr_step_draws(uint32_t seed, int ndeg, int steps, int with_barostat, double* out)
{
  nepx::SvrRng r(seed);
  for (int k = 0; k < steps; ++k) {
    out[3 * k] = r.gasdev();
    out[3 * k + 1] = r.sumnoises(ndeg - 1);
    out[3 * k + 2] = with_barostat ? r.gasdev() : 0.0;
  }
}

double resample(double kk, double sigma, int ndeg, double factor, double rr, double sum)
{
  return nepx::resample_kinetic(kk, sigma, ndeg, factor, rr, sum);
}
}

#include "../../dmg-md_b200/csrc/nhc.h"

extern "C" double nhc_step(double* pos, double* mom, const double* mass, double ek2, double kT,
                           double dN, double dt_half)
{
  return nepx::nhc_half_step(pos, mom, mass, ek2, kT, dN, dt_half);
}

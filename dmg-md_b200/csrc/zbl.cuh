// zbl.cuh -- ZBL screened-Coulomb pair term (universal, typewise and flexible).
// Included inside namespace nepx by nep_force.cu.
#pragma once

__device__ __forceinline__ void zbl_universal(float zizj, float a_inv, float r1, float r2, float d,
                                              float dinv, float& f, float& fp)
{
  // universal screening (reference nep_utilities.cuh:426-452)
  const float x = d * a_inv;
  f = 0.0f;
  fp = 0.0f;
  const float cp[8] = {0.18175f, 3.1998f, 0.50986f, 0.94229f, 0.28022f, 0.4029f, 0.02817f, 0.20162f};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float t = cp[2 * k] * expf(-cp[2 * k + 1] * x);
    f += t;
    fp -= cp[2 * k + 1] * t;
  }
  f *= zizj;
  fp *= zizj * a_inv;
  fp = fp * dinv - f * dinv * dinv;
  f *= dinv;
  float fc, fcp;
  if (d < r1) {
    fc = 1.0f;
    fcp = 0.0f;
  } else if (d < r2) {
    const float pf = 3.1415927f / (r2 - r1);
    float s, c;
    sincosf(pf * (d - r1), &s, &c);
    fc = 0.5f * c + 0.5f;
    fcp = -s * pf * 0.5f;
  } else {
    fc = 0.0f;
    fcp = 0.0f;
  }
  fp = fp * fc + f * fcp;
  f *= fc;
}

__device__ __forceinline__ void zbl_flexible(const float* zp, float zizj, float a_inv, float d,
                                             float dinv, float& f, float& fp)
{
  // flexible screening from the potential file (nep_utilities.cuh:454-475)
  const float x = d * a_inv;
  f = 0.0f;
  fp = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float t = zp[2 + 2 * k] * expf(-zp[3 + 2 * k] * x);
    f += t;
    fp -= zp[3 + 2 * k] * t;
  }
  f *= zizj;
  fp *= zizj * a_inv;
  fp = fp * dinv - f * dinv * dinv;
  f *= dinv;
  const float r1 = zp[0], r2 = zp[1];
  float fc, fcp;
  if (d < r1) {
    fc = 1.0f;
    fcp = 0.0f;
  } else if (d < r2) {
    const float pf = 3.1415927f / (r2 - r1);
    float s, c;
    sincosf(pf * (d - r1), &s, &c);
    fc = 0.5f * c + 0.5f;
    fcp = -s * pf * 0.5f;
  } else {
    fc = 0.0f;
    fcp = 0.0f;
  }
  fp = fp * fc + f * fcp;
  f *= fc;
}

// covalent radii for the typewise ZBL cutoff (nep_utilities.cuh:175)
__constant__ float c_covalent[94] = {
  0.426667f, 0.613333f, 1.6f, 1.25333f, 1.02667f, 1.0f, 0.946667f, 0.84f, 0.853333f, 0.893333f,
  1.86667f, 1.66667f, 1.50667f, 1.38667f, 1.46667f, 1.36f, 1.32f, 1.28f, 2.34667f, 2.05333f,
  1.77333f, 1.62667f, 1.61333f, 1.46667f, 1.42667f, 1.38667f, 1.33333f, 1.32f, 1.34667f, 1.45333f,
  1.49333f, 1.45333f, 1.53333f, 1.46667f, 1.52f, 1.56f, 2.52f, 2.22667f, 1.96f, 1.85333f,
  1.76f, 1.65333f, 1.53333f, 1.50667f, 1.50667f, 1.44f, 1.53333f, 1.64f, 1.70667f, 1.68f,
  1.68f, 1.64f, 1.76f, 1.74667f, 2.78667f, 2.34667f, 2.16f, 1.96f, 2.10667f, 2.09333f,
  2.08f, 2.06667f, 2.01333f, 2.02667f, 2.01333f, 2.0f, 1.98667f, 1.98667f, 1.97333f, 2.04f,
  1.94667f, 1.82667f, 1.74667f, 1.64f, 1.57333f, 1.54667f, 1.48f, 1.49333f, 1.50667f, 1.76f,
  1.73333f, 1.73333f, 1.81333f, 1.74667f, 1.84f, 1.89333f, 2.68f, 2.41333f, 2.22667f, 2.10667f,
  2.02667f, 2.04f, 2.05333f, 2.06667f};

// xbox.h -- the small-box criterion and expanded box of the reference, on
// host and device with the same roundings.
//
// Reference get_expanded_box (src/gpumd_compat/nep.cu:2002-2061) with
// Box::get_volume / get_area (box.cu:60-96): a periodic direction thinner
// than 2.5 (rc + 1) makes the box "small"; each periodic direction is then
// replicated ceil(2 rc / thickness) times and neighbours are enumerated over
// every atom and every replica.  The expanded box and its inverse are float,
// the inverse built from float cofactors and a float determinant divided in
// double.  The device copy uses the _rn intrinsics so no product is fused
// into an FMA: the values equal the host's.
#pragma once

#include <cmath>

#include "common.cuh"

namespace nepx {

#ifdef __CUDA_ARCH__
#define NEPX_FMUL(a, b) __fmul_rn((a), (b))
#define NEPX_FADD(a, b) __fadd_rn((a), (b))
#define NEPX_FSUB(a, b) __fsub_rn((a), (b))
#define NEPX_DMUL(a, b) __dmul_rn((a), (b))
#define NEPX_DADD(a, b) __dadd_rn((a), (b))
#define NEPX_DSUB(a, b) __dsub_rn((a), (b))
#else
#define NEPX_FMUL(a, b) ((a) * (b))
#define NEPX_FADD(a, b) ((a) + (b))
#define NEPX_FSUB(a, b) ((a) - (b))
#define NEPX_DMUL(a, b) ((a) * (b))
#define NEPX_DADD(a, b) ((a) + (b))
#define NEPX_DSUB(a, b) ((a) - (b))
#endif

__host__ __device__ inline double xbox_area(const double* a, const double* b)
{
  const double s1 = NEPX_DSUB(NEPX_DMUL(a[1], b[2]), NEPX_DMUL(a[2], b[1]));
  const double s2 = NEPX_DSUB(NEPX_DMUL(a[2], b[0]), NEPX_DMUL(a[0], b[2]));
  const double s3 = NEPX_DSUB(NEPX_DMUL(a[0], b[1]), NEPX_DMUL(a[1], b[0]));
  return sqrt(NEPX_DADD(NEPX_DADD(NEPX_DMUL(s1, s1), NEPX_DMUL(s2, s2)), NEPX_DMUL(s3, s3)));
}

// Fills si (box, small flag, images, expanded box) for cutoff rc (the
// largest radial cutoff).  Returns 0, or 1 when the box is small in one
// periodic direction and thicker than 10 rc in another (the reference stops
// there).  si.off / si.n are left to the caller.
__host__ __device__ inline int expanded_box(const Box& b, double rc, StructInfo& si)
{
  const double* h = b.h;
  const double vol = fabs(NEPX_DADD(
    NEPX_DADD(NEPX_DMUL(h[0], NEPX_DSUB(NEPX_DMUL(h[4], h[8]), NEPX_DMUL(h[5], h[7]))),
              NEPX_DMUL(h[1], NEPX_DSUB(NEPX_DMUL(h[5], h[6]), NEPX_DMUL(h[3], h[8])))),
    NEPX_DMUL(h[2], NEPX_DSUB(NEPX_DMUL(h[3], h[7]), NEPX_DMUL(h[4], h[6])))));
  const double va[3] = {h[0], h[3], h[6]};
  const double vb[3] = {h[1], h[4], h[7]};
  const double vc[3] = {h[2], h[5], h[8]};
  const double thick[3] = {vol / xbox_area(vb, vc), vol / xbox_area(vc, va),
                           vol / xbox_area(va, vb)};
  si.box = b;
  si.small = 0;
  si.nc[0] = si.nc[1] = si.nc[2] = 0;
  si.cell_base = 0;
  si.keep = 0;
  for (int d = 0; d < 3; ++d) {
    si.ncell[d] = b.pbc[d] ? static_cast<int>(ceil(2.0 * rc / thick[d])) : 1;
    if (b.pbc[d] && thick[d] <= 2.5 * (rc + 1.0)) si.small = 1;
  }
  for (int k = 0; k < 18; ++k) si.eh[k] = 0.0f;
  if (!si.small) return 0;
  for (int d = 0; d < 3; ++d)
    if (thick[d] > 10.0 * rc) return 1;
  float* e = si.eh;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      e[3 * r + c] = static_cast<float>(NEPX_DMUL(h[3 * r + c], static_cast<double>(si.ncell[c])));
  e[9] = NEPX_FSUB(NEPX_FMUL(e[4], e[8]), NEPX_FMUL(e[5], e[7]));
  e[10] = NEPX_FSUB(NEPX_FMUL(e[2], e[7]), NEPX_FMUL(e[1], e[8]));
  e[11] = NEPX_FSUB(NEPX_FMUL(e[1], e[5]), NEPX_FMUL(e[2], e[4]));
  e[12] = NEPX_FSUB(NEPX_FMUL(e[5], e[6]), NEPX_FMUL(e[3], e[8]));
  e[13] = NEPX_FSUB(NEPX_FMUL(e[0], e[8]), NEPX_FMUL(e[2], e[6]));
  e[14] = NEPX_FSUB(NEPX_FMUL(e[2], e[3]), NEPX_FMUL(e[0], e[5]));
  e[15] = NEPX_FSUB(NEPX_FMUL(e[3], e[7]), NEPX_FMUL(e[4], e[6]));
  e[16] = NEPX_FSUB(NEPX_FMUL(e[1], e[6]), NEPX_FMUL(e[0], e[7]));
  e[17] = NEPX_FSUB(NEPX_FMUL(e[0], e[4]), NEPX_FMUL(e[1], e[3]));
  const float detf = NEPX_FADD(
    NEPX_FADD(NEPX_FMUL(e[0], NEPX_FSUB(NEPX_FMUL(e[4], e[8]), NEPX_FMUL(e[5], e[7]))),
              NEPX_FMUL(e[1], NEPX_FSUB(NEPX_FMUL(e[5], e[6]), NEPX_FMUL(e[3], e[8])))),
    NEPX_FMUL(e[2], NEPX_FSUB(NEPX_FMUL(e[3], e[7]), NEPX_FMUL(e[4], e[6]))));
  const double det = detf;
  for (int k = 9; k < 18; ++k) e[k] = static_cast<float>(static_cast<double>(e[k]) / det);
  return 0;
}

}  // namespace nepx

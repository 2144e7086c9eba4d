// common.cuh -- shared device-side definitions of the nepx engine.
//
// Box and minimum image, NEP constants, cutoff and Chebyshev radial basis,
// and the real solid harmonics used by the descriptor and force kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nepx {

constexpr int kMaxTypes = 16;
constexpr int kMaxBasis = 17;   // basis_size + 1
constexpr int kMaxN = 13;       // n_max + 1
constexpr int kNumLM = 24;      // (L_max + 1)^2 - 1 at L_max = 4
constexpr int kNumLMHigh = 80;  // (L_max + 1)^2 - 1 at L_max = 8, the largest the format has
constexpr int kMaxDim = 128;
constexpr int kMaxInv = 6;      // q_222, q_1111, q_112, q_123, q_233, q_134
constexpr double kBoltzmann = 8.617343e-5;           // eV/K, GPUMD natural units
constexpr double kTimeUnit = 1.018051e+1;            // natural time unit in fs
constexpr double kPressureUnit = 1.602177e+2;        // eV/A^3 in GPa
constexpr float kCoulomb = 14.399645f;               // e^2/(4 pi eps0) in eV A

// Device-resident periodic box.  h is row-major with the cell vectors a, b, c
// as columns (the layout of the reference's Box::cpu_h[0..8]); hinv its
// inverse; fh the float copy (h then hinv) the FP32 kernels use.
struct Box {
  double h[9];
  double hinv[9];
  float fh[18];
  int pbc[3];
  int ortho;
};

// One structure of an explicit-row evaluation (the small-box path, and every
// structure of a batch): its box, the reference's expanded box for the image
// arithmetic, and its slice [off, off + n) of the concatenated atom arrays.
struct StructInfo {
  Box box;
  float eh[18];   // expanded box h (columns scaled by ncell) then its float inverse
  int ncell[3];   // images per direction (1 where not periodic)
  int small;      // 1: the reference's small-box image arithmetic; 0: minimum image
  int off, n;
  int nc[3];      // cell grid of a large structure's candidate search (nc[0] = 0: scan all atoms)
  int cell_base;  // first cell of this structure in the batch's cell arrays
  int keep;       // 1: keeps Verlet candidates across steps (cells sized for rc + skin)
};

// Packed neighbour of an explicit row: index j (low 28 bits) and type (high 4).
constexpr int kRowTypeShift = 28;
constexpr int kRowIndexMask = (1 << kRowTypeShift) - 1;

// Cell grid and rebuild bookkeeping of the Verlet list, device resident.
struct NeighborState {
  int rebuild;         // 1: rebuild the Verlet list before the next filter
  int overflow;        // bit 0 Verlet row, bit 1 radial row, bit 2 angular row
  int nc[3];           // cells per direction
  int ncell;
  int max_nn[3];       // largest Verlet / radial / angular row since the last stats read
  int call_nn[2];      // largest radial / angular row of the latest force evaluation
  int nonfinite;       // a force or energy came out NaN/Inf
  int box_error;       // the device box became unsupported (small in one direction, >10 rc in another)
  int ann_error;       // a tensor-core ANN tile gave up waiting for its MMAs
  int sync_error;      // the neighbour rebuild gave up waiting at a grid-wide barrier
  unsigned xr_builds;  // centers whose batch Verlet candidates were built (wraps)
  double box_scale;    // product of isotropic box factors since the last build (1 = none)
  double box_def[9];   // product of general box deformations since the last build (I = none)
};

// Minimum image of a float displacement, the arithmetic of the large-box
// path (reference box.cuh:84-127): half-box shortcut for orthogonal boxes,
// fractional nearbyint otherwise.
__device__ __forceinline__ void mic_f32(const Box& b, float& x, float& y, float& z)
{
  if (b.ortho) {
    const float lx2 = b.fh[0] * 0.5f, ly2 = b.fh[4] * 0.5f, lz2 = b.fh[8] * 0.5f;
    if (b.pbc[0] == 1) {
      if (x < -lx2) x += b.fh[0];
      else if (x > +lx2) x -= b.fh[0];
    }
    if (b.pbc[1] == 1) {
      if (y < -ly2) y += b.fh[4];
      else if (y > +ly2) y -= b.fh[4];
    }
    if (b.pbc[2] == 1) {
      if (z < -lz2) z += b.fh[8];
      else if (z > +lz2) z -= b.fh[8];
    }
  } else {
    float sx = b.fh[9] * x + b.fh[10] * y + b.fh[11] * z;
    float sy = b.fh[12] * x + b.fh[13] * y + b.fh[14] * z;
    float sz = b.fh[15] * x + b.fh[16] * y + b.fh[17] * z;
    if (b.pbc[0] == 1) sx -= nearbyintf(sx);
    if (b.pbc[1] == 1) sy -= nearbyintf(sy);
    if (b.pbc[2] == 1) sz -= nearbyintf(sz);
    x = b.fh[0] * sx + b.fh[1] * sy + b.fh[2] * sz;
    y = b.fh[3] * sx + b.fh[4] * sy + b.fh[5] * sz;
    z = b.fh[6] * sx + b.fh[7] * sy + b.fh[8] * sz;
  }
}

// Displacement r_j - r_i: the double difference rounded to float, then the
// float minimum image -- the operand order of the reference's filter
// (nep.cu:542-549), so neighbour predicates agree bit for bit.
__device__ __forceinline__ void displacement(const Box& b, const double* __restrict__ x,
                                             const double* __restrict__ y,
                                             const double* __restrict__ z, double xi, double yi,
                                             double zi, int j, float& dx, float& dy, float& dz)
{
  dx = __ldg(x + j) - xi;
  dy = __ldg(y + j) - yi;
  dz = __ldg(z + j) - zi;
  mic_f32(b, dx, dy, dz);
}

// One atom as the neighbour sweeps read it: position and type in one
// 32-byte record (one sector), repacked from the SoA inputs at every force
// call.  The SoA layout would touch four cache lines per neighbour.
struct __align__(32) Site {
  double x, y, z;
  long long type;
};

// A site record as two 16-byte loads: a = (x, y), c = (z, type bits).
__device__ __forceinline__ void site_load(const Site* __restrict__ sites, int j, double2& a,
                                          double2& c)
{
  a = __ldg(reinterpret_cast<const double2*>(sites + j));
  c = __ldg(reinterpret_cast<const double2*>(sites + j) + 1);
}

// Displacement from (xi, yi, zi) to a loaded site and the site's type, same
// arithmetic as displacement().
__device__ __forceinline__ void site_delta(const Box& b, const double2& a, const double2& c,
                                           double xi, double yi, double zi, float& dx, float& dy,
                                           float& dz, int& tj)
{
  dx = a.x - xi;
  dy = a.y - yi;
  dz = c.x - zi;
  tj = static_cast<int>(__double_as_longlong(c.y));
  mic_f32(b, dx, dy, dz);
}

// Displacement to site j and j's type.
__device__ __forceinline__ void site_displacement(const Box& b, const Site* __restrict__ sites,
                                                  double xi, double yi, double zi, int j,
                                                  float& dx, float& dy, float& dz, int& tj)
{
  double2 a, c;
  site_load(sites, j, a, c);
  site_delta(b, a, c, xi, yi, zi, dx, dy, dz, tj);
}

// Skin criterion of atom i at its new position (reference
// neighbor.cu:446-533, without the host round trip): packs its Site record
// for this step's neighbour sweeps and marks a rebuild when forced or when
// it moved more than skin/2 since the build.  Under an isotropic box scaling
// s since the build (x0 scaled along, so displacements are co-moving) a pair
// distance also drifts by up to |1 - s| (rc + skin), which shrinks the
// allowed displacement to (skin - |1 - s| (rc + skin)) / 2.  A general
// deformation M since the build moves a pair by at most ||M - I||_2
// (rc + skin); the bound used is sqrt(||M - I||_1 ||M - I||_inf) >= ||M - I||_2.
__device__ __forceinline__ void skin_check_atom(int N, int i, const Box& b, double xi, double yi,
                                                double zi, int type_i,
                                                const double* __restrict__ x0, NeighborState* st,
                                                Site* __restrict__ sites, double skin,
                                                double rc_v, int force)
{
  sites[i] = Site{xi, yi, zi, static_cast<long long>(type_i)};
  if (i == 0) {   // the first kernel of a force evaluation: its row maxima start here
    st->call_nn[0] = 0;
    st->call_nn[1] = 0;
  }
  if (force) {
    if (i == 0) st->rebuild = 1;
    return;
  }
  double col[3] = {0.0, 0.0, 0.0}, row_max = 0.0;
  for (int r = 0; r < 3; ++r) {
    double row = 0.0;
    for (int c = 0; c < 3; ++c) {
      const double a = fabs(st->box_def[3 * r + c] - (r == c ? 1.0 : 0.0));
      row += a;
      col[c] += a;
    }
    row_max = fmax(row_max, row);
  }
  const double def = sqrt(fmax(fmax(col[0], col[1]), col[2]) * row_max);
  const double strain = fmax(fabs(1.0 - st->box_scale), def);
  const double half = 0.5 * (skin - strain * rc_v);
  if (half <= 0.0) {
    st->rebuild = 1;
    return;
  }
  const double half_skin_sq = half * half;
  float dx = xi - x0[i];
  float dy = yi - x0[N + i];
  float dz = zi - x0[2 * N + i];
  mic_f32(b, dx, dy, dz);
  if ((dx * dx + dy * dy + dz * dz) > half_skin_sq) st->rebuild = 1;
}

// Cutoff function fc = (1 + cos(pi d / rc)) / 2 and its d-derivative.
// FAST (the mixed-precision kernels): sine and cosine from the hardware
// approximations (absolute error about 4e-7 on [0, pi)) in place of the
// correctly rounded sinpi/cospi.
template <bool FAST = false>
__device__ __forceinline__ void cutoff_fc(float rc, float rcinv, float d, float& fc, float& fcp)
{
  if (d < rc) {
    float s, c;
    if constexpr (FAST) __sincosf(3.14159265f * (d * rcinv), &s, &c);
    else sincospif(d * rcinv, &s, &c);
    fc = 0.5f * c + 0.5f;
    fcp = -1.5707963f * s * rcinv;
  } else {
    fc = 0.0f;
    fcp = 0.0f;
  }
}

// Edge length d and 1 / d from d^2: correctly rounded square root and
// division, or with FAST one hardware reciprocal square root (2 ulp).
template <bool FAST>
__device__ __forceinline__ void edge_length(float d2, float& d, float& dinv)
{
  if constexpr (FAST) {
    dinv = rsqrtf(d2);
    d = d2 * dinv;
  } else {
    d = sqrtf(d2);
    dinv = 1.0f / d;
  }
}

// Shifted Chebyshev radial basis f_k(d) = (T_k(x) + 1) / 2 * fc (f_0 = fc)
// with x = 2 (d/rc - 1)^2 - 1, k = 0..kmax-1.
template <int KMAX>
__device__ __forceinline__ void radial_basis(int kmax, float rcinv, float d, float fc, float* fn)
{
  const float u = d * rcinv - 1.0f;
  const float x = 2.0f * u * u - 1.0f;
  const float half_fc = 0.5f * fc;
  float t0 = 1.0f, t1 = x;
  fn[0] = fc;
#pragma unroll
  for (int k = 1; k < KMAX; ++k) {
    if (k < kmax) fn[k] = (t1 + 1.0f) * half_fc;
    const float t2 = 2.0f * x * t1 - t0;
    t0 = t1;
    t1 = t2;
  }
}

// Basis values and their d-derivatives.
template <int KMAX>
__device__ __forceinline__ void radial_basis_d(int kmax, float rcinv, float d, float fc,
                                               float fcp, float* fn, float* fnp)
{
  const float u = d * rcinv - 1.0f;
  const float x = 2.0f * u * u - 1.0f;
  const float dxdd = 4.0f * u * rcinv;
  float t0 = 1.0f, t1 = x;       // T_{k-1}, T_k
  float dt0 = 0.0f, dt1 = 1.0f;  // dT/dx
  fn[0] = fc;
  fnp[0] = fcp;
#pragma unroll
  for (int k = 1; k < KMAX; ++k) {
    if (k < kmax) {
      fn[k] = 0.5f * (t1 + 1.0f) * fc;
      fnp[k] = 0.5f * (dt1 * dxdd * fc + (t1 + 1.0f) * fcp);
    }
    const float t2 = 2.0f * x * t1 - t0;
    const float dt2 = 2.0f * t1 + 2.0f * x * dt1 - dt0;
    t0 = t1;
    t1 = t2;
    dt0 = dt1;
    dt1 = dt2;
  }
}

// Real solid harmonics of degree L = 1..4 at the unit vector (x, y, z):
// Y = Z_Lm(z) * Re/Im (x + i y)^m with the z-polynomials below, in the
// component order of the reference's blm moments (L^2 - 1 + {0, 2m-1, 2m});
// zp[k] = z^k.  Degrees 5..8 read their coefficients from a table
// (harmonic_tables.h).
__device__ __forceinline__ float zpoly(int L, int m, const float* zp, float* dzf)
{
  // coefficients of the reference's Z_COEFFICIENT_L tables (nep_utilities.cuh:89-117)
  float f = 0.0f, df = 0.0f;
  switch (L * 8 + m) {
    case 8 + 0: f = zp[1]; df = 1.0f; break;
    case 8 + 1: f = 1.0f; df = 0.0f; break;
    case 16 + 0: f = 3.0f * zp[2] - 1.0f; df = 6.0f * zp[1]; break;
    case 16 + 1: f = zp[1]; df = 1.0f; break;
    case 16 + 2: f = 1.0f; df = 0.0f; break;
    case 24 + 0: f = 5.0f * zp[3] - 3.0f * zp[1]; df = 15.0f * zp[2] - 3.0f; break;
    case 24 + 1: f = 5.0f * zp[2] - 1.0f; df = 10.0f * zp[1]; break;
    case 24 + 2: f = zp[1]; df = 1.0f; break;
    case 24 + 3: f = 1.0f; df = 0.0f; break;
    case 32 + 0: f = 35.0f * zp[4] - 30.0f * zp[2] + 3.0f; df = 140.0f * zp[3] - 60.0f * zp[1]; break;
    case 32 + 1: f = 7.0f * zp[3] - 3.0f * zp[1]; df = 21.0f * zp[2] - 3.0f; break;
    case 32 + 2: f = 7.0f * zp[2] - 1.0f; df = 14.0f * zp[1]; break;
    case 32 + 3: f = zp[1]; df = 1.0f; break;
    case 32 + 4: f = 1.0f; df = 0.0f; break;
    default: break;
  }
  *dzf = df;
  return f;
}

}  // namespace nepx

// nep_force.cu -- NEP energy, force and virial on sm_100a (plain FP32 path).
//
// Two kernels per force call (after the neighbour filter):
//
//  k_descriptor_ann_f12  one CTA per tile of kTile centers.
//    * radial and angular edges of the tile are processed edge-parallel in
//      chunks staged through shared memory (one edge per thread): geometry,
//      cutoff, Chebyshev basis, type-pair contraction g_n, harmonics Y_lm;
//    * owner threads (center, n) contract the chunk into the descriptors
//      q_rad[n] and the angular moments s[n][lm] held in shared memory, so
//      there is no atomic and the sum order is fixed;
//    * invariants q_L and q_222/q_1111/q_112/q_123/q_233/q_134, the
//      one-hidden-layer ANN (site energy, dE/dq) and the moment derivatives
//      a[n][lm] = dE/ds[n][lm] are formed per center in shared memory;
//    * a second edge-parallel sweep writes each directed angular partial
//      force f12(i,j) = grad_r sum_{n,lm} a[n][lm] g_n(d) Y_lm(r/d).
//    Reference: find_descriptor (nep.cu:569-748) and
//    find_partial_force_angular (nep.cu:890-991) with the accumulate_f12
//    ladder (nep_utilities.cuh:1240-1491); the angular harmonics and their
//    gradient are evaluated once per edge instead of once per (edge, n).
//
//  k_gather  a group of kGroup lanes per center: radial pair forces from both
//    site energies (reads the neighbour's dE/dq_rad), the angular exchange
//    F_i += f12(i,j) - f12(j,i) with the reverse slot found by binary search
//    in j's sorted row, ZBL, and the per-atom virial W_i = sum_j r_ij (x) f_ji.
//    Reference: find_force_radial (nep.cu:756-881), gpu_find_force_many_body
//    (potential.cu:81-210), find_force_ZBL (nep.cu:996-1111).
#include <cstdio>

#include "engine.h"

namespace nepx {

namespace {

constexpr int kTile = 16;        // centers per CTA
constexpr int kThreads = 128;    // threads per CTA = edges per chunk
constexpr int kGroup = 8;        // lanes per center in the gather

// three-body invariant weights (reference nep_utilities.cuh:52-75, L <= 4)
__constant__ float c_C3B[kNumLM] = {
  0.238732414637843f, 0.119366207318922f, 0.119366207318922f, 0.099471839432435f,
  0.596831036594608f, 0.596831036594608f, 0.149207759148652f, 0.149207759148652f,
  0.139260575205408f, 0.104445431404056f, 0.104445431404056f, 1.044454314040563f,
  1.044454314040563f, 0.174075719006761f, 0.174075719006761f, 0.011190581936149f,
  0.223811638722978f, 0.223811638722978f, 0.111905819361489f, 0.111905819361489f,
  1.566681471060845f, 1.566681471060845f, 0.195835183882606f, 0.195835183882606f};

// Many-body invariants as monomials c * s[i0] s[i1] s[i2] (s[i3]) of the raw
// moments, transcribed from the polynomials of find_q
// (nep_utilities.cuh:1661-1728).  Offsets index c_inv_start per invariant.
struct Monomial {
  float c;
  signed char i[4];
};
__constant__ Monomial c_mono[128];
__constant__ int c_inv_start[kMaxInv + 1];

// ---------------------------------------------------------------------------
// fused descriptor / ANN / angular partial force
// ---------------------------------------------------------------------------

struct DescLayout {
  int c, buf, s, a, q, fp, g, e;   // float offsets
  int ints;                        // int offset (after floats)
  int stride_e;                    // floats per staged edge
  int total_bytes;
};

__host__ __device__ inline int round4(int x) { return (x + 3) & ~3; }

__host__ __device__ inline DescLayout desc_layout(const ModelParams& p)
{
  DescLayout L;
  const int cN = p.T * p.T * (p.nR * p.kR + p.nA * p.kA);
  int se = p.nA + p.nlm;
  if (se < p.nR) se = p.nR;
  if ((se & 1) == 0) se += 1;   // odd stride: conflict-free row writes
  L.stride_e = se;
  int off = 0;
  L.c = off;   off += round4(cN);
  L.buf = off; off += round4(kThreads * se);
  L.s = off;   off += kTile * p.nA * kNumLM;
  L.a = off;   off += kTile * p.nA * kNumLM;
  L.q = off;   off += round4(kTile * p.dim);
  L.fp = off;  off += round4(kTile * p.dim);
  L.g = off;   off += round4(kTile * p.H);
  L.e = off;   off += round4(kTile * p.H);
  L.ints = off;
  L.total_bytes = off * 4 + (4 * kTile + 2 * (kTile + 1) + 4) * 4;
  return L;
}

__device__ __forceinline__ int find_owner(const int* off, int e)
{
  int lo = 0, hi = kTile;   // off[lo] <= e < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads)
k_descriptor_ann_f12(const ModelParams p, int N, const Box* __restrict__ box,
                     const double* __restrict__ pos, const int* __restrict__ type,
                     const int* __restrict__ nn_r, const int* __restrict__ nl_r, int mn_r,
                     const int* __restrict__ nn_a, const int* __restrict__ nl_a, int mn_a,
                     float* __restrict__ fp_rad, float4* __restrict__ f12,
                     double* __restrict__ pe_ann)
{
  extern __shared__ float sm[];
  const DescLayout L = desc_layout(p);
  float* s_c = sm + L.c;
  float* s_buf = sm + L.buf;
  float* s_s = sm + L.s;
  float* s_a = sm + L.a;
  float* s_q = sm + L.q;
  float* s_fp = sm + L.fp;
  float* s_g = sm + L.g;
  float* s_e = sm + L.e;
  int* s_atom = reinterpret_cast<int*>(sm + L.ints);
  int* s_type = s_atom + kTile;
  int* s_offr = s_type + kTile;
  int* s_offa = s_offr + kTile + 1;

  const int tid = threadIdx.x;
  const int T = p.T, nR = p.nR, nA = p.nA, kR = p.kR, kA = p.kA, nlm = p.nlm;
  const int dim = p.dim, H = p.H;
  const int cN = T * T * (nR * kR + nA * kA);
  for (int k = tid; k < cN; k += kThreads) s_c[k] = __ldg(p.c_pair + k);
  const int first = blockIdx.x * kTile;
  if (tid < kTile) {
    const int i = first + tid;
    s_atom[tid] = i < N ? i : -1;
    s_type[tid] = i < N ? type[i] : 0;
  }
  for (int k = tid; k < kTile * nA * kNumLM; k += kThreads) s_s[k] = 0.0f;
  for (int k = tid; k < kTile * dim; k += kThreads) s_q[k] = 0.0f;
  __syncthreads();
  if (tid == 0) {
    int r = 0, a = 0;
    for (int t = 0; t < kTile; ++t) {
      s_offr[t] = r;
      s_offa[t] = a;
      const int i = s_atom[t];
      if (i >= 0) {
        r += nn_r[i];
        a += nn_a[i];
      }
    }
    s_offr[kTile] = r;
    s_offa[kTile] = a;
  }
  __syncthreads();
  const Box b = *box;
  const double* x = pos;
  const double* y = pos + N;
  const double* z = pos + 2 * N;
  const int se = L.stride_e;

  // ---- radial descriptors ------------------------------------------------
  const int total_r = s_offr[kTile];
  for (int e0 = 0; e0 < total_r; e0 += kThreads) {
    const int e = e0 + tid;
    if (e < total_r) {
      const int a = find_owner(s_offr, e);
      const int i = s_atom[a];
      const int t1 = s_type[a];
      const int j = nl_r[static_cast<size_t>(i) * mn_r + (e - s_offr[a])];
      const int t2 = __ldg(type + j);
      float dx, dy, dz;
      displacement(b, x, y, z, x[i], y[i], z[i], j, dx, dy, dz);
      const float d = sqrtf(dx * dx + dy * dy + dz * dz);
      const float rc = (p.rc_r[t1] + p.rc_r[t2]) * 0.5f;
      const float rcinv = 1.0f / rc;
      float fc, fcp;
      cutoff_fc(rc, rcinv, d, fc, fcp);
      float fn[kMaxBasis];
      radial_basis<kMaxBasis>(kR, rcinv, d, fc, fn);
      const float* c = s_c + (t1 * T + t2) * nR * kR;
      for (int n = 0; n < nR; ++n) {
        float g = 0.0f;
#pragma unroll
        for (int k = 0; k < kMaxBasis; ++k)
          if (k < kR) g += fn[k] * c[n * kR + k];
        s_buf[tid * se + n] = g;
      }
    }
    __syncthreads();
    for (int own = tid; own < kTile * nR; own += kThreads) {
      const int a = own / nR, n = own % nR;
      const int lo = max(s_offr[a], e0), hi = min(s_offr[a + 1], e0 + kThreads);
      float acc = 0.0f;
      for (int e = lo; e < hi; ++e) acc += s_buf[(e - e0) * se + n];
      s_q[a * dim + n] += acc;
    }
    __syncthreads();
  }

  // ---- angular moments s[n][lm] -------------------------------------------
  const int total_a = s_offa[kTile];
  for (int e0 = 0; e0 < total_a; e0 += kThreads) {
    const int e = e0 + tid;
    if (e < total_a) {
      const int a = find_owner(s_offa, e);
      const int i = s_atom[a];
      const int t1 = s_type[a];
      const int j = nl_a[static_cast<size_t>(i) * mn_a + (e - s_offa[a])];
      const int t2 = __ldg(type + j);
      float dx, dy, dz;
      displacement(b, x, y, z, x[i], y[i], z[i], j, dx, dy, dz);
      const float d = sqrtf(dx * dx + dy * dy + dz * dz);
      const float rc = (p.rc_a[t1] + p.rc_a[t2]) * 0.5f;
      const float rcinv = 1.0f / rc;
      float fc, fcp;
      cutoff_fc(rc, rcinv, d, fc, fcp);
      float fn[kMaxBasis];
      radial_basis<kMaxBasis>(kA, rcinv, d, fc, fn);
      const float* c = s_c + p.num_c_radial + (t1 * T + t2) * nA * kA;
      float* row = s_buf + tid * se;
      for (int n = 0; n < nA; ++n) {
        float g = 0.0f;
#pragma unroll
        for (int k = 0; k < kMaxBasis; ++k)
          if (k < kA) g += fn[k] * c[n * kA + k];
        row[n] = g;
      }
      const float dinv = 1.0f / d;
      float Y[kNumLM];
      harmonics(p.L_max, dx * dinv, dy * dinv, dz * dinv, Y);
#pragma unroll
      for (int lm = 0; lm < kNumLM; ++lm)
        if (lm < nlm) row[nA + lm] = Y[lm];
    }
    __syncthreads();
    for (int own = tid; own < kTile * nA; own += kThreads) {
      const int a = own / nA, n = own % nA;
      const int lo = max(s_offa[a], e0), hi = min(s_offa[a + 1], e0 + kThreads);
      float acc[kNumLM];
#pragma unroll
      for (int lm = 0; lm < kNumLM; ++lm) acc[lm] = 0.0f;
      for (int e = lo; e < hi; ++e) {
        const float* row = s_buf + (e - e0) * se;
        const float g = row[n];
#pragma unroll
        for (int lm = 0; lm < kNumLM; ++lm)
          if (lm < nlm) acc[lm] += g * row[nA + lm];
      }
      float* srow = s_s + (a * nA + n) * kNumLM;
#pragma unroll
      for (int lm = 0; lm < kNumLM; ++lm)
        if (lm < nlm) srow[lm] += acc[lm];
    }
    __syncthreads();
  }

  // ---- invariants -> q, scaling ------------------------------------------
  for (int own = tid; own < kTile * nA; own += kThreads) {
    const int a = own / nA, n = own % nA;
    const float* s = s_s + (a * nA + n) * kNumLM;
    float* q = s_q + a * dim + nR;
    int col = 0;
    for (int Lq = 1; Lq <= p.L_max; ++Lq, ++col) {
      const int st = Lq * Lq - 1;
      float v = 0.0f;
      for (int k = 1; k < 2 * Lq + 1; ++k) v += c_C3B[st + k] * s[st + k] * s[st + k];
      v *= 2.0f;
      v += c_C3B[st] * s[st] * s[st];
      q[col * nA + n] = v;
    }
    for (int v = 0; v < p.num_inv; ++v, ++col) {
      const int id = p.inv_id[v];
      float acc = 0.0f;
      for (int m = c_inv_start[id]; m < c_inv_start[id + 1]; ++m) {
        const Monomial mo = c_mono[m];
        float t = mo.c * s[mo.i[0]] * s[mo.i[1]] * s[mo.i[2]];
        if (mo.i[3] >= 0) t *= s[mo.i[3]];
        acc += t;
      }
      q[col * nA + n] = acc;
    }
  }
  __syncthreads();
  for (int k = tid; k < kTile * dim; k += kThreads) s_q[k] *= __ldg(p.q_scaler + (k % dim));
  __syncthreads();

  // ---- ANN: hidden layer, site energy, dE/dq --------------------------------
  for (int own = tid; own < kTile * H; own += kThreads) {
    const int a = own / H, h = own % H;
    if (s_atom[a] < 0) continue;
    const int t = s_type[a];
    const float* w0 = p.w0 + (static_cast<size_t>(t) * H + h) * dim;
    const float* q = s_q + a * dim;
    float zsum = 0.0f;
    for (int d = 0; d < dim; ++d) zsum += __ldg(w0 + d) * q[d];
    const float x1 = tanhf(zsum - __ldg(p.b0 + t * H + h));
    const float w1 = __ldg(p.w1 + t * H + h);
    s_e[a * H + h] = w1 * x1;
    s_g[a * H + h] = w1 * (1.0f - x1 * x1);
  }
  __syncthreads();
  if (tid < kTile && s_atom[tid] >= 0) {
    float en = 0.0f;
    for (int h = 0; h < H; ++h) en += s_e[tid * H + h];
    en -= __ldg(p.out_bias + s_type[tid]);
    pe_ann[s_atom[tid]] = static_cast<double>(en);
  }
  for (int own = tid; own < kTile * dim; own += kThreads) {
    const int a = own / dim, d = own % dim;
    if (s_atom[a] < 0) continue;
    const int t = s_type[a];
    const float* w0 = p.w0 + static_cast<size_t>(t) * H * dim + d;
    const float* g = s_g + a * H;
    float acc = 0.0f;
    for (int h = 0; h < H; ++h) acc += g[h] * __ldg(w0 + static_cast<size_t>(h) * dim);
    acc *= __ldg(p.q_scaler + d);
    s_fp[own] = acc;
    if (d < nR) fp_rad[static_cast<size_t>(s_atom[a]) * nR + d] = acc;
  }
  __syncthreads();

  // ---- a[n][lm] = dE/ds[n][lm] ----------------------------------------------
  for (int own = tid; own < kTile * nA; own += kThreads) {
    const int a = own / nA, n = own % nA;
    const float* s = s_s + (a * nA + n) * kNumLM;
    float* av = s_a + (a * nA + n) * kNumLM;
    const float* fp = s_fp + a * dim + nR;
    for (int lm = 0; lm < kNumLM; ++lm) av[lm] = 0.0f;
    int col = 0;
    for (int Lq = 1; Lq <= p.L_max; ++Lq, ++col) {
      const int st = Lq * Lq - 1;
      const float f = fp[col * nA + n];
      av[st] = 2.0f * f * c_C3B[st] * s[st];
      for (int k = 1; k < 2 * Lq + 1; ++k) av[st + k] = 4.0f * f * c_C3B[st + k] * s[st + k];
    }
    for (int v = 0; v < p.num_inv; ++v, ++col) {
      const int id = p.inv_id[v];
      const float f = fp[col * nA + n];
      for (int m = c_inv_start[id]; m < c_inv_start[id + 1]; ++m) {
        const Monomial mo = c_mono[m];
        const int nf = mo.i[3] >= 0 ? 4 : 3;
        for (int q = 0; q < nf; ++q) {
          float t = f * mo.c;
          for (int r = 0; r < nf; ++r)
            if (r != q) t *= s[mo.i[r]];
          av[mo.i[q]] += t;
        }
      }
    }
  }
  __syncthreads();

  // ---- directed angular partial forces ---------------------------------------
  for (int e = tid; e < total_a; e += kThreads) {
    const int a = find_owner(s_offa, e);
    const int i = s_atom[a];
    const int t1 = s_type[a];
    const int k = e - s_offa[a];
    const int j = nl_a[static_cast<size_t>(i) * mn_a + k];
    const int t2 = __ldg(type + j);
    float dx, dy, dz;
    displacement(b, x, y, z, x[i], y[i], z[i], j, dx, dy, dz);
    const float d = sqrtf(dx * dx + dy * dy + dz * dz);
    const float dinv = 1.0f / d;
    const float ux = dx * dinv, uy = dy * dinv, uz = dz * dinv;
    const float rc = (p.rc_a[t1] + p.rc_a[t2]) * 0.5f;
    const float rcinv = 1.0f / rc;
    float fc, fcp;
    cutoff_fc(rc, rcinv, d, fc, fcp);
    float fn[kMaxBasis], fnp[kMaxBasis];
    radial_basis_d<kMaxBasis>(kA, rcinv, d, fc, fcp, fn, fnp);
    const float* c = s_c + p.num_c_radial + (t1 * T + t2) * nA * kA;
    float Acoef[kNumLM], Bcoef[kNumLM];
#pragma unroll
    for (int lm = 0; lm < kNumLM; ++lm) {
      Acoef[lm] = 0.0f;
      Bcoef[lm] = 0.0f;
    }
    for (int n = 0; n < nA; ++n) {
      float g = 0.0f, gp = 0.0f;
#pragma unroll
      for (int kk = 0; kk < kMaxBasis; ++kk)
        if (kk < kA) {
          const float cc = c[n * kA + kk];
          g += fn[kk] * cc;
          gp += fnp[kk] * cc;
        }
      const float* av = s_a + (a * nA + n) * kNumLM;
#pragma unroll
      for (int lm = 0; lm < kNumLM; ++lm)
        if (lm < nlm) {
          Acoef[lm] += av[lm] * g;
          Bcoef[lm] += av[lm] * gp;
        }
    }
    // walk the harmonics: SB = sum B Y, V = sum A dY/du (u components independent)
    float zp[5];
    zp[0] = 1.0f;
#pragma unroll
    for (int q = 1; q < 5; ++q) zp[q] = zp[q - 1] * uz;
    float SB = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
    int idx = 0;
#pragma unroll
    for (int Lq = 1; Lq <= 4; ++Lq) {
      if (Lq > p.L_max) break;
      float re0 = 1.0f, im0 = 0.0f;   // (ux + i uy)^(m-1)
#pragma unroll
      for (int m = 0; m <= Lq; ++m) {
        float dzf;
        const float zf = zpoly(Lq, m, zp, &dzf);
        if (m == 0) {
          SB += Bcoef[idx] * zf;
          vz += Acoef[idx] * dzf;
          ++idx;
        } else {
          const float re = ux * re0 - uy * im0;
          const float im = ux * im0 + uy * re0;
          const float Ar = Acoef[idx], Ai = Acoef[idx + 1];
          const float Br = Bcoef[idx], Bi = Bcoef[idx + 1];
          SB += (Br * re + Bi * im) * zf;
          const float mzf = m * zf;
          vx += mzf * (Ar * re0 + Ai * im0);
          vy += mzf * (Ai * re0 - Ar * im0);
          vz += dzf * (Ar * re + Ai * im);
          idx += 2;
          re0 = re;
          im0 = im;
        }
      }
    }
    const float uv = ux * vx + uy * vy + uz * vz;
    const float fx = SB * ux + (vx - uv * ux) * dinv;
    const float fy = SB * uy + (vy - uv * uy) * dinv;
    const float fz = SB * uz + (vz - uv * uz) * dinv;
    f12[static_cast<size_t>(i) * mn_a + k] = make_float4(fx, fy, fz, 0.0f);
  }
}

// ---------------------------------------------------------------------------
// gather
// ---------------------------------------------------------------------------

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

__global__ void __launch_bounds__(256)
k_gather(const ModelParams p, int N, const Box* __restrict__ box, const double* __restrict__ pos,
         const int* __restrict__ type, const int* __restrict__ nn_r, const int* __restrict__ nl_r,
         int mn_r, const int* __restrict__ nn_a, const int* __restrict__ nl_a, int mn_a,
         const float* __restrict__ fp_rad, const float4* __restrict__ f12,
         const double* __restrict__ pe_ann, double* __restrict__ pe, double* __restrict__ force,
         double* __restrict__ virial, int accumulate, NeighborState* st)
{
  extern __shared__ float s_c[];
  const int T = p.T, nR = p.nR, kR = p.kR;
  const int cR = T * T * nR * kR;
  for (int k = threadIdx.x; k < cR; k += blockDim.x) s_c[k] = __ldg(p.c_pair + k);
  __syncthreads();
  const int g = threadIdx.x % kGroup;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
  const bool active = i < N;
  const Box b = *box;
  const double* x = pos;
  const double* y = pos + N;
  const double* z = pos + 2 * N;
  float F[3] = {0.0f, 0.0f, 0.0f};
  float W[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float ezbl = 0.0f;
  if (active) {
    const double xi = x[i], yi = y[i], zi = z[i];
    const int t1 = type[i];
    float fpi[kMaxN];
#pragma unroll
    for (int n = 0; n < kMaxN; ++n) fpi[n] = n < nR ? fp_rad[static_cast<size_t>(i) * nR + n] : 0.0f;
    // radial pairs: dE_i/dr_ij and dE_j/dr_ji in one pass
    const int nr = nn_r[i];
    const int* rrow = nl_r + static_cast<size_t>(i) * mn_r;
    for (int k = g; k < nr; k += kGroup) {
      const int j = rrow[k];
      const int t2 = __ldg(type + j);
      float dx, dy, dz;
      displacement(b, x, y, z, xi, yi, zi, j, dx, dy, dz);
      const float d = sqrtf(dx * dx + dy * dy + dz * dz);
      const float dinv = 1.0f / d;
      const float rc = (p.rc_r[t1] + p.rc_r[t2]) * 0.5f;
      const float rcinv = 1.0f / rc;
      float fc, fcp;
      cutoff_fc(rc, rcinv, d, fc, fcp);
      float fn[kMaxBasis], fnp[kMaxBasis];
      radial_basis_d<kMaxBasis>(kR, rcinv, d, fc, fcp, fn, fnp);
      const float* c12 = s_c + (t1 * T + t2) * nR * kR;
      const float* c21 = s_c + (t2 * T + t1) * nR * kR;
      const float* fpj = fp_rad + static_cast<size_t>(j) * nR;
      float w12 = 0.0f, w21 = 0.0f;
      for (int n = 0; n < nR; ++n) {
        float gp12 = 0.0f, gp21 = 0.0f;
#pragma unroll
        for (int kk = 0; kk < kMaxBasis; ++kk)
          if (kk < kR) {
            gp12 += fnp[kk] * c12[n * kR + kk];
            gp21 += fnp[kk] * c21[n * kR + kk];
          }
        w12 += fpi[n] * gp12;
        w21 += __ldg(fpj + n) * gp21;
      }
      const float r[3] = {dx, dy, dz};
      const float s12 = w12 * dinv, s21 = w21 * dinv;
      // f12 = s12 r, f21 = -s21 r; F += f12 - f21; W += r (x) f21
      F[0] += (s12 + s21) * dx;
      F[1] += (s12 + s21) * dy;
      F[2] += (s12 + s21) * dz;
      const float f21[3] = {-s21 * dx, -s21 * dy, -s21 * dz};
      W[0] += r[0] * f21[0];
      W[1] += r[1] * f21[1];
      W[2] += r[2] * f21[2];
      W[3] += r[0] * f21[1];
      W[4] += r[0] * f21[2];
      W[5] += r[1] * f21[2];
      W[6] += r[1] * f21[0];
      W[7] += r[2] * f21[0];
      W[8] += r[2] * f21[1];
    }
    // angular exchange and ZBL
    const int na = nn_a[i];
    const int* arow = nl_a + static_cast<size_t>(i) * mn_a;
    const int zi_ = p.Z[t1];
    const float pow_zi = powf(static_cast<float>(zi_), 0.23f);
    for (int k = g; k < na; k += kGroup) {
      const int j = arow[k];
      float dx, dy, dz;
      displacement(b, x, y, z, xi, yi, zi, j, dx, dy, dz);
      const float4 a12 = f12[static_cast<size_t>(i) * mn_a + k];
      // reverse slot: i inside j's ascending row
      const int* jrow = nl_a + static_cast<size_t>(j) * mn_a;
      int lo = 0, hi = nn_a[j] - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(jrow + mid) < i) lo = mid + 1; else hi = mid;
      }
      float4 a21 = f12[static_cast<size_t>(j) * mn_a + lo];
      if (nn_a[j] == 0 || __ldg(jrow + lo) != i) {
        // only a truncated (overflowed) row can lose the reverse edge
        a21 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        atomicOr(&st->overflow, 4);
      }
      F[0] += a12.x - a21.x;
      F[1] += a12.y - a21.y;
      F[2] += a12.z - a21.z;
      W[0] += dx * a21.x;
      W[1] += dy * a21.y;
      W[2] += dz * a21.z;
      W[3] += dx * a21.y;
      W[4] += dx * a21.z;
      W[5] += dy * a21.z;
      W[6] += dy * a21.x;
      W[7] += dz * a21.x;
      W[8] += dz * a21.y;
      if (p.zbl) {
        const int t2 = __ldg(type + j);
        const float d = sqrtf(dx * dx + dy * dy + dz * dz);
        const float dinv = 1.0f / d;
        const int zj = p.Z[t2];
        const float a_inv = (pow_zi + powf(static_cast<float>(zj), 0.23f)) * 2.134563f;
        const float zizj = kCoulomb * zi_ * zj;
        float f, fpz;
        if (p.zbl_flexible) {
          const int ta = min(t1, t2), tb = max(t1, t2);
          const int idx = ta * p.T - (ta * (ta - 1)) / 2 + (tb - ta);
          float zpar[10];
#pragma unroll
          for (int q = 0; q < 10; ++q) zpar[q] = __ldg(p.zbl_para + 10 * idx + q);
          zbl_flexible(zpar, zizj, a_inv, d, dinv, f, fpz);
        } else {
          float r1 = p.zbl_rc_inner, r2 = p.zbl_rc_outer;
          if (p.typewise_zbl) {
            r2 = fminf((c_covalent[zi_ - 1] + c_covalent[zj - 1]) * p.typewise_factor, r2);
            r1 = 0.0f;
          }
          zbl_universal(zizj, a_inv, r1, r2, d, dinv, f, fpz);
        }
        const float f2 = fpz * dinv * 0.5f;
        const float h12[3] = {dx * f2, dy * f2, dz * f2};
        F[0] += 2.0f * h12[0];
        F[1] += 2.0f * h12[1];
        F[2] += 2.0f * h12[2];
        W[0] -= dx * h12[0];
        W[1] -= dy * h12[1];
        W[2] -= dz * h12[2];
        W[3] -= dx * h12[1];
        W[4] -= dx * h12[2];
        W[5] -= dy * h12[2];
        W[6] -= dy * h12[0];
        W[7] -= dz * h12[0];
        W[8] -= dz * h12[1];
        ezbl += 0.5f * f;
      }
    }
  }
  // reduce the group
#pragma unroll
  for (int off = kGroup / 2; off > 0; off >>= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) F[c] += __shfl_xor_sync(0xffffffffu, F[c], off);
#pragma unroll
    for (int c = 0; c < 9; ++c) W[c] += __shfl_xor_sync(0xffffffffu, W[c], off);
    ezbl += __shfl_xor_sync(0xffffffffu, ezbl, off);
  }
  if (active && g == 0) {
    const double e = pe_ann[i] + static_cast<double>(ezbl);
    bool finite = isfinite(e) && isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]);
    if (accumulate) {
      pe[i] += e;
      for (int c = 0; c < 3; ++c) force[static_cast<size_t>(c) * N + i] += F[c];
      for (int c = 0; c < 9; ++c) virial[static_cast<size_t>(c) * N + i] += W[c];
    } else {
      pe[i] = e;
      for (int c = 0; c < 3; ++c) force[static_cast<size_t>(c) * N + i] = F[c];
      for (int c = 0; c < 9; ++c) virial[static_cast<size_t>(c) * N + i] = W[c];
    }
    if (!finite) st->nonfinite = 1;
  }
}

}  // namespace

// Monomial tables of the many-body invariants, uploaded once per process.
void upload_invariant_tables()
{
  static bool done = false;
  if (done) return;
  struct M {
    float c;
    int a, b, cc, d;
  };
  const float C4B[5] = {-0.007499480826664f, -0.134990654879954f, 0.067495327439977f,
                        0.404971964639861f, -0.809943929279723f};
  const float C5B[3] = {0.026596810706114f, 0.053193621412227f, 0.026596810706114f};
  const float C4B2[5] = {0.027493550848847f, 0.164961305093080f, -0.013746775424423f,
                         0.041240326273270f, 0.082480652546540f};
  const float C123[7] = {-0.008418146349617f, -0.016836292699234f, -0.033672585398469f,
                         -0.042090731748086f, -0.067345170796937f, -0.084181463496172f,
                         -0.168362926992344f};
  const float C233[10] = {0.008572620635186f, 0.009644198214584f, 0.019288396429168f,
                          0.025717861905558f, 0.026789439484956f, 0.032147327381947f,
                          0.038576792858337f, 0.128589309527790f, 0.192883964291685f,
                          0.321473273819474f};
  const float C134[10] = {0.003645164295772f, 0.004860219061029f, 0.006075273826286f,
                          0.018225821478859f, 0.024301095305146f, 0.036451642957719f,
                          0.042526916784005f, 0.072903285915437f, 0.085053833568010f,
                          0.255161500704030f};
  const M q222[] = {{C4B[0], 3, 3, 3, -1}, {C4B[1], 3, 4, 4, -1}, {C4B[1], 3, 5, 5, -1},
                    {C4B[2], 3, 6, 6, -1}, {C4B[2], 3, 7, 7, -1}, {C4B[3], 6, 5, 5, -1},
                    {-C4B[3], 6, 4, 4, -1}, {C4B[4], 4, 5, 7, -1}};
  const M q1111[] = {{C5B[0], 0, 0, 0, 0}, {C5B[1], 0, 0, 1, 1}, {C5B[1], 0, 0, 2, 2},
                     {C5B[2], 1, 1, 1, 1}, {2.0f * C5B[2], 1, 1, 2, 2}, {C5B[2], 2, 2, 2, 2}};
  const M q112[] = {{C4B2[0], 0, 0, 3, -1}, {C4B2[1], 0, 1, 4, -1}, {C4B2[1], 0, 2, 5, -1},
                    {C4B2[2], 3, 1, 1, -1}, {C4B2[2], 3, 2, 2, -1}, {C4B2[3], 6, 1, 1, -1},
                    {-C4B2[3], 6, 2, 2, -1}, {C4B2[4], 1, 2, 7, -1}};
  const M q123[] = {{C123[6], 12, 2, 4, -1}, {-C123[6], 11, 2, 5, -1}, {C123[6], 1, 11, 4, -1},
                    {C123[6], 1, 12, 5, -1}, {C123[5], 0, 11, 6, -1},  {C123[5], 0, 12, 7, -1},
                    {C123[3], 14, 2, 6, -1}, {-C123[3], 13, 2, 7, -1}, {C123[3], 1, 13, 6, -1},
                    {C123[3], 1, 14, 7, -1}, {C123[4], 10, 0, 5, -1},  {C123[4], 0, 4, 9, -1},
                    {C123[1], 10, 2, 3, -1}, {C123[1], 0, 3, 8, -1},   {C123[1], 1, 3, 9, -1},
                    {C123[0], 10, 2, 6, -1}, {-C123[0], 10, 1, 7, -1}, {-C123[0], 2, 7, 9, -1},
                    {-C123[0], 1, 6, 9, -1}, {-C123[2], 2, 5, 8, -1},  {-C123[2], 1, 4, 8, -1}};
  const M q233[] = {{C233[0], 3, 8, 8, -1},    {C233[1], 10, 10, 3, -1},  {C233[1], 3, 9, 9, -1},
                    {-C233[2], 10, 10, 6, -1}, {C233[2], 6, 9, 9, -1},    {C233[3], 4, 8, 9, -1},
                    {C233[3], 10, 5, 8, -1},   {-C233[4], 13, 13, 3, -1}, {-C233[4], 14, 14, 3, -1},
                    {-C233[5], 14, 7, 9, -1},  {-C233[5], 13, 6, 9, -1},  {-C233[5], 10, 14, 6, -1},
                    {C233[5], 10, 13, 7, -1},  {C233[6], 10, 7, 9, -1},   {-C233[7], 11, 6, 8, -1},
                    {-C233[7], 12, 7, 8, -1},  {C233[8], 11, 4, 9, -1},   {C233[8], 12, 5, 9, -1},
                    {C233[8], 10, 12, 4, -1},  {-C233[8], 10, 11, 5, -1}, {C233[9], 12, 14, 4, -1},
                    {C233[9], 11, 14, 5, -1},  {C233[9], 13, 11, 4, -1},  {-C233[9], 13, 12, 5, -1}};
  const M q134[] = {{-C134[0], 10, 15, 2, -1}, {-C134[0], 1, 15, 9, -1},  {C134[1], 0, 15, 8, -1},
                    {-C134[2], 1, 13, 18, -1}, {-C134[2], 1, 14, 19, -1}, {-C134[2], 2, 14, 18, -1},
                    {C134[2], 2, 13, 19, -1},  {-C134[3], 10, 18, 2, -1}, {C134[3], 1, 10, 19, -1},
                    {C134[3], 1, 18, 9, -1},   {C134[3], 2, 19, 9, -1},   {C134[4], 1, 16, 8, -1},
                    {C134[4], 2, 17, 8, -1},   {C134[5], 0, 10, 17, -1},  {C134[5], 0, 16, 9, -1},
                    {-C134[5], 1, 11, 16, -1}, {-C134[5], 1, 12, 17, -1}, {-C134[5], 2, 12, 16, -1},
                    {C134[5], 2, 11, 17, -1},  {C134[6], 1, 13, 22, -1},  {C134[6], 1, 14, 23, -1},
                    {-C134[6], 2, 14, 22, -1}, {C134[6], 2, 13, 23, -1},  {C134[7], 0, 11, 18, -1},
                    {C134[7], 0, 12, 19, -1},  {C134[8], 0, 13, 20, -1},  {C134[8], 0, 14, 21, -1},
                    {C134[9], 1, 11, 20, -1},  {C134[9], 1, 12, 21, -1},  {-C134[9], 2, 12, 20, -1},
                    {C134[9], 2, 11, 21, -1}};
  const M* tabs[kMaxInv] = {q222, q1111, q112, q123, q233, q134};
  const int counts[kMaxInv] = {8, 6, 8, 21, 24, 31};
  Monomial host[128];
  int start[kMaxInv + 1];
  int k = 0;
  for (int v = 0; v < kMaxInv; ++v) {
    start[v] = k;
    for (int m = 0; m < counts[v]; ++m, ++k) {
      host[k].c = tabs[v][m].c;
      host[k].i[0] = static_cast<signed char>(tabs[v][m].a);
      host[k].i[1] = static_cast<signed char>(tabs[v][m].b);
      host[k].i[2] = static_cast<signed char>(tabs[v][m].cc);
      host[k].i[3] = static_cast<signed char>(tabs[v][m].d);
    }
  }
  start[kMaxInv] = k;
  cudaMemcpyToSymbol(c_mono, host, sizeof(Monomial) * k);
  cudaMemcpyToSymbol(c_inv_start, start, sizeof(start));
  done = true;
}

size_t descriptor_smem_bytes(const ModelParams& p) { return desc_layout(p).total_bytes; }

void launch_descriptor(Engine& e, int N, const double* pos, const int* type, cudaStream_t stream)
{
  const ModelParams& p = e.params;
  NeighborBuffers& nb = e.nbr;
  const int tiles = (N + kTile - 1) / kTile;
  k_descriptor_ann_f12<<<tiles, kThreads, e.smem_desc, stream>>>(
    p, N, e.d_box, pos, type, nb.nn_r, nb.nl_r, nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a,
    e.scratch.fp_rad, e.scratch.f12, e.scratch.pe_ann);
}

void launch_gather(Engine& e, int N, const double* pos, const int* type, double* pe,
                   double* force, double* virial, bool accumulate, cudaStream_t stream)
{
  const ModelParams& p = e.params;
  NeighborBuffers& nb = e.nbr;
  const int threads = 256;
  const size_t smem_g = static_cast<size_t>(p.T) * p.T * p.nR * p.kR * sizeof(float);
  const int blocks = static_cast<int>((static_cast<long long>(N) * kGroup + threads - 1) / threads);
  k_gather<<<blocks, threads, smem_g, stream>>>(
    p, N, e.d_box, pos, type, nb.nn_r, nb.nl_r, nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a,
    e.scratch.fp_rad, e.scratch.f12, e.scratch.pe_ann, pe, force, virial, accumulate ? 1 : 0,
    e.d_nstate);
}

void launch_force(Engine& e, int N, const double* pos, const int* type, double* pe,
                  double* force, double* virial, bool accumulate, cudaStream_t stream)
{
  launch_descriptor(e, N, pos, type, stream);
  launch_gather(e, N, pos, type, pe, force, virial, accumulate, stream);
}

void set_descriptor_smem_limit(size_t bytes)
{
  cudaFuncSetAttribute(k_descriptor_ann_f12, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(bytes));
}

}  // namespace nepx

// nep_force.cu -- NEP energy, force and virial on sm_100a.
//
// Four kernels per force call, each giving a group of G lanes (G = 4 or 8,
// chosen by the autotuner in engine.cu) to one center; every phase is local
// to the group, so no CTA-wide barrier follows the set-up (except in the
// tensor-core ANN, whose MMAs span the CTA's centers).
//
//  k_filter_radial  one sweep over the center's sorted Verlet row applies the
//    reference's FP32 typewise predicate (nep.cu:503-561), writes the radial
//    and angular rows in order (group ballot + popcount) and sums the radial
//    descriptors q_n = sum_j sum_k c(ti,tj)[n][k] f_k(d_ij) through per-type
//    bins of the basis values.
//  k_nep_fused  (descriptors + ANN)
//    1. the radial descriptors (explicit rows: evaluated here);
//    2. a sweep over the dense angular row accumulates the moments
//       s[n][lm] = sum_j g_n(d_ij) Y_lm(r_ij/d) in registers; a register
//       reduce-scatter across the group lands each lane's share in shared
//       memory;
//    3. per center: invariants q_L and q_222/q_1111/q_112/q_123/q_233/q_134,
//       the one-hidden-layer ANN (site energy, dE/dq), the moment derivatives
//       a[n][lm] = dE/ds[n][lm], and the radial force coefficients
//       alpha[t][k] = sum_n dE/dq_n c(ti,t)[n][k] (stored for the gather).
//    Mixed precision runs the ANN of the CTA's centers as two tcgen05 MMAs
//    (16-bit operands, FP32 accumulators in TMEM, tc_ann) in place of the
//    per-center FP32 contraction.  Reference: find_descriptor (nep.cu:569-748).
//  k_angular_f12  each directed partial force
//       f12(i,j) = (sum_lm B_lm Y_lm) r^ + (1/d)(I - r^r^T) sum_lm A_lm dY_lm/dr^
//    with A_lm = sum_n a[n][lm] g_n and B_lm = sum_n a[n][lm] g'_n: the
//    harmonic ladder runs once per edge, not once per (edge, n) as in
//    accumulate_f12 (nep_utilities.cuh:1240-1491).  Reference:
//    find_partial_force_angular (nep.cu:890-991).
//  k_gather  radial pair force from both site energies with the per-atom
//    alpha coefficients (w_ij = sum_k f'_k(d) alpha_i[tj][k]), the angular
//    exchange F_i += f12(i,j) - f12(j,i) with the reverse slot found by binary
//    search in j's sorted row (explicit rows: both directed forces evaluated
//    here), ZBL, and the per-atom virial W_i = sum_j r_ij (x) f_ji.
//    Reference: find_force_radial (nep.cu:756-881), gpu_find_force_many_body
//    (potential.cu:81-210), find_force_ZBL (nep.cu:996-1111).
//
// Harmonic degree: instances for l_max <= 4 (24 moment components per n) and
// l_max 5..8 (80 components).
#include <cstdio>
#include <mutex>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <utility>

#include "engine.h"
#include "harmonic_tables.h"
#include "invariants.h"
#include "tcgen05.cuh"

namespace nepx {

namespace {

constexpr int kBlock = 128;      // threads per CTA
constexpr int kChunkN = 5;       // radial functions per angular-moment sweep (3 CTAs per SM)
constexpr int kChunkN4 = 3;      // the same at 4 CTAs per SM (fewer live accumulators)
constexpr unsigned kFull = 0xffffffffu;

// Weights of the three-body invariants q_L and coefficients of the
// z-polynomials of the harmonics, degrees 1..8 (harmonic_tables.h; the
// reference's C3B and Z_COEFFICIENT_L tables, nep_utilities.cuh:51-187).
__constant__ float c_C3B[kNumLMHigh];
__constant__ float c_Zc[kHarmonicLMax + 1][kHarmonicLMax + 1][kHarmonicLMax + 1];

template <int LMAX>
__host__ __device__ constexpr int num_lm() { return (LMAX + 1) * (LMAX + 1) - 1; }

// Z_Lm(z) and dZ_Lm/dz with zp[k] = z^k; degrees above 4 from c_Zc.
__device__ __forceinline__ float zpoly_any(int L, int m, const float* zp, float* dzf)
{
  if (L <= 4) return zpoly(L, m, zp, dzf);
  float f = 0.0f, df = 0.0f;
#pragma unroll
  for (int k = 0; k <= kHarmonicLMax; ++k) {
    if (k <= L - m && ((L - m - k) & 1) == 0) {
      const float c = c_Zc[L][m][k];
      f += c * zp[k];
      if (k > 0) df += c * static_cast<float>(k) * zp[k - 1];
    }
  }
  *dzf = df;
  return f;
}

// Harmonics Y[lm], lm < (L_max + 1)^2 - 1, at the unit vector u, degrees up
// to LMAX (the instance's bound) and L_max (the model's), handed one at a
// time to f(lm, Y[lm]) with lm a compile-time index once unrolled (no array
// of all harmonics stays live).
template <int LMAX, typename F>
__device__ __forceinline__ void for_each_harmonic(int L_max, float ux, float uy, float uz, F&& f)
{
  float zp[LMAX + 1];
  zp[0] = 1.0f;
#pragma unroll
  for (int k = 1; k <= LMAX; ++k) zp[k] = zp[k - 1] * uz;
  int idx = 0;
#pragma unroll
  for (int L = 1; L <= LMAX; ++L) {
    if (L > L_max) break;
    float re = ux, im = uy;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      float dzf;
      const float zf = zpoly_any(L, m, zp, &dzf);
      if (m == 0) {
        f(idx++, zf);
      } else {
        f(idx++, zf * re);
        f(idx++, zf * im);
        const float r2 = ux * re - uy * im;
        im = ux * im + uy * re;
        re = r2;
      }
    }
  }
}

// Many-body invariants as monomials c * s[i0] s[i1] s[i2] (s[i3]) of the raw
// moments, transcribed from the polynomials of find_q
// (nep_utilities.cuh:1661-1728).  c_inv_start[v] .. c_inv_start[v+1] are the
// monomials of invariant v.
struct Monomial {
  float c;
  signed char i[4];
};
__constant__ Monomial c_mono[128];
__constant__ int c_inv_start[kMaxInv + 1];

// The same invariants for degrees <= 4 in registers: the monomial list of
// invariant ID (invariants.h) unrolled at compile time, so s and the
// derivatives a are register arrays of the 24 moment components of one n.
// Value: sum over monomials of c s[i0] s[i1] s[i2] (s[i3]), in list order.
template <int ID, int M>
__device__ __forceinline__ float inv_term(const float (&s)[kNumLM])
{
  constexpr InvMono mo = inv_mono(ID, M);
  float t = mo.c * s[mo.a] * s[mo.b] * s[mo.cc];
  if constexpr (mo.d >= 0) t *= s[mo.d];
  return t;
}

template <int ID, int... M>
__device__ __forceinline__ float inv_value(const float (&s)[kNumLM],
                                           std::integer_sequence<int, M...>)
{
  float acc = 0.0f;
  ((acc += inv_term<ID, M>(s)), ...);
  return acc;
}

template <int I>
__device__ __forceinline__ float inv_value_of(const float (&s)[kNumLM])
{
  return inv_value<I>(s, std::make_integer_sequence<int, inv_count(I)>{});
}

// Derivative terms: for every factor Q of monomial M, f c times the other
// factors in list order, added to a[factor Q].
template <int ID, int M, int Q, int R>
__device__ __forceinline__ float inv_grad_prod(const float (&s)[kNumLM], float t)
{
  constexpr InvMono mo = inv_mono(ID, M);
  constexpr int nf = mo.d >= 0 ? 4 : 3;
  if constexpr (R >= nf) {
    return t;
  } else {
    constexpr int i = R == 0 ? mo.a : R == 1 ? mo.b : R == 2 ? mo.cc : mo.d;
    if constexpr (R != Q) t *= s[i];
    return inv_grad_prod<ID, M, Q, R + 1>(s, t);
  }
}

template <int ID, int M, int Q>
__device__ __forceinline__ void inv_grad_factor(const float (&s)[kNumLM], float (&a)[kNumLM],
                                                float f)
{
  constexpr InvMono mo = inv_mono(ID, M);
  constexpr int nf = mo.d >= 0 ? 4 : 3;
  if constexpr (Q < nf) {
    constexpr int i = Q == 0 ? mo.a : Q == 1 ? mo.b : Q == 2 ? mo.cc : mo.d;
    a[i] += inv_grad_prod<ID, M, Q, 0>(s, f * mo.c);
    inv_grad_factor<ID, M, Q + 1>(s, a, f);
  }
}

template <int ID, int... M>
__device__ __forceinline__ void inv_grad(const float (&s)[kNumLM], float (&a)[kNumLM], float f,
                                         std::integer_sequence<int, M...>)
{
  (inv_grad_factor<ID, M, 0>(s, a, f), ...);
}

template <int I>
__device__ __forceinline__ void inv_grad_of(const float (&s)[kNumLM], float (&a)[kNumLM], float f)
{
  inv_grad<I>(s, a, f, std::make_integer_sequence<int, inv_count(I)>{});
}

// runtime invariant id -> its unrolled form
__device__ __forceinline__ float inv_value_id(int id, const float (&s)[kNumLM])
{
  switch (id) {
    case 0: return inv_value_of<0>(s);
    case 1: return inv_value_of<1>(s);
    case 2: return inv_value_of<2>(s);
    case 3: return inv_value_of<3>(s);
    case 4: return inv_value_of<4>(s);
    default: return inv_value_of<5>(s);
  }
}

__device__ __forceinline__ void inv_grad_id(int id, const float (&s)[kNumLM], float (&a)[kNumLM],
                                            float f)
{
  switch (id) {
    case 0: inv_grad_of<0>(s, a, f); break;
    case 1: inv_grad_of<1>(s, a, f); break;
    case 2: inv_grad_of<2>(s, a, f); break;
    case 3: inv_grad_of<3>(s, a, f); break;
    case 4: inv_grad_of<4>(s, a, f); break;
    default: inv_grad_of<5>(s, a, f); break;
  }
}

// The 24 moments of one n from shared memory (16-byte aligned) and back.
__device__ __forceinline__ void load24(const float* src, float (&v)[kNumLM])
{
#pragma unroll
  for (int q = 0; q < kNumLM / 4; ++q) {
    const float4 x = reinterpret_cast<const float4*>(src)[q];
    v[4 * q] = x.x;
    v[4 * q + 1] = x.y;
    v[4 * q + 2] = x.z;
    v[4 * q + 3] = x.w;
  }
}

__device__ __forceinline__ void store24(float* dst, const float (&v)[kNumLM])
{
#pragma unroll
  for (int q = 0; q < kNumLM / 4; ++q)
    reinterpret_cast<float4*>(dst)[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2],
                                                    v[4 * q + 3]);
}

#include "zbl.cuh"

__host__ __device__ constexpr int round4(int x) { return (x + 3) & ~3; }

// Asynchronous copy of one 32-byte Site record into shared memory (two 16-byte
// cp.async, cached in L1 like the plain loads they replace): a lane fetches
// the next neighbour's site while it works on the current one, without
// holding the record in registers.  Sites are 32-byte aligned (cudaMalloc
// base, 32-byte records), the destination 16-byte aligned.
__device__ __forceinline__ void site_fetch_async(unsigned dst, const Site* src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(dst + 16u),
               "l"(reinterpret_cast<const char*>(src) + 16)
               : "memory");
}
__device__ __forceinline__ void async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// all but the most recent group of this thread's copies have landed
__device__ __forceinline__ void async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared-memory layout of k_nep_fused (in floats; the tensor-core region in bytes).
struct FusedLayout {
  int kpr, kpa;        // basis sizes padded to float4
  int c_rad, c_ang;    // coefficient tables [T*T][n][kp]
  int wt;              // transposed ANN weights [T][dim][H4], or -1: read from global
  int per_atom;        // floats of per-center scratch
  int s, a, q, fp, gh; // offsets inside one center's scratch
  int atoms_base;      // offset of the per-center scratch
  int total_bytes;
  // tensor-core ANN (byte offsets from the start): 16-bit tiles of one chunk
  // of 128 stacked hidden units, W0 [128][dimk] and W0^T [dim][128], the CTA's
  // descriptors [APB][dimk] and hidden-layer derivatives [APB][128]; energy
  // partials [4][APB]; per type, the bit mask of the CTA's centers of that
  // type [kMaxTypes]; the mbarrier, the TMEM address and a flag
  int tc_w, tc_wt, tc_q, tc_g, tc_e, tc_type, tc_bar, tc_misc;
  // site prefetch slots of the angular sweep, two 32-byte records per thread
  // (offset in floats), or -1
  int pf;
};

// The descriptor builds that prefetch neighbour sites through shared memory:
// the Verlet-row path at three or fewer CTAs per SM (the four-CTA build has no
// shared memory to spare; explicit rows carry their displacements already).
__host__ __device__ constexpr bool fused_prefetch(bool xr, int minb) { return !xr && minb <= 3; }

// Shared memory one CTA may use with the ANN weights staged, when `minb`
// CTAs share an SM (228 KB per SM, 1 KB of it reserved per CTA).
__host__ __device__ constexpr int fused_smem_budget(int minb) { return 228 * 1024 / minb - 1024; }

// kp: row stride of the coefficient tables, the padded basis size of the
// kernel instance (rows are zero-filled up to it, so float4 dot products of
// the full compile-time width stay inside the row).
// tc: the layout of the tensor-core ANN build (16-bit tiles first, no FP32
// weights staged, no per-center hidden-unit scratch).  An MMA reads 128 rows
// of its A tile: rows past the stacked hidden units (or dim) are read from
// whatever follows in shared memory and only feed accumulator rows the
// epilogue never reads, so total_bytes covers the 128-row span of both A tiles.
// prefetch: room for the site prefetch slots at the end (fused_prefetch).
__host__ __device__ inline FusedLayout fused_layout(const ModelParams& p, int atoms_per_block,
                                                   int kp, int budget, bool tc = false,
                                                   bool prefetch = false)
{
  FusedLayout L;
  L.kpr = kp;
  L.kpa = kp;
  const int tt = p.T * p.T;
  int base = 0;   // floats before the tables
  if (tc) {
    auto up128 = [](int x) { return (x + 127) & ~127; };
    const int dimk = p.tc_dimk, th = p.T * p.H;
    const int rows = ((th < 128 ? th : 128) + 7) & ~7;
    L.tc_w = 0;
    L.tc_wt = up128(L.tc_w + rows * dimk * 2);
    L.tc_q = up128(L.tc_wt + ((p.dim + 7) & ~7) * 128 * 2);
    L.tc_g = up128(L.tc_q + atoms_per_block * dimk * 2);
    L.tc_e = up128(L.tc_g + atoms_per_block * 128 * 2);
    L.tc_type = L.tc_e + 4 * atoms_per_block * 4;
    L.tc_bar = (L.tc_type + kMaxTypes * 4 + 7) & ~7;
    L.tc_misc = L.tc_bar + 8;
    base = up128(L.tc_misc + 16) / 4;
  } else {
    L.tc_w = L.tc_wt = L.tc_q = L.tc_g = L.tc_e = L.tc_type = L.tc_bar = L.tc_misc = -1;
  }
  L.c_rad = base;
  L.c_ang = L.c_rad + tt * p.nR * L.kpr;
  L.s = 0;
  L.a = p.nA * p.nlm;
  L.q = 2 * p.nA * p.nlm;
  L.fp = L.q + round4(p.dim);
  L.gh = L.fp + round4(p.dim);
  // per-center stride: 16-byte aligned (float4 reads of the a[n][lm] rows)
  // and an odd number of 16-byte units, so float4 rows of neighbouring
  // centers start on different banks
  L.per_atom = round4(L.gh + (tc ? 0 : p.H));
  if ((L.per_atom / 4) % 2 == 0) L.per_atom += 4;
  const int tables = round4(L.c_ang + tt * p.nA * L.kpa);
  const int wsize = p.T * p.dim * p.H4;
  L.wt = tables;
  L.atoms_base = tables + wsize;
  L.total_bytes = 4 * (L.atoms_base + atoms_per_block * L.per_atom);
  const int pf_bytes = prefetch ? 2 * 32 * kBlock : 0;
  if (tc || L.total_bytes + pf_bytes > budget) {   // weights stay in global memory
    L.wt = -1;
    L.atoms_base = tables;
    L.total_bytes = 4 * (L.atoms_base + atoms_per_block * L.per_atom);
  }
  if (tc) {
    const int need_w = L.tc_w + 128 * p.tc_dimk * 2, need_wt = L.tc_wt + 128 * 128 * 2;
    L.total_bytes = (L.total_bytes > need_w ? L.total_bytes : need_w);
    L.total_bytes = (L.total_bytes > need_wt ? L.total_bytes : need_wt);
    L.total_bytes = (L.total_bytes + 15) & ~15;
  }
  L.pf = -1;
  if (prefetch) {
    L.pf = (L.total_bytes + 15) / 16 * 4;
    L.total_bytes = 4 * L.pf + pf_bytes;
  }
  return L;
}

// Cutoff of a type pair and its reciprocal: which 0 radial, 1 angular.  The
// exact builds read both from ModelParams::pair_cut (the correctly rounded
// reciprocal without a division per edge); the FAST builds form them from
// the per-type cutoffs with the hardware reciprocal, which costs less than
// the two loads.
template <bool FAST>
__device__ __forceinline__ void pair_cutoff(const ModelParams& p, int which, int t1, int t2,
                                            float& rc, float& rcinv)
{
  if constexpr (FAST) {
    rc = which == 0 ? (p.rc_r[t1] + p.rc_r[t2]) * 0.5f : (p.rc_a[t1] + p.rc_a[t2]) * 0.5f;
    rcinv = __fdividef(1.0f, rc);
  } else {
    const int tt = p.T * p.T, k = t1 * p.T + t2;
    rc = __ldg(p.pair_cut + 2 * which * tt + k);
    rcinv = __ldg(p.pair_cut + (2 * which + 1) * tt + k);
  }
}

// f[k] . c[k] over KM basis values with float4 loads of a padded row.
template <int KM>
__device__ __forceinline__ float dot_basis(const float* __restrict__ c, const float* f)
{
  float acc = 0.0f;
#pragma unroll
  for (int q = 0; q < (KM + 3) / 4; ++q) {
    const float4 cv = *reinterpret_cast<const float4*>(c + 4 * q);
    acc += cv.x * f[4 * q] + cv.y * f[4 * q + 1] + cv.z * f[4 * q + 2] + cv.w * f[4 * q + 3];
  }
  return acc;
}

// Shared memory of k_filter_radial: the coefficient table, then per-lane
// type bins of the basis sums when T * kp <= kFilterBinMax floats.
constexpr int kFilterBinMax = 48;
__host__ __device__ inline int filter_table_floats(const ModelParams& p, int kp)
{
  return round4(p.T * p.T * p.nR * kp);
}
__host__ __device__ inline int filter_bin_float4(const ModelParams& p, int kp)
{
  const int q = p.T * kp / 4;
  return q | 1;
}
__host__ __device__ inline bool filter_bins(const ModelParams& p, int kp)
{
  return p.T * kp <= kFilterBinMax;
}

// group ballot: the bits of the G lanes of this lane's group
template <int G>
__device__ __forceinline__ unsigned group_ballot(bool pred, int group)
{
  const unsigned b = __ballot_sync(kFull, pred);
  return (b >> (group * G)) & ((1u << G) - 1u);
}

template <int G>
__device__ __forceinline__ float group_sum(float v)
{
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Reduce-scatter of L values across the G lanes of a group: afterwards lane
// gl holds the group sums of v[base .. base + L/G) in v[0 .. L/G).
template <int L, int O>
__device__ __forceinline__ void rs_step(float* v, int gl, int& base)
{
  constexpr int half = L / 2;
  const bool hi = (gl & O) != 0;
#pragma unroll
  for (int i = 0; i < half; ++i) {
    const float send = hi ? v[i] : v[i + half];
    const float keep = hi ? v[i + half] : v[i];
    v[i] = keep + __shfl_xor_sync(kFull, send, O);
  }
  if (hi) base += half;
}

template <int G, int L>
__device__ __forceinline__ int reduce_scatter(float* v, int gl)
{
  static_assert(G == 2 || G == 4 || G == 8, "group of 2, 4 or 8 lanes");
  static_assert(L % G == 0, "share must divide evenly");
  int base = 0;
  if constexpr (G == 8) {
    rs_step<L, 4>(v, gl, base);
    rs_step<L / 2, 2>(v, gl, base);
    rs_step<L / 4, 1>(v, gl, base);
  } else if constexpr (G == 4) {
    rs_step<L, 2>(v, gl, base);
    rs_step<L / 2, 1>(v, gl, base);
  } else {
    rs_step<L, 1>(v, gl, base);
  }
  return base;
}

// Radial force coefficients of one center, alpha[t][k] = sum_n Fp[n] c(t1,t)[n][k]
// (the group's lanes split the T * kpr entries); c_rad: shared-memory table.
template <int G>
__device__ __forceinline__ void center_alpha(const ModelParams& p, int t1, const float* s_fp,
                                             const float* c_rad, int kpr, int gl, float* al)
{
  const int T = p.T, nR = p.nR;
  for (int e = gl; e < T * kpr; e += G) {
    const int t = e / kpr, kk = e % kpr;
    const float* c = c_rad + (t1 * T + t) * nR * kpr + kk;
    float acc = 0.0f;
    for (int n = 0; n < nR; ++n) acc += s_fp[n] * c[n * kpr];
    al[e] = acc;
  }
}

// Moment derivatives of one center, a[n][lm] = dE/ds[n][lm] (one lane owns
// one n); the monomial terms read the moments at run-time indices, so both
// live in shared memory.
template <int G, int NLM>
__device__ __forceinline__ void center_acoef(const ModelParams& p, const float* s_s, float* s_a,
                                             const float* s_fp, int gl)
{
  const int nR = p.nR, nA = p.nA;
  if constexpr (NLM == kNumLM) {
    // degrees <= 4: moments and derivatives of one n in registers
    const float* fp = s_fp + nR;
    for (int n = gl; n < nA; n += G) {
      float sv[kNumLM], av[kNumLM];
      load24(s_s + n * NLM, sv);
#pragma unroll
      for (int Lq = 1; Lq <= 4; ++Lq) {
        const int st0 = Lq * Lq - 1;
        const bool on = Lq <= p.L_max;
        const float f = on ? fp[(Lq - 1) * nA + n] : 0.0f;
        av[st0] = on ? 2.0f * f * c_C3B[st0] * sv[st0] : 0.0f;
#pragma unroll
        for (int k = 1; k < 2 * Lq + 1; ++k)
          av[st0 + k] = on ? 4.0f * f * c_C3B[st0 + k] * sv[st0 + k] : 0.0f;
      }
      int col = p.L_max;
      for (int w = 0; w < p.num_inv; ++w, ++col)
        inv_grad_id(p.inv_id[w], sv, av, fp[col * nA + n]);
      store24(s_a + n * NLM, av);
    }
  } else {
    for (int n = gl; n < nA; n += G) {
      const float* sv = s_s + n * NLM;
      float* av = s_a + n * NLM;
      const float* fp = s_fp + nR;
      int col = 0;
      for (int Lq = 1; Lq <= p.L_max; ++Lq, ++col) {
        const int st0 = Lq * Lq - 1;
        const float f = fp[col * nA + n];
        av[st0] = 2.0f * f * c_C3B[st0] * sv[st0];
        for (int k = 1; k < 2 * Lq + 1; ++k) av[st0 + k] = 4.0f * f * c_C3B[st0 + k] * sv[st0 + k];
      }
      for (int lm = (p.L_max + 1) * (p.L_max + 1) - 1; lm < NLM; ++lm) av[lm] = 0.0f;
      for (int w = 0; w < p.num_inv; ++w, ++col) {
        const int id = p.inv_id[w];
        const float f = fp[col * nA + n];
        for (int m = c_inv_start[id]; m < c_inv_start[id + 1]; ++m) {
          const Monomial mo = c_mono[m];
          const int nf = mo.i[3] >= 0 ? 4 : 3;
          for (int a = 0; a < nf; ++a) {
            float t = f * mo.c;
            for (int r = 0; r < nf; ++r)
              if (r != a) t *= sv[mo.i[r]];
            av[mo.i[a]] += t;
          }
        }
      }
    }
  }
}

// tanh of the mixed-precision ANN: the hardware approximation (PTX
// tanh.approx.f32, relative error about 2^-11, the size of an FP16 operand's
// rounding).
__device__ __forceinline__ float tanh_fast(float x)
{
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One FP32 value as a 16-bit MMA operand (FP16 or BF16, round to nearest).
__device__ __forceinline__ void store16(unsigned char* at, float v, bool bf16)
{
  *reinterpret_cast<unsigned short*>(at) =
    bf16 ? __bfloat16_as_ushort(__float2bfloat16_rn(v)) : __half_as_ushort(__float2half_rn(v));
}

// One chunk of the stacked weights into the tiles (16-byte rows of core
// matrices): rows m = 128 k .. of W0 (stacked m = t H + h) and columns
// 128 k .. of W0^T.
__device__ __forceinline__ void tc_stage_chunk(const ModelParams& p, const FusedLayout& Lay,
                                               unsigned char* smb, int k)
{
  const int dimk = p.tc_dimk, th = p.T * p.H, m0 = 128 * k;
  const int rows = th - m0 < 128 ? th - m0 : 128;
  const int cw = dimk / 8;
  const uint4* w = reinterpret_cast<const uint4*>(p.w0h + static_cast<size_t>(m0) * dimk);
  for (int e = threadIdx.x; e < rows * cw; e += kBlock)
    *reinterpret_cast<uint4*>(smb + Lay.tc_w + tc::off16(e / cw, 8 * (e % cw), dimk)) =
      __ldg(w + e);
  for (int e = threadIdx.x; e < p.dim * 16; e += kBlock) {
    const int d = e / 16, c = e % 16;
    *reinterpret_cast<uint4*>(smb + Lay.tc_wt + tc::off16(d, 8 * c, 128)) =
      __ldg(reinterpret_cast<const uint4*>(p.w0th + static_cast<size_t>(d) * p.tc_kt + m0 +
                                           8 * c));
  }
}

// Tensor-core set-up of a CTA of the mixed-precision descriptor kernel (before
// its first barrier): TMEM for the two accumulators, the mbarrier, flags, and
// with a single chunk of stacked hidden units the weight tiles.
template <int APB>
__device__ __forceinline__ void tc_ann_setup(const ModelParams& p, const FusedLayout& Lay,
                                             unsigned char* smb)
{
  constexpr int kCols = 2 * APB < 32 ? 32 : 2 * APB;   // D1 | D2, APB columns each
  uint32_t* misc = reinterpret_cast<uint32_t*>(smb + Lay.tc_misc);
  if (threadIdx.x < 32) tc::tmem_alloc(misc + 2, kCols);
  if (threadIdx.x == 0) {
    tc::mbar_init(tc::smem_u32(smb + Lay.tc_bar));
    misc[0] = 0u;   // largest |q| of the CTA (float bits)
  }
  unsigned* tmask = reinterpret_cast<unsigned*>(smb + Lay.tc_type);
  if (threadIdx.x < kMaxTypes) tmask[threadIdx.x] = 0u;   // centers of each type
  if (p.tc_kt == 128) {
    tc_stage_chunk(p, Lay, smb, 0);
    tc::fence_async_smem();
  }
}

// The per-atom ANN of all APB centers of the CTA on the tensor cores (whole
// CTA; s_q of every center holds its scaled descriptors).  The hidden units
// of all types are stacked, m = t H + h, and run in chunks of 128:
//   GEMM1 (M = 128 stacked units, N = APB centers, K = dim):
//     Z = W0 Q^T, from the 16-bit tiles of W0 * sw and Q * sq;
//   epilogue (thread = unit m = its TMEM lane, t = m / H): for the centers of
//     type t, x = tanh(z / (sw sq) - b0) (hardware tanh), E += w1 x,
//     G = w1 (1 - x^2) * sg (zero for the other centers);
//   GEMM2 (M = dim, N = APB, K = the chunk's 128 units): dE/dq += W0^T G^T,
//     accumulated over the chunks in TMEM.
// sw, sg are the model's power-of-two scales (nepx_set_precision), sq the
// CTA's (largest |q| to 2^14): in FP16 every operand keeps its 11-bit
// significand; unscaling by powers of two is exact.  Then each center's
// dE/dq (times q_scaler) lands in its s_fp and its site energy in pe_ann.
// Every wait is bounded: a timeout sets ann_error, waits (bounded again) for
// the MMAs in flight and lets the CTA finish with the error flagged.
template <int APB, int G>
__device__ void tc_ann(const ModelParams& p, const FusedLayout& Lay, float* sm, int slot,
                       int gl, bool active, int t1, int i, const float* s_q,
                       double* __restrict__ pe_ann, NeighborState* st)
{
  constexpr int kCols = 2 * APB < 32 ? 32 : 2 * APB;
  unsigned char* smb = reinterpret_cast<unsigned char*>(sm);
  unsigned char* Wt = smb + Lay.tc_w;
  unsigned char* Vt = smb + Lay.tc_wt;
  unsigned char* Qt = smb + Lay.tc_q;
  unsigned char* Gt = smb + Lay.tc_g;
  float* s_e = reinterpret_cast<float*>(smb + Lay.tc_e);
  unsigned* s_tmask = reinterpret_cast<unsigned*>(smb + Lay.tc_type);
  uint32_t* misc = reinterpret_cast<uint32_t*>(smb + Lay.tc_misc);
  const uint32_t bar = tc::smem_u32(smb + Lay.tc_bar);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int H = p.H, dim = p.dim, dimk = p.tc_dimk, th = p.T * H;
  const int chunks = p.tc_kt / 128;
  const bool bf16 = p.tc_bf16 != 0;

  // the CTA's largest |q| and the center types
  float qm = 0.0f;
  if (active)
    for (int d = gl; d < dim; d += G) qm = fmaxf(qm, fabsf(s_q[d]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) qm = fmaxf(qm, __shfl_xor_sync(kFull, qm, o));
  if (lane == 0) atomicMax(reinterpret_cast<int*>(misc), __float_as_int(qm));
  if (gl == 0 && active) atomicOr(s_tmask + t1, 1u << slot);
  __syncthreads();
  const float qmax = __int_as_float(static_cast<int>(misc[0]));
  int ex = 0;
  frexpf(qmax, &ex);
  const float sq = qmax > 0.0f ? ldexpf(1.0f, max(-60, min(60, 14 - ex))) : 1.0f;
  // this center's row of the descriptor tile, zero past dim and for idle slots
  for (int d = gl; d < dimk; d += G)
    store16(Qt + tc::off16(slot, d, dimk), (active && d < dim) ? s_q[d] * sq : 0.0f, bf16);
  tc::fence_async_smem();
  const uint32_t tmem = misc[2];
  const uint32_t lane_addr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  const uint32_t id = tc::idesc_f16(128, APB, bf16);
  const float unscale1 = 1.0f / (sq * p.tc_sw), unscale2 = 1.0f / (p.tc_sw * p.tc_sg);
  float e_acc[APB];
#pragma unroll
  for (int c = 0; c < APB; ++c) e_acc[c] = 0.0f;
  uint32_t phase = 0;
  bool failed = false;
  for (int k = 0; k < chunks; ++k) {
    if (chunks > 1) {
      // the previous chunk's MMAs are complete: its tiles may be overwritten
      tc_stage_chunk(p, Lay, smb, k);
      tc::fence_async_smem();
    }
    tc::before_sync();
    __syncthreads();
    tc::after_sync();
    if (tid == 0) {
      for (int s = 0; s < dimk / 16; ++s) {
        const uint64_t a = tc::smem_desc(tc::smem_u32(Wt + tc::off16(0, 16 * s, dimk)), dimk);
        const uint64_t b = tc::smem_desc(tc::smem_u32(Qt + tc::off16(0, 16 * s, dimk)), dimk);
        tc::mma_f16(tmem, a, b, id, s > 0 ? 1u : 0u);
      }
      tc::mma_commit(bar);
    }
    bool ok = tc::mbar_wait(bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    tc::after_sync();
    const int m = 128 * k + tid;
    const bool unit = m < th;
    const unsigned mine = unit ? s_tmask[m / H] : 0u;   // the centers of this unit's type
    const float b0m = unit ? __ldg(p.b0 + m) : 0.0f;   // b0 and w1 are [T][H]: index m
    const float w1m = unit ? __ldg(p.w1 + m) : 0.0f;
#pragma unroll
    for (int c0 = 0; c0 < APB; c0 += 16) {
      float z[16];
      tc::tmem_ld16(lane_addr + c0, z);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int c = c0 + q;
        float g = 0.0f;
        if ((mine >> c) & 1u) {
          const float x = tanh_fast(z[q] * unscale1 - b0m);
          e_acc[c] += w1m * x;
          g = w1m * (1.0f - x * x) * p.tc_sg;
        }
        store16(Gt + tc::off16(c, tid, 128), g, bf16);
      }
    }
    tc::fence_async_smem();
    tc::before_sync();
    __syncthreads();   // G complete, D1 read
    tc::after_sync();
    if (tid == 0) {
      for (int s = 0; s < 128 / 16; ++s) {
        const uint64_t a = tc::smem_desc(tc::smem_u32(Vt + tc::off16(0, 16 * s, 128)), 128);
        const uint64_t b = tc::smem_desc(tc::smem_u32(Gt + tc::off16(0, 16 * s, 128)), 128);
        tc::mma_f16(tmem + APB, a, b, id, (k > 0 || s > 0) ? 1u : 0u);
      }
      tc::mma_commit(bar);
    }
    ok = tc::mbar_wait(bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    tc::after_sync();
  }
  if (!failed) {
    // dE/dq: descriptor component d = this thread's TMEM lane, every center
    const int d = tid;
    const float qs = d < dim ? __ldg(p.q_scaler + d) : 0.0f;
#pragma unroll
    for (int c0 = 0; c0 < APB; c0 += 16) {
      float f[16];
      tc::tmem_ld16(lane_addr + APB + c0, f);
      if (d < dim)
#pragma unroll
        for (int q = 0; q < 16; ++q)
          sm[Lay.atoms_base + (c0 + q) * Lay.per_atom + Lay.fp + d] = f[q] * unscale2 * qs;
    }
  }
  // site energies: each warp's partial sums over its 32 hidden units, lane c
  // ends with center c's (fixed order), then the four warps in order
  if constexpr (APB == 16) {
#pragma unroll
    for (int c = 0; c < 16; ++c) e_acc[c] += __shfl_xor_sync(kFull, e_acc[c], 16);
  }
  int at = 0;
  if constexpr (APB == 32) rs_step<32, 16>(e_acc, lane, at);
  rs_step<16, 8>(e_acc, lane, at);
  rs_step<8, 4>(e_acc, lane, at);
  rs_step<4, 2>(e_acc, lane, at);
  rs_step<2, 1>(e_acc, lane, at);
  if (lane < APB) s_e[warp * APB + at] = e_acc[0];
  if (failed) {
    if (tid == 0) atomicOr(&st->ann_error, 1);
    tc::mbar_wait(bar, phase ^ 1u);   // the MMAs of the phase that timed out
  }
  tc::before_sync();
  __syncthreads();
  tc::after_sync();
  if (warp == 0) tc::tmem_dealloc(misc[2], kCols);
  if (active && gl == 0) {
    const float e = s_e[slot] + s_e[APB + slot] + s_e[2 * APB + slot] + s_e[3 * APB + slot];
    pe_ann[i] = static_cast<double>(e - __ldg(p.out_bias + t1));
  }
}

// Typewise filter and radial descriptors (large-box path): one group of G
// lanes per center sweeps its sorted Verlet row with the next candidate's
// site in flight, applies the reference's FP32 predicate bit for bit (double
// difference rounded to float, float minimum image, the same x*x + y*y + z*z
// expression; nep.cu:503-561) and writes the radial and angular rows in
// order (group ballot + popcount), summing
// q_n = sum_j sum_k c(ti,tj)[n][k] f_k(d_ij) on the way.  BIN: each lane
// sums its edges' basis values per neighbour type, B[tj][k] += f_k(d_ij), in
// its own shared-memory bins and contracts them with c once at the end
// (q_n = sum_t sum_k c(ti,t)[n][k] B[t][k]): a few float4 updates per edge
// instead of the nR x kR contraction.  Kept apart from k_nep_fused so this
// latency-bound sweep runs at the occupancy of its own register count.
// FAST: the mixed-precision build (hardware sqrt / reciprocal / sine-cosine
// approximations, see cutoff_fc), held to seven CTAs per SM (72 registers,
// as the exact build takes; it would take 78, rounded to 80: six CTAs).
template <int G, int NRM, int KM, bool BIN, bool FAST>
__global__ void __launch_bounds__(kBlock, (FAST ? 7 : 0))
k_filter_radial(const ModelParams p, int N, const Box* __restrict__ box,
                const Site* __restrict__ sites, NeighborState* st,
                const int* __restrict__ nn_v, const int* __restrict__ nl_v, int mn_v,
                int* __restrict__ nn_r, int* __restrict__ nl_r, int mn_r,
                int* __restrict__ nn_a, int* __restrict__ nl_a, int mn_a,
                float* __restrict__ qrad)
{
  constexpr int APW = 32 / G, APB = kBlock / G;
  constexpr int KP = (KM + 3) & ~3;
  extern __shared__ float sm[];   // radial coefficient table [T*T][nR][KP], then the bins
  const int tid = threadIdx.x;
  const int T = p.T, nR = p.nR, kR = p.kR;
  for (int k = tid; k < T * T * nR * KP; k += kBlock) {
    const int kk = k % KP, row = k / KP;
    sm[k] = kk < kR ? __ldg(p.c_pair + row * kR + kk) : 0.0f;
  }
  // this lane's bins [T][KP] (an odd number of float4 per lane: no bank conflicts)
  float4* bin = reinterpret_cast<float4*>(sm + filter_table_floats(p, KP)) +
                tid * filter_bin_float4(p, KP);
  if constexpr (BIN)
    for (int q = 0; q < T * KP / 4; ++q) bin[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (blockIdx.x == 0 && tid == 0) st->rebuild = 0;   // the Verlet list is consumed
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  const int group = lane / G, gl = lane % G;
  const int i = blockIdx.x * APB + warp * APW + group;
  const bool active = i < N;
  const Box b = *box;
  const Site me = active ? sites[i] : Site{0.0, 0.0, 0.0, 0};
  const double xi = me.x, yi = me.y, zi = me.z;
  const int t1 = static_cast<int>(me.type);
  const unsigned below = (1u << gl) - 1u;
  float qr[NRM];
#pragma unroll
  for (int n = 0; n < NRM; ++n) qr[n] = 0.0f;
  const int nv = active ? nn_v[i] : 0;
  const int nv_max = __reduce_max_sync(kFull, nv);
  const int* vrow = nl_v + static_cast<size_t>(i) * mn_v;
  int* rrow = nl_r + static_cast<size_t>(i) * mn_r;
  int* arow = nl_a + static_cast<size_t>(i) * mn_a;
  int cr = 0, ca = 0;
  // the next candidate's site and the index of the one after it in flight:
  // no load inside the loop waits on another
  int j_next = 0, j_after = 0;
  double2 sa_next = make_double2(0.0, 0.0), sc_next = make_double2(0.0, 0.0);
  if (gl < nv) {
    j_next = vrow[gl];
    site_load(sites, j_next, sa_next, sc_next);
  }
  if (gl + G < nv) j_after = vrow[gl + G];
  for (int base = 0; base < nv_max; base += G) {
    const int k = base + gl;
    const int j = j_next;
    const double2 sa = sa_next, sc = sc_next;
    if (k + G < nv) {
      j_next = j_after;
      site_load(sites, j_next, sa_next, sc_next);
    }
    if (k + 2 * G < nv) j_after = vrow[k + 2 * G];
    bool in_r = false, in_a = false;
    int t2 = 0;
    float x12 = 0.0f, y12 = 0.0f, z12 = 0.0f, d12_square = 0.0f, rc_radial = 1.0f;
    float rcinv_r = 1.0f;
    if (k < nv) {
      site_delta(b, sa, sc, xi, yi, zi, x12, y12, z12, t2);
      d12_square = x12 * x12 + y12 * y12 + z12 * z12;
      float rc_angular, rcinv_a;
      pair_cutoff<FAST>(p, 0, t1, t2, rc_radial, rcinv_r);
      pair_cutoff<FAST>(p, 1, t1, t2, rc_angular, rcinv_a);
      in_r = d12_square < rc_radial * rc_radial;
      in_a = in_r && d12_square < rc_angular * rc_angular;
    }
    const unsigned mr = group_ballot<G>(in_r, group);
    const unsigned ma = group_ballot<G>(in_a, group);
    if (in_r) {
      const int at = cr + __popc(mr & below);
      if (at < mn_r) rrow[at] = j;
      float d, dinv;
      edge_length<FAST>(d12_square, d, dinv);
      const float rcinv = rcinv_r;
      float fc, fcp;
      cutoff_fc<FAST>(rc_radial, rcinv, d, fc, fcp);
      float fn[KP];
#pragma unroll
      for (int kk = 0; kk < KP; ++kk) fn[kk] = 0.0f;
      radial_basis<KM>(kR, rcinv, d, fc, fn);
      if constexpr (BIN) {
        float4* bt = bin + t2 * (KP / 4);
#pragma unroll
        for (int q = 0; q < KP / 4; ++q) {
          float4 v = bt[q];
          v.x += fn[4 * q];
          v.y += fn[4 * q + 1];
          v.z += fn[4 * q + 2];
          v.w += fn[4 * q + 3];
          bt[q] = v;
        }
      } else {
        const float* c = sm + (t1 * T + t2) * nR * KP;
#pragma unroll
        for (int n = 0; n < NRM; ++n)
          if (n < nR) qr[n] += dot_basis<KM>(c + n * KP, fn);
      }
    }
    if (in_a) {
      const int at = ca + __popc(ma & below);
      if (at < mn_a) arow[at] = j;
    }
    cr += __popc(mr);
    ca += __popc(ma);
  }
  if constexpr (BIN) {
    const float* bf = reinterpret_cast<const float*>(bin);
    for (int t = 0; t < T; ++t) {
      const float* c = sm + (t1 * T + t) * nR * KP;
#pragma unroll
      for (int n = 0; n < NRM; ++n)
        if (n < nR) qr[n] += dot_basis<KM>(c + n * KP, bf + t * KP);
    }
  }
#pragma unroll
  for (int n = 0; n < NRM; ++n) qr[n] = group_sum<G>(qr[n]);
  if (active && gl == 0) {
    nn_r[i] = min(cr, mn_r);
    nn_a[i] = min(ca, mn_a);
    if (cr > mn_r) atomicOr(&st->overflow, 2);
    if (ca > mn_a) atomicOr(&st->overflow, 4);
    atomicMax(&st->max_nn[1], cr);
    atomicMax(&st->max_nn[2], ca);
    atomicMax(&st->call_nn[0], cr);
    atomicMax(&st->call_nn[1], ca);
#pragma unroll
    for (int n = 0; n < NRM; ++n)
      if (n < nR) qrad[static_cast<size_t>(i) * nR + n] = qr[n];
  }
}

// Directed angular partial force of a center on one neighbour at
// r = (dx, dy, dz) = r_j - r_i:
//   f12 = (sum_lm B_lm Y_lm) r^ + (1/d)(I - r^r^T) sum_lm A_lm dY_lm/dr^,
//   A_lm = sum_n a[n][lm] g_n(d), B_lm = sum_n a[n][lm] g'_n(d),
// with a[n][lm] = dE/ds[n][lm] of the center (av: global memory, or with AG
// false the center's shared-memory scratch) and c its angular coefficient
// table for the pair (nA rows of the padded basis, shared memory).
// Reference find_partial_force_angular (nep.cu:890-991) with the
// accumulate_f12 ladder (nep_utilities.cuh:1240-1491) evaluated once per edge
// instead of once per (edge, n).
template <int KM, int NAM, int LMAX, bool AG = true, bool FAST = false>
__device__ __forceinline__ float3 angular_edge_force(const ModelParams& p, const float* c,
                                                    const float* __restrict__ av, float rc,
                                                    float rcinv, float dx, float dy, float dz)
{
  constexpr int KP = (KM + 3) & ~3;
  constexpr int NLM = num_lm<LMAX>();
  const int nA = p.nA;
  float d, dinv;
  edge_length<FAST>(dx * dx + dy * dy + dz * dz, d, dinv);
  const float ux = dx * dinv, uy = dy * dinv, uz = dz * dinv;
  float fc, fcp;
  cutoff_fc<FAST>(rc, rcinv, d, fc, fcp);
  float fn[KP], fnp[KP];
#pragma unroll
  for (int kk = 0; kk < KP; ++kk) {
    fn[kk] = 0.0f;
    fnp[kk] = 0.0f;
  }
  radial_basis_d<KM>(p.kA, rcinv, d, fc, fcp, fn, fnp);
  float A[NLM], B[NLM];
#pragma unroll
  for (int lm = 0; lm < NLM; ++lm) {
    A[lm] = 0.0f;
    B[lm] = 0.0f;
  }
#pragma unroll
  for (int n = 0; n < NAM; ++n) {
    if (n < nA) {
      const float g = dot_basis<KM>(c + n * KP, fn);
      const float gp = dot_basis<KM>(c + n * KP, fnp);
      const float* an = av + n * NLM;
#pragma unroll
      for (int q = 0; q < NLM / 4; ++q) {
        const float4 a4 = AG ? __ldg(reinterpret_cast<const float4*>(an) + q)
                             : reinterpret_cast<const float4*>(an)[q];
        A[4 * q] += a4.x * g;
        A[4 * q + 1] += a4.y * g;
        A[4 * q + 2] += a4.z * g;
        A[4 * q + 3] += a4.w * g;
        B[4 * q] += a4.x * gp;
        B[4 * q + 1] += a4.y * gp;
        B[4 * q + 2] += a4.z * gp;
        B[4 * q + 3] += a4.w * gp;
      }
    }
  }
  // SB = sum B Y, V = sum A dY/du (u components independent)
  float zp[LMAX + 1];
  zp[0] = 1.0f;
#pragma unroll
  for (int q = 1; q <= LMAX; ++q) zp[q] = zp[q - 1] * uz;
  float SB = 0.0f, vx = 0.0f, vy = 0.0f, vz = 0.0f;
  int idx = 0;
#pragma unroll
  for (int Lq = 1; Lq <= LMAX; ++Lq) {
    if (Lq > p.L_max) break;
    float re0 = 1.0f, im0 = 0.0f;   // (ux + i uy)^(m-1)
#pragma unroll
    for (int m = 0; m <= Lq; ++m) {
      float dzf;
      const float zf = zpoly_any(Lq, m, zp, &dzf);
      if (m == 0) {
        SB += B[idx] * zf;
        vz += A[idx] * dzf;
        ++idx;
      } else {
        const float re = ux * re0 - uy * im0;
        const float im = ux * im0 + uy * re0;
        const float Ar = A[idx], Ai = A[idx + 1];
        SB += (B[idx] * re + B[idx + 1] * im) * zf;
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
  return make_float3(SB * ux + (vx - uv * ux) * dinv, SB * uy + (vy - uv * uy) * dinv,
                     SB * uz + (vz - uv * uz) * dinv);
}

// NRM/KM/NAM: compile-time bounds of nR, basis size + 1, nA for this instance.
// MINB: CTAs per SM the instance is built for (register cap 65536 / (128
// MINB)).  The small shape comes at 3 (168 registers, moments of five radial
// functions per sweep) and at 4 (128 registers, three per sweep: the angular
// row is swept twice but a third more warps hide the latency); the
// autotuner picks one.
// XR: explicit rows (small-box and batched paths) -- the radial and angular
// rows hold the displacement and packed neighbour of every edge (er, ea),
// built beforehand; phase 1 then only accumulates the radial descriptors.
// LMAX: 4 (moments of 24 components per n, five n per sweep) or 8 (80
// components, one n per sweep).
// TC: the ANN of the CTA's centers runs on the tensor cores (tc_ann, the
// mixed-precision path); otherwise in FP32 per center.
// FF (Verlet-row path only): the kernel ends with the directed angular partial
// forces f12 of the center's edges, from a[n][lm] in its shared-memory
// scratch, in place of handing a[n][lm] to k_angular_f12 through memory (the
// autotuner times both forms).
template <int G, int NRM, int KM, int NAM, bool XR, int LMAX, int MINB, bool TC, bool FF>
__global__ void __launch_bounds__(kBlock, MINB)
k_nep_fused(const ModelParams p, int N, const Box* __restrict__ box,
            const Site* __restrict__ sites, NeighborState* st,
            const int* __restrict__ nn_v, const int* __restrict__ nl_v, int mn_v,
            int* __restrict__ nn_r, int* __restrict__ nl_r, int mn_r, int* __restrict__ nn_a,
            int* __restrict__ nl_a, int mn_a, const float4* __restrict__ er,
            const float4* __restrict__ ea, const float* __restrict__ qrad,
            float* __restrict__ alpha, float* __restrict__ acoef, float4* __restrict__ f12,
            double* __restrict__ pe_ann)
{
  static_assert(!(FF && XR), "the fused angular force is built for Verlet rows only");
  // the mixed-precision build also takes the hardware approximations of
  // sqrt, reciprocal, sine and cosine (cutoff_fc)
  constexpr bool FAST = TC;
  constexpr int APW = 32 / G;             // centers per warp
  constexpr int APB = kBlock / G;         // centers per block
  constexpr int KP = (KM + 3) & ~3;
  constexpr int NLM = num_lm<LMAX>();
  // radial functions per moment sweep
  constexpr int CN = LMAX <= 4 ? (MINB >= 4 ? kChunkN4 : kChunkN) : 1;
  extern __shared__ __align__(128) float sm[];
  constexpr bool PF = fused_prefetch(XR, MINB);
  const FusedLayout Lay = fused_layout(p, APB, KP, fused_smem_budget(MINB), TC, PF);
  const int tid = threadIdx.x;
  const int T = p.T, nR = p.nR, nA = p.nA, kR = p.kR, kA = p.kA;
  const int dim = p.dim, H = p.H;
  // padded coefficient tables
  for (int k = tid; k < T * T * nR * Lay.kpr; k += kBlock) {
    const int kk = k % Lay.kpr, row = k / Lay.kpr;   // row = tp*nR + n
    sm[Lay.c_rad + k] = kk < kR ? __ldg(p.c_pair + row * kR + kk) : 0.0f;
  }
  for (int k = tid; k < T * T * nA * Lay.kpa; k += kBlock) {
    const int kk = k % Lay.kpa, row = k / Lay.kpa;
    sm[Lay.c_ang + k] = kk < kA ? __ldg(p.c_pair + p.num_c_radial + row * kA + kk) : 0.0f;
  }
  if (Lay.wt >= 0) {
    const float4* src = reinterpret_cast<const float4*>(p.w0t);
    float4* dst = reinterpret_cast<float4*>(sm + Lay.wt);
    for (int k = tid; k < T * dim * p.H4 / 4; k += kBlock) dst[k] = __ldg(src + k);
  }
  if (blockIdx.x == 0 && tid == 0) st->rebuild = 0;   // the Verlet list is consumed
  if constexpr (TC) {
    tc_ann_setup<APB>(p, Lay, reinterpret_cast<unsigned char*>(sm));
    tc::before_sync();
  }
  __syncthreads();
  if constexpr (TC) tc::after_sync();

  const int lane = tid & 31, warp = tid >> 5;
  const int group = lane / G, gl = lane % G;
  const int slot = warp * APW + group;                 // center within the block
  const int i = blockIdx.x * APB + slot;
  const bool active = i < N;
  float* mine = sm + Lay.atoms_base + slot * Lay.per_atom;
  float* s_s = mine + Lay.s;
  float* s_a = mine + Lay.a;
  float* s_q = mine + Lay.q;
  float* s_fp = mine + Lay.fp;
  float* s_gh = mine + Lay.gh;
  const Box b = *box;
  const Site me = active ? sites[i] : Site{0.0, 0.0, 0.0, 0};
  const double xi = me.x, yi = me.y, zi = me.z;
  const int t1 = static_cast<int>(me.type);

  // ---- 1. filter the Verlet row, radial descriptors -------------------------
  float qr[NRM];
#pragma unroll
  for (int n = 0; n < NRM; ++n) qr[n] = 0.0f;
  // q_n += sum_k c(t1,t2)[n][k] f_k(d) for one radial edge
  auto add_radial = [&](int t2, float d12_square) {
    float rc_radial, rcinv;
    pair_cutoff<FAST>(p, 0, t1, t2, rc_radial, rcinv);
    float d, dinv;
    edge_length<FAST>(d12_square, d, dinv);
    float fc, fcp;
    cutoff_fc<FAST>(rc_radial, rcinv, d, fc, fcp);
    float fn[KP];
#pragma unroll
    for (int kk = 0; kk < KP; ++kk) fn[kk] = 0.0f;
    radial_basis<KM>(kR, rcinv, d, fc, fn);
    const float* c = sm + Lay.c_rad + (t1 * T + t2) * nR * Lay.kpr;
#pragma unroll
    for (int n = 0; n < NRM; ++n)
      if (n < nR) qr[n] += dot_basis<KM>(c + n * Lay.kpr, fn);
  };
  int cr = 0, ca = 0;
  if constexpr (XR) {
    // explicit rows: counts clamped to capacity by the row builder
    cr = active ? nn_r[i] : 0;
    ca = active ? nn_a[i] : 0;
    const int cr_max = __reduce_max_sync(kFull, cr);
    const float4* erow = er + static_cast<size_t>(i) * mn_r;
    for (int base = 0; base < cr_max; base += G) {
      const int k = base + gl;
      if (k < cr) {
        const float4 e = erow[k];
        const int t2 = static_cast<int>(static_cast<unsigned>(__float_as_int(e.w)) >> kRowTypeShift);
        add_radial(t2, e.x * e.x + e.y * e.y + e.z * e.z);
      }
    }
  } else {
    // the typewise rows, their counts and the radial descriptors come from
    // k_filter_radial (lane 0 of the group holds q, the group sum spreads it)
    cr = active ? nn_r[i] : 0;
    ca = active ? nn_a[i] : 0;
    if (active && gl == 0)
#pragma unroll
      for (int n = 0; n < NRM; ++n)
        if (n < nR) qr[n] = qrad[static_cast<size_t>(i) * nR + n];
  }
#pragma unroll
  for (int n = 0; n < NRM; ++n) qr[n] = group_sum<G>(qr[n]);
  if (gl == 0)
#pragma unroll
    for (int n = 0; n < NRM; ++n)
      if (n < nR) s_q[n] = qr[n];
  __syncwarp();

  // ---- 2. angular moments s[n][lm] -----------------------------------------
  const int na = min(ca, mn_a);
  const int na_max = __reduce_max_sync(kFull, na);
  const int* arow = nl_a + static_cast<size_t>(i) * mn_a;
  const float4* earow = ea + static_cast<size_t>(i) * mn_a;
  for (int nc = 0; nc < nA; nc += CN) {
    float v[CN * NLM];
#pragma unroll
    for (int q = 0; q < CN * NLM; ++q) v[q] = 0.0f;
    // PF: the site of the lane's next edge is copied into the lane's other
    // shared-memory slot while the current one is worked on; the index of the
    // edge after that is loaded one iteration early, so no load waits on
    // another inside the loop
    const unsigned slots =
      PF ? static_cast<unsigned>(__cvta_generic_to_shared(sm + Lay.pf)) + 64u * tid : 0u;
    int j_next = 0;
    if constexpr (PF) {
      if (gl < na) site_fetch_async(slots, sites + arow[gl]);
      async_commit();
      if (gl + G < na) j_next = arow[gl + G];
    }
    for (int base = 0; base < na_max; base += G) {
      const int k = base + gl;
      const int par = (base / G) & 1;
      if constexpr (PF) {
        if (k + G < na) site_fetch_async(slots + 32u * (par ^ 1), sites + j_next);
        async_commit();
        if (k + 2 * G < na) j_next = arow[k + 2 * G];
        async_wait_prior();
      }
      if (k < na) {
        int t2;
        float dx, dy, dz;
        if constexpr (XR) {
          const float4 e = earow[k];
          dx = e.x;
          dy = e.y;
          dz = e.z;
          t2 = static_cast<int>(static_cast<unsigned>(__float_as_int(e.w)) >> kRowTypeShift);
        } else if constexpr (PF) {
          const double2* sl = reinterpret_cast<const double2*>(sm + Lay.pf + 16 * tid + 8 * par);
          site_delta(b, sl[0], sl[1], xi, yi, zi, dx, dy, dz, t2);
        } else {
          site_displacement(b, sites, xi, yi, zi, arow[k], dx, dy, dz, t2);
        }
        float d, dinv;
        edge_length<FAST>(dx * dx + dy * dy + dz * dz, d, dinv);
        float rc, rcinv;
        pair_cutoff<FAST>(p, 1, t1, t2, rc, rcinv);
        float fc, fcp;
        cutoff_fc<FAST>(rc, rcinv, d, fc, fcp);
        float fn[KP];
#pragma unroll
        for (int kk = 0; kk < KP; ++kk) fn[kk] = 0.0f;
        radial_basis<KM>(kA, rcinv, d, fc, fn);
        const float* c = sm + Lay.c_ang + ((t1 * T + t2) * nA + nc) * Lay.kpa;
        float g[CN];
#pragma unroll
        for (int n = 0; n < CN; ++n)
          g[n] = (nc + n < nA) ? dot_basis<KM>(c + n * Lay.kpa, fn) : 0.0f;
        for_each_harmonic<LMAX>(p.L_max, dx * dinv, dy * dinv, dz * dinv, [&](int lm, float y) {
#pragma unroll
          for (int n = 0; n < CN; ++n) v[n * NLM + lm] += g[n] * y;
        });
      }
    }
    if constexpr (PF) async_wait_all();
    const int at = reduce_scatter<G, CN * NLM>(v, gl);
    constexpr int share = CN * NLM / G;
    const int lim = (nA - nc < CN ? nA - nc : CN) * NLM;
#pragma unroll
    for (int q = 0; q < share; ++q)
      if (at + q < lim) s_s[nc * NLM + at + q] = v[q];
  }
  __syncwarp();

  // ---- 3. invariants, ANN, derivatives ---------------------------------------
  if constexpr (NLM == kNumLM) {
    // degrees <= 4: the n's 24 moments in registers, monomials unrolled
    for (int n = gl; n < nA; n += G) {
      float sv[kNumLM];
      load24(s_s + n * NLM, sv);
      float* q = s_q + nR;
#pragma unroll
      for (int Lq = 1; Lq <= 4; ++Lq) {
        if (Lq <= p.L_max) {
          const int st0 = Lq * Lq - 1;
          float val = 0.0f;
#pragma unroll
          for (int k = 1; k < 2 * Lq + 1; ++k) val += c_C3B[st0 + k] * sv[st0 + k] * sv[st0 + k];
          val *= 2.0f;
          val += c_C3B[st0] * sv[st0] * sv[st0];
          q[(Lq - 1) * nA + n] = val;
        }
      }
      int col = p.L_max;
      for (int w = 0; w < p.num_inv; ++w, ++col) q[col * nA + n] = inv_value_id(p.inv_id[w], sv);
    }
  } else {
    for (int n = gl; n < nA; n += G) {
      const float* s = s_s + n * NLM;
      float* q = s_q + nR;
      int col = 0;
      for (int Lq = 1; Lq <= p.L_max; ++Lq, ++col) {
        const int st0 = Lq * Lq - 1;
        float val = 0.0f;
        for (int k = 1; k < 2 * Lq + 1; ++k) val += c_C3B[st0 + k] * s[st0 + k] * s[st0 + k];
        val *= 2.0f;
        val += c_C3B[st0] * s[st0] * s[st0];
        q[col * nA + n] = val;
      }
      for (int w = 0; w < p.num_inv; ++w, ++col) {
        const int id = p.inv_id[w];
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
  }
  __syncwarp();
  // scaled descriptors; hidden-unit derivatives zero-padded to H4 for the
  // float4 dot products
  for (int d = gl; d < dim; d += G) s_q[d] *= __ldg(p.q_scaler + d);
  if constexpr (TC) {
    __syncwarp();
    tc_ann<APB, G>(p, Lay, sm, slot, gl, active, t1, i, s_q, pe_ann, st);
  } else {
    for (int h = H + gl; h < p.H4; h += G) s_gh[h] = 0.0f;
    __syncwarp();
    const float* w0t = Lay.wt >= 0 ? sm + Lay.wt : p.w0t;
    float e_part = 0.0f;
    if (active) {
      // hidden layer: each lane owns two groups of four consecutive hidden units
      // (float4 rows of the transposed w0; eight independent FMA chains in one
      // pass, each sequential in d as in the reference)
      const int hq = p.H4 / 4;
      const float4* wt =
        reinterpret_cast<const float4*>(w0t + static_cast<size_t>(t1) * dim * p.H4);
      auto finish = [&](int h, float z) {
        if (h < H) {
          const float x1 = tanhf(z - __ldg(p.b0 + t1 * H + h));
          const float w1 = __ldg(p.w1 + t1 * H + h);
          e_part += w1 * x1;
          s_gh[h] = w1 * (1.0f - x1 * x1);
        }
      };
      for (int h4 = gl; h4 < hq; h4 += 2 * G) {
        const bool has_b = h4 + G < hq;
        const int h4b = has_b ? h4 + G : h4;   // past the end: computed, dropped
        float z0 = 0.0f, z1 = 0.0f, z2 = 0.0f, z3 = 0.0f;
        float z4 = 0.0f, z5 = 0.0f, z6 = 0.0f, z7 = 0.0f;
#pragma unroll 2
        for (int d = 0; d < dim; ++d) {
          const float q = s_q[d];
          const float4 wa = wt[d * hq + h4];
          const float4 wb = wt[d * hq + h4b];
          z0 = fmaf(wa.x, q, z0);
          z1 = fmaf(wa.y, q, z1);
          z2 = fmaf(wa.z, q, z2);
          z3 = fmaf(wa.w, q, z3);
          z4 = fmaf(wb.x, q, z4);
          z5 = fmaf(wb.y, q, z5);
          z6 = fmaf(wb.z, q, z6);
          z7 = fmaf(wb.w, q, z7);
        }
        finish(4 * h4, z0);
        finish(4 * h4 + 1, z1);
        finish(4 * h4 + 2, z2);
        finish(4 * h4 + 3, z3);
        if (has_b) {
          finish(4 * h4b, z4);
          finish(4 * h4b + 1, z5);
          finish(4 * h4b + 2, z6);
          finish(4 * h4b + 3, z7);
        }
      }
    }
    e_part = group_sum<G>(e_part);
    if (active && gl == 0) pe_ann[i] = static_cast<double>(e_part - __ldg(p.out_bias + t1));
    __syncwarp();
    if (active) {
      // dE/dq: four descriptor components per lane at once (d0, d0 + G,
      // d0 + 2G, d0 + 3G), float4 over h, each sum in the same order as before
      const int hq = p.H4 / 4;
      const float4* g4 = reinterpret_cast<const float4*>(s_gh);
      const float4* wt =
        reinterpret_cast<const float4*>(w0t + static_cast<size_t>(t1) * dim * p.H4);
      for (int d0 = gl; d0 < dim; d0 += 4 * G) {
        int dd[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) dd[k] = min(d0 + k * G, dim - 1);   // past dim: dropped
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 2
        for (int h = 0; h < hq; ++h) {
          const float4 g = g4[h];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const float4 w = wt[dd[k] * hq + h];
            acc[k] = fmaf(g.x, w.x, acc[k]);
            acc[k] = fmaf(g.y, w.y, acc[k]);
            acc[k] = fmaf(g.z, w.z, acc[k]);
            acc[k] = fmaf(g.w, w.w, acc[k]);
          }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (d0 + k * G < dim) s_fp[d0 + k * G] = acc[k] * __ldg(p.q_scaler + d0 + k * G);
      }
    }
    __syncwarp();
  }
  if (active) center_alpha<G>(p, t1, s_fp, sm + Lay.c_rad, Lay.kpr, gl,
                              alpha + static_cast<size_t>(i) * T * Lay.kpr);
  center_acoef<G, NLM>(p, s_s, s_a, s_fp, gl);
  __syncwarp();

  // ---- 4. hand a[n][lm] to the angular-force kernel -------------------------
  if constexpr (!FF) {
    if (active) {
      float4* dst = reinterpret_cast<float4*>(acoef + static_cast<size_t>(i) * nA * NLM);
      const float4* src = reinterpret_cast<const float4*>(s_a);
      for (int q = gl; q < nA * NLM / 4; q += G) dst[q] = src[q];
    }
  } else {
    // ---- 4'. or evaluate the angular partial forces here (k_angular_f12's
    // arithmetic, the moments read from shared memory); the sites come again
    // through the lane's two prefetch slots (PF) or with the next index in
    // flight
    const float* ctab = sm + Lay.c_ang + t1 * T * nA * Lay.kpa;
    float4* frow = f12 + static_cast<size_t>(i) * mn_a;
    const unsigned slots =
      PF ? static_cast<unsigned>(__cvta_generic_to_shared(sm + Lay.pf)) + 64u * tid : 0u;
    int j_next = (gl < na) ? arow[gl] : 0;
    if constexpr (PF) {
      if (gl < na) site_fetch_async(slots, sites + j_next);
      async_commit();
      j_next = (gl + G < na) ? arow[gl + G] : 0;
    }
    for (int base = 0; base < na_max; base += G) {
      const int k = base + gl;
      const int par = (base / G) & 1;
      int j = 0;
      if constexpr (PF) {
        if (k + G < na) site_fetch_async(slots + 32u * (par ^ 1), sites + j_next);
        async_commit();
        if (k + 2 * G < na) j_next = arow[k + 2 * G];
        async_wait_prior();
      } else {
        j = j_next;
        if (k + G < na) j_next = arow[k + G];
      }
      if (k < na) {
        int t2;
        float dx, dy, dz;
        if constexpr (PF) {
          const double2* sl = reinterpret_cast<const double2*>(sm + Lay.pf + 16 * tid + 8 * par);
          site_delta(b, sl[0], sl[1], xi, yi, zi, dx, dy, dz, t2);
        } else {
          site_displacement(b, sites, xi, yi, zi, j, dx, dy, dz, t2);
        }
        float rc, rcinv;
        pair_cutoff<FAST>(p, 1, t1, t2, rc, rcinv);
        const float3 f = angular_edge_force<KM, NAM, LMAX, false, FAST>(
          p, ctab + t2 * nA * Lay.kpa, s_a, rc, rcinv, dx, dy, dz);
        frow[k] = make_float4(f.x, f.y, f.z, 0.0f);
      }
    }
    if constexpr (PF) async_wait_all();
  }
}

// Angular coefficient tables [T*T][nA][KP] into shared memory (zero-padded rows).
template <int KP>
__device__ __forceinline__ void load_angular_tables(const ModelParams& p, float* sm)
{
  const int T = p.T, nA = p.nA, kA = p.kA;
  for (int k = threadIdx.x; k < T * T * nA * KP; k += blockDim.x) {
    const int kk = k % KP, row = k / KP;
    sm[k] = kk < kA ? __ldg(p.c_pair + p.num_c_radial + row * kA + kk) : 0.0f;
  }
}

// One group of G lanes per center: the directed angular partial force of
// every edge of the center's angular row, f12[i][k] (float4, w unused).
// XR: explicit rows of a batch; only the centers of structures that are not
// small (each neighbour once in their rows) take this scheme.
// FAST builds held to four CTAs per SM (128 registers, as the exact build
// takes; they would take 142, rounded to 144: three CTAs).
template <int G, int KM, int NAM, bool XR, int LMAX, bool FAST>
__global__ void __launch_bounds__(kBlock, (FAST ? 4 : 0))
k_angular_f12(const ModelParams p, int N, const Box* __restrict__ box,
              const Site* __restrict__ sites,
              const int* __restrict__ nn_a, const int* __restrict__ nl_a, int mn_a,
              const float4* __restrict__ ea, const unsigned char* __restrict__ large,
              const float* __restrict__ acoef, float4* __restrict__ f12)
{
  constexpr int KP = (KM + 3) & ~3;
  extern __shared__ float sm[];
  load_angular_tables<KP>(p, sm);
  __syncthreads();
  const int tid = threadIdx.x;
  const int T = p.T, nA = p.nA;
  const int gl = tid % G;
  const int i = blockIdx.x * (kBlock / G) + tid / G;
  if (i >= N) return;
  if constexpr (XR) {
    if (!large[i]) return;
  }
  const Box b = *box;
  const Site me = sites[i];
  const double xi = me.x, yi = me.y, zi = me.z;
  const int t1 = static_cast<int>(me.type);
  const int na = nn_a[i];
  const int* arow = nl_a + static_cast<size_t>(i) * mn_a;
  const float* ai = acoef + static_cast<size_t>(i) * nA * num_lm<LMAX>();
  for (int k = gl; k < na; k += G) {
    int t2;
    float dx, dy, dz;
    if constexpr (XR) {
      const float4 e = ea[static_cast<size_t>(i) * mn_a + k];
      t2 = static_cast<int>(static_cast<unsigned>(__float_as_int(e.w)) >> kRowTypeShift);
      dx = e.x;
      dy = e.y;
      dz = e.z;
    } else {
      site_displacement(b, sites, xi, yi, zi, arow[k], dx, dy, dz, t2);
    }
    float rc, rcinv;
    pair_cutoff<FAST>(p, 1, t1, t2, rc, rcinv);
    const float3 f = angular_edge_force<KM, NAM, LMAX, true, FAST>(
      p, sm + (t1 * T + t2) * nA * KP, ai, rc, rcinv, dx, dy, dz);
    f12[static_cast<size_t>(i) * mn_a + k] = make_float4(f.x, f.y, f.z, 0.0f);
  }
}

// ---------------------------------------------------------------------------
// gather
// ---------------------------------------------------------------------------

// XR: explicit rows.  The rows then may hold one neighbour several times
// (periodic images), so the reverse partial force f12(j,i) is not looked up
// but evaluated here from j's moment derivatives at -r: the angular force
// work doubles and the f12 buffer and its kernel drop out.
// GMINB: CTAs of 256 per SM the instance is built for (register cap), 0 for
// none.  The Verlet-row gather comes uncapped (about 80 registers for the
// small shape, three CTAs) and at 4 (64 registers, a few spills, a third
// more warps); the autotuner picks one.  The small shape's explicit-row
// FAST build is held to two CTAs (128 registers: uncapped it would take 144,
// and one CTA per SM).
template <int G, int KM, int NAM, bool XR, int LMAX, int GMINB, bool FAST>
__global__ void __launch_bounds__(256, GMINB)
k_gather(const ModelParams p, int N, const Box* __restrict__ box,
         const Site* __restrict__ sites, const int* __restrict__ nn_r, const int* __restrict__ nl_r,
         int mn_r, const int* __restrict__ nn_a, const int* __restrict__ nl_a, int mn_a,
         const float4* __restrict__ er, const float4* __restrict__ ea,
         const float* __restrict__ acoef, const float* __restrict__ alpha,
         const float4* __restrict__ f12, const unsigned char* __restrict__ large,
         const double* __restrict__ pe_ann,
         double* __restrict__ pe, double* __restrict__ force, double* __restrict__ virial,
         int accumulate, NeighborState* st)
{
  constexpr int KP = (KM + 3) & ~3;
  extern __shared__ float sm[];
  if constexpr (XR) {
    load_angular_tables<KP>(p, sm);
    __syncthreads();
  }
  const int gl = threadIdx.x % G;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool active = i < N;
  const Box b = *box;
  const int T = p.T, kR = p.kR, kpr = KP;
  float F[3] = {0.0f, 0.0f, 0.0f};
  float W[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float ezbl = 0.0f;
  if (active) {
    const Site me = sites[i];
    const double xi = me.x, yi = me.y, zi = me.z;
    const int t1 = static_cast<int>(me.type);
    const float* ali = alpha + static_cast<size_t>(i) * T * kpr;
    // radial pairs: both site energies through the alpha coefficients
    const int nr = nn_r[i];
    const int* rrow = nl_r + static_cast<size_t>(i) * mn_r;
    // the next edge's index is loaded one iteration early: the site and alpha
    // loads of an edge then issue together at the top of its iteration
    int jr_next = (!XR && gl < nr) ? rrow[gl] : 0;
    for (int k = gl; k < nr; k += G) {
      int j, t2;
      float dx, dy, dz;
      const int jr = jr_next;
      if constexpr (!XR) {
        if (k + G < nr) jr_next = rrow[k + G];
      }
      if constexpr (XR) {
        const float4 e = er[static_cast<size_t>(i) * mn_r + k];
        const unsigned bits = static_cast<unsigned>(__float_as_int(e.w));
        j = static_cast<int>(bits & kRowIndexMask);
        t2 = static_cast<int>(bits >> kRowTypeShift);
        dx = e.x;
        dy = e.y;
        dz = e.z;
      } else {
        j = jr;
        site_displacement(b, sites, xi, yi, zi, j, dx, dy, dz, t2);
      }
      float d, dinv;
      edge_length<FAST>(dx * dx + dy * dy + dz * dz, d, dinv);
      float rc, rcinv;
      pair_cutoff<FAST>(p, 0, t1, t2, rc, rcinv);
      float fc, fcp;
      cutoff_fc<FAST>(rc, rcinv, d, fc, fcp);
      float fn[KP], fnp[KP];
#pragma unroll
      for (int kk = 0; kk < KP; ++kk) {
        fn[kk] = 0.0f;
        fnp[kk] = 0.0f;
      }
      radial_basis_d<KM>(kR, rcinv, d, fc, fcp, fn, fnp);
      const float w12 = dot_basis<KM>(ali + t2 * kpr, fnp);
      const float w21 = dot_basis<KM>(alpha + (static_cast<size_t>(j) * T + t1) * kpr, fnp);
      const float s12 = w12 * dinv, s21 = w21 * dinv;
      // f12 = s12 r, f21 = -s21 r; F += f12 - f21; W += r (x) f21
      F[0] += (s12 + s21) * dx;
      F[1] += (s12 + s21) * dy;
      F[2] += (s12 + s21) * dz;
      const float f21[3] = {-s21 * dx, -s21 * dy, -s21 * dz};
      W[0] += dx * f21[0];
      W[1] += dy * f21[1];
      W[2] += dz * f21[2];
      W[3] += dx * f21[1];
      W[4] += dx * f21[2];
      W[5] += dy * f21[2];
      W[6] += dy * f21[0];
      W[7] += dz * f21[0];
      W[8] += dz * f21[1];
    }
    // angular exchange and ZBL
    const int na = nn_a[i];
    const int* arow = nl_a + static_cast<size_t>(i) * mn_a;
    const bool large_i = XR && large[i];
    const int zi_ = p.Z[t1];
    const float pow_zi = p.zbl ? powf(static_cast<float>(zi_), 0.23f) : 0.0f;
    int ja_next = (!XR && gl < na) ? arow[gl] : 0;
    for (int k = gl; k < na; k += G) {
      int t2;
      float dx, dy, dz;
      float4 a12, a21;
      const int ja = ja_next;
      if constexpr (!XR) {
        if (k + G < na) ja_next = arow[k + G];
      }
      if constexpr (XR) {
        const float4 e = ea[static_cast<size_t>(i) * mn_a + k];
        const unsigned bits = static_cast<unsigned>(__float_as_int(e.w));
        const int j = static_cast<int>(bits & kRowIndexMask);
        t2 = static_cast<int>(bits >> kRowTypeShift);
        dx = e.x;
        dy = e.y;
        dz = e.z;
        if (large_i) {
          // a structure that is not small: j once in i's row and i once in
          // j's (rows ascend by the packed index), f12 from k_angular_f12
          a12 = f12[static_cast<size_t>(i) * mn_a + k];
          const int* jw = reinterpret_cast<const int*>(ea + static_cast<size_t>(j) * mn_a) + 3;
          const int nj = nn_a[j];
          int lo = 0, hi = nj - 1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((__ldg(jw + 4 * mid) & kRowIndexMask) < i) lo = mid + 1; else hi = mid;
          }
          a21 = f12[static_cast<size_t>(j) * mn_a + lo];
          if (nj == 0 || (__ldg(jw + 4 * lo) & kRowIndexMask) != i) {
            // only a truncated (overflowed) row can lose the reverse edge
            a21 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            atomicOr(&st->overflow, 4);
          }
        } else {
          float rc, rcinv;
          pair_cutoff<FAST>(p, 1, t1, t2, rc, rcinv);
          const int nA = p.nA;
          constexpr int NLM = num_lm<LMAX>();
          const float3 fij = angular_edge_force<KM, NAM, LMAX, true, FAST>(
            p, sm + (t1 * T + t2) * nA * KP, acoef + static_cast<size_t>(i) * nA * NLM, rc,
            rcinv, dx, dy, dz);
          const float3 fji = angular_edge_force<KM, NAM, LMAX, true, FAST>(
            p, sm + (t2 * T + t1) * nA * KP, acoef + static_cast<size_t>(j) * nA * NLM, rc,
            rcinv, -dx, -dy, -dz);
          a12 = make_float4(fij.x, fij.y, fij.z, 0.0f);
          a21 = make_float4(fji.x, fji.y, fji.z, 0.0f);
        }
      } else {
        const int j = ja;
        site_displacement(b, sites, xi, yi, zi, j, dx, dy, dz, t2);
        a12 = f12[static_cast<size_t>(i) * mn_a + k];
        // reverse slot: i inside j's ascending row
        const int* jrow = nl_a + static_cast<size_t>(j) * mn_a;
        const int nj = nn_a[j];
        int lo = 0, hi = nj - 1;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (__ldg(jrow + mid) < i) lo = mid + 1; else hi = mid;
        }
        a21 = f12[static_cast<size_t>(j) * mn_a + lo];
        if (nj == 0 || __ldg(jrow + lo) != i) {
          // only a truncated (overflowed) row can lose the reverse edge
          a21 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          atomicOr(&st->overflow, 4);
        }
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
#pragma unroll
  for (int c = 0; c < 3; ++c) F[c] = group_sum<G>(F[c]);
#pragma unroll
  for (int c = 0; c < 9; ++c) W[c] = group_sum<G>(W[c]);
  ezbl = group_sum<G>(ezbl);
  if (active && gl == 0) {
    const double e = pe_ann[i] + static_cast<double>(ezbl);
    const bool finite = isfinite(e) && isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]);
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

// shape classes: small (n_max <= 4, basis_size <= 8) and general
constexpr int kSmallN = 5, kSmallK = 9;
// Models with l_max 5..8 run one general-shape instance of each kernel (LMAX
// 8): their moments take 80 floats per n, so the descriptor and a-coefficient
// kernels take 16 centers per CTA (groups of 8 lanes), the force kernels 4.
constexpr int kHighFusedGroup = 8, kHighGroup = 4;

bool high_degree(const ModelParams& p) { return p.L_max > 4; }

// every kernel of a model uses one basis stride, so high-degree models take
// the general shape throughout
bool small_shape(const ModelParams& p)
{
  return !high_degree(p) && p.nR <= kSmallN && p.nA <= kSmallN && p.kR <= kSmallK &&
         p.kA <= kSmallK;
}

template <int G, int NRM, int KM, int NAM, bool XR, int LMAX, int MINB, bool TC, bool FF = false>
void launch_fused_t(Engine& e, int N, cudaStream_t s)
{
  NeighborBuffers& nb = e.nbr;
  constexpr int APB = kBlock / G;
  const int blocks = (N + APB - 1) / APB;
  const size_t smem = fused_layout(e.params, APB, (KM + 3) & ~3, fused_smem_budget(MINB), TC,
                                   fused_prefetch(XR, MINB))
                        .total_bytes;
  k_nep_fused<G, NRM, KM, NAM, XR, LMAX, MINB, TC, FF><<<blocks, kBlock, smem, s>>>(
    e.params, N, e.d_box, e.scratch.sites, e.d_nstate, nb.nn_v, nb.nl_v, nb.mn_v, nb.nn_r, nb.nl_r,
    nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a, e.xr.er, e.xr.ea, e.scratch.qrad, e.scratch.alpha,
    e.scratch.acoef, e.scratch.f12, e.scratch.pe_ann);
}

// The mixed precisions take the FAST builds of the filter, angular-force and
// gather kernels (and of the descriptor kernel, whose tensor-core build is
// FAST); they exist for the small shape, the others run the exact build.
inline bool fast_math(const Engine& e) { return e.precision != 0; }

template <int G, int NRM, int KM, bool FAST>
void launch_filter_tf(Engine& e, int N, cudaStream_t s)
{
  NeighborBuffers& nb = e.nbr;
  constexpr int APB = kBlock / G, KP = (KM + 3) & ~3;
  const ModelParams& p = e.params;
  const int blocks = (N + APB - 1) / APB;
  if (filter_bins(p, KP)) {
    const size_t smem =
      sizeof(float) * (filter_table_floats(p, KP) + 4 * kBlock * filter_bin_float4(p, KP));
    k_filter_radial<G, NRM, KM, true, FAST><<<blocks, kBlock, smem, s>>>(
      p, N, e.d_box, e.scratch.sites, e.d_nstate, nb.nn_v, nb.nl_v, nb.mn_v, nb.nn_r, nb.nl_r,
      nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a, e.scratch.qrad);
  } else {
    const size_t smem = sizeof(float) * filter_table_floats(p, KP);
    k_filter_radial<G, NRM, KM, false, FAST><<<blocks, kBlock, smem, s>>>(
      p, N, e.d_box, e.scratch.sites, e.d_nstate, nb.nn_v, nb.nl_v, nb.mn_v, nb.nn_r, nb.nl_r,
      nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a, e.scratch.qrad);
  }
}

template <int G, int NRM, int KM>
void launch_filter_t(Engine& e, int N, cudaStream_t s)
{
  if constexpr (KM == kSmallK) {
    if (fast_math(e)) {
      launch_filter_tf<G, NRM, KM, true>(e, N, s);
      return;
    }
  }
  launch_filter_tf<G, NRM, KM, false>(e, N, s);
}

template <int G, int KM, int NAM, int LMAX, bool FAST>
void launch_f12_tf(Engine& e, int N, cudaStream_t s)
{
  NeighborBuffers& nb = e.nbr;
  constexpr int APB = kBlock / G;
  const int blocks = (N + APB - 1) / APB;
  const size_t smem =
    sizeof(float) * e.params.T * e.params.T * e.params.nA * ((KM + 3) & ~3);
  if (e.use_xr)
    k_angular_f12<G, KM, NAM, true, LMAX, FAST><<<blocks, kBlock, smem, s>>>(
      e.params, N, e.d_box, e.scratch.sites, nb.nn_a, nb.nl_a, nb.mn_a, e.xr.ea, e.xr.large,
      e.scratch.acoef, e.scratch.f12);
  else
    k_angular_f12<G, KM, NAM, false, LMAX, FAST><<<blocks, kBlock, smem, s>>>(
      e.params, N, e.d_box, e.scratch.sites, nb.nn_a, nb.nl_a, nb.mn_a, e.xr.ea, e.xr.large,
      e.scratch.acoef, e.scratch.f12);
}

template <int G, int KM, int NAM, int LMAX>
void launch_f12_t(Engine& e, int N, cudaStream_t s)
{
  if constexpr (KM == kSmallK && LMAX == 4) {
    if (fast_math(e)) {
      launch_f12_tf<G, KM, NAM, LMAX, true>(e, N, s);
      return;
    }
  }
  launch_f12_tf<G, KM, NAM, LMAX, false>(e, N, s);
}

// FFI: the build also comes with the fused angular force (small shape)
template <int G, int NRM, int KM, int NAM, int LMAX, int MINB, bool TC, bool FFI = false>
void set_fused_smem_t(const ModelParams& p)
{
  auto bytes = [&](bool xr) {
    return fused_layout(p, kBlock / G, (KM + 3) & ~3, fused_smem_budget(MINB), TC,
                        fused_prefetch(xr, MINB))
      .total_bytes;
  };
  cudaFuncSetAttribute(k_nep_fused<G, NRM, KM, NAM, false, LMAX, MINB, TC, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes(false));
  cudaFuncSetAttribute(k_nep_fused<G, NRM, KM, NAM, true, LMAX, MINB, TC, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes(true));
  if constexpr (FFI)
    cudaFuncSetAttribute(k_nep_fused<G, NRM, KM, NAM, false, LMAX, MINB, TC, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes(false));
}

template <int G, int KM, int NAM, bool XR, int LMAX, int GMINB, bool FAST>
void launch_gather_tf(Engine& e, int N, double* pe, double* force, double* virial,
                      bool accumulate, cudaStream_t s)
{
  NeighborBuffers& nb = e.nbr;
  const int threads = 256;
  const int blocks = static_cast<int>((static_cast<long long>(N) * G + threads - 1) / threads);
  const size_t smem =
    XR ? sizeof(float) * e.params.T * e.params.T * e.params.nA * ((KM + 3) & ~3) : 0;
  k_gather<G, KM, NAM, XR, LMAX, GMINB, FAST><<<blocks, threads, smem, s>>>(
    e.params, N, e.d_box, e.scratch.sites, nb.nn_r, nb.nl_r, nb.mn_r, nb.nn_a, nb.nl_a, nb.mn_a,
    e.xr.er, e.xr.ea, e.scratch.acoef, e.scratch.alpha, e.scratch.f12, e.xr.large,
    e.scratch.pe_ann, pe,
    force, virial, accumulate ? 1 : 0, e.d_nstate);
}

template <int G, int KM, int NAM, bool XR, int LMAX, int GMINB = 0>
void launch_gather_t(Engine& e, int N, double* pe, double* force, double* virial,
                     bool accumulate, cudaStream_t s)
{
  if constexpr (KM == kSmallK && LMAX == 4) {
    if (fast_math(e)) {
      // the FAST builds are held to their occupancy: two CTAs per SM on
      // explicit rows, three for the uncapped Verlet-row build (it takes 84
      // registers unheld, which the 8-register allocation unit rounds to 88:
      // two CTAs of 256, and 1.5x the time)
      constexpr int fast_minb = XR ? 2 : (GMINB == 0 ? 3 : GMINB);
      launch_gather_tf<G, KM, NAM, XR, LMAX, fast_minb, true>(e, N, pe, force, virial,
                                                              accumulate, s);
      return;
    }
  }
  launch_gather_tf<G, KM, NAM, XR, LMAX, GMINB, false>(e, N, pe, force, virial, accumulate, s);
}

// the FP32 build or, for the mixed precisions, the tensor-core one
template <int G, int NRM, int KM, int NAM, int LMAX, int MINB>
void launch_fused_g(Engine& e, int N, cudaStream_t s)
{
  const bool tc = e.precision != 0;
  if (e.use_xr) {
    if (tc) launch_fused_t<G, NRM, KM, NAM, true, LMAX, MINB, true>(e, N, s);
    else launch_fused_t<G, NRM, KM, NAM, true, LMAX, MINB, false>(e, N, s);
  } else {
    if (tc) launch_fused_t<G, NRM, KM, NAM, false, LMAX, MINB, true>(e, N, s);
    else launch_fused_t<G, NRM, KM, NAM, false, LMAX, MINB, false>(e, N, s);
  }
}

// the small shape at 3 or 4 CTAs per SM (Engine::fused_minb, autotuned; the
// tensor-core build comes at 3)
template <int G>
void launch_fused_small(Engine& e, int N, cudaStream_t s)
{
  if (!e.use_xr && e.fuse_f12) {
    constexpr int n = kSmallN, k = kSmallK;
    if (e.precision != 0) launch_fused_t<G, n, k, n, false, 4, 3, true, true>(e, N, s);
    else if (e.fused_minb == 4) launch_fused_t<G, n, k, n, false, 4, 4, false, true>(e, N, s);
    else launch_fused_t<G, n, k, n, false, 4, 3, false, true>(e, N, s);
    return;
  }
  if (e.fused_minb == 4 && e.precision == 0) {
    if (e.use_xr) launch_fused_t<G, kSmallN, kSmallK, kSmallN, true, 4, 4, false>(e, N, s);
    else launch_fused_t<G, kSmallN, kSmallK, kSmallN, false, 4, 4, false>(e, N, s);
  } else {
    launch_fused_g<G, kSmallN, kSmallK, kSmallN, 4, 3>(e, N, s);
  }
}

template <int G, int KM, int NAM, int LMAX>
void launch_gather_g(Engine& e, int N, double* pe, double* force, double* virial,
                     bool accumulate, cudaStream_t s)
{
  if (e.use_xr) launch_gather_t<G, KM, NAM, true, LMAX, 0>(e, N, pe, force, virial, accumulate, s);
  else if (LMAX == 4 && e.gather_minb == 4)
    launch_gather_t<G, KM, NAM, false, LMAX, 4>(e, N, pe, force, virial, accumulate, s);
  else launch_gather_t<G, KM, NAM, false, LMAX, 0>(e, N, pe, force, virial, accumulate, s);
}

}  // namespace

#include "invariants_upload.inc"

// Padded basis width (row stride of the coefficient tables and of alpha).
int basis_stride(const ModelParams& p) { return small_shape(p) ? round4(kSmallK) : round4(kMaxBasis); }

bool fused_occupancy_variants(const ModelParams& p) { return small_shape(p); }

// Largest dynamic shared memory a descriptor-kernel variant this model runs needs.
size_t fused_smem_bytes(const ModelParams& p)
{
  if (high_degree(p))
    return fused_layout(p, kBlock / kHighFusedGroup, basis_stride(p), fused_smem_budget(2), false,
                        true)
      .total_bytes;
  return fused_layout(p, kBlock / 4, basis_stride(p), fused_smem_budget(small_shape(p) ? 3 : 2),
                      false, true)
    .total_bytes;
}

void set_fused_smem_limits(const ModelParams& p)
{
  // the tensor-core builds' layout needs the 16-bit tile sizes of the current
  // precision (set before this is called again by nepx_set_precision)
  const bool tc = p.tc_dimk > 0;
  if (high_degree(p)) {
    set_fused_smem_t<kHighFusedGroup, kMaxN, kMaxBasis, kMaxN, 8, 2, false>(p);
    if (tc) set_fused_smem_t<kHighFusedGroup, kMaxN, kMaxBasis, kMaxN, 8, 2, true>(p);
    return;
  }
  if (small_shape(p)) {
    set_fused_smem_t<4, kSmallN, kSmallK, kSmallN, 4, 3, false, true>(p);
    set_fused_smem_t<8, kSmallN, kSmallK, kSmallN, 4, 3, false, true>(p);
    set_fused_smem_t<4, kSmallN, kSmallK, kSmallN, 4, 4, false, true>(p);
    set_fused_smem_t<8, kSmallN, kSmallK, kSmallN, 4, 4, false, true>(p);
    if (tc) {
      set_fused_smem_t<4, kSmallN, kSmallK, kSmallN, 4, 3, true, true>(p);
      set_fused_smem_t<8, kSmallN, kSmallK, kSmallN, 4, 3, true, true>(p);
    }
  } else {
    set_fused_smem_t<4, kMaxN, kMaxBasis, kMaxN, 4, 2, false>(p);
    set_fused_smem_t<8, kMaxN, kMaxBasis, kMaxN, 4, 2, false>(p);
    if (tc) {
      set_fused_smem_t<4, kMaxN, kMaxBasis, kMaxN, 4, 2, true>(p);
      set_fused_smem_t<8, kMaxN, kMaxBasis, kMaxN, 4, 2, true>(p);
    }
  }
}

size_t fused_tc_smem_bytes(const ModelParams& p)
{
  if (high_degree(p))
    return fused_layout(p, kBlock / kHighFusedGroup, basis_stride(p), fused_smem_budget(2), true,
                        true)
      .total_bytes;
  return fused_layout(p, kBlock / 4, basis_stride(p), fused_smem_budget(small_shape(p) ? 3 : 2),
                      true, true)
    .total_bytes;
}

void launch_filter(Engine& e, int N, cudaStream_t s)
{
  const bool small = small_shape(e.params);
  if (e.filter_group == 8) {
    if (small) launch_filter_t<8, kSmallN, kSmallK>(e, N, s);
    else launch_filter_t<8, kMaxN, kMaxBasis>(e, N, s);
  } else {
    if (small) launch_filter_t<4, kSmallN, kSmallK>(e, N, s);
    else launch_filter_t<4, kMaxN, kMaxBasis>(e, N, s);
  }
}

// The descriptor kernel evaluates the angular partial forces itself (small
// shape, Verlet rows, when the autotuner picked it).
bool fused_angular_force(const Engine& e)
{
  return e.fuse_f12 && !e.use_xr && small_shape(e.params);
}

void launch_descriptor(Engine& e, int N, const double*, const int*, cudaStream_t stream)
{
  const bool small = small_shape(e.params);
  const bool high = high_degree(e.params);
  if (!e.use_xr) launch_filter(e, N, stream);
  if (high) launch_fused_g<kHighFusedGroup, kMaxN, kMaxBasis, kMaxN, 8, 2>(e, N, stream);
  else if (e.group == 8) {
    if (small) launch_fused_small<8>(e, N, stream);
    else launch_fused_g<8, kMaxN, kMaxBasis, kMaxN, 4, 2>(e, N, stream);
  } else {
    if (small) launch_fused_small<4>(e, N, stream);
    else launch_fused_g<4, kMaxN, kMaxBasis, kMaxN, 4, 2>(e, N, stream);
  }
  // a single explicit-row system: the gather evaluates both directed angular
  // forces itself; a batch's structures that are not small take f12 here
  if (e.use_xr && e.xr.from_box) return;
  if (fused_angular_force(e)) return;   // the descriptor kernel wrote f12
  if (high) launch_f12_t<kHighGroup, kMaxBasis, kMaxN, 8>(e, N, stream);
  else if (e.f12_group == 8) {
    if (small) launch_f12_t<8, kSmallK, kSmallN, 4>(e, N, stream);
    else launch_f12_t<8, kMaxBasis, kMaxN, 4>(e, N, stream);
  } else {
    if (small) launch_f12_t<4, kSmallK, kSmallN, 4>(e, N, stream);
    else launch_f12_t<4, kMaxBasis, kMaxN, 4>(e, N, stream);
  }
}

void launch_gather(Engine& e, int N, const double*, const int*, double* pe, double* force,
                   double* virial, bool accumulate, cudaStream_t stream)
{
  const bool small = small_shape(e.params);
  if (high_degree(e.params))
    launch_gather_g<kHighGroup, kMaxBasis, kMaxN, 8>(e, N, pe, force, virial, accumulate, stream);
  else if (e.gather_group == 4) {
    if (small) launch_gather_g<4, kSmallK, kSmallN, 4>(e, N, pe, force, virial, accumulate, stream);
    else launch_gather_g<4, kMaxBasis, kMaxN, 4>(e, N, pe, force, virial, accumulate, stream);
  } else {
    if (small) launch_gather_g<8, kSmallK, kSmallN, 4>(e, N, pe, force, virial, accumulate, stream);
    else launch_gather_g<8, kMaxBasis, kMaxN, 4>(e, N, pe, force, virial, accumulate, stream);
  }
}

void launch_force(Engine& e, int N, const double* pos, const int* type, double* pe,
                  double* force, double* virial, bool accumulate, cudaStream_t stream)
{
  launch_descriptor(e, N, pos, type, stream);
  launch_gather(e, N, pos, type, pe, force, virial, accumulate, stream);
}

}  // namespace nepx

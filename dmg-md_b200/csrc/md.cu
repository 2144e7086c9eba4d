// md.cu -- device-resident molecular dynamics: velocity Verlet in FP64 with
// the reference's ensembles (NVE, Berendsen / Nose-Hoover chain / Bussi
// NVT, Berendsen and stochastic-cell-rescaling NPT with the reference's
// isotropic coupling, plus anisotropic and triclinic couplings).
//
// Step order of the reference's single-rank loop (src/runtime.cu:747-848):
//   [NHC: scale v by the pre-force chain factor]
//   half kick + drift + wrap -> NEP force -> half kick -> thermo reduction
//   -> thermostat velocity factor -> barostat box factor -> scale v (and x, box)
// Every stage is a kernel on one stream; the thermostat / barostat scalars
// are computed on the device from the FP64 thermo sums, with the stochastic
// draws generated ahead on the host from the reference's random stream
// (svr_rng.h).  A step therefore never synchronises with the host, and a run
// replays CUDA graphs of captured steps (eight, then single ones) back to
// back.  The large-box path's skin check runs inside the first half kick.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/nepx.h"
#include "handle.h"
#include "md.h"
#include "nhc.h"

struct MdMirror {
  nepx::Box box;
  int status;
  nepx::NeighborState nstate;
};

struct nepx_md {
  nepx::Md md;
  MdMirror* mirror = nullptr;   // pinned host copy of the device status
  nepx_handle* pot = nullptr;
  double* h_noise = nullptr;   // pinned staging of the stochastic draws
  double* h_rows = nullptr;    // pinned staging of the thermo rows (rows_cap rows)
  double* pending_thermo = nullptr;   // the caller's row buffer, filled by md_finish
  int pending_rows = 0;
  cudaEvent_t noise_copied = nullptr;
  // one-step calls replay one graph: draws' upload, the call's scalar kernel,
  // the step and the publish; re-captured when any of its inputs changes
  cudaGraphExec_t graph_call = nullptr;
  struct CallKey {
    nepx::StepParams p;
    int precision, init, rows;
    double T0, tau;
    const void* bufs[5];
  } call_key{};
  bool own_stream = false;
  std::string error;
};

namespace nepx {

void launch_force(Engine& e, int N, const double* pos, const int* type, double* pe,
                  double* force, double* virial, bool accumulate, cudaStream_t stream);

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double box_volume(const Box& b)
{
  return fabs(b.h[0] * (b.h[4] * b.h[8] - b.h[5] * b.h[7]) +
              b.h[1] * (b.h[5] * b.h[6] - b.h[3] * b.h[8]) +
              b.h[2] * (b.h[3] * b.h[7] - b.h[4] * b.h[6]));
}

// block sum of 8 doubles per thread into partials[blockIdx.x * 8 + q]
__device__ __forceinline__ void block_reduce8(double* v, double* partials)
{
  __shared__ double s[kThreads / 32][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], off);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 8; ++q) s[warp][q] = v[q];
  __syncthreads();
  if (threadIdx.x < 8) {
    double acc = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) acc += s[w][threadIdx.x];
    partials[blockIdx.x * 8 + threadIdx.x] = acc;
  }
}

// Pre-force kinetic sum (NHC only): partials[b*8 + 0] = sum m v^2.
__global__ void k_ke_partials(int N, const double* __restrict__ mass,
                              const double* __restrict__ vel, double* partials)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i < N) {
    const double vx = vel[i], vy = vel[N + i], vz = vel[2 * N + i];
    v[0] = mass[i] * (vx * vx + vy * vy + vz * vz);
  }
  block_reduce8(v, partials);
}


__device__ __forceinline__ double target_temperature(const StepParams& p, long long step)
{
  const double fraction = static_cast<double>(step) / static_cast<double>(p.steps);
  return p.T0 + (p.T1 - p.T0) * fraction;
}

// Time step of the current step: the run's dt, or with an adaptive step
// min(dt, max_dist / max|v|) over the velocities at the start of the step
// (reference adaptive_time_step, runtime.cu:594-619).
__device__ __forceinline__ double step_dt(const StepParams& p, const MdScalars* sc)
{
  if (p.max_dist <= 0.0) return p.dt;
  const double v2 = __longlong_as_double(static_cast<long long>(sc->vmax2));
  const double limited = v2 == 0.0 ? p.dt : p.max_dist / sqrt(v2);
  return limited < p.dt ? limited : p.dt;
}

// max |v|^2 over the atoms (adaptive time step): a block maximum, then an
// integer atomicMax on the bits (ordered like the values for doubles >= 0)
__global__ void k_vmax(int N, const double* __restrict__ vel, MdScalars* sc)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v2 = 0.0;
  if (i < N) {
    const double vx = vel[i], vy = vel[N + i], vz = vel[2 * N + i];
    v2 = vx * vx + vy * vy + vz * vz;
  }
  for (int off = 16; off > 0; off >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, off));
  if ((threadIdx.x & 31) == 0 && v2 > 0.0)
    atomicMax(&sc->vmax2, static_cast<unsigned long long>(__double_as_longlong(v2)));
}

__global__ void k_nhc_pre(StepParams p, MdScalars* sc, const double* __restrict__ partials,
                          int nblocks)
{
  double ek2 = 0.0;
  for (int b = 0; b < nblocks; ++b) ek2 += partials[b * 8];
  const double kT = kBoltzmann * target_temperature(p, sc->step);
  // before_force hands over the kinetic energy (ek2/2) and doubles it again
  // (ensemble_control.cpp:186-198)
  sc->vfactor_pre = nhc_half_step(sc->nhc_pos, sc->nhc_mom, sc->nhc_mass, ek2 * 0.5 * 2.0, kT,
                                  3.0 * p.N, step_dt(p, sc) * 0.5);
}

// Skin check of the large-box neighbour path, done by k_vv1 on the new
// positions (enabled = 0: explicit rows, nothing to check).
struct SkinArgs {
  const int* type;
  const double* x0;
  NeighborState* st;
  Site* sites;
  double skin, rc_v;
  int enabled;
};

// v = v * f_pre + F/m dt/2 ; x += v dt ; wrap into the cell
// (runtime.cu:392-421, runtime_internal.hpp:648-681); then the skin check
// of the new position.
// With unwrapped != nullptr the unwrapped positions gain this step's
// displacement, new minus old position before the wrap (reference
// update_unwrapped, runtime.cu:423-438).
__global__ void k_vv1(StepParams p, const Box* __restrict__ box, const double* __restrict__ mass,
                      const double* __restrict__ force, double* pos, double* vel,
                      const MdScalars* __restrict__ sc, SkinArgs sk, double* unwrapped)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.N) return;
  const int N = p.N;
  const double f = sc->vfactor_pre;
  const double dt = step_dt(p, sc);
  const double half = dt * 0.5;
  const double im = 1.0 / mass[i];
  double r[3];
  for (int d = 0; d < 3; ++d) {
    const double v = vel[d * N + i] * f + force[d * N + i] * im * half;
    vel[d * N + i] = v;
    const double x0 = pos[d * N + i];
    r[d] = x0 + v * dt;
    if (unwrapped) unwrapped[d * N + i] += r[d] - x0;
  }
  const Box& b = *box;
  double s[3];
  for (int d = 0; d < 3; ++d) {
    s[d] = b.hinv[3 * d] * r[0] + b.hinv[3 * d + 1] * r[1] + b.hinv[3 * d + 2] * r[2];
    if (b.pbc[d] == 1) {
      if (s[d] < 0.0) s[d] += 1.0;
      else if (s[d] > 1.0) s[d] -= 1.0;
    }
  }
  double x[3];
  for (int d = 0; d < 3; ++d) {
    x[d] = b.h[3 * d] * s[0] + b.h[3 * d + 1] * s[1] + b.h[3 * d + 2] * s[2];
    pos[d * N + i] = x[d];
  }
  if (sk.enabled)
    skin_check_atom(N, i, b, x[0], x[1], x[2], sk.type[i], sk.x0, sk.st, sk.sites, sk.skin,
                    sk.rc_v, 0);
}

// second half kick and the FP64 thermo partial sums (runtime.cu:442-493)
__global__ void k_vv2_thermo(StepParams p, const double* __restrict__ mass,
                             const double* __restrict__ force, double* vel,
                             const double* __restrict__ pe, const double* __restrict__ virial,
                             double* partials, const MdScalars* __restrict__ sc)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = p.N;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (i < N) {
    const double half = step_dt(p, sc) * 0.5;
    const double m = mass[i];
    const double im = 1.0 / m;
    double vv[3];
    for (int d = 0; d < 3; ++d) {
      vv[d] = vel[d * N + i] + force[d * N + i] * im * half;
      vel[d * N + i] = vv[d];
    }
    v[0] = m * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
    v[1] = pe[i];
    v[2] = virial[i] + m * vv[0] * vv[0];
    v[3] = virial[N + i] + m * vv[1] * vv[1];
    v[4] = virial[2 * N + i] + m * vv[2] * vv[2];
    v[5] = virial[3 * N + i] + m * vv[0] * vv[1];
    v[6] = virial[4 * N + i] + m * vv[0] * vv[2];
    v[7] = virial[5 * N + i] + m * vv[1] * vv[2];
  }
  block_reduce8(v, partials);
}

// 3x3 products and inverse, row-major.
__device__ inline void mat3_mul(const double* a, const double* b, double* c)
{
  double t[9];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q)
      t[3 * r + q] = a[3 * r] * b[q] + a[3 * r + 1] * b[3 + q] + a[3 * r + 2] * b[6 + q];
  for (int k = 0; k < 9; ++k) c[k] = t[k];
}

__device__ inline bool mat3_inverse(const double* a, double* inv)
{
  const double c0 = a[4] * a[8] - a[5] * a[7];
  const double c1 = a[5] * a[6] - a[3] * a[8];
  const double c2 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c0 + a[1] * c1 + a[2] * c2;
  if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
  const double id = 1.0 / det;
  inv[0] = c0 * id;
  inv[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  inv[3] = c1 * id;
  inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  inv[6] = c2 * id;
  inv[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  return true;
}

// true when a periodic direction of the box is not thicker than t
__device__ inline bool box_thinner_than(const Box& b, double t)
{
  const double V = fabs(box_volume(b));
  for (int d = 0; d < 3; ++d) {
    if (!b.pbc[d]) continue;
    // thickness along d = V / |a_e x a_f|, a the cell vectors (columns of h)
    const int e = (d + 1) % 3, f = (d + 2) % 3;
    const double cx = b.h[3 + e] * b.h[6 + f] - b.h[6 + e] * b.h[3 + f];
    const double cy = b.h[6 + e] * b.h[f] - b.h[e] * b.h[6 + f];
    const double cz = b.h[e] * b.h[3 + f] - b.h[3 + e] * b.h[f];
    if (V / sqrt(cx * cx + cy * cy + cz * cz) <= t) return true;
  }
  return false;
}

// Per-component pressure coupling (the reference has only the isotropic
// one).  With the pressure tensor P (xx yy zz yz xz xy), targets P0 and
// couplings c = 1 / (3 tau_p C) (C the component's modulus):
//   Berendsen  mu_aa = 1 - c_a (P0_a - P_aa);  mu_ab = mu_ba = -c_ab (P0_ab - P_ab)
//   SCR        the same drift plus sqrt(2 c kT / V) eta on each diagonal strain
//              ln h_aa and sqrt(c kT / V) eta on each symmetric shear (the
//              fluctuation-dissipation pairing of each strain with its work
//              conjugate; with equal couplings and one shared draw the
//              volume fluctuation equals the isotropic formula's)
// and h' = mu h, positions with it.  Returns false on a non-positive or
// non-finite deformation.
__device__ bool apply_component_coupling(const StepParams& p, Box& b, const double* th,
                                         double V, double Tt, const double* eta, double* mu,
                                         NeighborState* nstate)
{
  const double P6[6] = {th[2], th[3], th[4], th[7], th[6], th[5]};
  const int nc = p.baro == kBaroAniso ? 3 : 6;
  const int slot[6][2] = {{0, 0}, {4, 4}, {8, 8}, {5, 7}, {2, 6}, {1, 3}};
  for (int c = 0; c < nc; ++c) {
    double m = -p.pc6[c] * (p.p6[c] - P6[c]);
    if (p.kind == kNptScr)
      m += sqrt((c < 3 ? 2.0 : 1.0) * p.pc6[c] * kBoltzmann * Tt / V) * eta[c];
    mu[slot[c][0]] += m;
    if (slot[c][1] != slot[c][0]) mu[slot[c][1]] += m;
  }
  for (int k = 0; k < 9; ++k)
    if (!isfinite(mu[k])) return false;
  if (!(mu[0] > 0.0 && mu[4] > 0.0 && mu[8] > 0.0)) return false;
  double h[9], hinv[9];
  mat3_mul(mu, b.h, h);
  if (!mat3_inverse(h, hinv)) return false;
  for (int k = 0; k < 9; ++k) {
    b.h[k] = h[k];
    b.hinv[k] = hinv[k];
    b.fh[k] = static_cast<float>(h[k]);
    b.fh[9 + k] = static_cast<float>(hinv[k]);
  }
  b.ortho = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 &&
            h[7] == 0.0;
  mat3_mul(mu, nstate->box_def, nstate->box_def);
  return true;
}

// Thermo normalisation, thermostat and barostat scalars, box update and the
// thermo row of this step (ensemble_control.cpp:180-306, npt_scr.cpp:21-33,
// box_control.cpp:9-68).  One block of 8 warps: warp q reduces quantity q
// of the block partials (lane l takes blocks l, l + 32, ..., then a fixed
// shuffle tree: a fixed order, so the sums are reproducible), thread 0 does
// the scalar work.
constexpr int kEnsembleThreads = 256;
__global__ void __launch_bounds__(kEnsembleThreads)
k_ensemble(StepParams p, Box* box, MdScalars* sc, const double* __restrict__ partials,
           int nblocks, const double* __restrict__ noise, double* rows, int rows_cap,
           NeighborState* nstate, int* status)
{
  __shared__ double s_sum[8];
  {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int b = lane; b < nblocks; b += 32) acc += partials[b * 8 + q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) s_sum[q] = acc;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const long long step = sc->step;
  const double dt = step_dt(p, sc);
  Box& b = *box;
  const double V = box_volume(b);
  double th[8];
  th[0] = s_sum[0] / (3.0 * p.N * kBoltzmann);
  th[1] = s_sum[1];
  for (int q = 2; q < 8; ++q) th[q] = s_sum[q] / V;
  for (int q = 0; q < 8; ++q) sc->thermo[q] = th[q];
  const double Tt = target_temperature(p, step);
  double vf = 1.0, bf = 1.0;
  const long long local = step - sc->step0;   // step within this call
  const double* nz = noise + kNoisePerStep * local;
  switch (p.kind) {
    case kNvtBer:
    case kNptBer: {
      const double coupling = 1.0 / p.Tdamp;
      if (coupling > 1.0e-5) vf = sqrt(1.0 + coupling * (Tt / th[0] - 1.0));
      break;
    }
    case kNvtNhc: {
      const double ek2 = th[0] * (3.0 * p.N * kBoltzmann);
      vf = nhc_half_step(sc->nhc_pos, sc->nhc_mom, sc->nhc_mass, ek2, kBoltzmann * Tt, 3.0 * p.N,
                         dt * 0.5);
      break;
    }
    case kNvtBdp:
    case kNptScr: {
      const int ndeg = 3 * p.N;
      const double old_ke = th[0] * ndeg * kBoltzmann * 0.5;
      const double sigma = ndeg * kBoltzmann * Tt * 0.5;
      const double new_ke = resample_kinetic(old_ke, sigma, ndeg, p.bdp_factor, nz[0], nz[1]);
      vf = sqrt(new_ke / old_ke);
      break;
    }
    default:
      break;
  }
  const bool npt = p.kind == kNptBer || p.kind == kNptScr;
  for (int k = 0; k < 9; ++k) sc->mu[k] = (k % 4 == 0) ? 1.0 : 0.0;
  if (npt && p.baro != kBaroIso) {
    if (!apply_component_coupling(p, b, th, V, Tt, nz + 2, sc->mu, nstate)) *status |= 2;
    else if (p.large_box && box_thinner_than(b, p.thick_min)) *status |= 4;
  } else if (npt) {
    const double p_inst = (th[2] + th[3] + th[4]) * 0.3333333333333333;
    bf = 1.0 - p.pc * (p.p_target - p_inst);
    if (p.kind == kNptScr)
      bf += sqrt(0.666666666666667 * p.pc * kBoltzmann * Tt / V) * nz[2];
    if (!(bf > 0.0) || !isfinite(bf)) {
      *status |= 2;
      bf = 1.0;
    } else if (bf != 1.0) {
      b.h[0] *= bf;
      b.h[4] *= bf;
      b.h[8] *= bf;
      const double det = b.h[0] * b.h[4] * b.h[8];
      b.hinv[0] = b.h[4] * b.h[8] / det;
      b.hinv[4] = b.h[0] * b.h[8] / det;
      b.hinv[8] = b.h[0] * b.h[4] / det;
      for (int k = 0; k < 9; ++k) {
        b.fh[k] = static_cast<float>(b.h[k]);
        b.fh[9 + k] = static_cast<float>(b.hinv[k]);
      }
      nstate->box_scale *= bf;
    }
  }
  if (!(vf > 0.0) || !isfinite(vf)) {
    *status |= 1;
    vf = 1.0;
  }
  sc->vfactor = vf;
  sc->bfactor = bf;
  if (p.thermo_every > 0 && (local + 1) % p.thermo_every == 0) {
    const long long row = (local + 1) / p.thermo_every - 1;
    if (row < rows_cap) {
      double* r = rows + row * kThermoCols;
      r[0] = th[0];
      r[1] = 1.5 * p.N * kBoltzmann * th[0];
      r[2] = th[1];
      r[3] = th[2] * kPressureUnit;
      r[4] = th[3] * kPressureUnit;
      r[5] = th[4] * kPressureUnit;
      r[6] = th[7] * kPressureUnit;
      r[7] = th[6] * kPressureUnit;
      r[8] = th[5] * kPressureUnit;
      const int cols[9] = {0, 3, 6, 1, 4, 7, 2, 5, 8};
      for (int k = 0; k < 9; ++k) r[9 + k] = b.h[cols[k]];
      r[18] = vf;
      r[19] = bf;
    }
  }
  sc->step = step + 1;
  sc->vfactor_pre = 1.0;
  sc->time += dt;
  sc->vmax2 = 0ull;   // the next step's k_vmax starts from zero
}

// v *= velocity factor; under a box change x and the Verlet reference x0
// scale with the box
__global__ void k_scale(int N, double* vel, double* pos, double* x0,
                        const MdScalars* __restrict__ sc)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double vf = sc->vfactor, bf = sc->bfactor;
  if (vf != 1.0)
    for (int d = 0; d < 3; ++d) vel[d * N + i] *= vf;
  if (bf != 1.0)
    for (int d = 0; d < 3; ++d) {
      pos[d * N + i] *= bf;
      x0[d * N + i] *= bf;
    }
  const double* mu = sc->mu;
  if (mu[0] != 1.0 || mu[1] != 0.0 || mu[2] != 0.0 || mu[3] != 0.0 || mu[4] != 1.0 ||
      mu[5] != 0.0 || mu[6] != 0.0 || mu[7] != 0.0 || mu[8] != 1.0) {
    double* arrs[2] = {pos, x0};
    for (double* a : arrs) {
      const double x = a[i], y = a[N + i], z = a[2 * N + i];
      a[i] = mu[0] * x + mu[1] * y + mu[2] * z;
      a[N + i] = mu[3] * x + mu[4] * y + mu[5] * z;
      a[2 * N + i] = mu[6] * x + mu[7] * y + mu[8] * z;
    }
  }
}

__global__ void k_init_scalars(MdScalars* sc, StepParams p, double T0, double tau)
{
  sc->step = 0;
  sc->step0 = 0;
  sc->time = 0.0;
  sc->vmax2 = 0ull;
  sc->vfactor_pre = 1.0;
  sc->vfactor = 1.0;
  sc->bfactor = 1.0;
  for (int k = 0; k < 9; ++k) sc->mu[k] = (k % 4 == 0) ? 1.0 : 0.0;
  // Nose-Hoover chain start (thermostat_nhc.cpp:25-41)
  const double kT = kBoltzmann * T0;
  for (int m = 0; m < kChain; ++m) {
    sc->nhc_pos[m] = 0.0;
    sc->nhc_mom[m] = (m % 2 == 0) ? 1.0 : -1.0;
    sc->nhc_mass[m] = kT * tau * tau;
  }
  sc->nhc_mass[0] *= 3.0 * p.N;
}

}  // namespace

// One MD step on the md's stream (captured into a graph by md_run).
void md_enqueue_step(Md& md, const StepParams& p, int* d_status)
{
  Engine& e = *md.engine;
  const int N = md.N;
  const int blocks = (N + kThreads - 1) / kThreads;
  cudaStream_t s = md.stream;
  if (p.max_dist > 0.0) k_vmax<<<blocks, kThreads, 0, s>>>(N, md.d_vel, md.d_sc);
  if (p.kind == kNvtNhc) {
    k_ke_partials<<<blocks, kThreads, 0, s>>>(N, md.d_mass, md.d_vel, md.d_partials);
    k_nhc_pre<<<1, 1, 0, s>>>(p, md.d_sc, md.d_partials, blocks);
  }
  const SkinArgs sk{md.d_type, e.nbr.x0, e.d_nstate, e.scratch.sites, e.skin,
                    static_cast<double>(e.model.rc_max) + e.skin, e.use_xr ? 0 : 1};
  k_vv1<<<blocks, kThreads, 0, s>>>(p, e.d_box, md.d_mass, md.d_force, md.d_pos, md.d_vel, md.d_sc,
                                    sk, p.unwrapped ? md.d_unwrapped : nullptr);
  launch_neighbor_update(e, N, md.d_pos, md.d_type, false, s, sk.enabled != 0);
  launch_force(e, N, md.d_pos, md.d_type, md.d_pe, md.d_force, md.d_virial, false, s);
  k_vv2_thermo<<<blocks, kThreads, 0, s>>>(p, md.d_mass, md.d_force, md.d_vel, md.d_pe,
                                          md.d_virial, md.d_partials, md.d_sc);
  k_ensemble<<<1, kEnsembleThreads, 0, s>>>(p, e.d_box, md.d_sc, md.d_partials, blocks,
                                            md.d_noise, md.d_rows, md.rows_cap, e.d_nstate,
                                            d_status);
  k_scale<<<blocks, kThreads, 0, s>>>(N, md.d_vel, md.d_pos, e.nbr.x0, md.d_sc);
}

// A call that continues a segment: thermostat state and segment step carry
// over; per-call buffers (draws, thermo rows) restart at this step.
__global__ void k_mark_call(MdScalars* sc) { sc->step0 = sc->step; }

void md_continue_scalars(Md& md) { k_mark_call<<<1, 1, 0, md.stream>>>(md.d_sc); }

// End of a call: the box, the status word, the neighbour state and the thermo
// rows, written straight into pinned host memory (device-addressable under
// unified addressing) -- one launch in place of four small copies.
__global__ void k_publish(const Box* __restrict__ box, const int* __restrict__ status,
                          const NeighborState* __restrict__ nstate, Box* h_box, int* h_status,
                          NeighborState* h_nstate, const double* __restrict__ rows, double* h_rows,
                          int n_vals)
{
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x == 0) {
    constexpr int kBoxWords = sizeof(Box) / sizeof(int);
    constexpr int kStateWords = sizeof(NeighborState) / sizeof(int);
    static_assert(sizeof(Box) % sizeof(int) == 0 && sizeof(NeighborState) % sizeof(int) == 0,
                  "word copies");
    const int* b = reinterpret_cast<const int*>(box);
    const int* n = reinterpret_cast<const int*>(nstate);
    for (int k = threadIdx.x; k < kBoxWords; k += blockDim.x) reinterpret_cast<int*>(h_box)[k] = b[k];
    for (int k = threadIdx.x; k < kStateWords; k += blockDim.x)
      reinterpret_cast<int*>(h_nstate)[k] = n[k];
    if (threadIdx.x == 0) *h_status = *status;
  }
  for (int k = tid; k < n_vals; k += gridDim.x * blockDim.x) h_rows[k] = rows[k];
}

void launch_publish(const Engine& e, const Md& md, const int* d_status, Box* h_box,
                    int* h_status, NeighborState* h_nstate, double* h_rows, int rows)
{
  const int n_vals = rows * kThermoCols;
  const int blocks = std::max(1, std::min(148, (n_vals + 255) / 256));
  k_publish<<<blocks, 256, 0, md.stream>>>(e.d_box, d_status, e.d_nstate, h_box, h_status,
                                           h_nstate, md.d_rows, h_rows, n_vals);
}

void md_init_scalars(Md& md, const StepParams& p, double T0, double tau)
{
  k_init_scalars<<<1, 1, 0, md.stream>>>(md.d_sc, p, T0, tau);
}

}  // namespace nepx

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

namespace {

int md_fail(nepx_md* m, int code, const std::string& msg)
{
  if (m) m->error = msg;
  return code;
}

int md_cuda(nepx_md* m, const char* what)
{
  const cudaError_t err = cudaGetLastError();
  return md_fail(m, NEPX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

template <typename T>
bool dalloc(T*& p, size_t n)
{
  return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)) ==
         cudaSuccess;
}

// Pinned host memory that kernels write directly: mapped into the device's
// address space under the same pointer (unified addressing), checked here.
template <typename T>
bool pinned_mapped(T*& p, size_t count)
{
  p = nullptr;
  if (cudaHostAlloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T),
                    cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return false;
  void* dp = nullptr;
  if (cudaHostGetDevicePointer(&dp, p, 0) != cudaSuccess || dp != p) {
    cudaFreeHost(p);
    p = nullptr;
    return false;
  }
  return true;
}

// The captured graphs hold the draw, row and status buffers' addresses as
// kernel and copy parameters: dropped (and captured again on the next run)
// whenever one of those buffers is reallocated.
void drop_graphs(nepx_md* m)
{
  for (cudaGraphExec_t* x : {&m->md.graph, &m->md.graph_multi, &m->graph_call}) {
    if (*x) cudaGraphExecDestroy(*x);
    *x = nullptr;
  }
}

int* status_buffer(nepx_md* m)
{
  // one int of device status behind the partials (allocated with them)
  return reinterpret_cast<int*>(m->md.d_partials + 8 * static_cast<size_t>(m->md.partial_blocks));
}

}  // namespace

extern "C" {

int nepx_md_create(nepx_t* pot, int n, const int* h_type, const double* h_mass,
                   const double* h_pos, const double* h_vel, const nepx_box* box, void* stream,
                   nepx_md_t** out)
{
  if (!pot || !h_type || !h_mass || !h_pos || !h_vel || !box || !out || n < 1)
    return NEPX_ERR_ARG;
  *out = nullptr;
  nepx::Engine& e = pot->engine;
  if (n > e.capacity) return NEPX_ERR_CAPACITY;
  for (int i = 0; i < n; ++i)
    if (h_type[i] < 0 || h_type[i] >= e.model.num_types || !(h_mass[i] > 0.0))
      return NEPX_ERR_ARG;
  auto* m = new (std::nothrow) nepx_md();
  if (!m) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  md.engine = &e;
  md.N = n;
  m->pot = pot;
  if (!nepx::make_box(box->h, box->pbc, md.box).empty()) {
    delete m;
    return NEPX_ERR_BOX;
  }
  // small boxes run on explicit rows rebuilt every step (the reference's
  // small-box path); the choice is made here for the whole trajectory
  const int kind = nepx::box_kind(e, md.box);
  if (kind < 0) {
    delete m;
    return NEPX_ERR_BOX;
  }
  md.xr = kind == 1 || !nepx::large_box_ok(e, md.box);
  if (md.xr && !nepx::engine_enable_xr(e, 1).empty()) {
    delete m;
    return NEPX_ERR_CUDA;
  }
  if (stream) {
    md.stream = static_cast<cudaStream_t>(stream);
  } else if (cudaStreamCreateWithFlags(&md.stream, cudaStreamNonBlocking) == cudaSuccess) {
    m->own_stream = true;
  }
  md.partial_blocks = (n + 255) / 256;
  bool ok = md.stream != nullptr;
  ok = ok && dalloc(md.d_type, n) && dalloc(md.d_mass, n) && dalloc(md.d_pos, 3 * size_t(n)) &&
       dalloc(md.d_vel, 3 * size_t(n)) && dalloc(md.d_force, 3 * size_t(n)) &&
       dalloc(md.d_pe, n) && dalloc(md.d_virial, 9 * size_t(n)) &&
       dalloc(md.d_partials, 8 * size_t(md.partial_blocks) + 2) && dalloc(md.d_sc, 1);
  ok = ok && cudaEventCreateWithFlags(&m->noise_copied, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && pinned_mapped(m->mirror, 1);
  if (ok) {
    std::memset(m->mirror, 0, sizeof(MdMirror));
    m->mirror->box = md.box;
  }
  if (ok) {
    // velocities arrive in A/fs; the engine integrates in natural units
    std::vector<double> v(h_vel, h_vel + 3 * size_t(n));
    for (double& x : v) x *= nepx::kTimeUnit;
    ok = cudaMemcpy(md.d_type, h_type, sizeof(int) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(md.d_mass, h_mass, sizeof(double) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(md.d_pos, h_pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(md.d_vel, v.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(status_buffer(m), 0, sizeof(int)) == cudaSuccess;
  }
  if (!ok) {
    nepx_md_destroy(m);
    return NEPX_ERR_CUDA;
  }
  *out = m;
  return NEPX_OK;
}

int nepx_md_destroy(nepx_md_t* m)
{
  if (!m) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  if (md.stream) cudaStreamSynchronize(md.stream);
  drop_graphs(m);
  void* ptrs[] = {md.d_type, md.d_mass,  md.d_pos,  md.d_vel,  md.d_force,    md.d_pe,
                  md.d_virial, md.d_partials, md.d_sc, md.d_noise, md.d_rows, md.d_unwrapped};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (m->h_noise) cudaFreeHost(m->h_noise);
  if (m->h_rows) cudaFreeHost(m->h_rows);
  if (m->mirror) cudaFreeHost(m->mirror);
  if (m->noise_copied) cudaEventDestroy(m->noise_copied);
  if (md.engine && md.engine->box_owner == &md) md.engine->box_owner = nullptr;
  if (m->own_stream && md.stream) cudaStreamDestroy(md.stream);
  delete m;
  return NEPX_OK;
}

const char* nepx_md_last_error(const nepx_md_t* m) { return m ? m->error.c_str() : "null handle"; }

int nepx_md_set_barostat(nepx_md_t* m, int coupling, const double* pressure_gpa,
                         const double* modulus_gpa)
{
  if (!m) return NEPX_ERR_ARG;
  nepx::EnsembleConfig& c = m->md.ens;
  if (c.kind != nepx::kNptBer && c.kind != nepx::kNptScr)
    return md_fail(m, NEPX_ERR_ARG, "set an NPT ensemble before its barostat coupling");
  if (coupling == NEPX_BARO_ISOTROPIC) {
    c.baro = nepx::kBaroIso;
    return NEPX_OK;
  }
  if (coupling != NEPX_BARO_ANISOTROPIC && coupling != NEPX_BARO_TRICLINIC)
    return md_fail(m, NEPX_ERR_ARG, "unknown barostat coupling");
  if (!pressure_gpa || !modulus_gpa) return md_fail(m, NEPX_ERR_ARG, "pressures or moduli missing");
  const int nc = coupling == NEPX_BARO_ANISOTROPIC ? 3 : 6;
  for (int k = 0; k < nc; ++k)
    if (!std::isfinite(pressure_gpa[k]) || !(modulus_gpa[k] > 0.0))
      return md_fail(m, NEPX_ERR_ARG, "barostat needs finite pressures and moduli > 0");
  c.baro = coupling == NEPX_BARO_ANISOTROPIC ? nepx::kBaroAniso : nepx::kBaroTri;
  for (int k = 0; k < 6; ++k) {
    c.p6_gpa[k] = k < nc ? pressure_gpa[k] : 0.0;
    c.c6_gpa[k] = k < nc ? modulus_gpa[k] : 1.0e300;   // uncoupled: no deformation
  }
  return NEPX_OK;
}

int nepx_md_set_ensemble(nepx_md_t* m, int kind, const double* params, unsigned seed)
{
  if (!m || kind < nepx::kNVE || kind > nepx::kNptScr) return NEPX_ERR_ARG;
  nepx::EnsembleConfig c;
  c.kind = kind;
  if (kind != nepx::kNVE) {
    if (!params) return md_fail(m, NEPX_ERR_ARG, "ensemble parameters missing");
    c.T0 = params[0];
    c.T1 = params[1];
    c.Tdamp = params[2];
    if (!(c.T0 > 0.0) || !(c.T1 > 0.0) || !(c.Tdamp >= 1.0))
      return md_fail(m, NEPX_ERR_ARG, "ensemble needs T0 > 0, T1 > 0 and Tdamp >= 1");
    if (kind == nepx::kNptBer || kind == nepx::kNptScr) {
      c.p_gpa = params[3];
      c.bulk_gpa = params[4];
      c.tau_p = params[5];
      if (!std::isfinite(c.p_gpa) || !(c.bulk_gpa > 0.0) || !(c.tau_p >= 1.0))
        return md_fail(m, NEPX_ERR_ARG, "NPT needs finite P, B > 0 and tau_p >= 1");
      // the box requirements of the coupling are checked when a run starts
    }
  }
  c.seed = seed;
  m->md.ens = c;
  m->md.rng = nepx::SvrRng(seed);
  return NEPX_OK;
}

}  // extern "C"

namespace {

// Enqueues `steps` steps on the md stream; nothing waits for the device.
int md_enqueue_run(nepx_md* m, int steps, double dt_fs, int thermo_every, double* h_thermo,
                   int first_step, int segment_steps)
{
  if (!m || steps < 1 || !(dt_fs >= 0.0) || thermo_every < 0) return NEPX_ERR_ARG;
  if (first_step < 0 || segment_steps < first_step + steps) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  nepx::Engine& e = *md.engine;
  const nepx::EnsembleConfig& c = md.ens;
  const int N = md.N;
  if (c.kind == nepx::kNptBer || c.kind == nepx::kNptScr) {
    const nepx::Box& b = md.box;
    if (!b.pbc[0] || !b.pbc[1] || !b.pbc[2])
      return md_fail(m, NEPX_ERR_UNSUPPORTED, "NPT needs a box periodic in all directions");
    if (c.baro == nepx::kBaroIso && !b.ortho)
      return md_fail(m, NEPX_ERR_UNSUPPORTED,
                     "isotropic NPT needs an orthogonal box (use a triclinic coupling)");
  }
  e.use_xr = md.xr;
  e.xr.from_box = true;
  nepx::StepParams p{};
  p.N = N;
  p.kind = c.kind;
  p.steps = segment_steps;
  p.thermo_every = thermo_every;
  p.dt = dt_fs / nepx::kTimeUnit;
  p.T0 = c.T0;
  p.T1 = c.T1;
  p.Tdamp = c.Tdamp;
  p.rc_v = e.model.rc_max + e.skin;
  p.skin = e.skin;
  p.max_dist = md.max_dist;
  p.unwrapped = md.d_unwrapped ? 1 : 0;
  if (p.max_dist > 0.0 && c.kind != nepx::kNVE && c.kind != nepx::kNvtBer)
    return md_fail(m, NEPX_ERR_UNSUPPORTED,
                   "the adaptive time step runs with nve and nvt_ber only, as in the reference");
  if (c.kind == nepx::kNptBer || c.kind == nepx::kNptScr) {
    p.p_target = c.p_gpa / nepx::kPressureUnit;
    // form pc in 1/GPa, then convert once (ensemble_control.cpp:84-95)
    p.pc = c.bulk_gpa > 2000.0 ? 0.0 : 1.0 / (3.0 * c.tau_p * c.bulk_gpa);
    p.pc *= nepx::kPressureUnit;
    p.baro = c.baro;
    for (int k = 0; k < 6; ++k) {
      p.p6[k] = c.p6_gpa[k] / nepx::kPressureUnit;
      p.pc6[k] = c.c6_gpa[k] > 2000.0 ? 0.0 : nepx::kPressureUnit / (3.0 * c.tau_p * c.c6_gpa[k]);
    }
    p.large_box = md.xr ? 0 : 1;
    p.thick_min = 2.5 * (e.model.rc_radial_max + 1.0);
  }
  p.bdp_factor = c.Tdamp > 0.1 ? std::exp(-1.0 / c.Tdamp) : 0.0;
  cudaStream_t s = md.stream;
  // stochastic draws of every step, in the reference's consumption order
  if (steps > md.noise_cap) {
    cudaStreamSynchronize(s);
    if (md.d_noise) cudaFree(md.d_noise);
    if (m->h_noise) cudaFreeHost(m->h_noise);
    drop_graphs(m);   // they hold the old buffers' addresses
    md.d_noise = nullptr;
    m->h_noise = nullptr;
    if (!dalloc(md.d_noise, nepx::kNoisePerStep * size_t(steps)) ||
        cudaMallocHost(reinterpret_cast<void**>(&m->h_noise),
                       sizeof(double) * nepx::kNoisePerStep * steps) != cudaSuccess)
      return md_cuda(m, "allocate noise buffers");
    md.noise_cap = steps;
  } else {
    cudaEventSynchronize(m->noise_copied);   // previous upload has left the staging buffer
  }
  const bool stochastic_v = c.kind == nepx::kNvtBdp || c.kind == nepx::kNptScr;
  const int box_draws = c.kind != nepx::kNptScr ? 0
                        : c.baro == nepx::kBaroIso ? 1 : (c.baro == nepx::kBaroAniso ? 3 : 6);
  for (int k = 0; k < steps; ++k) {
    double* z = m->h_noise + nepx::kNoisePerStep * k;
    for (int q = 0; q < nepx::kNoisePerStep; ++q) z[q] = 0.0;
    if (stochastic_v) {
      z[0] = md.rng.gasdev();
      z[1] = md.rng.sumnoises(3 * N - 1);
    }
    for (int q = 0; q < box_draws; ++q) z[2 + q] = md.rng.gasdev();
  }
  // a one-step call uploads its draws inside the call graph
  const bool fold = steps == 1;
  if (!fold) {
    cudaMemcpyAsync(md.d_noise, m->h_noise, sizeof(double) * nepx::kNoisePerStep * steps,
                    cudaMemcpyHostToDevice, s);
    cudaEventRecord(m->noise_copied, s);
  }
  const int rows = thermo_every > 0 ? steps / thermo_every : 0;
  if (rows > md.rows_cap) {
    cudaStreamSynchronize(s);
    if (md.d_rows) cudaFree(md.d_rows);
    if (m->h_rows) cudaFreeHost(m->h_rows);
    drop_graphs(m);   // they hold the old buffers' addresses
    md.d_rows = nullptr;
    m->h_rows = nullptr;
    if (!dalloc(md.d_rows, size_t(rows) * nepx::kThermoCols) ||
        !pinned_mapped(m->h_rows, size_t(rows) * nepx::kThermoCols))
      return md_cuda(m, "allocate rows");
    md.rows_cap = rows;
  }
  // the device box is authoritative while this md owns the engine; it is
  // re-uploaded only after the handle served another caller
  if (e.box_owner != &md) {
    nepx::launch_set_box(e, md.box, s);
    e.box_owner = &md;
    // the engine served another caller: its Verlet rows belong to that system
    if (md.forces_valid) nepx::launch_neighbor_update(e, N, md.d_pos, md.d_type, true, s);
  }
  const double tau = p.dt * c.Tdamp;
  if (!fold) {
    if (first_step == 0) nepx::md_init_scalars(md, p, c.T0, tau);
    else nepx::md_continue_scalars(md);
  }
  if (!md.forces_valid) {
    nepx::launch_neighbor_update(e, N, md.d_pos, md.d_type, true, s);
    if (!e.tuned) nepx::engine_autotune(e, N, md.d_pos, md.d_type, s);
    nepx::launch_force(e, N, md.d_pos, md.d_type, md.d_pe, md.d_force, md.d_virial, false, s);
    md.forces_valid = true;
  }
  e.force_rebuild = true;     // a later nepx_compute on this handle rebuilds
  e.have_box = false;
  int* d_status = status_buffer(m);
  // capture one step, and kGraphSteps steps back to back, as graphs (the step
  // counter lives on the device, so consecutive steps are the same kernels;
  // re-captured when the per-run constants change)
  if (!md.graph || std::memcmp(&p, &md.graph_params, sizeof(p)) != 0 ||
      md.graph_precision != e.precision) {
    for (cudaGraphExec_t* x : {&md.graph, &md.graph_multi}) {
      if (*x) cudaGraphExecDestroy(*x);
      *x = nullptr;
    }
    for (int reps : {1, nepx::kGraphSteps}) {
      cudaGraph_t g;
      if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return md_cuda(m, "begin capture");
      for (int r = 0; r < reps; ++r) nepx::md_enqueue_step(md, p, d_status);
      if (cudaStreamEndCapture(s, &g) != cudaSuccess) return md_cuda(m, "end capture");
      cudaGraphExec_t& x = reps == 1 ? md.graph : md.graph_multi;
      if (cudaGraphInstantiate(&x, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return md_cuda(m, "instantiate graph");
      }
      cudaGraphDestroy(g);
    }
    md.graph_params = p;
    md.graph_precision = e.precision;
  }
  // device-side status, box, neighbour flags and thermo rows land in pinned memory
  const int publish_rows = h_thermo ? rows : 0;
  if (fold) {
    nepx_md::CallKey key{};
    key.p = p;
    key.precision = e.precision;
    key.init = first_step == 0;
    key.rows = publish_rows;
    key.T0 = c.T0;
    key.tau = tau;
    key.bufs[0] = m->h_noise;
    key.bufs[1] = md.d_noise;
    key.bufs[2] = m->h_rows;
    key.bufs[3] = md.d_rows;
    key.bufs[4] = m->mirror;
    if (!m->graph_call || std::memcmp(&key, &m->call_key, sizeof(key)) != 0) {
      if (m->graph_call) cudaGraphExecDestroy(m->graph_call);
      m->graph_call = nullptr;
      cudaGraph_t g;
      if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return md_cuda(m, "begin capture");
      cudaMemcpyAsync(md.d_noise, m->h_noise, sizeof(double) * nepx::kNoisePerStep,
                      cudaMemcpyHostToDevice, s);
      if (key.init) nepx::md_init_scalars(md, p, c.T0, tau);
      else nepx::md_continue_scalars(md);
      nepx::md_enqueue_step(md, p, d_status);
      nepx::launch_publish(e, md, d_status, &m->mirror->box, &m->mirror->status,
                           &m->mirror->nstate, m->h_rows, publish_rows);
      if (cudaStreamEndCapture(s, &g) != cudaSuccess) return md_cuda(m, "end capture");
      if (cudaGraphInstantiate(&m->graph_call, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        m->graph_call = nullptr;
        return md_cuda(m, "instantiate graph");
      }
      cudaGraphDestroy(g);
      m->call_key = key;
    }
    if (cudaGraphLaunch(m->graph_call, s) != cudaSuccess) return md_cuda(m, "graph launch");
    // the staging buffer of the draws is free again once the graph has run
    cudaEventRecord(m->noise_copied, s);
  } else {
    int k = 0;
    for (; k + nepx::kGraphSteps <= steps; k += nepx::kGraphSteps)
      if (cudaGraphLaunch(md.graph_multi, s) != cudaSuccess) return md_cuda(m, "graph launch");
    for (; k < steps; ++k)
      if (cudaGraphLaunch(md.graph, s) != cudaSuccess) return md_cuda(m, "graph launch");
    nepx::launch_publish(e, md, d_status, &m->mirror->box, &m->mirror->status,
                         &m->mirror->nstate, m->h_rows, publish_rows);
  }
  m->pending_thermo = publish_rows > 0 ? h_thermo : nullptr;
  m->pending_rows = publish_rows;
  if (cudaPeekAtLastError() != cudaSuccess) return md_cuda(m, "enqueue run");
  return NEPX_OK;
}

// A bounded device wait that gave up: the tensor-core ANN's MMAs, or a grid
// barrier of the neighbour rebuild (whose counters are then reset before the
// next rebuild).
int wait_errors(nepx_md* m, const nepx::NeighborState& st)
{
  if (st.ann_error)
    return md_fail(m, NEPX_ERR_CUDA, "a tensor-core ANN tile timed out waiting for its MMAs");
  if (st.sync_error) {
    m->md.engine->nbr.gsync_dirty = true;
    m->md.forces_valid = false;
    return md_fail(m, NEPX_ERR_CUDA, "the neighbour-list rebuild timed out at a grid-wide barrier");
  }
  return NEPX_OK;
}

int md_finish(nepx_md* m)
{
  nepx::Md& md = m->md;
  if (cudaStreamSynchronize(md.stream) != cudaSuccess) return md_cuda(m, "run");
  if (m->pending_thermo) {
    std::memcpy(m->pending_thermo, m->h_rows,
                sizeof(double) * size_t(m->pending_rows) * nepx::kThermoCols);
    m->pending_thermo = nullptr;
  }
  md.box = m->mirror->box;
  const int status = m->mirror->status;
  const nepx::NeighborState& st = m->mirror->nstate;
  if (status & 1) return md_fail(m, NEPX_ERR_NONFINITE, "invalid thermostat velocity factor");
  if (status & 2) return md_fail(m, NEPX_ERR_NONFINITE, "invalid barostat box factor");
  if (status & 4)
    return md_fail(m, NEPX_ERR_BOX, "the barostat made a periodic direction thinner than "
                                    "2.5 (rc + 1): the large-box path no longer applies");
  if (st.overflow) return md_fail(m, NEPX_ERR_OVERFLOW, "a neighbour row exceeded its capacity");
  if (st.nonfinite) return md_fail(m, NEPX_ERR_NONFINITE, "non-finite energy or force");
  if (st.box_error)
    return md_fail(m, NEPX_ERR_BOX, "the box became small in one periodic direction and thicker "
                                    "than 10 rc in another (unsupported, as in the reference)");
  return wait_errors(m, st);
}

}  // namespace

extern "C" {

int nepx_md_run(nepx_md_t* m, int steps, double dt_fs, int thermo_every, double* h_thermo)
{
  const int rc = md_enqueue_run(m, steps, dt_fs, thermo_every, h_thermo, 0, steps);
  if (rc) return rc;
  return md_finish(m);
}

int nepx_md_run_segment(nepx_md_t* m, int steps, double dt_fs, int thermo_every,
                        double* h_thermo, int first_step, int segment_steps)
{
  const int rc = md_enqueue_run(m, steps, dt_fs, thermo_every, h_thermo, first_step,
                                segment_steps);
  if (rc) return rc;
  return md_finish(m);
}

int nepx_md_run_async(nepx_md_t* m, int steps, double dt_fs)
{
  return md_enqueue_run(m, steps, dt_fs, 0, nullptr, 0, steps);
}

int nepx_md_sync(nepx_md_t* m)
{
  if (!m) return NEPX_ERR_ARG;
  return md_finish(m);
}

int nepx_md_get(nepx_md_t* m, double* h_pos, double* h_vel, double* h_force, double* h_pe,
                double* h_virial, nepx_box* box)
{
  if (!m) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  const size_t n = md.N;
  cudaStreamSynchronize(md.stream);
  bool ok = true;
  if (h_pos) ok &= cudaMemcpy(h_pos, md.d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (h_vel) {
    ok &= cudaMemcpy(h_vel, md.d_vel, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost) == cudaSuccess;
    for (size_t k = 0; k < 3 * n; ++k) h_vel[k] /= nepx::kTimeUnit;
  }
  if (h_force) ok &= cudaMemcpy(h_force, md.d_force, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (h_pe) ok &= cudaMemcpy(h_pe, md.d_pe, sizeof(double) * n, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (h_virial) ok &= cudaMemcpy(h_virial, md.d_virial, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost) == cudaSuccess;
  if (box) {
    std::memcpy(box->h, md.box.h, sizeof(double) * 9);
    for (int d = 0; d < 3; ++d) box->pbc[d] = md.box.pbc[d];
  }
  return ok ? NEPX_OK : md_cuda(m, "copy state");
}

int nepx_md_set_velocity(nepx_md_t* m, const double* h_vel)
{
  if (!m || !h_vel) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  const size_t n = md.N;
  std::vector<double> v(h_vel, h_vel + 3 * n);
  for (double& x : v) {
    if (!std::isfinite(x)) return md_fail(m, NEPX_ERR_ARG, "non-finite velocity");
    x *= nepx::kTimeUnit;   // A/fs -> natural units
  }
  if (cudaStreamSynchronize(md.stream) != cudaSuccess ||
      cudaMemcpy(md.d_vel, v.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice) !=
        cudaSuccess)
    return md_cuda(m, "upload velocities");
  return NEPX_OK;
}

int nepx_md_compute_forces(nepx_md_t* m)
{
  if (!m) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  nepx::Engine& e = *md.engine;
  const int N = md.N;
  cudaStream_t s = md.stream;
  e.use_xr = md.xr;
  e.xr.from_box = true;
  bool rebuild = !md.forces_valid;
  if (e.box_owner != &md) {
    nepx::launch_set_box(e, md.box, s);
    e.box_owner = &md;
    rebuild = true;
  }
  nepx::launch_neighbor_update(e, N, md.d_pos, md.d_type, rebuild, s);
  if (!e.tuned) nepx::engine_autotune(e, N, md.d_pos, md.d_type, s);
  nepx::launch_force(e, N, md.d_pos, md.d_type, md.d_pe, md.d_force, md.d_virial, false, s);
  md.forces_valid = true;
  e.force_rebuild = true;     // a later nepx_compute on this handle rebuilds
  e.have_box = false;
  if (cudaMemcpyAsync(&m->mirror->nstate, e.d_nstate, sizeof(nepx::NeighborState),
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return md_cuda(m, "force evaluation");
  const nepx::NeighborState& st = m->mirror->nstate;
  if (st.overflow) return md_fail(m, NEPX_ERR_OVERFLOW, "a neighbour row exceeded its capacity");
  if (st.nonfinite) return md_fail(m, NEPX_ERR_NONFINITE, "non-finite energy or force");
  if (st.box_error)
    return md_fail(m, NEPX_ERR_BOX, "the box is small in one periodic direction and thicker "
                                    "than 10 rc in another (unsupported, as in the reference)");
  return wait_errors(m, st);
}

int nepx_md_neighbor_info(nepx_md_t* m, int* max_radial, int* max_angular)
{
  if (!m) return NEPX_ERR_ARG;
  if (cudaStreamSynchronize(m->md.stream) != cudaSuccess) return md_cuda(m, "synchronise");
  if (max_radial) *max_radial = m->mirror->nstate.call_nn[0];
  if (max_angular) *max_angular = m->mirror->nstate.call_nn[1];
  return NEPX_OK;
}

int nepx_md_set_max_distance(nepx_md_t* m, double max_distance)
{
  if (!m) return NEPX_ERR_ARG;
  if (!(max_distance >= 0.0) || !std::isfinite(max_distance))
    return md_fail(m, NEPX_ERR_ARG, "maximum distance per step should be >= 0");
  m->md.max_dist = max_distance;
  return NEPX_OK;
}

int nepx_md_time(nepx_md_t* m, double* time_fs)
{
  if (!m || !time_fs) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  double t = 0.0;
  if (cudaStreamSynchronize(md.stream) != cudaSuccess ||
      cudaMemcpy(&t, &md.d_sc->time, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return md_cuda(m, "read time");
  *time_fs = t * nepx::kTimeUnit;
  return NEPX_OK;
}

int nepx_md_enable_unwrapped(nepx_md_t* m)
{
  if (!m) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  if (md.d_unwrapped) return NEPX_OK;
  const size_t n = md.N;
  if (cudaStreamSynchronize(md.stream) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&md.d_unwrapped), sizeof(double) * 3 * n) !=
        cudaSuccess) {
    md.d_unwrapped = nullptr;
    return md_cuda(m, "allocate unwrapped positions");
  }
  if (cudaMemcpy(md.d_unwrapped, md.d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice) !=
      cudaSuccess)
    return md_cuda(m, "copy unwrapped positions");
  return NEPX_OK;
}

int nepx_md_get_unwrapped(nepx_md_t* m, double* h_unwrapped)
{
  if (!m || !h_unwrapped) return NEPX_ERR_ARG;
  nepx::Md& md = m->md;
  if (!md.d_unwrapped)
    return md_fail(m, NEPX_ERR_ARG, "unwrapped positions are not enabled (nepx_md_enable_unwrapped)");
  if (cudaStreamSynchronize(md.stream) != cudaSuccess ||
      cudaMemcpy(h_unwrapped, md.d_unwrapped, sizeof(double) * 3 * md.N,
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return md_cuda(m, "copy unwrapped positions");
  return NEPX_OK;
}

int nepx_md_device_state(nepx_md_t* m, double** d_pos, double** d_vel, double** d_force,
                         int** d_type, void** stream)
{
  if (!m) return NEPX_ERR_ARG;
  if (d_pos) *d_pos = m->md.d_pos;
  if (d_vel) *d_vel = m->md.d_vel;
  if (d_force) *d_force = m->md.d_force;
  if (d_type) *d_type = m->md.d_type;
  if (stream) *stream = m->md.stream;
  return NEPX_OK;
}

}  // extern "C"

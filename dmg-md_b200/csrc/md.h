// md.h -- device-resident molecular dynamics on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "engine.h"
#include "svr_rng.h"

namespace nepx {

enum EnsembleKind { kNVE = 0, kNvtBer = 1, kNvtNhc = 2, kNvtBdp = 3, kNptBer = 4, kNptScr = 5 };

// Pressure coupling of the NPT ensembles: the reference's isotropic one, and
// per-component couplings of an orthogonal (xx yy zz) or triclinic
// (xx yy zz yz xz xy) box, which the reference does not have
// (box_control.cpp:14-23 rejects them).
enum BarostatCoupling { kBaroIso = 0, kBaroAniso = 1, kBaroTri = 2 };
constexpr int kNoisePerStep = 8;   // two thermostat draws, up to six barostat draws

// run.in `ensemble` parameters (reference include/dmgmd/run_ir.hpp:12-117):
// T0 -> T1 linear ramp, Tdamp coupling in steps; NPT: target pressure (GPa),
// bulk modulus B (GPa) and pressure coupling tau_p (steps).
struct EnsembleConfig {
  int kind = kNVE;
  double T0 = 0.0, T1 = 0.0, Tdamp = 100.0;
  double p_gpa = 0.0, bulk_gpa = 0.0, tau_p = 1000.0;
  int baro = kBaroIso;
  double p6_gpa[6] = {0, 0, 0, 0, 0, 0};   // component targets, xx yy zz yz xz xy
  double c6_gpa[6] = {0, 0, 0, 0, 0, 0};   // component moduli
  uint32_t seed = 12345678u;   // reference default (ensemble_control.hpp:12-18)
};

constexpr int kChain = 4;      // Nose-Hoover chain length
constexpr int kGraphSteps = 8;   // steps per replay of the multi-step graph
constexpr int kThermoCols = 20;  // thermo.out's 18 columns + velocity and box factors

// Scalars the per-step kernels share, resident on the device.
struct MdScalars {
  long long step;      // step within the current segment
  long long step0;     // segment step at which the current call started
  double vfactor_pre;  // NHC scale applied before the first half kick
  double vfactor;      // thermostat scale after the second half kick
  double bfactor;      // isotropic box scale of this step
  double mu[9];        // box deformation of this step, h' = mu h (component couplings)
  double thermo[8];    // T, PE, stresses xx yy zz xy xz yz (natural units, volume-normalised)
  double nhc_pos[kChain], nhc_mom[kChain], nhc_mass[kChain];
  double time;         // simulated time since the segment's first step (natural units)
  unsigned long long vmax2;   // bits of max |v|^2 this step (adaptive time step; >= 0)
};

// Per-run constants passed by value.
struct StepParams {
  int N;
  int kind;
  int steps;           // segment length (the denominator of the temperature ramp)
  int thermo_every;
  double dt;           // natural time units
  double T0, T1, Tdamp;
  double p_target;     // eV/A^3
  double pc;           // Berendsen pressure coupling, (eV/A^3)^-1
  int baro;            // BarostatCoupling
  int large_box;       // the force path is the large-box one (box must stay thick)
  double p6[6];        // component targets, eV/A^3 (xx yy zz yz xz xy)
  double pc6[6];       // component couplings, (eV/A^3)^-1
  double thick_min;    // thinnest periodic thickness the large-box path accepts
  double bdp_factor;   // exp(-1/Tdamp) (0 when Tdamp <= 0.1)
  double rc_v;         // rc + skin, for the NPT rebuild criterion
  double skin;
  double max_dist;     // adaptive time step: largest displacement per step (A), 0 = off
  int unwrapped;       // accumulate unwrapped positions in the first half kick
};

struct Md {
  Engine* engine = nullptr;
  int N = 0;
  int* d_type = nullptr;
  double *d_mass = nullptr, *d_pos = nullptr, *d_vel = nullptr, *d_force = nullptr;
  double *d_pe = nullptr, *d_virial = nullptr;
  double* d_partials = nullptr;   // [blocks][8]
  int partial_blocks = 0;
  MdScalars* d_sc = nullptr;
  double* d_noise = nullptr;      // [steps][3]
  int noise_cap = 0;
  double* d_rows = nullptr;       // [rows][kThermoCols]
  int rows_cap = 0;
  double* d_scale = nullptr;      // cumulative box scale since the last Verlet build
  double* d_unwrapped = nullptr;  // [3][N] unwrapped positions (dump_xyz unwrapped_position)
  double max_dist = 0.0;          // adaptive time step bound (A), 0 = fixed step
  Box box{};
  EnsembleConfig ens;
  SvrRng rng{12345678u};
  bool forces_valid = false;
  bool xr = false;                // explicit-row (small-box) force path
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;        // one step
  cudaGraphExec_t graph_multi = nullptr;  // kGraphSteps steps back to back
  StepParams graph_params{};
  int graph_precision = -1;       // ANN precision the graph's kernels were captured with
};

}  // namespace nepx

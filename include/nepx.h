/*
 * nepx.h -- C ABI of the B200-native NEP molecular-dynamics engine.
 *
 * Plain pointers and sizes only.  A handle belongs to the CUDA device that is
 * current when it is created; calls on it expect that device to be current
 * (as cuBLAS handles do), and device pointers are memory of that device.
 * Handles are independent: different host threads may use different handles
 * at the same time.  `stream` is a cudaStream_t (NULL = legacy default
 * stream).  Every function returns 0 (NEPX_OK) or a positive
 * NEPX_ERR_* code; nepx_last_error() gives the message.  No function exits
 * the process.
 *
 * Each entry point names the reference (DMG-MD, zhangfeifan21/DMG-MD)
 * interface it replaces.
 */
#ifndef NEPX_H
#define NEPX_H

#ifdef __cplusplus
extern "C" {
#endif

#define NEPX_OK 0
#define NEPX_ERR_ARG 1          /* bad argument (null pointer, n out of range, ...) */
#define NEPX_ERR_FILE 2         /* potential file missing or malformed */
#define NEPX_ERR_UNSUPPORTED 3  /* valid input outside what the engine implements */
#define NEPX_ERR_CUDA 4         /* a CUDA call failed */
#define NEPX_ERR_CAPACITY 5     /* n above the capacity the handle was created with */
#define NEPX_ERR_OVERFLOW 6     /* a neighbour row exceeded MN (raise MN in nep.txt) */
#define NEPX_ERR_NONFINITE 7    /* an energy or force came out NaN/Inf */
#define NEPX_ERR_BOX 8          /* box too thin for the large-box path, or singular */

/* ANN precision (nepx_set_precision) */
#define NEPX_PRECISION_FP32 0        /* FP32 SIMT ANN: the reference's arithmetic */
#define NEPX_PRECISION_MIXED 1       /* ANN on the tensor cores: FP16 operands with per-layer
                                        power-of-two scaling, FP32 accumulation; descriptor and
                                        force kernels with the hardware square root, reciprocal
                                        and sine/cosine approximations */
#define NEPX_PRECISION_MIXED_BF16 2  /* the same with BF16 operands */

/* compute flags */
#define NEPX_ACCUMULATE 1u      /* add into pe/force/virial (the reference's += contract) */
#define NEPX_SYNC_CHECK 2u      /* synchronise the stream and report device-side errors */

typedef struct nepx_handle nepx_t;

/* Periodic box: h is row-major 3x3 with the cell vectors a, b, c as COLUMNS,
 * i.e. h = {ax, bx, cx, ay, by, cy, az, bz, cz} (the reference's
 * Box::cpu_h[0..8], src/gpumd_compat/box.cuh:53-70); pbc[d] = 1 periodic. */
typedef struct nepx_box {
  double h[9];
  int pbc[3];
} nepx_box;

/*
 * Parse a GPUMD-format nep.txt (nep4, nep4_zbl, nep5, nep5_zbl) and size the
 * per-atom scratch for up to max_atoms atoms.
 * Replaces NEP::NEP(const char*, int) (src/gpumd_compat/nep.cu:135-385) and
 * NEP::allocate_workspace (nep.cu:432-451).
 */
int nepx_create(const char* nep_path, int max_atoms, nepx_t** out);

/* Frees the handle and its device memory.  Replaces NEP::~NEP (nep.cu:397). */
int nepx_destroy(nepx_t* handle);

/* Message of the last error of this handle (never NULL).  With handle NULL:
 * why this thread's last nepx_create failed ("null handle" if it did not). */
const char* nepx_last_error(const nepx_t* handle);

/*
 * Model metadata. info[16]: version, num_types, zbl, zbl_flexible, n_max_radial,
 * n_max_angular, basis_radial, basis_angular, l_max, num_L, dim, H,
 * MN_radial, MN_angular (both x1.25 like the reference), has_q bitmask
 * (bit0 q_222 .. bit5 q_134), typewise_zbl.  rc[2*T]: rc_radial[t],
 * rc_angular[t].  Replaces NEP::params() (nep.cuh:200-201).
 */
int nepx_info(const nepx_t* handle, int* info, double* rc);

/*
 * Per-atom energy, force and virial of n atoms in a periodic box.
 *   d_type   n ints, 0-based in potential-file order
 *   d_pos    3n doubles SoA (x[0..n), y[0..n), z[0..n)), Angstrom
 *   d_pe     n doubles, eV
 *   d_force  3n doubles SoA, eV/Angstrom
 *   d_virial 9n doubles SoA, order xx yy zz xy xz yz yx zx zy, eV
 * Outputs are overwritten unless flags has NEPX_ACCUMULATE (then added, the
 * reference's += contract).  The call is asynchronous on `stream`; device
 * errors (row overflow, non-finite output) surface at the next call or
 * immediately with NEPX_SYNC_CHECK.
 * Replaces Potential::compute (src/gpumd_compat/potential.cuh:82-88) as
 * implemented by NEP::compute (nep.cu:2071-2100), large-box path
 * (nep.cu:1120-1280).  Boxes thinner than 2.5 (rc + skin) in a periodic
 * direction take the reference's small-box path (nep.cu:1844-2064).
 */
int nepx_compute(nepx_t* handle, const nepx_box* box, int n, const int* d_type,
                 const double* d_pos, double* d_pe, double* d_force, double* d_virial,
                 unsigned flags, void* stream);

/*
 * nepx_compute for callers that cannot allocate device memory while they run:
 * codes whose start-up hands all device memory to their own pool allocator,
 * and real-time or safety-reviewed drivers that forbid allocator calls after
 * initialisation.  This call allocates no device memory (no cudaMalloc,
 * cudaFree or allocating library routine) and, when it succeeds, no host
 * memory: all per-call scratch comes from one 16 MiB static device array
 * inside the library, held by every GPU that loads it until the process
 * exits.  n is limited by what fits in those 16 MiB for the handle's
 * neighbour capacities (about 6.4 KB per atom for MN_radial 250: some
 * 2,600 atoms); larger n returns NEPX_ERR_CAPACITY.  The handle
 * (nepx_create, max_atoms may be 1) supplies only the model parameters; the
 * handle's device must be current (else NEPX_ERR_ARG).  The ANN always runs
 * in FP32, whatever nepx_set_precision chose for the handle, and only the
 * large-box path is served (a box thinner than 2.5 (rc + skin) in a periodic
 * direction returns NEPX_ERR_BOX).  Errors of an earlier asynchronous
 * nepx_compute on the same handle are returned first, as nepx_compute
 * would.  The first call on a device resolves the array's device address;
 * make it before any stream capture.  Calls share the array: neighbour rows
 * are rebuilt and flags cleared on every call, and calls that overlap on
 * the GPU race.  Synchronises `stream`.  Arguments and outputs as
 * nepx_compute (outputs overwritten); error codes and messages as
 * nepx_compute with NEPX_SYNC_CHECK.
 * This entry point has no counterpart in the reference.
 */
int nepx_compute_noalloc(nepx_t* handle, const nepx_box* box, int n, const int* d_type,
                         const double* d_pos, double* d_pe, double* d_force, double* d_virial,
                         void* stream);

/* Forces a Verlet rebuild at the next compute.  Replaces
 * NEP::notify_box_changed (src/gpumd_compat/nep.cuh:170). */
int nepx_notify_box_changed(nepx_t* handle);

/* Verlet skin in Angstrom (reference default 1.0, neighbor.cuh). */
int nepx_set_skin(nepx_t* handle, double skin);

/*
 * Copies the typewise neighbour rows of the last compute (which = 0 radial,
 * 1 angular) into device buffers: d_nn[n] counts, d_nl[n*mn] row-major, rows
 * ascending.  Test and diagnostics hook; the reference exposes the same rows
 * through NEP::get_NN_radial_ptr / get_NL_radial_ptr (nep.cuh:254-256) in
 * ordinal-major layout.
 */
int nepx_neighbors(nepx_t* handle, int which, int n, int* d_nn, int* d_nl, int mn, void* stream);

/*
 * Largest row seen since the last call (radial, angular, Verlet) and device
 * error bits; synchronises `stream`.  Replaces the neighbor.out occupancy
 * record (nep.cu:1156-1176).
 */
int nepx_neighbor_stats(nepx_t* handle, int* max_radial, int* max_angular, int* max_verlet,
                        void* stream);

/*
 * Per-stage device time of the force path, averaged over `reps` calls after
 * one settling call: ms[0] neighbour update (skin check, conditional
 * rebuild, typewise filter), ms[1] descriptor + ANN + angular partial
 * forces, ms[2] force / virial gather, ms[3] the whole force call.
 * Arguments as nepx_compute.  Replaces the wall-clock log_timing of the
 * reference (src/mpi_runtime.cu:2048-2080) with CUDA events per kernel.
 */
int nepx_profile(nepx_t* handle, const nepx_box* box, int n, const int* d_type,
                 const double* d_pos, double* d_pe, double* d_force, double* d_virial, int reps,
                 double* ms, void* stream);

/* ------------------------------------------------------------------------
 * Molecular dynamics on one GPU (velocity Verlet, FP64 integration).
 * Replaces the single-rank loop run_segment / run_m1_replicated
 * (src/runtime.cu:680-971) with its ensembles (src/ensemble_control.cpp).
 * ---------------------------------------------------------------------- */

typedef struct nepx_md nepx_md_t;

/* ensemble kinds (run.in keywords) */
#define NEPX_NVE 0
#define NEPX_NVT_BER 1   /* Berendsen */
#define NEPX_NVT_NHC 2   /* Nose-Hoover chain, length 4 */
#define NEPX_NVT_BDP 3   /* Bussi-Donadio-Parrinello (stochastic velocity rescaling) */
#define NEPX_NPT_BER 4   /* isotropic Berendsen barostat + Berendsen thermostat */
#define NEPX_NPT_SCR 5   /* isotropic stochastic cell rescaling + BDP thermostat */

/*
 * A system of n atoms driven by `pot` (which must have capacity >= n).
 * Host inputs: types, masses (amu), positions 3n SoA (A), velocities 3n SoA
 * (A/fs, the model.xyz unit).  stream: cudaStream_t to run on (NULL = the
 * engine creates a non-blocking stream).  Replaces the device-atom setup of
 * run_m1_replicated (runtime.cu:855-905).
 */
int nepx_md_create(nepx_t* pot, int n, const int* h_type, const double* h_mass,
                   const double* h_pos, const double* h_vel, const nepx_box* box, void* stream,
                   nepx_md_t** out);
int nepx_md_destroy(nepx_md_t* md);
const char* nepx_md_last_error(const nepx_md_t* md);

/*
 * params (kind != NEPX_NVE): {T0, T1, Tdamp[, P_GPa, B_GPa, tau_p]} as the
 * reference's `ensemble` command (run_parser.cpp:158-315); seed of the
 * stochastic thermostat / barostat stream (reference default 12345678,
 * env DMGMD_ENSEMBLE_SEED).  Replaces EnsembleController
 * (src/ensemble_control.cpp:57-306).
 */
int nepx_md_set_ensemble(nepx_md_t* md, int kind, const double* params, unsigned seed);

/*
 * Pressure coupling of the NPT ensemble set last (nepx_md_set_ensemble
 * selects NEPX_BARO_ISOTROPIC, the reference's only one).  The other two
 * have no counterpart in the reference, which rejects them
 * (src/box_control.cpp:14-23); they follow GPUMD's component syntax:
 *   NEPX_BARO_ANISOTROPIC  pressure_gpa[3], modulus_gpa[3]: xx yy zz
 *   NEPX_BARO_TRICLINIC    pressure_gpa[6], modulus_gpa[6]: xx yy zz yz xz xy
 * Each component a deforms the box by mu_a = 1 - (P0_a - P_a) / (3 tau_p C_a)
 * per step (npt_scr adds its component noise), h' = mu h with positions
 * following; a modulus above 2000 GPa leaves the component uncoupled.  A run
 * needs a box periodic in all three directions (and an orthogonal one for
 * the isotropic coupling); a run whose box becomes thinner than the
 * large-box criterion returns NEPX_ERR_BOX.
 */
#define NEPX_BARO_ISOTROPIC 0
#define NEPX_BARO_ANISOTROPIC 1
#define NEPX_BARO_TRICLINIC 2
int nepx_md_set_barostat(nepx_md_t* md, int coupling, const double* pressure_gpa,
                         const double* modulus_gpa);

/*
 * `steps` steps of dt_fs femtoseconds.  Every thermo_every steps (0 = never)
 * one row of 20 doubles is written to h_thermo (rows = steps / thermo_every,
 * may be NULL): the 18 thermo.out columns (T KE PE sxx syy szz syz sxz sxy
 * ax ay az bx by bz cx cy cz; stresses in GPa) followed by that step's
 * thermostat velocity factor and barostat box factor.  The target
 * temperature ramps from T0 to T1 over the run, as in the reference.
 * Synchronises the md stream before returning.
 */
int nepx_md_run(nepx_md_t* md, int steps, double dt_fs, int thermo_every, double* h_thermo);

/* nepx_md_run without thermo rows and without waiting for the device:
 * consecutive calls queue back to back on the md stream.  Device-side errors
 * are reported by the next nepx_md_sync (or nepx_md_run).  Interleaving
 * nepx_compute on the same potential handle requires nepx_md_sync first. */
int nepx_md_run_async(nepx_md_t* md, int steps, double dt_fs);

/* Part of one segment: steps [first_step, first_step + steps) of a segment of
 * segment_steps steps (the reference's `run segment_steps`).  first_step = 0
 * starts the segment (thermostat state initialised, temperature ramp from
 * T0); later calls continue it (thermostat state kept, ramp continued), so a
 * driver can stop between steps for output without changing the trajectory.
 * Thermo rows count from this call's first step.  nepx_md_run(md, n, ...)
 * equals nepx_md_run_segment(md, n, ..., 0, n). */
int nepx_md_run_segment(nepx_md_t* md, int steps, double dt_fs, int thermo_every,
                        double* h_thermo, int first_step, int segment_steps);
int nepx_md_sync(nepx_md_t* md);

/* Copies the current state to host arrays (any may be NULL); velocities in
 * A/fs; virial 9n in the compute order. */
int nepx_md_get(nepx_md_t* md, double* h_pos, double* h_vel, double* h_force, double* h_pe,
                double* h_virial, nepx_box* box);

/* Replaces the velocities (host [3][n], A/fs), e.g. after a host-side
 * momentum correction.  Replaces DeviceAtoms::upload_velocity as used by
 * correct_device_velocity (src/runtime.cu:620-655). */
int nepx_md_set_velocity(nepx_md_t* md, const double* h_vel);

/* Evaluates energy, forces and virials at the current positions (what the
 * reference does at the start of every run segment, force.compute before the
 * step loop, src/runtime.cu:746); synchronous.  Recomputing at unchanged
 * positions gives the same forces bit for bit. */
int nepx_md_compute_forces(nepx_md_t* md);

/* Largest radial and angular neighbour row of the md's latest force
 * evaluation: the `actual` values of the reference's neighbor.out record
 * (src/gpumd_compat/nep.cu:1156-1176).  Synchronises the md stream. */
int nepx_md_neighbor_info(nepx_md_t* md, int* max_radial, int* max_angular);

/* Adaptive time step: every later step takes dt = min(dt_fs, max_distance /
 * max |v|) over the velocities at the start of the step, computed on the
 * device (reference adaptive_time_step, src/runtime.cu:594-619, `time_step dt
 * max_distance` in run.in).  max_distance in A; 0 turns it off.  Runs with
 * NEPX_NVE and NEPX_NVT_BER only, as in the reference (other ensembles
 * return NEPX_ERR_UNSUPPORTED at run time). */
int nepx_md_set_max_distance(nepx_md_t* md, double max_distance);

/* Simulated time (fs) since the first step of the current segment (the sum
 * of the steps' time steps; with a fixed step, steps * dt).  Replaces the
 * reference's global_time bookkeeping (src/runtime.cu:759-760). */
int nepx_md_time(nepx_md_t* md, double* time_fs);

/* Starts tracking unwrapped positions from the current positions (no-op when
 * already on): each later first half kick adds the step's displacement
 * before the wrap into the box.  Replaces DeviceAtoms::enable_unwrapped and
 * update_unwrapped (src/runtime.cu:80-90, 423-438) behind dump_xyz
 * unwrapped_position. */
int nepx_md_enable_unwrapped(nepx_md_t* md);

/* Copies the unwrapped positions (host [3][n], A); NEPX_ERR_ARG unless
 * enabled. */
int nepx_md_get_unwrapped(nepx_md_t* md, double* h_unwrapped);

/* Device pointers of the state (positions, velocities in natural units,
 * forces, types) and the stream the md runs on. */
int nepx_md_device_state(nepx_md_t* md, double** d_pos, double** d_vel, double** d_force,
                         int** d_type, void** stream);

/*
 * Chooses how the per-atom ANN runs for every later call on this handle
 * (compute, batch, MD, server): NEPX_PRECISION_FP32 (default), or the two
 * ANN contractions as tcgen05 tensor-core MMAs inside the descriptor kernel,
 * over the centers of each CTA (M = 128 hidden units or descriptor
 * components, N = the CTA's 16 or 32 centers), with 16-bit operands and
 * FP32 accumulation: NEPX_PRECISION_MIXED (FP16; W0, w1 (1 - x^2) and each
 * CTA's descriptors scaled by powers of two to use FP16's range) or
 * NEPX_PRECISION_MIXED_BF16.  Descriptors, forces and the rest of the ANN
 * (tanh, energy sum) stay FP32 arithmetic; in the mixed modes the descriptor
 * and force kernels (models with n_max <= 4, basis <= 8, l_max <= 4) take
 * the hardware approximations of 1/sqrt (edge lengths), 1/x and sine/cosine
 * (the cutoff function), 2 ulp or about 4e-7 absolute, in place of the
 * correctly rounded functions the FP32 mode keeps for parity with the
 * reference.  NEPX_ERR_UNSUPPORTED for models with dim >
 * 128 or more than 256 hidden units.  No counterpart in the reference (its
 * ANN is FP32 only).
 */
int nepx_set_precision(nepx_t* handle, int mode);

/*
 * Launch choices of the force kernels, as NEPX_TUNING_FIELDS ints:
 *   [0] lanes per center of the typewise filter (4 or 8)
 *   [1] lanes per center of the descriptor kernel (4 or 8)
 *   [2] CTAs per SM the descriptor kernel is built for (3 or 4; the
 *       tensor-core build runs at 3 whatever is set)
 *   [3] lanes per center of the angular-force kernel (4 or 8)
 *   [4] lanes per center of the gather (4 or 8)
 *   [5] 1: the descriptor kernel evaluates the angular partial forces itself
 *       (models with n_max <= 4, basis <= 8, l_max <= 4, on the Verlet-row
 *       path), 0: k_angular_f12 does
 *   [6] the Verlet-row gather's build (models with l_max <= 4): 3 = unheld
 *       (about 80 registers, three CTAs of 256 per SM), 4 = held to four CTAs
 *       (64 registers, some spills, a third more warps)
 * The first compute of a handle times the variants and keeps the fastest
 * (the autotuner; its picks are shared by the handles of the process and,
 * with NEPX_TUNE_FILE set, kept in that file).  nepx_get_tuning reports the
 * current choices and *tuned = 1 once they are fixed.  nepx_set_tuning fixes
 * them for every later call on the handle (no timing runs), for example to
 * repeat a run's summation order bit for bit; values outside the lists
 * above return NEPX_ERR_ARG.  nepx_set_precision with a new mode lets the
 * autotuner choose again.  No counterpart in the reference (fixed launch
 * shapes).
 */
#define NEPX_TUNING_FIELDS 7
int nepx_get_tuning(nepx_t* handle, int* values, int* tuned);
int nepx_set_tuning(nepx_t* handle, const int* values);

/* ---- many independent structures --------------------------------------- */

/* One structure of a batch: n atoms, consecutive in the batch arrays. */
typedef struct nepx_struct_desc {
  int n;
  nepx_box box;
} nepx_struct_desc;

/*
 * Energy, force and virial of nstruct independent structures in one launch
 * sequence.  The batch arrays hold the structures' atoms back to back, T =
 * sum of descs[s].n atoms: d_type[T], d_pos[3][T] (SoA, stride T), outputs
 * d_pe[T], d_force[3][T], d_virial[9][T] (order as nepx_compute).  Each
 * structure is evaluated as nepx_compute would evaluate it alone, on
 * explicit neighbour rows (any box the reference accepts, small or large),
 * and its results do not depend on the other structures of the batch.  T
 * must not exceed the handle's max_atoms.  No counterpart in the reference
 * (it evaluates one system per process); the per-structure contract is
 * Potential::compute (potential.cuh:82-88).
 */
int nepx_compute_batch(nepx_t* handle, const nepx_struct_desc* descs, int nstruct,
                       const int* d_type, const double* d_pos, double* d_pe, double* d_force,
                       double* d_virial, unsigned flags, void* stream);

/*
 * Serving loop: a worker thread owns the potential handle and a device
 * arena of max_atoms atoms and max_struct structure slots.  Requests are
 * admitted while their device memory fits the server's budget (continuous
 * batching: new requests join between steps while others are mid-segment):
 * each request counts its atoms' bytes (explicit neighbour rows and partial
 * forces at the model's row capacities, descriptor scratch, arena and I/O
 * buffers), a structure slot and the cells of its grid; every step evaluates all
 * resident structures in one launch sequence, runs the NVE velocity-Verlet
 * half steps of the MD segments, and retires finished requests (results
 * copied to the caller's host buffers).  The handle must not be used by the
 * caller while the server exists.  No counterpart in the reference.
 */
typedef struct nepx_server nepx_server_t;

typedef struct nepx_request {
  int n;                  /* atoms */
  nepx_box box;
  const int* type;        /* host [n] */
  const double* pos;      /* host [3][n] */
  int md_steps;           /* 0: single point; > 0: NVE steps after the first force call */
  double dt_fs;           /* MD time step */
  const double* mass;     /* host [n] amu (MD only) */
  const double* vel;      /* host [3][n] A/fs (MD only) */
} nepx_request;

typedef struct nepx_result {
  double* pe;             /* [n] per-atom energy of the final state (eV) */
  double* force;          /* [3][n] */
  double* virial;         /* [9][n] or NULL */
  double* pos;            /* [3][n] final positions (MD) or NULL */
  double* vel;            /* [3][n] final velocities A/fs (MD) or NULL */
  double t_submit, t_admit, t_done;   /* seconds on the server's steady clock */
} nepx_result;

int nepx_server_create(nepx_t* handle, int max_atoms, int max_struct, nepx_server_t** out);
/* The same with the arena sized from a device-memory budget in bytes (at most
 * the handle's max_atoms atoms): requests are admitted while the resident
 * requests' bytes stay within hbm_bytes.  No counterpart in the reference. */
int nepx_server_create_budget(nepx_t* handle, double hbm_bytes, int max_struct,
                              nepx_server_t** out);
/* info[4]: the byte budget, bytes per served atom, bytes per structure slot,
 * mean resident bytes per step. */
int nepx_server_memory(nepx_server_t* server, double* info);
/* Stops the worker after the queued requests are done, then frees the arena. */
int nepx_server_destroy(nepx_server_t* server);
const char* nepx_server_last_error(const nepx_server_t* server);
/* Copies the request's inputs and queues it; *ticket identifies it.  `out`
 * must stay valid until the request is done. */
int nepx_server_submit(nepx_server_t* server, const nepx_request* req, nepx_result* out,
                       long long* ticket);
/* *done = 1 once the results are in `out` (status: the request's own code). */
int nepx_server_poll(nepx_server_t* server, long long ticket, int* done, int* status);
int nepx_server_wait(nepx_server_t* server, long long ticket, int* status);
/* Blocks until every submitted request is done. */
int nepx_server_drain(nepx_server_t* server);
/* stats[8]: requests done, steps run, atom-steps, busy seconds (GPU steps),
 * mean resident atoms per step, mean resident structures per step, current
 * queue length, seconds since creation. */
int nepx_server_stats(nepx_server_t* server, double* stats);
/* Row reuse of MD segments (on by default): a segment admitted while it is on
 * keeps, per atom, the neighbours within the cutoff plus the handle's Verlet
 * skin (small boxes: with their image) and filters them into its rows at each
 * step, rebuilding them when one of its atoms has moved more than skin / 2
 * since the build; the rows are those a fresh build gives.  Off: every step
 * builds every row afresh.  Applies to requests admitted afterwards.  The
 * Verlet idea of Neighbor::find_neighbor_global (neighbor.cu:537-582) for the
 * batched rows; no counterpart in the reference. */
int nepx_server_set_row_reuse(nepx_server_t* server, int on);
/* info[2]: centers whose candidates were (re)built, centers of candidate-
 * keeping structures summed over the steps (reuse = 1 - info[0] / info[1]). */
int nepx_server_rows(nepx_server_t* server, double* info);

#ifdef __cplusplus
}
#endif
#endif

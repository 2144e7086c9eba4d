// engine.h -- state of one nepx handle: the potential on the device, the
// neighbour lists, per-atom scratch, and the launch entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "common.cuh"
#include "model.h"

namespace nepx {

struct NeighborBuffers {
  int mn_v = 0, mn_r = 0, mn_a = 0, pow2_v = 0;
  int* nn_v = nullptr;
  int* nl_v = nullptr;   // [N][mn_v] row-major
  int* nn_r = nullptr;
  int* nl_r = nullptr;   // [N][mn_r]
  int* nn_a = nullptr;
  int* nl_a = nullptr;   // [N][mn_a]
  // the cooperative rebuild kernel: its grid-barrier counters (arrivals,
  // generation), per-block partial sums of the cell scan, its block count
  unsigned* gsync = nullptr;         // [2]
  int* scan_part = nullptr;          // [rebuild_blocks]
  int rebuild_blocks = 0;
  bool gsync_dirty = false;          // a barrier timed out: reset the counters first
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* cell_atoms = nullptr;
  int* cell_of = nullptr;
  Site* cell_sites = nullptr;   // [N] site records in cell order (beside cell_atoms)
  int cell_cap = 0;
  double* x0 = nullptr;  // positions at the last Verlet build (3N SoA)
};

struct ForceScratch {
  Site* sites = nullptr;     // [N] position + type records, packed by the skin check
  float* qrad = nullptr;     // [N][nR] radial descriptors from the typewise filter
  float* alpha = nullptr;    // [N][T][kp] radial force coefficients sum_n dE/dq_n c(ti,t)[n][k]
  float4* f12 = nullptr;     // [N][mn_a] directed angular partial forces
  float* acoef = nullptr;    // [N][nA][24] dE/ds[n][lm] of each center
  double* pe_ann = nullptr;  // [N] site energy of the ANN
  double* tune_out = nullptr;  // [13 N] throw-away outputs of the autotuning calls
};

// Verlet candidates of the explicit rows of a batch (the server's MD
// segments): per center, the structure-local neighbours (small boxes: with
// their image) within the cutoff plus the skin at the last build, in the
// order of the rows.  Each step filters them into the rows; a structure
// rebuilds them when it is new or one of its atoms has moved more than
// skin / 2 since the build.  sflag == nullptr: off (every row built afresh).
struct BatchVerlet {
  const int* sflag = nullptr;      // per structure: bit 1 keeps candidates, bit 2 new (build)
  const double* dmax2 = nullptr;   // per structure: largest squared displacement since the build
  double half_skin2 = 0.0;         // (skin / 2)^2
  float skin = 0.0f;
  int mn = 0;                      // candidates per center
  int* vcnt = nullptr;             // [N] candidates of each center
  int* vrow = nullptr;             // [N][mn]
  double* x0 = nullptr;            // [3][N] positions at the build
};

// Candidate code of a small-box structure: local index (20 bits) and the
// image (4 bits per direction).
constexpr int kCandIndexBits = 20;
constexpr int kCandMaxImages = 16;

// Explicit-row state: the small-box path (one structure, rebuilt from the
// device box at every call) and the batched path (many structures).
struct ExplicitRows {
  float4* er = nullptr;       // [N][mn_r] radial edges (r_ij, packed j | type << 28)
  float4* ea = nullptr;       // [N][mn_a] angular edges
  StructInfo* d_si = nullptr; // [max_struct] structures
  int* d_soff = nullptr;      // [max_struct + 1] first atom of each structure, then the total
  int max_struct = 0;
  int n_struct = 0;
  bool from_box = true;       // one structure whose StructInfo follows the device box
  // cell lists of the large structures of a batch (candidate search)
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* cell_atoms = nullptr;  // [N]
  int* cell_of = nullptr;     // [N], -1: the atom's structure scans all its atoms
  int cell_cap = 0;
  int n_cells = 0;            // cells in use (set with the structure table)
  // [N] 1: the center's structure is not small (a batch only), so its rows
  // hold each neighbour once, ascending, and its angular forces take the
  // directed-f12 scheme of the large-box path
  unsigned char* large = nullptr;
  BatchVerlet bv;
};

struct Engine {
  NepModel model;
  ModelParams params{};
  int capacity = 0;          // atoms the buffers are sized for
  int device = 0;            // the CUDA device current at creation, which owns every buffer
  double skin = 1.0;         // Verlet skin (A), the reference's default
  // device copies of the model
  float* d_params = nullptr; // one allocation holding all parameter blocks
  float* d_rc_r = nullptr;
  float* d_rc_a = nullptr;
  Box* d_box = nullptr;
  NeighborState* d_nstate = nullptr;
  NeighborBuffers nbr;
  ForceScratch scratch;
  ExplicitRows xr;
  bool use_xr = false;       // neighbour rows with explicit displacements (small box, batch)
  int precision = 0;         // 0: FP32 SIMT ANN; 1 / 2: ANN on the tensor cores, FP16 / BF16
  unsigned short* d_w16 = nullptr;   // the 16-bit ANN weights of the mixed path
  // host-side bookkeeping
  Box last_box{};
  bool have_box = false;
  bool force_rebuild = true;
  const void* box_owner = nullptr;   // md whose box the device copy holds (nullptr: none)
  int last_n = -1;
  int group = 4;             // lanes per center in the fused kernel (autotuned)
  int fused_minb = 3;        // CTAs per SM the small-shape fused kernel is built for (autotuned)
  int filter_group = 8;      // lanes per center in the typewise filter (autotuned)
  int f12_group = 4;         // lanes per center in the angular-force kernel (autotuned)
  int gather_group = 8;      // lanes per center in the gather (autotuned)
  int gather_minb = 3;       // Verlet-row gather build: 3 unheld, 4 held to four CTAs (autotuned)
  bool fuse_f12 = false;     // the descriptor kernel evaluates f12 itself (autotuned)
  bool tuned = false;
  std::string error;
};

// Padded basis width of the kernel instance serving this model (row stride
// of the shared-memory coefficient tables and of ForceScratch::alpha).
int basis_stride(const ModelParams& p);
size_t fused_smem_bytes(const ModelParams& p);
// The same for the tensor-core (mixed-precision) build; needs the tc_* fields.
size_t fused_tc_smem_bytes(const ModelParams& p);
// True when the descriptor kernel comes in two occupancy builds (3 or 4 CTAs
// per SM, Engine::fused_minb) for this model's shape.
bool fused_occupancy_variants(const ModelParams& p);
// True when the descriptor kernel writes the angular partial forces itself
// (Engine::fuse_f12 on a small-shape model and Verlet rows): no k_angular_f12.
bool fused_angular_force(const Engine& e);
void set_fused_smem_limits(const ModelParams& p);

// Times each kernel variant on the given system (a few calls each, stream
// synchronised) and keeps the fastest: the lane-group size of the filter,
// descriptor, angular-force and gather kernels, the CTAs per SM of the
// descriptor kernel and of the gather, and whether the descriptor kernel
// evaluates the angular partial forces itself.  The picks are kept per (device, model shape, precision, row
// path, size class log2 N) for every later handle of the process, and in the
// file NEPX_TUNE_FILE names, when set, across runs.  Neighbour rows must be
// current.
void engine_autotune(Engine& e, int N, const double* pos, const int* type, cudaStream_t stream);

// Loads the potential, uploads it and sizes every buffer for max_atoms.
std::string engine_create(Engine& e, const std::string& nep_path, int max_atoms);
void engine_destroy(Engine& e);

// Host-side box: fills hinv, the float copy and the orthogonality flag.
std::string make_box(const double* h, const int* pbc, Box& b);

// True when the box is thick enough for the Verlet-list (large-box) path.
bool large_box_ok(const Engine& e, const Box& b);

// Writes the box to the device copy in stream order.
void launch_set_box(Engine& e, const Box& b, cudaStream_t stream);

// Site packing, skin check and conditional Verlet rebuild.  The force
// launches read positions and types from the packed sites, so every force
// launch follows a neighbour update at the same positions.
// skin_done: the caller has packed the site records and applied the skin
// criterion itself (the MD step does it in its first half kick).
// Blocks of the cooperative neighbour rebuild that fit on the current device
// at once for Verlet rows padded to pow2_v (0 on failure).
int neighbor_rebuild_blocks(int pow2_v);
void launch_neighbor_update(Engine& e, int N, const double* pos, const int* type, bool force,
                            cudaStream_t stream, bool skin_done = false);

// Device bytes one atom and one structure slot of a served request occupy
// (serve.cu): the server admits requests by these against its byte budget.
size_t served_bytes_per_atom(const Engine& e);
size_t served_bytes_per_struct();

// Explicit rows: allocates them for the handle's capacity and max_struct
// structures (once; later calls only check the size).
std::string engine_enable_xr(Engine& e, int max_struct);

// Cell grids of the large structures of a batch: each gets cells at least
// rc / 2 thick, (rc + skin) / 2 where it keeps Verlet candidates (at most
// cell_cap in total, else it scans all its atoms); returns the number of
// cells.  Structures are described by si[0..n).
int assign_cells(const Engine& e, StructInfo* si, int n);
// Cells of a structure's grid (0: small, or too few cells for the stencil,
// so its rows scan all its atoms); nc_out (may be null) gets the grid.
int structure_cells(const Engine& e, const StructInfo& s, int* nc_out);

// Small-box test of the reference with its cutoff (largest radial cutoff)
// and skin 1 A; returns 0 large, 1 small, -1 small in one direction and
// thicker than 10 rc in another (unsupported, as in the reference).
int box_kind(const Engine& e, const Box& b);

// Rebuilds the explicit rows (and the site records) from the positions: for
// from_box mode first the single StructInfo from the device box.
void launch_explicit_rows(Engine& e, int N, const double* pos, const int* type,
                          cudaStream_t stream);
// True when a structure can keep Verlet candidates: every periodic width at
// least 4 skins (its skin check takes minimum-image displacements) and, for
// a small box, candidates that fit the code (local index below 2^20, at most
// 16 images per direction).
bool verlet_encodable(const StructInfo& s, double skin);

// Neighbour indices of the explicit rows (which = 0 radial, 1 angular) into
// caller arrays nn[n], nl[n][mn] (row-major), as for the Verlet-path rows.
void launch_explicit_row_indices(const Engine& e, int which, int n, int* nn, int* nl, int mn,
                                 cudaStream_t stream);

// Switches the ANN precision (0 FP32, 1 FP16 / 2 BF16 tensor-core ANN inside
// the descriptor kernel); uploads the 16-bit weights.
std::string engine_set_precision(Engine& e, int mode);

// Descriptor + ANN + angular partial forces, then the force/virial gather.
// accumulate = add into pe/force/virial instead of overwriting them.
void launch_force(Engine& e, int N, const double* pos, const int* type, double* pe,
                  double* force, double* virial, bool accumulate, cudaStream_t stream);
void launch_descriptor(Engine& e, int N, const double* pos, const int* type, cudaStream_t stream);
// The typewise filter + radial descriptors alone (large-box path).
void launch_filter(Engine& e, int N, cudaStream_t stream);
void launch_gather(Engine& e, int N, const double* pos, const int* type, double* pe,
                   double* force, double* virial, bool accumulate, cudaStream_t stream);

}  // namespace nepx

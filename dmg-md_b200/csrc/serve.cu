// serve.cu -- many independent structures on one GPU: nepx_compute_batch and
// the continuous-batching server (include/nepx.h).
//
// Both run the explicit-row force path (explicit.cu) over structures packed
// back to back in one atom range; each structure's rows, descriptors and
// forces depend on its own atoms only, so a structure gets the same result
// alone and in any mix.
//
// Server design.  A worker thread owns the potential handle and an arena of
// max_atoms atoms (SoA arrays, double-buffered).  Each step it
//   1. admits queued requests in arrival order while they fit the arena,
//   2. rebuilds the arena: survivors move to their new offsets and the new
//      requests' inputs arrive in one host-to-device copy of a pinned block,
//      scattered by one kernel (k_arena_build); the structure table
//      (StructInfo, offsets, per-structure step flags) is one more copy,
//   3. runs the NVE first half step for the MD segments, the explicit rows,
//      the descriptor/ANN kernel and the gather over every resident atom,
//      then the second half step,
//   4. gathers the outputs of the requests that finish with this step into
//      one block (k_pack_out) and copies it back in one transfer.
// A single-point request finishes with its first step; an MD segment of k
// steps after 1 + k steps (the first evaluates the initial forces).  The
// velocity-Verlet arithmetic is that of the nepx_md NVE path (md.cu), with
// positions wrapped into each structure's own box.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/nepx.h"
#include "handle.h"
#include "xbox.h"

namespace nepx {
namespace {

constexpr int kThreads = 256;
constexpr int kOutFields = 19;   // pe, force 3, virial 9, pos 3, vel 3

__device__ __forceinline__ int find_struct(const int* __restrict__ soff, int S, int i)
{
  int lo = 0, hi = S - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (soff[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// New arena from the old one and the incoming block.  src[s].x >= 0: the
// structure's old offset; else src[s].y is its offset in the incoming block
// (SoA doubles pos 3, vel 3, mass with stride t_in, then t_in ints of type).
__global__ void k_arena_build(int T, int S, const int* __restrict__ soff,
                              const int2* __restrict__ src, int t_old,
                              const int* __restrict__ o_type, const double* __restrict__ o_pos,
                              const double* __restrict__ o_vel, const double* __restrict__ o_mass,
                              const double* __restrict__ o_force, int t_in,
                              const double* __restrict__ in_d, const int* __restrict__ in_type,
                              int* n_type, int* n_sid, double* n_pos, double* n_vel,
                              double* n_mass, double* n_force, const int* __restrict__ o_vcnt,
                              const double* __restrict__ o_x0, int* n_vcnt, double* n_x0)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const int s = find_struct(soff, S, i);
  const int local = i - soff[s];
  const int2 sr = src[s];
  n_sid[i] = s;
  if (sr.x >= 0) {
    const int j = sr.x + local;
    n_type[i] = o_type[j];
    n_mass[i] = o_mass[j];
    n_vcnt[i] = o_vcnt[j];
    for (int d = 0; d < 3; ++d) {
      n_pos[d * T + i] = o_pos[d * t_old + j];
      n_vel[d * T + i] = o_vel[d * t_old + j];
      n_force[d * T + i] = o_force[d * t_old + j];
      n_x0[d * T + i] = o_x0[d * t_old + j];
    }
  } else {
    const int j = sr.y + local;
    n_type[i] = in_type[j];
    n_mass[i] = in_d[6 * t_in + j];
    n_vcnt[i] = 0;
    for (int d = 0; d < 3; ++d) {
      n_pos[d * T + i] = in_d[d * t_in + j];
      n_vel[d * T + i] = in_d[(3 + d) * t_in + j];
      n_force[d * T + i] = 0.0;
      n_x0[d * T + i] = 0.0;
    }
  }
}

// Verlet candidates of the surviving structures that keep them (flag bit 1)
// into the new arena: one warp per atom, coalesced over the row.
__global__ void k_arena_rows(int T, int S, const int* __restrict__ soff,
                             const int2* __restrict__ src, const int* __restrict__ sflag,
                             const int* __restrict__ n_vcnt, const int* __restrict__ o_vrow,
                             int* __restrict__ n_vrow, int mn)
{
  const int lane = threadIdx.x & 31;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= T) return;
  const int s = find_struct(soff, S, i);
  const int2 sr = src[s];
  if (sr.x < 0 || !(sflag[s] & 2)) return;
  const int j = sr.x + (i - soff[s]);
  const int n = n_vcnt[i];
  const int* from = o_vrow + static_cast<size_t>(j) * mn;
  int* to = n_vrow + static_cast<size_t>(i) * mn;
  for (int k = lane; k < n; k += 32) to[k] = from[k];
}

// First half kick and drift of the atoms whose structure steps (flag bit 0),
// wrapped into the structure's box: the arithmetic of md.cu k_vv1 (NVE).
// Structures that keep Verlet candidates (bit 1) record the largest squared
// displacement of their atoms since the build (dmax2, as the ordered bits of
// a non-negative double); in a large box by minimum image, exact while an
// atom has moved less than half the box's thinnest periodic width, which
// holds for the boxes that keep candidates (at least 4 skins thick: an atom
// is caught at skin / 2).
__global__ void k_vv1_batch(int T, const int* __restrict__ sid, const int* __restrict__ sflag,
                            const double* __restrict__ sdt, const StructInfo* __restrict__ si,
                            const double* __restrict__ mass, const double* __restrict__ force,
                            double* pos, double* vel, const double* __restrict__ x0,
                            double* dmax2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const int s = sid[i];
  if (!(sflag[s] & 1)) return;
  const double dt = sdt[s];
  const double half = dt * 0.5;
  const double im = 1.0 / mass[i];
  double r[3];
  for (int d = 0; d < 3; ++d) {
    const double v = vel[d * T + i] * 1.0 + force[d * T + i] * im * half;
    vel[d * T + i] = v;
    r[d] = pos[d * T + i] + v * dt;
  }
  const Box& b = si[s].box;
  double f[3];
  for (int d = 0; d < 3; ++d) {
    f[d] = b.hinv[3 * d] * r[0] + b.hinv[3 * d + 1] * r[1] + b.hinv[3 * d + 2] * r[2];
    if (b.pbc[d] == 1) {
      if (f[d] < 0.0) f[d] += 1.0;
      else if (f[d] > 1.0) f[d] -= 1.0;
    }
  }
  double x[3];
  for (int d = 0; d < 3; ++d) {
    x[d] = b.h[3 * d] * f[0] + b.h[3 * d + 1] * f[1] + b.h[3 * d + 2] * f[2];
    pos[d * T + i] = x[d];
  }
  if (sflag[s] & 2) {
    // displacement since the build.  A large box's candidates are plain
    // indices, whose displacement is taken by minimum image: an atom that
    // crossed a periodic face has not moved a box length.  A small box's
    // candidates name images relative to the wrapped positions, so there a
    // wrap counts as the box-length jump it is and forces a rebuild.
    const bool mic = !si[s].small;
    double u[3], g[3];
    for (int d = 0; d < 3; ++d) u[d] = x[d] - x0[d * T + i];
    for (int d = 0; d < 3; ++d) {
      g[d] = b.hinv[3 * d] * u[0] + b.hinv[3 * d + 1] * u[1] + b.hinv[3 * d + 2] * u[2];
      if (mic && b.pbc[d] == 1) g[d] -= rint(g[d]);
    }
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double w = b.h[3 * d] * g[0] + b.h[3 * d + 1] * g[1] + b.h[3 * d + 2] * g[2];
      d2 += w * w;
    }
    atomicMax(reinterpret_cast<unsigned long long*>(dmax2 + s),
              static_cast<unsigned long long>(__double_as_longlong(d2)));
  }
}

// Second half kick (md.cu k_vv2_thermo without the thermo sums).
__global__ void k_vv2_batch(int T, const int* __restrict__ sid, const int* __restrict__ sflag,
                            const double* __restrict__ sdt, const double* __restrict__ mass,
                            const double* __restrict__ force, double* vel)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const int s = sid[i];
  if (!(sflag[s] & 1)) return;
  const double half = sdt[s] * 0.5;
  const double im = 1.0 / mass[i];
  for (int d = 0; d < 3; ++d) vel[d * T + i] = vel[d * T + i] + force[d * T + i] * im * half;
}

// Outputs of the finishing structures into one block, SoA with stride t_out:
// pe, force 3, virial 9, pos 3, vel 3.  fin[k] = (arena offset, out offset).
__global__ void k_pack_out(int t_out, int nfin, const int* __restrict__ fin_out_off,
                           const int* __restrict__ fin_arena_off, int T,
                           const double* __restrict__ pe, const double* __restrict__ force,
                           const double* __restrict__ virial, const double* __restrict__ pos,
                           const double* __restrict__ vel, double* out)
{
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= t_out) return;
  const int k = find_struct(fin_out_off, nfin, o);
  const int a = fin_arena_off[k] + (o - fin_out_off[k]);
  out[o] = pe[a];
  for (int d = 0; d < 3; ++d) out[(1 + d) * t_out + o] = force[d * T + a];
  for (int d = 0; d < 9; ++d) out[(4 + d) * t_out + o] = virial[d * T + a];
  for (int d = 0; d < 3; ++d) out[(13 + d) * t_out + o] = pos[d * T + a];
  for (int d = 0; d < 3; ++d) out[(16 + d) * t_out + o] = vel[d * T + a];
}

std::string struct_info(const Engine& e, const nepx_box& box, int off, int n, StructInfo& si)
{
  Box b;
  const std::string err = make_box(box.h, box.pbc, b);
  if (!err.empty()) return err;
  if (expanded_box(b, e.model.rc_radial_max, si))
    return "box thinner than 2.5 (rc + 1) in one periodic direction and thicker than 10 rc "
           "in another (unsupported, as in the reference)";
  si.off = off;
  si.n = n;
  return "";
}

template <typename T>
bool dalloc(T*& p, size_t n)
{
  return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)) ==
         cudaSuccess;
}

template <typename T>
bool halloc(T*& p, size_t n)
{
  return cudaMallocHost(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)) ==
         cudaSuccess;
}

int grid(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

// Device bytes one served atom occupies: the handle's per-atom buffers of the
// explicit-row path (radial and angular rows, angular partial forces, site
// records, cell slots, descriptor scratch) and the server's two arena
// buffers and I/O blocks.
size_t served_bytes_per_atom(const Engine& e)
{
  const NeighborBuffers& nb = e.nbr;
  const ModelParams& p = e.params;
  size_t b = 16 * static_cast<size_t>(nb.mn_r + nb.mn_a);   // explicit rows (float4)
  b += 16 * static_cast<size_t>(nb.mn_a);                    // angular partial forces
  b += 2 * sizeof(int) + sizeof(Site) + 1 + 2 * sizeof(int); // counts, sites, flag, cell slots
  b += sizeof(float) * (static_cast<size_t>(p.nA) * p.nlm + p.T * basis_stride(p) + p.nR);
  b += sizeof(double);                                       // site energy
  b += 2 * (2 * sizeof(int) + 10 * sizeof(double));          // arenas: type, sid, pos, vel, mass, force
  b += 2 * (sizeof(int) * (1 + static_cast<size_t>(nb.mn_v)) + 3 * sizeof(double));   // candidates
  b += sizeof(double) * (1 + 9 + kOutFields + 8);            // pe, virial, output and input blocks
  return b;
}

// Device bytes of one structure slot: its table entry, offset, control words
// and step size (its cell grid is counted per cell).
size_t served_bytes_per_struct() { return sizeof(StructInfo) + 6 * sizeof(int) + sizeof(double); }

// Explicit rows + force over structures already described in e.xr (d_si,
// d_soff, n_struct uploaded).  Shared by the batch call and the server.
void launch_batch_force(Engine& e, int T, const double* pos, const int* type, double* pe,
                        double* force, double* virial, bool accumulate, cudaStream_t s)
{
  e.use_xr = true;
  e.xr.from_box = false;
  launch_explicit_rows(e, T, pos, type, s);
  if (!e.tuned) engine_autotune(e, T, pos, type, s);
  launch_force(e, T, pos, type, pe, force, virial, accumulate, s);
  // the Verlet-path state of the handle no longer matches its last box
  e.force_rebuild = true;
  e.have_box = false;
  e.box_owner = nullptr;
}

}  // namespace nepx

// ---------------------------------------------------------------------------
// the server
// ---------------------------------------------------------------------------

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  long long ticket = 0;
  int n = 0, md_steps = 0;
  int cells = 0;            // cells of its grid in the batch's cell lists
  size_t bytes = 0;         // device bytes it occupies while resident
  double dt = 0.0;          // fs
  nepx_box box{};
  std::vector<int> type;
  std::vector<double> pos, vel, mass;   // vel in natural units
  nepx_result* out = nullptr;
  double t_submit = 0.0;
};

struct Resident {
  long long ticket = 0;
  int n = 0, md_steps = 0, steps_done = 0;
  int cells = 0;
  size_t bytes = 0;
  bool fresh = true;        // initial forces not evaluated yet
  double dt = 0.0;          // fs
  nepx::StructInfo si{};
  int off = 0;              // offset in the current arena
  nepx_result* out = nullptr;
  double t_submit = 0.0, t_admit = 0.0;
};

// Device arrays of one arena buffer.
struct Arena {
  int* type = nullptr;
  int* sid = nullptr;
  double *pos = nullptr, *vel = nullptr, *mass = nullptr, *force = nullptr;
  // Verlet candidates of the MD segments' centers (explicit.cu BatchVerlet)
  int *vcnt = nullptr, *vrow = nullptr;
  double* x0 = nullptr;
};

}  // namespace

struct nepx_server {
  nepx_t* h = nullptr;
  int max_atoms = 0, max_struct = 0;
  // admission by device memory: a request is admitted while the resident
  // requests' bytes plus its own stay within the budget (and the arena's atom,
  // slot and cell capacities hold)
  size_t bytes_per_atom = 0, bytes_per_struct = 0, budget = 0;
  cudaStream_t stream = nullptr;
  Arena arena[2];
  int cur = 0;
  double *d_pe = nullptr, *d_virial = nullptr, *d_out = nullptr, *d_in = nullptr;
  int* d_ctl = nullptr;       // per-structure src (int2), flags, finishing lists
  double* d_sdt = nullptr;
  double* d_dmax2 = nullptr;  // per structure: largest squared displacement since its candidates' build
  int mn_cand = 0;            // Verlet candidates per served atom
  bool row_reuse = true;      // MD segments admitted from now on keep Verlet candidates
  // pinned host staging, two copies (the worker stages one step while the
  // previous one runs)
  double *h_in[2] = {}, *h_out[2] = {}, *h_sdt[2] = {};
  int* h_ctl[2] = {};
  nepx::StructInfo* h_si[2] = {};
  int* h_soff[2] = {};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<Pending> queue;
  std::unordered_map<long long, int> status;   // -1 pending, else the request's code
  long long next_ticket = 1;
  bool stopping = false;
  std::string error;
  Clock::time_point t0;
  // statistics
  double done = 0, steps = 0, atom_steps = 0, busy = 0, resident_atoms = 0, resident_structs = 0;
  double resident_bytes = 0;
  double cand_builds = 0, kept_center_steps = 0;
  unsigned last_builds = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  void run();
};

namespace {

void free_server(nepx_server* S)
{
  for (auto& a : S->arena) {
    void* ptrs[] = {a.type, a.sid, a.pos, a.vel, a.mass, a.force, a.vcnt, a.vrow, a.x0};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
  void* dptrs[] = {S->d_pe, S->d_virial, S->d_out, S->d_in, S->d_ctl, S->d_sdt, S->d_dmax2};
  for (void* p : dptrs)
    if (p) cudaFree(p);
  for (int c = 0; c < 2; ++c) {
    void* hptrs[] = {S->h_in[c], S->h_out[c], S->h_sdt[c], S->h_ctl[c], S->h_si[c], S->h_soff[c]};
    for (void* p : hptrs)
      if (p) cudaFreeHost(p);
  }
  if (S->stream) cudaStreamDestroy(S->stream);
}

}  // namespace

// The worker loop.  Once step k is done on the GPU, the worker admits the
// requests queued meanwhile, stages and enqueues step k+1, and only then
// copies step k's results out to their callers, while step k+1 runs.  The
// pinned staging buffers alternate between two copies, so step k's outputs
// stay readable while step k+1 writes its own.  (Staging step k+1 while step
// k runs hid a little more host time, 2% more structures/s on the serving
// stream, but every request arriving during step k then waited one more step:
// p50 latency 0.57 -> 0.85 ms at 60% load.)
void nepx_server::run()
{
  using namespace nepx;
  Engine& e = h->engine;
  // a new host thread starts on device 0: work on the handle's device
  cudaSetDevice(e.device);
  cudaStream_t s = stream;
  std::vector<Resident> res;   // arena order, after the step in flight
  int fly_T = 0;               // atoms in the arena the last enqueued step writes (its stride)
  const int MS = max_struct;
  // control block layout (ints): src int2[MS] | flags[MS] | fin_out_off[MS+1] | fin_arena_off[MS]
  const size_t ctl_ints = 2 * MS + MS + (MS + 1) + MS;
  // a finishing request of a staged or running step
  struct Finishing {
    long long ticket;
    nepx_result* out;
    int n, base;
    double t_submit, t_admit;
  };
  struct Step {
    int par = 0, T = 0, S = 0, t_in = 0, t_out = 0, n_cells = 0;
    double t_tick = 0.0, bytes = 0.0;
    double kept = 0.0;           // atoms of structures that keep Verlet candidates
    std::vector<Finishing> fin;
  };
  Step fly;                    // the step on the GPU
  bool flying = false;
  int par = 0;                 // staging copy of the next step
  for (;;) {
    // ---- 1. finish the step in flight ------------------------------------------
    int code = NEPX_OK;
    std::string msg;
    double t_end = 0.0;
    double fly_builds = 0.0;
    if (flying) {
      const cudaError_t cerr = cudaStreamSynchronize(s);
      t_end = now();
      if (cerr != cudaSuccess) {
        code = NEPX_ERR_CUDA;
        msg = std::string("server step: ") + cudaGetErrorString(cerr);
      } else {
        const NeighborState& st = *h->h_state;
        fly_builds = static_cast<double>(st.xr_builds - last_builds);   // wraps
        last_builds = st.xr_builds;
        if (st.overflow) {
          code = NEPX_ERR_OVERFLOW;
          msg = "a neighbour row exceeded its capacity; raise MN_radial/MN_angular in nep.txt";
        } else if (st.nonfinite) {
          code = NEPX_ERR_NONFINITE;
          msg = "non-finite energy or force";
        }
        if (code) {
          NeighborState cleared = st;
          cleared.overflow = 0;
          cleared.nonfinite = 0;
          cudaMemcpy(e.d_nstate, &cleared, sizeof(cleared), cudaMemcpyHostToDevice);
        }
      }
    }
    // ---- 2. admission --------------------------------------------------------
    std::vector<Pending> adm;
    bool keep_new = true;
    {
      std::unique_lock<std::mutex> lk(mu);
      if (!flying) cv.wait(lk, [&] { return !queue.empty() || !res.empty() || stopping; });
      if (!flying && queue.empty() && res.empty()) break;   // stopping with nothing left
      keep_new = row_reuse;
      int atoms = 0;
      int nst = static_cast<int>(res.size());
      int cells = 0;
      size_t bytes = 0;
      for (const Resident& r : res) {
        atoms += r.n;
        cells += r.cells;
        bytes += r.bytes;
      }
      while (!queue.empty()) {
        Pending& p = queue.front();
        if (atoms + p.n > max_atoms || nst + 1 > MS || bytes + p.bytes > budget ||
            cells + p.cells > e.xr.cell_cap)
          break;
        atoms += p.n;
        ++nst;
        cells += p.cells;
        bytes += p.bytes;
        adm.push_back(std::move(p));
        queue.pop_front();
      }
    }
    const bool stage = !res.empty() || !adm.empty();
    Step nx;
    if (stage) {
      // ---- 3. stage the next step: survivors in order, then the admitted ------
      nx.par = par;
      nx.t_tick = now();
      double* hin = h_in[par];
      int* c_src = h_ctl[par];
      int* c_flag = c_src + 2 * MS;
      int* c_fout = c_flag + MS;
      int* c_farena = c_fout + MS + 1;
      const int S_old = static_cast<int>(res.size());
      int t_in = 0;
      for (const Pending& p : adm) t_in += p.n;
      std::vector<int> in_off(adm.size());
      {
        int o = 0;
        for (size_t k = 0; k < adm.size(); ++k) {
          in_off[k] = o;
          o += adm[k].n;
        }
      }
      int Tn = 0;
      for (int k = 0; k < S_old; ++k) {
        c_src[2 * k] = res[k].off;
        c_src[2 * k + 1] = 0;
        res[k].off = Tn;
        Tn += res[k].n;
      }
      for (size_t k = 0; k < adm.size(); ++k) {
        Pending& p = adm[k];
        Resident r;
        r.ticket = p.ticket;
        r.n = p.n;
        r.cells = p.cells;
        r.bytes = p.bytes;
        r.md_steps = p.md_steps;
        r.dt = p.dt;
        r.out = p.out;
        r.t_submit = p.t_submit;
        r.t_admit = nx.t_tick;
        r.off = Tn;
        struct_info(e, p.box, 0, p.n, r.si);   // validated at submit
        r.si.n = p.n;
        r.si.keep = (keep_new && p.md_steps > 0 && verlet_encodable(r.si, e.skin)) ? 1 : 0;
        const int idx = static_cast<int>(res.size());
        c_src[2 * idx] = -1;
        c_src[2 * idx + 1] = in_off[k];
        // incoming block: pos 3, vel 3, mass (doubles, stride t_in), then types
        for (int d = 0; d < 3; ++d) {
          std::memcpy(hin + static_cast<size_t>(d) * t_in + in_off[k], p.pos.data() + d * p.n,
                      sizeof(double) * p.n);
          if (!p.vel.empty())
            std::memcpy(hin + static_cast<size_t>(3 + d) * t_in + in_off[k],
                        p.vel.data() + d * p.n, sizeof(double) * p.n);
          else
            std::memset(hin + static_cast<size_t>(3 + d) * t_in + in_off[k], 0,
                        sizeof(double) * p.n);
        }
        for (int a = 0; a < p.n; ++a)
          hin[static_cast<size_t>(6) * t_in + in_off[k] + a] = p.mass.empty() ? 1.0 : p.mass[a];
        std::memcpy(reinterpret_cast<int*>(hin + static_cast<size_t>(7) * t_in) + in_off[k],
                    p.type.data(), sizeof(int) * p.n);
        Tn += p.n;
        res.push_back(r);
      }
      const int S = static_cast<int>(res.size());
      // structure table, offsets, step flags and the finishing requests
      for (int k = 0; k < S; ++k) {
        Resident& r = res[k];
        r.si.off = r.off;
        r.si.n = r.n;
        h_si[par][k] = r.si;
        h_soff[par][k] = r.off;
        // bit 0 steps, bit 1 keeps Verlet candidates, bit 2 builds them (new)
        c_flag[k] = (r.fresh ? 0 : 1) | (r.si.keep ? 2 : 0) | (r.fresh && r.si.keep ? 4 : 0);
        if (r.si.keep) nx.kept += r.n;
        h_sdt[par][k] = r.dt / kTimeUnit;
        nx.bytes += static_cast<double>(r.bytes);
        const bool finishes = r.fresh ? r.md_steps == 0 : r.steps_done + 1 == r.md_steps;
        if (finishes) {
          c_fout[nx.fin.size()] = nx.t_out;
          c_farena[nx.fin.size()] = r.off;
          nx.fin.push_back({r.ticket, r.out, r.n, nx.t_out, r.t_submit, r.t_admit});
          nx.t_out += r.n;
        }
      }
      h_soff[par][S] = Tn;
      c_fout[nx.fin.size()] = nx.t_out;
      nx.n_cells = assign_cells(e, h_si[par], S);
      nx.T = Tn;
      nx.S = S;
      nx.t_in = t_in;
      // what is left after this step: the next admission sees these
      std::vector<Resident> keep;
      keep.reserve(res.size());
      for (Resident& r : res) {
        const bool fin = r.fresh ? r.md_steps == 0 : r.steps_done + 1 == r.md_steps;
        if (!r.fresh) ++r.steps_done;
        r.fresh = false;
        if (!fin) keep.push_back(r);
      }
      res.swap(keep);
    }
    // ---- 4. enqueue the staged step ---------------------------------------------
    if (stage) {
      const int p = nx.par;
      Arena& A = arena[cur];
      Arena& B = arena[1 - cur];
      int* d_src = d_ctl;
      const int* d_flag = d_ctl + 2 * MS;
      const int* d_fout = d_flag + MS;
      const int* d_farena = d_fout + MS + 1;
      if (nx.t_in > 0)
        cudaMemcpyAsync(d_in, h_in[p], (sizeof(double) * 7 + sizeof(int)) * nx.t_in,
                        cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(d_ctl, h_ctl[p], sizeof(int) * ctl_ints, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(d_sdt, h_sdt[p], sizeof(double) * nx.S, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(e.xr.d_si, h_si[p], sizeof(StructInfo) * nx.S, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(e.xr.d_soff, h_soff[p], sizeof(int) * (nx.S + 1), cudaMemcpyHostToDevice,
                      s);
      e.xr.n_struct = nx.S;
      e.xr.n_cells = nx.n_cells;
      k_arena_build<<<grid(nx.T), kThreads, 0, s>>>(
        nx.T, nx.S, e.xr.d_soff, reinterpret_cast<const int2*>(d_src), fly_T, A.type, A.pos,
        A.vel, A.mass, A.force, nx.t_in, d_in,
        reinterpret_cast<const int*>(d_in + static_cast<size_t>(7) * nx.t_in), B.type, B.sid,
        B.pos, B.vel, B.mass, B.force, A.vcnt, A.x0, B.vcnt, B.x0);
      if (nx.kept > 0)
        k_arena_rows<<<(nx.T + 7) / 8, kThreads, 0, s>>>(
          nx.T, nx.S, e.xr.d_soff, reinterpret_cast<const int2*>(d_src), d_flag, B.vcnt, A.vrow,
          B.vrow, mn_cand);
      cur = 1 - cur;
      Arena& R = arena[cur];
      cudaMemsetAsync(d_dmax2, 0, sizeof(double) * nx.S, s);
      k_vv1_batch<<<grid(nx.T), kThreads, 0, s>>>(nx.T, R.sid, d_flag, d_sdt, e.xr.d_si, R.mass,
                                                  R.force, R.pos, R.vel, R.x0, d_dmax2);
      if (nx.kept > 0) {
        BatchVerlet& bv = e.xr.bv;
        bv.sflag = d_flag;
        bv.dmax2 = d_dmax2;
        bv.skin = static_cast<float>(e.skin);
        bv.half_skin2 = 0.25 * e.skin * e.skin;
        bv.mn = mn_cand;
        bv.vcnt = R.vcnt;
        bv.vrow = R.vrow;
        bv.x0 = R.x0;
      }
      launch_batch_force(e, nx.T, R.pos, R.type, d_pe, R.force, d_virial, false, s);
      e.xr.bv = BatchVerlet{};
      k_vv2_batch<<<grid(nx.T), kThreads, 0, s>>>(nx.T, R.sid, d_flag, d_sdt, R.mass, R.force,
                                                  R.vel);
      const int nfin = static_cast<int>(nx.fin.size());
      if (nfin > 0) {
        k_pack_out<<<grid(nx.t_out), kThreads, 0, s>>>(nx.t_out, nfin, d_fout, d_farena, nx.T,
                                                       d_pe, R.force, d_virial, R.pos, R.vel,
                                                       d_out);
        cudaMemcpyAsync(h_out[p], d_out, sizeof(double) * kOutFields * nx.t_out,
                        cudaMemcpyDeviceToHost, s);
      }
      cudaMemcpyAsync(h->h_state, e.d_nstate, sizeof(NeighborState), cudaMemcpyDeviceToHost, s);
      fly_T = nx.T;
      par = 1 - par;
    }
    // ---- 5. deliver the finished step while the staged one runs ---------------
    if (flying) {
      const double* hout = h_out[fly.par];
      for (const Finishing& f : fly.fin) {
        nepx_result* o = f.out;
        const int n = f.n;
        auto take = [&](double* dst, int field0, int nf, double scale) {
          if (!dst) return;
          for (int q = 0; q < nf; ++q)
            for (int a = 0; a < n; ++a)
              dst[static_cast<size_t>(q) * n + a] =
                hout[static_cast<size_t>(field0 + q) * fly.t_out + f.base + a] * scale;
        };
        take(o->pe, 0, 1, 1.0);
        take(o->force, 1, 3, 1.0);
        take(o->virial, 4, 9, 1.0);
        take(o->pos, 13, 3, 1.0);
        take(o->vel, 16, 3, 1.0 / kTimeUnit);
        o->t_submit = f.t_submit;
        o->t_admit = f.t_admit;
        o->t_done = t_end;
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        for (const Finishing& f : fly.fin) status[f.ticket] = code;
        if (code) error = msg;
        done += static_cast<double>(fly.fin.size());
        steps += 1;
        atom_steps += fly.T;
        busy += t_end - fly.t_tick;
        resident_atoms += fly.T;
        resident_structs += fly.S;
        resident_bytes += fly.bytes;
        cand_builds += fly_builds;
        kept_center_steps += fly.kept;
      }
      if (!fly.fin.empty()) done_cv.notify_all();
    }
    flying = stage;
    if (stage) fly = std::move(nx);
  }
}

extern "C" {

int nepx_compute_batch(nepx_t* h, const nepx_struct_desc* descs, int nstruct, const int* d_type,
                       const double* d_pos, double* d_pe, double* d_force, double* d_virial,
                       unsigned flags, void* stream)
{
  if (!h) return NEPX_ERR_ARG;
  if (!descs || nstruct < 1 || !d_type || !d_pos || !d_pe || !d_force || !d_virial) {
    h->error = "null pointer or nstruct < 1";
    return NEPX_ERR_ARG;
  }
  nepx::Engine& e = h->engine;
  std::vector<nepx::StructInfo> si(nstruct);
  std::vector<int> soff(nstruct + 1);
  long long T = 0;
  for (int k = 0; k < nstruct; ++k) {
    if (descs[k].n < 1) {
      h->error = "structure " + std::to_string(k) + " has no atoms";
      return NEPX_ERR_ARG;
    }
    const std::string err = nepx::struct_info(e, descs[k].box, static_cast<int>(T), descs[k].n,
                                              si[k]);
    if (!err.empty()) {
      h->error = "structure " + std::to_string(k) + ": " + err;
      return NEPX_ERR_BOX;
    }
    soff[k] = static_cast<int>(T);
    T += descs[k].n;
  }
  soff[nstruct] = static_cast<int>(T);
  if (T > e.capacity) {
    h->error = std::to_string(T) + " atoms exceed the capacity " + std::to_string(e.capacity) +
               " of this handle";
    return NEPX_ERR_CAPACITY;
  }
  const std::string err = nepx::engine_enable_xr(e, nstruct);
  if (!err.empty()) {
    h->error = err;
    return NEPX_ERR_CUDA;
  }
  auto s = static_cast<cudaStream_t>(stream);
  // a copy of the flags of an earlier call may still be landing in h_state
  if (h->state_pending) cudaEventSynchronize(h->state_ready);
  h->state_pending = false;
  e.xr.n_cells = nepx::assign_cells(e, si.data(), nstruct);
  // pageable sources: the copies complete before the calls return
  cudaMemcpyAsync(e.xr.d_si, si.data(), sizeof(nepx::StructInfo) * nstruct,
                  cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(e.xr.d_soff, soff.data(), sizeof(int) * (nstruct + 1), cudaMemcpyHostToDevice,
                  s);
  e.xr.n_struct = nstruct;
  nepx::launch_batch_force(e, static_cast<int>(T), d_pos, d_type, d_pe, d_force, d_virial,
                           (flags & NEPX_ACCUMULATE) != 0, s);
  if (cudaPeekAtLastError() != cudaSuccess) {
    h->error = std::string("kernel launch: ") + cudaGetErrorString(cudaGetLastError());
    return NEPX_ERR_CUDA;
  }
  cudaMemcpyAsync(h->h_state, e.d_nstate, sizeof(nepx::NeighborState), cudaMemcpyDeviceToHost, s);
  cudaEventRecord(h->state_ready, s);
  h->state_pending = true;
  if (flags & NEPX_SYNC_CHECK) {
    if (cudaEventSynchronize(h->state_ready) != cudaSuccess) {
      h->error = "stream sync failed";
      return NEPX_ERR_CUDA;
    }
    h->state_pending = false;
    const nepx::NeighborState& st = *h->h_state;
    if (st.overflow) {
      h->error = "a neighbour row exceeded its capacity; raise MN_radial/MN_angular in nep.txt";
      return NEPX_ERR_OVERFLOW;
    }
    if (st.nonfinite) {
      h->error = "non-finite energy or force";
      return NEPX_ERR_NONFINITE;
    }
  }
  return NEPX_OK;
}

int nepx_server_create(nepx_t* h, int max_atoms, int max_struct, nepx_server_t** out)
{
  if (!h || !out || max_atoms < 1 || max_struct < 1) return NEPX_ERR_ARG;
  *out = nullptr;
  nepx::Engine& e = h->engine;
  if (max_atoms > e.capacity) {
    h->error = "server arena larger than the handle's max_atoms";
    return NEPX_ERR_CAPACITY;
  }
  if (!nepx::engine_enable_xr(e, max_struct).empty()) return NEPX_ERR_CUDA;
  auto* S = new (std::nothrow) nepx_server();
  if (!S) return NEPX_ERR_ARG;
  S->h = h;
  S->max_atoms = max_atoms;
  S->max_struct = max_struct;
  S->bytes_per_atom = nepx::served_bytes_per_atom(e);
  S->bytes_per_struct = nepx::served_bytes_per_struct();
  S->budget = static_cast<size_t>(max_atoms) * S->bytes_per_atom +
              static_cast<size_t>(max_struct) * S->bytes_per_struct +
              sizeof(int) * 2 * static_cast<size_t>(e.xr.cell_cap);
  S->t0 = Clock::now();
  const size_t N = max_atoms, MS = max_struct;
  bool ok = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) == cudaSuccess;
  S->mn_cand = e.nbr.mn_v;
  for (auto& a : S->arena)
    ok = ok && nepx::dalloc(a.type, N) && nepx::dalloc(a.sid, N) &&
         nepx::dalloc(a.pos, 3 * N) && nepx::dalloc(a.vel, 3 * N) && nepx::dalloc(a.mass, N) &&
         nepx::dalloc(a.force, 3 * N) && nepx::dalloc(a.vcnt, N) &&
         nepx::dalloc(a.vrow, N * static_cast<size_t>(S->mn_cand)) && nepx::dalloc(a.x0, 3 * N);
  ok = ok && nepx::dalloc(S->d_pe, N) && nepx::dalloc(S->d_virial, 9 * N) &&
       nepx::dalloc(S->d_out, size_t(nepx::kOutFields) * N) && nepx::dalloc(S->d_in, 8 * N) &&
       nepx::dalloc(S->d_ctl, 5 * MS + 1) && nepx::dalloc(S->d_sdt, MS) &&
       nepx::dalloc(S->d_dmax2, MS);
  for (int c = 0; c < 2; ++c)
    ok = ok && nepx::halloc(S->h_in[c], 8 * N) &&
         nepx::halloc(S->h_out[c], nepx::kOutFields * N) && nepx::halloc(S->h_sdt[c], MS) &&
         nepx::halloc(S->h_ctl[c], 5 * MS + 1) && nepx::halloc(S->h_si[c], MS) &&
         nepx::halloc(S->h_soff[c], MS + 1);
  if (ok) ok = cudaMemsetAsync(S->arena[0].force, 0, sizeof(double) * 3 * N, S->stream) ==
               cudaSuccess;
  if (ok) ok = cudaMemsetAsync(S->arena[0].x0, 0, sizeof(double) * 3 * N, S->stream) ==
               cudaSuccess;
  if (ok) {
    // candidate builds are counted from the handle's running device counter
    nepx::NeighborState now{};
    ok = cudaMemcpy(&now, e.d_nstate, sizeof(now), cudaMemcpyDeviceToHost) == cudaSuccess;
    S->last_builds = now.xr_builds;
  }
  if (!ok) {
    free_server(S);
    delete S;
    h->error = "server allocation failed";
    return NEPX_ERR_CUDA;
  }
  S->worker = std::thread([S] { S->run(); });
  *out = S;
  return NEPX_OK;
}

int nepx_server_destroy(nepx_server_t* S)
{
  if (!S) return NEPX_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv.notify_all();
  if (S->worker.joinable()) S->worker.join();
  free_server(S);
  delete S;
  return NEPX_OK;
}

const char* nepx_server_last_error(const nepx_server_t* S)
{
  return S ? S->error.c_str() : "null server";
}

int nepx_server_submit(nepx_server_t* S, const nepx_request* req, nepx_result* out,
                       long long* ticket)
{
  if (!S || !req || !out || !ticket || req->n < 1 || !req->type || !req->pos)
    return NEPX_ERR_ARG;
  if (req->md_steps < 0 || (req->md_steps > 0 && (!req->mass || !req->vel || !(req->dt_fs > 0))))
    return NEPX_ERR_ARG;
  const nepx::Engine& e = S->h->engine;
  if (req->n > S->max_atoms) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->error = "request of " + std::to_string(req->n) + " atoms is larger than the arena";
    return NEPX_ERR_CAPACITY;
  }
  nepx::StructInfo si;
  const std::string err = nepx::struct_info(e, req->box, 0, req->n, si);
  if (!err.empty()) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->error = err;
    return NEPX_ERR_BOX;
  }
  for (int a = 0; a < req->n; ++a)
    if (req->type[a] < 0 || req->type[a] >= e.model.num_types) return NEPX_ERR_ARG;
  Pending p;
  p.n = req->n;
  p.cells = nepx::structure_cells(e, si, nullptr);
  p.bytes = static_cast<size_t>(req->n) * S->bytes_per_atom + S->bytes_per_struct +
            sizeof(int) * 2 * static_cast<size_t>(p.cells);
  if (p.bytes > S->budget || p.cells > e.xr.cell_cap) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->error = "request of " + std::to_string(req->n) + " atoms needs more device memory than "
               "the server's budget";
    return NEPX_ERR_CAPACITY;
  }
  p.md_steps = req->md_steps;
  p.dt = req->dt_fs;
  p.box = req->box;
  p.type.assign(req->type, req->type + req->n);
  p.pos.assign(req->pos, req->pos + 3 * static_cast<size_t>(req->n));
  if (req->md_steps > 0) {
    p.mass.assign(req->mass, req->mass + req->n);
    p.vel.resize(3 * static_cast<size_t>(req->n));
    for (size_t k = 0; k < p.vel.size(); ++k) p.vel[k] = req->vel[k] * nepx::kTimeUnit;
  }
  p.out = out;
  p.t_submit = S->now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    p.ticket = S->next_ticket++;
    *ticket = p.ticket;
    S->status[p.ticket] = -1;
    S->queue.push_back(std::move(p));
  }
  S->cv.notify_one();
  return NEPX_OK;
}

int nepx_server_poll(nepx_server_t* S, long long ticket, int* done, int* status)
{
  if (!S || !done) return NEPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->status.find(ticket);
  if (it == S->status.end()) return NEPX_ERR_ARG;
  *done = it->second >= 0;
  if (status) *status = it->second;
  return NEPX_OK;
}

int nepx_server_wait(nepx_server_t* S, long long ticket, int* status)
{
  if (!S) return NEPX_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->status.find(ticket);
  if (it == S->status.end()) return NEPX_ERR_ARG;
  S->done_cv.wait(lk, [&] { return S->status[ticket] >= 0; });
  if (status) *status = S->status[ticket];
  return NEPX_OK;
}

int nepx_server_drain(nepx_server_t* S)
{
  if (!S) return NEPX_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  S->done_cv.wait(lk, [&] {
    for (const auto& kv : S->status)
      if (kv.second < 0) return false;
    return true;
  });
  return NEPX_OK;
}

int nepx_server_create_budget(nepx_t* h, double hbm_bytes, int max_struct, nepx_server_t** out)
{
  if (!h || !out || max_struct < 1 || !(hbm_bytes > 0.0)) return NEPX_ERR_ARG;
  *out = nullptr;
  nepx::Engine& e = h->engine;
  const double per_atom = static_cast<double>(nepx::served_bytes_per_atom(e)) + 2.0 * sizeof(int);
  const double slots = static_cast<double>(max_struct) * nepx::served_bytes_per_struct();
  const double atoms = std::floor((hbm_bytes - slots) / per_atom);
  if (atoms < 1.0) {
    h->error = "a device-memory budget of " + std::to_string(hbm_bytes) +
               " bytes holds no atom of this model";
    return NEPX_ERR_CAPACITY;
  }
  const int max_atoms = static_cast<int>(std::min<double>(atoms, e.capacity));
  const int rc = nepx_server_create(h, max_atoms, max_struct, out);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk((*out)->mu);
  (*out)->budget = static_cast<size_t>(hbm_bytes);
  return NEPX_OK;
}

int nepx_server_memory(nepx_server_t* S, double* info)
{
  if (!S || !info) return NEPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  info[0] = static_cast<double>(S->budget);
  info[1] = static_cast<double>(S->bytes_per_atom);
  info[2] = static_cast<double>(S->bytes_per_struct);
  info[3] = S->steps > 0 ? S->resident_bytes / S->steps : 0.0;
  return NEPX_OK;
}

int nepx_server_set_row_reuse(nepx_server_t* S, int on)
{
  if (!S) return NEPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->row_reuse = on != 0;
  return NEPX_OK;
}

int nepx_server_rows(nepx_server_t* S, double* info)
{
  if (!S || !info) return NEPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  info[0] = S->cand_builds;
  info[1] = S->kept_center_steps;
  return NEPX_OK;
}

int nepx_server_stats(nepx_server_t* S, double* stats)
{
  if (!S || !stats) return NEPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  stats[0] = S->done;
  stats[1] = S->steps;
  stats[2] = S->atom_steps;
  stats[3] = S->busy;
  stats[4] = S->steps > 0 ? S->resident_atoms / S->steps : 0.0;
  stats[5] = S->steps > 0 ? S->resident_structs / S->steps : 0.0;
  stats[6] = static_cast<double>(S->queue.size());
  stats[7] = S->now();
  return NEPX_OK;
}

}  // extern "C"

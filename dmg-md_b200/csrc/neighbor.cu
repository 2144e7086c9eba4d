// neighbor.cu -- Verlet list (cutoff + skin) on a cell grid; the per-step
// typewise radial / angular filter of its rows is k_filter_radial
// (nep_force.cu).
//
// Reference behaviour (src/gpumd_compat/neighbor.cu:90-582, nep.cu:503-561):
// the Verlet list of all pairs with float d^2 < (rc + skin)^2 is rebuilt when
// any atom moved more than skin/2 since the last build; every force call
// filters it into typewise radial and angular lists with float
// d^2 < ((rc_t1 + rc_t2)/2)^2.  Rows are ascending in atom index.
//
// B200 design: everything stays on the device.  The skin check sets a device
// flag that the rebuild kernels read (they return at once when it is clear),
// so a step never waits on the host.  Rows are row-major (atom i owns the
// contiguous slots [i*MN, i*MN + count)) so the warp that owns a center reads
// and writes coalesced.  The cell list is a counting sort on a grid of cells
// at least (rc + skin)/2 wide with a 5x5x5 stencil; each Verlet row is sorted
// in shared memory, which makes every later sum over neighbours ordered and
// bitwise reproducible.
#include <algorithm>
#include <climits>

#include "engine.h"

namespace nepx {

namespace {

__device__ __forceinline__ int wrapped_cell(double s, int nc, int pbc)
{
  if (!pbc) return 0;
  s -= floor(s);
  int c = static_cast<int>(s * nc);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__device__ __forceinline__ void cell_coords(const Box& b, const NeighborState& st, double x,
                                            double y, double z, int& cx, int& cy, int& cz)
{
  const double sx = b.hinv[0] * x + b.hinv[1] * y + b.hinv[2] * z;
  const double sy = b.hinv[3] * x + b.hinv[4] * y + b.hinv[5] * z;
  const double sz = b.hinv[6] * x + b.hinv[7] * y + b.hinv[8] * z;
  cx = wrapped_cell(sx, st.nc[0], b.pbc[0]);
  cy = wrapped_cell(sy, st.nc[1], b.pbc[1]);
  cz = wrapped_cell(sz, st.nc[2], b.pbc[2]);
}

// Packs each atom into its Site record for the neighbour sweeps of this
// step and applies the skin criterion (skin_check_atom, common.cuh).  The MD
// step does the same inside its first half kick instead.
__global__ void k_skin_check(int N, const Box* __restrict__ box, const double* __restrict__ pos,
                             const int* __restrict__ type, const double* __restrict__ x0,
                             NeighborState* st, Site* __restrict__ sites, double skin,
                             double rc_v, int force)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  skin_check_atom(N, i, *box, pos[i], pos[N + i], pos[2 * N + i], type[i], x0, st, sites, skin,
                  rc_v, force);
}

// Cell grid from the current box (cells at least rc_v/2 thick, at most
// cell_cap of them), then clears the counts.  One block.
__global__ void k_cell_setup(const Box* __restrict__ box, NeighborState* st, int* cell_count,
                             double rc_v, int cell_cap)
{
  __shared__ int s_ncell;
  if (!st->rebuild) return;
  if (threadIdx.x == 0) {
    st->box_scale = 1.0;
    for (int k = 0; k < 9; ++k) st->box_def[k] = (k % 4 == 0) ? 1.0 : 0.0;
    const Box& b = *box;
    double vol = fabs(b.h[0] * (b.h[4] * b.h[8] - b.h[5] * b.h[7]) +
                      b.h[1] * (b.h[5] * b.h[6] - b.h[3] * b.h[8]) +
                      b.h[2] * (b.h[3] * b.h[7] - b.h[4] * b.h[6]));
    int nc[3];
    double width = 0.5 * rc_v;
    for (int pass = 0; pass < 64; ++pass) {
      long long total = 1;
      for (int d = 0; d < 3; ++d) {
        // thickness along direction d = 1 / |row d of hinv|
        const double* r = b.hinv + 3 * d;
        const double thick = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        nc[d] = b.pbc[d] ? max(1, static_cast<int>(floor(thick / width))) : 1;
        total *= nc[d];
      }
      if (total <= cell_cap) break;
      width *= 1.25;
    }
    (void)vol;
    st->nc[0] = nc[0];
    st->nc[1] = nc[1];
    st->nc[2] = nc[2];
    st->ncell = nc[0] * nc[1] * nc[2];
    s_ncell = st->ncell;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < s_ncell; c += blockDim.x) cell_count[c] = 0;
}

__global__ void k_cell_count(int N, const Box* __restrict__ box, const double* __restrict__ pos,
                             const NeighborState* __restrict__ st, int* cell_of, int* cell_count)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!st->rebuild || i >= N) return;
  int cx, cy, cz;
  cell_coords(*box, *st, pos[i], pos[N + i], pos[2 * N + i], cx, cy, cz);
  const int c = (cz * st->nc[1] + cy) * st->nc[0] + cx;
  cell_of[i] = c;
  atomicAdd(cell_count + c, 1);
}

// Exclusive scan of the cell counts (one block); resets the counts to serve
// as fill cursors.
__global__ void k_cell_scan(const NeighborState* __restrict__ st, int* cell_count, int* cell_start)
{
  __shared__ int s_part[1024];
  if (!st->rebuild) return;
  const int n = st->ncell;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per;
  const int hi = min(n, lo + per);
  int sum = 0;
  for (int c = lo; c < hi; ++c) sum += cell_count[c];
  s_part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < blockDim.x; off <<= 1) {
    int v = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0;
    __syncthreads();
    s_part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = s_part[threadIdx.x] - sum;
  for (int c = lo; c < hi; ++c) {
    const int k = cell_count[c];
    cell_start[c] = run;
    run += k;
    cell_count[c] = 0;
  }
}

__global__ void k_cell_fill(int N, const NeighborState* __restrict__ st, const int* __restrict__ cell_of,
                            int* cell_count, const int* __restrict__ cell_start, int* cell_atoms)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (!st->rebuild || i >= N) return;
  const int c = cell_of[i];
  const int slot = atomicAdd(cell_count + c, 1);
  cell_atoms[cell_start[c] + slot] = i;
}

// One warp per center: gathers every candidate of the 5x5x5 stencil with
// float d^2 < (rc + skin)^2, sorts the row in shared memory (bitonic), and
// writes it with the reference positions for the next skin check.
__global__ void k_verlet_build(int N, const Box* __restrict__ box, const Site* __restrict__ sites,
                               NeighborState* st, const int* __restrict__ cell_count,
                               const int* __restrict__ cell_start, const int* __restrict__ cell_atoms,
                               const int* __restrict__ cell_of, int* nn_v, int* nl_v, int mn_v,
                               int pow2, float cutoff_square, double* x0)
{
  extern __shared__ int s_rows[];
  if (!st->rebuild) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  int* buf = s_rows + warp * (pow2 + 1);
  int* count = buf + pow2;
  const Box b = *box;
  for (int i = blockIdx.x * wpb + warp; i < N; i += gridDim.x * wpb) {
  if (lane == 0) *count = 0;
  __syncwarp();
  const double xi = sites[i].x, yi = sites[i].y, zi = sites[i].z;
  const int nc0 = st->nc[0], nc1 = st->nc[1], nc2 = st->nc[2];
  const int ci = cell_of[i];
  const int cx = ci % nc0, cy = (ci / nc0) % nc1, cz = ci / (nc0 * nc1);
  // per direction: 5 wrapped offsets when the grid is wide enough, else
  // every cell of that direction exactly once
  const int span0 = (b.pbc[0] && nc0 >= 5) ? 5 : nc0;
  const int span1 = (b.pbc[1] && nc1 >= 5) ? 5 : nc1;
  const int span2 = (b.pbc[2] && nc2 >= 5) ? 5 : nc2;
  const int ncand = span0 * span1 * span2;
  for (int s = lane; s < ncand; s += 32) {
    const int s0 = s % span0, s1 = (s / span0) % span1, s2 = s / (span0 * span1);
    int gx = span0 == 5 ? cx + s0 - 2 : s0;
    int gy = span1 == 5 ? cy + s1 - 2 : s1;
    int gz = span2 == 5 ? cz + s2 - 2 : s2;
    if (gx < 0) gx += nc0; else if (gx >= nc0) gx -= nc0;
    if (gy < 0) gy += nc1; else if (gy >= nc1) gy -= nc1;
    if (gz < 0) gz += nc2; else if (gz >= nc2) gz -= nc2;
    const int c = (gz * nc1 + gy) * nc0 + gx;
    const int start = cell_start[c];
    const int cnt = cell_count[c];
    for (int m = 0; m < cnt; ++m) {
      const int j = cell_atoms[start + m];
      if (j == i) continue;
      float dx, dy, dz;
      int tj;
      site_displacement(b, sites, xi, yi, zi, j, dx, dy, dz, tj);
      const float d2 = dx * dx + dy * dy + dz * dz;
      if (d2 < cutoff_square) {
        const int slot = atomicAdd(count, 1);
        if (slot < pow2) buf[slot] = j;
      }
    }
  }
  __syncwarp();
  const int total = *count;
  const int used = min(total, pow2);
  // bitonic sort of the smallest power of two that holds the row (padding
  // INT_MAX), one compare-exchange pair per lane and pass
  int p2 = 1;
  while (p2 < used) p2 <<= 1;
  for (int k = used + lane; k < p2; k += 32) buf[k] = INT_MAX;
  __syncwarp();
  for (int k = 2; k <= p2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < (p2 >> 1); q += 32) {
        const int t = ((q & ~(j - 1)) << 1) | (q & (j - 1));   // lower index of the pair
        const int u = t | j;
        const int a = buf[t], c = buf[u];
        const bool up = (t & k) == 0;
        if ((a > c) == up) {
          buf[t] = c;
          buf[u] = a;
        }
      }
      __syncwarp();
    }
  }
  const int keep = min(total, mn_v);
  int* row = nl_v + static_cast<size_t>(i) * mn_v;
  for (int k = lane; k < keep; k += 32) row[k] = buf[k];
  if (lane == 0) {
    nn_v[i] = keep;
    if (total > mn_v) atomicOr(&st->overflow, 1);
    atomicMax(&st->max_nn[0], total);
    x0[i] = xi;
    x0[N + i] = yi;
    x0[2 * N + i] = zi;
  }
  __syncwarp();   // the row buffer is reused by this warp's next center
  }
}

}  // namespace

void launch_neighbor_update(Engine& e, int N, const double* pos, const int* type, bool force,
                            cudaStream_t stream, bool skin_done)
{
  if (e.use_xr) {
    launch_explicit_rows(e, N, pos, type, stream);
    return;
  }
  NeighborBuffers& nb = e.nbr;
  const int threads = 256;
  const int grid = (N + threads - 1) / threads;
  const double rc_v_d = static_cast<double>(e.model.rc_max) + e.skin;
  if (!skin_done)
    k_skin_check<<<grid, threads, 0, stream>>>(N, e.d_box, pos, type, nb.x0, e.d_nstate,
                                                e.scratch.sites, e.skin, rc_v_d, force ? 1 : 0);
  k_cell_setup<<<1, 1024, 0, stream>>>(e.d_box, e.d_nstate, nb.cell_count, rc_v_d, nb.cell_cap);
  k_cell_count<<<grid, threads, 0, stream>>>(N, e.d_box, pos, e.d_nstate, nb.cell_of,
                                             nb.cell_count);
  k_cell_scan<<<1, 1024, 0, stream>>>(e.d_nstate, nb.cell_count, nb.cell_start);
  k_cell_fill<<<grid, threads, 0, stream>>>(N, e.d_nstate, nb.cell_of, nb.cell_count,
                                            nb.cell_start, nb.cell_atoms);
  // cell counts were consumed as cursors; they now hold the per-cell totals again
  // a grid of at most 16 CTAs per SM walks all centers, so the launch is
  // cheap on the (common) steps whose skin check found nothing to rebuild
  const int warps = 4;
  const size_t smem = static_cast<size_t>(warps) * (nb.pow2_v + 1) * sizeof(int);
  const int vblocks = std::min((N + warps - 1) / warps, 148 * 16);
  k_verlet_build<<<vblocks, warps * 32, smem, stream>>>(
    N, e.d_box, e.scratch.sites, e.d_nstate, nb.cell_count, nb.cell_start, nb.cell_atoms, nb.cell_of,
    nb.nn_v, nb.nl_v, nb.mn_v, nb.pow2_v, static_cast<float>(rc_v_d * rc_v_d), nb.x0);
  // the typewise radial / angular filter follows in k_filter_radial
}

}  // namespace nepx

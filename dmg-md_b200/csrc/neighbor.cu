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
// B200 design: everything stays on the device, in one cooperative launch.
// Its phases -- skin check, cell grid, counting sort of the atoms into cells,
// Verlet rows -- are separated by grid-wide barriers (every
// block is resident, and every wait is bounded); a step whose skin check
// finds nothing to rebuild costs that one launch, which returns at once, and
// never waits on the host.  Rows are row-major (atom i owns the contiguous
// slots [i*MN, i*MN + count)) so the warp that owns a center reads and writes
// coalesced.  The cell list is a counting sort on a grid of cells at least
// (rc + skin)/2 wide with a 5x5x5 stencil; each Verlet row is sorted in
// shared memory, which makes every later sum over neighbours ordered and
// bitwise reproducible.
#include <algorithm>
#include <climits>

#include "engine.h"

namespace nepx {

namespace {

constexpr int kRebuildThreads = 128;                 // four warps: a center per warp in the row build
constexpr int kRebuildWarps = kRebuildThreads / 32;
constexpr long long kGridWaitCycles = 4000000000ll;  // ~2 s at the B200 clock

__device__ __forceinline__ int wrapped_cell(double s, int nc, int pbc)
{
  if (!pbc) return 0;
  s -= floor(s);
  int c = static_cast<int>(s * nc);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

// Packs each atom into its Site record for the neighbour sweeps of this
// step and applies the skin criterion (skin_check_atom, common.cuh).  The MD
// step does the same inside its first half kick instead.
__device__ __forceinline__ void skin_phase(int N, const Box& b, const double* __restrict__ pos,
                                           const int* __restrict__ type,
                                           const double* __restrict__ x0, NeighborState* st,
                                           Site* __restrict__ sites, double skin, double rc_v,
                                           int force)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    skin_check_atom(N, i, b, pos[i], pos[N + i], pos[2 * N + i], type[i], x0, st, sites, skin,
                    rc_v, force);
}

// Grid-wide barrier of the cooperative rebuild.  A generation counter: the
// last block to arrive resets the arrival count and advances the generation,
// the others wait for the advance -- at most kGridWaitCycles, after which they
// record the timeout in sync_error and go on (the call then reports an error).
__device__ void grid_sync(unsigned* gs, NeighborState* st)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = gs + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(gs, 1u) == gridDim.x - 1) {
      atomicExch(gs, 0u);
      __threadfence();
      atomicAdd(gs + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (*gen == g) {
        if (clock64() - t0 > kGridWaitCycles) {
          atomicOr(&st->sync_error, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Sum over the block (kRebuildThreads threads).
__device__ int block_sum(int v, int* s_tmp)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_tmp[warp] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < kRebuildWarps; ++w) t += s_tmp[w];
  return t;
}

// Inclusive prefix sum over the block; *total gets the block's sum.
__device__ int block_scan(int v, int* s_tmp, int* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) s_tmp[warp] = x;
  __syncthreads();
  int before = 0, t = 0;
  for (int w = 0; w < kRebuildWarps; ++w) {
    if (w < warp) before += s_tmp[w];
    t += s_tmp[w];
  }
  *total = t;
  return x + before;
}

// Compare-exchange of two values held by one lane: the pair's lower element
// keeps the smaller value when its block sorts ascending.
__device__ __forceinline__ void cx_pair(int& lo, int& hi, bool ascending)
{
  const int a = min(lo, hi), c = max(lo, hi);
  lo = ascending ? a : c;
  hi = ascending ? c : a;
}

// Ascending bitonic sort of the first p2 (a power of two, at most 128)
// values of a warp, four per lane: element e = lane + 32 r is v[r] (padding
// INT_MAX).  Partners e ^ jj exchange by shuffle (jj < 32) or inside the
// lane (jj = 32, 64); e keeps the smaller value when (e < partner) matches the
// ascending direction (e & k) == 0 of its block.
__device__ __forceinline__ void warp_sort128(int (&v)[4], int p2, int lane)
{
  for (int k = 2; k <= p2; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      if (jj == 64) {
        cx_pair(v[0], v[2], (lane & k) == 0);
        cx_pair(v[1], v[3], ((lane + 32) & k) == 0);
      } else if (jj == 32) {
        cx_pair(v[0], v[1], (lane & k) == 0);
        cx_pair(v[2], v[3], ((lane + 64) & k) == 0);
      } else {
        const bool lower = (lane & jj) == 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int pv = __shfl_xor_sync(0xffffffffu, v[r], jj);
          const bool asc = ((lane + 32 * r) & k) == 0;
          v[r] = (lower == asc) ? min(v[r], pv) : max(v[r], pv);
        }
      }
    }
  }
}

struct RebuildArgs {
  int N;
  const Box* box;
  const double* pos;
  const int* type;
  NeighborState* st;
  Site* sites;
  int* cell_count;
  int* cell_start;
  int* cell_atoms;
  int* cell_of;
  Site* cell_sites;    // the site records in cell order (beside cell_atoms)
  int* nn_v;
  int* nl_v;
  double* x0;
  unsigned* gsync;
  int* part;           // [gridDim.x] per-block sums of the cell scan
  int mn_v, pow2, cell_cap;
  double skin, rc_v;
  float cutoff_square;
  double prune_square; // (rc_v (1 + 1e-5) + 1e-5)^2: the stencil rows' trimming bound
  int skin_check;      // 1: pack the sites and apply the skin criterion first
  int force;           // with skin_check: rebuild whatever the displacements
};

// The whole neighbour update in one cooperative launch (grid-stride phases,
// grid_sync between them):
//   0. (skin_check) site records and the skin criterion;
//   1. cell grid from the current box (cells at least rc_v/2 thick, at most
//      cell_cap of them), counts cleared;
//   2. cell of every atom, counts;
//   3. exclusive scan of the counts (per-block chunks, then block offsets);
//   4. atoms into their cells (index and site record, in cell order);
//   5. Verlet rows: one warp per center gathers every candidate of the 5x5x5
//      stencil (its rows along x, trimmed to the cells in reach) with float
//      d^2 < (rc + skin)^2, sorts the row (bitonic, in registers up to 128
//      entries) and writes it with the reference positions of the next skin
//      check.
// Phases 1-5 run only when the rebuild flag is set; the flag is the same for
// every block, so all of them return together.
__global__ void __launch_bounds__(kRebuildThreads, 12)
k_neighbor_rebuild(const RebuildArgs a)
{
  extern __shared__ int s_rows[];
  __shared__ int s_tmp[kRebuildWarps];
  __shared__ int s_grid[4];
  NeighborState* st = a.st;
  const int N = a.N;
  const int tid = threadIdx.x;
  const int gtid = blockIdx.x * blockDim.x + tid, nthreads = gridDim.x * blockDim.x;
  const Box b = *a.box;
  if (a.skin_check) {
    skin_phase(N, b, a.pos, a.type, a.x0, st, a.sites, a.skin, a.rc_v, a.force);
    grid_sync(a.gsync, st);
  }
  if (!*reinterpret_cast<volatile int*>(&st->rebuild)) return;

  // 1. cell grid (every block derives the same one; block 0 records it)
  if (tid == 0) {
    int nc[3];
    double width = 0.5 * a.rc_v;
    for (int pass = 0; pass < 64; ++pass) {
      long long total = 1;
      for (int d = 0; d < 3; ++d) {
        // thickness along direction d = 1 / |row d of hinv|
        const double* r = b.hinv + 3 * d;
        const double thick = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        nc[d] = b.pbc[d] ? max(1, static_cast<int>(floor(thick / width))) : 1;
        total *= nc[d];
      }
      if (total <= a.cell_cap) break;
      width *= 1.25;
    }
    s_grid[0] = nc[0];
    s_grid[1] = nc[1];
    s_grid[2] = nc[2];
    s_grid[3] = nc[0] * nc[1] * nc[2];
    if (blockIdx.x == 0) {
      st->box_scale = 1.0;
      for (int k = 0; k < 9; ++k) st->box_def[k] = (k % 4 == 0) ? 1.0 : 0.0;
      st->nc[0] = nc[0];
      st->nc[1] = nc[1];
      st->nc[2] = nc[2];
      st->ncell = s_grid[3];
    }
  }
  __syncthreads();
  const int nc0 = s_grid[0], nc1 = s_grid[1], nc2 = s_grid[2], ncell = s_grid[3];
  for (int c = gtid; c < ncell; c += nthreads) a.cell_count[c] = 0;
  grid_sync(a.gsync, st);

  // 2. cells and counts
  for (int i = gtid; i < N; i += nthreads) {
    const double x = a.pos[i], y = a.pos[N + i], z = a.pos[2 * N + i];
    const double sx = b.hinv[0] * x + b.hinv[1] * y + b.hinv[2] * z;
    const double sy = b.hinv[3] * x + b.hinv[4] * y + b.hinv[5] * z;
    const double sz = b.hinv[6] * x + b.hinv[7] * y + b.hinv[8] * z;
    const int c = (wrapped_cell(sz, nc2, b.pbc[2]) * nc1 + wrapped_cell(sy, nc1, b.pbc[1])) * nc0 +
                  wrapped_cell(sx, nc0, b.pbc[0]);
    a.cell_of[i] = c;
    atomicAdd(a.cell_count + c, 1);
  }
  grid_sync(a.gsync, st);

  // 3. exclusive scan: block sums of contiguous chunks, then each block
  //    scans its chunk from the sum of the chunks before it; the counts
  //    are reset to serve as fill cursors
  const int chunk = (ncell + gridDim.x - 1) / gridDim.x;
  const int c0 = min(ncell, static_cast<int>(blockIdx.x) * chunk), c1 = min(ncell, c0 + chunk);
  {
    int sum = 0;
    for (int c = c0 + tid; c < c1; c += blockDim.x) sum += a.cell_count[c];
    sum = block_sum(sum, s_tmp);
    if (tid == 0) a.part[blockIdx.x] = sum;
  }
  grid_sync(a.gsync, st);
  {
    int off = 0;
    for (int q = tid; q < static_cast<int>(blockIdx.x); q += blockDim.x) off += a.part[q];
    off = block_sum(off, s_tmp);
    for (int base = c0; base < c1; base += blockDim.x) {
      const int c = base + tid;
      const int v = c < c1 ? a.cell_count[c] : 0;
      int tile = 0;
      const int incl = block_scan(v, s_tmp, &tile);
      if (c < c1) {
        a.cell_start[c] = off + incl - v;
        a.cell_count[c] = 0;
      }
      off += tile;
    }
  }
  grid_sync(a.gsync, st);

  // 4. fill (the counts are the cell totals again afterwards); each atom's
  //    site record goes beside its index, so a cell's candidates are one
  //    contiguous run of records
  for (int i = gtid; i < N; i += nthreads) {
    const int c = a.cell_of[i];
    const int slot = atomicAdd(a.cell_count + c, 1);
    const int at = a.cell_start[c] + slot;
    a.cell_atoms[at] = i;
    a.cell_sites[at] = a.sites[i];
  }
  grid_sync(a.gsync, st);

  // 5. Verlet rows, one warp per center.  The 5x5x5 stencil is taken as its
  //    25 rows of cells along x (span1 x span2 of them on narrow grids); a
  //    row's cells are consecutive in the cell order, so its atoms are one
  //    contiguous run of the cell-ordered arrays (two where the row wraps
  //    around the box).  In an orthogonal box each row is trimmed to the
  //    cells that can hold a neighbour: a row whose y-z distance from the
  //    center exceeds rc + skin is dropped, and the x extent keeps the
  //    offsets whose distance along x fits in what is left (the bound is the
  //    exact geometric distance to the cell, widened by 1e-5 relative so
  //    that no pair the float predicate accepts is ever cut).  Lane r takes
  //    row r, a warp prefix sum of the runs flattens them into one range,
  //    and the warp sweeps it 32 candidates at a time, reading the
  //    cell-ordered index and site record side by side.  Hits are compacted
  //    in order of discovery (ballot + popcount) and the row is sorted: in
  //    registers, four values per lane, up to 128 entries; in shared memory
  //    above.
  const int lane = tid & 31, warp = tid >> 5;
  const unsigned below = (1u << lane) - 1u;
  const int pow2 = a.pow2;
  int* buf = s_rows + warp * (pow2 + 1);
  const int span0 = (b.pbc[0] && nc0 >= 5) ? 5 : nc0;
  const int span1 = (b.pbc[1] && nc1 >= 5) ? 5 : nc1;
  const int span2 = (b.pbc[2] && nc2 >= 5) ? 5 : nc2;
  const int nrows = span1 * span2;   // at most 25
  const bool prune = b.ortho != 0;
  const double w0 = b.h[0] / nc0, w1 = b.h[4] / nc1, w2 = b.h[8] / nc2;
  const double r2 = a.prune_square;
  for (int i = blockIdx.x * kRebuildWarps + warp; i < N; i += gridDim.x * kRebuildWarps) {
    // the site records may have been written by this launch (phase 0): plain
    // loads, which the barriers order, not the read-only path
    const double xi = a.sites[i].x, yi = a.sites[i].y, zi = a.sites[i].z;
    const int ci = a.cell_of[i];
    const int cx = ci % nc0, cy = (ci / nc0) % nc1, cz = ci / (nc0 * nc1);
    int st1 = 0, n1 = 0, st2 = 0, n2 = 0;
    if (lane < nrows) {
      const int q1 = lane % span1, q2 = lane / span1;
      // the center's position inside its cell, in cell widths (phase 2's
      // fractional coordinates)
      auto frac = [&](int d, int c, int nc) {
        double sd = b.hinv[3 * d] * xi + b.hinv[3 * d + 1] * yi + b.hinv[3 * d + 2] * zi;
        sd -= floor(sd);
        return fmin(fmax(sd * nc - c, 0.0), 1.0);
      };
      // distance from the center to the cells k rows away along a direction
      auto gap = [](int k, double u, double w) {
        return k > 0 ? (k - u) * w : (k < 0 ? (u - k - 1) * w : 0.0);
      };
      double dyz2 = 0.0;
      double ux = 0.0;
      if (prune) {
        if (span1 == 5) {
          const double g = gap(q1 - 2, frac(1, cy, nc1), w1);
          dyz2 += g * g;
        }
        if (span2 == 5) {
          const double g = gap(q2 - 2, frac(2, cz, nc2), w2);
          dyz2 += g * g;
        }
        if (span0 == 5) ux = frac(0, cx, nc0);
      }
      if (dyz2 < r2) {
        int gy = span1 == 5 ? cy + q1 - 2 : q1;
        int gz = span2 == 5 ? cz + q2 - 2 : q2;
        if (gy < 0) gy += nc1; else if (gy >= nc1) gy -= nc1;
        if (gz < 0) gz += nc2; else if (gz >= nc2) gz -= nc2;
        const int row = (gz * nc1 + gy) * nc0;
        // atoms of the row's cells c0..c1 (consecutive)
        auto run = [&](int c0, int c1, int& st, int& n) {
          st = a.cell_start[row + c0];
          n = a.cell_start[row + c1] + a.cell_count[row + c1] - st;
        };
        if (span0 < 5) {
          run(0, nc0 - 1, st1, n1);
        } else {
          int klo = -2, khi = 2;
          if (prune) {
            const double rx2 = r2 - dyz2;
            auto within = [&](int k) {
              const double g = gap(k, ux, w0);
              return g * g < rx2;
            };
            klo = within(-1) ? (within(-2) ? -2 : -1) : 0;
            khi = within(1) ? (within(2) ? 2 : 1) : 0;
          }
          const int g0 = cx + klo, g1 = cx + khi;
          if (g0 < 0) {
            run(g0 + nc0, nc0 - 1, st1, n1);
            run(0, g1, st2, n2);
          } else if (g1 >= nc0) {
            run(g0, nc0 - 1, st1, n1);
            run(0, g1 - nc0, st2, n2);
          } else {
            run(g0, g1, st1, n1);
          }
        }
      }
    }
    const int my_cnt = n1 + n2;
    int incl = my_cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total_c = __shfl_sync(0xffffffffu, incl, 31);
    int total = 0;
    for (int base = 0; base < total_c; base += 32) {
      const int k = base + lane;
      // stencil row of candidate k: the first lane whose inclusive count exceeds k
      int lo = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
        if (v <= k) lo += step;
      }
      const int r_incl = __shfl_sync(0xffffffffu, incl, lo);
      const int r_cnt = __shfl_sync(0xffffffffu, my_cnt, lo);
      const int r_st1 = __shfl_sync(0xffffffffu, st1, lo);
      const int r_n1 = __shfl_sync(0xffffffffu, n1, lo);
      const int r_st2 = __shfl_sync(0xffffffffu, st2, lo);
      bool hit = false;
      int j = 0;
      if (k < total_c) {
        const int local = k - (r_incl - r_cnt);
        const int at = local < r_n1 ? r_st1 + local : r_st2 + (local - r_n1);
        j = a.cell_atoms[at];
        const double2 sa = reinterpret_cast<const double2*>(a.cell_sites + at)[0];
        const double2 sc = reinterpret_cast<const double2*>(a.cell_sites + at)[1];
        float dx, dy, dz;
        int tj;
        site_delta(b, sa, sc, xi, yi, zi, dx, dy, dz, tj);
        const float d2 = dx * dx + dy * dy + dz * dz;
        hit = j != i && d2 < a.cutoff_square;
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const int slot = total + __popc(m & below);
        if (slot < pow2) buf[slot] = j;
      }
      total += __popc(m);
    }
    __syncwarp();
    const int used = min(total, pow2);
    int p2 = 1;
    while (p2 < used) p2 <<= 1;
    const int keep = min(total, a.mn_v);
    int* row = a.nl_v + static_cast<size_t>(i) * a.mn_v;
    if (p2 <= 128) {
      int v[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) v[r] = lane + 32 * r < used ? buf[lane + 32 * r] : INT_MAX;
      warp_sort128(v, p2, lane);
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (lane + 32 * r < keep) row[lane + 32 * r] = v[r];
    } else {
      // bitonic sort of the smallest power of two that holds the row (padding
      // INT_MAX), one compare-exchange pair per lane and pass
      for (int k = used + lane; k < p2; k += 32) buf[k] = INT_MAX;
      __syncwarp();
      for (int k = 2; k <= p2; k <<= 1) {
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
          for (int q = lane; q < (p2 >> 1); q += 32) {
            const int t = ((q & ~(jj - 1)) << 1) | (q & (jj - 1));   // lower index of the pair
            const int u = t | jj;
            const int x = buf[t], y = buf[u];
            const bool up = (t & k) == 0;
            if ((x > y) == up) {
              buf[t] = y;
              buf[u] = x;
            }
          }
          __syncwarp();
        }
      }
      for (int k = lane; k < keep; k += 32) row[k] = buf[k];
    }
    if (lane == 0) {
      a.nn_v[i] = keep;
      if (total > a.mn_v) atomicOr(&st->overflow, 1);
      atomicMax(&st->max_nn[0], total);
      a.x0[i] = xi;
      a.x0[N + i] = yi;
      a.x0[2 * N + i] = zi;
    }
    __syncwarp();   // the row buffer is reused by this warp's next center
  }
}

size_t rebuild_smem(int pow2) { return sizeof(int) * kRebuildWarps * (pow2 + 1); }

}  // namespace

// Blocks of the cooperative rebuild: as many as can be resident at once (the
// launch fails rather than oversubscribe), at most 16 per SM.
int neighbor_rebuild_blocks(int pow2_v)
{
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_neighbor_rebuild, kRebuildThreads,
                                                    rebuild_smem(pow2_v)) != cudaSuccess)
    return 0;
  return sms * std::min(per_sm, 16);
}

void launch_neighbor_update(Engine& e, int N, const double* pos, const int* type, bool force,
                            cudaStream_t stream, bool skin_done)
{
  if (e.use_xr) {
    launch_explicit_rows(e, N, pos, type, stream);
    return;
  }
  NeighborBuffers& nb = e.nbr;
  if (nb.gsync_dirty) {
    // a barrier gave up waiting in an earlier launch: restart its counters
    cudaMemsetAsync(nb.gsync, 0, 2 * sizeof(unsigned), stream);
    nb.gsync_dirty = false;
  }
  RebuildArgs a;
  a.N = N;
  a.box = e.d_box;
  a.pos = pos;
  a.type = type;
  a.st = e.d_nstate;
  a.sites = e.scratch.sites;
  a.cell_count = nb.cell_count;
  a.cell_start = nb.cell_start;
  a.cell_atoms = nb.cell_atoms;
  a.cell_of = nb.cell_of;
  a.cell_sites = nb.cell_sites;
  a.nn_v = nb.nn_v;
  a.nl_v = nb.nl_v;
  a.x0 = nb.x0;
  a.gsync = nb.gsync;
  a.part = nb.scan_part;
  a.mn_v = nb.mn_v;
  a.pow2 = nb.pow2_v;
  a.cell_cap = nb.cell_cap;
  a.skin = e.skin;
  a.rc_v = static_cast<double>(e.model.rc_max) + e.skin;
  a.cutoff_square = static_cast<float>(a.rc_v * a.rc_v);
  const double rp = a.rc_v * (1.0 + 1e-5) + 1e-5;
  a.prune_square = rp * rp;
  a.skin_check = skin_done ? 0 : 1;
  a.force = force ? 1 : 0;
  // small systems take fewer blocks: cheaper barriers, nothing to share out
  const int want = std::max(1, (N + kRebuildWarps - 1) / kRebuildWarps);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(std::min(nb.rebuild_blocks, want)));
  cfg.blockDim = dim3(kRebuildThreads);
  cfg.dynamicSmemBytes = rebuild_smem(nb.pow2_v);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_neighbor_rebuild, a);
  // the typewise radial / angular filter follows in k_filter_radial (which
  // clears the rebuild flag)
}

}  // namespace nepx

// explicit.cu -- neighbour rows with explicit displacements: the small-box
// path and the batched path.
//
// Reference small-box path (src/gpumd_compat/nep_small_box.cuh:56-120,
// find_neighbor_list_small_box; nep.cu:1900-2000, compute_small_box): when a
// periodic direction is thinner than 2.5 (rc + 1) every center scans every
// atom of its system and every image of the expanded box, keeping the pairs
// inside the typewise radial / angular cutoffs together with the float
// displacement r12 of that image.  Rows follow (j ascending, then images
// ia, ib, ic) and are rebuilt at every force call.
//
// Here one warp owns a center and its lanes take consecutive candidates j;
// per 32-candidate chunk each lane counts its edges over all images, a warp
// scan gives every lane its write offset and a second pass writes the edges,
// so rows keep the reference's order.  The same kernel serves any number of
// structures packed into one atom range (the batched path): a center finds
// its structure by binary search over the structure offsets.  Structures
// that are not small use the large-box arithmetic (double difference rounded
// to float, float minimum image, reference nep.cu:503-561); their candidates
// come from a cell grid of their own (cells at least rc/2 thick, 5x5x5 stencil,
// a counting sort per batch scanned per structure), and each row is sorted
// (warp-shuffle bitonic network up to 64 entries, shared memory above), which
// yields the large-box path's typewise rows exactly.  Those structures' rows
// hold each neighbour once, so a batch marks their centers (large[]) for the
// directed-f12 scheme of the large-box path.
//
// Row entry: float4 (x12, y12, z12, bits of j | type(j) << 28), row-major
// [center][slot]; radial and angular rows are separate.
#include <algorithm>
#include <climits>
#include <cmath>
#include <string>

#include "engine.h"
#include "xbox.h"

namespace nepx {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__global__ void k_pack_sites(int N, const double* __restrict__ pos, const int* __restrict__ type,
                             Site* __restrict__ sites, NeighborState* st)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (i == 0) {   // the first kernel of a force evaluation: its row maxima start here
    st->call_nn[0] = 0;
    st->call_nn[1] = 0;
  }
  sites[i] = Site{pos[i], pos[N + i], pos[2 * N + i], static_cast<long long>(type[i])};
}

// One structure spanning all N atoms, its StructInfo from the device box.
__global__ void k_struct_from_box(const Box* __restrict__ box, double rc, int N, StructInfo* si,
                                  int* soff, NeighborState* st)
{
  StructInfo s;
  if (expanded_box(*box, rc, s)) st->box_error = 1;
  s.off = 0;
  s.n = N;
  *si = s;
  soff[0] = 0;
  soff[1] = N;
}

// Minimum image in the expanded box (reference nep_small_box.cuh:39-54).
__device__ __forceinline__ void mic_small_box(const StructInfo& s, float& x12, float& y12,
                                              float& z12)
{
  const float* e = s.eh;
  float sx12 = e[9] * x12 + e[10] * y12 + e[11] * z12;
  float sy12 = e[12] * x12 + e[13] * y12 + e[14] * z12;
  float sz12 = e[15] * x12 + e[16] * y12 + e[17] * z12;
  if (s.box.pbc[0] == 1) sx12 -= nearbyintf(sx12);
  if (s.box.pbc[1] == 1) sy12 -= nearbyintf(sy12);
  if (s.box.pbc[2] == 1) sz12 -= nearbyintf(sz12);
  x12 = e[0] * sx12 + e[1] * sy12 + e[2] * sz12;
  y12 = e[3] * sx12 + e[4] * sy12 + e[5] * sz12;
  z12 = e[6] * sx12 + e[7] * sy12 + e[8] * sz12;
}

// Displacement from a center (float position) to atom j (double position) at
// image (ia, ib, ic) of the expanded box: the reference's small-box
// arithmetic (nep_small_box.cuh:134-143).  Shared by the row builder and the
// Verlet-candidate filter, so both produce the same float values.
__device__ __forceinline__ void small_box_delta(const StructInfo& s, float x1, float y1,
                                                float z1, double xj, double yj, double zj,
                                                int ia, int ib, int ic, float& x12, float& y12,
                                                float& z12)
{
  const float* fh = s.box.fh;
  const float d0 = fh[0] * ia + fh[1] * ib + fh[2] * ic;
  const float d1 = fh[3] * ia + fh[4] * ib + fh[5] * ic;
  const float d2 = fh[6] * ia + fh[7] * ib + fh[8] * ic;
  x12 = xj + d0 - x1;
  y12 = yj + d1 - y1;
  z12 = zj + d2 - z1;
  mic_small_box(s, x12, y12, z12);
}

__device__ __forceinline__ float4 row_entry(float x, float y, float z, int j, int t)
{
  return make_float4(x, y, z, __int_as_float(j | (t << kRowTypeShift)));
}

__global__ void __launch_bounds__(256)
k_rows_explicit(const ModelParams p, int total, const StructInfo* __restrict__ si,
                const int* __restrict__ soff, int S, const double* __restrict__ pos,
                const int* __restrict__ type, int* __restrict__ nn_r, float4* __restrict__ er,
                int mn_r, int* __restrict__ nn_a, float4* __restrict__ ea, int mn_a,
                const int* __restrict__ cell_count, const int* __restrict__ cell_start,
                const int* __restrict__ cell_atoms, const int* __restrict__ cell_of, int p2r,
                const Site* __restrict__ sites, unsigned char* __restrict__ large, int mark_large,
                const BatchVerlet bv, NeighborState* st)
{
  extern __shared__ int s_rows[];   // per warp: p2r row slots + a counter
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < total; i += gridDim.x * wpb) {
    // structure of center i: the last s with soff[s] <= i
    int lo = 0, hi = S - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (soff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    const StructInfo& s = si[lo];
    const int off = s.off, n = s.n;
    const int t1 = type[i];
    const float rr1 = p.rc_r[t1], ra1 = p.rc_a[t1];
    // a structure that keeps Verlet candidates: (re)build them here when it is
    // new or has moved more than skin / 2 since the build; its rows come from
    // them in k_rows_verlet
    const int sf = bv.sflag ? bv.sflag[lo] : 0;
    const bool keep = (sf & 2) != 0;
    if (keep && !(sf & 4) && bv.dmax2[lo] <= bv.half_skin2) continue;
    auto cand_cut = [&](int tj) {
      return fmaxf((rr1 + p.rc_r[tj]) * 0.5f, (ra1 + p.rc_a[tj]) * 0.5f) + bv.skin;
    };
    float4* rrow = er + static_cast<size_t>(i) * mn_r;
    float4* arow = ea + static_cast<size_t>(i) * mn_a;
    int cr = 0, ca = 0;
    if (!s.small) {
      const double xi = pos[i], yi = pos[total + i], zi = pos[2 * total + i];
      const Box b = s.box;   // the structure's box, held in registers for this center
      int* buf = s_rows + (threadIdx.x >> 5) * (p2r + 1);
      int* count = buf + p2r;
      if (lane == 0) *count = 0;
      __syncwarp();
      auto consider = [&](int j) {
        // the site record: position and type in one 32-byte sector
        float x12, y12, z12;
        int tj;
        site_displacement(b, sites, xi, yi, zi, j, x12, y12, z12, tj);
        const float d12_square = x12 * x12 + y12 * y12 + z12 * z12;
        const float rcut = keep ? cand_cut(tj) : (rr1 + p.rc_r[tj]) * 0.5f;
        if (d12_square < rcut * rcut) {
          const int slot = atomicAdd(count, 1);
          if (slot < p2r) buf[slot] = j;
        }
      };
      if (s.nc[0] > 0) {
        // the 5x5x5 cells (at least rc/2 wide) around the center's, every cell
        // once where the grid is narrower.  In rounds of 32 stencil cells:
        // lane q takes a cell, a warp prefix sum of the cell counts flattens
        // their atoms into one range, and the warp sweeps that range 32
        // candidates at a time (one cell per pass would leave most lanes idle)
        const int nc0 = s.nc[0], nc1 = s.nc[1], nc2 = s.nc[2];
        const int lc = cell_of[i] - s.cell_base;
        const int cx = lc % nc0, cy = (lc / nc0) % nc1, cz = lc / (nc0 * nc1);
        const int sp0 = (b.pbc[0] && nc0 >= 5) ? 5 : nc0;
        const int sp1 = (b.pbc[1] && nc1 >= 5) ? 5 : nc1;
        const int sp2 = (b.pbc[2] && nc2 >= 5) ? 5 : nc2;
        const int ns = sp0 * sp1 * sp2;   // at most 125
        const bool full = sp0 == 5 && sp1 == 5 && sp2 == 5;   // usual: constant divisors
        for (int r0 = 0; r0 < ns; r0 += 32) {
          int my_start = 0, my_cnt = 0;
          if (r0 + lane < ns) {
            const int q = r0 + lane;
            int q0, q1, q2;
            if (full) {
              q0 = q % 5;
              q1 = (q / 5) % 5;
              q2 = q / 25;
            } else {
              q0 = q % sp0;
              q1 = (q / sp0) % sp1;
              q2 = q / (sp0 * sp1);
            }
            int gx = sp0 == 5 ? cx + q0 - 2 : q0;
            int gy = sp1 == 5 ? cy + q1 - 2 : q1;
            int gz = sp2 == 5 ? cz + q2 - 2 : q2;
            if (gx < 0) gx += nc0; else if (gx >= nc0) gx -= nc0;
            if (gy < 0) gy += nc1; else if (gy >= nc1) gy -= nc1;
            if (gz < 0) gz += nc2; else if (gz >= nc2) gz -= nc2;
            const int c = s.cell_base + (gz * nc1 + gy) * nc0 + gx;
            my_start = cell_start[c];
            my_cnt = cell_count[c];
          }
          int incl = my_cnt;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
          }
          const int total_c = __shfl_sync(kFull, incl, 31);
          for (int base = 0; base < total_c; base += 32) {
            const int k = base + lane;
            // stencil cell of candidate k: the first lane whose inclusive count exceeds k
            int lo = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
              const int probe = lo + step - 1;
              const int v = __shfl_sync(kFull, incl, probe);
              if (v <= k) lo += step;
            }
            const int cstart = __shfl_sync(kFull, my_start, lo);
            const int cincl = __shfl_sync(kFull, incl, lo);
            const int ccnt = __shfl_sync(kFull, my_cnt, lo);
            if (k < total_c) {
              const int j = cell_atoms[cstart + (k - (cincl - ccnt))];
              if (j != i) consider(j);
            }
          }
        }
      } else {
        for (int base = 0; base < n; base += 32) {
          const int j = off + base + lane;
          if (base + lane < n && j != i) consider(j);
        }
      }
      __syncwarp();
      const int found = *count;
      const int used = min(found, p2r);
      int p2 = 1;
      while (p2 < used) p2 <<= 1;
      if (p2 <= 64) {
        // bitonic sort in registers: element e = lane in a, e = lane + 32 in
        // c; partners e ^ jj exchange by shuffle (jj < 32) or inside the lane
        // (jj = 32); e keeps the smaller value when (e < partner) matches the
        // ascending direction (e & k) == 0 of its block
        int a = lane < used ? buf[lane] : INT_MAX;
        int c = lane + 32 < used ? buf[lane + 32] : INT_MAX;
        const bool two = p2 > 32;   // warp-uniform
        for (int k = 2; k <= p2; k <<= 1) {
          for (int jj = k >> 1; jj > 0; jj >>= 1) {
            if (jj == 32) {
              const int lo_v = min(a, c);
              c = max(a, c);
              a = lo_v;
            } else {
              const bool lower = (lane & jj) == 0;
              const int pa = __shfl_xor_sync(kFull, a, jj);
              a = (lower == ((lane & k) == 0)) ? min(a, pa) : max(a, pa);
              if (two) {
                const int pc = __shfl_xor_sync(kFull, c, jj);
                c = (lower == (((lane + 32) & k) == 0)) ? min(c, pc) : max(c, pc);
              }
            }
          }
        }
        __syncwarp();   // every lane has read buf before it is overwritten
        if (lane < used) buf[lane] = a;
        if (lane + 32 < used) buf[lane + 32] = c;
        __syncwarp();
      } else {
        for (int k = used + lane; k < p2; k += 32) buf[k] = INT_MAX;
        __syncwarp();
        for (int k = 2; k <= p2; k <<= 1) {   // bitonic sort, one pair per lane and pass
          for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int q = lane; q < (p2 >> 1); q += 32) {
              const int t = ((q & ~(jj - 1)) << 1) | (q & (jj - 1));
              const int u = t | jj;
              const int a = buf[t], c = buf[u];
              if ((a > c) == ((t & k) == 0)) {
                buf[t] = c;
                buf[u] = a;
              }
            }
            __syncwarp();
          }
        }
      }
      if (keep) {
        // ascending candidates, structure-local
        int* vr = bv.vrow + static_cast<size_t>(i) * bv.mn;
        for (int k = lane; k < used && k < bv.mn; k += 32) vr[k] = buf[k] - off;
        if (lane == 0) {
          bv.vcnt[i] = min(found, bv.mn);
          if (found > bv.mn || found > p2r) atomicOr(&st->overflow, 1);
          bv.x0[i] = xi;
          bv.x0[total + i] = yi;
          bv.x0[2 * total + i] = zi;
          atomicAdd(&st->xr_builds, 1u);
        }
        __syncwarp();   // the buffer is reused by this warp's next center
        continue;
      }
      // ascending radial row; the angular row is its subset inside the angular cutoff
      for (int k0 = 0; k0 < used; k0 += 32) {
        const int k = k0 + lane;
        bool in_a = false;
        float4 entry = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (k < used) {
          const int j = buf[k];
          float x12, y12, z12;
          int t2;
          site_displacement(b, sites, xi, yi, zi, j, x12, y12, z12, t2);
          const float d12_square = x12 * x12 + y12 * y12 + z12 * z12;
          const float rc_angular = (ra1 + p.rc_a[t2]) * 0.5f;
          in_a = d12_square < rc_angular * rc_angular;
          entry = row_entry(x12, y12, z12, j, t2);
          if (k < mn_r) rrow[k] = entry;
        }
        const unsigned ma = __ballot_sync(kFull, in_a);
        if (in_a) {
          const int at = ca + __popc(ma & below);
          if (at < mn_a) arow[at] = entry;
        }
        ca += __popc(ma);
      }
      cr = found;
      __syncwarp();   // the buffer is reused by this warp's next center
    } else if (keep) {
      // candidates (j, image) within the cutoff plus the skin, in row order:
      // j ascending, then the images; count per lane, scan, then write
      const float x1 = pos[i], y1 = pos[total + i], z1 = pos[2 * total + i];
      int* vr = bv.vrow + static_cast<size_t>(i) * bv.mn;
      int cv = 0;
      for (int base = 0; base < n; base += 32) {
        const int j = off + base + lane;
        const bool valid = base + lane < n;
        const float rcut = cand_cut(valid ? type[j] : 0);
        const double xj = valid ? pos[j] : 0.0, yj = valid ? pos[total + j] : 0.0,
                     zj = valid ? pos[2 * total + j] : 0.0;
        const unsigned jl = static_cast<unsigned>(j - off);
        int wv = 0;
        for (int pass = 0; pass < 2; ++pass) {
          int kv = 0;
          if (valid) {
            for (int ia = 0; ia < s.ncell[0]; ++ia)
              for (int ib = 0; ib < s.ncell[1]; ++ib)
                for (int ic = 0; ic < s.ncell[2]; ++ic) {
                  if (ia == 0 && ib == 0 && ic == 0 && j == i) continue;   // self
                  float x12, y12, z12;
                  small_box_delta(s, x1, y1, z1, xj, yj, zj, ia, ib, ic, x12, y12, z12);
                  if (x12 * x12 + y12 * y12 + z12 * z12 < rcut * rcut) {
                    if (pass == 1 && wv + kv < bv.mn)
                      vr[wv + kv] = static_cast<int>(
                        jl | (static_cast<unsigned>(ia) << kCandIndexBits) |
                        (static_cast<unsigned>(ib) << (kCandIndexBits + 4)) |
                        (static_cast<unsigned>(ic) << (kCandIndexBits + 8)));
                    ++kv;
                  }
                }
          }
          if (pass == 0) {
            int sv = kv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const int u = __shfl_up_sync(kFull, sv, o);
              if (lane >= o) sv += u;
            }
            wv = cv + sv - kv;
            cv += __shfl_sync(kFull, sv, 31);
          }
        }
      }
      if (lane == 0) {
        bv.vcnt[i] = min(cv, bv.mn);
        if (cv > bv.mn) atomicOr(&st->overflow, 1);
        bv.x0[i] = pos[i];
        bv.x0[total + i] = pos[total + i];
        bv.x0[2 * total + i] = pos[2 * total + i];
        atomicAdd(&st->xr_builds, 1u);
      }
      continue;
    } else {
      // the small-box arithmetic: float center, double image position
      const float x1 = pos[i], y1 = pos[total + i], z1 = pos[2 * total + i];
      for (int base = 0; base < n; base += 32) {
        const int j = off + base + lane;
        const bool valid = base + lane < n;
        const int t2 = valid ? type[j] : 0;
        const float rc_radial = (rr1 + p.rc_r[t2]) * 0.5f;
        const float rc_angular = (ra1 + p.rc_a[t2]) * 0.5f;
        const double xj = valid ? pos[j] : 0.0, yj = valid ? pos[total + j] : 0.0,
                     zj = valid ? pos[2 * total + j] : 0.0;
        // pass 0 counts this lane's edges, pass 1 writes them at the scanned offsets
        int wr = 0, wa = 0;
        for (int pass = 0; pass < 2; ++pass) {
          int kr = 0, ka = 0;
          if (valid) {
            for (int ia = 0; ia < s.ncell[0]; ++ia)
              for (int ib = 0; ib < s.ncell[1]; ++ib)
                for (int ic = 0; ic < s.ncell[2]; ++ic) {
                  if (ia == 0 && ib == 0 && ic == 0 && j == i) continue;   // self
                  float x12, y12, z12;
                  small_box_delta(s, x1, y1, z1, xj, yj, zj, ia, ib, ic, x12, y12, z12);
                  const float d12_square = x12 * x12 + y12 * y12 + z12 * z12;
                  if (d12_square < rc_radial * rc_radial) {
                    if (pass == 1 && wr + kr < mn_r)
                      rrow[wr + kr] = row_entry(x12, y12, z12, j, t2);
                    ++kr;
                  }
                  if (d12_square < rc_angular * rc_angular) {
                    if (pass == 1 && wa + ka < mn_a)
                      arow[wa + ka] = row_entry(x12, y12, z12, j, t2);
                    ++ka;
                  }
                }
          }
          if (pass == 0) {
            // exclusive warp scan of the per-lane counts
            int sr = kr, sa = ka;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const int ur = __shfl_up_sync(kFull, sr, o), ua = __shfl_up_sync(kFull, sa, o);
              if (lane >= o) {
                sr += ur;
                sa += ua;
              }
            }
            wr = cr + sr - kr;
            wa = ca + sa - ka;
            cr += __shfl_sync(kFull, sr, 31);
            ca += __shfl_sync(kFull, sa, 31);
          }
        }
      }
    }
    if (lane == 0) {
      nn_r[i] = min(cr, mn_r);
      nn_a[i] = min(ca, mn_a);
      large[i] = mark_large && !s.small ? 1 : 0;
      if (cr > mn_r) atomicOr(&st->overflow, 2);
      if (ca > mn_a) atomicOr(&st->overflow, 4);
      atomicMax(&st->max_nn[1], cr);
      atomicMax(&st->max_nn[2], ca);
      atomicMax(&st->call_nn[0], cr);
      atomicMax(&st->call_nn[1], ca);
    }
  }
}

// Rows of the centers whose structure keeps Verlet candidates: one warp per
// center filters its candidates (in row order) with the predicates and the
// arithmetic of k_rows_explicit, so the rows equal a fresh build's bit for
// bit while no atom of the structure has moved more than skin / 2 since the
// candidates were built.  Radial and angular rows are written in order by
// warp ballot + popcount.
__global__ void __launch_bounds__(256)
k_rows_verlet(const ModelParams p, int total, const StructInfo* __restrict__ si,
              const int* __restrict__ soff, int S, const double* __restrict__ pos,
              const int* __restrict__ type, int* __restrict__ nn_r, float4* __restrict__ er,
              int mn_r, int* __restrict__ nn_a, float4* __restrict__ ea, int mn_a,
              const Site* __restrict__ sites, unsigned char* __restrict__ large,
              const BatchVerlet bv, NeighborState* st)
{
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < total; i += gridDim.x * wpb) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (soff[mid] <= i) lo = mid; else hi = mid - 1;
    }
    if (!(bv.sflag[lo] & 2)) continue;
    const StructInfo& s = si[lo];
    const int off = s.off;
    const int t1 = type[i];
    const float rr1 = p.rc_r[t1], ra1 = p.rc_a[t1];
    float4* rrow = er + static_cast<size_t>(i) * mn_r;
    float4* arow = ea + static_cast<size_t>(i) * mn_a;
    const int* vr = bv.vrow + static_cast<size_t>(i) * bv.mn;
    const int nv = bv.vcnt[i];
    int cr = 0, ca = 0;
    const double xi = pos[i], yi = pos[total + i], zi = pos[2 * total + i];
    const float x1 = static_cast<float>(xi), y1 = static_cast<float>(yi),
                z1 = static_cast<float>(zi);
    for (int k0 = 0; k0 < nv; k0 += 32) {
      const int k = k0 + lane;
      bool in_r = false, in_a = false;
      float4 entry = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (k < nv) {
        const unsigned code = static_cast<unsigned>(vr[k]);
        int j, t2;
        float x12, y12, z12;
        if (!s.small) {
          j = off + static_cast<int>(code);
          site_displacement(s.box, sites, xi, yi, zi, j, x12, y12, z12, t2);
        } else {
          j = off + static_cast<int>(code & ((1u << kCandIndexBits) - 1u));
          const int ia = static_cast<int>((code >> kCandIndexBits) & 15u);
          const int ib = static_cast<int>((code >> (kCandIndexBits + 4)) & 15u);
          const int ic = static_cast<int>(code >> (kCandIndexBits + 8));
          t2 = type[j];
          small_box_delta(s, x1, y1, z1, pos[j], pos[total + j], pos[2 * total + j], ia, ib,
                          ic, x12, y12, z12);
        }
        const float d12_square = x12 * x12 + y12 * y12 + z12 * z12;
        const float rc_radial = (rr1 + p.rc_r[t2]) * 0.5f;
        const float rc_angular = (ra1 + p.rc_a[t2]) * 0.5f;
        in_r = d12_square < rc_radial * rc_radial;
        // large structures: the angular row is the radial row's subset (as
        // k_rows_explicit builds it); small boxes test both cutoffs apart
        in_a = (s.small || in_r) && d12_square < rc_angular * rc_angular;
        entry = row_entry(x12, y12, z12, j, t2);
      }
      const unsigned mr = __ballot_sync(kFull, in_r);
      const unsigned ma = __ballot_sync(kFull, in_a);
      if (in_r) {
        const int at = cr + __popc(mr & below);
        if (at < mn_r) rrow[at] = entry;
      }
      if (in_a) {
        const int at = ca + __popc(ma & below);
        if (at < mn_a) arow[at] = entry;
      }
      cr += __popc(mr);
      ca += __popc(ma);
    }
    if (lane == 0) {
      nn_r[i] = min(cr, mn_r);
      nn_a[i] = min(ca, mn_a);
      large[i] = s.small ? 0 : 1;
      if (cr > mn_r) atomicOr(&st->overflow, 2);
      if (ca > mn_a) atomicOr(&st->overflow, 4);
      atomicMax(&st->max_nn[1], cr);
      atomicMax(&st->max_nn[2], ca);
      atomicMax(&st->call_nn[0], cr);
      atomicMax(&st->call_nn[1], ca);
    }
  }
}

// Cell of every atom of a large structure (fractional coordinates, wrapped
// where periodic, one cell where not), counted per cell.
__global__ void k_xcell_assign(int total, const StructInfo* __restrict__ si,
                               const int* __restrict__ soff, int S, const double* __restrict__ pos,
                               int* cell_count, int* cell_of)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int lo = 0, hi = S - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (soff[mid] <= i) lo = mid; else hi = mid - 1;
  }
  const StructInfo& s = si[lo];
  if (s.small || s.nc[0] == 0) {
    cell_of[i] = -1;
    return;
  }
  const double r[3] = {pos[i], pos[total + i], pos[2 * total + i]};
  int c[3];
  for (int d = 0; d < 3; ++d) {
    double f = s.box.hinv[3 * d] * r[0] + s.box.hinv[3 * d + 1] * r[1] + s.box.hinv[3 * d + 2] * r[2];
    f -= floor(f);
    int k = static_cast<int>(f * s.nc[d]);
    c[d] = k < 0 ? 0 : (k >= s.nc[d] ? s.nc[d] - 1 : k);
  }
  const int cell = s.cell_base + (c[2] * s.nc[1] + c[1]) * s.nc[0] + c[0];
  cell_of[i] = cell;
  atomicAdd(cell_count + cell, 1);
}

// Exclusive scan of the cell counts, one block per structure: a structure's
// cells are contiguous and its atoms fill [off, off + n) of cell_atoms, so
// its cells start at off plus the scan of its own counts (coalesced chunks
// of blockDim.x cells with a running carry).  Counts reset as fill cursors.
__global__ void k_xcell_scan(const StructInfo* __restrict__ si, int* cell_count, int* cell_start)
{
  __shared__ int warp_sum[32];
  __shared__ int carry_s;
  const StructInfo& s = si[blockIdx.x];
  if (s.nc[0] == 0) return;   // block-uniform: the structure scans all its atoms
  const int ncs = s.nc[0] * s.nc[1] * s.nc[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int carry = s.off;
  for (int c0 = 0; c0 < ncs; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;
    const int v = c < ncs ? cell_count[s.cell_base + c] : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int w = lane < nw ? warp_sum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += u;
      }
      if (lane < nw) warp_sum[lane] = w;   // inclusive over warps
      if (lane == 31) carry_s = w;         // chunk total
    }
    __syncthreads();
    const int before = (warp > 0 ? warp_sum[warp - 1] : 0) + incl - v;
    if (c < ncs) {
      cell_start[s.cell_base + c] = carry + before;
      cell_count[s.cell_base + c] = 0;
    }
    carry += carry_s;
    __syncthreads();   // warp_sum and carry_s are rewritten by the next chunk
  }
}

__global__ void k_xcell_fill(int total, const int* __restrict__ cell_of, int* cell_count,
                             const int* __restrict__ cell_start, int* cell_atoms)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = cell_of[i];
  if (c < 0) return;
  cell_atoms[cell_start[c] + atomicAdd(cell_count + c, 1)] = i;
}

__global__ void k_row_indices(int n, const int* __restrict__ cnt, const float4* __restrict__ rows,
                              int src_mn, int* nn, int* nl, int mn)
{
  const int i = blockIdx.x;
  if (i >= n) return;
  const int c = cnt[i];
  if (threadIdx.x == 0) nn[i] = c;
  for (int k = threadIdx.x; k < c; k += blockDim.x)
    nl[static_cast<size_t>(i) * mn + k] =
      __float_as_int(rows[static_cast<size_t>(i) * src_mn + k].w) & kRowIndexMask;
}

template <typename T>
cudaError_t dalloc(T*& ptr, size_t count)
{
  return cudaMalloc(reinterpret_cast<void**>(&ptr), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

int structure_cells(const Engine& e, const StructInfo& s, int* nc_out)
{
  if (s.small) return 0;
  // cells at least half the candidate radius: the cutoff, plus the skin for
  // a structure that keeps Verlet candidates
  const double rc = s.keep ? e.model.rc_max + e.skin : e.model.rc_radial_max;
  int nc[3], cells = 1;
  for (int d = 0; d < 3; ++d) {
    const double* r = s.box.hinv + 3 * d;
    const double thick = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    nc[d] = s.box.pbc[d] ? std::max(1, static_cast<int>(thick / (0.5 * rc))) : 1;
    cells *= nc[d];
  }
  // a 5x5x5 stencil of cells at least rc/2 wide covers the cutoff; grids of
  // fewer than 125 cells scan all the structure's atoms instead
  if (cells < 125) return 0;
  if (nc_out)
    for (int d = 0; d < 3; ++d) nc_out[d] = nc[d];
  return cells;
}

int assign_cells(const Engine& e, StructInfo* si, int n)
{
  int used = 0;
  for (int k = 0; k < n; ++k) {
    StructInfo& s = si[k];
    s.nc[0] = s.nc[1] = s.nc[2] = 0;
    s.cell_base = 0;
    int nc[3];
    const int cells = structure_cells(e, s, nc);
    if (cells == 0 || used + cells > e.xr.cell_cap) continue;
    for (int d = 0; d < 3; ++d) s.nc[d] = nc[d];
    s.cell_base = used;
    used += cells;
  }
  return used;
}

int box_kind(const Engine& e, const Box& b)
{
  StructInfo s;
  if (expanded_box(b, e.model.rc_radial_max, s)) return -1;
  return s.small;
}

std::string engine_enable_xr(Engine& e, int max_struct)
{
  ExplicitRows& x = e.xr;
  if (x.er && x.max_struct >= max_struct) return "";
  const size_t N = e.capacity;
  if (N > static_cast<size_t>(kRowIndexMask))
    return "explicit neighbour rows address at most 2^28 atoms";
  if (!x.er) {
    x.cell_cap = static_cast<int>(std::max<size_t>(N, 4096));
    bool ok = dalloc(x.er, N * e.nbr.mn_r) == cudaSuccess;
    ok &= dalloc(x.ea, N * e.nbr.mn_a) == cudaSuccess;
    ok &= dalloc(x.cell_count, x.cell_cap) == cudaSuccess;
    ok &= dalloc(x.cell_start, x.cell_cap) == cudaSuccess;
    ok &= dalloc(x.cell_atoms, N) == cudaSuccess;
    ok &= dalloc(x.cell_of, N) == cudaSuccess;
    ok &= dalloc(x.large, N) == cudaSuccess;
    if (!ok) return "cudaMalloc failed (explicit neighbour rows)";
  }
  if (x.max_struct < max_struct) {
    if (x.d_si) cudaFree(x.d_si);
    if (x.d_soff) cudaFree(x.d_soff);
    x.d_si = nullptr;
    x.d_soff = nullptr;
    bool ok = dalloc(x.d_si, max_struct) == cudaSuccess;
    ok &= dalloc(x.d_soff, max_struct + 1) == cudaSuccess;
    if (!ok) return "cudaMalloc failed (structure table)";
    x.max_struct = max_struct;
  }
  return "";
}

void launch_explicit_rows(Engine& e, int N, const double* pos, const int* type,
                          cudaStream_t stream)
{
  ExplicitRows& x = e.xr;
  const int threads = 256;
  k_pack_sites<<<(N + threads - 1) / threads, threads, 0, stream>>>(N, pos, type,
                                                                     e.scratch.sites, e.d_nstate);
  if (x.from_box) {
    k_struct_from_box<<<1, 1, 0, stream>>>(e.d_box, e.model.rc_radial_max, N, x.d_si, x.d_soff,
                                           e.d_nstate);
    x.n_struct = 1;
  }
  if (!x.from_box && x.n_cells > 0) {
    cudaMemsetAsync(x.cell_count, 0, sizeof(int) * x.n_cells, stream);
    k_xcell_assign<<<(N + threads - 1) / threads, threads, 0, stream>>>(
      N, x.d_si, x.d_soff, x.n_struct, pos, x.cell_count, x.cell_of);
    k_xcell_scan<<<x.n_struct, 1024, 0, stream>>>(x.d_si, x.cell_count, x.cell_start);
    k_xcell_fill<<<(N + threads - 1) / threads, threads, 0, stream>>>(
      N, x.cell_of, x.cell_count, x.cell_start, x.cell_atoms);
  }
  const bool verlet = !x.from_box && x.bv.sflag != nullptr;
  int p2r = 1;
  while (p2r < std::max(e.nbr.mn_r, verlet ? x.bv.mn : 0)) p2r <<= 1;
  const int warps = threads / 32;
  const int blocks = std::min((N + warps - 1) / warps, 148 * 8);
  const size_t smem = sizeof(int) * warps * (p2r + 1);
  BatchVerlet bv = x.bv;
  if (!verlet) bv.sflag = nullptr;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_rows_explicit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
  k_rows_explicit<<<blocks, threads, smem, stream>>>(
    e.params, N, x.d_si, x.d_soff, x.n_struct, pos, type, e.nbr.nn_r, x.er, e.nbr.mn_r,
    e.nbr.nn_a, x.ea, e.nbr.mn_a, x.cell_count, x.cell_start, x.cell_atoms, x.cell_of, p2r,
    e.scratch.sites, x.large, x.from_box ? 0 : 1, bv, e.d_nstate);
  if (verlet)
    k_rows_verlet<<<blocks, threads, 0, stream>>>(
      e.params, N, x.d_si, x.d_soff, x.n_struct, pos, type, e.nbr.nn_r, x.er, e.nbr.mn_r,
      e.nbr.nn_a, x.ea, e.nbr.mn_a, e.scratch.sites, x.large, bv, e.d_nstate);
}

bool verlet_encodable(const StructInfo& s, double skin)
{
  for (int d = 0; d < 3; ++d) {
    const double* r = s.box.hinv + 3 * d;
    const double thick = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (s.box.pbc[d] && thick < 4.0 * skin) return false;
  }
  if (!s.small) return true;
  return s.n <= (1 << kCandIndexBits) && s.ncell[0] <= kCandMaxImages &&
         s.ncell[1] <= kCandMaxImages && s.ncell[2] <= kCandMaxImages;
}

void launch_explicit_row_indices(const Engine& e, int which, int n, int* nn, int* nl, int mn,
                                 cudaStream_t stream)
{
  const int src_mn = which == 0 ? e.nbr.mn_r : e.nbr.mn_a;
  k_row_indices<<<n, 64, 0, stream>>>(n, which == 0 ? e.nbr.nn_r : e.nbr.nn_a,
                                      which == 0 ? e.xr.er : e.xr.ea, src_mn, nn, nl, mn);
}

}  // namespace nepx

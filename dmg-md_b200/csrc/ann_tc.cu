// ann_tc.cu -- the per-atom ANN of the mixed-precision path on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM).
//
// The NEP ANN (reference apply_ann_one_layer, nep_utilities.cuh, one hidden
// tanh layer per center type) is two dense contractions per center:
//     z = W0_t q - b0_t,  x = tanh z,  E = w1_t . x - bias_t,
//     dE/dq = W0_t^T (w1_t (1 - x^2)) * q_scaler.
// Here centers are sorted by type (k_type_*), and one CTA takes a tile of
// 128 consecutive sorted centers: the tile's descriptors are the M = 128
// rows of GEMM1 (K = dim, N = hidden units), whose epilogue (tanh, energy,
// w1 (1 - x^2)) writes the A operand of GEMM2 (K = hidden units, N = dim)
// back to shared memory.  The hidden layer streams through in chunks of 64
// (or 32, 16) units -- GEMM1 chunk, epilogue, GEMM2 accumulating over the
// chunks in TMEM -- so the tiles of any model up to dim ~ 128 fit one SM.
// Both contractions run as 3xTF32 (a = a_hi + a_lo with a_hi the TF32 part:
// a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulation in TMEM), which keeps
// FP32-level accuracy (relative error ~1e-6) at tensor-core rate.  A tile
// that holds centers of several types runs the contractions once per type
// and keeps each row's result for its own type.
//
// Operands sit in shared memory in the K-major, no-swizzle canonical layout
// of tcgen05: 8-row x 16-byte core matrices, the two K-adjacent core
// matrices of one MMA (K = 8 TF32) 128 bytes apart (leading byte offset),
// consecutive 8-row groups K/4 * 128 bytes apart (stride byte offset).  One
// thread issues the MMAs and commits them to an mbarrier; every wait on it
// is bounded (a timeout sets the error flag, the kernel frees its TMEM and
// returns).
#include <cstdint>

#include "engine.h"

namespace nepx {

namespace {

constexpr int kRows = 128;                        // centers per tile = MMA M = TMEM lanes
constexpr long long kWaitCycles = 4000000000ll;   // ~2 s at the B200 clock

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in a K-major no-swizzle tile with K columns
__host__ __device__ __forceinline__ uint32_t core_off(int r, int k, int K)
{
  return static_cast<uint32_t>(((r >> 3) * (K >> 2) + (k >> 2)) * 128 + (r & 7) * 16 +
                               (k & 3) * 4);
}

// Shared-memory matrix descriptor: start address, leading byte offset 128
// (K-adjacent core matrices), stride byte offset K/4 * 128 (8-row groups),
// descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int K)
{
  const uint64_t lbo = 128u >> 4;
  const uint64_t sbo = static_cast<uint64_t>((K >> 2) * 128) >> 4;
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N and M as given.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
    "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                 mbar)
               : "memory");
}

__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Bounded wait for the phase of the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

// 16 consecutive TMEM columns of this thread's lane; the wait is part of the
// same statement so no register is read before the load lands.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
    "%12, %13, %14, %15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;\n"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(taddr)
    : "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// a = hi + lo with hi the TF32 value (round to nearest) and lo the exact rest
__device__ __forceinline__ void split_tf32(float a, float& hi, float& lo)
{
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(a));
  hi = __uint_as_float(h);
  lo = a - hi;
}

struct AnnTcLayout {
  int dimK, dimN;       // K of GEMM1 (dim to 8), N of GEMM2 (dim to 16)
  int HC, Hn;           // hidden units per chunk (N of GEMM1, K of GEMM2), H rounded to HC
  int q, w, g, v;       // byte offsets of the hi tiles (the lo tile follows each)
  int qsz, wsz, gsz, vsz;
  int bar, slot, total;
  int cols;             // TMEM columns allocated
};

__host__ __device__ inline AnnTcLayout ann_tc_layout(const ModelParams& p, int HC)
{
  AnnTcLayout L;
  L.dimK = (p.dim + 7) & ~7;
  L.dimN = (p.dim + 15) & ~15;
  L.HC = HC;
  L.Hn = (p.H + HC - 1) / HC * HC;
  L.qsz = kRows * L.dimK * 4;
  L.wsz = HC * L.dimK * 4;
  L.gsz = kRows * HC * 4;
  L.vsz = L.dimN * HC * 4;
  L.q = 0;
  L.w = L.q + 2 * L.qsz;
  L.g = L.w + 2 * L.wsz;
  L.v = L.g + 2 * L.gsz;
  L.bar = L.v + 2 * L.vsz;
  L.slot = L.bar + 8;
  L.total = L.slot + 8;
  int need = HC + L.dimN, cols = 32;
  while (cols < need) cols *= 2;
  L.cols = cols;
  return L;
}

constexpr int kSmemLimit = 227 * 1024;

// Hidden-unit chunk: the largest (64, 32, 16) whose tiles let two CTAs share
// an SM, else the largest that fits one.
__host__ __device__ inline int ann_tc_chunk(const ModelParams& p)
{
  for (int hc = 64; hc >= 16; hc /= 2)
    if (ann_tc_layout(p, hc).total <= kSmemLimit / 2 - 1024) return hc;
  for (int hc = 64; hc >= 16; hc /= 2)
    if (ann_tc_layout(p, hc).total <= kSmemLimit) return hc;
  return 0;
}

__global__ void __launch_bounds__(kRows, 2)
k_ann_tc(const ModelParams p, int N, int HC, const int* __restrict__ order,
         const Site* __restrict__ sites, const float* __restrict__ qbuf,
         double* __restrict__ pe_ann, float* __restrict__ fpbuf, int* err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  const AnnTcLayout L = ann_tc_layout(p, HC);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int dim = p.dim, H = p.H, dimK = L.dimK, dimN = L.dimN;
  unsigned char* Qh = smem + L.q;
  unsigned char* Ql = smem + L.q + L.qsz;
  unsigned char* Wh = smem + L.w;
  unsigned char* Wl = smem + L.w + L.wsz;
  unsigned char* Gh = smem + L.g;
  unsigned char* Gl = smem + L.g + L.gsz;
  unsigned char* Vh = smem + L.v;
  unsigned char* Vl = smem + L.v + L.vsz;
  const uint32_t bar = smem_u32(smem + L.bar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + L.slot);
  auto put = [](unsigned char* base, uint32_t off, float x) {
    *reinterpret_cast<float*>(base + off) = x;
  };

  const int first = blockIdx.x * kRows;
  const int idx = first + tid;
  const int c = idx < N ? order[idx] : -1;
  const int tc = c >= 0 ? static_cast<int>(sites[c].type) : -1;
  // type range of the tile (a reduction, so any row order is handled)
  __shared__ int s_trange[2];
  if (tid == 0) {
    s_trange[0] = kMaxTypes;
    s_trange[1] = -1;
  }
  __syncthreads();
  if (tc >= 0) {
    atomicMin(&s_trange[0], tc);
    atomicMax(&s_trange[1], tc);
  }
  __syncthreads();
  const int t_lo = s_trange[0], t_hi = s_trange[1];

  // this row of the descriptor tile (zero rows past N)
  const float4* qrow = reinterpret_cast<const float4*>(qbuf + static_cast<size_t>(c < 0 ? 0 : c) *
                                                                p.dimK);
  for (int k4 = 0; k4 < dimK / 4; ++k4) {
    const float4 x4 = c >= 0 ? __ldg(qrow + k4) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float xs[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float hi, lo;
      split_tf32(xs[u], hi, lo);
      put(Qh, core_off(tid, 4 * k4 + u, dimK), hi);
      put(Ql, core_off(tid, 4 * k4 + u, dimK), lo);
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
                 "r"(L.cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *slot;
  const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  const uint32_t z_col = 0, f_col = static_cast<uint32_t>(HC);
  const uint32_t id1 = idesc_tf32(kRows, HC), id2 = idesc_tf32(kRows, dimN);
  uint32_t phase = 0;
  bool failed = false;

  for (int t = t_lo; t <= t_hi && !failed; ++t) {
    const float* wt = p.w0t + static_cast<size_t>(t) * dim * p.H4;   // [dim][H4]
    float e_row = 0.0f;
    for (int h0 = 0; h0 < L.Hn && !failed; h0 += HC) {
      // chunk of the weights: B1 = W0_t rows h0..h0+HC (K = dimK), B2 = W0_t^T (N = dimN, K = HC)
      for (int e = tid; e < HC * dimK; e += kRows) {
        const int hh = e / dimK, d = e % dimK, h = h0 + hh;
        const float x = (h < H && d < dim) ? __ldg(wt + static_cast<size_t>(d) * p.H4 + h) : 0.0f;
        float hi, lo;
        split_tf32(x, hi, lo);
        put(Wh, core_off(hh, d, dimK), hi);
        put(Wl, core_off(hh, d, dimK), lo);
      }
      for (int e = tid; e < dimN * HC; e += kRows) {
        const int d = e / HC, hh = e % HC, h = h0 + hh;
        const float x = (d < dim && h < H) ? __ldg(wt + static_cast<size_t>(d) * p.H4 + h) : 0.0f;
        float hi, lo;
        split_tf32(x, hi, lo);
        put(Vh, core_off(d, hh, HC), hi);
        put(Vl, core_off(d, hh, HC), lo);
      }
      fence_async_smem();
      tc_before_sync();
      __syncthreads();
      tc_after_sync();
      // GEMM1: Z[128][HC] = Q W0_chunk^T
      if (tid == 0) {
        for (int s = 0; s < dimK / 8; ++s) {
          const uint32_t ko = static_cast<uint32_t>(s * 256);
          const uint64_t qh = smem_desc(smem_u32(Qh) + ko, dimK);
          const uint64_t ql = smem_desc(smem_u32(Ql) + ko, dimK);
          const uint64_t wh = smem_desc(smem_u32(Wh) + ko, dimK);
          const uint64_t wl = smem_desc(smem_u32(Wl) + ko, dimK);
          mma_tf32(tmem + z_col, qh, wh, id1, s > 0 ? 1u : 0u);
          mma_tf32(tmem + z_col, qh, wl, id1, 1u);
          mma_tf32(tmem + z_col, ql, wh, id1, 1u);
        }
        mma_commit(bar);
      }
      bool ok = mbar_wait(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      tc_after_sync();
      // epilogue 1: x = tanh(z - b0), E += w1 . x, G = w1 (1 - x^2) as the A operand of GEMM2
      for (int c0 = 0; c0 < HC; c0 += 16) {
        float z[16];
        tmem_ld16(lane_base + z_col + c0, z);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int h = h0 + c0 + k;
          float g = 0.0f;
          if (h < H) {
            const float x1 = tanhf(z[k] - __ldg(p.b0 + t * H + h));
            const float w1 = __ldg(p.w1 + t * H + h);
            e_row += w1 * x1;
            g = w1 * (1.0f - x1 * x1);
          }
          float hi, lo;
          split_tf32(g, hi, lo);
          put(Gh, core_off(tid, c0 + k, HC), hi);
          put(Gl, core_off(tid, c0 + k, HC), lo);
        }
      }
      fence_async_smem();
      tc_before_sync();
      __syncthreads();
      tc_after_sync();
      // GEMM2: F[128][dimN] += G_chunk W0_chunk
      if (tid == 0) {
        for (int s = 0; s < HC / 8; ++s) {
          const uint32_t ko = static_cast<uint32_t>(s * 256);
          const uint64_t gh = smem_desc(smem_u32(Gh) + ko, HC);
          const uint64_t gl = smem_desc(smem_u32(Gl) + ko, HC);
          const uint64_t vh = smem_desc(smem_u32(Vh) + ko, HC);
          const uint64_t vl = smem_desc(smem_u32(Vl) + ko, HC);
          mma_tf32(tmem + f_col, gh, vh, id2, (h0 > 0 || s > 0) ? 1u : 0u);
          mma_tf32(tmem + f_col, gh, vl, id2, 1u);
          mma_tf32(tmem + f_col, gl, vh, id2, 1u);
        }
        mma_commit(bar);
      }
      ok = mbar_wait(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      tc_after_sync();   // the next chunk overwrites W, V and G only after GEMM2 is done
    }
    if (failed) break;
    // epilogue 2: rows of type t keep dE/dq and their energy
    for (int d0 = 0; d0 < dimN; d0 += 16) {
      float f[16];
      tmem_ld16(lane_base + f_col + d0, f);
      if (tc == t) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int d = d0 + k;
          if (d < dim) fpbuf[static_cast<size_t>(c) * p.dimK + d] = f[k] * __ldg(p.q_scaler + d);
        }
      }
    }
    if (tc == t) pe_ann[c] = static_cast<double>(e_row - __ldg(p.out_bias + t));
    tc_before_sync();
    __syncthreads();   // TMEM is rewritten by the next type
    tc_after_sync();
  }
  if (failed) {
    if (tid == 0) atomicOr(err, 1);
    // let the MMAs of the phase that timed out finish before their TMEM is freed
    mbar_wait(bar, phase ^ 1u);
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L.cols)
                 : "memory");
}

// Centers sorted by type: a histogram, one scan, a scatter, with one atomic
// per warp and type (order within a type is arbitrary; every center's result
// is independent of it).  Unless `always`, the sort runs only when the Verlet
// list is rebuilt: the types of a system do not change between rebuilds, and
// k_ann_tc takes each tile's type range from its rows, so a stale order costs
// speed, never correctness.
__global__ void k_type_clear(int* counts, const NeighborState* st)
{
  if (st->rebuild && threadIdx.x < 2 * kMaxTypes) counts[threadIdx.x] = 0;
}

__global__ void k_type_hist(int N, const Site* __restrict__ sites, int T, int* counts,
                            const NeighborState* st, int always)
{
  if (!always && !st->rebuild) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = i < N ? static_cast<int>(sites[i].type) : -1;
  const int lane = threadIdx.x & 31;
  for (int u = 0; u < T; ++u) {
    const unsigned m = __ballot_sync(0xffffffffu, t == u);
    if (m && lane == __ffs(m) - 1) atomicAdd(counts + u, __popc(m));
  }
}

__global__ void k_type_scan(int T, int* counts, const NeighborState* st, int always)
{
  if (!always && !st->rebuild) return;
  // counts[0..T) -> exclusive starts in counts[T..2T), cursors reset to them
  int acc = 0;
  for (int t = 0; t < T; ++t) {
    const int c = counts[t];
    counts[T + t] = acc;
    counts[t] = acc;
    acc += c;
  }
}

__global__ void k_type_scatter(int N, const Site* __restrict__ sites, int T, int* cursor,
                               int* order, const NeighborState* st, int always)
{
  if (!always && !st->rebuild) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = i < N ? static_cast<int>(sites[i].type) : -1;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  for (int u = 0; u < T; ++u) {
    const unsigned m = __ballot_sync(0xffffffffu, t == u);
    if (!m) continue;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cursor + u, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (t == u) order[base + __popc(m & below)] = i;
  }
}

}  // namespace

size_t ann_tc_smem_bytes(const ModelParams& p)
{
  const int hc = ann_tc_chunk(p);
  return hc ? ann_tc_layout(p, hc).total : 0;
}

bool ann_tc_supported(const ModelParams& p, std::string& why)
{
  const int hc = ann_tc_chunk(p);
  if (!hc || ((p.dim + 15) & ~15) > 256) {
    why = "the tensor-core ANN tiles of this model do not fit one SM";
    return false;
  }
  return true;
}

void ann_tc_prepare(const ModelParams& p)
{
  cudaFuncSetAttribute(k_ann_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(ann_tc_smem_bytes(p)));
}

void launch_type_order(Engine& e, int N, bool always, cudaStream_t s)
{
  const ModelParams& p = e.params;
  ForceScratch& sc = e.scratch;
  const int threads = 256, grid = (N + threads - 1) / threads;
  if (always) cudaMemsetAsync(sc.type_counts, 0, sizeof(int) * 2 * kMaxTypes, s);
  else k_type_clear<<<1, 32, 0, s>>>(sc.type_counts, e.d_nstate);
  k_type_hist<<<grid, threads, 0, s>>>(N, sc.sites, p.T, sc.type_counts, e.d_nstate, always);
  k_type_scan<<<1, 1, 0, s>>>(p.T, sc.type_counts, e.d_nstate, always);
  k_type_scatter<<<grid, threads, 0, s>>>(N, sc.sites, p.T, sc.type_counts, sc.order, e.d_nstate,
                                          always);
}

void launch_ann_tc(Engine& e, int N, cudaStream_t s)
{
  const ModelParams& p = e.params;
  ForceScratch& sc = e.scratch;
  const int tiles = (N + kRows - 1) / kRows;
  k_ann_tc<<<tiles, kRows, ann_tc_smem_bytes(p), s>>>(p, N, ann_tc_chunk(p), sc.order, sc.sites,
                                                       sc.q, sc.pe_ann, sc.fp,
                                                       &e.d_nstate->ann_error);
}

}  // namespace nepx

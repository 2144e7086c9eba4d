// engine.cu -- handle construction, device uploads and box handling.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <vector>

#include "engine.h"

namespace nepx {

void upload_invariant_tables();

namespace {

__global__ void k_set_box(Box* dst, Box src) { *dst = src; }

template <typename T>
cudaError_t dalloc(T*& ptr, size_t count)
{
  return cudaMalloc(reinterpret_cast<void**>(&ptr), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

std::string make_box(const double* h, const int* pbc, Box& b)
{
  std::memcpy(b.h, h, sizeof(double) * 9);
  for (int d = 0; d < 3; ++d) b.pbc[d] = pbc[d] ? 1 : 0;
  // inverse with the cofactor order of the reference (box.cu:101-118)
  b.hinv[0] = h[4] * h[8] - h[5] * h[7];
  b.hinv[1] = h[2] * h[7] - h[1] * h[8];
  b.hinv[2] = h[1] * h[5] - h[2] * h[4];
  b.hinv[3] = h[5] * h[6] - h[3] * h[8];
  b.hinv[4] = h[0] * h[8] - h[2] * h[6];
  b.hinv[5] = h[2] * h[3] - h[0] * h[5];
  b.hinv[6] = h[3] * h[7] - h[4] * h[6];
  b.hinv[7] = h[1] * h[6] - h[0] * h[7];
  b.hinv[8] = h[0] * h[4] - h[1] * h[3];
  const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  if (!std::isfinite(det) || det == 0.0) return "singular or non-finite box";
  for (int k = 0; k < 9; ++k) b.hinv[k] /= det;
  b.ortho = h[1] == 0 && h[2] == 0 && h[3] == 0 && h[5] == 0 && h[6] == 0 && h[7] == 0;
  for (int k = 0; k < 9; ++k) {
    b.fh[k] = static_cast<float>(b.h[k]);
    b.fh[9 + k] = static_cast<float>(b.hinv[k]);
  }
  return "";
}

bool large_box_ok(const Engine& e, const Box& b)
{
  // small-box criterion of the reference (nep.cu:2002-2030): a periodic
  // thickness <= 2.5 (rc + 1) takes the image-expansion path
  const double rc = e.model.rc_max;
  for (int d = 0; d < 3; ++d) {
    if (!b.pbc[d]) continue;
    const double* r = b.hinv + 3 * d;
    const double thick = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    if (thick <= 2.5 * (rc + e.skin)) return false;
  }
  return true;
}

void launch_set_box(Engine& e, const Box& b, cudaStream_t stream)
{
  k_set_box<<<1, 1, 0, stream>>>(e.d_box, b);
}

std::string engine_create(Engine& e, const std::string& nep_path, int max_atoms)
{
  std::string err = load_nep(nep_path, e.model);
  if (!err.empty()) return err;
  if (cudaGetDevice(&e.device) != cudaSuccess) return "no CUDA device";
  const NepModel& m = e.model;
  ModelParams& p = e.params;
  std::memset(&p, 0, sizeof(p));
  p.version = m.version;
  p.T = m.num_types;
  p.nR = m.n_max_radial + 1;
  p.nA = m.n_max_angular + 1;
  p.kR = m.basis_radial + 1;
  p.kA = m.basis_angular + 1;
  p.L_max = m.L_max;
  p.nlm = m.L_max > 4 ? kNumLMHigh : kNumLM;   // moment stride per n
  p.num_L = m.num_L;
  p.dim = m.dim;
  p.dimK = (m.dim + 7) & ~7;
  p.H = m.H;
  p.num_inv = 0;
  for (int v = 0; v < kMaxInv; ++v)
    if (m.has_inv[v]) p.inv_id[p.num_inv++] = v;
  for (int t = 0; t < m.num_types; ++t) {
    p.rc_r[t] = m.rc_radial[t];
    p.rc_a[t] = m.rc_angular[t];
    p.Z[t] = m.Z[t];
  }
  p.zbl = m.zbl;
  p.zbl_flexible = m.zbl_flexible;
  p.typewise_zbl = m.typewise_zbl;
  p.zbl_rc_inner = m.zbl_rc_inner;
  p.zbl_rc_outer = m.zbl_rc_outer;
  p.typewise_factor = m.typewise_factor;
  p.num_c_radial = p.T * p.T * p.nR * p.kR;
  if (p.T * p.T * (p.nR * p.kR + p.nA * p.kA) > 12288)
    return "descriptor coefficient table too large for shared memory";

  upload_invariant_tables();
  // one parameter allocation: c_pair | w0 | b0 | w0t | w1 | out_bias | q_scaler | zbl | rc_r |
  // rc_a
  std::vector<float> blob;
  auto append = [&blob](const std::vector<float>& v) {
    const size_t at = blob.size();
    blob.insert(blob.end(), v.begin(), v.end());
    while (blob.size() % 4) blob.push_back(0.0f);   // 16-byte aligned blocks
    return at;
  };
  // w0 transposed for the ANN, rows zero-padded to H4 (float4 over hidden units)
  p.H4 = (p.H + 3) & ~3;
  std::vector<float> w0t(static_cast<size_t>(p.T) * p.dim * p.H4, 0.0f);
  for (int t = 0; t < p.T; ++t)
    for (int h = 0; h < p.H; ++h)
      for (int d = 0; d < p.dim; ++d)
        w0t[(static_cast<size_t>(t) * p.dim + d) * p.H4 + h] =
          m.w0[(static_cast<size_t>(t) * p.H + h) * p.dim + d];
  const size_t o_c = append(m.c_pair), o_w0 = append(m.w0), o_b0 = append(m.b0);
  const size_t o_w0t = append(w0t);
  const size_t o_w1 = append(m.w1), o_ob = append(m.out_bias), o_qs = append(m.q_scaler);
  const size_t o_z = append(m.zbl_para.empty() ? std::vector<float>(1, 0.0f) : m.zbl_para);
  const size_t o_rr = append(std::vector<float>(m.rc_radial, m.rc_radial + kMaxTypes));
  const size_t o_ra = append(std::vector<float>(m.rc_angular, m.rc_angular + kMaxTypes));
  std::vector<float> pc(4 * static_cast<size_t>(p.T) * p.T);
  const size_t tt = static_cast<size_t>(p.T) * p.T;
  for (int t1 = 0; t1 < p.T; ++t1)
    for (int t2 = 0; t2 < p.T; ++t2) {
      const size_t k = static_cast<size_t>(t1) * p.T + t2;
      const float rr = (p.rc_r[t1] + p.rc_r[t2]) * 0.5f, ra = (p.rc_a[t1] + p.rc_a[t2]) * 0.5f;
      pc[k] = rr;
      pc[tt + k] = 1.0f / rr;
      pc[2 * tt + k] = ra;
      pc[3 * tt + k] = 1.0f / ra;
    }
  const size_t o_pc = append(pc);
  if (dalloc(e.d_params, blob.size()) != cudaSuccess) return "cudaMalloc failed (parameters)";
  if (cudaMemcpy(e.d_params, blob.data(), blob.size() * sizeof(float), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return "cudaMemcpy failed (parameters)";
  p.c_pair = e.d_params + o_c;
  p.w0 = e.d_params + o_w0;
  p.w0t = e.d_params + o_w0t;
  p.b0 = e.d_params + o_b0;
  p.w1 = e.d_params + o_w1;
  p.out_bias = e.d_params + o_ob;
  p.q_scaler = e.d_params + o_qs;
  p.zbl_para = e.d_params + o_z;
  e.d_rc_r = e.d_params + o_rr;
  e.d_rc_a = e.d_params + o_ra;
  p.pair_cut = e.d_params + o_pc;

  // neighbour rows: the reference's MN_radial*1.25 scaled by ((rc+skin)/rc)^3
  const int N = std::max(max_atoms, 1);
  e.capacity = N;
  NeighborBuffers& nb = e.nbr;
  nb.mn_r = m.MN_radial;
  nb.mn_a = m.MN_angular;
  const double rc = m.rc_max, rv = rc + e.skin;
  nb.mn_v = static_cast<int>(m.MN_radial * rv * rv * rv / (rc * rc * rc));
  nb.mn_v = std::max(nb.mn_v, nb.mn_r);
  if (nb.mn_v > 2048) return "Verlet row capacity above 2048 is not supported";
  nb.pow2_v = 32;
  while (nb.pow2_v < nb.mn_v) nb.pow2_v <<= 1;
  nb.cell_cap = std::max(N, 4096);
  bool ok = true;
  ok &= dalloc(nb.nn_v, N) == cudaSuccess;
  ok &= dalloc(nb.nl_v, static_cast<size_t>(N) * nb.mn_v) == cudaSuccess;
  ok &= dalloc(nb.nn_r, N) == cudaSuccess;
  ok &= dalloc(nb.nl_r, static_cast<size_t>(N) * nb.mn_r) == cudaSuccess;
  ok &= dalloc(nb.nn_a, N) == cudaSuccess;
  ok &= dalloc(nb.nl_a, static_cast<size_t>(N) * nb.mn_a) == cudaSuccess;
  nb.rebuild_blocks = neighbor_rebuild_blocks(nb.pow2_v);
  if (nb.rebuild_blocks < 1) return "the neighbour rebuild kernel cannot be resident on this device";
  ok &= dalloc(nb.gsync, 2) == cudaSuccess;
  ok &= dalloc(nb.scan_part, nb.rebuild_blocks) == cudaSuccess;
  ok &= dalloc(nb.cell_count, nb.cell_cap) == cudaSuccess;
  ok &= dalloc(nb.cell_start, nb.cell_cap) == cudaSuccess;
  ok &= dalloc(nb.cell_atoms, N) == cudaSuccess;
  ok &= dalloc(nb.cell_of, N) == cudaSuccess;
  ok &= dalloc(nb.cell_sites, N) == cudaSuccess;
  ok &= dalloc(nb.x0, 3 * static_cast<size_t>(N)) == cudaSuccess;
  ok &= dalloc(e.scratch.sites, N) == cudaSuccess;
  ok &= dalloc(e.scratch.qrad, static_cast<size_t>(N) * p.nR) == cudaSuccess;
  ok &= dalloc(e.scratch.alpha, static_cast<size_t>(N) * p.T * basis_stride(p)) == cudaSuccess;
  ok &= dalloc(e.scratch.f12, static_cast<size_t>(N) * nb.mn_a) == cudaSuccess;
  ok &= dalloc(e.scratch.pe_ann, N) == cudaSuccess;
  ok &= dalloc(e.scratch.acoef, static_cast<size_t>(N) * p.nA * p.nlm) == cudaSuccess;
  ok &= dalloc(e.scratch.tune_out, 13 * static_cast<size_t>(N)) == cudaSuccess;
  ok &= dalloc(e.d_box, 1) == cudaSuccess;
  ok &= dalloc(e.d_nstate, 1) == cudaSuccess;
  if (!ok) return "cudaMalloc failed (per-atom buffers)";
  NeighborState init{};
  init.box_scale = 1.0;
  for (int k = 0; k < 9; ++k) init.box_def[k] = (k % 4 == 0) ? 1.0 : 0.0;
  if (cudaMemcpy(e.d_nstate, &init, sizeof(init), cudaMemcpyHostToDevice) != cudaSuccess)
    return "cudaMemcpy failed (neighbour state)";
  if (cudaMemset(nb.nn_a, 0, sizeof(int) * N) != cudaSuccess ||
      cudaMemset(nb.gsync, 0, 2 * sizeof(unsigned)) != cudaSuccess)
    return "cudaMemset failed";
  if (fused_smem_bytes(p) > 227 * 1024)
    return "descriptor kernel needs more shared memory than a CTA has (not supported)";
  set_fused_smem_limits(p);
  if (cudaGetLastError() != cudaSuccess) return "CUDA error during setup";
  return "";
}

namespace {

// Launch shapes the autotuner picked, per (device, model shape, precision,
// row path, size class): every handle of the process reuses them, and with
// NEPX_TUNE_FILE set they are read from and appended to that file, so later
// runs skip the timing calls too.
struct TuneKey {
  int v[14];
  bool operator==(const TuneKey& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};
struct TuneVal {
  int filter_group, group, fused_minb, f12_group, gather_group, fuse_f12, gather_minb;
};

std::mutex g_tune_mu;
std::vector<std::pair<TuneKey, TuneVal>> g_tune;
bool g_tune_loaded = false;

TuneKey tune_key(const Engine& e, int N)
{
  const ModelParams& p = e.params;
  int size_class = 0;
  while ((1 << (size_class + 1)) <= N) ++size_class;   // floor(log2 N)
  TuneKey k{{e.device, e.use_xr ? 1 : 0, e.precision, p.T, p.nR, p.nA, p.kR, p.kA, p.L_max,
             p.dim, p.H, p.num_inv, size_class, 3}};
  return k;
}

void tune_load_file()
{
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("NEPX_TUNE_FILE");
  if (!path) return;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    TuneKey k;
    TuneVal v;
    bool ok = true;
    for (int& x : k.v) ok = ok && static_cast<bool>(ls >> x);
    ok = ok && static_cast<bool>(ls >> v.filter_group >> v.group >> v.fused_minb >> v.f12_group >>
                                 v.gather_group >> v.fuse_f12 >> v.gather_minb);
    // only the shapes the launchers instantiate; anything else is ignored
    auto lanes = [](int g) { return g == 4 || g == 8; };
    ok = ok && lanes(v.filter_group) && lanes(v.group) && lanes(v.f12_group) &&
         lanes(v.gather_group) && (v.fused_minb == 3 || v.fused_minb == 4) &&
         (v.fuse_f12 == 0 || v.fuse_f12 == 1) && (v.gather_minb == 3 || v.gather_minb == 4);
    if (ok) g_tune.emplace_back(k, v);
  }
}

bool tune_lookup(const TuneKey& k, TuneVal& v)
{
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_load_file();
  for (const auto& kv : g_tune)
    if (kv.first == k) {
      v = kv.second;
      return true;
    }
  return false;
}

void tune_store(const TuneKey& k, const TuneVal& v)
{
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (const auto& kv : g_tune)
    if (kv.first == k) return;
  g_tune.emplace_back(k, v);
  if (const char* path = std::getenv("NEPX_TUNE_FILE")) {
    std::ofstream out(path, std::ios::app);
    for (int x : k.v) out << x << ' ';
    out << v.filter_group << ' ' << v.group << ' ' << v.fused_minb << ' ' << v.f12_group << ' '
        << v.gather_group << ' ' << v.fuse_f12 << ' ' << v.gather_minb << '\n';
  }
}

}  // namespace

void engine_autotune(Engine& e, int N, const double* pos, const int* type, cudaStream_t stream)
{
  const TuneKey key = tune_key(e, N);
  TuneVal known{};
  if (tune_lookup(key, known)) {
    e.filter_group = known.filter_group;
    e.group = known.group;
    e.fused_minb = known.fused_minb;
    e.f12_group = known.f12_group;
    e.gather_group = known.gather_group;
    e.fuse_f12 = known.fuse_f12 != 0;
    e.gather_minb = known.gather_minb;
    e.tuned = true;
    return;
  }
  // candidate lanes per center; each variant runs 3 times, the median counts
  const int groups[2] = {4, 8};
  float best_f = 1e30f, best_g = 1e30f;
  int pick_f = e.group, pick_g = e.gather_group;
  cudaEvent_t a, b, c;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventCreate(&c);
  int pick_a = e.f12_group;
  if (!e.use_xr) {
    float best = 1e30f;
    int pick = e.filter_group;
    // each grouping: one untimed launch, then the median of five
    for (int g : groups) {
      e.filter_group = g;
      float t[6];
      for (int r = 0; r < 6; ++r) {
        cudaEventRecord(a, stream);
        launch_filter(e, N, stream);
        cudaEventRecord(b, stream);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t[r], a, b);
      }
      std::sort(t + 1, t + 6);
      if (t[3] < best) {
        best = t[3];
        pick = g;
      }
    }
    e.filter_group = pick;
  }
  // the descriptor kernel's occupancy builds (CTAs per SM), when the shape has
  // two (the FP32 build of the small shape; the tensor-core build comes at 3)
  const int minbs[2] = {3, 4};
  const int n_minb = (fused_occupancy_variants(e.params) && e.precision == 0) ? 2 : 1;
  if (n_minb == 1) e.fused_minb = 3;
  int pick_m = e.fused_minb;
  // the descriptor kernel with and without the angular partial forces (the
  // fused form exists for the small shape on Verlet rows)
  e.fuse_f12 = true;
  const int n_ff = fused_angular_force(e) ? 2 : 1;
  e.fuse_f12 = false;
  bool pick_ff = false;
  for (int ff = 0; ff < n_ff; ++ff)
  for (int gf : groups) {
    for (int mi = 0; mi < n_minb; ++mi)
    for (int gg : groups) {
      e.fuse_f12 = ff == 1;
      e.group = gf;
      e.fused_minb = minbs[mi];
      e.f12_group = gg;   // angular-force grouping varies together with the gather's
      e.gather_group = gg;
      // with the fused form the angular-force grouping plays no part (the
      // gather's groupings are timed with the separate form)
      if (e.fuse_f12 && gg != groups[0]) continue;
      float tf[3], tg[3];
      // one untimed call first: each build's first launch pays for its
      // instruction cache and the rows' way into L2
      launch_descriptor(e, N, pos, type, stream);
      for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a, stream);
        launch_descriptor(e, N, pos, type, stream);
        cudaEventRecord(b, stream);
        double* out = e.scratch.tune_out;   // 13 N doubles: pe, force, virial
        launch_gather(e, N, pos, type, out, out + N, out + 4 * static_cast<size_t>(N), false,
                      stream);
        cudaEventRecord(c, stream);
        cudaEventSynchronize(c);
        cudaEventElapsedTime(&tf[r], a, b);
        cudaEventElapsedTime(&tg[r], b, c);
      }
      std::sort(tf, tf + 3);
      std::sort(tg, tg + 3);
      if (tf[1] < best_f) {
        best_f = tf[1];
        pick_f = gf;
        pick_m = e.fused_minb;
        pick_a = gg;
        pick_ff = e.fuse_f12;
      }
      if (tg[1] < best_g) {
        best_g = tg[1];
        pick_g = gg;
      }
    }
  }
  // the Verlet-row gather's two occupancy builds, with each grouping (the
  // rows, alpha and f12 of the last descriptor call serve every variant)
  int pick_gm = 3;
  if (!e.use_xr && e.params.L_max <= 4) {
    best_g = 1e30f;
    for (int gm = 3; gm <= 4; ++gm)
      for (int gg : groups) {
        e.gather_minb = gm;
        e.gather_group = gg;
        // one untimed launch, then the median of five (short kernels: the
        // picks must not follow the noise of single launches)
        float tg[6];
        for (int r = 0; r < 6; ++r) {
          cudaEventRecord(a, stream);
          double* out = e.scratch.tune_out;
          launch_gather(e, N, pos, type, out, out + N, out + 4 * static_cast<size_t>(N), false,
                        stream);
          cudaEventRecord(b, stream);
          cudaEventSynchronize(b);
          cudaEventElapsedTime(&tg[r], a, b);
        }
        std::sort(tg + 1, tg + 6);
        if (tg[3] < best_g) {
          best_g = tg[3];
          pick_g = gg;
          pick_gm = gm;
        }
      }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaEventDestroy(c);
  e.gather_minb = pick_gm;
  e.group = pick_f;
  e.fused_minb = pick_m;
  e.f12_group = pick_a;
  e.gather_group = pick_g;
  e.fuse_f12 = pick_ff;
  e.tuned = true;
  tune_store(key, TuneVal{e.filter_group, e.group, e.fused_minb, e.f12_group, e.gather_group,
                          e.fuse_f12 ? 1 : 0, e.gather_minb});
  if (std::getenv("NEPX_VERBOSE"))
    std::fprintf(stderr,
                 "nepx autotune (N=%d): filter G=%d, fused G=%d at %d CTAs/SM, angular force "
                 "%s, G=%d, gather G=%d at %d CTAs/SM\n",
                 N, e.filter_group, e.group, e.fused_minb,
                 e.fuse_f12 ? "in the descriptor kernel" : "own kernel", e.f12_group,
                 e.gather_group, e.gather_minb);
}

namespace {

// Largest power of two p with max_abs * p <= 2^14 (1 when max_abs is 0): the
// per-layer scale that keeps 16-bit operands inside FP16's range with room
// for the products' accumulation.
float pow2_scale(float max_abs)
{
  if (!(max_abs > 0.0f) || !std::isfinite(max_abs)) return 1.0f;
  int ex = 0;
  std::frexp(max_abs, &ex);   // max_abs < 2^ex
  return std::ldexp(1.0f, std::max(-60, std::min(60, 14 - ex)));
}

unsigned short to16(float x, bool bf16)
{
  if (bf16) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<const unsigned short*>(&h);
  }
  const __half h = __float2half_rn(x);
  return *reinterpret_cast<const unsigned short*>(&h);
}

}  // namespace

std::string engine_set_precision(Engine& e, int mode)
{
  if (mode < 0 || mode > 2) return "precision mode must be 0 (FP32), 1 (FP16) or 2 (BF16)";
  ModelParams& p = e.params;
  if (mode != 0) {
    // the descriptor kernel's MMAs: M = 128 stacked hidden units per chunk
    // (m = t H + h over all types) and M = 128 descriptor components
    if (p.dim > 128 || p.T * p.H > 1024)
      return "the tensor-core ANN takes dim <= 128 and at most 1024 hidden units over all types";
    const NepModel& m = e.model;
    const bool bf16 = mode == 2;
    p.tc_dimk = (p.dim + 15) & ~15;
    p.tc_kt = (p.T * p.H + 127) / 128 * 128;
    float wmax = 0.0f, w1max = 0.0f;
    for (float x : m.w0) wmax = std::max(wmax, std::fabs(x));
    for (float x : m.w1) w1max = std::max(w1max, std::fabs(x));
    p.tc_sw = pow2_scale(wmax);
    p.tc_sg = pow2_scale(w1max);   // |w1 (1 - x^2)| <= |w1|
    const size_t nw = static_cast<size_t>(p.T) * p.H * p.tc_dimk;
    const size_t nwt = static_cast<size_t>(p.dim) * p.tc_kt;
    std::vector<unsigned short> h16(nw + nwt, to16(0.0f, bf16));
    for (int t = 0; t < p.T; ++t)
      for (int h = 0; h < p.H; ++h)
        for (int d = 0; d < p.dim; ++d) {
          const size_t mrow = static_cast<size_t>(t) * p.H + h;
          const float w = m.w0[mrow * p.dim + d] * p.tc_sw;
          h16[mrow * p.tc_dimk + d] = to16(w, bf16);
          h16[nw + static_cast<size_t>(d) * p.tc_kt + mrow] = to16(w, bf16);
        }
    // one buffer per handle (its size depends on the model only): captured MD
    // graphs keep its address, so a later precision switch overwrites it in place
    if (!e.d_w16 &&
        cudaMalloc(reinterpret_cast<void**>(&e.d_w16), sizeof(unsigned short) * h16.size()) !=
          cudaSuccess) {
      e.d_w16 = nullptr;
      return "cudaMalloc failed (16-bit ANN weights)";
    }
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(e.d_w16, h16.data(), sizeof(unsigned short) * h16.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return "cudaMemcpy failed (16-bit ANN weights)";
    p.w0h = e.d_w16;
    p.w0th = e.d_w16 + nw;
    p.tc_bf16 = bf16 ? 1 : 0;
    if (fused_tc_smem_bytes(p) > 227 * 1024)
      return "the tensor-core ANN tiles of this model do not fit one CTA's shared memory";
    set_fused_smem_limits(p);
    if (cudaGetLastError() != cudaSuccess) return "CUDA error setting up the tensor-core ANN";
  }
  if (e.precision != mode) e.tuned = false;
  e.precision = mode;
  return "";
}

void engine_destroy(Engine& e)
{
  NeighborBuffers& nb = e.nbr;
  void* ptrs[] = {e.d_params, e.d_box, e.d_nstate, nb.nn_v, nb.nl_v, nb.nn_r, nb.nl_r,
                  nb.nn_a, nb.nl_a, nb.gsync, nb.scan_part, nb.cell_count, nb.cell_start, nb.cell_atoms, nb.cell_of,
                  nb.cell_sites, nb.x0, e.scratch.alpha, e.scratch.f12, e.scratch.pe_ann, e.d_w16,
                  e.scratch.tune_out, e.scratch.acoef, e.scratch.sites, e.scratch.qrad,
                  e.xr.er, e.xr.ea, e.xr.large,
                  e.xr.d_si, e.xr.d_soff};
  for (void* q : ptrs)
    if (q) cudaFree(q);
}

}  // namespace nepx

// capi.cu -- the extern "C" boundary declared in include/nepx.h.
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "../../include/nepx.h"
#include "engine.h"

#include "handle.h"

namespace {

int fail(nepx_handle* h, int code, const std::string& msg)
{
  if (h) h->error = msg;
  return code;
}

int cuda_fail(nepx_handle* h, const char* what)
{
  const cudaError_t err = cudaGetLastError();
  return fail(h, NEPX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

const char* const kUnsupportedBox =
  "box thinner than 2.5 (rc + 1) in one periodic direction and thicker than 10 rc in another "
  "(unsupported, as in the reference)";

}  // namespace

namespace nepx {

int decode_state(nepx_handle* h, const NeighborState& s)
{
  if (s.overflow) {
    const char* which = (s.overflow & 1) ? "Verlet" : (s.overflow & 2) ? "radial" : "angular";
    return fail(h, NEPX_ERR_OVERFLOW,
                std::string("a ") + which +
                  " neighbour row exceeded its capacity; raise MN_radial/MN_angular in nep.txt");
  }
  if (s.nonfinite) return fail(h, NEPX_ERR_NONFINITE, "non-finite energy or force");
  if (s.box_error) return fail(h, NEPX_ERR_BOX, kUnsupportedBox);
  if (s.ann_error)
    return fail(h, NEPX_ERR_CUDA, "a tensor-core ANN tile timed out waiting for its MMAs");
  if (s.sync_error) {
    h->engine.nbr.gsync_dirty = true;
    h->engine.force_rebuild = true;
    return fail(h, NEPX_ERR_CUDA, "the neighbour-list rebuild timed out at a grid-wide barrier");
  }
  return NEPX_OK;
}

int check_state(nepx_handle* h, bool wait)
{
  if (!h->state_pending) return NEPX_OK;
  if (wait) {
    if (cudaEventSynchronize(h->state_ready) != cudaSuccess) return cuda_fail(h, "event sync");
  } else if (cudaEventQuery(h->state_ready) != cudaSuccess) {
    cudaGetLastError();   // clear cudaErrorNotReady
    return NEPX_OK;
  }
  h->state_pending = false;
  return decode_state(h, *h->h_state);
}

}  // namespace nepx

using nepx::check_state;

// Why the last nepx_create of this thread failed (no handle to hold it).
thread_local std::string t_create_error;

extern "C" {

int nepx_create(const char* nep_path, int max_atoms, nepx_t** out)
{
  t_create_error.clear();
  if (!nep_path || !out || max_atoms < 1) {
    t_create_error = "nepx_create: null path or handle pointer, or max_atoms < 1";
    return NEPX_ERR_ARG;
  }
  *out = nullptr;
  auto* h = new (std::nothrow) nepx_handle();
  if (!h) {
    t_create_error = "nepx_create: out of host memory";
    return NEPX_ERR_CAPACITY;
  }
  std::string err = nepx::engine_create(h->engine, nep_path, max_atoms);
  if (!err.empty()) {
    t_create_error = "nepx_create: " + err;
    int code = NEPX_ERR_FILE;
    if (err.find("cuda") != std::string::npos || err.find("CUDA") != std::string::npos)
      code = NEPX_ERR_CUDA;
    else if (err.find("not supported") != std::string::npos)
      code = NEPX_ERR_UNSUPPORTED;
    nepx::engine_destroy(h->engine);
    delete h;
    return code;
  }
  if (cudaMallocHost(reinterpret_cast<void**>(&h->h_state), sizeof(nepx::NeighborState)) !=
        cudaSuccess ||
      cudaEventCreateWithFlags(&h->state_ready, cudaEventDisableTiming) != cudaSuccess) {
    nepx::engine_destroy(h->engine);
    delete h;
    t_create_error = "nepx_create: pinned host buffer or event creation failed";
    return NEPX_ERR_CUDA;
  }
  std::memset(h->h_state, 0, sizeof(nepx::NeighborState));
  *out = h;
  return NEPX_OK;
}

int nepx_destroy(nepx_t* h)
{
  if (!h) return NEPX_ERR_ARG;
  cudaDeviceSynchronize();
  nepx::engine_destroy(h->engine);
  if (h->h_state) cudaFreeHost(h->h_state);
  if (h->state_ready) cudaEventDestroy(h->state_ready);
  delete h;
  return NEPX_OK;
}

const char* nepx_last_error(const nepx_t* h)
{
  if (!h) return t_create_error.empty() ? "null handle" : t_create_error.c_str();
  return h->error.c_str();
}

int nepx_info(const nepx_t* h, int* info, double* rc)
{
  if (!h || !info) return NEPX_ERR_ARG;
  const nepx::NepModel& m = h->engine.model;
  int mask = 0;
  for (int v = 0; v < nepx::kMaxInv; ++v)
    if (m.has_inv[v]) mask |= 1 << v;
  const int vals[16] = {m.version,     m.num_types,     m.zbl ? 1 : 0, m.zbl_flexible ? 1 : 0,
                        m.n_max_radial, m.n_max_angular, m.basis_radial, m.basis_angular,
                        m.L_max,       m.num_L,         m.dim,         m.H,
                        m.MN_radial,   m.MN_angular,    mask,          m.typewise_zbl ? 1 : 0};
  std::memcpy(info, vals, sizeof(vals));
  if (rc)
    for (int t = 0; t < m.num_types; ++t) {
      rc[2 * t] = m.rc_radial[t];
      rc[2 * t + 1] = m.rc_angular[t];
    }
  return NEPX_OK;
}

int nepx_compute(nepx_t* h, const nepx_box* box, int n, const int* d_type, const double* d_pos,
                 double* d_pe, double* d_force, double* d_virial, unsigned flags, void* stream)
{
  if (!h) return NEPX_ERR_ARG;
  if (!box || !d_type || !d_pos || !d_pe || !d_force || !d_virial || n < 1)
    return fail(h, NEPX_ERR_ARG, "null pointer or n < 1");
  nepx::Engine& e = h->engine;
  if (n > e.capacity)
    return fail(h, NEPX_ERR_CAPACITY, "n = " + std::to_string(n) + " exceeds the capacity " +
                                        std::to_string(e.capacity) + " of this handle");
  int rc = check_state(h, false);
  if (rc) return rc;
  nepx::Box b;
  std::string err = nepx::make_box(box->h, box->pbc, b);
  if (!err.empty()) return fail(h, NEPX_ERR_BOX, err);
  // small boxes (and boxes too thin for the Verlet cell grid) take the
  // explicit-row path, rebuilt at every call like the reference's small-box path
  const int kind = nepx::box_kind(e, b);
  if (kind < 0) return fail(h, NEPX_ERR_BOX, kUnsupportedBox);
  const bool xr = kind == 1 || !nepx::large_box_ok(e, b);
  if (xr) {
    err = nepx::engine_enable_xr(e, 1);
    if (!err.empty()) return fail(h, NEPX_ERR_CUDA, err);
    e.xr.from_box = true;
  }
  e.use_xr = xr;
  const bool changed = !e.have_box || std::memcmp(&b, &e.last_box, sizeof(nepx::Box)) != 0;
  const bool rebuild = e.force_rebuild || changed || n != e.last_n;
  auto s = static_cast<cudaStream_t>(stream);
  nepx::launch_set_box(e, b, s);
  e.box_owner = nullptr;
  nepx::launch_neighbor_update(e, n, d_pos, d_type, rebuild, s);
  if (!e.tuned) nepx::engine_autotune(e, n, d_pos, d_type, s);
  nepx::launch_force(e, n, d_pos, d_type, d_pe, d_force, d_virial,
                     (flags & NEPX_ACCUMULATE) != 0, s);
  if (cudaPeekAtLastError() != cudaSuccess) return cuda_fail(h, "kernel launch");
  cudaMemcpyAsync(h->h_state, e.d_nstate, sizeof(nepx::NeighborState), cudaMemcpyDeviceToHost, s);
  cudaEventRecord(h->state_ready, s);
  h->state_pending = true;
  e.last_box = b;
  e.have_box = true;
  e.force_rebuild = false;
  e.last_n = n;
  if (flags & NEPX_SYNC_CHECK) {
    rc = check_state(h, true);
    if (rc) return rc;
    if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail(h, "stream sync");
  }
  return NEPX_OK;
}

int nepx_profile(nepx_t* h, const nepx_box* box, int n, const int* d_type, const double* d_pos,
                 double* d_pe, double* d_force, double* d_virial, int reps, double* ms,
                 void* stream)
{
  if (!h || !ms || reps < 1) return NEPX_ERR_ARG;
  nepx::Engine& e = h->engine;
  // first call settles the lists (and validates the arguments)
  int rc = nepx_compute(h, box, n, d_type, d_pos, d_pe, d_force, d_virial, NEPX_SYNC_CHECK, stream);
  if (rc) return rc;
  auto s = static_cast<cudaStream_t>(stream);
  cudaEvent_t ev[5];
  for (auto& x : ev) cudaEventCreate(&x);
  double acc[4] = {0, 0, 0, 0};
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(ev[0], s);
    nepx::launch_neighbor_update(e, n, d_pos, d_type, false, s);
    cudaEventRecord(ev[1], s);
    nepx::launch_descriptor(e, n, d_pos, d_type, s);
    cudaEventRecord(ev[2], s);
    nepx::launch_gather(e, n, d_pos, d_type, d_pe, d_force, d_virial, false, s);
    cudaEventRecord(ev[3], s);
    cudaEventSynchronize(ev[3]);
    float t;
    for (int k = 0; k < 3; ++k) {
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      acc[k] += t;
    }
    cudaEventElapsedTime(&t, ev[0], ev[3]);
    acc[3] += t;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  for (int k = 0; k < 4; ++k) ms[k] = acc[k] / reps;
  if (cudaPeekAtLastError() != cudaSuccess) return cuda_fail(h, "profile");
  return check_state(h, true);
}

int nepx_notify_box_changed(nepx_t* h)
{
  if (!h) return NEPX_ERR_ARG;
  h->engine.force_rebuild = true;
  return NEPX_OK;
}

int nepx_set_skin(nepx_t* h, double skin)
{
  if (!h) return NEPX_ERR_ARG;
  if (!(skin >= 0.0) || !std::isfinite(skin)) return fail(h, NEPX_ERR_ARG, "bad skin");
  if (skin > h->engine.skin)
    return fail(h, NEPX_ERR_UNSUPPORTED, "skin above the one the handle was sized for");
  h->engine.skin = skin;
  h->engine.force_rebuild = true;
  return NEPX_OK;
}

int nepx_neighbors(nepx_t* h, int which, int n, int* d_nn, int* d_nl, int mn, void* stream)
{
  if (!h || !d_nn || !d_nl || n < 1 || n > h->engine.capacity) return NEPX_ERR_ARG;
  const nepx::NeighborBuffers& nb = h->engine.nbr;
  const int src_mn = which == 0 ? nb.mn_r : nb.mn_a;
  if (mn < src_mn) return fail(h, NEPX_ERR_ARG, "mn smaller than the row capacity");
  auto s = static_cast<cudaStream_t>(stream);
  if (h->engine.use_xr) {
    nepx::launch_explicit_row_indices(h->engine, which, n, d_nn, d_nl, mn, s);
    if (cudaPeekAtLastError() != cudaSuccess) return cuda_fail(h, "copy neighbour rows");
    return NEPX_OK;
  }
  const int* nn = which == 0 ? nb.nn_r : nb.nn_a;
  const int* nl = which == 0 ? nb.nl_r : nb.nl_a;
  if (cudaMemcpyAsync(d_nn, nn, sizeof(int) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
      cudaMemcpy2DAsync(d_nl, sizeof(int) * mn, nl, sizeof(int) * src_mn, sizeof(int) * src_mn, n,
                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return cuda_fail(h, "copy neighbour rows");
  return NEPX_OK;
}

int nepx_set_precision(nepx_t* h, int mode)
{
  if (!h) return NEPX_ERR_ARG;
  if (mode != NEPX_PRECISION_FP32 && mode != NEPX_PRECISION_MIXED &&
      mode != NEPX_PRECISION_MIXED_BF16)
    return fail(h, NEPX_ERR_ARG, "unknown precision mode");
  const std::string err = nepx::engine_set_precision(h->engine, mode);
  if (!err.empty()) return fail(h, NEPX_ERR_UNSUPPORTED, err);
  return NEPX_OK;
}

int nepx_get_tuning(nepx_t* h, int* v, int* tuned)
{
  if (!h || !v) return NEPX_ERR_ARG;
  const nepx::Engine& e = h->engine;
  v[0] = e.filter_group;
  v[1] = e.group;
  v[2] = e.fused_minb;
  v[3] = e.f12_group;
  v[4] = e.gather_group;
  v[5] = e.fuse_f12 ? 1 : 0;
  v[6] = e.gather_minb;
  if (tuned) *tuned = e.tuned ? 1 : 0;
  return NEPX_OK;
}

int nepx_set_tuning(nepx_t* h, const int* v)
{
  if (!h || !v) return NEPX_ERR_ARG;
  auto lanes = [](int g) { return g == 4 || g == 8; };
  if (!lanes(v[0]) || !lanes(v[1]) || !(v[2] == 3 || v[2] == 4) || !lanes(v[3]) ||
      !lanes(v[4]) || !(v[5] == 0 || v[5] == 1) || !(v[6] == 3 || v[6] == 4))
    return fail(h, NEPX_ERR_ARG, "launch choice outside the built variants");
  nepx::Engine& e = h->engine;
  e.filter_group = v[0];
  e.group = v[1];
  e.fused_minb = v[2];
  e.f12_group = v[3];
  e.gather_group = v[4];
  e.fuse_f12 = v[5] == 1;
  e.gather_minb = v[6];
  e.tuned = true;
  return NEPX_OK;
}

int nepx_neighbor_stats(nepx_t* h, int* max_radial, int* max_angular, int* max_verlet,
                        void* stream)
{
  if (!h) return NEPX_ERR_ARG;
  auto s = static_cast<cudaStream_t>(stream);
  nepx::NeighborState st;
  if (cudaMemcpyAsync(&st, h->engine.d_nstate, sizeof(st), cudaMemcpyDeviceToHost, s) !=
        cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return cuda_fail(h, "read neighbour state");
  if (max_radial) *max_radial = st.max_nn[1];
  if (max_angular) *max_angular = st.max_nn[2];
  if (max_verlet) *max_verlet = st.max_nn[0];
  nepx::NeighborState cleared = st;
  cleared.max_nn[0] = cleared.max_nn[1] = cleared.max_nn[2] = 0;
  cleared.overflow = 0;
  cleared.nonfinite = 0;
  cleared.box_error = 0;
  cudaMemcpy(h->engine.d_nstate, &cleared, sizeof(cleared), cudaMemcpyHostToDevice);
  if (st.overflow) return fail(h, NEPX_ERR_OVERFLOW, "a neighbour row exceeded its capacity");
  if (st.nonfinite) return fail(h, NEPX_ERR_NONFINITE, "non-finite energy or force");
  return NEPX_OK;
}

}  // extern "C"

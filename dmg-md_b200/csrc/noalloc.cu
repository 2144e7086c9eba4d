// noalloc.cu -- nepx_compute_noalloc: the force call without any allocation.
//
// Some callers cannot call cudaMalloc once they are running: codes that hand
// all device memory to their own pool allocator at start-up (a library
// cudaMalloc then fails or fragments that pool), and real-time or
// safety-reviewed MD drivers whose rules forbid allocator calls after
// initialisation.  For them this entry point evaluates energy, force and
// virial with every per-call scratch buffer -- cell list, Verlet and typewise
// neighbour rows, descriptor derivatives, angular partial forces, the device
// box and the error flags -- carved from one file-scope static device array
// of kStaticScratchBytes (16 MiB) that each GPU loading the library holds
// until the process exits.  The handle still supplies the model parameters
// (uploaded once by nepx_create, which may be given max_atoms = 1).
//
// Setup: the first call on a device, with that device current, resolves the
// array's device address with cudaGetSymbolAddress (a host-side name of a
// __device__ array is not a device address).  Make that first call before
// any stream capture.  Every call shares the one array and keeps the last
// call's contents, so the flags are cleared and the neighbour rows rebuilt
// on every call; calls that overlap on the GPU (other streams, other host
// threads) race on it.  The call synchronises its stream before returning
// so the device flags can be checked.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/nepx.h"
#include "handle.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_static_scratch on the current device, resolved once
// per device (cudaGetSymbolAddress; the host-side name of a __device__ array
// is only a stand-in, not a device address).
cudaError_t static_scratch(void** out)
{
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_static_scratch);
    if (err != cudaSuccess) return err;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

// Bump carving of the static array in 256-byte aligned pieces.
struct Carver {
  unsigned char* base;
  size_t used = 0;
  template <typename T>
  T* take(size_t count)
  {
    used = (used + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += count * sizeof(T);
    return p;
  }
};

size_t bytes_needed(const nepx::Engine& e, int n)
{
  Carver c{nullptr};
  const nepx::NeighborBuffers& nb = e.nbr;
  const size_t N = n;
  const size_t cells = std::max<size_t>(N, 4096);
  c.take<nepx::Box>(1);
  c.take<nepx::NeighborState>(1);
  c.take<int>(N);               // nn_v
  c.take<int>(N * nb.mn_v);     // nl_v
  c.take<int>(N);               // nn_r
  c.take<int>(N * nb.mn_r);     // nl_r
  c.take<int>(N);               // nn_a
  c.take<int>(N * nb.mn_a);     // nl_a
  c.take<unsigned>(2);                   // grid-barrier counters
  c.take<int>(nb.rebuild_blocks);        // cell-scan partial sums
  c.take<int>(cells);           // cell_count
  c.take<int>(cells);           // cell_start
  c.take<int>(N);               // cell_atoms
  c.take<int>(N);               // cell_of
  c.take<nepx::Site>(N);        // cell_sites
  c.take<double>(3 * N);        // x0
  c.take<nepx::Site>(N);
  c.take<float>(N * e.params.nR);
  c.take<float>(N * e.params.T * nepx::basis_stride(e.params));
  c.take<float4>(N * nb.mn_a);
  c.take<double>(N);
  c.take<float>(N * e.params.nA * e.params.nlm);
  return c.used;
}

// The handle's engine runs the launches with its per-call buffers pointed
// into the static array for the duration of one call; the destructor puts the
// handle's own buffers back on every exit path.  Only plain pointer and
// scalar fields change hands (the model's host vectors are never copied), so
// nothing is allocated on the host either.
struct BorrowedBuffers {
  nepx::Engine& e;
  nepx::Box* d_box;
  nepx::NeighborState* d_nstate;
  nepx::NeighborBuffers nbr;
  nepx::ForceScratch scratch;
  int capacity;
  bool tuned, use_xr;
  int precision;
  explicit BorrowedBuffers(nepx::Engine& eng)
    : e(eng), d_box(eng.d_box), d_nstate(eng.d_nstate), nbr(eng.nbr), scratch(eng.scratch),
      capacity(eng.capacity), tuned(eng.tuned), use_xr(eng.use_xr), precision(eng.precision)
  {
  }
  ~BorrowedBuffers()
  {
    e.d_box = d_box;
    e.d_nstate = d_nstate;
    e.nbr = nbr;
    e.scratch = scratch;
    e.capacity = capacity;
    e.tuned = tuned;
    e.use_xr = use_xr;
    e.precision = precision;
  }
};

}  // namespace

extern "C" int nepx_compute_noalloc(nepx_t* h, const nepx_box* box, int n, const int* d_type,
                                    const double* d_pos, double* d_pe, double* d_force,
                                    double* d_virial, void* stream)
{
  if (!h) return NEPX_ERR_ARG;
  if (!box || !d_type || !d_pos || !d_pe || !d_force || !d_virial || n < 1) {
    h->error = "null pointer or n < 1";
    return NEPX_ERR_ARG;
  }
  nepx::Engine& e = h->engine;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != e.device) {
    cudaGetLastError();
    h->error = "the current CUDA device is not the one the handle was created on";
    return NEPX_ERR_ARG;
  }
  if (bytes_needed(e, n) > kStaticScratchBytes) {
    h->error = "n = " + std::to_string(n) +
               " needs more than the 16 MiB static scratch of nepx_compute_noalloc";
    return NEPX_ERR_CAPACITY;
  }
  nepx::Box b;
  std::string err = nepx::make_box(box->h, box->pbc, b);
  if (!err.empty() || !nepx::large_box_ok(e, b)) {
    h->error = err.empty() ? "box thinner than 2.5 (rc + skin) in a periodic direction" : err;
    return NEPX_ERR_BOX;
  }
  void* base = nullptr;
  if (static_scratch(&base) != cudaSuccess) {
    cudaGetLastError();
    h->error = "cudaGetSymbolAddress of the static scratch failed";
    return NEPX_ERR_CUDA;
  }
  // an earlier asynchronous nepx_compute on this handle may still have its
  // flags on the way into the pinned mirror: report its errors before this
  // call reuses the mirror
  int rc = nepx::check_state(h, true);
  if (rc) return rc;
  auto s = static_cast<cudaStream_t>(stream);
  {
    BorrowedBuffers keep(e);
    Carver c{static_cast<unsigned char*>(base)};
    const size_t N = n;
    const size_t cells = std::max<size_t>(N, 4096);
    nepx::NeighborBuffers& nb = e.nbr;
    e.d_box = c.take<nepx::Box>(1);
    e.d_nstate = c.take<nepx::NeighborState>(1);
    nb.nn_v = c.take<int>(N);
    nb.nl_v = c.take<int>(N * nb.mn_v);
    nb.nn_r = c.take<int>(N);
    nb.nl_r = c.take<int>(N * nb.mn_r);
    nb.nn_a = c.take<int>(N);
    nb.nl_a = c.take<int>(N * nb.mn_a);
    nb.gsync = c.take<unsigned>(2);
    nb.scan_part = c.take<int>(nb.rebuild_blocks);
    nb.gsync_dirty = false;
    nb.cell_count = c.take<int>(cells);
    nb.cell_start = c.take<int>(cells);
    nb.cell_atoms = c.take<int>(N);
    nb.cell_of = c.take<int>(N);
    nb.cell_sites = c.take<nepx::Site>(N);
    nb.x0 = c.take<double>(3 * N);
    nb.cell_cap = static_cast<int>(cells);
    e.scratch.sites = c.take<nepx::Site>(N);
    e.scratch.qrad = c.take<float>(N * e.params.nR);
    e.scratch.alpha = c.take<float>(N * e.params.T * nepx::basis_stride(e.params));
    e.scratch.f12 = c.take<float4>(N * nb.mn_a);
    e.scratch.pe_ann = c.take<double>(N);
    e.scratch.acoef = c.take<float>(N * e.params.nA * e.params.nlm);
    e.capacity = n;
    e.tuned = true;      // keeps the handle's kernel variants; no timing runs here
    e.precision = 0;     // FP32 ANN: the mixed path's buffers are not in the static array
    e.use_xr = false;
    // the array keeps the previous call's contents: clear the flags, rebuild
    cudaMemsetAsync(e.d_nstate, 0, sizeof(nepx::NeighborState), s);
    cudaMemsetAsync(nb.gsync, 0, 2 * sizeof(unsigned), s);
    nepx::launch_set_box(e, b, s);
    nepx::launch_neighbor_update(e, n, d_pos, d_type, true, s);
    nepx::launch_force(e, n, d_pos, d_type, d_pe, d_force, d_virial, false, s);
    if (cudaPeekAtLastError() != cudaSuccess) {
      h->error = std::string("kernel launch: ") + cudaGetErrorString(cudaGetLastError());
      return NEPX_ERR_CUDA;
    }
    // h_state is the handle's pinned flag mirror, allocated by nepx_create
    cudaMemcpyAsync(h->h_state, e.d_nstate, sizeof(nepx::NeighborState),
                    cudaMemcpyDeviceToHost, s);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    h->error = std::string("stream: ") + cudaGetErrorString(cudaGetLastError());
    return NEPX_ERR_CUDA;
  }
  return nepx::decode_state(h, *h->h_state);
}

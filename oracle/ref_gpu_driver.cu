// ref_gpu_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own FP32 GPU NEP (src/gpumd_compat, GPUMD-derived),
// compiled for sm_100a from its sources into oracle/_ref/libnep_ref_gpu.so by
// `make -C oracle ref-gpu`, through its public interface: NEP(path, N) and
// Potential::compute(box, type, position, potential, force, virial)
// (potential.cuh:82-88, nep.cu:2071-2100), with N1 = 0, N2 = N and zeroed
// outputs as NepForce::compute does (runtime.cu:557-568).  It is the "the
// reference's own NEP evaluation" the parity tests compare against, and the
// reference GPU timing of bench.py.  The reference appends neighbor.out in
// the working directory every 1000 calls, as it does in DMG-MD.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "gpumd_compat/box.cuh"
#include "gpumd_compat/gpu_vector.cuh"
#include "gpumd_compat/nep.cuh"

namespace {

struct RefGpu {
  gpumd_compat::NEP* nep = nullptr;
  gpumd_compat::GPU_Vector<int> type;
  gpumd_compat::GPU_Vector<double> pos, pe, force, virial;
  int n = 0;
};

}  // namespace

extern "C" void* refgpu_create(const char* path, int n)
{
  auto* r = new RefGpu();
  r->nep = new gpumd_compat::NEP(path, n);
  r->nep->N1 = 0;
  r->nep->N2 = n;
  r->n = n;
  r->type.resize(n);
  r->pos.resize(3 * static_cast<size_t>(n));
  r->pe.resize(n);
  r->force.resize(3 * static_cast<size_t>(n));
  r->virial.resize(9 * static_cast<size_t>(n));
  return r;
}

extern "C" void refgpu_destroy(void* p)
{
  auto* r = static_cast<RefGpu*>(p);
  delete r->nep;
  delete r;
}

// Loads type/position (device pointers) into the reference's buffers.
extern "C" int refgpu_set_atoms(void* p, const int* d_type, const double* d_pos)
{
  auto* r = static_cast<RefGpu*>(p);
  r->type.copy_from_device(d_type);
  r->pos.copy_from_device(d_pos);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// One force call; outputs copied to device pointers when they are non-null.
extern "C" int refgpu_compute(void* p, const double* h, const int* pbc, double* d_pe,
                              double* d_force, double* d_virial)
{
  auto* r = static_cast<RefGpu*>(p);
  gpumd_compat::Box box;
  std::memcpy(box.cpu_h, h, sizeof(double) * 9);
  box.pbc_x = pbc[0];
  box.pbc_y = pbc[1];
  box.pbc_z = pbc[2];
  box.get_inverse();
  box.set_is_orthogonal();
  cudaMemset(r->pe.data(), 0, sizeof(double) * r->n);
  cudaMemset(r->force.data(), 0, sizeof(double) * 3 * r->n);
  cudaMemset(r->virial.data(), 0, sizeof(double) * 9 * r->n);
  r->nep->compute(box, r->type, r->pos, r->pe, r->force, r->virial);
  if (d_pe) r->pe.copy_to_device(d_pe);
  if (d_force) r->force.copy_to_device(d_force);
  if (d_virial) r->virial.copy_to_device(d_virial);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Typewise rows of the last large-box compute (which = 0 radial, 1 angular),
// copied to host arrays: nn[n] and nl[n*mn] row-major (the reference stores
// them ordinal-major, NL[k*N + i], nep.cu:543-556).
extern "C" int refgpu_neighbors(void* p, int which, int* nn, int* nl, int mn)
{
  auto* r = static_cast<RefGpu*>(p);
  const int n = r->n;
  auto& NN = which == 0 ? r->nep->nep_data.NN_radial : r->nep->nep_data.NN_angular;
  auto& NL = which == 0 ? r->nep->nep_data.NL_radial : r->nep->nep_data.NL_angular;
  std::vector<int> hnn(n), hnl(NL.size());
  NN.copy_to_host(hnn.data(), n);
  NL.copy_to_host(hnl.data(), NL.size());
  const size_t cap = NL.size() / n;
  for (int i = 0; i < n; ++i) {
    nn[i] = hnn[i];
    for (int k = 0; k < hnn[i] && k < mn && static_cast<size_t>(k) < cap; ++k)
      nl[static_cast<size_t>(i) * mn + k] = hnl[static_cast<size_t>(k) * n + i];
  }
  return 0;
}

// Typewise rows of the last small-box compute (which = 0 radial, 1 angular):
// the neighbour index of every (atom, image) edge in the reference's order,
// copied row-major like refgpu_neighbors (small_box_data, nep.cu:2080-2095).
extern "C" int refgpu_neighbors_small(void* p, int which, int* nn, int* nl, int mn)
{
  auto* r = static_cast<RefGpu*>(p);
  const int n = r->n;
  auto& sb = r->nep->small_box_data;
  auto& NN = which == 0 ? sb.NN_radial : sb.NN_angular;
  auto& NL = which == 0 ? sb.NL_radial : sb.NL_angular;
  if (NN.size() != static_cast<size_t>(n)) return 1;
  std::vector<int> hnn(n), hnl(NL.size());
  NN.copy_to_host(hnn.data(), n);
  NL.copy_to_host(hnl.data(), NL.size());
  const size_t cap = NL.size() / n;
  for (int i = 0; i < n; ++i) {
    nn[i] = hnn[i];
    for (int k = 0; k < hnn[i] && k < mn && static_cast<size_t>(k) < cap; ++k)
      nl[static_cast<size_t>(i) * mn + k] = hnl[static_cast<size_t>(k) * n + i];
  }
  return 0;
}

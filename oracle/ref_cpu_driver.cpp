// ref_cpu_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own FP64 CPU NEP evaluator, NEP3_CPU
// (third_party/lammps-matpl-overlay/files/src/nep_cpu.cpp:2385-2479), the way
// the LAMMPS pair style does (files/src/pair_nep.cpp:260-283): periodic ghost
// atoms, a full neighbour list per center, Newton scatter onto neighbours and
// ghosts, then a fold of ghost forces and virials back onto their owners (the
// job of LAMMPS' reverse communication).  Compiled from the reference sources
// into oracle/_ref/libnep_ref_cpu.so by oracle/Makefile; it is the
// "reference" CPU baseline of bench.py and a parity pin for the oracle.
#include "nep_cpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Handle {
  std::string path;
  std::vector<std::unique_ptr<NEP3_CPU>> workers;
  double rc = 0.0;
};

NEP3_CPU* make_worker(const std::string& path, int num_types)
{
  auto* w = new NEP3_CPU();
  w->read_neptxt(path, false);
  w->map_atom_type_idx.resize(num_types);
  for (int t = 0; t < num_types; ++t) w->map_atom_type_idx[t] = t;
  return w;
}

struct Image {
  std::vector<double> x;     // 3 per atom (local then ghosts)
  std::vector<int> type;     // LAMMPS 1-based
  std::vector<int> owner;
};

void inverse3(const double* h, double* hi)
{
  const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) + h[1] * (h[5] * h[6] - h[3] * h[8]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  hi[0] = (h[4] * h[8] - h[5] * h[7]) / det;
  hi[1] = (h[2] * h[7] - h[1] * h[8]) / det;
  hi[2] = (h[1] * h[5] - h[2] * h[4]) / det;
  hi[3] = (h[5] * h[6] - h[3] * h[8]) / det;
  hi[4] = (h[0] * h[8] - h[2] * h[6]) / det;
  hi[5] = (h[2] * h[3] - h[0] * h[5]) / det;
  hi[6] = (h[3] * h[7] - h[4] * h[6]) / det;
  hi[7] = (h[1] * h[6] - h[0] * h[7]) / det;
  hi[8] = (h[0] * h[4] - h[1] * h[3]) / det;
}

}  // namespace

extern "C" void* nepref_create(const char* path)
{
  auto* h = new Handle();
  h->path = path;
  std::unique_ptr<NEP3_CPU> probe(new NEP3_CPU());
  probe->read_neptxt(path, false);
  h->rc = std::max(probe->paramb.rc_radial, probe->paramb.rc_angular);
  return h;
}

extern "C" void nepref_destroy(void* p) { delete static_cast<Handle*>(p); }

// Centers [begin, end) of an n-atom periodic box h (row-major, cell vectors
// as columns), SoA positions.  Outputs (n entries each, SoA) are overwritten:
// pe for the centers, forces and virials (xx yy zz xy xz yz yx zx zy) summed
// over all edges of those centers and folded onto owners.
extern "C" int nepref_compute_range(void* p, int n, const int* type, const double* h,
                                    const double* pos, int threads, int begin, int end,
                                    double* pe, double* force, double* virial)
{
  auto* H = static_cast<Handle*>(p);
  if (n <= 0 || begin < 0 || end > n || begin > end) return 1;
  int num_types = 0;
  for (int i = 0; i < n; ++i) num_types = std::max(num_types, type[i] + 1);
  double hi[9];
  inverse3(h, hi);
  const double rc = H->rc;
  // thickness of the cell along each fractional direction
  double thick[3];
  const double vol = std::fabs(h[0] * (h[4] * h[8] - h[5] * h[7]) +
                               h[1] * (h[5] * h[6] - h[3] * h[8]) +
                               h[2] * (h[3] * h[7] - h[4] * h[6]));
  for (int d = 0; d < 3; ++d) {
    const double len = std::sqrt(hi[3 * d] * hi[3 * d] + hi[3 * d + 1] * hi[3 * d + 1] +
                                 hi[3 * d + 2] * hi[3 * d + 2]);
    thick[d] = 1.0 / len;
  }
  (void)vol;
  // wrapped fractional coordinates of the local atoms
  std::vector<double> frac(3 * n);
  for (int i = 0; i < n; ++i) {
    const double r[3] = {pos[i], pos[n + i], pos[2 * n + i]};
    for (int d = 0; d < 3; ++d) {
      double s = hi[3 * d] * r[0] + hi[3 * d + 1] * r[1] + hi[3 * d + 2] * r[2];
      s -= std::floor(s);
      frac[3 * i + d] = s;
    }
  }
  // local atoms then ghosts within a fractional skin of rc / thickness
  Image im;
  double skin[3];
  int img[3];
  for (int d = 0; d < 3; ++d) {
    skin[d] = rc / thick[d];
    img[d] = static_cast<int>(std::ceil(skin[d]));
  }
  auto push = [&](int owner, const double* s) {
    for (int d = 0; d < 3; ++d)
      im.x.push_back(h[3 * d] * s[0] + h[3 * d + 1] * s[1] + h[3 * d + 2] * s[2]);
    im.type.push_back(type[owner] + 1);
    im.owner.push_back(owner);
  };
  for (int i = 0; i < n; ++i) push(i, &frac[3 * i]);
  for (int ia = -img[0]; ia <= img[0]; ++ia)
    for (int ib = -img[1]; ib <= img[1]; ++ib)
      for (int ic = -img[2]; ic <= img[2]; ++ic) {
        if (!ia && !ib && !ic) continue;
        for (int i = 0; i < n; ++i) {
          const double s[3] = {frac[3 * i] + ia, frac[3 * i + 1] + ib, frac[3 * i + 2] + ic};
          bool keep = true;
          for (int d = 0; d < 3; ++d)
            if (s[d] < -skin[d] || s[d] >= 1.0 + skin[d]) keep = false;
          if (keep) push(i, s);
        }
      }
  const int total = static_cast<int>(im.owner.size());
  // fractional bins covering [-skin, 1 + skin) with width >= skin
  int nb[3];
  for (int d = 0; d < 3; ++d) nb[d] = std::max(1, static_cast<int>((1.0 + 2.0 * skin[d]) / skin[d]));
  std::vector<int> bin_of(total), head(nb[0] * nb[1] * nb[2], -1), next(total, -1);
  auto bin_index = [&](const double* s, int* b3) {
    for (int d = 0; d < 3; ++d) {
      int b = static_cast<int>((s[d] + skin[d]) / (1.0 + 2.0 * skin[d]) * nb[d]);
      b3[d] = std::min(std::max(b, 0), nb[d] - 1);
    }
  };
  std::vector<double> sfrac(3 * total);
  for (int a = 0; a < total; ++a) {
    const double* r = &im.x[3 * a];
    for (int d = 0; d < 3; ++d)
      sfrac[3 * a + d] = hi[3 * d] * r[0] + hi[3 * d + 1] * r[1] + hi[3 * d + 2] * r[2];
    int b3[3];
    bin_index(&sfrac[3 * a], b3);
    const int b = (b3[2] * nb[1] + b3[1]) * nb[0] + b3[0];
    bin_of[a] = b;
    next[a] = head[b];
    head[b] = a;
  }
  // full neighbour lists of the centers
  const double rc2 = rc * rc;
  std::vector<std::vector<int>> nbrs(n);
  for (int i = begin; i < end; ++i) {
    int b3[3];
    bin_index(&sfrac[3 * i], b3);
    std::vector<int>& row = nbrs[i];
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int cx = b3[0] + dx, cy = b3[1] + dy, cz = b3[2] + dz;
          if (cx < 0 || cy < 0 || cz < 0 || cx >= nb[0] || cy >= nb[1] || cz >= nb[2]) continue;
          for (int a = head[(cz * nb[1] + cy) * nb[0] + cx]; a >= 0; a = next[a]) {
            if (a == i) continue;
            const double r[3] = {im.x[3 * a] - im.x[3 * i], im.x[3 * a + 1] - im.x[3 * i + 1],
                                 im.x[3 * a + 2] - im.x[3 * i + 2]};
            if (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] < rc2) row.push_back(a);
          }
        }
    std::sort(row.begin(), row.end());
  }
  // threads over disjoint center slices, private accumulators
  threads = std::max(1, std::min(threads, end - begin > 0 ? end - begin : 1));
  while (static_cast<int>(H->workers.size()) < threads)
    H->workers.emplace_back(make_worker(H->path, std::max(num_types, 1)));
  std::vector<std::vector<double>> f_acc(threads), v_acc(threads), e_acc(threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      const int lo = begin + static_cast<int>(static_cast<long long>(end - begin) * t / threads);
      const int hi_ = begin + static_cast<int>(static_cast<long long>(end - begin) * (t + 1) / threads);
      NEP3_CPU* w = H->workers[t].get();
      w->map_atom_type_idx.resize(std::max(num_types, 1));
      for (int k = 0; k < num_types; ++k) w->map_atom_type_idx[k] = k;
      std::vector<int> ilist;
      for (int i = lo; i < hi_; ++i) ilist.push_back(i);
      std::vector<int> numneigh(total, 0);
      std::vector<int*> firstneigh(total, nullptr);
      for (int i = lo; i < hi_; ++i) {
        numneigh[i] = static_cast<int>(nbrs[i].size());
        firstneigh[i] = nbrs[i].data();
      }
      std::vector<double> xs(im.x);
      std::vector<double*> xp(total);
      for (int a = 0; a < total; ++a) xp[a] = &xs[3 * a];
      f_acc[t].assign(3 * total, 0.0);
      v_acc[t].assign(9 * total, 0.0);
      e_acc[t].assign(total, 0.0);
      std::vector<double*> fp(total), vp(total);
      for (int a = 0; a < total; ++a) {
        fp[a] = &f_acc[t][3 * a];
        vp[a] = &v_acc[t][9 * a];
      }
      std::vector<int> types(im.type);
      double etot = 0.0, vtot[6] = {0, 0, 0, 0, 0, 0};
      if (!ilist.empty())
        w->compute_for_lammps(n, static_cast<int>(ilist.size()), ilist.data(), numneigh.data(),
                              firstneigh.data(), types.data(), xp.data(), etot, vtot,
                              e_acc[t].data(), fp.data(), vp.data(), 9, 0, h[0], h[4], h[8],
                              h[1], h[2], h[5], "none", n, 0);
    });
  }
  for (auto& th : pool) th.join();
  std::memset(pe, 0, sizeof(double) * n);
  std::memset(force, 0, sizeof(double) * 3 * n);
  std::memset(virial, 0, sizeof(double) * 9 * n);
  for (int t = 0; t < threads; ++t)
    for (int a = 0; a < total; ++a) {
      const int o = im.owner[a];
      pe[o] += e_acc[t][a];
      for (int d = 0; d < 3; ++d) force[d * n + o] += f_acc[t][3 * a + d];
      for (int c = 0; c < 9; ++c) virial[c * n + o] += v_acc[t][9 * a + c];
    }
  return 0;
}

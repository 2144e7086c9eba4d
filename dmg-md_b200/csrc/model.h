// model.h -- NEP potential file (nep.txt) loader and its device image.
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

namespace nepx {

// Host copy of a parsed NEP4 / NEP5 / NEP-ZBL potential.  Field meanings
// follow the reference loader NEP::NEP (src/gpumd_compat/nep.cu:135-415).
struct NepModel {
  int version = 4;                 // 4 or 5
  int num_types = 0;
  std::vector<std::string> symbols;
  int Z[kMaxTypes] = {0};          // atomic numbers (ZBL)
  bool zbl = false, zbl_flexible = false, typewise_zbl = false;
  float zbl_rc_inner = 1.0f, zbl_rc_outer = 2.0f, typewise_factor = 0.0f;
  std::vector<float> zbl_para;     // 10 per type pair (flexible ZBL)
  float rc_radial[kMaxTypes] = {0}, rc_angular[kMaxTypes] = {0};
  float rc_radial_max = 0.0f, rc_max = 0.0f;
  int MN_radial = 0, MN_angular = 0;   // enlarged by 1.25 like the reference
  int n_max_radial = 0, n_max_angular = 0, basis_radial = 0, basis_angular = 0;
  int L_max = 0, num_L = 0, dim = 0, H = 0;
  int has_inv[kMaxInv] = {0};
  // device-layout parameter blocks (float)
  std::vector<float> c_pair;       // [T*T][nR*kR] then [T*T][nA*kA]
  std::vector<float> w0;           // [T][H][dim]
  std::vector<float> b0;           // [T][H]
  std::vector<float> w1;           // [T][H]
  std::vector<float> out_bias;     // [T]: energy -= out_bias[t]
  std::vector<float> q_scaler;     // [dim]
};

// Returns an empty string on success, else the reason.
std::string load_nep(const std::string& path, NepModel& m);

// Kernel-side view (passed by value; pointers are device pointers).
struct ModelParams {
  int version, T, nR, nA, kR, kA, L_max, num_L, dim, H;
  int nlm;            // moment components stored per n: 24 (l_max <= 4) or 80 (l_max 5..8)
  int dimK;           // dim rounded up to 8: row stride of the descriptor and dE/dq buffers
  int num_inv, inv_id[kMaxInv];
  float rc_r[kMaxTypes], rc_a[kMaxTypes];
  // per type pair t1 * T + t2: [0] radial cutoff (rc_r[t1] + rc_r[t2]) / 2,
  // [1] its reciprocal, [2] angular cutoff, [3] its reciprocal, T * T floats
  // each (computed on the host with the same float operations: the kernels'
  // results are unchanged, each edge saves a division)
  const float* pair_cut;
  int zbl, zbl_flexible, typewise_zbl;
  float zbl_rc_inner, zbl_rc_outer, typewise_factor;
  int Z[kMaxTypes];
  const float* c_pair;
  const float* w0;
  const float* w0t;   // [T][dim][H4]: w0 transposed, rows zero-padded
  int H4;
  const float* b0;
  const float* w1;
  const float* out_bias;
  const float* q_scaler;
  const float* zbl_para;
  int num_c_radial;
  // mixed-precision ANN: 16-bit tensor-core operands (set by nepx_set_precision).
  // The hidden units of all types are stacked, m = t H + h, in chunks of 128.
  int tc_dimk;                // dim rounded up to 16 (GEMM1's K)
  int tc_kt;                  // T H rounded up to 128 (GEMM2's K over all chunks)
  int tc_bf16;                // operand format: 0 FP16, 1 BF16
  float tc_sw, tc_sg;         // power-of-two scales of W0 and of w1 (1 - x^2)
  const unsigned short* w0h;  // [T H][tc_dimk] W0 * tc_sw, row m = t H + h
  const unsigned short* w0th; // [dim][tc_kt] W0^T * tc_sw, column m
};

}  // namespace nepx

// model.cu -- NEP potential file loader.
//
// Accepts the GPUMD nep.txt format the reference reads in
// src/gpumd_compat/nep.cu:135-415 (nep4, nep4_zbl, nep5, nep5_zbl; global or
// per-type cutoffs; l_max line with 4 to 8 items) and repacks the flat
// parameter block into the per-type layouts the kernels use.  Malformed input
// returns an error string; the reference exits the process instead.
#include "model.h"

#include <cmath>
#include <fstream>
#include <sstream>

namespace nepx {

namespace {

const char* kElementSymbols[94] = {
  "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S",
  "Cl", "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
  "As", "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd",
  "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd",
  "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg",
  "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu"};

bool next_tokens(std::ifstream& in, std::vector<std::string>& tok)
{
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    tok.clear();
    std::string t;
    while (ss >> t) tok.push_back(t);
    if (!tok.empty()) return true;
  }
  tok.clear();
  return false;
}

bool to_int(const std::string& s, int& v)
{
  char* end = nullptr;
  long x = std::strtol(s.c_str(), &end, 10);
  if (!end || *end) return false;
  v = static_cast<int>(x);
  return true;
}

bool to_double(const std::string& s, double& v)
{
  char* end = nullptr;
  v = std::strtod(s.c_str(), &end);
  return end && !*end && std::isfinite(v);
}

}  // namespace

std::string load_nep(const std::string& path, NepModel& m)
{
  std::ifstream in(path);
  if (!in.is_open()) return "cannot open potential file " + path;
  std::vector<std::string> tok;
  if (!next_tokens(in, tok) || tok.size() < 3) return "first line needs at least 3 items";
  const std::string& kind = tok[0];
  if (kind == "nep4") {
    m.version = 4;
  } else if (kind == "nep4_zbl") {
    m.version = 4;
    m.zbl = true;
  } else if (kind == "nep5") {
    m.version = 5;
  } else if (kind == "nep5_zbl") {
    m.version = 5;
    m.zbl = true;
  } else {
    return "unsupported model '" + kind + "' (nep4, nep4_zbl, nep5, nep5_zbl)";
  }
  if (!to_int(tok[1], m.num_types) || m.num_types < 1 || m.num_types > kMaxTypes)
    return "bad number of types";
  if (static_cast<int>(tok.size()) != 2 + m.num_types)
    return "first line should list " + std::to_string(m.num_types) + " symbols";
  for (int t = 0; t < m.num_types; ++t) {
    m.symbols.push_back(tok[2 + t]);
    m.Z[t] = 0;
    for (int e = 0; e < 94; ++e)
      if (tok[2 + t] == kElementSymbols[e]) m.Z[t] = e + 1;
    if (m.zbl && m.Z[t] == 0) return "unknown element " + tok[2 + t];
  }
  double v;
  if (m.zbl) {
    if (!next_tokens(in, tok) || (tok.size() != 3 && tok.size() != 4))
      return "zbl line should be zbl rc_inner rc_outer [factor]";
    double a, b;
    if (!to_double(tok[1], a) || !to_double(tok[2], b)) return "bad zbl cutoffs";
    m.zbl_rc_inner = static_cast<float>(a);
    m.zbl_rc_outer = static_cast<float>(b);
    if (a == 0 && b == 0) {
      m.zbl_flexible = true;
    } else if (tok.size() == 4) {
      if (!to_double(tok[3], v)) return "bad zbl factor";
      m.typewise_zbl = true;
      m.typewise_factor = static_cast<float>(v);
    }
  }
  if (!next_tokens(in, tok)) return "missing cutoff line";
  const int T = m.num_types;
  if (tok.size() == 5) {
    double a, b;
    if (!to_double(tok[1], a) || !to_double(tok[2], b)) return "bad cutoffs";
    for (int t = 0; t < T; ++t) {
      m.rc_radial[t] = static_cast<float>(a);
      m.rc_angular[t] = static_cast<float>(b);
    }
  } else if (static_cast<int>(tok.size()) == 2 * T + 3) {
    for (int t = 0; t < T; ++t) {
      double a, b;
      if (!to_double(tok[1 + 2 * t], a) || !to_double(tok[2 + 2 * t], b)) return "bad cutoffs";
      m.rc_radial[t] = static_cast<float>(a);
      m.rc_angular[t] = static_cast<float>(b);
    }
  } else {
    return "cutoff line should have 4 or 2*num_types+2 parameters";
  }
  for (int t = 0; t < T; ++t) {
    m.rc_radial_max = std::max(m.rc_radial_max, m.rc_radial[t]);
    m.rc_max = std::max(m.rc_max, std::max(m.rc_radial[t], m.rc_angular[t]));
  }
  int mnr, mna;
  if (!to_int(tok[tok.size() - 2], mnr) || !to_int(tok[tok.size() - 1], mna))
    return "bad MN_radial / MN_angular";
  if (mnr > 819) return "MN_radial exceeds 819";
  m.MN_radial = static_cast<int>(std::ceil(mnr * 1.25));
  m.MN_angular = static_cast<int>(std::ceil(mna * 1.25));
  if (!next_tokens(in, tok) || tok.size() != 3 || !to_int(tok[1], m.n_max_radial) ||
      !to_int(tok[2], m.n_max_angular))
    return "n_max line should be n_max n_max_radial n_max_angular";
  if (!next_tokens(in, tok) || tok.size() != 3 || !to_int(tok[1], m.basis_radial) ||
      !to_int(tok[2], m.basis_angular))
    return "basis_size line should be basis_size radial angular";
  if (m.n_max_radial + 1 > kMaxN || m.n_max_angular + 1 > kMaxN)
    return "n_max above " + std::to_string(kMaxN - 1) + " is not supported";
  if (m.basis_radial + 1 > kMaxBasis || m.basis_angular + 1 > kMaxBasis)
    return "basis_size above 16 is not supported";
  if (!next_tokens(in, tok) || tok.size() < 4 || tok.size() > 8)
    return "l_max line should be l_max L has_q_222 has_q_1111 [has_q_112 ...]";
  if (!to_int(tok[1], m.L_max) || m.L_max < 0) return "bad l_max";
  if (m.L_max > 8) return "l_max above 8 is not supported (the harmonics stop at degree 8)";
  m.num_L = m.L_max;
  for (int k = 0; k < kMaxInv; ++k) {
    int f = 0;
    if (2 + k < static_cast<int>(tok.size()) && !to_int(tok[2 + k], f)) return "bad l_max flag";
    m.has_inv[k] = f ? 1 : 0;
    m.num_L += m.has_inv[k];
  }
  if (!next_tokens(in, tok) || tok.size() != 3 || !to_int(tok[1], m.H) || m.H < 1)
    return "ANN line should be ANN num_neurons 0";
  const int nR = m.n_max_radial + 1, nA = m.n_max_angular + 1;
  const int kR = m.basis_radial + 1, kA = m.basis_angular + 1;
  m.dim = nR + nA * m.num_L;
  if (m.dim > kMaxDim) return "descriptor dimension above 128 is not supported";
  const int H = m.H, dim = m.dim;
  const int num_ann = m.version == 4 ? (dim + 2) * H * T + 1 : ((dim + 2) * H + 1) * T + 1;
  const int num_c_radial = T * T * nR * kR;
  const int num_desc = T * T * (nR * kR + nA * kA);
  const int total = num_ann + num_desc + dim;
  std::vector<double> p(total);
  for (int k = 0; k < total; ++k) {
    if (!next_tokens(in, tok) || !to_double(tok[0], p[k]))
      return "potential file ends or is malformed at parameter " + std::to_string(k);
  }
  if (m.zbl_flexible) {
    const int npair = T * (T + 1) / 2;
    m.zbl_para.resize(10 * npair);
    for (int k = 0; k < 10 * npair; ++k) {
      if (!next_tokens(in, tok) || !to_double(tok[0], v)) return "missing flexible ZBL parameter";
      m.zbl_para[k] = static_cast<float>(v);
    }
  }
  // ANN blocks per type (reference nep.cu:464-496)
  m.w0.resize(static_cast<size_t>(T) * H * dim);
  m.b0.resize(static_cast<size_t>(T) * H);
  m.w1.resize(static_cast<size_t>(T) * H);
  m.out_bias.resize(T);
  size_t off = 0;
  std::vector<double> extra_bias(T, 0.0);
  for (int t = 0; t < T; ++t) {
    for (int k = 0; k < H * dim; ++k) m.w0[static_cast<size_t>(t) * H * dim + k] = static_cast<float>(p[off + k]);
    off += static_cast<size_t>(H) * dim;
    for (int k = 0; k < H; ++k) m.b0[static_cast<size_t>(t) * H + k] = static_cast<float>(p[off + k]);
    off += H;
    for (int k = 0; k < H; ++k) m.w1[static_cast<size_t>(t) * H + k] = static_cast<float>(p[off + k]);
    off += H;
    if (m.version == 5) extra_bias[t] = p[off++];
  }
  const double b1 = p[off++];
  for (int t = 0; t < T; ++t) {
    // NEP4: E -= b1; NEP5: E -= w1[H] + b1, both in float like the reference
    m.out_bias[t] = m.version == 5 ? static_cast<float>(extra_bias[t]) + static_cast<float>(b1)
                                   : static_cast<float>(b1);
  }
  // descriptor coefficients: file basis-major -> type-pair major (nep.cu:103-126)
  m.c_pair.resize(num_desc);
  for (int tp = 0; tp < T * T; ++tp) {
    for (int b = 0; b < nR * kR; ++b)
      m.c_pair[static_cast<size_t>(tp) * nR * kR + b] = static_cast<float>(p[num_ann + static_cast<size_t>(b) * T * T + tp]);
    for (int b = 0; b < nA * kA; ++b)
      m.c_pair[num_c_radial + static_cast<size_t>(tp) * nA * kA + b] =
        static_cast<float>(p[num_ann + num_c_radial + static_cast<size_t>(b) * T * T + tp]);
  }
  m.q_scaler.resize(dim);
  for (int d = 0; d < dim; ++d) m.q_scaler[d] = static_cast<float>(p[num_ann + num_desc + d]);
  return "";
}

}  // namespace nepx

// run_input.cpp -- run.in / model.xyz / nep.txt-header parsing for nepx-md.
#include "run_input.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <unordered_set>

namespace nepx_run {

std::string InputError::describe() const
{
  std::ostringstream o;
  if (!source.file.empty()) {
    o << source.file;
    if (source.line) o << ":" << source.line;
    o << ": ";
  }
  o << what();
  if (!source.text.empty()) o << "\n    " << source.text;
  return o.str();
}

std::vector<std::string> tokens(const std::string& line)
{
  std::istringstream in(line);
  std::vector<std::string> out;
  std::string t;
  while (in >> t) out.push_back(t);
  return out;
}

namespace {

[[noreturn]] void fail(const Source& s, const std::string& msg) { throw InputError(s, msg); }

int to_int(const std::string& tok, const Source& s, const std::string& name)
{
  char* end = nullptr;
  errno = 0;
  const long v = std::strtol(tok.c_str(), &end, 0);
  if (errno || end == tok.c_str() || *end != '\0' || v < INT_MIN || v > INT_MAX)
    fail(s, name + " should be an integer");
  return static_cast<int>(v);
}

double to_real(const std::string& tok, const Source& s, const std::string& name)
{
  char* end = nullptr;
  errno = 0;
  const double v = std::strtod(tok.c_str(), &end);
  if (errno || end == tok.c_str() || *end != '\0' || !std::isfinite(v))
    fail(s, name + " should be a finite real number");
  return v;
}

void need(const std::vector<std::string>& t, size_t n, const Source& s, const std::string& msg)
{
  if (t.size() != n) fail(s, msg);
}

[[noreturn]] void unsupported(const Source& s, const std::string& what)
{
  fail(s, "unsupported command '" + what + "'");
}

DumpXyzCmd dump_xyz(const std::vector<std::string>& t, const Source& s)
{
  if (t.size() < 3) fail(s, "dump_xyz should have at least 2 parameters");
  DumpXyzCmd c;
  c.interval = to_int(t[1], s, "dump interval");
  if (c.interval <= 0) fail(s, "dump interval should be > 0");
  c.file = t[2];
  bool group_seen = false, precision_seen = false;
  for (size_t k = 3; k < t.size(); ++k) {
    const std::string& w = t[k];
    if (w == "group") {
      if (group_seen) fail(s, "option 'group' is specified more than once in dump_xyz");
      if (k + 2 >= t.size()) fail(s, "option 'group' requires a grouping method and group ID");
      c.grouping = to_int(t[k + 1], s, "grouping method");
      c.group_id = to_int(t[k + 2], s, "group ID");
      if (*c.grouping < 0 || *c.group_id < 0)
        fail(s, "grouping method and group ID should be >= 0");
      group_seen = true;
      k += 2;
    } else if (w == "precision") {
      if (precision_seen) fail(s, "option 'precision' is specified more than once in dump_xyz");
      if (k + 1 >= t.size()) fail(s, "option 'precision' requires single or double");
      if (t[k + 1] == "single") c.double_precision = false;
      else if (t[k + 1] == "double") c.double_precision = true;
      else fail(s, "invalid dump_xyz precision '" + t[k + 1] + "'");
      precision_seen = true;
      ++k;
    } else if (w == "mass") c.mass = true;
    else if (w == "charge") c.charge = true;
    else if (w == "velocity") c.velocity = true;
    else if (w == "force") c.force = true;
    else if (w == "potential") c.potential = true;
    else if (w == "unwrapped_position") c.unwrapped = true;
    else if (w == "virial") c.virial = true;
    else if (w == "group_labels") c.group_labels = true;
    else if (w == "bec") unsupported(s, "dump_xyz bec");
    else fail(s, "unrecognized dump_xyz argument '" + w + "'");
  }
  return c;
}

EnsembleCmd ensemble(const std::vector<std::string>& t, const Source& s)
{
  if (t.size() < 2) fail(s, "ensemble type is missing");
  EnsembleCmd c;
  const std::string& name = t[1];
  if (name == "nve") {
    need(t, 2, s, "ensemble nve should have 0 parameters");
    return c;
  }
  if (name == "npt_ber" || name == "npt_scr") {
    // the reference's isotropic 8-token form, plus GPUMD's anisotropic
    // (Pxx Pyy Pzz Cxx Cyy Czz) and triclinic (Pxx Pyy Pzz Pyz Pxz Pxy, six
    // moduli) forms, which the reference rejects
    if (t.size() > 8 && t.size() != 12 && t.size() != 18)
      fail(s, name + ": v1 supports isotropic 8-token syntax only (and the anisotropic 12-token "
                     "and triclinic 18-token forms of this engine)");
    need(t, t.size() > 8 ? t.size() : 8, s,
         "ensemble " + name + " should have 6 parameters (isotropic 8-token syntax)");
    c.kind = name == "npt_ber" ? Ensemble::npt_ber : Ensemble::npt_scr;
    c.T0 = to_real(t[2], s, "initial temperature");
    c.T1 = to_real(t[3], s, "final temperature");
    c.Tdamp = to_real(t[4], s, "temperature coupling");
    if (t.size() == 8) {
      c.p_gpa = to_real(t[5], s, "target pressure (GPa)");
      c.bulk_gpa = to_real(t[6], s, "bulk modulus (GPa)");
    } else {
      const int nc = t.size() == 12 ? 3 : 6;
      c.baro = nc == 3 ? 1 : 2;
      for (int k = 0; k < nc; ++k) {
        c.p6_gpa[k] = to_real(t[5 + k], s, "target pressure component (GPa)");
        c.c6_gpa[k] = to_real(t[5 + nc + k], s, "elastic modulus component (GPa)");
        if (c.c6_gpa[k] <= 0.0) fail(s, "elastic moduli should be > 0");
      }
      // the isotropic fields stay valid for the ensemble call
      c.p_gpa = (c.p6_gpa[0] + c.p6_gpa[1] + c.p6_gpa[2]) / 3.0;
      c.bulk_gpa = c.c6_gpa[0];
    }
    c.tau_p = to_real(t.back(), s, "pressure coupling time");
    if (c.T0 <= 0.0 || c.T1 <= 0.0) fail(s, "initial and final temperatures should be > 0");
    if (c.Tdamp < 1.0) fail(s, "temperature coupling should be >= 1");
    if (c.bulk_gpa <= 0.0) fail(s, "bulk modulus should be > 0");
    if (c.tau_p < 1.0) fail(s, "pressure coupling time should be >= 1");
    return c;
  }
  if (name == "nvt_ber" || name == "nvt_nhc" || name == "nvt_bdp") {
    need(t, 5, s, "ensemble " + name + " should have 3 parameters");
    c.kind = name == "nvt_ber" ? Ensemble::nvt_ber
             : name == "nvt_nhc" ? Ensemble::nvt_nhc : Ensemble::nvt_bdp;
    c.T0 = to_real(t[2], s, "initial temperature");
    c.T1 = to_real(t[3], s, "final temperature");
    c.Tdamp = to_real(t[4], s, "temperature coupling");
    if (c.T0 <= 0.0 || c.T1 <= 0.0) fail(s, "initial and final temperatures should be > 0");
    if (c.Tdamp < 1.0) fail(s, "temperature coupling should be >= 1");
    return c;
  }
  fail(s, "unsupported command 'ensemble " + name + "' in the current version");
}

CommandData command(const std::vector<std::string>& t, const Source& s)
{
  const std::string& key = t.front();
  if (key == "potential") {
    if (t.size() == 3) unsupported(s, "potential partition direction");
    need(t, 2, s, "potential should have 1 parameter");
    return PotentialCmd{t[1]};
  }
  if (key == "velocity") {
    if (t.size() != 2 && t.size() != 4) fail(s, "velocity should have 1 or 3 parameters");
    VelocityCmd c;
    c.temperature = to_real(t[1], s, "initial temperature");
    if (c.temperature <= 0.0) fail(s, "initial temperature should be > 0");
    if (t.size() == 4) c.seed = to_int(t[3], s, "seed");
    return c;
  }
  if (key == "time_step") {
    if (t.size() != 2 && t.size() != 3) fail(s, "time_step should have 1 or 2 parameters");
    TimeStepCmd c;
    c.fs = to_real(t[1], s, "time_step");
    if (t.size() == 3) {
      const double v = to_real(t[2], s, "maximum distance per step");
      if (v <= 0.0) fail(s, "maximum distance per step should be > 0");
      c.max_distance = v;
    }
    return c;
  }
  if (key == "ensemble") return ensemble(t, s);
  if (key == "correct_velocity") {
    if (t.size() != 2 && t.size() != 3) fail(s, "correct_velocity should have 1 or 2 parameters");
    CorrectVelocityCmd c;
    c.interval = to_int(t[1], s, "velocity correction interval");
    if (c.interval < 10) fail(s, "velocity correction interval should be >= 10");
    if (t.size() == 3) {
      c.grouping = to_int(t[2], s, "velocity correction grouping method");
      if (*c.grouping < 0) fail(s, "velocity correction grouping method should be >= 0");
    }
    return c;
  }
  if (key == "dump_thermo") {
    need(t, 2, s, "dump_thermo should have 1 parameter");
    const int v = to_int(t[1], s, "thermo dump interval");
    if (v <= 0) fail(s, "thermo dump interval should be > 0");
    return DumpThermoCmd{v};
  }
  if (key == "dump_xyz") return dump_xyz(t, s);
  if (key == "dump_restart") {
    need(t, 2, s, "dump_restart should have 1 parameter");
    const int v = to_int(t[1], s, "restart dump interval");
    if (v <= 0) fail(s, "restart dump interval should be > 0");
    return DumpRestartCmd{v};
  }
  if (key == "run") {
    need(t, 2, s, "run should have 1 parameter");
    return RunCmd{to_int(t[1], s, "number of steps")};
  }
  // GPUMD commands outside the NEP MD path, rejected by name
  static const std::unordered_set<std::string> known = {
    "active", "add_efield", "add_force", "add_random_force", "add_spring", "change_box",
    "compute", "compute_adf", "compute_angular_rdf", "compute_chunk", "compute_cohesive",
    "compute_dos", "compute_dpdt", "compute_elastic", "compute_es", "compute_extrapolation",
    "compute_gkma", "compute_hac", "compute_hnema", "compute_hnemd", "compute_hnemdec",
    "compute_ic", "compute_lsqt", "compute_msd", "compute_orientorder", "compute_phonon",
    "compute_rdf", "compute_sdc", "compute_shc", "compute_viscosity", "deform", "dftd3",
    "dump_beads", "dump_cg", "dump_dipole", "dump_exyz", "dump_force", "dump_netcdf",
    "dump_observer", "dump_polarizability", "dump_position", "dump_shock_nemd",
    "dump_velocity", "electron_stop", "fix", "kspace", "mc", "minimize", "move", "neighbor",
    "plumed", "replicate"};
  if (known.count(key)) unsupported(s, key);
  unsupported(s, key + " (unknown)");
}

}  // namespace

std::vector<Command> parse_run_file(const std::string& path)
{
  std::ifstream in(path);
  if (!in) throw InputError(Source{path, 0, {}}, "cannot open run.in");
  std::vector<Command> program;
  std::string line;
  size_t no = 0;
  while (std::getline(in, line)) {
    ++no;
    std::vector<std::string> t;
    for (std::string& w : tokens(line)) {
      if (!w.empty() && w.front() == '#') break;   // a comment runs to the end of the line
      t.push_back(std::move(w));
    }
    if (t.empty()) continue;
    const Source s{path, no, line};
    if (t.size() > 32) fail(s, "the number of tokens should be <= 32");
    program.push_back(Command{s, command(t, s)});
  }
  return program;
}

void validate_program(const std::vector<Command>& program)
{
  Ensemble selected = Ensemble::nve;
  bool adaptive = false, correction = false;
  double dt = 1.0;
  for (const Command& c : program) {
    if (const auto* ts = std::get_if<TimeStepCmd>(&c.data)) {
      adaptive = ts->max_distance.has_value();
      dt = ts->fs;
    }
    if (std::holds_alternative<CorrectVelocityCmd>(c.data)) correction = true;
    if (std::holds_alternative<RunCmd>(c.data)) {
      const bool npt = selected == Ensemble::npt_ber || selected == Ensemble::npt_scr;
      const std::string npt_name = selected == Ensemble::npt_ber ? "npt_ber" : "npt_scr";
      if (npt && correction)
        fail(c.source, "ensemble " + npt_name + " does not support correct_velocity");
      if (npt && adaptive)
        fail(c.source, "ensemble " + npt_name + " does not support adaptive time_step");
      if (npt && !(std::isfinite(dt) && dt > 0.0))
        fail(c.source, "ensemble " + npt_name + " requires a finite positive time_step");
      if (selected == Ensemble::nvt_nhc || selected == Ensemble::nvt_bdp) {
        const std::string name = selected == Ensemble::nvt_nhc ? "nvt_nhc" : "nvt_bdp";
        if (correction) fail(c.source, "ensemble " + name + " does not support correct_velocity");
        if (adaptive) fail(c.source, "ensemble " + name + " does not support adaptive time_step");
        if (!(std::isfinite(dt) && dt > 0.0))
          fail(c.source, "ensemble " + name + " requires a finite positive time_step");
      }
      correction = false;
      adaptive = false;
    }
    if (const auto* e = std::get_if<EnsembleCmd>(&c.data)) selected = e->kind;
  }
}

// ---- nep.txt header --------------------------------------------------------------

PotentialHeader read_potential_header(const std::string& path)
{
  std::ifstream in(path);
  std::string line;
  if (!in || !std::getline(in, line))
    throw InputError(Source{path, 1, {}}, "cannot open or read potential file");
  const auto t = tokens(line);
  const Source s{path, 1, line};
  if (t.size() < 3) fail(s, "potential header should have at least 3 items");
  if (t[0] != "nep4" && t[0] != "nep5" && t[0] != "nep4_zbl" && t[0] != "nep5_zbl")
    fail(s, "unsupported NEP model '" + t[0] + "'");
  const int types = to_int(t[1], s, "number of atom types");
  if (types <= 0 || t.size() != static_cast<size_t>(types + 2))
    fail(s, "potential header atom-symbol count mismatch");
  return PotentialHeader{t[0], std::vector<std::string>(t.begin() + 2, t.end())};
}

// ---- model.xyz -------------------------------------------------------------------

namespace {

// Standard atomic weights (u) of H..Lr, GPUMD's default masses when
// model.xyz has no mass column.
const char* const kMassTable =
  "H 1.008 He 4.002602 Li 6.94 Be 9.0121831 B 10.81 C 12.011 N 14.007 O 15.999 "
  "F 18.998403163 Ne 20.1797 Na 22.98976928 Mg 24.305 Al 26.9815385 Si 28.085 "
  "P 30.973761998 S 32.06 Cl 35.45 Ar 39.948 K 39.0983 Ca 40.078 Sc 44.955908 Ti 47.867 "
  "V 50.9415 Cr 51.9961 Mn 54.938044 Fe 55.845 Co 58.933194 Ni 58.6934 Cu 63.546 Zn 65.38 "
  "Ga 69.723 Ge 72.63 As 74.921595 Se 78.971 Br 79.904 Kr 83.798 Rb 85.4678 Sr 87.62 "
  "Y 88.90584 Zr 91.224 Nb 92.90637 Mo 95.95 Tc 98 Ru 101.07 Rh 102.9055 Pd 106.42 "
  "Ag 107.8682 Cd 112.414 In 114.818 Sn 118.71 Sb 121.76 Te 127.6 I 126.90447 Xe 131.293 "
  "Cs 132.90545196 Ba 137.327 La 138.90547 Ce 140.116 Pr 140.90766 Nd 144.242 Pm 145 "
  "Sm 150.36 Eu 151.964 Gd 157.25 Tb 158.92535 Dy 162.5 Ho 164.93033 Er 167.259 "
  "Tm 168.93422 Yb 173.045 Lu 174.9668 Hf 178.49 Ta 180.94788 W 183.84 Re 186.207 "
  "Os 190.23 Ir 192.217 Pt 195.084 Au 196.96657 Hg 200.592 Tl 204.38 Pb 207.2 "
  "Bi 208.9804 Po 210 At 210 Rn 222 Fr 223 Ra 226 Ac 227 Th 232.0377 Pa 231.03588 "
  "U 238.02891 Np 237 Pu 244 Am 243 Cm 247 Bk 247 Cf 251 Es 252 Fm 257 Md 258 No 259 Lr 262";

bool default_mass(const std::string& symbol, double& mass)
{
  const auto t = tokens(kMassTable);
  for (size_t k = 0; k + 1 < t.size(); k += 2)
    if (t[k] == symbol) {
      mass = std::strtod(t[k + 1].c_str(), nullptr);
      return true;
    }
  return false;
}

std::string lower(std::string v)
{
  for (char& c : v) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return v;
}

// value of key=... on the comment line (case-insensitive key, optional
// spaces around '=', double-quoted or bare value); empty when absent
std::string keyed(const std::string& line, const std::string& key, const Source& s)
{
  const std::string low = lower(line), k = lower(key);
  size_t at = low.find(k + "=");
  if (at == std::string::npos) {
    at = low.find(k);
    if (at == std::string::npos) return {};
    size_t c = at + k.size();
    while (c < line.size() && std::isspace(static_cast<unsigned char>(line[c]))) ++c;
    if (c >= line.size() || line[c] != '=') return {};
    at = c;
  } else {
    at += k.size();
  }
  size_t c = at + 1;
  while (c < line.size() && std::isspace(static_cast<unsigned char>(line[c]))) ++c;
  if (c >= line.size()) return {};
  if (line[c] == '"') {
    const size_t end = line.find('"', c + 1);
    if (end == std::string::npos) fail(s, "unterminated quoted value for " + key);
    return line.substr(c + 1, end - c - 1);
  }
  const size_t end = line.find_first_of(" \t\r\n", c);
  return line.substr(c, end == std::string::npos ? std::string::npos : end - c);
}

struct Column {
  std::string name;
  char type;
  int width;
  size_t offset;
};

}  // namespace

Model parse_model_file(const std::string& path, const PotentialHeader& pot)
{
  std::ifstream in(path);
  if (!in) throw InputError(Source{path, 0, {}}, "cannot open model.xyz");
  std::string l1, l2;
  if (!std::getline(in, l1) || !std::getline(in, l2))
    fail(Source{path, 1, l1}, "model.xyz should contain at least two lines");
  const auto c1 = tokens(l1);
  const Source s1{path, 1, l1}, s2{path, 2, l2};
  if (c1.size() != 1) fail(s1, "the first line should have one value");
  const int n = to_int(c1[0], s1, "number of atoms");
  if (n < 2) fail(s1, "number of atoms should be >= 2");
  Model m;
  m.n = n;
  const std::string pbc = keyed(l2, "pbc", s2);
  if (!pbc.empty()) {
    const auto f = tokens(pbc);
    if (f.size() != 3) fail(s2, "pbc should contain three T/F values");
    for (int d = 0; d < 3; ++d) {
      const std::string v = lower(f[d]);
      if (v != "t" && v != "f") fail(s2, "pbc should contain only T or F");
      m.pbc[d] = v == "t";
    }
  }
  const auto lat = tokens(keyed(l2, "lattice", s2));
  if (lat.size() != 9) fail(s2, "Lattice should contain nine values");
  // Lattice lists a, b, c; h holds them as columns
  for (int k = 0; k < 9; ++k) m.h[(k % 3) * 3 + k / 3] = to_real(lat[k], s2, "lattice value");
  // Properties=name:type:width triples
  const std::string schema = lower(keyed(l2, "properties", s2));
  std::vector<std::string> parts;
  for (size_t a = 0;;) {
    const size_t b = schema.find(':', a);
    parts.push_back(schema.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  if (parts.empty() || parts.size() % 3) fail(s2, "Properties should contain name:type:width triples");
  std::vector<Column> cols;
  size_t offset = 0;
  for (size_t k = 0; k < parts.size(); k += 3) {
    const int w = to_int(parts[k + 2], s2, "property width");
    if (w <= 0 || parts[k + 1].empty()) fail(s2, "property width should be > 0");
    cols.push_back(Column{parts[k], parts[k + 1][0], w, offset});
    offset += w;
  }
  auto col = [&cols](const char* name) -> const Column* {
    for (const Column& c : cols)
      if (c.name == name) return &c;
    return nullptr;
  };
  const Column *sp = col("species"), *ps = col("pos"), *ms = col("mass"), *vl = col("vel"),
               *gr = col("group");
  if (!sp || !ps) fail(s2, "Properties should contain species and pos");
  m.species.resize(n);
  m.type.resize(n);
  m.mass.resize(n);
  m.pos.assign(3 * static_cast<size_t>(n), 0.0);
  m.vel.assign(3 * static_cast<size_t>(n), 0.0);
  m.has_velocity = vl != nullptr;
  if (gr) m.groups.assign(gr->width, std::vector<int>(n));
  for (int a = 0; a < n; ++a) {
    std::string line;
    if (!std::getline(in, line))
      fail(Source{path, static_cast<size_t>(a) + 3, {}}, "model.xyz has fewer atom lines than declared");
    const Source s{path, static_cast<size_t>(a) + 3, line};
    const auto t = tokens(line);
    if (t.size() != offset) fail(s, "number of columns does not match Properties");
    m.species[a] = t[sp->offset];
    const auto it = std::find(pot.symbols.begin(), pot.symbols.end(), m.species[a]);
    if (it == pot.symbols.end())
      fail(s, "species '" + m.species[a] + "' is not allowed by the potential");
    m.type[a] = static_cast<int>(it - pot.symbols.begin());
    for (int d = 0; d < 3; ++d)
      m.pos[static_cast<size_t>(d) * n + a] = to_real(t[ps->offset + d], s, "position");
    if (ms) {
      m.mass[a] = to_real(t[ms->offset], s, "atom mass");
    } else if (!default_mass(m.species[a], m.mass[a])) {
      fail(s, "no GPUMD default mass for species '" + m.species[a] + "'");
    }
    if (m.mass[a] <= 0.0) fail(s, "atom mass should be > 0");
    if (vl)
      for (int d = 0; d < 3; ++d)
        m.vel[static_cast<size_t>(d) * n + a] = to_real(t[vl->offset + d], s, "velocity");
    if (gr)
      for (int g = 0; g < gr->width; ++g) {
        const int label = to_int(t[gr->offset + g], s, "group label");
        if (label < 0 || label >= n) fail(s, "group label should be >= 0 and < N");
        m.groups[g][a] = label;
      }
  }
  return m;
}

}  // namespace nepx_run

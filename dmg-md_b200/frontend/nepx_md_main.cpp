// nepx_md_main.cpp -- nepx-md: a GPUMD-format MD job on one GPU.
//
// Reads run.in, model.xyz and the potential named by run.in from the working
// directory, as the reference's dmg-md does (src/dmgmd_main.cpp:29-90), and
// runs each `run` segment through the nepx C ABI (include/nepx.h):
// velocity Verlet with the selected ensemble on the GPU, outputs written by
// the host between steps.  Outputs follow the reference's writers
// (src/runtime.cu:1139-1313): thermo.out (a header per segment, one row per
// dump_thermo interval), dump_xyz files (appended; a trailing '*' in the name
// writes one file per output step) and restart.xyz (rewritten).
//
//   nepx-md                     run the job in the working directory
//   nepx-md --precision mixed   the ANN on the tensor cores (FP16; mixed_bf16: BF16)
//   nepx-md --check             parse and validate the inputs only (no GPU)
//
// The ensemble RNG seed is DMGMD_ENSEMBLE_SEED when set (decimal), else
// 12345678, restarted for every segment (reference runtime.cu:705-709).
#include <algorithm>
#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <numeric>
#include <optional>
#include <string>
#include <vector>

#include "../../include/nepx.h"
#include "run_input.h"

using namespace nepx_run;

namespace {

constexpr double kTimeUnit = 10.18051;       // fs per natural time unit
constexpr double kBoltzmann = 8.617343e-5;   // eV/K
constexpr double kPressureUnit = 160.2177;   // GPa per eV/A^3

struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(int rc, const char* what, const char* message)
{
  if (rc) throw Failure(std::string(what) + ": " + (message ? message : "error"));
}

// ---- velocities (reference runtime.cu:1002-1109) ---------------------------------

// Removes the linear momentum of the atoms `idx`, then their rigid rotation
// about their center of mass (angular momentum over the inertia tensor):
// the reference's correct_velocity_subset (runtime.cu:979-1063).
void correct_subset(const std::vector<double>& mass, const std::vector<double>& pos,
                    std::vector<double>& vel, const std::vector<size_t>& idx)
{
  if (idx.empty()) return;
  const size_t n = mass.size();
  double M = 0.0, p[3] = {0, 0, 0};
  for (size_t a : idx) {
    M += mass[a];
    for (int d = 0; d < 3; ++d) p[d] += mass[a] * vel[d * n + a];
  }
  if (M == 0.0) return;
  for (int d = 0; d < 3; ++d) p[d] /= M;
  for (size_t a : idx)
    for (int d = 0; d < 3; ++d) vel[d * n + a] -= p[d];
  double c[3] = {0, 0, 0};
  for (size_t a : idx)
    for (int d = 0; d < 3; ++d) c[d] += pos[d * n + a] * mass[a];
  for (double& v : c) v /= M;
  double L[3] = {0, 0, 0}, I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (size_t a : idx) {
    const double x = pos[a] - c[0], y = pos[n + a] - c[1], z = pos[2 * n + a] - c[2];
    const double vx = vel[a], vy = vel[n + a], vz = vel[2 * n + a], m = mass[a];
    L[0] += m * (y * vz - z * vy);
    L[1] += m * (z * vx - x * vz);
    L[2] += m * (x * vy - y * vx);
    I[0][0] += m * (y * y + z * z);
    I[1][1] += m * (x * x + z * z);
    I[2][2] += m * (x * x + y * y);
    I[0][1] -= m * x * y;
    I[1][2] -= m * y * z;
    I[0][2] -= m * x * z;
  }
  I[1][0] = I[0][1];
  I[2][1] = I[1][2];
  I[2][0] = I[0][2];
  const double det = I[0][0] * I[1][1] * I[2][2] + I[0][1] * I[1][2] * I[2][0] +
                     I[0][2] * I[1][0] * I[2][1] - I[0][0] * I[1][2] * I[2][1] -
                     I[0][1] * I[1][0] * I[2][2] - I[2][0] * I[1][1] * I[0][2];
  if (std::fabs(det) < 1.0e-10) return;
  // adjugate of I
  const double A[3][3] = {
    {I[1][1] * I[2][2] - I[1][2] * I[2][1], -(I[0][1] * I[2][2] - I[0][2] * I[2][1]),
     I[0][1] * I[1][2] - I[0][2] * I[1][1]},
    {-(I[1][0] * I[2][2] - I[1][2] * I[2][0]), I[0][0] * I[2][2] - I[0][2] * I[2][0],
     -(I[0][0] * I[1][2] - I[0][2] * I[1][0])},
    {I[1][0] * I[2][1] - I[1][1] * I[2][0], -(I[0][0] * I[2][1] - I[0][1] * I[2][0]),
     I[0][0] * I[1][1] - I[0][1] * I[1][0]}};
  double w[3] = {0, 0, 0};
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) w[r] += A[r][k] / det * L[k];
  for (size_t a : idx) {
    const double x = pos[a] - c[0], y = pos[n + a] - c[1], z = pos[2 * n + a] - c[2];
    vel[a] -= w[1] * z - w[2] * y;
    vel[n + a] -= w[2] * x - w[0] * z;
    vel[2 * n + a] -= w[0] * y - w[1] * x;
  }
}

void zero_momenta(const std::vector<double>& mass, const std::vector<double>& pos,
                  std::vector<double>& vel)
{
  std::vector<size_t> all(mass.size());
  std::iota(all.begin(), all.end(), size_t(0));
  correct_subset(mass, pos, vel, all);
}

// correct_velocity: every atom at once, or each group of one grouping method
// of model.xyz in turn (reference correct_device_velocity, runtime.cu:620-655).
void correct_velocity(const Model& m, const CorrectVelocityCmd& c, const std::vector<double>& pos,
                      std::vector<double>& vel)
{
  if (!c.grouping) {
    zero_momenta(m.mass, pos, vel);
    return;
  }
  if (*c.grouping >= static_cast<int>(m.groups.size()))
    throw std::runtime_error("correct_velocity grouping method is out of range");
  const std::vector<int>& label = m.groups[*c.grouping];
  int top = -1;
  for (int g : label) top = std::max(top, g);
  for (int g = 0; g <= top; ++g) {
    std::vector<size_t> subset;
    for (size_t a = 0; a < label.size(); ++a)
      if (label[a] == g) subset.push_back(a);
    correct_subset(m.mass, pos, vel, subset);
  }
}

// Uniform random components (libc rand; per-component srand(seed + 3 id +
// axis) when seeded), zero momenta, scaled to T.  Velocities in A/fs.
void random_velocities(const Model& m, double T, const int* seed, std::vector<double>& vel)
{
  const size_t n = m.n;
  vel.assign(3 * n, 0.0);
  for (size_t a = 0; a < n; ++a)
    for (int d = 0; d < 3; ++d) {
      if (seed) std::srand(static_cast<unsigned>(*seed + static_cast<int>(a) * 3 + d));
      vel[d * n + a] = -1.0 + (std::rand() * 2.0) / static_cast<double>(RAND_MAX);
    }
  zero_momenta(m.mass, m.pos, vel);
  double t = 0.0;
  for (size_t a = 0; a < n; ++a)
    t += m.mass[a] * (vel[a] * vel[a] + vel[n + a] * vel[n + a] + vel[2 * n + a] * vel[2 * n + a]);
  t /= 3.0 * kBoltzmann * static_cast<double>(n);
  const double f = std::sqrt(T / t);
  for (double& v : vel) v *= f / kTimeUnit;   // natural units -> A/fs
}

// ---- writers (reference runtime.cu:1139-1313) --------------------------------------

struct State {
  std::vector<double> pos, vel, force, pe, virial;
  std::vector<double> unwrapped;   // when a dump_xyz asks for unwrapped_position
  nepx_box box;
};

void print_tensor(FILE* f, const char* name, const char* fmt, const double* t)
{
  std::fprintf(f, " %s=\"", name);
  for (int k = 0; k < 9; ++k) std::fprintf(f, k == 0 ? fmt + 1 : fmt, t[k]);
  std::fprintf(f, "\"");
}

void write_thermo_header(FILE* f, int interval, int n, double dt_fs)
{
  std::fprintf(f, "# dump_thermo %d\n", interval);
  std::fprintf(f, "# format_version 1\n");
  std::fprintf(f, "# num_atoms %d\n", n);
  std::fprintf(f, "# dt_output %.10e fs\n", dt_fs * interval);
  std::fprintf(f, "# columns T KE PE sxx syy szz syz sxz sxy ax ay az bx by bz cx cy cz\n");
}

void write_thermo_row(FILE* f, const double* row)
{
  for (int k = 0; k < 18; ++k) std::fprintf(f, "%20.10e", row[k]);
  std::fprintf(f, "\n");
  std::fflush(f);
}

void write_xyz(const DumpXyzCmd& c, int step, double time_fs, const Model& m, const State& s,
               const double* thermo)
{
  std::string name = c.file;
  const bool separated = !name.empty() && name.back() == '*';
  if (separated) {
    name.pop_back();
    name += std::to_string(step + 1);
  }
  FILE* f = std::fopen(name.c_str(), separated ? "w" : "a");
  if (!f) throw Failure("cannot open dump_xyz output '" + name + "'");
  const char* fmt = c.double_precision ? " %.17g" : " %.9g";
  const size_t n = m.n;
  std::vector<size_t> order;
  for (size_t a = 0; a < n; ++a) {
    if (c.grouping) {
      if (*c.grouping >= static_cast<int>(m.groups.size()))
        throw Failure("dump_xyz grouping method is out of range");
      if (m.groups[*c.grouping][a] != *c.group_id) continue;
    }
    order.push_back(a);
  }
  std::fprintf(f, "%zu\n", order.size());
  std::fprintf(f, "Time=%.8f", time_fs);
  std::fprintf(f, " pbc=\"%c %c %c\"", s.box.pbc[0] ? 'T' : 'F', s.box.pbc[1] ? 'T' : 'F',
               s.box.pbc[2] ? 'T' : 'F');
  const double* h = s.box.h;
  const double lattice[9] = {h[0], h[3], h[6], h[1], h[4], h[7], h[2], h[5], h[8]};
  print_tensor(f, "Lattice", fmt, lattice);
  double pe = 0.0;
  for (size_t a = 0; a < n; ++a) pe += s.pe[a];
  std::fprintf(f, " energy=");
  std::fprintf(f, fmt + 1, pe);
  double w[6] = {0, 0, 0, 0, 0, 0};
  for (size_t a = 0; a < n; ++a)
    for (int k = 0; k < 6; ++k) w[k] += s.virial[k * n + a];
  const double vir[9] = {w[0], w[3], w[4], w[3], w[1], w[5], w[4], w[5], w[2]};
  print_tensor(f, "virial", fmt, vir);
  // thermo row stresses (GPa, order sxx syy szz syz sxz sxy) back to eV/A^3
  const double sxx = thermo[3] / kPressureUnit, syy = thermo[4] / kPressureUnit,
               szz = thermo[5] / kPressureUnit, syz = thermo[6] / kPressureUnit,
               sxz = thermo[7] / kPressureUnit, sxy = thermo[8] / kPressureUnit;
  const double stress[9] = {sxx, sxy, sxz, sxy, syy, syz, sxz, syz, szz};
  print_tensor(f, "stress", fmt, stress);
  std::fprintf(f, " Properties=species:S:1:pos:R:3");
  if (c.mass) std::fprintf(f, ":mass:R:1");
  if (c.charge) std::fprintf(f, ":charge:R:1");
  if (c.velocity) std::fprintf(f, ":vel:R:3");
  if (c.force) std::fprintf(f, ":forces:R:3");
  if (c.potential) std::fprintf(f, ":energy_atom:R:1");
  if (c.unwrapped) std::fprintf(f, ":unwrapped_position:R:3");
  if (c.virial) std::fprintf(f, ":virial:R:9");
  if (c.group_labels) std::fprintf(f, ":group:I:%zu", m.groups.size());
  std::fprintf(f, "\n");
  const int rowmajor[9] = {0, 3, 4, 6, 1, 5, 7, 8, 2};
  for (size_t a : order) {
    std::fprintf(f, "%s", m.species[a].c_str());
    for (int d = 0; d < 3; ++d) std::fprintf(f, fmt, s.pos[d * n + a]);
    if (c.mass) std::fprintf(f, fmt, m.mass[a]);
    if (c.charge) std::fprintf(f, fmt, 0.0);
    if (c.velocity)
      for (int d = 0; d < 3; ++d) std::fprintf(f, fmt, s.vel[d * n + a]);
    if (c.force)
      for (int d = 0; d < 3; ++d) std::fprintf(f, fmt, s.force[d * n + a]);
    if (c.potential) std::fprintf(f, fmt, s.pe[a]);
    if (c.unwrapped)
      for (int d = 0; d < 3; ++d) std::fprintf(f, fmt, s.unwrapped[d * n + a]);
    if (c.virial)
      for (int k : rowmajor) std::fprintf(f, fmt, s.virial[k * n + a]);
    if (c.group_labels)
      for (const auto& g : m.groups) std::fprintf(f, " %d", g[a]);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}

void write_restart(const Model& m, const State& s)
{
  FILE* f = std::fopen("restart.xyz", "w");
  if (!f) throw Failure("cannot open restart.xyz");
  const size_t n = m.n;
  const double* h = s.box.h;
  std::fprintf(f, "%zu\n", n);
  std::fprintf(f, "pbc=\"%c %c %c\" ", s.box.pbc[0] ? 'T' : 'F', s.box.pbc[1] ? 'T' : 'F',
               s.box.pbc[2] ? 'T' : 'F');
  std::fprintf(f, "Lattice=\"%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\" ", h[0], h[3],
               h[6], h[1], h[4], h[7], h[2], h[5], h[8]);
  if (m.groups.empty())
    std::fprintf(f, "Properties=species:S:1:pos:R:3:mass:R:1:vel:R:3\n");
  else
    std::fprintf(f, "Properties=species:S:1:pos:R:3:mass:R:1:vel:R:3:group:I:%zu\n",
                 m.groups.size());
  for (size_t a = 0; a < n; ++a) {
    std::fprintf(f, "%s %.17g %.17g %.17g %.17g %.17g %.17g %.17g ", m.species[a].c_str(),
                 s.pos[a], s.pos[n + a], s.pos[2 * n + a], m.mass[a], s.vel[a], s.vel[n + a],
                 s.vel[2 * n + a]);
    for (const auto& g : m.groups) std::fprintf(f, "%d ", g[a]);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}

// ---- the job --------------------------------------------------------------------------

struct Job {
  Model model;
  nepx_t* pot = nullptr;
  nepx_md_t* md = nullptr;
  std::vector<double> vel;   // A/fs until the md exists
  double dt_fs = 1.0;
  double time_fs = 0.0;
  std::uint32_t seed = 12345678u;
  // per run (the reference clears them after every run, runtime.cu:950-952)
  std::optional<CorrectVelocityCmd> correction;
  double max_distance = 0.0;     // adaptive time step bound (A), 0 = fixed step
  bool want_unwrapped = false;   // a dump_xyz asked for unwrapped positions
  long long force_calls = 0;     // force evaluations so far (neighbor.out numbering)

  State state(bool unwrapped = false)
  {
    State s;
    const size_t n = model.n;
    s.pos.resize(3 * n);
    s.vel.resize(3 * n);
    s.force.resize(3 * n);
    s.pe.resize(n);
    s.virial.resize(9 * n);
    check(nepx_md_get(md, s.pos.data(), s.vel.data(), s.force.data(), s.pe.data(),
                      s.virial.data(), &s.box),
          "nepx_md_get", nepx_md_last_error(md));
    if (unwrapped) {
      s.unwrapped.resize(3 * n);
      check(nepx_md_get_unwrapped(md, s.unwrapped.data()), "nepx_md_get_unwrapped",
            nepx_md_last_error(md));
    }
    return s;
  }

  void ensure_md()
  {
    if (md) return;
    nepx_box box;
    std::memcpy(box.h, model.h, sizeof(box.h));
    std::memcpy(box.pbc, model.pbc, sizeof(box.pbc));
    const int rc = nepx_md_create(pot, model.n, model.type.data(), model.mass.data(),
                                  model.pos.data(), vel.data(), &box, nullptr, &md);
    if (rc) throw Failure("nepx_md_create failed (code " + std::to_string(rc) + "): " +
                          nepx_last_error(pot));
  }

  // The reference appends a neighbor.out line at every 1000th force
  // evaluation of the process, counted from 0 (nep.cu:1156-1176): the largest
  // radial and angular row of that evaluation next to their capacities.
  void neighbor_record(long long call)
  {
    if (call % 1000 != 0) return;
    int info[16];
    check(nepx_info(pot, info, nullptr), "nepx_info", nepx_last_error(pot));
    int r = 0, a = 0;
    check(nepx_md_neighbor_info(md, &r, &a), "nepx_md_neighbor_info", nepx_md_last_error(md));
    FILE* f = std::fopen("neighbor.out", "a");
    if (!f) throw Failure("cannot open neighbor.out");
    std::fprintf(f, "Neighbor info at step %lld: radial(max=%d,actual=%d), angular(max=%d,actual=%d).\n",
                 call, info[12], r, info[13], a);
    std::fclose(f);
  }

  void correct_now()
  {
    std::vector<double> pos(3 * model.n), v(3 * model.n);
    check(nepx_md_get(md, pos.data(), v.data(), nullptr, nullptr, nullptr, nullptr),
          "nepx_md_get", nepx_md_last_error(md));
    correct_velocity(model, *correction, pos, v);
    check(nepx_md_set_velocity(md, v.data()), "nepx_md_set_velocity", nepx_md_last_error(md));
  }

  void run(int steps, const EnsembleCmd& ens, const std::vector<int>& thermo,
           const std::vector<DumpXyzCmd>& xyz, const std::vector<int>& restart)
  {
    ensure_md();
    const double params[6] = {ens.T0, ens.T1, ens.Tdamp, ens.p_gpa, ens.bulk_gpa, ens.tau_p};
    check(nepx_md_set_ensemble(md, static_cast<int>(ens.kind), params, seed),
          "nepx_md_set_ensemble", nepx_md_last_error(md));
    if (ens.baro)
      check(nepx_md_set_barostat(md, ens.baro, ens.p6_gpa, ens.c6_gpa), "nepx_md_set_barostat",
            nepx_md_last_error(md));
    if (want_unwrapped)
      check(nepx_md_enable_unwrapped(md), "nepx_md_enable_unwrapped", nepx_md_last_error(md));
    check(nepx_md_set_max_distance(md, max_distance), "time_step", nepx_md_last_error(md));
    // the reference evaluates the forces once before the steps of every run
    // (runtime.cu:746); it is a force evaluation of the neighbor.out count
    check(nepx_md_compute_forces(md), "force evaluation", nepx_md_last_error(md));
    neighbor_record(force_calls++);
    const long long call0 = force_calls;   // the force evaluation of step 0
    // stop at every multiple of the gcd of the output intervals
    int g = 0;
    for (int v : thermo) g = std::gcd(g, v);
    for (const auto& d : xyz) g = std::gcd(g, d.interval);
    for (int v : restart) g = std::gcd(g, v);
    if (g == 0) g = steps;
    bool unwrapped_out = false;
    for (const auto& d : xyz) unwrapped_out |= d.unwrapped;
    FILE* tf = nullptr;
    if (!thermo.empty()) {
      tf = std::fopen("thermo.out", "a");
      if (!tf) throw Failure("cannot open thermo.out");
      write_thermo_header(tf, thermo.back(), model.n, dt_fs);
    }
    const double time0 = time_fs;
    double row[20];
    for (int done = 0; done < steps;) {
      if (correction && done % correction->interval == 0) correct_now();
      // the chunk ends at the next output step, the next velocity correction,
      // or right after the step whose force evaluation neighbor.out records
      int next = std::min(steps, (done / g + 1) * g);
      if (correction) next = std::min(next, (done / correction->interval + 1) * correction->interval);
      const long long to_record = (1000 - (call0 + done) % 1000) % 1000;
      if (done + to_record < steps) next = std::min<long long>(next, done + to_record + 1);
      const int k = next - done;
      check(nepx_md_run_segment(md, k, dt_fs, k, row, done, steps), "run",
            nepx_md_last_error(md));
      done = next;
      if (max_distance > 0.0) {
        double t = 0.0;
        check(nepx_md_time(md, &t), "nepx_md_time", nepx_md_last_error(md));
        time_fs = time0 + t;
      } else {
        time_fs += k * dt_fs;
      }
      neighbor_record(call0 + done - 1);
      if (tf && done % thermo.back() == 0) write_thermo_row(tf, row);
      bool need_state = false;
      for (const auto& d : xyz) need_state |= done % d.interval == 0;
      for (int v : restart) need_state |= done % v == 0;
      if (!need_state) continue;
      const State s = state(unwrapped_out);
      for (const auto& d : xyz)
        if (done % d.interval == 0) write_xyz(d, done - 1, time_fs, model, s, row);
      for (int v : restart)
        if (done % v == 0) write_restart(model, s);
    }
    force_calls = call0 + steps;
    if (tf) std::fclose(tf);
  }
};

}  // namespace

int main(int argc, char** argv)
{
  int precision = NEPX_PRECISION_FP32;
  bool check_only = false;
  for (int a = 1; a < argc; ++a) {
    const std::string arg = argv[a];
    if (arg == "--check") {
      check_only = true;
    } else if (arg == "--precision" && a + 1 < argc) {
      const std::string v = argv[++a];
      if (v == "mixed") precision = NEPX_PRECISION_MIXED;
      else if (v == "mixed_bf16") precision = NEPX_PRECISION_MIXED_BF16;
      else if (v != "fp32") {
        std::cerr << "nepx-md: --precision takes fp32, mixed or mixed_bf16\n";
        return EXIT_FAILURE;
      }
    } else {
      std::cerr << "usage: nepx-md [--precision fp32|mixed|mixed_bf16] [--check]   (run.in and "
                   "model.xyz in the working directory)\n";
      return EXIT_FAILURE;
    }
  }
  Job job;
  try {
    const std::vector<Command> program = parse_run_file("run.in");
    validate_program(program);
    std::string potential;
    for (const Command& c : program) {
      if (const auto* p = std::get_if<PotentialCmd>(&c.data)) {
        if (!potential.empty())
          throw InputError(c.source, "multiple potential commands are unsupported");
        potential = p->file;
      }
    }
    if (potential.empty())
      throw InputError(Source{"run.in", 0, {}}, "run.in does not contain a potential command");
    const PotentialHeader header = read_potential_header(potential);
    job.model = parse_model_file("model.xyz", header);
    if (check_only) {
      int runs = 0;
      for (const Command& c : program) runs += std::holds_alternative<RunCmd>(c.data);
      std::printf("ok: %d atoms, %zu types (%s), %zu commands, %d runs\n", job.model.n,
                  header.symbols.size(), header.model.c_str(), program.size(), runs);
      return EXIT_SUCCESS;
    }
    if (const char* s = std::getenv("DMGMD_ENSEMBLE_SEED")) {
      char* end = nullptr;
      const unsigned long v = std::strtoul(s, &end, 10);
      if (!*s || *end || v > 0xffffffffUL)
        throw Failure("DMGMD_ENSEMBLE_SEED must contain decimal digits only");
      job.seed = static_cast<std::uint32_t>(v);
    }
    check(nepx_create(potential.c_str(), job.model.n, &job.pot), "nepx_create", potential.c_str());
    if (precision != NEPX_PRECISION_FP32)
      check(nepx_set_precision(job.pot, precision), "nepx_set_precision", nepx_last_error(job.pot));
    if (job.model.has_velocity) {
      job.vel = job.model.vel;
    } else {
      std::srand(static_cast<unsigned>(
        std::chrono::system_clock::now().time_since_epoch().count()));
      random_velocities(job.model, 300.0, nullptr, job.vel);
    }
    EnsembleCmd ensemble;
    bool have_ensemble = false, have_potential = false;
    std::vector<int> thermo, restart;
    std::vector<DumpXyzCmd> xyz;
    for (const Command& c : program) {
      try {
        if (std::holds_alternative<PotentialCmd>(c.data)) {
          have_potential = true;
        } else if (const auto* v = std::get_if<VelocityCmd>(&c.data)) {
          if (!job.model.has_velocity) {
            if (job.md) throw Failure("velocity after a run is not supported by nepx-md");
            random_velocities(job.model, v->temperature, v->seed ? &*v->seed : nullptr, job.vel);
          }
        } else if (const auto* t = std::get_if<TimeStepCmd>(&c.data)) {
          job.dt_fs = t->fs;
          job.max_distance = t->max_distance.value_or(0.0);
        } else if (const auto* v = std::get_if<CorrectVelocityCmd>(&c.data)) {
          job.correction = *v;
        } else if (const auto* e = std::get_if<EnsembleCmd>(&c.data)) {
          ensemble = *e;
          have_ensemble = true;
        } else if (const auto* d = std::get_if<DumpThermoCmd>(&c.data)) {
          thermo.push_back(d->interval);
        } else if (const auto* d = std::get_if<DumpXyzCmd>(&c.data)) {
          xyz.push_back(*d);
          job.want_unwrapped |= d->unwrapped;
        } else if (const auto* d = std::get_if<DumpRestartCmd>(&c.data)) {
          restart.push_back(d->interval);
        } else if (const auto* r = std::get_if<RunCmd>(&c.data)) {
          if (!have_potential) throw Failure("run requires a preceding potential command");
          if (!have_ensemble) throw Failure("run requires a preceding ensemble command");
          if (r->steps > 0) job.run(r->steps, ensemble, thermo, xyz, restart);
          thermo.clear();
          xyz.clear();
          restart.clear();
          job.correction.reset();
          job.max_distance = 0.0;
        }
      } catch (const Failure& f) {
        throw InputError(c.source, f.what());
      }
    }
    if (!thermo.empty() || !xyz.empty() || !restart.empty())
      throw InputError(Source{"run.in", 0, {}}, "dump command is not followed by run");
  } catch (const InputError& e) {
    std::cerr << "nepx-md input error: " << e.describe() << "\n";
    if (job.md) nepx_md_destroy(job.md);
    if (job.pot) nepx_destroy(job.pot);
    return EXIT_FAILURE;
  } catch (const std::exception& e) {
    std::cerr << "nepx-md runtime error: " << e.what() << "\n";
    if (job.md) nepx_md_destroy(job.md);
    if (job.pot) nepx_destroy(job.pot);
    return EXIT_FAILURE;
  }
  if (job.md) nepx_md_destroy(job.md);
  if (job.pot) nepx_destroy(job.pot);
  return EXIT_SUCCESS;
}

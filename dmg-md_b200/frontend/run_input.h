// run_input.h -- the GPUMD-format input surface of the nepx-md driver:
// run.in programs, model.xyz structures and the nep.txt header.
//
// Same commands, argument rules and error messages as the reference's
// parse_run_file (src/run_parser.cpp:160-319) and parse_model_file
// (src/model_parser.cpp:279-418); every rejection carries the file, line and
// text it comes from.
#pragma once

#include <optional>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

namespace nepx_run {

struct Source {
  std::string file;
  size_t line = 0;
  std::string text;
};

class InputError : public std::runtime_error {
 public:
  InputError(Source source, const std::string& message)
      : std::runtime_error(message), source(std::move(source)) {}
  Source source;
  std::string describe() const;
};

// ---- run.in ------------------------------------------------------------------

enum class Ensemble { nve, nvt_ber, nvt_nhc, nvt_bdp, npt_ber, npt_scr };

struct PotentialCmd { std::string file; };
struct VelocityCmd { double temperature = 0; std::optional<int> seed; };
struct TimeStepCmd { double fs = 0; std::optional<double> max_distance; };
struct EnsembleCmd {
  Ensemble kind = Ensemble::nve;
  double T0 = 0, T1 = 0, Tdamp = 0;        // temperatures (K), coupling (steps)
  double p_gpa = 0, bulk_gpa = 0, tau_p = 0;
  int baro = 0;                  // 0 isotropic, 1 anisotropic (xx yy zz), 2 triclinic
  double p6_gpa[6] = {0, 0, 0, 0, 0, 0};   // component targets, xx yy zz yz xz xy
  double c6_gpa[6] = {0, 0, 0, 0, 0, 0};   // component moduli
};
struct CorrectVelocityCmd { int interval = 0; std::optional<int> grouping; };
struct DumpThermoCmd { int interval = 0; };
struct DumpXyzCmd {
  int interval = 0;
  std::string file;
  std::optional<int> grouping, group_id;
  bool double_precision = false;   // "precision double"; default single
  bool mass = false, charge = false, velocity = false, force = false, potential = false;
  bool unwrapped = false, virial = false, group_labels = false;
};
struct DumpRestartCmd { int interval = 0; };
struct RunCmd { int steps = 0; };

using CommandData = std::variant<PotentialCmd, VelocityCmd, TimeStepCmd, EnsembleCmd,
                                 CorrectVelocityCmd, DumpThermoCmd, DumpXyzCmd, DumpRestartCmd,
                                 RunCmd>;
struct Command {
  Source source;
  CommandData data;
};

std::vector<Command> parse_run_file(const std::string& path);

// Program-level checks of the reference (validate_runtime_ensembles,
// src/run_parser.cpp:321-395) plus what this driver does not run.
void validate_program(const std::vector<Command>& program);

// ---- nep.txt header and model.xyz ----------------------------------------------

struct PotentialHeader {
  std::string model;                  // nep4, nep5, nep4_zbl, nep5_zbl
  std::vector<std::string> symbols;   // type order
};
PotentialHeader read_potential_header(const std::string& path);

struct Model {
  int n = 0;
  double h[9] = {0};      // row-major, cell vectors as columns
  int pbc[3] = {1, 1, 1};
  std::vector<std::string> species;
  std::vector<int> type;
  std::vector<double> mass;
  std::vector<double> pos;   // [3][n]
  std::vector<double> vel;   // [3][n] A/fs (zero when the file has none)
  bool has_velocity = false;
  std::vector<std::vector<int>> groups;   // [method][n]
};
Model parse_model_file(const std::string& path, const PotentialHeader& potential);

// Whitespace tokens of a line (no comment handling).
std::vector<std::string> tokens(const std::string& line);

}  // namespace nepx_run

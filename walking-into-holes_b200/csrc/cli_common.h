// Command-line layer shared by the wih_twos and wih_adjoint executables.
//
// Keeps the reference's flag set, defaults, validation rules, exit codes and
// output formats (benchmarks/compiled_bunny/src/wih_twos.cpp:73-240 for the
// options, 1711-1793 for the field CSV and summary JSON) so the reference's
// Python drivers run unchanged against these executables.  Two flags are
// added: --precision {mixed,fp64} (default mixed) and --device N.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "twos.h"

namespace twos_cli {

struct Options {
  std::string mode = "twos";
  std::string source_mode = "affine";
  std::string mesh_path, points_path, output_path, summary_path, trace_path, cavities_path;
  std::string precision = "mixed";
  std::array<int, 3> grid{54, 64, 48};
  int walks = 16;
  int repeats = 3;
  int max_steps = 512;
  int threads = 0;
  int trace_sites = 0;
  int mg_cycles = 60, mg_pre_smooth = 3, mg_post_smooth = 3, mg_coarse_smooth = 80;
  int device = 0;
  uint64_t seed = 20260912ULL;
  double epsilon = 5.0e-4;
  double source_y_slope = 0.65;
  double validation_radius_cap = 0.1;
  double validation_value_cap = 0.1;
  double cavity_radius = 0.0;
  double diff_offset = 0.02;
  double mg_tolerance = 1.0e-8;
  double mg_omega = 0.72;
};

// Thrown instead of exiting so the --serve loop can answer `DONE 2`.
struct UsageError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void print_usage(const std::string &message) {
  if (!message.empty()) std::cerr << "error: " << message << "\n\n";
  std::cerr << "Usage: wih_twos --mesh MESH.ply --points POINTS.csv --output FIELD.csv\n"
            << "                 --summary SUMMARY.json [options]\n\n"
            << "Options (B200 backend):\n"
            << "  --mode NAME           twos (default), diffwos or validate; voxel and mg are\n"
            << "                        not provided by this backend\n"
            << "  --walks N             paths per evaluation site (default 16)\n"
            << "  --repeats N           timed repetitions; median is reported (default 3)\n"
            << "  --threads N           accepted for compatibility (host threads)\n"
            << "  --epsilon X           WoS termination shell (default 5e-4)\n"
            << "  --max-steps N         maximum spheres per path (default 512)\n"
            << "  --seed N              deterministic base seed\n"
            << "  --source-mode NAME    affine or housing (default affine)\n"
            << "  --source-y-slope X    f=1+slope*(y+0.5) (default 0.65)\n"
            << "  --cavities FILE       optional CSV of spherical cavity centers\n"
            << "  --cavity-radius X     common cavity radius (default 0)\n"
            << "  --precision NAME      mixed (FP32 query, FP64 accumulation; default) or fp64\n"
            << "  --device N            CUDA device (default 0)\n"
            << "  --grid, --mg-*, --diff-offset, --validation-*, --trace-*  accepted and\n"
            << "                        validated as by the reference\n";
}

inline Options parse_options(const std::vector<std::string> &argv) {
  Options o;
  std::unordered_map<std::string, std::string *> strings = {
      {"--mode", &o.mode},         {"--source-mode", &o.source_mode}, {"--mesh", &o.mesh_path},
      {"--points", &o.points_path}, {"--output", &o.output_path},      {"--summary", &o.summary_path},
      {"--trace-output", &o.trace_path}, {"--cavities", &o.cavities_path}, {"--precision", &o.precision},
  };
  for (size_t i = 0; i < argv.size(); ++i) {
    const std::string key = argv[i];
    if (key == "--help" || key == "-h") throw UsageError("");
    if (i + 1 >= argv.size()) throw UsageError("missing value for " + key);
    const std::string value = argv[++i];
    try {
      if (auto it = strings.find(key); it != strings.end()) {
        *it->second = value;
      } else if (key == "--walks") {
        o.walks = std::stoi(value);
      } else if (key == "--validation-radius-cap") {
        o.validation_radius_cap = std::stod(value);
      } else if (key == "--validation-value-cap") {
        o.validation_value_cap = std::stod(value);
      } else if (key == "--repeats") {
        o.repeats = std::stoi(value);
      } else if (key == "--max-steps") {
        o.max_steps = std::stoi(value);
      } else if (key == "--threads") {
        o.threads = std::stoi(value);
      } else if (key == "--trace-sites") {
        o.trace_sites = std::stoi(value);
      } else if (key == "--mg-cycles") {
        o.mg_cycles = std::stoi(value);
      } else if (key == "--mg-pre-smooth") {
        o.mg_pre_smooth = std::stoi(value);
      } else if (key == "--mg-post-smooth") {
        o.mg_post_smooth = std::stoi(value);
      } else if (key == "--mg-coarse-smooth") {
        o.mg_coarse_smooth = std::stoi(value);
      } else if (key == "--seed") {
        o.seed = std::stoull(value);
      } else if (key == "--epsilon") {
        o.epsilon = std::stod(value);
      } else if (key == "--source-y-slope") {
        o.source_y_slope = std::stod(value);
      } else if (key == "--cavity-radius") {
        o.cavity_radius = std::stod(value);
      } else if (key == "--diff-offset") {
        o.diff_offset = std::stod(value);
      } else if (key == "--mg-tolerance") {
        o.mg_tolerance = std::stod(value);
      } else if (key == "--mg-omega") {
        o.mg_omega = std::stod(value);
      } else if (key == "--device") {
        o.device = std::stoi(value);
      } else if (key == "--grid") {
        std::string parsed = value;
        std::replace(parsed.begin(), parsed.end(), ',', ' ');
        std::istringstream values(parsed);
        if (!(values >> o.grid[0] >> o.grid[1] >> o.grid[2])) throw UsageError("--grid must have the form NX,NY,NZ");
      } else {
        throw UsageError("unknown option " + key);
      }
    } catch (const std::invalid_argument &) {
      throw UsageError("invalid value for " + key);
    } catch (const std::out_of_range &) {
      throw UsageError("invalid value for " + key);
    }
  }
  if (o.mesh_path.empty() || o.points_path.empty() || o.output_path.empty() || o.summary_path.empty())
    throw UsageError("--mesh, --points, --output, and --summary are required");
  if ((o.mode != "twos" && o.mode != "diffwos" && o.mode != "voxel" && o.mode != "mg" && o.mode != "validate") ||
      (o.source_mode != "affine" && o.source_mode != "housing") || o.walks < 2 || o.repeats < 1 ||
      o.max_steps < 1 || o.epsilon <= 0.0 || o.trace_sites < 0 || o.validation_radius_cap <= 0 ||
      o.validation_value_cap <= 0 || o.mg_cycles < 1 || o.mg_pre_smooth < 1 || o.mg_post_smooth < 1 ||
      o.mg_coarse_smooth < 1 || o.diff_offset <= o.epsilon || o.mg_tolerance <= 0.0 || o.mg_omega <= 0.0 ||
      o.mg_omega >= 1.0 || o.cavity_radius < 0.0 || (!o.cavities_path.empty() && o.cavity_radius <= 0.0) ||
      (o.precision != "mixed" && o.precision != "fp64"))
    throw UsageError("invalid numeric option");
  if (o.mode == "diffwos" && o.cavities_path.empty()) throw UsageError("Differential WoS requires --cavities");
  for (int extent : o.grid)
    if (extent < 3) throw UsageError("every --grid extent must be at least three");
  if (o.mode == "mg")
    for (int extent : o.grid)
      if (extent % 2 == 0) throw UsageError("geometric multigrid requires odd --grid extents");
  return o;
}

inline twos_source_term make_term(int kind, double amp, int axis = 0, double offset = 0.0, double div = 1.0,
                                  std::array<double, 3> c = {0, 0, 0}, std::array<double, 3> w = {1, 1, 1}) {
  twos_source_term t{};
  t.kind = kind;
  t.axis = axis;
  t.amp = amp;
  t.offset = offset;
  t.div = div;
  for (int a = 0; a < 3; ++a) {
    t.c[a] = c[a];
    t.w[a] = w[a];
  }
  return t;
}

// The reference's source (wih_twos.cpp:546-567) as source terms.
inline void set_source(twos_request &r, const Options &o) {
  if (o.source_mode == "affine") {
    r.source[0] = make_term(TWOS_TERM_CONST, 1.0);
    r.source[1] = make_term(TWOS_TERM_LINEAR, o.source_y_slope, 1, 0.5);
    r.n_source = 2;
    r.green = 0;
  } else {
    r.source[0] = make_term(TWOS_TERM_CONST, 0.08);
    r.source[1] = make_term(TWOS_TERM_GAUSS, 5.2, 0, 0, 1, {-0.48, -0.18, -0.08}, {0.24, 0.22, 0.16});
    r.source[2] = make_term(TWOS_TERM_GAUSS, 4.6, 0, 0, 1, {0.43, 0.19, -0.07}, {0.21, 0.20, 0.15});
    r.source[3] = make_term(TWOS_TERM_GAUSS, 2.0, 0, 0, 1, {0.02, -0.31, -0.02}, {0.30, 0.16, 0.19});
    r.n_source = 4;
    r.green = 1;
  }
}

inline twos_request base_request(const Options &o) {
  twos_request r{};
  r.mode = TWOS_MODE_COMPLIANCE;
  r.precision = o.precision == "fp64" ? TWOS_PREC_FP64 : TWOS_PREC_MIXED;
  r.walks = o.walks;
  r.max_steps = o.max_steps;
  r.seed = o.seed;
  r.repeat = 0;
  r.stream = 0;
  r.epsilon = o.epsilon;
  r.cavity_radius = o.cavity_radius;
  r.query_radius = 4.0;
  set_source(r, o);
  return r;
}

inline double median(std::vector<double> values) {
  std::sort(values.begin(), values.end());
  const size_t middle = values.size() / 2;
  if (values.size() % 2 == 1) return values[middle];
  return 0.5 * (values[middle - 1] + values[middle]);
}

inline double peak_rss_megabytes() {
  std::ifstream status("/proc/self/status");
  std::string key;
  while (status >> key) {
    if (key == "VmHWM:") {
      double kilobytes = 0.0;
      std::string unit;
      status >> kilobytes >> unit;
      return kilobytes / 1024.0;
    }
    std::string rest;
    std::getline(status, rest);
  }
  return std::numeric_limits<double>::quiet_NaN();
}

inline std::vector<double> read_points(const std::string &path) {
  std::ifstream input(path);
  if (!input) throw std::runtime_error("cannot open points: " + path);
  std::vector<double> points;
  std::string line;
  while (std::getline(input, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::replace(line.begin(), line.end(), ',', ' ');
    std::istringstream values(line);
    double x, y, z;
    if (values >> x >> y >> z) {
      points.push_back(x);
      points.push_back(y);
      points.push_back(z);
    }
  }
  if (points.empty()) throw std::runtime_error("points file contains no points");
  return points;
}

inline std::vector<double> read_optional_points(const std::string &path) {
  if (path.empty()) return {};
  return read_points(path);
}

inline void throw_on(int rc) {
  if (rc != TWOS_OK) throw std::runtime_error(twos_last_error());
}

inline int effective_threads(const Options &o) {
  return o.threads > 0 ? o.threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
}

// Differential field CSV (write_differential_field, wih_twos.cpp:1576-1602):
// site,x,y,z then per cavity i dc{i}_x,_y,_z, dc{i}_se_x,_y,_z, dR{i},
// dR{i}_se, at 17 significant digits.
inline void write_differential_field(const std::string &path, const std::vector<double> &points,
                                     const std::vector<twos_diff_result> &rows, size_t n_cav) {
  std::ofstream output(path);
  if (!output) throw std::runtime_error("cannot write differential field output: " + path);
  output << "site,x,y,z";
  for (size_t c = 0; c < n_cav; ++c)
    output << ",dc" << c << "_x,dc" << c << "_y,dc" << c << "_z,dc" << c << "_se_x,dc" << c << "_se_y,dc" << c
           << "_se_z,dR" << c << ",dR" << c << "_se";
  output << "\n" << std::setprecision(17);
  const size_t n = points.size() / 3;
  for (size_t s = 0; s < n; ++s) {
    output << s << ',' << points[3 * s] << ',' << points[3 * s + 1] << ',' << points[3 * s + 2];
    for (size_t c = 0; c < n_cav; ++c) {
      const twos_diff_result &d = rows[s * n_cav + c];
      output << ',' << d.dc[0] << ',' << d.dc[1] << ',' << d.dc[2] << ',' << d.dc_se[0] << ',' << d.dc_se[1] << ','
             << d.dc_se[2] << ',' << d.dR << ',' << d.dR_se;
    }
    output << '\n';
  }
}

// Runs twos_diffwos, accepting its "unsafe differential path" return (rows
// and statistics are written) so the caller applies its own policy to caps
// and unsafe offsets; any other failure throws.
inline twos_summary run_diffwos(twos_mesh *mesh, const twos_request &r, double offset, int enclosure_fallback,
                                const std::vector<double> &points, const std::vector<double> &cavities,
                                std::vector<twos_diff_result> &rows, std::vector<twos_diff_stats> &stats) {
  const size_t n = points.size() / 3, n_cav = cavities.size() / 3;
  rows.assign(n * n_cav, twos_diff_result{});
  stats.assign(n, twos_diff_stats{});
  twos_summary s{};
  const int rc = twos_diffwos(mesh, &r, offset, enclosure_fallback, points.data(), static_cast<uint32_t>(n),
                              cavities.data(), static_cast<uint32_t>(n_cav), rows.data(), stats.data(), &s);
  if (rc != TWOS_OK && !(rc == TWOS_ERR_RUNTIME && s.error_flags == 0 &&
                         std::string(twos_last_error()).rfind("unsafe differential path", 0) == 0))
    throw_on(rc);
  return s;
}

}  // namespace twos_cli

// wih_study family: drop-in executables for the submission-study backend
// (benchmarks/submission_study/study.cpp), on libtwos.so.
//
//   wih_study             study.cpp as built plain: paired/hot estimates with a
//                         Beta(2,2) Green point per step, --diff 1 gradients.
//   wih_analytic_query    study.cpp with WIH_ANALYTIC_SOURCE (analytic_query.cpp):
//                         each step adds the exact ball integral of every heat
//                         bump (and of the sensor for p) instead of a sample.
//   wih_compliance_query  with WIH_ANALYTIC_SOURCE and WIH_AFFINE_COMPLIANCE
//                         (compliance_query.cpp): f = 1 + 0.65 y for both u and
//                         p, integrated exactly as r^2/6 f(y).
//
// Argv as study.cpp:273-292: the wih_twos options plus --config FILE (a
// sensor "x y z r" then heat records "x y z r A", study.cpp:37-42; the sensor
// there overrides --sensor-side, as in the reference's order of operations),
// --diff 0|1, --fd 0|1, --sensor-side -1|1, --hot-only 0|1.  --mode twos
// only (mg is a grid baseline this backend does not provide); --fd 1 (the
// coupled finite-difference baseline) is refused the same way.
//
// Outputs, at 17 significant digits:
//   paired/hot: CSV site,u,p,score,same_index,steps,caps; summary
//     {total_seconds, peak_rss_megabytes, distance_queries, parity_rays,
//      enclosure_fallbacks, relative_residual, steps, caps} (study.cpp:345-353);
//     a request whose walks hit --max-steps writes its CSV, then fails.
//   --diff 1: the differential field CSV and {total_seconds, steps, caps,
//     peak_rss_megabytes, distance_queries, parity_rays, enclosure_fallbacks}
//     (study.cpp:304-316), with the enclosure fallback on; an unsafe offset or
//     a capped path fails the request after the field is written.
// Runtime errors print the message and return 1; usage errors return 2.
// `--serve` keeps one mesh per session and reads "<argc>\n" + argc lines per
// request, answering "DONE <code>" and stopping after a non-zero code; bad
// framing exits 2 (study.cpp:358-379).
#include <memory>

#include "cli_common.h"

#ifndef TWOS_STUDY_ANALYTIC
#define TWOS_STUDY_ANALYTIC 0
#endif
#ifndef TWOS_STUDY_AFFINE
#define TWOS_STUDY_AFFINE 0
#endif

using namespace twos_cli;

namespace {

constexpr double kPi = 3.141592653589793;

struct Session {
  twos_mesh *mesh = nullptr;
  std::string path;
  ~Session() { twos_mesh_close(mesh); }
};

struct StudyConfig {
  std::array<double, 3> sensor{0.55, 0.18, -0.03};
  double sensor_radius = 0.13;
  std::vector<std::array<double, 5>> heat;  // x y z r A
};

// load_config (study.cpp:37-42): one whitespace stream.
StudyConfig load_config(const std::string &path, const std::array<double, 3> &sensor) {
  StudyConfig c;
  c.sensor = sensor;
  std::ifstream f(path);
  if (!(f >> c.sensor[0] >> c.sensor[1] >> c.sensor[2] >> c.sensor_radius))
    throw std::runtime_error("bad sensor config");
  std::array<double, 5> h{};
  while (f >> h[0] >> h[1] >> h[2] >> h[3] >> h[4]) c.heat.push_back(h);
  if (c.heat.empty()) throw std::runtime_error("missing compact heat sources");
  return c;
}

// custom_source (study.cpp:30-36) as source terms.
int set_custom_source(twos_source_term *terms, const StudyConfig &c) {
  if (TWOS_STUDY_AFFINE) {
    terms[0] = make_term(TWOS_TERM_CONST, 1.0);
    terms[1] = make_term(TWOS_TERM_LINEAR, 0.65, 1, 0.0);
    return 2;
  }
  if (c.heat.size() > TWOS_MAX_TERMS) throw std::runtime_error("too many heat sources");
  int n = 0;
  for (const auto &h : c.heat) terms[n++] = make_term(TWOS_TERM_BUMP, h[4], 0, 0.0, 1.0, {h[0], h[1], h[2]}, {h[3], 0, 0});
  return n;
}

// sensor_source (study.cpp:44-52): the bump divided by its integral
// 32 pi R^3 / 105; in the exact mode its amplitude is that reciprocal,
// written as study.cpp:100-101 writes it.
int set_sensor_source(twos_source_term *terms, const StudyConfig &c) {
  if (TWOS_STUDY_AFFINE) return set_custom_source(terms, c);
  const double R = c.sensor_radius;
  if (TWOS_STUDY_ANALYTIC)
    terms[0] = make_term(TWOS_TERM_BUMP, 105 / (32 * kPi * std::pow(R, 3)), 0, 0.0, 1.0, c.sensor, {R, 0, 0});
  else
    terms[0] = make_term(TWOS_TERM_BUMP, 1.0, 0, 0.0, 32 * kPi * std::pow(R, 3) / 105, c.sensor, {R, 0, 0});
  return 1;
}

bool inside_cavity(const double *x, const std::vector<double> &holes, double radius) {
  for (size_t i = 0; i + 2 < holes.size(); i += 3) {
    const double dx = x[0] - holes[i], dy = x[1] - holes[i + 1], dz = x[2] - holes[i + 2];
    if (std::sqrt(dx * dx + dy * dy + dz * dz) <= radius) return true;
  }
  return false;
}

int process_request(const std::vector<std::string> &argv, Session &session) {
  try {
    std::array<double, 3> sensor{0.55, 0.18, -0.03};
    bool hot = false, fd = false, diff = false;
    std::string config;
    std::vector<std::string> args;
    for (size_t i = 1; i < argv.size(); ++i) {
      const std::string &key = argv[i];
      if (key == "--config" || key == "--fd" || key == "--diff") {
        if (i + 1 == argv.size()) throw std::runtime_error("missing value for " + key);
        const std::string &value = argv[++i];
        if (key == "--config")
          config = value;
        else if (key == "--fd")
          fd = std::stoi(value) != 0;
        else
          diff = std::stoi(value) != 0;
      } else if (key == "--sensor-side") {
        if (i + 1 == argv.size()) throw std::runtime_error("missing sensor side");
        const int side = std::stoi(argv[++i]);
        if (side != 1 && side != -1) throw std::runtime_error("sensor side must be -1 or 1");
        sensor = {0.55 * side, 0.18 * side, -0.03};
      } else if (key == "--hot-only") {
        if (i + 1 == argv.size()) throw std::runtime_error("missing hot flag");
        hot = std::stoi(argv[++i]) != 0;
      } else {
        args.push_back(key);
      }
    }
    Options o;
    try {
      o = parse_options(args);
    } catch (const UsageError &e) {
      print_usage(e.what());
      return 2;
    }
    const StudyConfig cfg = load_config(config, sensor);
    if (o.mode != "twos" && o.mode != "mg") throw std::runtime_error("use twos or mg");
    if (o.mode == "mg") throw std::runtime_error("mode mg is not provided by the TWoS B200 backend");
    const auto start = std::chrono::steady_clock::now();
    if (!session.mesh) {
      throw_on(twos_mesh_open_ply(o.mesh_path.c_str(), o.device, &session.mesh));
      session.path = o.mesh_path;
    }
    if (session.path != o.mesh_path) throw std::runtime_error("a session must retain the same outer mesh");
    const std::vector<double> points = read_points(o.points_path);
    const std::vector<double> holes = read_optional_points(o.cavities_path);
    const size_t n = points.size() / 3;
    twos_request r = base_request(o);
    r.n_source = set_custom_source(r.source, cfg);

    if (diff) {
      // The nested walks are wih_twos.cpp's walk with custom_source: a Green
      // point in housing mode, the ball centre otherwise (wih_twos.cpp:646-653).
      r.mode = TWOS_MODE_COMPLIANCE;
      r.green = o.source_mode == "housing" ? TWOS_SOURCE_GREEN : TWOS_SOURCE_CENTER;
      r.skip_cavity_sites = 0;
      std::vector<twos_diff_result> rows;
      std::vector<twos_diff_stats> stats;
      const twos_summary s = run_diffwos(session.mesh, r, o.diff_offset, 1, points, holes, rows, stats);
      write_differential_field(o.output_path, points, rows, holes.size() / 3);
      uint64_t steps = 0, unsafe = 0, caps = 0;
      for (const twos_diff_stats &d : stats) {
        steps += d.outer_steps + d.nested_steps;
        unsafe += d.unsafe_offset;
        caps += d.limits;
      }
      if (unsafe || caps)
        throw std::runtime_error("unsafe differential path: unsafe=" + std::to_string(unsafe) +
                                 " caps=" + std::to_string(caps));
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
      std::ofstream f(o.summary_path);
      if (!f) throw std::runtime_error("cannot write summary: " + o.summary_path);
      f << std::setprecision(17) << "{\"total_seconds\":" << sec << ",\"steps\":" << steps << ",\"caps\":" << caps
        << ",\"peak_rss_megabytes\":" << peak_rss_megabytes() << ",\"distance_queries\":" << s.queries
        << ",\"parity_rays\":" << s.node_tests << ",\"enclosure_fallbacks\":" << s.plane_tests << "}\n";
      return 0;
    }
    if (fd) throw std::runtime_error("the finite-difference baseline (--fd 1) is not provided by the TWoS B200 backend");

    r.mode = hot ? TWOS_MODE_HOT : TWOS_MODE_PAIRED;
    r.green = TWOS_STUDY_ANALYTIC ? TWOS_SOURCE_EXACT : TWOS_SOURCE_GREEN;
    r.skip_cavity_sites = 1;
    r.n_adjoint = set_sensor_source(r.adjoint, cfg);
    std::vector<twos_site_result> values(n);
    twos_summary s{};
    const int rc = twos_estimate(session.mesh, &r, points.data(), static_cast<uint32_t>(n), holes.data(),
                                 static_cast<uint32_t>(holes.size() / 3), values.data(), &s);
    if (rc != TWOS_OK && !(rc == TWOS_ERR_RUNTIME && s.error_flags == 0 && s.caps > 0)) throw_on(rc);
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    uint64_t steps = 0, caps = 0, queries = 0;
    std::ofstream f(o.output_path);
    if (!f) throw std::runtime_error("cannot write field output: " + o.output_path);
    f << "site,u,p,score,same_index,steps,caps\n" << std::setprecision(17);
    for (size_t i = 0; i < n; ++i) {
      const twos_site_result &v = values[i];
      steps += v.steps;
      caps += v.caps;
      // One distance query per step, plus the terminal one of every path
      // that was not capped; sites inside a cavity run no walk.
      if (!inside_cavity(&points[3 * i], holes, o.cavity_radius))
        queries += v.steps + static_cast<uint64_t>(o.walks) - v.caps;
      const double p = hot ? 0.0 : v.p;
      const double same = hot ? 0.0 : v.same_index;
      f << i << ',' << v.u << ',' << p << ',' << v.score << ',' << same << ',' << v.steps << ',' << v.caps << '\n';
    }
    f.close();
    if (caps) throw std::runtime_error("walk step limit reached");
    std::ofstream sm(o.summary_path);
    if (!sm) throw std::runtime_error("cannot write summary: " + o.summary_path);
    sm << std::setprecision(17) << "{\"total_seconds\":" << seconds << ",\"peak_rss_megabytes\":"
       << peak_rss_megabytes() << ",\"distance_queries\":" << queries << ",\"parity_rays\":0"
       << ",\"enclosure_fallbacks\":0,\"relative_residual\":0,\"steps\":" << steps << ",\"caps\":" << caps
       << ",\"gpu_kernel_seconds\":" << s.kernel_seconds << ",\"gpu_precision\":\"" << o.precision << "\"}\n";
    return 0;
  } catch (const std::exception &e) {
    std::cerr << e.what() << '\n';
    return 1;
  }
}

}  // namespace

int main(int argc, char **argv) {
  Session session;
  if (argc == 2 && std::string(argv[1]) == "--serve") {
    std::string line;
    while (std::getline(std::cin, line)) {
      int n = 0;
      try {
        n = std::stoi(line);
      } catch (...) {
        return 2;
      }
      if (n <= 0 || n > 200) return 2;
      std::vector<std::string> values(static_cast<size_t>(n));
      for (auto &value : values)
        if (!std::getline(std::cin, value)) return 2;
      const int code = process_request(values, session);
      std::cout << "DONE " << code << std::endl;
      if (code) return code;
    }
    return 0;
  }
  return process_request(std::vector<std::string>(argv, argv + argc), session);
}

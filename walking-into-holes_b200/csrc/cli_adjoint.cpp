// wih_adjoint: drop-in executable for the reference's paired primal/adjoint
// backend (benchmarks/distinct_adjoint/adjoint.cpp:91-158), on libtwos.so.
//
// One walk set carries u (the --source-mode source) and p (the sensor bump
// (1 - |x-c|^2/0.13^2)_+^2 about c = (0.55 s, 0.18 s, -0.03), s from
// --sensor-side) evaluated at a shared Beta(2,2) Green point per step.
// Output CSV `site,u,p,score,same_index,steps,caps` at 17 digits and the
// summary JSON {total_seconds, peak_rss_megabytes, relative_residual, steps,
// caps}; --hot-only 1 reports score = mean u.  Sites inside a cavity get
// all-zero rows.  A request whose walks hit --max-steps writes its CSV and then
// fails with code 1.
//
// `wih_adjoint --serve` keeps one mesh for the session and reads requests from
// stdin as "<argc>\n" followed by argc lines (the first is the program name);
// each is answered with "DONE <code>", and the server exits after a non-zero
// code.  Malformed framing exits with 2.  A request naming another mesh is an
// error, as in the reference.
#include <memory>

#include "cli_common.h"

using namespace twos_cli;

namespace {

struct Session {
  twos_mesh *mesh = nullptr;
  std::string path;
  int device = -1;
  ~Session() { twos_mesh_close(mesh); }
};

int process_request(const std::vector<std::string> &argv, Session &session) {
  try {
    double side = 1.0;
    bool hot = false;
    std::vector<std::string> args;
    for (size_t i = 1; i < argv.size(); ++i) {
      const std::string &key = argv[i];
      if (key == "--sensor-side") {
        if (i + 1 == argv.size()) throw std::runtime_error("missing sensor side");
        const int s = std::stoi(argv[++i]);
        if (s != 1 && s != -1) throw std::runtime_error("sensor side must be -1 or 1");
        side = s;
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
    if (o.mode != "twos" && o.mode != "mg") throw std::runtime_error("use twos or mg");
    if (o.mode == "mg") throw std::runtime_error("mode mg is not provided by the TWoS B200 backend");
    const auto start = std::chrono::steady_clock::now();
    if (!session.mesh) {
      throw_on(twos_mesh_open_ply(o.mesh_path.c_str(), o.device, &session.mesh));
      session.path = o.mesh_path;
      session.device = o.device;
    }
    if (session.path != o.mesh_path) throw std::runtime_error("a session must retain the same outer mesh");
    const std::vector<double> points = read_points(o.points_path);
    const std::vector<double> holes = read_optional_points(o.cavities_path);
    const size_t n = points.size() / 3;
    twos_request r = base_request(o);
    r.mode = hot ? TWOS_MODE_HOT : TWOS_MODE_PAIRED;
    r.green = 1;  // paired_site always draws the Green point (adjoint.cpp:31)
    r.skip_cavity_sites = 1;
    r.adjoint[0] = make_term(TWOS_TERM_BUMP, 1.0, 0, 0.0, 1.0, {0.55 * side, 0.18 * side, -0.03}, {0.13, 0.0, 0.0});
    r.n_adjoint = 1;
    std::vector<twos_site_result> values(n);
    twos_summary s{};
    const int rc = twos_estimate(session.mesh, &r, points.data(), static_cast<uint32_t>(n), holes.data(),
                                 static_cast<uint32_t>(holes.size() / 3), values.data(), &s);
    if (rc != TWOS_OK && !(rc == TWOS_ERR_RUNTIME && s.error_flags == 0 && s.caps > 0)) throw_on(rc);
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    uint64_t steps = 0, caps = 0;
    std::ofstream f(o.output_path);
    if (!f) throw std::runtime_error("cannot write field output: " + o.output_path);
    f << "site,u,p,score,same_index,steps,caps\n" << std::setprecision(17);
    for (size_t i = 0; i < n; ++i) {
      const twos_site_result &v = values[i];
      steps += v.steps;
      caps += v.caps;
      const double p = hot ? 0.0 : v.p;
      const double same = hot ? 0.0 : v.same_index;
      f << i << ',' << v.u << ',' << p << ',' << v.score << ',' << same << ',' << v.steps << ',' << v.caps << '\n';
    }
    f.close();
    if (caps) throw std::runtime_error("walk step limit reached");
    std::ofstream sm(o.summary_path);
    if (!sm) throw std::runtime_error("cannot write summary: " + o.summary_path);
    sm << std::setprecision(17) << "{\"total_seconds\":" << seconds << ",\"peak_rss_megabytes\":"
       << peak_rss_megabytes() << ",\"relative_residual\":" << 0 << ",\"steps\":" << steps << ",\"caps\":" << caps
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

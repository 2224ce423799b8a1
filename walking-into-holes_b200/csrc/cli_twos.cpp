// wih_twos: drop-in executable for the reference's compliance TWoS backend
// (benchmarks/compiled_bunny/src/wih_twos.cpp:1799-1864, --mode twos), on
// libtwos.so.  Same argv, same field CSV `site,x,y,z,u,score,score_se,steps,
// limit_hits` at 17 significant digits, same summary JSON keys (plus gpu_*
// keys), same exit codes: 2 for usage errors, 1 with "fatal: ..." for runtime
// errors, including any retained path that hits --max-steps.
#include <memory>

#include "cli_common.h"

using namespace twos_cli;

namespace {

struct MeshHandle {
  twos_mesh *m = nullptr;
  ~MeshHandle() { twos_mesh_close(m); }
};

void write_field(const std::string &path, const std::vector<double> &points,
                 const std::vector<twos_site_result> &results) {
  std::ofstream output(path);
  if (!output) throw std::runtime_error("cannot write field output: " + path);
  output << "site,x,y,z,u,score,score_se,steps,limit_hits\n";
  output << std::setprecision(17);
  for (size_t i = 0; i < results.size(); ++i) {
    output << i << ',' << points[3 * i] << ',' << points[3 * i + 1] << ',' << points[3 * i + 2] << ','
           << results[i].u << ',' << results[i].score << ',' << results[i].score_se << ',' << results[i].steps
           << ',' << results[i].caps << '\n';
  }
}

void write_summary(const std::string &path, const twos_mesh_info &info, size_t n_cavities, const Options &o,
                   size_t site_count, const std::vector<double> &times, const std::vector<double> &kernel_times,
                   uint64_t total_steps, uint64_t total_limits) {
  const double runtime = median(times);
  const double paths = static_cast<double>(site_count) * o.walks;
  std::ofstream out(path);
  if (!out) throw std::runtime_error("cannot write summary: " + path);
  const double input_mb =
      static_cast<double>(info.vertices * 3 * sizeof(double) + info.faces * 3 * sizeof(uint32_t)) / (1024.0 * 1024.0);
  out << std::setprecision(17) << "{\n"
      << "  \"engine\": \"TWoS B200 sm_100a\",\n"
      << "  \"vertices\": " << info.vertices << ",\n"
      << "  \"faces\": " << info.faces << ",\n"
      << "  \"source_mode\": \"" << o.source_mode << "\",\n"
      << "  \"cavities\": " << n_cavities << ",\n"
      << "  \"cavity_radius\": " << o.cavity_radius << ",\n"
      << "  \"sites\": " << site_count << ",\n"
      << "  \"walks_per_site\": " << o.walks << ",\n"
      << "  \"repeats\": " << o.repeats << ",\n"
      << "  \"threads\": " << effective_threads(o) << ",\n"
      << "  \"epsilon\": " << o.epsilon << ",\n"
      << "  \"mesh_build_seconds\": " << info.build_seconds << ",\n"
      << "  \"runtime_seconds_median\": " << runtime << ",\n"
      << "  \"runtime_seconds_min\": " << *std::min_element(times.begin(), times.end()) << ",\n"
      << "  \"paths_per_second\": " << paths / runtime << ",\n"
      << "  \"distance_queries_per_second\": " << (static_cast<double>(total_steps) + paths) / runtime << ",\n"
      << "  \"mean_steps\": " << static_cast<double>(total_steps) / paths << ",\n"
      << "  \"max_step_limit_hits\": " << total_limits << ",\n"
      << "  \"mesh_input_megabytes\": " << input_mb << ",\n"
      << "  \"peak_rss_megabytes\": " << peak_rss_megabytes() << ",\n"
      << "  \"gpu_precision\": \"" << o.precision << "\",\n"
      << "  \"gpu_device\": " << info.device << ",\n"
      << "  \"gpu_kernel_seconds_median\": " << median(kernel_times) << ",\n"
      << "  \"gpu_bvh_nodes\": " << info.bvh_nodes << ",\n"
      << "  \"gpu_bvh_depth\": " << info.bvh_depth << ",\n"
      << "  \"gpu_mixed_delta\": " << info.mixed_delta << ",\n"
      << "  \"timings_seconds\": [";
  for (size_t i = 0; i < times.size(); ++i) {
    if (i) out << ", ";
    out << times[i];
  }
  out << "]\n}\n";
}

int run(const Options &o) {
  if (o.mode != "twos")
    throw std::runtime_error("mode " + o.mode + " is not provided by the TWoS B200 backend");
  MeshHandle mesh;
  throw_on(twos_mesh_open_ply(o.mesh_path.c_str(), o.device, &mesh.m));
  twos_mesh_info info{};
  throw_on(twos_mesh_get_info(mesh.m, &info));
  const std::vector<double> points = read_points(o.points_path);
  const std::vector<double> cavities = read_optional_points(o.cavities_path);
  const size_t n = points.size() / 3;
  twos_request r = base_request(o);
  std::vector<double> times, kernel_times;
  std::vector<twos_site_result> retained(n);
  uint64_t retained_steps = 0, retained_limits = 0;
  for (int repeat = 0; repeat < o.repeats; ++repeat) {
    std::vector<twos_site_result> results(n);
    r.repeat = static_cast<uint32_t>(repeat);
    twos_summary s{};
    const auto start = std::chrono::steady_clock::now();
    const int rc = twos_estimate(mesh.m, &r, points.data(), static_cast<uint32_t>(n), cavities.data(),
                                 static_cast<uint32_t>(cavities.size() / 3), results.data(), &s);
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    // A step cap is judged on the retained repeat only (wih_twos.cpp:1842-1848).
    if (rc != TWOS_OK && !(rc == TWOS_ERR_RUNTIME && s.error_flags == 0 && s.caps > 0)) throw_on(rc);
    times.push_back(elapsed);
    kernel_times.push_back(s.kernel_seconds);
    if (repeat == 0) {
      retained = std::move(results);
      retained_steps = s.steps;
      retained_limits = s.caps;
    }
  }
  if (retained_limits != 0) throw std::runtime_error("one or more paths hit --max-steps");
  write_field(o.output_path, points, retained);
  if (!o.trace_path.empty() && o.trace_sites > 0)
    std::cerr << "warning: --trace-output is not written by the TWoS B200 backend\n";
  write_summary(o.summary_path, info, cavities.size() / 3, o, n, times, kernel_times, retained_steps,
                retained_limits);
  std::cout << "TWoS B200: " << n << " sites x " << o.walks << " walks, median " << median(times) << " s, "
            << std::fixed << std::setprecision(0) << (static_cast<double>(n) * o.walks / median(times))
            << " paths/s\n";
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  Options o;
  try {
    o = parse_options(std::vector<std::string>(argv + 1, argv + argc));
  } catch (const UsageError &e) {
    print_usage(e.what());
    return 2;
  }
  try {
    return run(o);
  } catch (const std::exception &e) {
    std::cerr << "fatal: " << e.what() << '\n';
    return 1;
  }
}

// wih_twos: drop-in executable for the reference's compliance TWoS backend
// (benchmarks/compiled_bunny/src/wih_twos.cpp:1799-1864, --mode twos and
// --mode diffwos), on libtwos.so.  Same argv, same field CSV `site,x,y,z,u,score,score_se,steps,
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
                   uint64_t total_steps, uint64_t total_limits, uint64_t grid_steps) {
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
      << "  \"gpu_grid_steps\": " << grid_steps << ",\n"
      << "  \"timings_seconds\": [";
  for (size_t i = 0; i < times.size(); ++i) {
    if (i) out << ", ";
    out << times[i];
  }
  out << "]\n}\n";
}

// --mode diffwos (run_differential_wos, wih_twos.cpp:1604-1709): retained
// repeat 0, an error when any outer or nested path hit --max-steps (unsafe
// offsets are counted, not errors, in this executable), field CSV and the
// differential summary JSON.
int run_differential(const Options &o, twos_mesh *mesh, const twos_mesh_info &info,
                     const std::vector<double> &points, const std::vector<double> &cavities) {
  const size_t n = points.size() / 3, n_cav = cavities.size() / 3;
  twos_request r = base_request(o);
  std::vector<double> times;
  std::vector<twos_diff_result> retained;
  std::vector<twos_diff_stats> stats;
  for (int repeat = 0; repeat < o.repeats; ++repeat) {
    r.repeat = static_cast<uint32_t>(repeat);
    std::vector<twos_diff_result> rows;
    std::vector<twos_diff_stats> st;
    const auto start = std::chrono::steady_clock::now();
    run_diffwos(mesh, r, o.diff_offset, 0, points, cavities, rows, st);
    times.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count());
    if (repeat == 0) {
      retained = std::move(rows);
      stats = std::move(st);
    }
  }
  uint64_t outer = 0, nested = 0, cav = 0, seam = 0, seg = 0, unsafe = 0, limits = 0;
  for (const twos_diff_stats &s : stats) {
    outer += s.outer_steps;
    nested += s.nested_steps;
    cav += s.cavity_terminations;
    seam += s.near_seam;
    seg += s.segment_unsafe;
    unsafe += s.unsafe_offset;
    limits += s.limits;
  }
  if (limits != 0) throw std::runtime_error("one or more differential paths hit --max-steps");
  write_differential_field(o.output_path, points, retained, n_cav);
  const double runtime = median(times);
  const double paths = static_cast<double>(n) * o.walks;
  std::ofstream out(o.summary_path);
  if (!out) throw std::runtime_error("cannot write differential summary: " + o.summary_path);
  out << std::setprecision(17) << "{\n"
      << "  \"engine\": \"TWoS B200 sm_100a Differential WoS\",\n"
      << "  \"mode\": \"diffwos\",\n"
      << "  \"vertices\": " << info.vertices << ",\n"
      << "  \"faces\": " << info.faces << ",\n"
      << "  \"source_mode\": \"" << o.source_mode << "\",\n"
      << "  \"cavities\": " << n_cav << ",\n"
      << "  \"gradient_parameters\": " << 4 * n_cav << ",\n"
      << "  \"cavity_radius\": " << o.cavity_radius << ",\n"
      << "  \"sites\": " << n << ",\n"
      << "  \"walks_per_site\": " << o.walks << ",\n"
      << "  \"seed\": " << o.seed << ",\n"
      << "  \"epsilon\": " << o.epsilon << ",\n"
      << "  \"normal_offset\": " << o.diff_offset << ",\n"
      << "  \"seam_strip_multiplier\": 1,\n"
      << "  \"runtime_seconds_median\": " << runtime << ",\n"
      << "  \"outer_mean_steps\": " << static_cast<double>(outer) / paths << ",\n"
      << "  \"nested_mean_steps_per_outer_path\": " << static_cast<double>(nested) / paths << ",\n"
      << "  \"cavity_termination_fraction\": " << static_cast<double>(cav) / paths << ",\n"
      << "  \"near_seam_fraction\": " << static_cast<double>(seam) / paths << ",\n"
      << "  \"segment_unsafe_fraction\": " << static_cast<double>(seg) / paths << ",\n"
      << "  \"unsafe_offset_fraction\": " << static_cast<double>(unsafe) / paths << ",\n"
      << "  \"unsafe_given_cavity_fraction\": "
      << (cav == 0 ? 0.0 : static_cast<double>(unsafe) / static_cast<double>(cav)) << ",\n"
      << "  \"near_seam_terminations\": " << seam << ",\n"
      << "  \"segment_unsafe_terminations\": " << seg << ",\n"
      << "  \"unsafe_offset_terminations\": " << unsafe << ",\n"
      << "  \"mesh_build_seconds\": " << info.build_seconds << ",\n"
      << "  \"peak_rss_megabytes\": " << peak_rss_megabytes() << ",\n"
      << "  \"gpu_precision\": \"" << o.precision << "\",\n"
      << "  \"timings_seconds\": [";
  for (size_t i = 0; i < times.size(); ++i) {
    if (i) out << ", ";
    out << times[i];
  }
  out << "]\n}\n";
  std::cout << "TWoS B200 Differential WoS: " << n << " sites x " << o.walks << " walks, " << 4 * n_cav
            << " parameters, median " << runtime << " s\n";
  return 0;
}

// --mode validate (run_minimum_benefit, minimum_benefit.hpp:145-188): the
// per-sample CSV site,sample,value,steps,capped,clipped and the stage JSON;
// a containment failure fails the request after both are written.  The
// samples come from the validation stream (stream 2) of --seed.
int run_validate(const Options &o, twos_mesh *mesh, const twos_mesh_info &info, const std::vector<double> &points,
                 const std::vector<double> &cavities) {
  const size_t n = points.size() / 3, n_cav = cavities.size() / 3;
  twos_request r = base_request(o);
  r.precision = TWOS_PREC_FP64;
  r.stream = 2;
  twos_validate_params vp{o.validation_radius_cap, o.validation_value_cap};
  std::vector<twos_cert_sample> samples(n * static_cast<size_t>(o.walks));
  std::vector<twos_validate_stage> stages(n * TWOS_VALIDATE_MAX_STAGES);
  uint32_t n_stages = 0;
  twos_summary s{};
  const int rc = twos_validate(mesh, &r, &vp, points.data(), static_cast<uint32_t>(n), cavities.data(),
                               static_cast<uint32_t>(n_cav), samples.data(), stages.data(), &n_stages, &s);
  const bool containment = rc == TWOS_ERR_RUNTIME && s.error_flags == 0 && s.node_tests > 0;
  if (rc != TWOS_OK && !containment) throw_on(rc);
  std::ofstream output(o.output_path);
  if (!output) throw std::runtime_error("cannot write validation output: " + o.output_path);
  output << std::setprecision(17) << "site,sample,value,steps,capped,clipped\n";
  for (size_t i = 0; i < n; ++i)
    for (int j = 0; j < o.walks; ++j) {
      const twos_cert_sample &v = samples[i * o.walks + j];
      output << i << ',' << j << ',' << v.value << ',' << v.steps << ',' << int(v.capped) << ',' << int(v.clipped)
             << '\n';
    }
  std::ofstream summary(o.summary_path);
  if (!summary) throw std::runtime_error("cannot write summary: " + o.summary_path);
  summary << std::setprecision(17)
          << "{\"scope\":\"conditional ideal-sampling certificate; conservative box geometry and source "
             "arithmetic\",\n"
          << "\"distance_tree_build_seconds\":" << info.build_seconds
          << ",\n\"distance_mode\":\"triangle_AABB_union_lower_bound\",\n"
          << "\"sample_cap\":" << o.validation_value_cap << ",\"radius_cap\":" << o.validation_radius_cap
          << ",\"stages\":[\n";
  bool first = true;
  for (size_t i = 0; i < n; ++i)
    for (uint32_t k = 0; k < n_stages; ++k) {
      const twos_validate_stage &st = stages[i * TWOS_VALIDATE_MAX_STAGES + k];
      if (!first) summary << ",\n";
      first = false;
      // Device time apportioned to the stage's prefix of the site's walks.
      const double elapsed = s.kernel_seconds * (static_cast<double>(st.n) / o.walks) / static_cast<double>(n);
      summary << "{\"site\":" << st.site << ",\"n\":" << st.n << ",\"mean\":" << st.mean
              << ",\"mean_steps\":" << st.mean_steps << ",\"clipped\":" << st.clipped
              << ",\"path_caps\":" << st.path_caps << ",\"elapsed_seconds\":" << elapsed
              << ",\"center_clearance_lower\":" << st.center_clearance_lower
              << ",\"embree_center_distance\":" << st.center_distance << "}";
    }
  summary << "\n],\"containment_failures\":" << s.node_tests << "}\n";
  if (containment) throw std::runtime_error("sample containment guard failed; validation record must be rejected");
  return 0;
}

int run(const Options &o) {
  if (o.mode != "twos" && o.mode != "diffwos" && o.mode != "validate")
    throw std::runtime_error("mode " + o.mode + " is not provided by the TWoS B200 backend");
  if (o.mode == "validate") {
    MeshHandle mesh;
    throw_on(twos_mesh_open_ply(o.mesh_path.c_str(), o.device, &mesh.m));
    twos_mesh_info info{};
    throw_on(twos_mesh_get_info(mesh.m, &info));
    return run_validate(o, mesh.m, info, read_points(o.points_path), read_optional_points(o.cavities_path));
  }
  if (o.mode == "diffwos") {
    MeshHandle mesh;
    throw_on(twos_mesh_open_ply(o.mesh_path.c_str(), o.device, &mesh.m));
    twos_mesh_info info{};
    throw_on(twos_mesh_get_info(mesh.m, &info));
    return run_differential(o, mesh.m, info, read_points(o.points_path), read_optional_points(o.cavities_path));
  }
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
  uint64_t retained_steps = 0, retained_limits = 0, retained_grid_steps = 0;
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
      retained_grid_steps = s.grid_steps;
    }
  }
  if (retained_limits != 0) throw std::runtime_error("one or more paths hit --max-steps");
  write_field(o.output_path, points, retained);
  if (!o.trace_path.empty() && o.trace_sites > 0)
    std::cerr << "warning: --trace-output is not written by the TWoS B200 backend\n";
  write_summary(o.summary_path, info, cavities.size() / 3, o, n, times, kernel_times, retained_steps,
                retained_limits, retained_grid_steps);
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

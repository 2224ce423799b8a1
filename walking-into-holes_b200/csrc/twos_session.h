// The mesh session of libtwos.so and the host helpers its entry points share
// (twos_abi.cpp, noalloc.cu).  Not part of the public ABI.
#pragma once

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "twos_internal.h"

namespace twos {

// Records `msg` as this thread's last error and returns `code`.
int fail(int code, const std::string &msg);
// Throws std::runtime_error naming `what` when `e` is not cudaSuccess.
void check(cudaError_t e, const char *what);

// Grow-only device allocation.
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t n) {
    if (n <= bytes) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    check(cudaMalloc(&ptr, std::max<size_t>(n, 256)), "cudaMalloc");
    bytes = std::max<size_t>(n, 256);
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// What a group of launches reports back to the entry point that ran them.
struct RunOut {
  double kernel_seconds = 0.0;
  double walk_seconds = 0.0;
  uint32_t launches = 0;
  uint32_t error_flags = 0;
  uint64_t steps = 0, caps = 0;
  uint64_t node_tests = 0, plane_tests = 0, triangle_tests = 0, grid_steps = 0;
};

int validate_request(const twos_request *r, uint32_t n_sites, uint32_t n_cav, bool allow_boundary = false);
// Fills `summary` (when not NULL) from `ro` and maps device error bits and
// step caps onto the ABI's return codes and last-error messages.
int finish(const RunOut &ro, uint32_t n_sites, const twos_request *r, twos_summary *summary, double t_total,
           uint64_t h2d, uint64_t d2h);
JobDesc make_job(twos_mesh *mesh, const twos_request *r, uint32_t n_sites, uint32_t site_begin,
                 uint32_t site_offset, uint32_t geo, uint64_t walk_begin, uint32_t site_rank, uint32_t cav_begin,
                 uint32_t n_cav, std::vector<TermDev> &terms);

}  // namespace twos

struct twos_mesh {
  int device = 0;
  std::vector<double> vertices;
  std::vector<uint32_t> faces;
  twos::HostBvh bvh;
  double bmin[3], bmax[3], center[3];
  double delta = 0.0;
  double build_seconds = 0.0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;  // stream in use
  cudaStream_t own_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evw = nullptr;
  twos::DevBuf nodes_f, tris_f, nodes_d, tris_d;
  twos::DevBuf grid;   // distance-bound grid (16-byte corner record per cell), may be empty
  twos::DevBuf nodes4_f;  // the four-wide BVH (mixed form, bvh_width 4)
  twos::DevBuf geo;  // one GeoDesc
  twos::GeoDesc geo_host{};
  uint64_t resident_bytes = 0;
  // Scratch, grown on demand.
  twos::DevBuf jobs, geos, terms, cavities, sites, out, u, p, grad, steps, first, counter, totals, points, dist, closest,
      topk, wf;
  size_t max_launch_walks = size_t(1) << 30;
  int block = 128;         // walk-kernel threads per block
  int refill = 1;          // lanes idle before a warp refills from the queue
  int step_threshold = 1;  // finished queries before a warp takes its walk step
  int blocks_per_sm = 0;   // 0: as many as fit
  int vote = 0;            // 1: one kind of traversal unit per warp iteration
  int warm = 1;            // 1: seed each step's query with the previous nearest triangle
  float grid_tau = 0.1f;   // mixed-form grid steps need a bound of this many spacings; 0 = off
  int units = 8;           // traversal units per lane per warp-loop iteration
  int lane_walks = 1;      // walks a lane claims from the queue at once
  uint32_t wavefront = 0;  // > 0: mixed centre-source walks run in the wavefront form with this many slots
  int entry_start = 1;     // 1: mixed-form queries start at the entry-node table's node
  int grid_fp64 = 0;       // 1: the FP64 compliance form uses the grid and entry nodes too
  int bvh_width = 2;       // mixed form: 2 (binary) or 4 (four-wide) BVH traversal
};

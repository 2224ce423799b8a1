// Device side of the design loop: scout -> top-k shortlist -> fresh
// validation -> lower-confidence-bound choice -> accept/reject -> insert a
// ball cavity, with every decision taken on the device so a whole iteration
// can be captured once as a CUDA graph and replayed.
//
// Follows select_twos (benchmarks/stanford_bunny/run_bunny_benchmark.py:302-337):
// feasible candidates are scouted, the top `k` by scout score are rescored
// with fresh samples, lower = score - z * se, and the argmax of lower is the
// choice (run_bunny_benchmark.py:330-331); here the choice is inserted only
// when lower > threshold (the accept test of
// benchmarks/minimum_benefit/run_application_validation.py:221, 245-248 with a
// normal bound), and candidates closer than the pair clearance to an inserted
// cavity become infeasible (feasible_mask, run_bunny_benchmark.py:290-299).
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>

#include "twos_internal.h"

namespace twos {

__global__ void design_keys_kernel(const DesignLaunch D) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n_candidates; i += gridDim.x * blockDim.x) {
    const double s = D.scout_rows[i].score;
    D.keys[i] = (D.feasible[i] && !isnan(s)) ? s : -CUDART_INF;
  }
}

__global__ void design_gather_kernel(const DesignLaunch D) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < D.k; j += gridDim.x * blockDim.x) {
    const uint32_t c = D.shortlist[j];
    const bool ok = c < D.n_candidates;
    for (int a = 0; a < 3; ++a) D.val_sites[3 * j + a] = ok ? D.candidates[3 * c + a] : 0.0;
  }
}

// One warp: argmax of lower = score - z*se over the shortlist (ties to the
// earlier shortlist slot, i.e. the higher scout score), the accept test and
// the insertion.  The next iteration's sample keys advance with `repeat`.
__global__ void design_select_kernel(const DesignLaunch D) {
  const unsigned lane = threadIdx.x & 31u;
  double best = -CUDART_INF;
  uint32_t arg = 0xffffffffu;
  for (uint32_t j = lane; j < D.k; j += 32) {
    const twos_site_result r = D.val_rows[j];
    const double lower = r.score - D.z * r.score_se;
    if (!isnan(lower) && D.shortlist[j] < D.n_candidates && (arg == 0xffffffffu || lower > best)) {
      best = lower;
      arg = j;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const uint32_t oa = __shfl_xor_sync(0xffffffffu, arg, o);
    if (oa != 0xffffffffu && (arg == 0xffffffffu || ob > best || (ob == best && oa < arg))) {
      best = ob;
      arg = oa;
    }
  }
  if (lane != 0) return;
  const uint32_t it = *D.iteration;
  DesignStep h;
  h.chosen = 0xffffffffu;
  h.accepted = 0u;
  h.scout_score = CUDART_NAN;
  h.score = CUDART_NAN;
  h.score_se = CUDART_NAN;
  h.lower = CUDART_NAN;
  h.slot = 0xffffffffu;
  h.n_cavities = D.scout_job->n_cav;
  if (arg != 0xffffffffu) {
    const uint32_t c = D.shortlist[arg];
    const twos_site_result r = D.val_rows[arg];
    h.chosen = c;
    h.slot = arg;
    h.scout_score = D.scout_rows[c].score;
    h.score = r.score;
    h.score_se = r.score_se;
    h.lower = best;
    const uint32_t n_cav = D.scout_job->n_cav;
    if (best > D.threshold && n_cav < D.max_cav) {
      h.accepted = 1u;
      for (int a = 0; a < 3; ++a) D.cavities[3 * n_cav + a] = D.candidates[3 * c + a];
      D.scout_job->n_cav = n_cav + 1;
      D.val_job->n_cav = n_cav + 1;
    }
  }
  if (it < D.max_iterations) D.history[it] = h;
  D.scout_job->repeat = it + 1;
  D.val_job->repeat = it + 1;
  *D.iteration = it + 1;
}

// Candidates within the pair clearance of a cavity inserted this iteration
// become infeasible.
__global__ void design_mask_kernel(const DesignLaunch D) {
  const uint32_t it = *D.iteration;
  if (it == 0 || it > D.max_iterations) return;
  const DesignStep h = D.history[it - 1];
  if (!h.accepted) return;
  const uint32_t n_cav = D.scout_job->n_cav;
  const double *c = D.cavities + 3ull * (n_cav - 1);
  const double r2 = D.pair_clearance * D.pair_clearance;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n_candidates; i += gridDim.x * blockDim.x) {
    const double dx = D.candidates[3 * i] - c[0], dy = D.candidates[3 * i + 1] - c[1],
                 dz = D.candidates[3 * i + 2] - c[2];
    if (dx * dx + dy * dy + dz * dz < r2) D.feasible[i] = 0;
  }
}

static int blocks_for(uint32_t n) { return static_cast<int>(std::min<uint32_t>((n + 255) / 256, 148u * 8)); }

cudaError_t launch_design_keys(const DesignLaunch &D, cudaStream_t s) {
  design_keys_kernel<<<blocks_for(D.n_candidates), 256, 0, s>>>(D);
  return cudaGetLastError();
}
cudaError_t launch_design_gather(const DesignLaunch &D, cudaStream_t s) {
  design_gather_kernel<<<blocks_for(D.k), 256, 0, s>>>(D);
  return cudaGetLastError();
}
cudaError_t launch_design_select(const DesignLaunch &D, cudaStream_t s) {
  design_select_kernel<<<1, 32, 0, s>>>(D);
  return cudaGetLastError();
}
cudaError_t launch_design_mask(const DesignLaunch &D, cudaStream_t s) {
  design_mask_kernel<<<blocks_for(D.n_candidates), 256, 0, s>>>(D);
  return cudaGetLastError();
}

}  // namespace twos

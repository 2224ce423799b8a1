// twos_estimate_noalloc: the device-buffer estimator without any device
// allocation, for callers that cannot call cudaMalloc -- code that runs while
// a framework owns the device memory pool (a raw cudaMalloc bypasses its
// allocator and fragments memory it manages), and long-running services with
// a fixed device-memory budget that must not grow per request.
//
// All per-call device scratch of an estimate -- the launch's job, geometry and
// term tables, the cavities, the per-site first-query distances, the work-
// queue counter, the totals/error words and the per-walk sample buffers -- is
// carved out of one file-scope static device array of kNoallocScratchBytes
// (16 MiB).  Every GPU that loads the library holds this array until the
// process exits.  The caller passes the sites and the result rows (device
// memory) and a mesh session opened earlier.  The call returns after the work
// on the session's stream has completed, and reports errors and its summary
// through the same mapping as twos_estimate_device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <limits>
#include <mutex>

#include "twos_session.h"

namespace twos {

constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
static_assert(kNoallocScratchBytes == TWOS_NOALLOC_SCRATCH_BYTES, "header and library disagree");

// The scratch.  In host code this name is only a host-side stand-in; its
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on `device` (which must be current), looked
// up once per device.
void *scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices) throw std::runtime_error("device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    void *ptr = nullptr;
    check(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(no-allocation scratch)");
    g_scratch_ptr[device] = ptr;
  }
  return g_scratch_ptr[device];
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
  size_t totals, counter, job, geo, terms, cav, first, u, p, steps, end;
};

Layout plan(size_t n_terms, size_t n_cav, size_t n_sites, size_t walks_total, size_t vbytes, bool paired) {
  Layout L{};
  size_t at = 0;
  L.totals = at;
  at = align256(at + 8 * sizeof(unsigned long long));
  L.counter = at;
  at = align256(at + sizeof(unsigned long long));
  L.job = at;
  at = align256(at + sizeof(JobDesc));
  L.geo = at;
  at = align256(at + sizeof(GeoDesc));
  L.terms = at;
  at = align256(at + std::max<size_t>(1, n_terms) * sizeof(TermDev));
  L.cav = at;
  at = align256(at + std::max<size_t>(1, n_cav) * 3 * sizeof(double));
  L.first = at;
  at = align256(at + n_sites * sizeof(double));
  L.u = at;
  at = align256(at + walks_total * vbytes);
  L.p = at;
  if (paired) at = align256(at + walks_total * vbytes);
  L.steps = at;
  at = align256(at + walks_total * sizeof(uint32_t));
  L.end = at;
  return L;
}

}  // namespace
}  // namespace twos

using namespace twos;

extern "C" int twos_estimate_noalloc(twos_mesh *m, const twos_request *r, const double *d_sites, uint32_t n_sites,
                                     const double *cavities, uint32_t n_cavities, twos_site_result *d_out,
                                     twos_summary *summary) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  if (int rc = validate_request(r, n_sites, n_cavities)) return rc;
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!d_sites || !d_out || (n_cavities && !cavities)) return fail(TWOS_ERR_USAGE, "null buffer");
  const bool mixed = r->precision == TWOS_PREC_MIXED;
  const bool paired = r->mode == TWOS_MODE_PAIRED;
  const size_t vbytes = mixed ? sizeof(float) : sizeof(double);
  const size_t walks_total = static_cast<size_t>(n_sites) * static_cast<size_t>(r->walks);
  const Layout lay = plan(static_cast<size_t>(r->n_source + r->n_adjoint), n_cavities, n_sites, walks_total, vbytes,
                          paired);
  if (lay.end > kNoallocScratchBytes) {
    const size_t per_walk = vbytes * (paired ? 2 : 1) + sizeof(uint32_t);
    return fail(TWOS_ERR_USAGE, "request needs " + std::to_string(lay.end) +
                                    " bytes of scratch; twos_estimate_noalloc holds " +
                                    std::to_string(kNoallocScratchBytes) + " (about " +
                                    std::to_string(kNoallocScratchBytes / per_walk) +
                                    " walks per call at this mode and precision)");
  }
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    unsigned char *base = static_cast<unsigned char *>(scratch_address(m->device));
    std::vector<TermDev> terms;
    const JobDesc J = make_job(m, r, n_sites, 0, r->site_offset, 0, 0, 0, 0, n_cavities, terms);
    if (terms.empty()) terms.push_back(TermDev{});
    cudaStream_t st = m->stream;
    // The array keeps the previous call's contents: everything the kernels
    // read is written here first, and the counters start at zero.
    check(cudaMemsetAsync(base + lay.totals, 0, 8 * sizeof(unsigned long long), st), "memset");
    check(cudaMemsetAsync(base + lay.counter, 0, sizeof(unsigned long long), st), "memset");
    check(cudaMemcpyAsync(base + lay.job, &J, sizeof(JobDesc), cudaMemcpyHostToDevice, st), "upload job");
    check(cudaMemcpyAsync(base + lay.geo, &m->geo_host, sizeof(GeoDesc), cudaMemcpyHostToDevice, st), "upload geo");
    check(cudaMemcpyAsync(base + lay.terms, terms.data(), terms.size() * sizeof(TermDev), cudaMemcpyHostToDevice, st),
          "upload terms");
    if (n_cavities)
      check(cudaMemcpyAsync(base + lay.cav, cavities, n_cavities * 3 * sizeof(double), cudaMemcpyHostToDevice, st),
            "upload cavities");
    unsigned long long *totals = reinterpret_cast<unsigned long long *>(base + lay.totals);
    WosLaunch L{};
    L.jobs = reinterpret_cast<JobDesc *>(base + lay.job);
    L.n_jobs = 1;
    L.geos = reinterpret_cast<GeoDesc *>(base + lay.geo);
    L.n_geos = 1;
    L.sites = d_sites;
    L.terms = reinterpret_cast<TermDev *>(base + lay.terms);
    L.n_terms = static_cast<uint32_t>(terms.size());
    L.cavities = reinterpret_cast<double *>(base + lay.cav);
    L.total_walks = walks_total;
    L.counter = reinterpret_cast<unsigned long long *>(base + lay.counter);
    L.error = reinterpret_cast<uint32_t *>(totals + 2);
    L.u_out = base + lay.u;
    L.p_out = paired ? base + lay.p : nullptr;
    L.steps_out = reinterpret_cast<uint32_t *>(base + lay.steps);
    L.refill = m->refill;
    L.step_threshold = m->step_threshold;
    L.vote = m->vote;
    L.warm = m->warm;
    L.grid_tau = m->grid_tau;
    L.units = m->units;
    L.lane_walks = m->lane_walks;
    L.entry = m->entry_start;
    L.grid64 = m->grid_fp64;
    L.wide = m->bvh_width == 4;
    L.counters = totals + 3;
    L.site_best2 = base + lay.first;
    L.total_sites = n_sites;
    const int block = m->block;
    const int per_sm = wos_max_blocks_per_sm(r->precision, r->mode, r->green, block, L);
    if (per_sm <= 0) throw std::runtime_error("WoS kernel cannot be resident on this device");
    const int grid = std::min(per_sm, m->blocks_per_sm > 0 ? m->blocks_per_sm : per_sm) * m->num_sms;
    FinalizeLaunch F{};
    F.jobs = L.jobs;
    F.n_jobs = 1;
    F.total_sites = n_sites;
    F.totals = totals;
    F.u = L.u_out;
    F.p = L.p_out;
    F.steps = L.steps_out;
    F.out = d_out;
    check(cudaEventRecord(m->ev0, st), "event");
    check(launch_site_prepass(r->precision, L, st), "site pre-pass");
    check(launch_wos(r->precision, r->mode, r->green, L, grid, block, st), "WoS launch");
    check(cudaEventRecord(m->evw, st), "event");
    check(launch_finalize(r->precision, r->mode, F, st), "finalize launch");
    check(cudaEventRecord(m->ev1, st), "event");
    unsigned long long tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    check(cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, st), "download totals");
    check(cudaStreamSynchronize(st), "WoS kernels");
    float ms = 0.f, msw = 0.f;
    check(cudaEventElapsedTime(&ms, m->ev0, m->ev1), "event time");
    check(cudaEventElapsedTime(&msw, m->ev0, m->evw), "event time");
    ro.kernel_seconds = ms * 1e-3;
    ro.walk_seconds = msw * 1e-3;
    ro.launches = 3;
    ro.steps = tot[0];
    ro.caps = tot[1];
    std::memcpy(&ro.error_flags, &tot[2], sizeof(uint32_t));
    ro.node_tests = tot[3];
    ro.plane_tests = tot[4];
    ro.triangle_tests = tot[5];
    ro.grid_steps = tot[6];
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return finish(ro, n_sites, r, summary, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(),
                0, 0);
}

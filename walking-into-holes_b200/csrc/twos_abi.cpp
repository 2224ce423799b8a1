// C ABI of libtwos.so (include/twos.h): mesh sessions, request validation,
// device memory, chunked kernel launches and the mapping of device error bits
// and step caps onto the reference's error behaviour.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "twos_session.h"

namespace twos {

static thread_local std::string g_error;

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

void counter_key(uint64_t seed, uint32_t stream, uint32_t &k0, uint32_t &k1) {
  uint64_t x = seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(stream) + 1);
  // SplitMix64 finaliser (Steele, Lea & Flood 2014).
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30U)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27U)) * 0x94d049bb133111ebULL;
  x = x ^ (x >> 31U);
  k0 = static_cast<uint32_t>(x);
  k1 = static_cast<uint32_t>(x >> 32);
}

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace twos

using namespace twos;

namespace twos {

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Sizes and fills the mixed form's distance-bound grid of a session whose
// BVH is on the device and whose geo_host describes it (m->geo allocated).
// About 1024 vertices per triangle, at most 2^28 (4 GB of 16-byte cell
// records; 512 MB of vertex values while it is built), over the bounding
// box padded by one spacing (environment TWOS_GRID_VERTICES sets the count,
// up to 2^30; 0 builds none).  On the 327,680-triangle noise sphere the walk
// kernel took 2.42 / 2.32 / 2.17 / 2.11 / 2.08 s with 2^25 / 2^26 / 2^27 /
// 2^28 / 2^29 vertices (entry cells of one spacing from 2^26 up): a finer
// grid answers more steps and its entry cells start queries deeper.  2^28
// keeps the mesh open within a few seconds.
// Values are FP32 distances less 2 delta (the mixed form's own error bound,
// covering the FP32 query and the vertex placement), in steps of h/128.
std::vector<int32_t> build_entry_table(twos_mesh *m);

void build_distance_grid(twos_mesh *m, size_t n_tris) {
  GeoDesc &g = m->geo_host;
  g.grid = nullptr;
  uint64_t target = std::min<uint64_t>(std::max<uint64_t>(1024ull * n_tris, 4096ull), 1ull << 28);
  if (const char *e = std::getenv("TWOS_GRID_VERTICES"))
    target = std::min<uint64_t>(std::strtoull(e, nullptr, 10), 1ull << 30);
  const uint64_t cap = std::max<uint64_t>(target, 1ull << 25);
  double ext[3], emax = 0.0;
  for (int a = 0; a < 3; ++a) {
    ext[a] = m->bmax[a] - m->bmin[a];
    emax = std::max(emax, ext[a]);
  }
  if (target < 64 || !(emax > 0.0)) return;
  double vol = 1.0;
  for (int a = 0; a < 3; ++a) vol *= std::max(ext[a], 1e-3 * emax);
  double h = std::cbrt(vol / static_cast<double>(target));
  uint64_t n[3];
  for (int it = 0;; ++it) {
    for (int a = 0; a < 3; ++a) n[a] = static_cast<uint64_t>(std::ceil(ext[a] / h)) + 3;
    const uint64_t total = n[0] * n[1] * n[2];
    if ((total <= target + target / 2 && total <= cap) || it > 200) break;
    h *= 1.03;
  }
  if (n[0] * n[1] * n[2] > cap) return;
  for (int a = 0; a < 3; ++a) {
    g.grid_lo[a] = static_cast<float>(m->bmin[a] - h - m->center[a]);
    g.grid_n[a] = static_cast<uint32_t>(n[a]);
  }
  g.grid_h = static_cast<float>(h);
  g.grid_inv_h = 1.0f / g.grid_h;
  g.grid_q = g.grid_h / 128.0f;
  const uint64_t count = n[0] * n[1] * n[2];
  const uint64_t cells = (n[0] - 1) * (n[1] - 1) * (n[2] - 1);
  check(cudaMemcpy(m->geo.ptr, &g, sizeof(GeoDesc), cudaMemcpyHostToDevice), "upload");
  // Per-vertex values first, then the per-cell records the walks read.
  DevBuf values;
  struct Release {
    DevBuf &b;
    ~Release() { b.release(); }
  } release_values{values};
  values.reserve(count * sizeof(uint16_t));
  uint32_t *err = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
  check(cudaMemset(err, 0, sizeof(uint32_t)), "memset");
  check(launch_grid_build(m->geo.as<GeoDesc>(), count, 2.0 * m->delta, values.as<uint16_t>(), err, nullptr),
        "grid build");
  check(cudaDeviceSynchronize(), "grid build");
  uint32_t build_err = 0;
  check(cudaMemcpy(&build_err, err, sizeof(uint32_t), cudaMemcpyDeviceToHost), "download");
  if (build_err) {
    // A vertex whose query overran its bounds holds 0: still a lower bound,
    // but no upper bound, so the session runs without the grid.
    return;
  }
  // The entry-node table, folded into the records with the corner values.
  const std::vector<int32_t> table = build_entry_table(m);
  DevBuf dtable;
  struct Release2 {
    DevBuf &b;
    ~Release2() { b.release(); }
  } release_table{dtable};
  if (!table.empty()) {
    dtable.reserve(table.size() * sizeof(int32_t));
    check(cudaMemcpy(dtable.ptr, table.data(), table.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "upload");
  }
  m->grid.reserve(cells * sizeof(uint4));
  check(launch_grid_pack(values.as<uint16_t>(), g.grid_n, table.empty() ? nullptr : dtable.as<int32_t>(),
                         g.entry_shift, g.entry_n, m->grid.as<uint4>(), nullptr),
        "grid pack");
  check(cudaDeviceSynchronize(), "grid pack");
  g.grid = m->grid.as<uint4>();
  m->resident_bytes += cells * sizeof(uint4);
}

// The entry-node table over the distance grid: cells of 2^s grid spacings
// (by default one spacing while the table takes at most 1 GiB -- 1 GiB for
// 2^28 grid vertices -- else two; TWOS_ENTRY_CELLS sets 1, 2, 4, 8 or 16, 0
// builds none), each with the node whose subtree holds every triangle within
// one cell size (plus 4 delta) of the cell.  A query whose initial bound is
// below one cell size starts there instead of at the root.  Built on the
// host; the grid's cell records carry it (empty: no table).
std::vector<int32_t> build_entry_table(twos_mesh *m) {
  GeoDesc &g = m->geo_host;
  const uint64_t vertices = static_cast<uint64_t>(g.grid_n[0]) * g.grid_n[1] * g.grid_n[2];
  uint32_t shift = vertices * sizeof(int32_t) <= (1ull << 30) ? 0 : 1;
  if (const char *e = std::getenv("TWOS_ENTRY_CELLS")) {
    const long c = std::strtol(e, nullptr, 10);
    if (c <= 0) return {};
    shift = 0;
    while (shift < 4 && (1L << (shift + 1)) <= c) ++shift;
  }
  const uint32_t c = 1u << shift;
  const double h = static_cast<double>(g.grid_h);
  double origin[3];
  for (int a = 0; a < 3; ++a) {
    origin[a] = static_cast<double>(g.grid_lo[a]) + m->center[a];
    g.entry_n[a] = (g.grid_n[a] - 1 + c - 1) / c;
  }
  const double cell = c * h;
  g.entry_shift = shift;
  g.entry_radius = static_cast<float>(cell);
  return twos::build_entry_table(m->bvh, origin, cell, g.entry_n, cell + 4.0 * m->delta, 0.01 * h);
}

int open_impl(std::vector<double> &&v, std::vector<uint32_t> &&f, int device, twos_mesh **out) {
  if (!out) return fail(TWOS_ERR_USAGE, "null output pointer");
  *out = nullptr;
  if (f.empty() || v.empty()) return fail(TWOS_ERR_USAGE, "expected a nonempty triangle mesh");
  const size_t nv = v.size() / 3;
  for (uint32_t idx : f)
    if (idx >= nv) return fail(TWOS_ERR_USAGE, "face index out of range");
  for (double x : v)
    if (!std::isfinite(x)) return fail(TWOS_ERR_USAGE, "non-finite vertex coordinate");
  auto m = std::make_unique<twos_mesh>();
  m->device = device;
  m->vertices = std::move(v);
  m->faces = std::move(f);
  try {
    check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop;
    check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    m->num_sms = prop.multiProcessorCount;
    const auto t0 = std::chrono::steady_clock::now();
    for (int a = 0; a < 3; ++a) {
      m->bmin[a] = std::numeric_limits<double>::infinity();
      m->bmax[a] = -std::numeric_limits<double>::infinity();
    }
    for (size_t i = 0; i < nv; ++i)
      for (int a = 0; a < 3; ++a) {
        m->bmin[a] = std::min(m->bmin[a], m->vertices[3 * i + a]);
        m->bmax[a] = std::max(m->bmax[a], m->vertices[3 * i + a]);
      }
    double reach = 0.0;
    for (int a = 0; a < 3; ++a) {
      m->center[a] = 0.5 * (m->bmin[a] + m->bmax[a]);
      reach = std::max(reach, 0.5 * (m->bmax[a] - m->bmin[a]));
    }
    // FP32 distance error bound for the mixed form: coordinates within
    // `reach` of the centre carry at most ulp(reach)/2 representation error
    // each; the closest-point arithmetic adds a few ulps.  32 * 2^-24 * reach
    // covers both with margin (checked against FP64 in the tests).
    m->delta = 32.0 * std::ldexp(1.0, -24) * std::max(reach, 1e-30);
    build_bvh(m->vertices, m->faces, m->bvh);
    std::vector<NodeF> nf;
    std::vector<TriF> tf;
    std::vector<NodeD> nd;
    std::vector<TriD> td;
    pack_bvh_f32(m->bvh, m->vertices, m->faces, m->center, nf, tf);
    std::vector<Node4F> n4;
    std::vector<int32_t> cover4;
    pack_bvh4_f32(m->bvh, nf, n4, cover4);
    pack_bvh_f64(m->bvh, m->vertices, m->faces, nd, td);
    check(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    m->stream = m->own_stream;
    check(cudaEventCreate(&m->ev0), "cudaEventCreate");
    check(cudaEventCreate(&m->ev1), "cudaEventCreate");
    check(cudaEventCreate(&m->evw), "cudaEventCreate");
    m->nodes_f.reserve(nf.size() * sizeof(NodeF));
    m->tris_f.reserve(tf.size() * sizeof(TriF));
    m->nodes_d.reserve(nd.size() * sizeof(NodeD));
    m->tris_d.reserve(td.size() * sizeof(TriD));
    check(cudaMemcpy(m->nodes_f.ptr, nf.data(), nf.size() * sizeof(NodeF), cudaMemcpyHostToDevice), "upload");
    m->nodes4_f.reserve(n4.size() * sizeof(Node4F));
    check(cudaMemcpy(m->nodes4_f.ptr, n4.data(), n4.size() * sizeof(Node4F), cudaMemcpyHostToDevice), "upload");
    check(cudaMemcpy(m->tris_f.ptr, tf.data(), tf.size() * sizeof(TriF), cudaMemcpyHostToDevice), "upload");
    check(cudaMemcpy(m->nodes_d.ptr, nd.data(), nd.size() * sizeof(NodeD), cudaMemcpyHostToDevice), "upload");
    check(cudaMemcpy(m->tris_d.ptr, td.data(), td.size() * sizeof(TriD), cudaMemcpyHostToDevice), "upload");
    m->resident_bytes = nf.size() * sizeof(NodeF) + n4.size() * sizeof(Node4F) + tf.size() * sizeof(TriF) +
                        nd.size() * sizeof(NodeD) +
                        td.size() * sizeof(TriD);
    GeoDesc &g = m->geo_host;
    g.nodes_f = m->nodes_f.as<NodeF>();
    g.nodes4_f = m->nodes4_f.as<Node4F>();
    g.tris_f = m->tris_f.as<TriF>();
    g.nodes_d = m->nodes_d.as<NodeD>();
    g.tris_d = m->tris_d.as<TriD>();
    for (int a = 0; a < 3; ++a) g.center[a] = m->center[a];
    g.delta = static_cast<float>(m->delta);
    // A query visits each node and tests each triangle at most once.
    g.max_iter = static_cast<uint32_t>(
        std::min<uint64_t>(2ull * (m->bvh.nodes.size() + m->faces.size() / 3) + 16, 0xffffffffull));
    m->geo.reserve(sizeof(GeoDesc));
    m->counter.reserve(16);
    m->totals.reserve(64);
    build_distance_grid(m.get(), tf.size());
    check(cudaMemcpy(m->geo.ptr, &g, sizeof(GeoDesc), cudaMemcpyHostToDevice), "upload");
    m->build_seconds = seconds_since(t0);
    if (const char *e = std::getenv("TWOS_MAX_LAUNCH_WALKS")) m->max_launch_walks = std::strtoull(e, nullptr, 10);
    if (const char *e = std::getenv("TWOS_REFILL")) m->refill = std::max(1, std::atoi(e));
    if (const char *e = std::getenv("TWOS_STEP_THRESHOLD")) m->step_threshold = std::max(1, std::atoi(e));
    if (const char *e = std::getenv("TWOS_BLOCKS_PER_SM")) m->blocks_per_sm = std::max(0, std::atoi(e));
    if (const char *e = std::getenv("TWOS_VOTE")) m->vote = std::atoi(e) != 0;
    if (const char *e = std::getenv("TWOS_WARM")) m->warm = std::atoi(e) != 0;
    if (const char *e = std::getenv("TWOS_UNITS")) m->units = std::min(64, std::max(1, std::atoi(e)));
    if (const char *e = std::getenv("TWOS_LANE_WALKS")) m->lane_walks = std::min(64, std::max(1, std::atoi(e)));
    if (const char *e = std::getenv("TWOS_WAVEFRONT")) {
      const long v = std::atol(e);
      if (v >= 0 && v <= (1l << 26) && v % 256 == 0) m->wavefront = static_cast<uint32_t>(v);
    }
    if (const char *e = std::getenv("TWOS_ENTRY")) m->entry_start = std::atoi(e) != 0;
    if (const char *e = std::getenv("TWOS_BVH_WIDTH")) m->bvh_width = std::atoi(e) == 4 ? 4 : 2;
    if (const char *e = std::getenv("TWOS_BLOCK")) {
      const int b = std::atoi(e);
      if (b == 128 || b == 256 || b == 512) m->block = b;
    }
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  *out = m.release();
  return TWOS_OK;
}

int validate_request(const twos_request *r, uint32_t n_sites, uint32_t n_cav, bool allow_boundary) {
  if (!r) return fail(TWOS_ERR_USAGE, "null request");
  if (r->mode < 0 || r->mode > 2) return fail(TWOS_ERR_USAGE, "invalid mode");
  if (r->precision != TWOS_PREC_FP64 && r->precision != TWOS_PREC_MIXED)
    return fail(TWOS_ERR_USAGE, "invalid precision");
  if (r->walks < 2) return fail(TWOS_ERR_USAGE, "walks must be at least 2");
  if (r->max_steps < 1) return fail(TWOS_ERR_USAGE, "max_steps must be at least 1");
  if (!(r->epsilon > 0.0)) return fail(TWOS_ERR_USAGE, "epsilon must be positive");
  if (r->cavity_radius < 0.0 || (n_cav > 0 && !(r->cavity_radius > 0.0)))
    return fail(TWOS_ERR_USAGE, "cavities need a positive cavity radius");
  if (r->n_source < 0 || r->n_source > TWOS_MAX_TERMS || r->n_adjoint < 0 || r->n_adjoint > TWOS_MAX_TERMS)
    return fail(TWOS_ERR_USAGE, "too many source terms");
  for (int i = 0; i < r->n_source + r->n_adjoint; ++i) {
    const twos_source_term &t = i < r->n_source ? r->source[i] : r->adjoint[i - r->n_source];
    if (t.kind < TWOS_TERM_CONST || t.kind > TWOS_TERM_QUAD) return fail(TWOS_ERR_USAGE, "unknown source term");
    if (t.kind == TWOS_TERM_LINEAR && (t.axis < 0 || t.axis > 2)) return fail(TWOS_ERR_USAGE, "bad term axis");
    if (r->green == TWOS_SOURCE_EXACT && t.kind != TWOS_TERM_CONST && t.kind != TWOS_TERM_LINEAR &&
        t.kind != TWOS_TERM_BUMP)
      return fail(TWOS_ERR_USAGE, "the exact source integral takes constant, linear and bump terms only");
  }
  if (r->green < TWOS_SOURCE_CENTER || r->green > TWOS_SOURCE_EXACT)
    return fail(TWOS_ERR_USAGE, "invalid source integration mode");
  if (r->n_boundary > TWOS_MAX_TERMS) return fail(TWOS_ERR_USAGE, "too many boundary terms");
  if (r->n_boundary && !allow_boundary)
    return fail(TWOS_ERR_USAGE, "Dirichlet boundary data is taken by twos_estimate_gradient");
  for (uint32_t i = 0; i < r->n_boundary; ++i) {
    const twos_source_term &t = r->boundary[i];
    if (t.kind < TWOS_TERM_CONST || t.kind > TWOS_TERM_QUAD) return fail(TWOS_ERR_USAGE, "unknown boundary term");
    if (t.kind == TWOS_TERM_LINEAR && (t.axis < 0 || t.axis > 2)) return fail(TWOS_ERR_USAGE, "bad term axis");
  }
  if (n_cav > 4096) return fail(TWOS_ERR_USAGE, "at most 4096 cavities per request");
  (void)n_sites;
  return TWOS_OK;
}

// Translates a term into the FP32 frame about `c` (identity for FP64).
TermDev frame_term(const twos_source_term &t, const double c[3]) {
  TermDev d;
  std::memcpy(&d, &t, sizeof(d));
  switch (t.kind) {
    case TWOS_TERM_LINEAR:
      d.offset = t.offset + c[t.axis];
      break;
    case TWOS_TERM_GAUSS:
    case TWOS_TERM_BUMP:
    case TWOS_TERM_BALL:
    case TWOS_TERM_QUAD:
      for (int a = 0; a < 3; ++a) d.c[a] = t.c[a] - c[a];
      break;
    case TWOS_TERM_BOX:
      for (int a = 0; a < 3; ++a) {
        d.c[a] = t.c[a] - c[a];
        d.w[a] = t.w[a] - c[a];
      }
      break;
    default:
      break;
  }
  return d;
}

// The device descriptor of one job; its source terms are appended to `terms`
// in the job geometry's frame.
JobDesc make_job(twos_mesh *mesh, const twos_request *r, uint32_t n_sites, uint32_t site_begin,
                 uint32_t site_offset, uint32_t geo, uint64_t walk_begin, uint32_t site_rank, uint32_t cav_begin,
                 uint32_t n_cav, std::vector<TermDev> &terms) {
  const double zero[3] = {0.0, 0.0, 0.0};
  const double *frame = r->precision == TWOS_PREC_MIXED ? mesh->center : zero;
  JobDesc J{};
  J.walk_begin = walk_begin;
  J.n_sites = n_sites;
  J.walks = static_cast<uint32_t>(r->walks);
  J.site_begin = site_begin;
  J.site_offset = site_offset;
  J.geo = geo;
  counter_key(r->seed, r->stream, J.k0, J.k1);
  J.repeat = r->repeat;
  J.max_steps = r->max_steps;
  J.flags = (r->green == TWOS_SOURCE_GREEN ? kJobGreen : 0u) |
            (r->green == TWOS_SOURCE_EXACT ? kJobExactSource : 0u) |
            (r->skip_cavity_sites ? kJobSkipCavitySites : 0u);
  J.epsilon = r->epsilon;
  const double qr = r->query_radius > 0.0 ? r->query_radius : std::numeric_limits<double>::infinity();
  J.query_radius2 = qr * qr;
  J.cavity_radius = r->cavity_radius;
  J.src_begin = static_cast<uint32_t>(terms.size());
  J.n_src = static_cast<uint32_t>(r->n_source);
  for (int i = 0; i < r->n_source; ++i) terms.push_back(frame_term(r->source[i], frame));
  J.adj_begin = static_cast<uint32_t>(terms.size());
  J.n_adj = static_cast<uint32_t>(r->n_adjoint);
  for (int i = 0; i < r->n_adjoint; ++i) terms.push_back(frame_term(r->adjoint[i], frame));
  J.cav_begin = cav_begin;
  J.n_cav = n_cav;
  J.site_rank = site_rank;
  J.bnd_begin = static_cast<uint32_t>(terms.size());
  J.n_bnd = r->n_boundary;
  for (uint32_t i = 0; i < r->n_boundary; ++i) terms.push_back(frame_term(r->boundary[i], frame));
  return J;
}

// One job of a launch plan, before device layout.
struct JobSpec {
  twos_mesh *mesh;
  const twos_request *r;
  uint32_t n_sites;
  uint32_t site_begin;   // into the launch's site / result arrays
  uint32_t site_offset;  // RNG site index base
  const double *cav;     // host cavities
  uint32_t n_cav;
};

// Runs one persistent launch over a group of jobs (walk kernel + finalize)
// on `owner`'s stream; sites and rows are device arrays indexed by
// JobSpec::site_begin.  All jobs share mode, precision and the Green flag.
// A device record of every grid step of a launch (tests).
struct TraceOut {
  float4 *rec;
  unsigned long long *count;
  uint32_t cap;
};

void run_launch(twos_mesh *owner, const std::vector<JobSpec> &specs, const double *d_sites, twos_site_result *d_out,
                RunOut &ro, twos_gradient_result *d_grad = nullptr, const TraceOut *trace = nullptr) {
  const twos_request *r0 = specs.front().r;
  const bool mixed = r0->precision == TWOS_PREC_MIXED;
  // d_grad selects the gradient form (paired walks with first-ball gradient
  // samples, finalized into twos_gradient_result rows).
  const int mode = d_grad ? kModeGradient : r0->mode;
  const bool paired = mode == TWOS_MODE_PAIRED || mode == kModeGradient;
  const int green = r0->green;
  std::vector<JobDesc> jobs;
  std::vector<GeoDesc> geos;
  std::vector<twos_mesh *> geo_mesh;
  std::vector<TermDev> terms;
  std::vector<double> cav;
  uint64_t walk_total = 0;
  uint32_t site_total = 0;
  for (const JobSpec &js : specs) {
    const twos_request *r = js.r;
    uint32_t geo = 0;
    while (geo < geo_mesh.size() && geo_mesh[geo] != js.mesh) ++geo;
    if (geo == geo_mesh.size()) {
      geo_mesh.push_back(js.mesh);
      geos.push_back(js.mesh->geo_host);
    }
    JobDesc J = make_job(js.mesh, r, js.n_sites, js.site_begin, js.site_offset, geo, walk_total, site_total,
                         static_cast<uint32_t>(cav.size() / 3), js.n_cav, terms);
    cav.insert(cav.end(), js.cav, js.cav + 3 * static_cast<size_t>(js.n_cav));
    jobs.push_back(J);
    walk_total += static_cast<uint64_t>(js.n_sites) * static_cast<uint64_t>(r->walks);
    site_total += js.n_sites;
  }
  if (terms.empty()) terms.push_back(TermDev{});
  twos_mesh *m = owner;
  const size_t vbytes = mixed ? sizeof(float) : sizeof(double);
  m->jobs.reserve(jobs.size() * sizeof(JobDesc));
  m->geos.reserve(geos.size() * sizeof(GeoDesc));
  m->terms.reserve(terms.size() * sizeof(TermDev));
  m->cavities.reserve(std::max<size_t>(1, cav.size()) * sizeof(double));
  m->u.reserve(walk_total * vbytes);
  if (paired) m->p.reserve(walk_total * vbytes);
  m->steps.reserve(walk_total * sizeof(uint32_t));
  if (d_grad) m->grad.reserve(walk_total * 6 * vbytes);
  m->first.reserve(static_cast<size_t>(site_total) * sizeof(double));
  check(cudaMemcpyAsync(m->jobs.ptr, jobs.data(), jobs.size() * sizeof(JobDesc), cudaMemcpyHostToDevice, m->stream),
        "upload jobs");
  check(cudaMemcpyAsync(m->geos.ptr, geos.data(), geos.size() * sizeof(GeoDesc), cudaMemcpyHostToDevice, m->stream),
        "upload geometries");
  check(cudaMemcpyAsync(m->terms.ptr, terms.data(), terms.size() * sizeof(TermDev), cudaMemcpyHostToDevice,
                        m->stream),
        "upload terms");
  if (!cav.empty())
    check(cudaMemcpyAsync(m->cavities.ptr, cav.data(), cav.size() * sizeof(double), cudaMemcpyHostToDevice,
                          m->stream),
          "upload cavities");
  check(cudaMemsetAsync(m->counter.ptr, 0, sizeof(unsigned long long), m->stream), "memset");
  WosLaunch L{};
  L.jobs = m->jobs.as<JobDesc>();
  L.n_jobs = static_cast<uint32_t>(jobs.size());
  L.geos = m->geos.as<GeoDesc>();
  L.n_geos = static_cast<uint32_t>(geos.size());
  L.sites = d_sites;
  L.terms = m->terms.as<TermDev>();
  L.n_terms = static_cast<uint32_t>(terms.size());
  L.cavities = m->cavities.as<double>();
  L.total_walks = walk_total;
  L.counter = m->counter.as<unsigned long long>();
  L.error = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
  L.u_out = m->u.ptr;
  L.p_out = paired ? m->p.ptr : nullptr;
  L.steps_out = m->steps.as<uint32_t>();
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
  L.counters = m->totals.as<unsigned long long>() + 3;
  L.site_best2 = m->first.ptr;
  L.total_sites = site_total;
  L.grad_out = d_grad ? m->grad.ptr : nullptr;
  const int block = m->block;
  const int per_sm = wos_max_blocks_per_sm(r0->precision, mode, green, block, L);
  if (per_sm <= 0) throw std::runtime_error("WoS kernel cannot be resident on this device");
  const int grid = std::min(per_sm, m->blocks_per_sm > 0 ? m->blocks_per_sm : per_sm) * m->num_sms;
  FinalizeLaunch F{};
  F.jobs = L.jobs;
  F.n_jobs = L.n_jobs;
  F.total_sites = site_total;
  F.totals = m->totals.as<unsigned long long>();
  F.u = L.u_out;
  F.p = L.p_out;
  F.steps = L.steps_out;
  F.out = d_out;
  check(cudaEventRecord(m->ev0, m->stream), "event");
  check(launch_site_prepass(r0->precision, L, m->stream), "site pre-pass");
  if (trace) {
    L.trace = trace->rec;
    L.trace_count = trace->count;
    L.trace_cap = trace->cap;
    check(launch_wos_traced(L, per_sm * m->num_sms, m->stream), "traced WoS launch");
  } else if (m->wavefront > 0 && mixed && green == TWOS_SOURCE_CENTER &&
             (mode == TWOS_MODE_COMPLIANCE || mode == TWOS_MODE_PAIRED || mode == TWOS_MODE_HOT) &&
             walk_total < (1ull << 32)) {
    // Wavefront form: no more slots than walks (rounded up to a step block).
    const uint32_t slots = static_cast<uint32_t>(std::min<uint64_t>(m->wavefront, (walk_total + 255) / 256 * 256));
    m->wf.reserve(wf_slot_bytes(slots));
    int max_steps = 1;
    for (const JobSpec &js : specs) max_steps = std::max(max_steps, js.r->max_steps);
    // Every live slot steps once per iteration: a generous bound.
    const uint64_t bound = (walk_total / slots + 2) * static_cast<uint64_t>(max_steps) + 1024;
    check(launch_wos_wavefront(mode, L, m->wf.ptr, slots, m->num_sms, bound, m->stream), "wavefront WoS launch");
  } else {
    check(launch_wos(r0->precision, mode, green, L, grid, block, m->stream), "WoS launch");
  }
  check(cudaEventRecord(m->evw, m->stream), "event");
  if (d_grad) {
    // One job per launch in the gradient form: its rows start at the job's site_begin.
    GradFinalizeLaunch G{};
    G.n_sites = site_total;
    G.walks = static_cast<uint32_t>(r0->walks);
    G.u = L.u_out;
    G.p = L.p_out;
    G.grad = L.grad_out;
    G.steps = L.steps_out;
    G.out = d_grad + specs.front().site_begin;
    G.totals = m->totals.as<unsigned long long>();
    check(launch_grad_finalize(r0->precision, G, m->stream), "gradient finalize launch");
  } else {
    check(launch_finalize(r0->precision, mode, F, m->stream), "finalize launch");
  }
  check(cudaEventRecord(m->ev1, m->stream), "event");
  check(cudaEventSynchronize(m->ev1), "WoS kernels");
  float ms = 0.f, msw = 0.f;
  check(cudaEventElapsedTime(&ms, m->ev0, m->ev1), "event time");
  check(cudaEventElapsedTime(&msw, m->ev0, m->evw), "event time");
  ro.kernel_seconds += ms * 1e-3;
  ro.walk_seconds += msw * 1e-3;
  ro.launches += 3;
}

void begin_totals(twos_mesh *m) {
  // totals: [0] steps, [1] caps, [2] error bits, [3..5] traversal counters.
  check(cudaMemsetAsync(m->totals.ptr, 0, 8 * sizeof(unsigned long long), m->stream), "memset");
}

void end_totals(twos_mesh *m, RunOut &ro) {
  unsigned long long tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  check(cudaMemcpyAsync(tot, m->totals.ptr, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, m->stream),
        "download totals");
  check(cudaStreamSynchronize(m->stream), "sync");
  ro.steps = tot[0];
  ro.caps = tot[1];
  uint32_t err = 0;
  std::memcpy(&err, &tot[2], sizeof(uint32_t));
  ro.error_flags = err;
  ro.node_tests = tot[3];
  ro.plane_tests = tot[4];
  ro.triangle_tests = tot[5];
  ro.grid_steps = tot[6];
}

// Runs the estimator over device-resident sites into device-resident rows,
// chunked by sites so one launch holds at most max_launch_walks walks.  With
// `keep`, the request must fit one launch and its per-walk samples stay in
// the session's u/p/steps buffers.
void run_estimate(twos_mesh *m, const twos_request *r, const double *d_sites, uint32_t n_sites,
                  const double *cav, uint32_t n_cav, twos_site_result *d_out, RunOut &ro, bool keep) {
  const size_t walks = static_cast<size_t>(r->walks);
  const size_t chunk_sites =
      std::max<size_t>(1, std::min<size_t>(n_sites, std::max<size_t>(1, m->max_launch_walks / walks)));
  if (keep && chunk_sites < n_sites) throw std::runtime_error("sample request exceeds one launch");
  begin_totals(m);
  for (size_t first = 0; first < n_sites; first += chunk_sites) {
    const uint32_t count = static_cast<uint32_t>(std::min<size_t>(chunk_sites, n_sites - first));
    JobSpec js{m, r, count, static_cast<uint32_t>(first), r->site_offset + static_cast<uint32_t>(first), cav, n_cav};
    run_launch(m, {js}, d_sites, d_out, ro);
  }
  end_totals(m, ro);
}

int finish(const RunOut &ro, uint32_t n_sites, const twos_request *r, twos_summary *summary, double t_total,
           uint64_t h2d, uint64_t d2h) {
  if (summary) {
    summary->kernel_seconds = ro.kernel_seconds;
    summary->walk_seconds = ro.walk_seconds;
    summary->total_seconds = t_total;
    summary->paths = static_cast<uint64_t>(n_sites) * static_cast<uint64_t>(r->walks);
    summary->steps = ro.steps;
    summary->caps = ro.caps;
    summary->queries = ro.steps + summary->paths;
    summary->h2d_bytes = h2d;
    summary->d2h_bytes = d2h;
    summary->launches = ro.launches;
    summary->error_flags = ro.error_flags;
    summary->node_tests = ro.node_tests;
    summary->plane_tests = ro.plane_tests;
    summary->triangle_tests = ro.triangle_tests;
    summary->grid_steps = ro.grid_steps;
  }
  if (ro.error_flags & TWOS_DEVERR_QUERY) return fail(TWOS_ERR_RUNTIME, "closest-point query failed");
  if (ro.error_flags & TWOS_DEVERR_STACK) return fail(TWOS_ERR_RUNTIME, "BVH traversal stack bound exceeded");
  if (ro.error_flags & TWOS_DEVERR_ITER) return fail(TWOS_ERR_RUNTIME, "BVH traversal iteration bound exceeded");
  if (ro.error_flags & TWOS_DEVERR_SOURCE) return fail(TWOS_ERR_RUNTIME, "negative analytic Green integral");
  if (ro.error_flags) return fail(TWOS_ERR_RUNTIME, "device error");
  if (ro.caps) return fail(TWOS_ERR_RUNTIME, "one or more paths hit --max-steps");
  return TWOS_OK;
}

}  // namespace

extern "C" {

int twos_abi_version(void) { return TWOS_ABI_VERSION; }

const char *twos_last_error(void) { return g_error.c_str(); }

int twos_mesh_open(const double *vertices, uint64_t n_vertices, const uint32_t *faces, uint64_t n_faces,
                   int device, twos_mesh **out) {
  if (!vertices || !faces) return fail(TWOS_ERR_USAGE, "null mesh buffers");
  std::vector<double> v(vertices, vertices + 3 * n_vertices);
  std::vector<uint32_t> f(faces, faces + 3 * n_faces);
  return open_impl(std::move(v), std::move(f), device, out);
}

int twos_mesh_open_ply(const char *path, int device, twos_mesh **out) {
  if (!path) return fail(TWOS_ERR_USAGE, "null path");
  std::vector<double> v;
  std::vector<uint32_t> f;
  try {
    load_ascii_ply(path, v, f);
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return open_impl(std::move(v), std::move(f), device, out);
}

void twos_mesh_close(twos_mesh *m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (DevBuf *b : {&m->nodes_f, &m->tris_f, &m->nodes_d, &m->tris_d, &m->geo, &m->jobs, &m->geos, &m->terms, &m->cavities,
                    &m->sites, &m->out, &m->u, &m->p, &m->steps, &m->first, &m->counter, &m->totals, &m->points, &m->dist,
                    &m->closest, &m->topk, &m->grid, &m->grad, &m->nodes4_f, &m->wf})
    b->release();
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->evw) cudaEventDestroy(m->evw);
  if (m->own_stream) cudaStreamDestroy(m->own_stream);
  delete m;
}

int twos_mesh_set_stream(twos_mesh *m, void *stream) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  m->stream = stream ? static_cast<cudaStream_t>(stream) : m->own_stream;
  return TWOS_OK;
}

int twos_mesh_set_tuning(twos_mesh *m, const twos_tuning *t) {
  if (!m || !t) return fail(TWOS_ERR_USAGE, "null argument");
  if ((t->block != 128 && t->block != 256 && t->block != 512) || t->refill < 1 || t->refill > 32 ||
      t->step_threshold < 1 || t->step_threshold > 32 || t->blocks_per_sm < 0 ||
      !(t->grid_threshold == 0.0f || (t->grid_threshold >= 0.1f && t->grid_threshold <= 1e6f)) ||
      t->units < 1 || t->units > 64 || (t->entry != 0 && t->entry != 1) ||
      (t->grid_fp64 != 0 && t->grid_fp64 != 1) || (t->bvh_width != 2 && t->bvh_width != 4) || t->lane_walks < 1 || t->lane_walks > 64 ||
      (t->lane_walks > 1 && t->bvh_width == 4) || t->wavefront < 0 ||
      t->wavefront > (1 << 26) || t->wavefront % 256 != 0)
    return fail(TWOS_ERR_USAGE, "invalid tuning");
  m->block = t->block;
  m->refill = t->refill;
  m->step_threshold = t->step_threshold;
  m->blocks_per_sm = t->blocks_per_sm;
  m->grid_tau = t->grid_threshold;
  m->units = t->units;
  m->entry_start = t->entry;
  m->grid_fp64 = t->grid_fp64;
  m->bvh_width = t->bvh_width;
  m->lane_walks = t->lane_walks;
  m->wavefront = static_cast<uint32_t>(t->wavefront);
  return TWOS_OK;
}

int twos_mesh_get_tuning(const twos_mesh *m, twos_tuning *t) {
  if (!m || !t) return fail(TWOS_ERR_USAGE, "null argument");
  t->block = m->block;
  t->refill = m->refill;
  t->step_threshold = m->step_threshold;
  t->blocks_per_sm = m->blocks_per_sm;
  t->grid_threshold = m->grid_tau;
  t->units = m->units;
  t->entry = m->entry_start;
  t->grid_fp64 = m->grid_fp64;
  t->bvh_width = m->bvh_width;
  t->lane_walks = m->lane_walks;
  t->wavefront = static_cast<int32_t>(m->wavefront);
  return TWOS_OK;
}

int twos_mesh_get_info(const twos_mesh *m, twos_mesh_info *info) {
  if (!m || !info) return fail(TWOS_ERR_USAGE, "null argument");
  info->vertices = m->vertices.size() / 3;
  info->faces = m->faces.size() / 3;
  info->bvh_nodes = m->bvh.nodes.size();
  info->bvh_depth = static_cast<uint32_t>(m->bvh.depth);
  info->device = static_cast<uint32_t>(m->device);
  for (int a = 0; a < 3; ++a) {
    info->bounds_min[a] = m->bmin[a];
    info->bounds_max[a] = m->bmax[a];
    info->center[a] = m->center[a];
  }
  info->mixed_delta = m->delta;
  info->build_seconds = m->build_seconds;
  info->device_bytes = m->resident_bytes;
  for (int a = 0; a < 3; ++a) info->grid_dims[a] = m->geo_host.grid ? m->geo_host.grid_n[a] : 0u;
  info->grid_pad = 0;
  info->grid_spacing = m->geo_host.grid ? static_cast<double>(m->geo_host.grid_h) : 0.0;
  return TWOS_OK;
}

int twos_closest_point(twos_mesh *m, int precision, const double *points, uint64_t n, double query_radius,
                       double *distance, double *closest) {
  if (!m || (!points && n) || (!distance && n)) return fail(TWOS_ERR_USAGE, "null argument");
  if (precision != TWOS_PREC_FP64 && precision != TWOS_PREC_MIXED) return fail(TWOS_ERR_USAGE, "invalid precision");
  if (n == 0) return TWOS_OK;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->points.reserve(n * 3 * sizeof(double));
    m->dist.reserve(n * sizeof(double));
    if (closest) m->closest.reserve(n * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->points.ptr, points, n * 3 * sizeof(double), cudaMemcpyHostToDevice, m->stream),
          "upload points");
    check(cudaMemsetAsync(m->totals.ptr, 0, 64, m->stream), "memset");
    const double qr = query_radius > 0.0 ? query_radius : std::numeric_limits<double>::infinity();
    uint32_t *err = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
    check(launch_closest(precision, m->geo.as<GeoDesc>(), m->points.as<double>(), n, qr * qr,
                         m->dist.as<double>(), closest ? m->closest.as<double>() : nullptr, err, m->stream),
          "closest launch");
    check(cudaMemcpyAsync(distance, m->dist.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
          "download");
    if (closest)
      check(cudaMemcpyAsync(closest, m->closest.ptr, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
            "download");
    uint32_t e = 0;
    check(cudaMemcpyAsync(&e, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, m->stream), "download");
    check(cudaStreamSynchronize(m->stream), "closest kernel");
    if (e & (TWOS_DEVERR_STACK | TWOS_DEVERR_ITER)) return fail(TWOS_ERR_RUNTIME, "BVH traversal bound exceeded");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return TWOS_OK;
}

int twos_mesh_distance_bound(twos_mesh *m, const double *points, uint64_t n, double *bound) {
  if (!m || (n && (!points || !bound))) return fail(TWOS_ERR_USAGE, "null argument");
  if (n == 0) return TWOS_OK;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->points.reserve(n * 3 * sizeof(double));
    m->dist.reserve(n * sizeof(double));
    check(cudaMemcpyAsync(m->points.ptr, points, n * 3 * sizeof(double), cudaMemcpyHostToDevice, m->stream),
          "upload points");
    check(launch_grid_bound(m->geo.as<GeoDesc>(), m->points.as<double>(), n, m->dist.as<double>(), m->stream),
          "grid bound launch");
    check(cudaMemcpyAsync(bound, m->dist.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download");
    check(cudaStreamSynchronize(m->stream), "grid bound");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return TWOS_OK;
}

int twos_estimate_device(twos_mesh *m, const twos_request *r, const double *d_sites, uint32_t n_sites,
                         const double *cavities, uint32_t n_cavities, twos_site_result *d_out,
                         twos_summary *summary) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  if (int rc = validate_request(r, n_sites, n_cavities)) return rc;
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!d_sites || !d_out || (n_cavities && !cavities)) return fail(TWOS_ERR_USAGE, "null buffer");
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    run_estimate(m, r, d_sites, n_sites, cavities, n_cavities, d_out, ro, false);
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return finish(ro, n_sites, r, summary, seconds_since(t0), 0, 0);
}

int twos_estimate(twos_mesh *m, const twos_request *r, const double *sites, uint32_t n_sites,
                  const double *cavities, uint32_t n_cavities, twos_site_result *out, twos_summary *summary) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  if (int rc = validate_request(r, n_sites, n_cavities)) return rc;
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!sites || !out || (n_cavities && !cavities)) return fail(TWOS_ERR_USAGE, "null buffer");
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  const uint64_t h2d = static_cast<uint64_t>(n_sites) * 3 * sizeof(double) + n_cavities * 3 * sizeof(double);
  const uint64_t d2h = static_cast<uint64_t>(n_sites) * sizeof(twos_site_result);
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    m->out.reserve(static_cast<size_t>(n_sites) * sizeof(twos_site_result));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    run_estimate(m, r, m->sites.as<double>(), n_sites, cavities, n_cavities, m->out.as<twos_site_result>(), ro,
                 false);
    check(cudaMemcpyAsync(out, m->out.ptr, d2h, cudaMemcpyDeviceToHost, m->stream), "download results");
    check(cudaStreamSynchronize(m->stream), "sync");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return finish(ro, n_sites, r, summary, seconds_since(t0), h2d, d2h);
}

int twos_estimate_batch(twos_mesh *const *meshes, const twos_request *requests, uint32_t n_jobs,
                        const double *const *sites, const uint32_t *n_sites, const double *const *cavities,
                        const uint32_t *n_cavities, twos_site_result *const *out, twos_summary *summary) {
  if (!meshes || !requests || !sites || !n_sites || !out || n_jobs == 0)
    return fail(TWOS_ERR_USAGE, "null argument");
  twos_mesh *owner = meshes[0];
  uint64_t total_sites = 0, total_paths = 0, h2d = 0;
  for (uint32_t j = 0; j < n_jobs; ++j) {
    if (!meshes[j]) return fail(TWOS_ERR_USAGE, "null mesh in batch");
    if (meshes[j]->device != owner->device) return fail(TWOS_ERR_USAGE, "batch meshes must share one device");
    const uint32_t nc = n_cavities ? n_cavities[j] : 0;
    if (int rc = validate_request(&requests[j], n_sites[j], nc)) return rc;
    if (requests[j].mode != requests[0].mode || requests[j].precision != requests[0].precision ||
        requests[j].green != requests[0].green)
      return fail(TWOS_ERR_USAGE, "batch requests must share mode, precision and green");
    if ((n_sites[j] && (!sites[j] || !out[j])) || (nc && (!cavities || !cavities[j])))
      return fail(TWOS_ERR_USAGE, "null buffer in batch");
    if (nc > 4096) return fail(TWOS_ERR_USAGE, "at most 4096 cavities per job");
    total_sites += n_sites[j];
    total_paths += static_cast<uint64_t>(n_sites[j]) * static_cast<uint64_t>(requests[j].walks);
    h2d += static_cast<uint64_t>(n_sites[j]) * 3 * sizeof(double) + nc * 3 * sizeof(double);
  }
  if (total_sites > 0xffffffffull) return fail(TWOS_ERR_USAGE, "too many sites in one batch");
  if (n_jobs > 256) return fail(TWOS_ERR_USAGE, "at most 256 jobs per batch");
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  try {
    check(cudaSetDevice(owner->device), "cudaSetDevice");
    owner->sites.reserve(std::max<uint64_t>(1, total_sites) * 3 * sizeof(double));
    owner->out.reserve(std::max<uint64_t>(1, total_sites) * sizeof(twos_site_result));
    std::vector<uint32_t> begin(n_jobs);
    uint32_t at = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
      begin[j] = at;
      if (n_sites[j])
        check(cudaMemcpyAsync(owner->sites.as<double>() + 3ull * at, sites[j], n_sites[j] * 3 * sizeof(double),
                              cudaMemcpyHostToDevice, owner->stream),
              "upload sites");
      at += n_sites[j];
    }
    // Queue order: the walks of consecutive jobs overlap in flight at each
    // job boundary, so two geometries whose data fill much of the L2 should
    // not follow each other.  Jobs go largest, smallest, second largest,
    // second smallest, ... by the bytes their form reads (BVH and triangles,
    // plus the distance grid's cell records in the mixed form).  Results do
    // not depend on the order: every walk's samples are keyed by its own job.
    const bool mixed = requests[0].precision == TWOS_PREC_MIXED;
    auto footprint = [&](uint32_t j) {
      const twos_mesh *mj = meshes[j];
      return mixed ? mj->nodes_f.bytes + mj->tris_f.bytes + mj->grid.bytes : mj->nodes_d.bytes + mj->tris_d.bytes;
    };
    std::vector<uint32_t> by_size(n_jobs);
    for (uint32_t j = 0; j < n_jobs; ++j) by_size[j] = j;
    std::stable_sort(by_size.begin(), by_size.end(),
                     [&](uint32_t a, uint32_t b) { return footprint(a) > footprint(b); });
    std::vector<uint32_t> order;
    for (uint32_t lo = 0, hi = n_jobs; lo < hi;) {
      order.push_back(by_size[lo++]);
      if (lo < hi) order.push_back(by_size[--hi]);
    }
    // Group consecutive jobs into launches of at most max_launch_walks walks
    // (a single larger job runs alone) whose job, geometry and term tables
    // fit the walk kernel's shared-memory budget: a launch that must read
    // them from global memory pays for it at every step (measured: 32
    // jobs in one launch 2.34 s, one launch per job 2.23 s).
    begin_totals(owner);
    std::vector<JobSpec> group;
    std::vector<const twos_mesh *> group_geos;
    uint64_t group_walks = 0;
    uint32_t group_terms = 0;
    const int precision = requests[0].precision;
    for (uint32_t q = 0; q <= n_jobs; ++q) {
      const uint32_t j = q < n_jobs ? order[q] : n_jobs;
      const uint64_t w = j < n_jobs ? static_cast<uint64_t>(n_sites[j]) * requests[j].walks : 0;
      bool fits = true;
      if (j < n_jobs && !group.empty()) {
        const bool new_geo = std::find(group_geos.begin(), group_geos.end(), meshes[j]) == group_geos.end();
        const uint32_t terms = group_terms + static_cast<uint32_t>(requests[j].n_source + requests[j].n_adjoint);
        fits = launch_tables_in_smem(precision, static_cast<uint32_t>(group.size()) + 1,
                                     static_cast<uint32_t>(group_geos.size()) + (new_geo ? 1u : 0u),
                                     std::max(1u, terms));
      }
      if (!group.empty() && (j == n_jobs || group_walks + w > owner->max_launch_walks || !fits)) {
        run_launch(owner, group, owner->sites.as<double>(), owner->out.as<twos_site_result>(), ro);
        group.clear();
        group_geos.clear();
        group_walks = 0;
        group_terms = 0;
      }
      if (j == n_jobs) break;
      if (n_sites[j] == 0) continue;
      const uint32_t nc = n_cavities ? n_cavities[j] : 0;
      group.push_back(JobSpec{meshes[j], &requests[j], n_sites[j], begin[j], requests[j].site_offset,
                              nc ? cavities[j] : nullptr, nc});
      if (std::find(group_geos.begin(), group_geos.end(), meshes[j]) == group_geos.end())
        group_geos.push_back(meshes[j]);
      group_walks += w;
      group_terms += static_cast<uint32_t>(requests[j].n_source + requests[j].n_adjoint);
    }
    end_totals(owner, ro);
    for (uint32_t j = 0; j < n_jobs; ++j)
      if (n_sites[j])
        check(cudaMemcpyAsync(out[j], owner->out.as<twos_site_result>() + begin[j],
                              n_sites[j] * sizeof(twos_site_result), cudaMemcpyDeviceToHost, owner->stream),
              "download results");
    check(cudaStreamSynchronize(owner->stream), "sync");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  twos_request agg = requests[0];
  const int rc = finish(ro, 0, &agg, summary, seconds_since(t0), h2d, total_sites * sizeof(twos_site_result));
  if (summary) {
    summary->paths = total_paths;
    summary->queries = ro.steps + total_paths;
  }
  return rc;
}

int twos_design_loop(twos_mesh *m, const twos_request *scout, const twos_request *validate,
                     const double *candidates, uint32_t n, const double *cavities, uint32_t n_cav0,
                     const twos_design_params *P, twos_design_step *history, double *cavities_out,
                     uint32_t *n_cavities_out, twos_summary *summary) {
  if (!m || !scout || !validate || !candidates || !P || !history || !cavities_out || !n_cavities_out)
    return fail(TWOS_ERR_USAGE, "null argument");
  if (n == 0 || P->iterations == 0) return fail(TWOS_ERR_USAGE, "need candidates and iterations");
  if (P->shortlist == 0 || P->shortlist > 1024 || P->shortlist > n)
    return fail(TWOS_ERR_USAGE, "shortlist must be in [1, min(1024, candidates)]");
  if (!(P->cavity_radius > 0.0) || !(P->z >= 0.0)) return fail(TWOS_ERR_USAGE, "invalid design parameters");
  if (n_cav0 && !cavities) return fail(TWOS_ERR_USAGE, "null cavities");
  twos_request rs = *scout, rv = *validate;
  rs.cavity_radius = rv.cavity_radius = P->cavity_radius;
  // Iteration i draws its samples with repeat = i; validation walks are keyed
  // by their shortlist slot, on the validate request's own stream.
  rs.repeat = rv.repeat = 0;
  const uint32_t max_cav = n_cav0 + P->iterations;
  if (int rc = validate_request(&rs, n, max_cav)) return rc;
  if (int rc = validate_request(&rv, P->shortlist, max_cav)) return rc;
  if (rs.precision != rv.precision || rs.mode != rv.mode || rs.mode == TWOS_MODE_HOT)
    return fail(TWOS_ERR_USAGE, "scout and validate must share precision and a TD mode");
  const uint32_t k = P->shortlist;
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  DevBuf cand, feas, keys, idx, vsites, rows_s, rows_v, cav, jobs_s, jobs_v, iter, hist, terms_d, topk, dist,
      first_v;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    cand.reserve(static_cast<size_t>(n) * 3 * sizeof(double));
    check(cudaMemcpyAsync(cand.ptr, candidates, static_cast<size_t>(n) * 3 * sizeof(double), cudaMemcpyHostToDevice,
                          m->stream),
          "upload candidates");
    // Feasibility against the surface and the initial cavities (host, once).
    dist.reserve(static_cast<size_t>(n) * sizeof(double));
    check(launch_closest(TWOS_PREC_FP64, m->geo.as<GeoDesc>(), cand.as<double>(), n,
                         std::numeric_limits<double>::infinity(), dist.as<double>(), nullptr,
                         reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2), m->stream),
          "closest launch");
    std::vector<double> d(n);
    check(cudaMemcpyAsync(d.data(), dist.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download");
    check(cudaStreamSynchronize(m->stream), "sync");
    const double pair = 2.0 * P->cavity_radius + P->pair_gap;
    std::vector<uint8_t> mask(n);
    for (uint32_t i = 0; i < n; ++i) {
      bool ok = d[i] >= P->cavity_radius + P->outer_clearance;
      for (uint32_t c = 0; c < n_cav0 && ok; ++c) {
        const double dx = candidates[3 * i] - cavities[3 * c], dy = candidates[3 * i + 1] - cavities[3 * c + 1],
                     dz = candidates[3 * i + 2] - cavities[3 * c + 2];
        ok = dx * dx + dy * dy + dz * dz >= pair * pair;
      }
      mask[i] = ok ? 1 : 0;
    }
    feas.reserve(n);
    check(cudaMemcpyAsync(feas.ptr, mask.data(), n, cudaMemcpyHostToDevice, m->stream), "upload mask");
    keys.reserve(static_cast<size_t>(n) * sizeof(double));
    idx.reserve(k * sizeof(uint32_t));
    vsites.reserve(static_cast<size_t>(k) * 3 * sizeof(double));
    rows_s.reserve(static_cast<size_t>(n) * sizeof(twos_site_result));
    rows_v.reserve(static_cast<size_t>(k) * sizeof(twos_site_result));
    cav.reserve(static_cast<size_t>(max_cav) * 3 * sizeof(double));
    if (n_cav0)
      check(cudaMemcpyAsync(cav.ptr, cavities, n_cav0 * 3 * sizeof(double), cudaMemcpyHostToDevice, m->stream),
            "upload cavities");
    std::vector<TermDev> terms;
    const JobDesc Js = make_job(m, &rs, n, 0, rs.site_offset, 0, 0, 0, 0, n_cav0, terms);
    const JobDesc Jv = make_job(m, &rv, k, 0, rv.site_offset, 0, 0, 0, 0, n_cav0, terms);
    if (terms.empty()) terms.push_back(TermDev{});
    terms_d.reserve(terms.size() * sizeof(TermDev));
    jobs_s.reserve(sizeof(JobDesc));
    jobs_v.reserve(sizeof(JobDesc));
    check(cudaMemcpyAsync(terms_d.ptr, terms.data(), terms.size() * sizeof(TermDev), cudaMemcpyHostToDevice,
                          m->stream),
          "upload terms");
    check(cudaMemcpyAsync(jobs_s.ptr, &Js, sizeof(JobDesc), cudaMemcpyHostToDevice, m->stream), "upload job");
    check(cudaMemcpyAsync(jobs_v.ptr, &Jv, sizeof(JobDesc), cudaMemcpyHostToDevice, m->stream), "upload job");
    iter.reserve(sizeof(uint32_t));
    check(cudaMemsetAsync(iter.ptr, 0, sizeof(uint32_t), m->stream), "memset");
    hist.reserve(static_cast<size_t>(P->iterations) * sizeof(DesignStep));
    const bool mixed = rs.precision == TWOS_PREC_MIXED;
    const bool paired = rs.mode == TWOS_MODE_PAIRED;
    const size_t vbytes = mixed ? sizeof(float) : sizeof(double);
    const size_t walks_max = std::max<size_t>(static_cast<size_t>(n) * rs.walks, static_cast<size_t>(k) * rv.walks);
    m->u.reserve(walks_max * vbytes);
    if (paired) m->p.reserve(walks_max * vbytes);
    m->steps.reserve(walks_max * sizeof(uint32_t));
    const size_t tk = topk_scratch_bytes(n, k);
    topk.reserve(tk);
    begin_totals(m);

    WosLaunch Ls{};
    Ls.jobs = jobs_s.as<JobDesc>();
    Ls.n_jobs = 1;
    Ls.geos = m->geo.as<GeoDesc>();
    Ls.n_geos = 1;
    Ls.sites = cand.as<double>();
    Ls.terms = terms_d.as<TermDev>();
    Ls.n_terms = static_cast<uint32_t>(terms.size());
    Ls.cavities = cav.as<double>();
    Ls.total_walks = static_cast<uint64_t>(n) * rs.walks;
    Ls.counter = m->counter.as<unsigned long long>();
    Ls.error = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
    Ls.u_out = m->u.ptr;
    Ls.p_out = paired ? m->p.ptr : nullptr;
    Ls.steps_out = m->steps.as<uint32_t>();
    Ls.refill = m->refill;
    Ls.step_threshold = m->step_threshold;
    Ls.vote = m->vote;
    Ls.warm = m->warm;
    Ls.grid_tau = m->grid_tau;
    Ls.units = m->units;
    Ls.lane_walks = m->lane_walks;
    Ls.entry = m->entry_start;
    Ls.grid64 = m->grid_fp64;
    Ls.wide = m->bvh_width == 4;
    Ls.counters = m->totals.as<unsigned long long>() + 3;
    m->first.reserve(static_cast<size_t>(n) * sizeof(double));
    first_v.reserve(static_cast<size_t>(k) * sizeof(double));
    Ls.site_best2 = m->first.ptr;
    Ls.total_sites = n;
    WosLaunch Lv = Ls;
    // The validation stage decides acceptance; it runs without the mixed
    // form's distance grid, so the mixed and FP64 forms validate a candidate
    // with the same samples (the grid changes the walks' radii) and their
    // accept decisions for the same candidate agree.  The scout keeps it.
    Lv.grid_tau = 0.f;
    Lv.site_best2 = first_v.ptr;
    Lv.total_sites = k;
    Lv.jobs = jobs_v.as<JobDesc>();
    Lv.sites = vsites.as<double>();
    Lv.total_walks = static_cast<uint64_t>(k) * rv.walks;
    FinalizeLaunch Fs{};
    Fs.jobs = Ls.jobs;
    Fs.n_jobs = 1;
    Fs.total_sites = n;
    Fs.totals = m->totals.as<unsigned long long>();
    Fs.u = Ls.u_out;
    Fs.p = Ls.p_out;
    Fs.steps = Ls.steps_out;
    Fs.out = rows_s.as<twos_site_result>();
    FinalizeLaunch Fv = Fs;
    Fv.jobs = Lv.jobs;
    Fv.total_sites = k;
    Fv.out = rows_v.as<twos_site_result>();
    DesignLaunch D{};
    D.candidates = cand.as<double>();
    D.n_candidates = n;
    D.k = k;
    D.scout_rows = rows_s.as<twos_site_result>();
    D.feasible = feas.as<uint8_t>();
    D.keys = keys.as<double>();
    D.shortlist = idx.as<uint32_t>();
    D.val_sites = vsites.as<double>();
    D.val_rows = rows_v.as<twos_site_result>();
    D.scout_job = jobs_s.as<JobDesc>();
    D.val_job = jobs_v.as<JobDesc>();
    D.cavities = cav.as<double>();
    D.max_cav = max_cav;
    D.max_iterations = P->iterations;
    D.z = P->z;
    D.threshold = P->accept_threshold;
    D.pair_clearance = pair;
    D.iteration = iter.as<uint32_t>();
    D.history = hist.as<DesignStep>();
    const int block = m->block;
    const int per_s = wos_max_blocks_per_sm(rs.precision, rs.mode, rs.green, block, Ls);
    const int per_v = wos_max_blocks_per_sm(rv.precision, rv.mode, rv.green, block, Lv);
    if (per_s <= 0 || per_v <= 0) throw std::runtime_error("WoS kernel cannot be resident on this device");
    const int cap = m->blocks_per_sm > 0 ? m->blocks_per_sm : 1 << 20;
    const int grid_s = std::min(per_s, cap) * m->num_sms, grid_v = std::min(per_v, cap) * m->num_sms;
    auto iteration = [&]() {
      check(cudaMemsetAsync(m->counter.ptr, 0, sizeof(unsigned long long), m->stream), "memset");
      check(launch_site_prepass(rs.precision, Ls, m->stream), "scout pre-pass");
      check(launch_wos(rs.precision, rs.mode, rs.green, Ls, grid_s, block, m->stream), "scout launch");
      check(launch_finalize(rs.precision, rs.mode, Fs, m->stream), "scout finalize");
      check(launch_design_keys(D, m->stream), "keys");
      check(launch_topk(D.keys, n, k, idx.as<uint32_t>(), topk.ptr, topk.bytes, m->stream), "top-k");
      check(launch_design_gather(D, m->stream), "gather");
      check(cudaMemsetAsync(m->counter.ptr, 0, sizeof(unsigned long long), m->stream), "memset");
      check(launch_site_prepass(rv.precision, Lv, m->stream), "validate pre-pass");
      check(launch_wos(rv.precision, rv.mode, rv.green, Lv, grid_v, block, m->stream), "validate launch");
      check(launch_finalize(rv.precision, rv.mode, Fv, m->stream), "validate finalize");
      check(launch_design_select(D, m->stream), "select");
      check(launch_design_mask(D, m->stream), "mask");
    };
    if (P->use_graph) {
      check(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeRelaxed), "begin capture");
      iteration();
      check(cudaStreamEndCapture(m->stream, &graph), "end capture");
      check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    }
    check(cudaEventRecord(m->ev0, m->stream), "event");
    for (uint32_t it = 0; it < P->iterations; ++it) {
      if (exec)
        check(cudaGraphLaunch(exec, m->stream), "graph launch");
      else
        iteration();
    }
    check(cudaEventRecord(m->ev1, m->stream), "event");
    check(cudaEventSynchronize(m->ev1), "design loop");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, m->ev0, m->ev1), "event time");
    ro.kernel_seconds = ms * 1e-3;
    ro.launches = P->iterations * 11;
    check(cudaMemcpyAsync(history, hist.ptr, P->iterations * sizeof(DesignStep), cudaMemcpyDeviceToHost, m->stream),
          "download history");
    JobDesc Jout{};
    check(cudaMemcpyAsync(&Jout, jobs_s.ptr, sizeof(JobDesc), cudaMemcpyDeviceToHost, m->stream), "download job");
    check(cudaMemcpyAsync(cavities_out, cav.ptr, max_cav * 3 * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
          "download cavities");
    end_totals(m, ro);
    *n_cavities_out = Jout.n_cav;
  } catch (const std::exception &e) {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (DevBuf *b : {&cand, &feas, &keys, &idx, &vsites, &rows_s, &rows_v, &cav, &jobs_s, &jobs_v, &iter, &hist,
                      &terms_d, &topk, &dist, &first_v})
      b->release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (DevBuf *b : {&cand, &feas, &keys, &idx, &vsites, &rows_s, &rows_v, &cav, &jobs_s, &jobs_v, &iter, &hist,
                    &terms_d, &topk, &dist, &first_v})
    b->release();
  const int rc = finish(ro, 0, &rs, summary, seconds_since(t0), 0, 0);
  if (summary) {
    summary->paths = static_cast<uint64_t>(P->iterations) *
                     (static_cast<uint64_t>(n) * rs.walks + static_cast<uint64_t>(k) * rv.walks);
    summary->queries = ro.steps + summary->paths;
  }
  return rc;
}

int twos_validate(twos_mesh *m, const twos_request *r, const twos_validate_params *vp, const double *sites,
                  uint32_t n_sites, const double *cavities, uint32_t n_cav, twos_cert_sample *samples,
                  twos_validate_stage *stages, uint32_t *n_stages, twos_summary *summary) {
  if (!m || !r || !vp) return fail(TWOS_ERR_USAGE, "null mesh, request or parameters");
  if (int rc = validate_request(r, n_sites, n_cav)) return rc;
  if (r->green != TWOS_SOURCE_CENTER && r->green != TWOS_SOURCE_GREEN)
    return fail(TWOS_ERR_USAGE, "validation takes the centre or the Green-point source rule");
  if (!(vp->radius_cap > 0.0) || !(vp->value_cap > 0.0))
    return fail(TWOS_ERR_USAGE, "validation caps must be positive");
  for (int i = 0; i < r->n_source; ++i) {
    const twos_source_term &t = r->source[i];
    const bool lead_const = i == 0 && t.kind == TWOS_TERM_CONST;
    const bool ok = lead_const || (t.kind == TWOS_TERM_LINEAR && t.amp >= 0.0) ||
                    (t.kind == TWOS_TERM_GAUSS && t.amp >= 0.0 && t.w[0] > 0.0 && t.w[1] > 0.0 && t.w[2] > 0.0);
    if (!ok)
      return fail(TWOS_ERR_USAGE,
                  "validation sources: a leading constant, then nonnegative linear and Gaussian terms");
  }
  if (n_sites == 0) {
    if (n_stages) *n_stages = 0;
    return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  }
  if (!sites || !samples || !stages || !n_stages || (n_cav && !cavities)) return fail(TWOS_ERR_USAGE, "null buffer");
  // Every candidate must be inside the mesh and outside every cavity
  // (minimum_benefit.hpp:158-159).
  {
    std::vector<uint8_t> inside(n_sites);
    if (int rc = twos_inside(m, sites, n_sites, inside.data())) return rc;
    for (uint32_t s = 0; s < n_sites; ++s) {
      bool in_cav = false;
      for (uint32_t c = 0; c < n_cav; ++c) {
        const double dx = sites[3 * s] - cavities[3 * c], dy = sites[3 * s + 1] - cavities[3 * c + 1],
                     dz = sites[3 * s + 2] - cavities[3 * c + 2];
        in_cav = in_cav || std::sqrt(dx * dx + dy * dy + dz * dz) <= r->cavity_radius;
      }
      if (!inside[s] || in_cav)
        return fail(TWOS_ERR_RUNTIME, "candidate classified outside; exact driver predicate is also required");
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  const size_t walks = static_cast<size_t>(r->walks);
  const size_t total = static_cast<size_t>(n_sites) * walks;
  DevBuf dsamp, dclear, dcenter, dterms;
  unsigned long long tot[2] = {0, 0};
  std::vector<double> clearance(n_sites), center(n_sites);
  RunOut ro;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    m->cavities.reserve(std::max<size_t>(1, n_cav) * 3 * sizeof(double));
    if (n_cav)
      check(cudaMemcpyAsync(m->cavities.ptr, cavities, static_cast<size_t>(n_cav) * 3 * sizeof(double),
                            cudaMemcpyHostToDevice, m->stream),
            "upload cavities");
    dterms.reserve(std::max(1, r->n_source) * sizeof(TermDev));
    if (r->n_source)
      check(cudaMemcpyAsync(dterms.ptr, r->source, r->n_source * sizeof(TermDev), cudaMemcpyHostToDevice, m->stream),
            "upload terms");
    dsamp.reserve(total * sizeof(twos_cert_sample));
    dclear.reserve(n_sites * sizeof(double));
    dcenter.reserve(n_sites * sizeof(double));
    begin_totals(m);
    ValidateLaunch V{};
    V.geo = m->geo.as<GeoDesc>();
    V.sites = m->sites.as<double>();
    V.n_sites = n_sites;
    V.walks = static_cast<uint32_t>(walks);
    V.cavities = m->cavities.as<double>();
    V.n_cav = n_cav;
    V.terms = dterms.as<TermDev>();
    V.n_terms = static_cast<uint32_t>(r->n_source);
    V.green = r->green == TWOS_SOURCE_GREEN;
    counter_key(r->seed, r->stream, V.k0, V.k1);
    V.repeat = r->repeat;
    V.site_offset = r->site_offset;
    V.max_steps = r->max_steps;
    V.epsilon = r->epsilon;
    V.cavity_radius = r->cavity_radius;
    V.radius_cap = vp->radius_cap;
    V.value_cap = vp->value_cap;
    V.samples = dsamp.as<twos_cert_sample>();
    V.clearance = dclear.as<double>();
    V.center_distance = dcenter.as<double>();
    V.totals = m->totals.as<unsigned long long>() + 3;  // [3] failures, [4] steps
    V.error = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
    check(cudaEventRecord(m->ev0, m->stream), "event");
    check(launch_validate(V, m->stream), "validate launch");
    check(cudaEventRecord(m->ev1, m->stream), "event");
    ro.launches = 2;
    check(cudaMemcpyAsync(samples, dsamp.ptr, total * sizeof(twos_cert_sample), cudaMemcpyDeviceToHost, m->stream),
          "download samples");
    check(cudaMemcpyAsync(clearance.data(), dclear.ptr, n_sites * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
          "download clearance");
    check(cudaMemcpyAsync(center.data(), dcenter.ptr, n_sites * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
          "download centre distance");
    end_totals(m, ro);
    tot[0] = ro.node_tests;  // totals[3]: containment failures
    tot[1] = ro.plane_tests; // totals[4]: steps
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, m->ev0, m->ev1), "event time");
    ro.kernel_seconds = ro.walk_seconds = ms / 1e3;
  } catch (const std::exception &e) {
    for (DevBuf *b : {&dsamp, &dclear, &dcenter, &dterms}) b->release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  for (DevBuf *b : {&dsamp, &dclear, &dcenter, &dterms}) b->release();
  // Stage statistics: prefixes n in {1024, 4096, 16384, 65536} below walks,
  // then walks; sums in long double in sample order (minimum_benefit.hpp:160-176).
  std::vector<uint32_t> ns;
  for (uint32_t n : {1024u, 4096u, 16384u, 65536u})
    if (n < walks) ns.push_back(n);
  ns.push_back(static_cast<uint32_t>(walks));
  uint64_t caps_total = 0;
  for (uint32_t s = 0; s < n_sites; ++s) {
    const twos_cert_sample *v = samples + static_cast<size_t>(s) * walks;
    long double sum = 0.0L;
    uint64_t steps = 0, clipped = 0, capped = 0;
    uint32_t j = 0;
    for (size_t k = 0; k < ns.size(); ++k) {
      for (; j < ns[k]; ++j) {
        sum += v[j].value;
        steps += v[j].steps;
        clipped += v[j].clipped;
        capped += v[j].capped;
      }
      twos_validate_stage &st = stages[static_cast<size_t>(s) * TWOS_VALIDATE_MAX_STAGES + k];
      st.site = s;
      st.n = ns[k];
      st.mean = static_cast<double>(sum / ns[k]);
      st.mean_steps = static_cast<double>(steps) / ns[k];
      st.clipped = clipped;
      st.path_caps = capped;
      st.center_clearance_lower = clearance[s];
      st.center_distance = center[s];
    }
    caps_total += capped;
  }
  *n_stages = static_cast<uint32_t>(ns.size());
  if (summary) {
    std::memset(summary, 0, sizeof(*summary));
    summary->kernel_seconds = summary->walk_seconds = ro.kernel_seconds;
    summary->total_seconds = seconds_since(t0);
    summary->paths = total;
    summary->steps = tot[1];
    summary->caps = caps_total;
    summary->launches = ro.launches;
    summary->error_flags = ro.error_flags;
    summary->node_tests = tot[0];  // containment failures
  }
  if (ro.error_flags & TWOS_DEVERR_STACK) return fail(TWOS_ERR_RUNTIME, "BVH traversal stack bound exceeded");
  if (ro.error_flags & TWOS_DEVERR_ITER) return fail(TWOS_ERR_RUNTIME, "BVH traversal iteration bound exceeded");
  if (ro.error_flags) return fail(TWOS_ERR_RUNTIME, "device error");
  if (tot[0])
    return fail(TWOS_ERR_RUNTIME, "sample containment guard failed; validation record must be rejected");
  return TWOS_OK;
}

int twos_estimate_gradient(twos_mesh *m, const twos_request *r, const double *sites, uint32_t n_sites,
                           const double *cavities, uint32_t n_cav, twos_gradient_result *out,
                           twos_summary *summary) {
  if (!m || !r) return fail(TWOS_ERR_USAGE, "null mesh or request");
  if (int rc = validate_request(r, n_sites, n_cav, true)) return rc;
  if (r->mode != TWOS_MODE_PAIRED) return fail(TWOS_ERR_USAGE, "the gradient form takes a paired request");
  if (r->green == TWOS_SOURCE_EXACT)
    return fail(TWOS_ERR_USAGE, "the gradient form takes the centre or the Green-point source rule");
  if (r->walks < 3) return fail(TWOS_ERR_USAGE, "the gradient form needs at least 3 walks per site");
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!sites || !out || (n_cav && !cavities)) return fail(TWOS_ERR_USAGE, "null buffer");
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  DevBuf rows;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    rows.reserve(static_cast<size_t>(n_sites) * sizeof(twos_gradient_result));
    const size_t walks = static_cast<size_t>(r->walks);
    const size_t chunk =
        std::max<size_t>(1, std::min<size_t>(n_sites, std::max<size_t>(1, m->max_launch_walks / walks)));
    begin_totals(m);
    for (size_t first = 0; first < n_sites; first += chunk) {
      const uint32_t count = static_cast<uint32_t>(std::min<size_t>(chunk, n_sites - first));
      JobSpec js{m, r, count, static_cast<uint32_t>(first), r->site_offset + static_cast<uint32_t>(first), cavities,
                 n_cav};
      run_launch(m, {js}, m->sites.as<double>(), nullptr, ro, rows.as<twos_gradient_result>());
    }
    check(cudaMemcpyAsync(out, rows.ptr, static_cast<size_t>(n_sites) * sizeof(twos_gradient_result),
                          cudaMemcpyDeviceToHost, m->stream),
          "download rows");
    end_totals(m, ro);
  } catch (const std::exception &e) {
    rows.release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  rows.release();
  return finish(ro, n_sites, r, summary, seconds_since(t0), static_cast<uint64_t>(n_sites) * 24,
                static_cast<uint64_t>(n_sites) * sizeof(twos_gradient_result));
}

int twos_rqmc(twos_mesh *m, const twos_request *r, const twos_rqmc_params *rp, const double *sites, uint32_t n_sites,
              double *batch_u, double *batch_p, double *td, twos_summary *summary) {
  if (!m || !r || !rp) return fail(TWOS_ERR_USAGE, "null mesh, request or parameters");
  if (int rc = validate_request(r, n_sites, 0)) return rc;
  // Korobov generators a of the 3D lattice (i/n, a i/n, a^2 i/n): for each n
  // the odd a with the largest minimum toroidal distance between lattice
  // points (the reference's table, sampling.py:16, serves its 2D (1, a)
  // lattice).
  uint32_t generator = 0;
  switch (r->walks) {
    case 32: generator = 3; break;
    case 64: generator = 5; break;
    case 128: generator = 5; break;
    case 256: generator = 13; break;
    case 512: generator = 101; break;
    case 1024: generator = 35; break;
    default: return fail(TWOS_ERR_USAGE, "RQMC walks must be a power of two from 32 to 1024");
  }
  if (rp->method != TWOS_RQMC_MC && rp->method != TWOS_RQMC_ARRAY && rp->method != TWOS_RQMC_NEIGHBOUR &&
      rp->method != TWOS_RQMC_SOBOL)
    return fail(TWOS_ERR_USAGE, "invalid RQMC method");
  // The Poisson kernel reweights a walk's exit value only: a source's path
  // integral depends on where the walk started (sampling.py runs the
  // neighbour estimator on the harmonic problem alone).
  if (rp->method == TWOS_RQMC_NEIGHBOUR && r->n_source)
    return fail(TWOS_ERR_USAGE, "neighbour reuse needs a harmonic problem (no source terms)");
  if (rp->batches < 2) return fail(TWOS_ERR_USAGE, "RQMC needs at least 2 batches");
  if (rp->n_u_boundary > TWOS_MAX_TERMS || rp->n_p_boundary > TWOS_MAX_TERMS)
    return fail(TWOS_ERR_USAGE, "too many boundary terms");
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!sites || !batch_u || !batch_p || !td) return fail(TWOS_ERR_USAGE, "null buffer");
  const auto t0 = std::chrono::steady_clock::now();
  const bool mixed = r->precision == TWOS_PREC_MIXED;
  const double zero[3] = {0.0, 0.0, 0.0};
  const double *frame = mixed ? m->center : zero;
  std::vector<TermDev> terms;
  for (int i = 0; i < r->n_source; ++i) terms.push_back(frame_term(r->source[i], frame));
  for (uint32_t i = 0; i < rp->n_u_boundary; ++i) terms.push_back(frame_term(rp->u_boundary[i], frame));
  for (uint32_t i = 0; i < rp->n_p_boundary; ++i) terms.push_back(frame_term(rp->p_boundary[i], frame));
  if (terms.empty()) terms.push_back(TermDev{});
  const size_t nb = static_cast<size_t>(rp->batches) * n_sites;
  const size_t nw = nb * static_cast<size_t>(r->walks);
  const bool reuse = rp->method == TWOS_RQMC_NEIGHBOUR;
  const bool rec_first = reuse || rp->walk_first || rp->site_radius, rec_walk = reuse || rp->walk_u || rp->walk_p;
  RunOut ro;
  DevBuf dterms, du, dp, dfirst, dwu, dwp, drad, dsobol;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    if (rp->method == TWOS_RQMC_SOBOL) {
      // Two coordinates per step for the first kSobolSteps steps; computed
      // once per process (a few hundred primitive polynomials).
      static const std::vector<uint32_t> table = sobol_directions(2 * kSobolSteps, kSobolBits);
      dsobol.reserve(table.size() * sizeof(uint32_t));
      check(cudaMemcpyAsync(dsobol.ptr, table.data(), table.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            m->stream),
            "upload Sobol directions");
    }
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    dterms.reserve(terms.size() * sizeof(TermDev));
    check(cudaMemcpyAsync(dterms.ptr, terms.data(), terms.size() * sizeof(TermDev), cudaMemcpyHostToDevice, m->stream),
          "upload terms");
    du.reserve(nb * sizeof(double));
    dp.reserve(nb * sizeof(double));
    if (rec_first) {
      dfirst.reserve(nw * 3 * sizeof(double));
      drad.reserve(static_cast<size_t>(n_sites) * sizeof(double));
      check(cudaMemsetAsync(dfirst.ptr, 0, nw * 3 * sizeof(double), m->stream), "memset");
      check(cudaMemsetAsync(drad.ptr, 0, static_cast<size_t>(n_sites) * sizeof(double), m->stream), "memset");
    }
    if (rec_walk) {
      dwu.reserve(nw * sizeof(double));
      dwp.reserve(nw * sizeof(double));
    }
    begin_totals(m);
    RqmcLaunch R{};
    R.geo = m->geo.as<GeoDesc>();
    R.sites = m->sites.as<double>();
    R.n_sites = n_sites;
    R.walks = static_cast<uint32_t>(r->walks);
    R.batches = rp->batches;
    R.method = rp->method;
    R.generator = generator;
    R.generator2 = static_cast<uint32_t>((static_cast<uint64_t>(generator) * generator) % R.walks);
    R.terms = dterms.as<TermDev>();
    R.n_src = static_cast<uint32_t>(r->n_source);
    R.n_ub = rp->n_u_boundary;
    R.n_pb = rp->n_p_boundary;
    counter_key(r->seed, r->stream, R.k0, R.k1);
    R.repeat = r->repeat;
    R.max_steps = r->max_steps;
    R.epsilon = r->epsilon;
    for (int a = 0; a < 3; ++a) {
      R.lo[a] = m->bmin[a] - frame[a];
      R.inv_extent[a] = 1.0 / std::max(m->bmax[a] - m->bmin[a], 1e-300);
    }
    R.batch_u = du.as<double>();
    R.batch_p = dp.as<double>();
    R.walk_first = rec_first ? dfirst.as<double>() : nullptr;
    R.site_radius = rec_first ? drad.as<double>() : nullptr;
    R.walk_u = rec_walk ? dwu.as<double>() : nullptr;
    R.walk_p = rec_walk ? dwp.as<double>() : nullptr;
    R.totals = m->totals.as<unsigned long long>();
    R.error = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
    if (rp->method == TWOS_RQMC_SOBOL) {
      R.sobol_v = dsobol.as<uint32_t>();
      while ((1u << R.sobol_bits) < R.walks) ++R.sobol_bits;
    }
    check(cudaEventRecord(m->ev0, m->stream), "event");
    check(launch_rqmc(r->precision, R, m->stream), "RQMC launch");
    ro.launches = 1;
    if (reuse) {
      check(launch_rqmc_reuse(R, m->stream), "neighbour reuse launch");
      ro.launches = 2;
    }
    check(cudaEventRecord(m->ev1, m->stream), "event");
    check(cudaMemcpyAsync(batch_u, du.ptr, nb * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download");
    check(cudaMemcpyAsync(batch_p, dp.ptr, nb * sizeof(double), cudaMemcpyDeviceToHost, m->stream), "download");
    const std::pair<double *, DevBuf *> records[] = {
        {rp->walk_first, &dfirst}, {rp->walk_u, &dwu}, {rp->walk_p, &dwp}, {rp->site_radius, &drad}};
    const size_t record_bytes[] = {nw * 3 * sizeof(double), nw * sizeof(double), nw * sizeof(double),
                                   static_cast<size_t>(n_sites) * sizeof(double)};
    for (int i = 0; i < 4; ++i)
      if (records[i].first)
        check(cudaMemcpyAsync(records[i].first, records[i].second->ptr, record_bytes[i], cudaMemcpyDeviceToHost,
                              m->stream),
              "download");
    end_totals(m, ro);
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, m->ev0, m->ev1), "event time");
    ro.kernel_seconds = ro.walk_seconds = ms / 1e3;
  } catch (const std::exception &e) {
    for (DevBuf *b : {&dterms, &du, &dp, &dfirst, &dwu, &dwp, &drad, &dsobol}) b->release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  for (DevBuf *b : {&dterms, &du, &dp, &dfirst, &dwu, &dwp, &drad, &dsobol}) b->release();
  // Cross-fitting over batches (crossfit, sampling.py:90-92).
  const double R = rp->batches;
  for (uint32_t s = 0; s < n_sites; ++s) {
    double sa = 0.0, sb = 0.0, sab = 0.0;
    for (uint32_t b = 0; b < rp->batches; ++b) {
      const double a = batch_u[static_cast<size_t>(b) * n_sites + s], c = batch_p[static_cast<size_t>(b) * n_sites + s];
      sa += a;
      sb += c;
      sab += a * c;
    }
    td[s] = -(sa * sb - sab) / (R * (R - 1.0));
  }
  twos_request rr = *r;
  rr.walks = r->walks * static_cast<int>(rp->batches);
  const uint64_t record_d2h = (rp->walk_first ? nw * 24 : 0) + (rp->walk_u ? nw * 8 : 0) + (rp->walk_p ? nw * 8 : 0) +
                              (rp->site_radius ? static_cast<uint64_t>(n_sites) * 8 : 0);
  return finish(ro, n_sites, &rr, summary, seconds_since(t0), static_cast<uint64_t>(n_sites) * 24,
                nb * 16 + record_d2h);
}

int twos_ball_green_integral(const double *cases, uint32_t n, double *out, int device) {
  if (n == 0) return TWOS_OK;
  if (!cases || !out) return fail(TWOS_ERR_USAGE, "null buffer");
  DevBuf dc, dout, derr;
  uint32_t err = 0;
  try {
    check(cudaSetDevice(device), "cudaSetDevice");
    dc.reserve(static_cast<size_t>(n) * 4 * sizeof(double));
    dout.reserve(static_cast<size_t>(n) * sizeof(double));
    derr.reserve(sizeof(uint32_t));
    check(cudaMemcpy(dc.ptr, cases, static_cast<size_t>(n) * 4 * sizeof(double), cudaMemcpyHostToDevice), "upload");
    check(cudaMemset(derr.ptr, 0, sizeof(uint32_t)), "memset");
    check(launch_ball_green(dc.as<double>(), n, dout.as<double>(), derr.as<uint32_t>(), nullptr), "launch");
    check(cudaMemcpy(out, dout.ptr, static_cast<size_t>(n) * sizeof(double), cudaMemcpyDeviceToHost), "download");
    check(cudaMemcpy(&err, derr.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost), "download");
  } catch (const std::exception &e) {
    for (DevBuf *b : {&dc, &dout, &derr}) b->release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  for (DevBuf *b : {&dc, &dout, &derr}) b->release();
  if (err) return fail(TWOS_ERR_RUNTIME, "negative analytic Green integral");
  return TWOS_OK;
}

int twos_diffwos(twos_mesh *m, const twos_request *r, double diff_offset, int enclosure_fallback,
                 const double *sites, uint32_t n_sites, const double *cavities, uint32_t n_cav,
                 twos_diff_result *out, twos_diff_stats *stats, twos_summary *summary) {
  if (!m || !r) return fail(TWOS_ERR_USAGE, "null mesh or request");
  if (r->mode == TWOS_MODE_PAIRED) return fail(TWOS_ERR_USAGE, "Differential WoS takes one source");
  if (n_cav == 0 || !cavities) return fail(TWOS_ERR_USAGE, "Differential WoS requires --cavities");
  if (!(diff_offset > r->epsilon)) return fail(TWOS_ERR_USAGE, "diff_offset must exceed epsilon");
  if (int rc = validate_request(r, n_sites, n_cav)) return rc;
  if (n_sites == 0) return finish(RunOut{}, 0, r, summary, 0.0, 0, 0);
  if (!sites || !out) return fail(TWOS_ERR_USAGE, "null buffer");
  const auto t0 = std::chrono::steady_clock::now();
  RunOut ro;
  unsigned long long tot[kDiffTotals] = {};
  DevBuf hits, osteps, flags, start, nu, nsteps, rows, st, dtot;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    const bool mixed = r->precision == TWOS_PREC_MIXED;
    const size_t vbytes = mixed ? sizeof(float) : sizeof(double);
    const size_t walks = static_cast<size_t>(r->walks);
    const size_t chunk = std::max<size_t>(1, std::min<size_t>(n_sites, std::max<size_t>(1, m->max_launch_walks / walks)));
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    m->cavities.reserve(static_cast<size_t>(n_cav) * 3 * sizeof(double));
    check(cudaMemcpyAsync(m->cavities.ptr, cavities, static_cast<size_t>(n_cav) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload cavities");
    const size_t cw = chunk * walks;
    hits.reserve(cw * sizeof(HitRec));
    osteps.reserve(cw * sizeof(uint32_t));
    flags.reserve(cw * sizeof(uint32_t));
    start.reserve(cw * 3 * sizeof(double));
    nu.reserve(cw * vbytes);
    nsteps.reserve(cw * sizeof(uint32_t));
    rows.reserve(static_cast<size_t>(n_sites) * n_cav * sizeof(twos_diff_result));
    st.reserve(static_cast<size_t>(n_sites) * sizeof(twos_diff_stats));
    dtot.reserve(sizeof(tot));
    check(cudaMemsetAsync(dtot.ptr, 0, sizeof(tot), m->stream), "memset");
    begin_totals(m);
    // Outer walks (no payoff) on stream s; nested walks on stream s + 1.
    twos_request ro_req = *r;
    ro_req.n_source = ro_req.n_adjoint = 0;
    ro_req.green = 0;
    ro_req.skip_cavity_sites = 0;
    twos_request rn_req = *r;
    rn_req.mode = TWOS_MODE_COMPLIANCE;
    rn_req.stream = r->stream + 1;
    rn_req.skip_cavity_sites = 0;
    for (size_t first = 0; first < n_sites; first += chunk) {
      const uint32_t count = static_cast<uint32_t>(std::min<size_t>(chunk, n_sites - first));
      const uint64_t cwalks = static_cast<uint64_t>(count) * walks;
      for (int pass = 0; pass < 2; ++pass) {
        const twos_request *rq = pass == 0 ? &ro_req : &rn_req;
        std::vector<TermDev> terms;
        const JobDesc J = make_job(m, rq, count, static_cast<uint32_t>(first), r->site_offset + static_cast<uint32_t>(first),
                                   0, 0, 0, 0, n_cav, terms);
        if (terms.empty()) terms.push_back(TermDev{});
        m->jobs.reserve(sizeof(JobDesc));
        m->terms.reserve(terms.size() * sizeof(TermDev));
        check(cudaMemcpyAsync(m->jobs.ptr, &J, sizeof(JobDesc), cudaMemcpyHostToDevice, m->stream), "upload job");
        check(cudaMemcpyAsync(m->terms.ptr, terms.data(), terms.size() * sizeof(TermDev), cudaMemcpyHostToDevice,
                              m->stream),
              "upload terms");
        check(cudaMemsetAsync(m->counter.ptr, 0, sizeof(unsigned long long), m->stream), "memset");
        WosLaunch L{};
        L.jobs = m->jobs.as<JobDesc>();
        L.n_jobs = 1;
        L.geos = m->geo.as<GeoDesc>();
        L.n_geos = 1;
        L.sites = m->sites.as<double>();
        L.terms = m->terms.as<TermDev>();
        L.n_terms = static_cast<uint32_t>(terms.size());
        L.cavities = m->cavities.as<double>();
        L.total_walks = cwalks;
        L.counter = m->counter.as<unsigned long long>();
        L.error = reinterpret_cast<uint32_t *>(m->totals.as<unsigned long long>() + 2);
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
        L.counters = m->totals.as<unsigned long long>() + 3;
        L.site_best2 = nullptr;
        L.total_sites = count;
        const int mode = pass == 0 ? kModeBoundary : TWOS_MODE_COMPLIANCE;
        const int green = pass == 1 ? rq->green : TWOS_SOURCE_CENTER;
        if (pass == 0) {
          L.hits = hits.as<HitRec>();
          L.steps_out = osteps.as<uint32_t>();
          L.u_out = nu.ptr;  // unused in boundary mode
        } else {
          L.walk_start = start.as<double>();
          L.u_out = nu.ptr;
          L.steps_out = nsteps.as<uint32_t>();
        }
        const int block = m->block;
        const int per_sm = wos_max_blocks_per_sm(r->precision, mode, green, block, L);
        if (per_sm <= 0) throw std::runtime_error("WoS kernel cannot be resident on this device");
        const int grid = std::min(per_sm, m->blocks_per_sm > 0 ? m->blocks_per_sm : per_sm) * m->num_sms;
        check(launch_wos(r->precision, mode, green, L, grid, block, m->stream), "walk launch");
        ro.launches += 1;
        if (pass == 0) {
          DiffLaunch D{};
          D.geo = m->geo.as<GeoDesc>();
          D.cavities = m->cavities.as<double>();
          D.n_cav = n_cav;
          D.cavity_radius = r->cavity_radius;
          D.diff_offset = diff_offset;
          D.epsilon = r->epsilon;
          D.enclosure_fallback = enclosure_fallback;
          D.total_walks = cwalks;
          D.hits = hits.as<HitRec>();
          D.outer_steps = osteps.as<uint32_t>();
          D.flags = flags.as<uint32_t>();
          D.start = start.as<double>();
          D.totals = dtot.as<unsigned long long>();
          D.error = L.error;
          check(launch_diff_classify(D, m->stream), "classify launch");
          ro.launches += 1;
        }
      }
      DiffLaunch D{};
      D.n_cav = n_cav;
      D.diff_offset = diff_offset;
      D.n_sites = count;
      D.walks = static_cast<uint32_t>(walks);
      D.site_begin = static_cast<uint32_t>(first);
      D.hits = hits.as<HitRec>();
      D.outer_steps = osteps.as<uint32_t>();
      D.flags = flags.as<uint32_t>();
      D.nested_u = nu.ptr;
      D.nested_steps = nsteps.as<uint32_t>();
      D.out = rows.as<twos_diff_result>();
      D.stats = st.as<twos_diff_stats>();
      D.totals = dtot.as<unsigned long long>();
      check(launch_diff_reduce(r->precision, D, m->stream), "reduce launch");
      ro.launches += 1;
    }
    check(cudaMemcpyAsync(out, rows.ptr, static_cast<size_t>(n_sites) * n_cav * sizeof(twos_diff_result),
                          cudaMemcpyDeviceToHost, m->stream),
          "download rows");
    if (stats)
      check(cudaMemcpyAsync(stats, st.ptr, static_cast<size_t>(n_sites) * sizeof(twos_diff_stats),
                            cudaMemcpyDeviceToHost, m->stream),
            "download stats");
    check(cudaMemcpyAsync(tot, dtot.ptr, sizeof(tot), cudaMemcpyDeviceToHost, m->stream), "download totals");
    end_totals(m, ro);
  } catch (const std::exception &e) {
    for (DevBuf *b : {&hits, &osteps, &flags, &start, &nu, &nsteps, &rows, &st, &dtot}) b->release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  for (DevBuf *b : {&hits, &osteps, &flags, &start, &nu, &nsteps, &rows, &st, &dtot}) b->release();
  const double secs = seconds_since(t0);
  // Queries as the study backend counts them: one closest-point query per
  // step of the outer and nested walks plus the terminal one of every walk
  // that was not capped, and the classification's distance queries.
  const uint64_t outer_walks = static_cast<uint64_t>(n_sites) * static_cast<uint64_t>(r->walks);
  const uint64_t nested_walks = tot[7] - tot[6];
  if (summary) {
    std::memset(summary, 0, sizeof(*summary));
    summary->kernel_seconds = secs;
    summary->total_seconds = secs;
    summary->paths = outer_walks;
    summary->steps = tot[3] + tot[4];
    summary->caps = tot[5];
    summary->queries = tot[3] + (outer_walks - tot[8]) + tot[4] + (nested_walks - tot[9]) + tot[0];
    summary->launches = ro.launches;
    summary->error_flags = ro.error_flags;
    summary->node_tests = tot[1];       // parity rays
    summary->plane_tests = tot[2];      // enclosure fallbacks
    summary->triangle_tests = tot[6];   // unsafe offsets
  }
  if (ro.error_flags & TWOS_DEVERR_QUERY) return fail(TWOS_ERR_RUNTIME, "closest-point query failed");
  if (ro.error_flags) return fail(TWOS_ERR_RUNTIME, "device error");
  if (tot[6] || tot[5])
    return fail(TWOS_ERR_RUNTIME, "unsafe differential path: unsafe=" + std::to_string(tot[6]) +
                                      " caps=" + std::to_string(tot[5]));
  return TWOS_OK;
}

int twos_walk_samples(twos_mesh *m, const twos_request *r, const double *sites, uint32_t n_sites,
                      const double *cavities, uint32_t n_cavities, double *u, double *p, uint32_t *steps) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  if (int rc = validate_request(r, n_sites, n_cavities)) return rc;
  if (n_sites == 0) return TWOS_OK;
  if (!sites || !u || !steps) return fail(TWOS_ERR_USAGE, "null buffer");
  const size_t total = static_cast<size_t>(n_sites) * static_cast<size_t>(r->walks);
  if (total > m->max_launch_walks) return fail(TWOS_ERR_USAGE, "too many walks for one sample request");
  RunOut ro;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    m->out.reserve(static_cast<size_t>(n_sites) * sizeof(twos_site_result));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    run_estimate(m, r, m->sites.as<double>(), n_sites, cavities, n_cavities, m->out.as<twos_site_result>(), ro,
                 true);
    const bool mixed = r->precision == TWOS_PREC_MIXED;
    const bool paired = r->mode == TWOS_MODE_PAIRED;
    if (mixed) {
      std::vector<float> tmp(total);
      check(cudaMemcpy(tmp.data(), m->u.ptr, total * sizeof(float), cudaMemcpyDeviceToHost), "download");
      for (size_t i = 0; i < total; ++i) u[i] = tmp[i];
      if (p) {
        if (paired) {
          check(cudaMemcpy(tmp.data(), m->p.ptr, total * sizeof(float), cudaMemcpyDeviceToHost), "download");
          for (size_t i = 0; i < total; ++i) p[i] = tmp[i];
        } else {
          std::fill(p, p + total, 0.0);
        }
      }
    } else {
      check(cudaMemcpy(u, m->u.ptr, total * sizeof(double), cudaMemcpyDeviceToHost), "download");
      if (p) {
        if (paired)
          check(cudaMemcpy(p, m->p.ptr, total * sizeof(double), cudaMemcpyDeviceToHost), "download");
        else
          std::fill(p, p + total, 0.0);
      }
    }
    check(cudaMemcpy(steps, m->steps.ptr, total * sizeof(uint32_t), cudaMemcpyDeviceToHost), "download");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  if (ro.error_flags & TWOS_DEVERR_QUERY) return fail(TWOS_ERR_RUNTIME, "closest-point query failed");
  if (ro.error_flags) return fail(TWOS_ERR_RUNTIME, "device error");
  return TWOS_OK;
}

int twos_trace_grid_steps(twos_mesh *m, const twos_request *r, const double *sites, uint32_t n_sites,
                          uint64_t capacity, double *points, double *bounds, uint64_t *count) {
  if (!m || !count || (capacity && (!points || !bounds))) return fail(TWOS_ERR_USAGE, "null argument");
  if (int rc = validate_request(r, n_sites, 0)) return rc;
  if (r->precision != TWOS_PREC_MIXED || r->mode != TWOS_MODE_COMPLIANCE || r->green != TWOS_SOURCE_CENTER)
    return fail(TWOS_ERR_USAGE, "the grid-step trace runs the mixed compliance form with the centre source");
  if (capacity > 0xffffffffull) return fail(TWOS_ERR_USAGE, "trace capacity too large");
  if (n_sites == 0) {
    *count = 0;
    return TWOS_OK;
  }
  if (!sites) return fail(TWOS_ERR_USAGE, "null buffer");
  const size_t walks = static_cast<size_t>(n_sites) * static_cast<size_t>(r->walks);
  if (walks > m->max_launch_walks) return fail(TWOS_ERR_USAGE, "too many walks for one traced launch");
  RunOut ro;
  DevBuf rec, cnt;
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    rec.reserve(std::max<uint64_t>(capacity, 1) * sizeof(float4));
    cnt.reserve(sizeof(unsigned long long));
    check(cudaMemsetAsync(cnt.ptr, 0, sizeof(unsigned long long), m->stream), "memset");
    m->sites.reserve(static_cast<size_t>(n_sites) * 3 * sizeof(double));
    m->out.reserve(static_cast<size_t>(n_sites) * sizeof(twos_site_result));
    check(cudaMemcpyAsync(m->sites.ptr, sites, static_cast<size_t>(n_sites) * 3 * sizeof(double),
                          cudaMemcpyHostToDevice, m->stream),
          "upload sites");
    begin_totals(m);
    const TraceOut t{rec.as<float4>(), cnt.as<unsigned long long>(), static_cast<uint32_t>(capacity)};
    JobSpec js{m, r, n_sites, 0, r->site_offset, nullptr, 0};
    run_launch(m, {js}, m->sites.as<double>(), m->out.as<twos_site_result>(), ro, nullptr, &t);
    end_totals(m, ro);
    unsigned long long total = 0;
    check(cudaMemcpy(&total, cnt.ptr, sizeof(total), cudaMemcpyDeviceToHost), "download count");
    const uint64_t kept = std::min<uint64_t>(total, capacity);
    std::vector<float4> host(kept);
    if (kept) check(cudaMemcpy(host.data(), rec.ptr, kept * sizeof(float4), cudaMemcpyDeviceToHost), "download trace");
    for (uint64_t i = 0; i < kept; ++i) {
      // FP32 frame -> original coordinates (exact in FP64).
      points[3 * i] = static_cast<double>(host[i].x) + m->center[0];
      points[3 * i + 1] = static_cast<double>(host[i].y) + m->center[1];
      points[3 * i + 2] = static_cast<double>(host[i].z) + m->center[2];
      bounds[i] = static_cast<double>(host[i].w);
    }
    *count = total;
  } catch (const std::exception &e) {
    rec.release();
    cnt.release();
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  rec.release();
  cnt.release();
  if (ro.error_flags) return fail(TWOS_ERR_RUNTIME, "device error");
  return TWOS_OK;
}

int twos_sobol_directions(uint32_t dims, uint32_t bits, uint32_t *out) {
  if (!out || dims == 0 || dims > 65536 || bits == 0 || bits > 32)
    return fail(TWOS_ERR_USAGE, "invalid Sobol direction arguments");
  try {
    const std::vector<uint32_t> t = sobol_directions(dims, bits);
    std::copy(t.begin(), t.end(), out);
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return TWOS_OK;
}

int twos_l2_read_gbs(int device, uint64_t bytes, uint32_t passes, double *gbs) {
  if (!gbs || bytes < 1024 || bytes % 32 || passes == 0) return fail(TWOS_ERR_USAGE, "invalid L2 probe arguments");
  void *buf = nullptr;
  uint32_t *sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = TWOS_OK;
  try {
    check(cudaSetDevice(device), "cudaSetDevice");
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device attribute");
    check(cudaMalloc(&buf, bytes), "cudaMalloc");
    check(cudaMalloc(&sink, sizeof(uint32_t)), "cudaMalloc");
    check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    check(cudaMemsetAsync(buf, 0, bytes, st), "memset");
    const int blocks = 8 * sms;  // 2048 threads per SM
    check(launch_l2_read(buf, bytes, 2, sink, blocks, st), "L2 probe");  // warm the L2
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
      check(cudaEventRecord(e0, st), "event");
      check(launch_l2_read(buf, bytes, static_cast<int>(passes), sink, blocks, st), "L2 probe");
      check(cudaEventRecord(e1, st), "event");
      check(cudaEventSynchronize(e1), "L2 probe");
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, e0, e1), "event time");
      best = std::max(best, static_cast<double>(bytes) * passes / (ms * 1e-3) / 1e9);
    }
    *gbs = best;
  } catch (const std::exception &e) {
    rc = fail(TWOS_ERR_RUNTIME, e.what());
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (buf) cudaFree(buf);
  if (sink) cudaFree(sink);
  return rc;
}

int twos_finalize_samples(twos_mesh *m, int precision, int mode, const double *u, const double *p,
                          const uint32_t *steps, uint32_t n_sites, uint32_t walks, twos_site_result *out) {
  if (!m) return fail(TWOS_ERR_USAGE, "null mesh");
  if (precision != TWOS_PREC_FP64 && precision != TWOS_PREC_MIXED) return fail(TWOS_ERR_USAGE, "invalid precision");
  if (mode != TWOS_MODE_COMPLIANCE && mode != TWOS_MODE_PAIRED && mode != TWOS_MODE_HOT)
    return fail(TWOS_ERR_USAGE, "invalid mode");
  if (walks < 2) return fail(TWOS_ERR_USAGE, "walks must be at least 2");
  if (n_sites == 0) return TWOS_OK;
  const bool paired = mode == TWOS_MODE_PAIRED;
  if (!u || !out || (paired && !p)) return fail(TWOS_ERR_USAGE, "null buffer");
  const size_t total = static_cast<size_t>(n_sites) * walks;
  if (total > m->max_launch_walks) return fail(TWOS_ERR_USAGE, "too many samples for one launch");
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    const bool mixed = precision == TWOS_PREC_MIXED;
    const size_t vbytes = mixed ? sizeof(float) : sizeof(double);
    m->u.reserve(total * vbytes);
    if (paired) m->p.reserve(total * vbytes);
    m->steps.reserve(total * sizeof(uint32_t));
    m->out.reserve(static_cast<size_t>(n_sites) * sizeof(twos_site_result));
    m->jobs.reserve(sizeof(JobDesc));
    auto upload = [&](const double *src, DevBuf &dst) {
      if (mixed) {
        std::vector<float> tmp(src, src + total);
        check(cudaMemcpy(dst.ptr, tmp.data(), total * sizeof(float), cudaMemcpyHostToDevice), "upload samples");
      } else {
        check(cudaMemcpy(dst.ptr, src, total * sizeof(double), cudaMemcpyHostToDevice), "upload samples");
      }
    };
    upload(u, m->u);
    if (paired) upload(p, m->p);
    if (steps)
      check(cudaMemcpy(m->steps.ptr, steps, total * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload steps");
    else
      check(cudaMemset(m->steps.ptr, 0, total * sizeof(uint32_t)), "memset");
    JobDesc J{};
    J.n_sites = n_sites;
    J.walks = walks;
    check(cudaMemcpy(m->jobs.ptr, &J, sizeof(JobDesc), cudaMemcpyHostToDevice), "upload job");
    begin_totals(m);
    FinalizeLaunch F{};
    F.jobs = m->jobs.as<JobDesc>();
    F.n_jobs = 1;
    F.total_sites = n_sites;
    F.totals = m->totals.as<unsigned long long>();
    F.u = m->u.ptr;
    F.p = paired ? m->p.ptr : m->u.ptr;
    F.steps = m->steps.as<uint32_t>();
    F.out = m->out.as<twos_site_result>();
    check(launch_finalize(precision, mode, F, m->stream), "finalize launch");
    check(cudaMemcpyAsync(out, m->out.ptr, static_cast<size_t>(n_sites) * sizeof(twos_site_result),
                          cudaMemcpyDeviceToHost, m->stream),
          "download results");
    check(cudaStreamSynchronize(m->stream), "finalize");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return TWOS_OK;
}

int twos_inside(twos_mesh *m, const double *points, uint64_t n, uint8_t *inside) {
  if (!m || (n && (!points || !inside))) return fail(TWOS_ERR_USAGE, "null argument");
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t threads = std::min<uint64_t>(hw, std::max<uint64_t>(1, n / 1024));
  std::vector<std::string> errs(threads);
  std::vector<int> codes(threads, 0);
  std::vector<std::thread> pool;
  for (uint64_t t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      for (uint64_t i = t; i < n; i += threads) {
        bool in = false;
        if (inside_parity(m->bvh, m->vertices, m->faces, points + 3 * i, in, errs[t])) {
          codes[t] = 1;
          return;
        }
        inside[i] = in ? 1 : 0;
      }
    });
  }
  for (auto &th : pool) th.join();
  for (uint64_t t = 0; t < threads; ++t)
    if (codes[t]) return fail(TWOS_ERR_RUNTIME, errs[t]);
  return TWOS_OK;
}

int twos_topk_device(twos_mesh *m, const double *d_keys, uint32_t n, uint32_t k, uint32_t *d_index) {
  if (!m || (n && (!d_keys || !d_index))) return fail(TWOS_ERR_USAGE, "null argument");
  if (k > 1024) return fail(TWOS_ERR_USAGE, "k must be at most 1024");
  if (k > n) return fail(TWOS_ERR_USAGE, "k must not exceed n");
  try {
    check(cudaSetDevice(m->device), "cudaSetDevice");
    const size_t bytes = topk_scratch_bytes(n, k);
    m->topk.reserve(bytes);
    check(launch_topk(d_keys, n, k, d_index, m->topk.ptr, m->topk.bytes, m->stream), "topk launch");
    check(cudaStreamSynchronize(m->stream), "topk kernels");
  } catch (const std::exception &e) {
    return fail(TWOS_ERR_RUNTIME, e.what());
  }
  return TWOS_OK;
}

}  // extern "C"

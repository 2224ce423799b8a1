// Internal layouts shared by the host code (twos_abi.cpp, bvh.cpp) and the
// CUDA kernels (kernels.cu) of libtwos.so.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "twos.h"

namespace twos {

// ---------------------------------------------------------------- BVH layouts
// Binary BVH; each node stores both children's boxes so one node fetch gives
// the two box tests.  Child encoding: >= 0 internal node index; < 0 leaf with
// ~child = (first_triangle << 3) | count (count 0..7, 0 = empty child whose
// box is inverted so it is never entered).
constexpr int kLeafMax = 4;
constexpr int kMaxDepth = 24;    // builder bound (<= 4 * 2^24 triangles); one stack entry per level
constexpr int kStack = 24;

// Each child also carries a normal slab: a unit direction n (the child's
// area-weighted mean normal) and the interval [smin, smax] of n.v over its
// vertices, rounded outward.  A child whose normals cancel gets n = 0 and
// [0, 0], which bounds nothing.

// FP32 node: 96 bytes, six 16-byte loads.  x = (l.lo.x, r.lo.x, l.hi.x, r.hi.x),
// likewise y and z; nl = (l.n, l.smin), nr = (r.n, r.smin);
// tail = (l.smax, r.smax, left child bits, right child bits).
struct alignas(32) NodeF {
  float4 x, y, z;
  float4 nl, nr;
  float4 tail;
};
static_assert(sizeof(NodeF) == 96, "NodeF layout");

// Four-wide FP32 node (the mixed form's BVH width 4, collapsed from the
// binary BVH: a node's slots are its binary children, each internal child
// replaced by its own two children): 192 bytes, six 32-byte loads.  Slot c
// of every float4 is child c: box lo/hi per axis, normal slab (n, smin,
// smax), child code as in the binary layout.  An empty slot has an inverted
// box and n = 0, so it is never entered.
struct alignas(32) Node4F {
  float4 xlo, xhi, ylo, yhi, zlo, zhi;
  float4 nx, ny, nz, smin, smax;
  int4 child;
};
static_assert(sizeof(Node4F) == 192, "Node4F layout");

// FP64 node: 192 bytes.  lo/hi pairs (left, right) per axis, slabs, children.
struct alignas(16) NodeD {
  double2 xlo, xhi, ylo, yhi, zlo, zhi;
  double2 nl_xy, nl_zmin, nr_xy, nr_zmin, smax;
  int4 child;
};
static_assert(sizeof(NodeD) == 192, "NodeD layout");

// FP32 triangle: 64 bytes: plane slab (n.xyz, dmin), (a.xyz, dmax),
// (b.xyz, original id bits), (c.xyz, 0).  n is the unit normal; the vertices
// satisfy dmin <= n.v <= dmax (rounded outward); degenerate triangles carry
// n = 0, which never rejects.
struct alignas(64) TriF {
  float4 plane, a, b, c;
};
static_assert(sizeof(TriF) == 64, "TriF layout");

// FP64 triangle: 128 bytes, eight 16-byte loads.
struct alignas(16) TriD {
  double2 nxy, nzmin, dmax_id;
  double2 axy, azbx, bybz, cxy, czpad;
};
static_assert(sizeof(TriD) == 128, "TriD layout");

// Host-side BVH produced by the builder (bvh.cpp).
struct HostBvh {
  struct Node {
    double lo[2][3], hi[2][3];  // child boxes (left, right)
    int32_t child[2];
  };
  std::vector<Node> nodes;      // nodes[0] is the root (always internal)
  std::vector<uint32_t> order;  // leaf triangle order -> original triangle index
  int depth = 0;
};

void build_bvh(const std::vector<double> &vertices, const std::vector<uint32_t> &faces, HostBvh &out);

// Packs the host BVH into device layouts.  FP32 coordinates are taken about
// `center`; boxes are taken from the rounded FP32 vertices so they contain the
// FP32 triangles exactly.
void pack_bvh_f32(const HostBvh &bvh, const std::vector<double> &vertices, const std::vector<uint32_t> &faces,
                  const double center[3], std::vector<NodeF> &nodes, std::vector<TriF> &tris);
void pack_bvh_f64(const HostBvh &bvh, const std::vector<double> &vertices, const std::vector<uint32_t> &faces,
                  std::vector<NodeD> &nodes, std::vector<TriD> &tris);

// Entry-node table of the mixed form's closest-point query: for each cell of
// a uniform grid (cell size `cell`, `dims` cells from `origin`, original
// coordinates), the deepest BVH node whose subtree holds every triangle
// within `radius` of the cell grown by `pad` (0, the root, when none is).
// A query at a point of the cell whose initial bound is below `radius`
// (less the FP32 error) may start its traversal there: every triangle
// outside that subtree is farther than the bound.
std::vector<int32_t> build_entry_table(const HostBvh &bvh, const double origin[3], double cell, const uint32_t dims[3],
                                       double radius, double pad);

// The four-wide FP32 BVH collapsed from the packed binary one; cover[n] is,
// for every binary node n, the four-wide node whose subtree is n's or holds
// it (n's own node, or its parent's when n was absorbed into it).
void pack_bvh4_f32(const HostBvh &bvh, const std::vector<NodeF> &binary, std::vector<Node4F> &nodes4,
                   std::vector<int32_t> &cover);

// Host ray-parity membership over the host BVH (EmbreeMesh::inside).
int inside_parity(const HostBvh &bvh, const std::vector<double> &vertices, const std::vector<uint32_t> &faces,
                  const double p[3], bool &inside, std::string &err);

// ASCII PLY reader with the reference's rules; throws std::runtime_error.
void load_ascii_ply(const std::string &path, std::vector<double> &vertices, std::vector<uint32_t> &faces);
// CSV/whitespace point reader (wih_twos.cpp:508-522); throws when empty.
std::vector<double> read_points(const std::string &path);

// ---------------------------------------------------------------- launch descriptors
// One geometry resident on the device.
struct GeoDesc {
  const NodeF *nodes_f;
  const Node4F *nodes4_f;  // the same BVH four wide (mixed form, bvh_width 4)
  const TriF *tris_f;
  const NodeD *nodes_d;
  const TriD *tris_d;
  double center[3];   // FP32 frame origin (mixed form)
  float delta;        // FP32 distance error bound (mixed form)
  uint32_t max_iter;  // traversal iteration bound (node + leaf visits)
  // Distance-bound grid of the mixed form (null: none).  Vertex (i, j, k)
  // sits at grid_lo + (i, j, k) * grid_h in the FP32 frame; D(v) * grid_q
  // is a lower bound of its distance to the surface.  Stored by cell, so a
  // lookup is one 16-byte load: record grid[(i * (n1 - 1) + j) * (n2 - 1) + k]
  // of cell (i, j, k) holds in .z (low 16 bits) the smallest D of its eight
  // corners (i + a, j + b, k + c), in byte corner & 3 of .x (corners 0-3) or
  // .y (corners 4-7), corner = a * 4 + b * 2 + c, each corner's D minus that
  // base (255: saturated or too far above the base -- the base alone is used
  // and the corner gives no upper bound), and in .w the cell's entry node
  // (-1: none).  D varies by at most sqrt(3) h / grid_q + 1 < 224 over a
  // cell, so the bytes hold every unsaturated corner exactly.
  const uint4 *grid;
  float grid_lo[3];
  float grid_h, grid_inv_h, grid_q;
  uint32_t grid_n[3];
  // Entry nodes (in the grid's records): the BVH node a query may start
  // from at a point of the cell when its initial bound is below
  // entry_radius (every triangle outside that node's subtree is farther).
  // The host table behind them has cells of 2^entry_shift grid cells per
  // axis, entry_n[] of them.
  uint32_t entry_shift;
  uint32_t entry_n[3];
  float entry_radius;
};

// One job = one geometry x a contiguous range of sites with one request.
struct JobDesc {
  uint64_t walk_begin;   // first global walk id of the job
  uint32_t n_sites;
  uint32_t walks;
  uint32_t site_begin;   // index of the job's first site in the sites/results arrays
  uint32_t site_offset;  // added to the local site index in the sample key
  uint32_t geo;
  uint32_t k0, k1;       // Philox key
  uint32_t repeat;
  int32_t max_steps;
  uint32_t flags;        // kJobGreen | kJobSkipCavitySites | kJobExactSource
  double epsilon;
  double query_radius2;  // squared initial radius (+inf when unbounded)
  double cavity_radius;
  uint32_t src_begin, n_src, adj_begin, n_adj;
  uint32_t cav_begin, n_cav;
  uint32_t site_rank;    // sites of the launch's earlier jobs (finalize lookup)
  uint32_t bnd_begin, n_bnd;  // Dirichlet data of u on the mesh (term range)
  uint32_t pad;
};
constexpr uint32_t kJobGreen = 1u;
constexpr uint32_t kJobSkipCavitySites = 2u;
constexpr uint32_t kJobExactSource = 4u;  // TWOS_SOURCE_EXACT

struct TermDev {
  int32_t kind;
  int32_t axis;
  double amp, offset, div;
  double c[3], w[3];
};
static_assert(sizeof(TermDev) == sizeof(twos_source_term), "term layout");

struct WosLaunch {
  const JobDesc *jobs;
  uint32_t n_jobs;
  const GeoDesc *geos;
  uint32_t n_geos;
  const double *sites;      // [n][3], original coordinates
  const TermDev *terms;     // job term ranges index this table (frame of the job's geometry)
  uint32_t n_terms;
  const double *cavities;   // [n][3]
  uint64_t total_walks;
  unsigned long long *counter;  // work-queue head, zeroed before launch
  uint32_t *error;              // TWOS_DEVERR_* bits
  void *u_out;                  // per-walk u: float (mixed) or double (fp64)
  void *p_out;                  // per-walk p (paired), same type
  uint32_t *steps_out;          // per-walk steps | cap << 31
  int refill;                   // refill a warp once this many lanes are idle
  int step_threshold;           // step a warp's walks once this many queries are done
  unsigned long long *counters; // [0] node tests, [1] triangle plane tests, [2] full triangle tests,
                                // [3] grid steps
  // Squared mesh distance at each launch site (index site_rank + site), from
  // the pre-pass; every walk of a site starts from the same point, so its
  // first query is answered from here (-1 when nothing is within range).
  void *site_best2;
  uint32_t total_sites;
  int vote;  // 1: a warp runs one kind of traversal unit per iteration (majority vote)
  // 1: a step's query starts from the distance to the previous query's
  // nearest triangle (an upper bound attained by a real triangle, so the
  // traversal's minimum -- and every walk -- is unchanged; it only prunes
  // from the first node on).
  int warm;
  // Per-walk start points [total_walks][3] (original coordinates); a walk whose
  // start is NaN is skipped (zero value, zero steps).  Null: walks start at
  // their site.
  const double *walk_start;
  // Boundary mode (kModeBoundary): per-walk boundary hit of the terminal step.
  struct HitRec *hits;
  // Gradient mode (kModeGradient): per-walk grad U and grad P, 6 values of
  // the walk type per walk.
  void *grad_out;
  // Mixed form: a step whose grid bound is at least grid_tau spacings takes
  // it as the ball radius instead of querying the BVH (0: never).
  float grid_tau;
  // Traversal units (node visits / triangle tests) a lane runs back to back
  // per iteration of the warp loop (>= 1).
  int units;
  // Walks a lane claims from the work queue at once and runs one after
  // another (>= 1).
  int lane_walks;
  // Mixed form: whether a query may start at the entry-node table's node.
  int entry;
  // FP64 compliance form with the mixed form's distance grid and entry nodes
  // (a comparison of precision alone; off for the plain FP64 form).
  int grid64;
  // Mixed form: traverse the four-wide BVH (compliance, paired and hot
  // modes with the centre or Green-point source; others stay binary).
  int wide;
  // Optional record of every grid step (tests): position in the FP32 frame
  // and the bound used, at most trace_cap records; trace_count counts all.
  float4 *trace;
  unsigned long long *trace_count;
  uint32_t trace_cap;
};

// Walk-to-boundary mode of the walk kernel (walk_to_boundary,
// wih_twos.cpp:725-740): no payoff; each walk records its terminal hit.
constexpr int kModeBoundary = 3;
// Paired walks that also return first-ball gradient samples
// (twos_estimate_gradient).
constexpr int kModeGradient = 4;

// Boundary hit of a walk's terminal step (closest_boundary, wih_twos.cpp:
// 602-626), original coordinates.  cavity = -1 for the mesh, -2 when the
// walk hit the step cap or was skipped.
struct HitRec {
  double point[3];
  double normal[3];
  int32_t cavity;
  int32_t pad;
};

// Fills L.site_best2 (T per site, T = float for mixed, double for FP64).
cudaError_t launch_site_prepass(int precision, const WosLaunch &L, cudaStream_t s);

struct FinalizeLaunch {
  const JobDesc *jobs;
  uint32_t n_jobs;
  uint32_t total_sites;           // sites of this launch (sum of job n_sites)
  unsigned long long *totals;     // [0] += steps, [1] += caps
  const void *u;
  const void *p;
  const uint32_t *steps;
  twos_site_result *out;
};

// Array-RQMC / matched MC lockstep walks (rqmc.cuh): one block per
// (site, batch), blockDim = walks.
struct RqmcLaunch {
  const GeoDesc *geo;
  const double *sites;
  uint32_t n_sites, walks, batches;
  int method;                  // TWOS_RQMC_*
  uint32_t generator;          // Korobov generator a for `walks`
  uint32_t generator2;         // a^2 mod walks
  const TermDev *terms;        // [src | u boundary | p boundary]
  uint32_t n_src, n_ub, n_pb;
  uint32_t k0, k1, repeat;
  int max_steps;
  double epsilon;
  double lo[3], inv_extent[3];  // Hilbert quantization box (geometry frame of T)
  double *batch_u, *batch_p;   // [batches][n_sites]
  double *walk_first;          // optional [batches][n_sites][walks][3] (original coordinates)
  double *walk_u, *walk_p;     // optional [batches][n_sites][walks]
  double *site_radius;         // optional [n_sites]
  unsigned long long *totals;  // [0] steps, [1] caps
  uint32_t *error;
  // SOBOL: direction numbers [2 * kSobolSteps][kSobolBits] (sobol_directions)
  // and log2(walks), the index bits of a walk.
  const uint32_t *sobol_v;
  uint32_t sobol_bits;
};
cudaError_t launch_rqmc(int precision, const RqmcLaunch &R, cudaStream_t s);

// Sobol-over-steps RQMC: steps 0 .. kSobolSteps - 1 of a walk take the two
// coordinates (2k, 2k + 1) of its Sobol' point; later steps draw the matched
// MC stream.  kSobolBits index bits cover up to 1024 walks.
constexpr uint32_t kSobolSteps = 256, kSobolBits = 10;

// Sobol' direction numbers, `bits` per dimension, most significant digit
// first: v[d * bits + b] = m_{d, b+1} 2^(31-b).  Dimension 0 is van der
// Corput's (m = 1); dimension d >= 1 takes the d-th primitive polynomial over
// GF(2) (by degree, then by coefficient bits) with odd initial m_k < 2^k
// from SplitMix64 and Sobol's recurrence beyond its degree.
std::vector<uint32_t> sobol_directions(uint32_t dims, uint32_t bits);
cudaError_t launch_rqmc_reuse(const RqmcLaunch &R, cudaStream_t s);

// Gradient-mode finalize: one warp per site over u, p, grad u, grad p.
struct GradFinalizeLaunch {
  uint32_t n_sites, walks;
  const void *u, *p, *grad;     // per walk (float or double); grad 6 per walk
  const uint32_t *steps;
  twos_gradient_result *out;
  unsigned long long *totals;   // [0] += steps, [1] += caps
};
cudaError_t launch_grad_finalize(int precision, const GradFinalizeLaunch &F, cudaStream_t s);

// Differential WoS pass over one chunk of sites (diffwos.cuh).
constexpr uint32_t kDiffCavity = 1u, kDiffNearSeam = 2u, kDiffSegmentUnsafe = 4u, kDiffUnsafe = 8u;
struct DiffLaunch {
  const GeoDesc *geo;             // device
  const double *cavities;         // [n_cav][3], original coordinates
  uint32_t n_cav;
  double cavity_radius, diff_offset, epsilon;
  int enclosure_fallback;
  uint64_t total_walks;           // n_sites * walks
  uint32_t n_sites, walks, site_begin;
  const HitRec *hits;             // outer walks' terminal hits
  const uint32_t *outer_steps;    // steps | cap << 31
  uint32_t *flags;                // kDiff* per walk
  double *start;                  // nested start points [walks][3] (NaN = none)
  const void *nested_u;           // nested walk values (float or double)
  const uint32_t *nested_steps;
  twos_diff_result *out;          // [sites][n_cav], indexed by site_begin + site
  twos_diff_stats *stats;         // [sites] or null
  unsigned long long *totals;     // [0] queries [1] rays [2] fallbacks [3] outer steps [4] nested steps
                                  // [5] limits [6] unsafe [7] cavity terminations
                                  // [8] outer caps [9] nested caps (kDiffTotals words)
  uint32_t *error;
};
constexpr int kDiffTotals = 10;
cudaError_t launch_diff_classify(const DiffLaunch &D, cudaStream_t s);
cudaError_t launch_diff_reduce(int precision, const DiffLaunch &D, cudaStream_t s);

// One design-loop iteration record (layout of twos_design_step).
struct DesignStep {
  uint32_t chosen;
  uint32_t accepted;
  double scout_score, score, score_se, lower;
  uint32_t slot, n_cavities;
};
static_assert(sizeof(DesignStep) == sizeof(twos_design_step), "design step layout");

// Device buffers of the design loop (design.cu).
struct DesignLaunch {
  const double *candidates;            // [n][3]
  uint32_t n_candidates;
  uint32_t k;                          // shortlist size
  const twos_site_result *scout_rows;  // [n]
  uint8_t *feasible;                   // [n]
  double *keys;                        // [n]
  const uint32_t *shortlist;           // [k]
  double *val_sites;                   // [k][3]
  const twos_site_result *val_rows;    // [k]
  JobDesc *scout_job;
  JobDesc *val_job;
  double *cavities;                    // [max_cav][3]
  uint32_t max_cav;
  uint32_t max_iterations;
  double z, threshold, pair_clearance;
  uint32_t *iteration;
  DesignStep *history;                 // [max_iterations]
};

cudaError_t launch_design_keys(const DesignLaunch &D, cudaStream_t s);
cudaError_t launch_design_gather(const DesignLaunch &D, cudaStream_t s);
cudaError_t launch_design_select(const DesignLaunch &D, cudaStream_t s);
cudaError_t launch_design_mask(const DesignLaunch &D, cudaStream_t s);

// Kernel launchers (kernels.cu).  They return cudaGetLastError() of the launch.
cudaError_t launch_wos_traced(const WosLaunch &L, int grid, cudaStream_t s);
// Whether a walk-kernel launch of this many jobs, geometries and source
// terms keeps its descriptor tables in shared memory (else it reads them
// from global memory at every step).
bool launch_tables_in_smem(int precision, uint32_t n_jobs, uint32_t n_geos, uint32_t n_terms);

// Wavefront form of the mixed-precision walk (wavefront.cuh): the walks in
// flight live in `slots` slot records in device memory.
struct WfSlots {
  float4 *pos;       // FP32-frame position; w: the next step's squared radius
  uint4 *meta;       // launch walk id, steps, nearest triangle, flags | job << 8
  float2 *val;       // u, p accumulators
  int *node;         // start node of the slot's pending query
  uint32_t *queue;   // slots with a pending query
  uint32_t *counts;  // [0] queue length, [1] live slots after the step kernel
  uint32_t slots;
};
size_t wf_slot_bytes(uint32_t slots);
// Runs every walk of L (FP32, centre-point source, compliance / paired /
// hot; total walks below 2^32) through the wavefront kernels on stream s and
// waits for it.  max_iterations bounds the iterations (an error beyond).
cudaError_t launch_wos_wavefront(int mode, const WosLaunch &L, void *slot_mem, uint32_t slots, int num_sms,
                                 uint64_t max_iterations, cudaStream_t s);
cudaError_t launch_wos(int precision, int mode, int src, const WosLaunch &L, int grid, int block,
                       cudaStream_t s);
int wos_max_blocks_per_sm(int precision, int mode, int src, int block, const WosLaunch &L);
cudaError_t launch_finalize(int precision, int mode, const FinalizeLaunch &F, cudaStream_t s);
// Certified validation walks (validate.cuh), FP64 with directed rounding.
struct ValidateLaunch {
  const GeoDesc *geo;          // device descriptor (FP64 BVH and triangles used)
  const double *sites;         // [n_sites][3]
  uint32_t n_sites, walks;
  const double *cavities;      // [n_cav][3]
  uint32_t n_cav;
  const TermDev *terms;        // source terms (validated host-side)
  uint32_t n_terms;
  int green;                   // 1: Beta(2,2) Green point per step
  uint32_t k0, k1, repeat, site_offset;
  int max_steps;
  double epsilon, cavity_radius, radius_cap, value_cap;
  twos_cert_sample *samples;   // [n_sites * walks]
  double *clearance;           // [n_sites] certified distance at the site
  double *center_distance;     // [n_sites] FP64 domain distance at the site
  unsigned long long *totals;  // [0] containment failures [1] steps
  uint32_t *error;
};
cudaError_t launch_validate(const ValidateLaunch &V, cudaStream_t s);

// Exact ball integrals of bump sources: cases[4i..4i+3] = (d, r, R, A).
cudaError_t launch_ball_green(const double *cases, uint32_t n, double *out, uint32_t *error, cudaStream_t s);
// L2 read probe: `passes` sweeps of 32-byte loads over `bytes` of buf.
cudaError_t launch_l2_read(const void *buf, uint64_t bytes, int passes, uint32_t *sink, int blocks, cudaStream_t s);
cudaError_t launch_closest(int precision, const GeoDesc *geo_dev, const double *pts, uint64_t n,
                           double query_radius2, double *dist, double *closest, uint32_t *error, cudaStream_t s);
// Fills a geometry's distance-bound grid (n = vertices of the grid described
// in *geo_dev; its `grid` pointer is not read).
cudaError_t launch_grid_build(const GeoDesc *geo_dev, uint64_t n, double margin, uint16_t *out, uint32_t *error,
                              cudaStream_t s);
// Packs the per-vertex values (n[0] x n[1] x n[2], k fastest) and the entry
// table (may be null; entry_n[] cells of 2^shift grid cells) into the cell
// records of GeoDesc::grid.
cudaError_t launch_grid_pack(const uint16_t *vertices, const uint32_t n[3], const int32_t *table, uint32_t shift,
                             const uint32_t entry_n[3], uint4 *cells, cudaStream_t s);
// The walk step's grid bound at each point (original coordinates); NaN
// outside the grid.
cudaError_t launch_grid_bound(const GeoDesc *geo_dev, const double *pts, uint64_t n, double *out, cudaStream_t s);
cudaError_t launch_topk(const double *keys, uint32_t n, uint32_t k, uint32_t *index, void *scratch,
                        size_t scratch_bytes, cudaStream_t s);
size_t topk_scratch_bytes(uint32_t n, uint32_t k);

// Host copy of the counter-based key derivation (shared definition with the
// device draw layout): key = splitmix64(seed + golden * (stream + 1)).
void counter_key(uint64_t seed, uint32_t stream, uint32_t &k0, uint32_t &k1);

}  // namespace twos

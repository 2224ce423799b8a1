/*
 * twos.h -- C ABI of the B200-native TWoS (Topological Walk on Spheres)
 * estimator, libtwos.so.
 *
 * This is the drop-in boundary for the reference's compiled Embree/OpenMP
 * backend (hertjo/walking-into-holes).  The reference exposes that backend to
 * Python only as executables driven by argv, files and a --serve pipe
 * (benchmarks/compiled_bunny/src/wih_twos.cpp:137-240, 1799-1864;
 * benchmarks/distinct_adjoint/adjoint.cpp:91-158).  The executables built
 * from this library (wih_twos, wih_adjoint) keep that contract byte for byte;
 * this header is the in-process call underneath them, which a ctypes, cgo or
 * JNI binding can reach directly.  Each entry point names the reference code
 * it replaces.
 *
 * Conventions
 *   - Return codes: TWOS_OK (0), TWOS_ERR_RUNTIME (1: cap hit, non-finite
 *     distance, CUDA error, device wait limit), TWOS_ERR_USAGE (2: invalid
 *     argument).  These are the reference's process exit codes
 *     (wih_twos.cpp:134, 1860-1863).  twos_last_error() gives the message
 *     (thread-local, valid until the next call on the same thread).
 *   - Buffers passed to the host entry points are caller-owned host memory;
 *     device buffers are owned by the mesh session.  No C++ exception crosses
 *     this ABI.
 *   - A session is not thread-safe; it issues all work on one CUDA stream.
 *   - Points, cavities and vertices are arrays of 3 doubles (x, y, z).
 */
#ifndef TWOS_H
#define TWOS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TWOS_ABI_VERSION 2

enum { TWOS_OK = 0, TWOS_ERR_RUNTIME = 1, TWOS_ERR_USAGE = 2 };

/* Estimator modes.
 *   COMPLIANCE: one walk set, U = sum f r^2/6; score = (S^2 - S2)/(N(N-1))
 *               (wih_twos.cpp:674-717, the compliance TD -D_T = u^2).
 *   PAIRED:     one walk set with two payoffs u (source) and p (adjoint
 *               source) at a shared Green point; score = (SuSp - Sup)/(N(N-1))
 *               (adjoint.cpp:18-42, study.cpp:80-120).
 *   HOT:        PAIRED with the adjoint switched off; score = mean u
 *               (adjoint.cpp:38, --hot-only 1). */
enum { TWOS_MODE_COMPLIANCE = 0, TWOS_MODE_PAIRED = 1, TWOS_MODE_HOT = 2 };

/* Arithmetic of the walk.
 *   FP64:  positions, BVH boxes, triangles and distances in FP64 (the plain
 *          form; termination at r <= epsilon exactly as wih_twos.cpp:647).
 *   MIXED: positions, boxes, triangles and distances in FP32 about the mesh
 *          centre; each step radius is shrunk by a bound delta on the FP32
 *          distance error, and the walk stops when the shrunk radius is
 *          <= epsilon, so no walk steps through the boundary.  Per-site
 *          U-statistic accumulation stays in FP64. */
enum { TWOS_PREC_FP64 = 0, TWOS_PREC_MIXED = 1 };

/* Source terms; a source f(x) is the ordered sum of up to TWOS_MAX_TERMS terms.
 *   CONST  amp
 *   LINEAR amp * (x[axis] + offset)                 (affine, wih_twos.cpp:551)
 *   GAUSS  amp * exp(-sum_k ((x_k - c_k)/w_k)^2)     (housing, wih_twos.cpp:553-565)
 *   BUMP   amp * max(0, 1 - |x-c|^2/w0^2)^2 / div   (sensor, adjoint.cpp:11-15,
 *                                                    study.cpp:45-47)
 *   BOX    amp if c <= x <= w componentwise, else 0
 *   BALL   amp if |x - c| <= w0, else 0
 *   QUAD   amp * sum_k w_k (x_k - c_k)^2            (harmonic when sum w = 0;
 *                                                    boundary data, no
 *                                                    reference counterpart) */
enum {
  TWOS_TERM_CONST = 0,
  TWOS_TERM_LINEAR = 1,
  TWOS_TERM_GAUSS = 2,
  TWOS_TERM_BUMP = 3,
  TWOS_TERM_BOX = 4,
  TWOS_TERM_BALL = 5,
  TWOS_TERM_QUAD = 6
};

/* Per-step source integral over the walk's ball B_r(y), added to u (p):
 *   CENTER  r^2/6 f(y)                          (wih_twos.cpp:648-651, affine)
 *   GREEN   r^2/6 f(a), a = y + r beta w with beta ~ Beta(2,2), w uniform
 *           (wih_twos.cpp:569-575; adjoint.cpp:31; study.cpp:106-108)
 *   EXACT   the exact integral of the ball's Green function against f
 *           (study.cpp WIH_ANALYTIC_SOURCE, 53-77, 96-104): CONST and
 *           LINEAR terms contribute r^2/6 f(y) (f harmonic), each BUMP term
 *           A (1 - |x-c|^2/R^2)_+^2 (A = amp / div) its closed-form Newton-
 *           potential difference; other term kinds are rejected. */
enum {
  TWOS_SOURCE_CENTER = 0,
  TWOS_SOURCE_GREEN = 1,
  TWOS_SOURCE_EXACT = 2
};

#define TWOS_MAX_TERMS 8

typedef struct twos_source_term {
  int32_t kind;
  int32_t axis;
  double amp;
  double offset;
  double div;
  double c[3];
  double w[3];
} twos_source_term; /* 80 bytes */

/* One estimation request (the reference's Options, wih_twos.cpp:73-101, plus
 * the paired flags of adjoint.cpp:95-107). */
typedef struct twos_request {
  int32_t mode;       /* TWOS_MODE_* */
  int32_t precision;  /* TWOS_PREC_* */
  int32_t walks;      /* N >= 2 walks per site (--walks) */
  int32_t max_steps;  /* step cap per walk (--max-steps); reaching it is an error */
  uint64_t seed;      /* --seed */
  uint32_t repeat;    /* repeat index, part of the sample key */
  uint32_t stream;    /* independent stream id (0 estimate, 1 fresh validation, ...) */
  double epsilon;     /* termination shell (--epsilon) */
  double cavity_radius;  /* common radius of the spherical cavities (--cavity-radius) */
  double query_radius;   /* initial closest-point radius; nothing at or beyond it is
                            found (wih_twos.cpp:348 uses 4.0); <= 0 means unbounded */
  int32_t green;         /* TWOS_SOURCE_*: how each ball's source integral is
                            taken (centre, Green point, or exact) */
  int32_t n_source;
  int32_t n_adjoint;
  int32_t skip_cavity_sites; /* 1: sites inside a cavity get all-zero rows
                                (adjoint.cpp:123-126) */
  uint32_t site_offset;      /* added to the site index in the sample key */
  uint32_t n_boundary;       /* terms of the primal's Dirichlet data g on the
                                mesh (0: u = 0 there, as the reference) */
  twos_source_term source[TWOS_MAX_TERMS];
  twos_source_term adjoint[TWOS_MAX_TERMS];
  /* Dirichlet data of u on the mesh surface, added to a walk's u at its exit
   * point (the nearest surface point when the walk stops within epsilon of
   * the mesh; cavities keep u = 0).  No reference counterpart: the
   * reference's walks carry zero terminal data.  The adjoint keeps zero
   * data. */
  twos_source_term boundary[TWOS_MAX_TERMS];
} twos_request;

/* Per-site result (SiteResult wih_twos.cpp:666-672 and PairValue
 * adjoint.cpp:16).  COMPLIANCE fills u = mean, score, score_se (jackknife),
 * p = u and same_index = sum u^2 / N.  PAIRED/HOT fill u, p (means), score,
 * score_se (jackknife of the cross statistic), same_index = sum u p / N. */
typedef struct twos_site_result {
  double u;
  double p;
  double score;
  double score_se;
  double same_index;
  uint64_t steps;
  uint64_t caps;
} twos_site_result; /* 56 bytes */

typedef struct twos_summary {
  double kernel_seconds;   /* device time of the walk + finalize kernels */
  double walk_seconds;     /* device time of the walk kernel alone */
  double total_seconds;    /* host wall time of the call */
  uint64_t paths;          /* walks run */
  uint64_t steps;          /* sum of steps */
  uint64_t caps;           /* walks that hit max_steps */
  uint64_t queries;        /* closest-point queries = steps + paths (wih_twos.cpp:1779) */
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint32_t launches;       /* kernels launched by the call */
  uint32_t error_flags;    /* TWOS_DEVERR_* bits raised on the device */
  uint64_t node_tests;     /* BVH node fetches (two child bounds each) */
  uint64_t plane_tests;    /* triangle plane-slab tests */
  uint64_t triangle_tests; /* full closest-point-on-triangle tests */
  uint64_t grid_steps;     /* steps whose radius came from the distance-bound
                              grid instead of a closest-point query (mixed form) */
} twos_summary;

/* Device-side error bits (set by kernels, never by a trap). */
enum {
  TWOS_DEVERR_QUERY = 1u,     /* no surface point within query_radius / non-finite */
  TWOS_DEVERR_STACK = 2u,     /* traversal stack bound exceeded */
  TWOS_DEVERR_ITER = 4u,      /* traversal iteration bound exceeded */
  TWOS_DEVERR_CONFIG = 8u,
  TWOS_DEVERR_SOURCE = 16u    /* an exact ball integral came out negative beyond
                                 round-off (study.cpp:74) */
};

typedef struct twos_mesh twos_mesh;

typedef struct twos_mesh_info {
  uint64_t vertices;
  uint64_t faces;
  uint64_t bvh_nodes;
  uint32_t bvh_depth;
  uint32_t device;
  double bounds_min[3];
  double bounds_max[3];
  double center[3];
  double mixed_delta;         /* FP32 distance error bound used by TWOS_PREC_MIXED */
  double build_seconds;       /* host BVH build + upload + distance grid */
  uint64_t device_bytes;      /* BVH + triangle + grid bytes resident on the device */
  uint32_t grid_dims[3];      /* distance-bound grid vertices per axis (0: no grid) */
  uint32_t grid_pad;
  double grid_spacing;        /* its spacing h */
} twos_mesh_info;

/* Library version and the message of the last failed call on this thread. */
int twos_abi_version(void);
const char *twos_last_error(void);

/* Build a session from an in-memory triangle mesh: host BVH build, upload of
 * the FP32 and FP64 layouts to `device`, and the distance-bound grid of the
 * mixed form: a uniform grid over the padded bounding box (about 1,024
 * vertices per triangle, at most 2^28; environment TWOS_GRID_VERTICES sets
 * it, up to 2^30; 0 builds none) holding at each vertex v a lower bound of
 * the distance from v to the surface (the FP32 distance minus twice the
 * mixed form's error bound, rounded down to 1/128 of the spacing h, 16
 * bits), stored as one 16-byte record per cell with the cell's entry node
 * (about 16 bytes per vertex: 4 GB at 2^28 vertices, built in a few
 * seconds).  The distance function is 1-Lipschitz, so D(v) - |x - v| bounds
 * the distance at any x from below: a mixed-form step may take that as its
 * ball radius -- the ball still lies in the domain, so the walk stays an
 * unbiased walk-on-spheres -- and skip the closest-point query.  Replaces
 * EmbreeMesh's constructor (wih_twos.cpp:298-325; rtcCommitScene is the BVH
 * build). */
int twos_mesh_open(const double *vertices, uint64_t n_vertices, const uint32_t *faces,
                   uint64_t n_faces, int device, twos_mesh **out);

/* Same from an ASCII PLY file with the reference's accept/reject rules and
 * messages (EmbreeMesh::load_ascii_ply, wih_twos.cpp:437-493). */
int twos_mesh_open_ply(const char *path, int device, twos_mesh **out);

void twos_mesh_close(twos_mesh *mesh);

int twos_mesh_get_info(const twos_mesh *mesh, twos_mesh_info *info);

/* Issue the session's work on `stream` (a cudaStream_t of the session's
 * device) instead of its own stream; NULL restores the session's stream.
 * Lets a caller time the kernels with events on its own stream.  No
 * reference counterpart (the reference has no device work). */
int twos_mesh_set_stream(twos_mesh *mesh, void *stream);

/* Launch tuning of a session's walk kernel (chosen by the autotuner of
 * twos_b200/autotune.py; no reference counterpart).
 *   block:          threads per block, 128, 256 or 512
 *   refill:         a warp refills from the work queue once this many lanes
 *                   are idle (1..32)
 *   step_threshold: a warp takes its batched walk step once this many lanes
 *                   have finished their closest-point query (1..32)
 *   blocks_per_sm:  resident blocks per SM, 0 = as many as fit
 *   grid_threshold: see below */
typedef struct twos_tuning {
  int32_t block;
  int32_t refill;
  int32_t step_threshold;
  int32_t blocks_per_sm;
  float grid_threshold;  /* mixed form: a step takes its radius from the
                            distance-bound grid when the bound is at least
                            this many grid spacings (>= 0.1); 0 = every step
                            queries the BVH.  Default 0.1. */
  int32_t units;         /* traversal units (node visits or triangle tests) a
                            lane runs back to back before its warp returns to
                            the refill and step ballots (1..64).  Default 8. */
  int32_t entry;         /* mixed form: 1 lets a closest-point query whose
                            initial bound is below one entry cell start at
                            the entry-node table's node instead of the root
                            (same result, fewer node visits); 0 = root. */
  int32_t grid_fp64;     /* 1: the FP64 compliance form (centre source) also
                            takes the distance grid's steps and entry nodes,
                            for comparing precision alone; 0 (default): the
                            plain FP64 form, the reference's algorithm. */
  int32_t bvh_width;     /* mixed form: 2 traverses the binary BVH, 4 the same
                            BVH collapsed to four-wide nodes (compliance,
                            paired and hot modes with the centre or Green
                            source; the others stay binary).  The same
                            minima up to FP32 rounding ties between a node
                            bound and a triangle distance.  Default 2. */
  int32_t lane_walks;    /* walks a lane claims from the work queue at once
                            and runs one after another (1..64): mixed form,
                            centre-point source, compliance / paired / hot
                            modes on the binary BVH (not with bvh_width 4);
                            the other forms claim one.  Every walk keeps its
                            own counter stream, so the rows do not change.
                            Default 1. */
  int32_t wavefront;     /* mixed form, centre-point source, compliance /
                            paired / hot modes: 0 runs the persistent walk
                            kernel; N > 0 (a multiple of 256, at most 2^26)
                            runs the wavefront form with N walks in flight --
                            a step kernel over all of them, then a query
                            kernel over those whose next radius needs a BVH
                            query, once per step.  Same rows.  Default 0. */
} twos_tuning;

int twos_mesh_set_tuning(twos_mesh *mesh, const twos_tuning *tuning);
int twos_mesh_get_tuning(const twos_mesh *mesh, twos_tuning *tuning);

/* Batched unsigned distance and closest point to the mesh surface
 * (EmbreeMesh::closest_point + point_query_callback, wih_twos.cpp:339-359,
 * 416-430).  `closest` may be NULL.  Host buffers. */
int twos_closest_point(twos_mesh *mesh, int precision, const double *points, uint64_t n,
                       double query_radius, double *distance, double *closest);

/* The mixed form's distance-grid lower bound at each point (the radius a
 * grid step would take before the threshold test: the largest D(v) - |x - v|
 * over the corners v of x's grid cell), NaN outside the grid or when the
 * session has none.
 * Never above the distance to the surface.  Host buffers.  No reference
 * counterpart. */
int twos_mesh_distance_bound(twos_mesh *mesh, const double *points, uint64_t n, double *bound);

/* Per-site TWoS estimates for n_sites sites (the OpenMP site loop of
 * wih_twos.cpp:1825-1841 with evaluate_site 674-717, or the paired loop of
 * adjoint.cpp:121-127 with paired_site 18-42).  Host buffers; `summary` may
 * be NULL.  Returns TWOS_ERR_RUNTIME when any walk hit max_steps (the rows
 * are still written, with caps > 0) or a device error bit was raised. */
int twos_estimate(twos_mesh *mesh, const twos_request *request, const double *sites,
                  uint32_t n_sites, const double *cavities, uint32_t n_cavities,
                  twos_site_result *out, twos_summary *summary);

/* As twos_estimate with device-resident sites (d_sites, 3 doubles each) and
 * results (d_out); cavities stay host memory.  Work is ordered on the
 * session's stream and the call returns after it completes. */
int twos_estimate_device(twos_mesh *mesh, const twos_request *request, const double *d_sites,
                         uint32_t n_sites, const double *cavities, uint32_t n_cavities,
                         twos_site_result *d_out, twos_summary *summary);

/* twos_estimate_device for callers that cannot allocate device memory.  No
 * counterpart in the reference (whose backend has no device code).
 *
 * Some callers must not call cudaMalloc: code running while a framework owns
 * the device memory pool (a raw cudaMalloc bypasses its allocator and
 * fragments memory it manages), and services with a fixed device-memory
 * budget that must not grow per request.  This entry point allocates nothing:
 * every per-call device buffer (launch tables, cavities, first-query
 * distances, queue counter, totals and the per-walk samples) is carved out of
 * one static device array of TWOS_NOALLOC_SCRATCH_BYTES (16 MiB) that every
 * GPU loading the library holds until the process exits.  The mesh session
 * (opened earlier with twos_mesh_open*), the sites (d_sites, 3 doubles each)
 * and the result rows (d_out) belong to the caller.
 *
 * Limit: the scratch holds the per-walk samples of one call (a value per walk
 * for u, another for p in paired mode, 4 bytes of step count), so
 * n_sites * walks may be at most about 2.0 M in mixed compliance mode
 * (8 bytes per walk), 1.39 M in mixed paired or FP64 compliance mode (12) and
 * 0.83 M in FP64 paired mode (20), less a few KB of tables and 8 bytes per
 * site; larger requests are rejected with TWOS_ERR_USAGE and a message giving
 * the bytes needed.  The first call on a device looks up the array's device
 * address (once per device); make that first call before any stream capture.
 * All calls share the one array and it keeps the previous call's contents
 * (the call clears what must start at zero): calls that overlap on the GPU,
 * from different threads, streams or sessions, race on it and must be
 * serialised by the caller.  Work runs on the session's stream and the call
 * returns after that stream has completed it.  Rows equal
 * twos_estimate_device's, and errors and the summary are reported the same
 * way (h2d_bytes and d2h_bytes are 0). */
#define TWOS_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int twos_estimate_noalloc(twos_mesh *mesh, const twos_request *request, const double *d_sites,
                          uint32_t n_sites, const double *cavities, uint32_t n_cavities,
                          twos_site_result *d_out, twos_summary *summary);

/* Several meshes in persistent launches over one work queue: job j runs
 * request[j] over sites[j] (n_sites[j] sites, 3 doubles each) on meshes[j]
 * with cavities[j] (may be NULL when n_cavities[j] == 0) and writes out[j].
 * All meshes must be sessions on the same device; all requests must share
 * mode, precision and the Green-point flag.  Walks of the jobs of a launch
 * share one device work queue, so a batch of uneven meshes, site counts and
 * walk counts keeps every SM busy; the queue takes the jobs largest
 * geometry, smallest, second largest, ... so two geometries that each fill
 * much of the L2 are not in flight at once, and is cut into as few launches
 * as keep each launch's job and geometry descriptors in shared memory.
 * Results equal those of one twos_estimate call per job with the same
 * requests.  The work runs on meshes[0]'s stream; `summary` totals the batch.
 * Replaces a driver loop of one process call per geometry (e.g.
 * benchmarks/bunny_budget/run_study.py:41-62). */
int twos_estimate_batch(twos_mesh *const *meshes, const twos_request *requests, uint32_t n_jobs,
                        const double *const *sites, const uint32_t *n_sites, const double *const *cavities,
                        const uint32_t *n_cavities, twos_site_result *const *out, twos_summary *summary);

/* Design loop (select_twos, benchmarks/stanford_bunny/run_bunny_benchmark.py:
 * 302-337, and run_design 450-491): each iteration scouts every feasible
 * candidate with `scout`, rescored the top `shortlist` by scout score with
 * `validate` (its own stream, so fresh samples), takes the argmax of
 * lower = score - z * score_se, and inserts a ball cavity of radius
 * cavity_radius at it when lower > accept_threshold.  A candidate is feasible
 * when its surface distance is >= cavity_radius + outer_clearance and it is
 * at least 2 * cavity_radius + pair_gap from every cavity (feasible_mask,
 * run_bunny_benchmark.py:290-299).  Every decision is taken on the device;
 * with use_graph one iteration is captured as a CUDA graph and replayed.
 * Iteration i keys its scout walks by (repeat i, candidate index) and its
 * validation walks by (repeat i, shortlist slot); the validation stage runs
 * without the mixed form's distance grid, so both precisions validate a
 * candidate with the same samples.  history[i].slot and .n_cavities record
 * what a replay of that validation needs. */
typedef struct twos_design_params {
  uint32_t iterations;
  uint32_t shortlist;       /* <= 1024 */
  double cavity_radius;
  double z;                 /* confidence multiplier (1.96) */
  double accept_threshold;
  double outer_clearance;
  double pair_gap;
  int32_t use_graph;
  int32_t reserved;
} twos_design_params;

typedef struct twos_design_step {
  uint32_t chosen;          /* candidate index, UINT32_MAX when none was feasible */
  uint32_t accepted;
  double scout_score;
  double score;             /* validation estimate */
  double score_se;
  double lower;             /* score - z * score_se */
  uint32_t slot;            /* the choice's shortlist slot: its validation walks' site index */
  uint32_t n_cavities;      /* cavities present while it was validated */
} twos_design_step;

/* history[iterations]; cavities_out holds up to n_cavities + iterations
 * centres (initial ones first); *n_cavities_out is set.  Host buffers. */
int twos_design_loop(twos_mesh *mesh, const twos_request *scout, const twos_request *validate,
                     const double *candidates, uint32_t n_candidates, const double *cavities,
                     uint32_t n_cavities, const twos_design_params *params, twos_design_step *history,
                     double *cavities_out, uint32_t *n_cavities_out, twos_summary *summary);

/* Differential WoS (evaluate_differential_site, wih_twos.cpp:839-928;
 * --mode diffwos, run_differential_wos 1604-1709; study.cpp --diff 1,
 * 304-316): at each probe site, the derivatives of u with respect to every
 * cavity's centre and radius.  Each of request->walks outer walks runs to the
 * boundary; one that ends on cavity i is offset inward by diff_offset along
 * the normal, checked for seam/segment safety and membership (ray parity,
 * with the enclosure fallback when enclosure_fallback != 0), and a nested
 * walk from the offset point gives the samples n u/l (centre) and -u/l
 * (radius).  out is [n_sites][n_cavities]; stats ([n_sites]) may be NULL.
 * The request's source terms and green flag drive the nested walks.
 * Returns TWOS_ERR_RUNTIME when a walk hit max_steps or an offset was unsafe
 * (rows and stats are still written), as the study backend does
 * (study.cpp:309-310).  In `summary`, queries counts closest-point queries as
 * the study backend's note_query(0) does, node_tests the parity rays
 * (note_query(1)), plane_tests the enclosure fallbacks taken and
 * triangle_tests the unsafe offsets. */
typedef struct twos_diff_result {
  double dc[3];
  double dc_se[3];
  double dR;
  double dR_se;
} twos_diff_result; /* 64 bytes */

typedef struct twos_diff_stats {
  uint64_t outer_steps;
  uint64_t nested_steps;
  uint64_t cavity_terminations;
  uint64_t near_seam;
  uint64_t segment_unsafe;
  uint64_t unsafe_offset;
  uint64_t limits;
} twos_diff_stats;

int twos_diffwos(twos_mesh *mesh, const twos_request *request, double diff_offset, int enclosure_fallback,
                 const double *sites, uint32_t n_sites, const double *cavities, uint32_t n_cavities,
                 twos_diff_result *out, twos_diff_stats *stats, twos_summary *summary);

/* Gradient estimates and the cross-index gradient product (the Neumann-
 * cavity topological derivative of the plain method on the unit sphere; no
 * reference counterpart: the reference implements only Dirichlet cavities,
 * paper/sections/03_problem.tex:153).  A paired request (source = the
 * primal's f, adjoint = the adjoint's source q, boundary = the primal's
 * Dirichlet data; green CENTER or GREEN) runs one walk set; each walk i
 * gives gradient samples at the site from its first ball B_R(x):
 *   grad U_i = (3/R) U'_i w + R (1 - t^3) f(x + t R w') w'
 * with w the first step direction, U'_i the walk's u after its first step
 * (the sphere term of the mean-value gradient formula), and t ~ U(0,1), w'
 * uniform an extra draw for the ball's source term (the gradient of the
 * ball's Green function, sampled with a bounded weight); likewise grad P_i.
 * cross = sum_{i != j} grad U_i . grad P_j / (N (N-1)) estimates
 * grad u . grad p without the i = j bias, with its leave-one-out jackknife
 * SE.  For a small Neumann sphere at x the topological derivative of
 * J = int q u is D_T = (3/2) grad u . grad p - q(x) u(x) - f(x) p(x) (the
 * dipole of a Neumann sphere in a uniform field, 3D polarization 3/2, plus
 * the removed volume); u_se and p_se with cross_se bound the standard error
 * of an assembled D_T. */
typedef struct twos_gradient_result {
  double u, p;
  double grad_u[3], grad_p[3];
  double cross, cross_se;
  uint64_t steps, caps;
  double u_se, p_se; /* standard errors of the means u and p */
} twos_gradient_result; /* 112 bytes */

int twos_estimate_gradient(twos_mesh *mesh, const twos_request *request, const double *sites, uint32_t n_sites,
                           const double *cavities, uint32_t n_cavities, twos_gradient_result *out,
                           twos_summary *summary);

/* Array-RQMC, matched Monte Carlo and neighbour reuse (benchmarks/
 * critical_baselines/sampling.py:49-110, the reference's 2D study, here in
 * 3D on the mesh).  Each site's request->walks walks (a power of two,
 * 32..1024) advance in lockstep, one CUDA block per (site, batch).  ARRAY: at
 * every step the active walks are ordered by the 3D Hilbert index of their
 * position (10 bits per axis in the mesh's bounding box; finished walks last)
 * and the walk of rank i takes the 3D Korobov lattice point
 * (i/n, g i/n, g^2 i/n) mod 1 shifted by one random (U1, U2) per (site,
 * batch, step) (Ho and Owen's Array-RQMC; the first coordinate is the
 * ordering, the other two give the step direction; g maximises the lattice's
 * minimum distance).  MC: independent uniforms.  NEIGHBOUR: the MC walks,
 * then each site's batch mean pools the walks of every site y whose first
 * ball B(y, r_y) contains it, each walk reweighted by the Poisson kernel
 * ratio r_y (r_y^2 - |x-y|^2) / |x - z|^3 (z the walk's first step point)
 * and each site y weighted by (1-a)^4 / (1+a)^2, a = |x-y| / r_y (reused_means,
 * sampling.py:76-88, in 3D; harmonic problems only: no request->source).
 * SOBOL: Sobol-over-steps RQMC (sampling.py:49-60 in 3D): walk i of a
 * (site, batch) holds point i of a Sobol' sequence scrambled once per
 * (site, batch) (a random lower-triangular digit matrix and a digital shift
 * per coordinate) and takes coordinates 2k and 2k + 1 at step k, for steps
 * k < 256; later steps draw the MC stream.  The direction numbers come from
 * the primitive polynomials over GF(2) in order, with seeded odd initial
 * values (not the reference's scipy table).
 * A walk's payoff is request->source at each ball centre times r^2/6 plus
 * u_boundary (primal) or p_boundary (adjoint) at its exit point on the mesh.
 * The cross-fitting unit is a whole batch (an independent randomization):
 * batch_u/batch_p [batches][n_sites] are the batch means and
 * td[site] = -(sum a sum b - sum ab) / (R (R - 1)) over the R batches
 * (crossfit, sampling.py:90-92).  Capped walks are an error (sampling.py:
 * 72-73).  No reference counterpart in the compiled backend. */
enum { TWOS_RQMC_MC = 0, TWOS_RQMC_ARRAY = 1, TWOS_RQMC_NEIGHBOUR = 2, TWOS_RQMC_SOBOL = 3 };

typedef struct twos_rqmc_params {
  int32_t method;    /* TWOS_RQMC_* */
  uint32_t batches;  /* >= 2 */
  uint32_t n_u_boundary, n_p_boundary;
  twos_source_term u_boundary[TWOS_MAX_TERMS];
  twos_source_term p_boundary[TWOS_MAX_TERMS];
  /* Optional per-walk record (host buffers, each may be NULL):
   * walk_first [batches][n_sites][walks][3] the first step's point,
   * walk_u / walk_p [batches][n_sites][walks] each walk's payoffs, and
   * site_radius [n_sites] the first ball's radius at each site (the record
   * reused_means takes, sampling.py:49-88). */
  double *walk_first, *walk_u, *walk_p, *site_radius;
} twos_rqmc_params;

int twos_rqmc(twos_mesh *mesh, const twos_request *request, const twos_rqmc_params *params, const double *sites,
              uint32_t n_sites, double *batch_u, double *batch_p, double *td, twos_summary *summary);

/* Test hook for the mixed form's distance grid: runs the mixed compliance
 * estimate of `request` (centre-point source, no cavities) over `sites` in a
 * walk kernel that records every grid step -- the walk's position (original
 * coordinates, the FP32 position exactly) and the bound it used as the
 * ball's radius before the delta shrink -- keeping the first `capacity`
 * records in points [capacity][3] and bounds [capacity]; *count is the total
 * number of grid steps.  Host buffers.  No reference counterpart. */
int twos_trace_grid_steps(twos_mesh *mesh, const twos_request *request, const double *sites, uint32_t n_sites,
                          uint64_t capacity, double *points, double *bounds, uint64_t *count);

/* Measured L2 read bandwidth of `device` in GB/s: the best of five timed
 * launches that each stream a zeroed `bytes` buffer (an L2-resident size,
 * e.g. 64 MiB) `passes` times with 32-byte vector loads from every SM, the
 * walk kernel's load form.  The roofline denominator for kernels whose
 * working set is L2-resident.  No reference counterpart (a measurement). */
int twos_l2_read_gbs(int device, uint64_t bytes, uint32_t passes, double *gbs);

/* The Sobol' direction numbers of twos_rqmc's SOBOL method, host only:
 * out [dims][bits], out[d * bits + b] = m_{d,b+1} 2^(31-b) (most significant
 * digit first).  Dimension 0 is van der Corput's; dimension d >= 1 takes the
 * d-th primitive polynomial over GF(2) by degree, then coefficient bits,
 * with odd initial values m_k < 2^k from SplitMix64 and Sobol's recurrence
 * (the reference's study takes scipy's Joe-Kuo table instead,
 * critical_baselines/sampling.py:53).  dims <= 65536, bits 1..32. */
int twos_sobol_directions(uint32_t dims, uint32_t bits, uint32_t *out);

/* The estimator's per-site reduction on caller-supplied per-walk samples:
 * u and p (p may be NULL outside paired mode) [n_sites][walks] as doubles,
 * steps (may be NULL) with bit 31 set on a cap, out one row per site -- all
 * host buffers.  The rows are what twos_estimate writes for walks with these
 * payoffs: compliance the U-statistic (S^2 - S2)/(N(N-1)) with its
 * leave-one-out jackknife SE (evaluate_site, wih_twos.cpp:686-715, and
 * crossfit_square, stanford_bunny/run_bunny_benchmark.py:257-269); paired
 * (S_u S_p - S_up)/(N(N-1)), i.e. minus crossfit_product of
 * experiments/run_controlled_experiments.py:79-87, with the same jackknife;
 * hot the mean.  With TWOS_PREC_MIXED the samples are rounded to float
 * first, as the mixed walk kernel stores them.  `mesh` supplies the device
 * and stream.  Used to check the device reduction on identical inputs. */
int twos_finalize_samples(twos_mesh *mesh, int precision, int mode, const double *u, const double *p,
                          const uint32_t *steps, uint32_t n_sites, uint32_t walks, twos_site_result *out);

/* Per-walk samples (the `values` vector of wih_twos.cpp:678-690): u and p
 * (p may be NULL) as doubles, steps per walk with bit 31 set on a cap, laid
 * out [site][walk].  Host buffers.  Used by parity tests. */
int twos_walk_samples(twos_mesh *mesh, const twos_request *request, const double *sites,
                      uint32_t n_sites, const double *cavities, uint32_t n_cavities, double *u,
                      double *p, uint32_t *steps);

/* Ray-parity point membership (EmbreeMesh::inside, wih_twos.cpp:361-394):
 * inside[i] = 1 when a ray in the reference's fixed oblique direction crosses
 * the surface an odd number of times.  Host buffers. */
int twos_inside(twos_mesh *mesh, const double *points, uint64_t n, uint8_t *inside);

/* The EXACT source's ball integral on the device (exact_bump_green,
 * study.cpp:64-77, as read by wih_analytic_integral_audit,
 * analytic_integral_audit.cpp): for case i, cases[4i..4i+3] = (d, r, R, A)
 * with the bump centred at distance d from the ball centre, out[i] =
 * integral over B_r of G_r(0, z) A (1 - |z-c|^2/R^2)_+^2 dz.  Host buffers;
 * runs on `device`.  A negative integral beyond round-off returns
 * TWOS_ERR_RUNTIME with the values written. */
int twos_ball_green_integral(const double *cases, uint32_t n, double *out, int device);

/* Certified fresh-sample validation (--mode validate: run_minimum_benefit,
 * cert_walk, CertDistanceTree and cert_source_lower of
 * benchmarks/compiled_bunny/src/minimum_benefit.hpp:13-188).  Each of
 * request->walks walks per site takes as its distance the distance to the
 * union of the triangles' bounding boxes and to the cavities, every positive
 * operation rounded one ulp down after rounding to nearest; steps of radius
 * min(radius_cap, 0.95 d); a rounded-down lower bound of the source at the
 * ball centre (green 0) or at a Beta(2,2) Green point (green 1) times
 * r^2/6; the value clipped at value_cap; a walk whose sampled point might
 * leave its ball stops and is counted as a containment failure.  FP64 in
 * both precision forms (request->precision is ignored).
 *
 * Sources: an optional leading CONST term, then LINEAR (amp >= 0) and GAUSS
 * (amp >= 0) terms; anything else is TWOS_ERR_USAGE.  Every site must be
 * inside the mesh (ray parity) and outside every cavity, else
 * TWOS_ERR_RUNTIME.  samples is [n_sites][walks]; stages is
 * [n_sites][TWOS_VALIDATE_MAX_STAGES] with *n_stages per site: the prefixes
 * n in {1024, 4096, 16384, 65536} below walks, then walks, as the
 * reference's stage JSON.  Containment failures return TWOS_ERR_RUNTIME
 * with everything written ("validation record must be rejected"). */
#define TWOS_VALIDATE_MAX_STAGES 5

typedef struct twos_validate_params {
  double radius_cap; /* --validation-radius-cap */
  double value_cap;  /* --validation-value-cap */
} twos_validate_params;

typedef struct twos_cert_sample {
  double value;
  uint32_t steps;
  uint8_t capped;    /* hit max_steps */
  uint8_t clipped;   /* reached value_cap */
  uint8_t contained; /* 0: containment failure (the sample must not be used) */
  uint8_t pad;
} twos_cert_sample; /* 16 bytes */

typedef struct twos_validate_stage {
  uint32_t site;
  uint32_t n;
  double mean;                   /* long-double sum of the first n values / n */
  double mean_steps;
  uint64_t clipped;
  uint64_t path_caps;
  double center_clearance_lower; /* certified domain distance at the site */
  double center_distance;        /* exact FP64 domain distance at the site */
} twos_validate_stage; /* 56 bytes */

int twos_validate(twos_mesh *mesh, const twos_request *request, const twos_validate_params *params,
                  const double *sites, uint32_t n_sites, const double *cavities, uint32_t n_cavities,
                  twos_cert_sample *samples, twos_validate_stage *stages, uint32_t *n_stages,
                  twos_summary *summary);

/* Indices of the k largest keys, highest first, ties to the lower index
 * (np.argpartition(...)[-k:] of run_bunny_benchmark.py:324 with a
 * deterministic order).  Device buffers, k <= 1024. */
int twos_topk_device(twos_mesh *mesh, const double *d_keys, uint32_t n, uint32_t k,
                     uint32_t *d_index);

#ifdef __cplusplus
}
#endif

#endif /* TWOS_H */

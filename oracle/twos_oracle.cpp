// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the TWoS estimator.
//
// This file restates, on the host and in plain FP64, the algorithm of the
// reference backend (hertjo/walking-into-holes,
// benchmarks/compiled_bunny/src/wih_twos.cpp and
// benchmarks/distinct_adjoint/adjoint.cpp).  It is the checker that the CUDA
// product is compared with; nothing in the product links, loads or calls it.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
//
// Two random streams are provided:
//   * RNG_REFERENCE -- the reference's own per-walk std::mt19937_64 stream,
//     keyed exactly as wih_twos.cpp:681-686 (compliance) and adjoint.cpp:22
//     (paired).  Because the same libstdc++ <random> and libm are used, the
//     integer step counts reproduce the reference's tracked output files.
//   * RNG_COUNTER -- the counter-based Philox4x32-10 stream that the GPU
//     kernels use (a pure function of seed, stream, repeat, site, walk, step,
//     draw), so GPU and oracle walk the same paths from the same samples.
//
// Closest-point queries use an exact FP64 minimum over triangles through a
// binary SAH BVH (<= 4 triangles per leaf, nearest-child-first traversal,
// pruning a box when its lower-bound distance is >= the current best).  The
// same traversal is instrumented to count AABB and triangle tests; those
// counts define the algorithmic bytes per query used for the roofline.
//
// Build: g++ -O2 -fopenmp -ffp-contract=off -shared -fPIC (no -march flags, so
// no FMA contraction, matching the reference's default x86-64 Release build).

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Vec3 {
  double x = 0.0, y = 0.0, z = 0.0;
};
inline Vec3 operator+(const Vec3 &a, const Vec3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(const Vec3 &a, const Vec3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator*(const Vec3 &a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(const Vec3 &a, const Vec3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(const Vec3 &a) { return std::sqrt(dot(a, a)); }
inline double coord(const Vec3 &v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Ericson's closest point on a triangle (Real-Time Collision Detection,
// section 5.1.5), the case analysis wih_twos.cpp:247-289 uses.
Vec3 closest_point_triangle(const Vec3 &p, const Vec3 &a, const Vec3 &b, const Vec3 &c) {
  const Vec3 ab = b - a, ac = c - a, ap = p - a;
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const Vec3 bp = p - b;
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return b;
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    return a + ab * v;
  }
  const Vec3 cp = p - c;
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    return a + ac * w;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
    const Vec3 bc = c - b;
    const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return b + bc * w;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  return a + ab * v + ac * w;
}

struct Box {
  Vec3 lo{std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
          std::numeric_limits<double>::infinity()};
  Vec3 hi{-std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
          -std::numeric_limits<double>::infinity()};
  void grow(const Vec3 &p) {
    lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
    hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
  }
  void grow(const Box &b) {
    grow(b.lo);
    grow(b.hi);
  }
  double area() const {
    const double dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    if (!(dx >= 0.0)) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
  }
  // Squared distance from p to the box (0 inside).
  double dist2(const Vec3 &p) const {
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double g = std::max({0.0, coord(lo, a) - coord(p, a), coord(p, a) - coord(hi, a)});
      s += g * g;
    }
    return s;
  }
};

// Binary SAH BVH with at most 4 triangles per leaf (the canonical traversal).
struct Bvh {
  struct Node {
    Box box;
    int left = -1, right = -1;  // internal: children; leaf: left = -1
    int begin = 0, count = 0;   // leaf triangle range into order
  };
  std::vector<Node> nodes;
  std::vector<uint32_t> order;
  int depth = 0;
};

struct Mesh {
  std::vector<Vec3> v;
  std::vector<std::array<uint32_t, 3>> f;
  Bvh bvh;
};

constexpr int kLeafMax = 4;
constexpr int kBins = 32;

int build_node(Mesh &m, std::vector<Box> &tb, std::vector<Vec3> &cent, int begin, int end, int depth) {
  Bvh &b = m.bvh;
  const int index = static_cast<int>(b.nodes.size());
  b.nodes.emplace_back();
  b.depth = std::max(b.depth, depth);
  Box box, cbox;
  for (int i = begin; i < end; ++i) {
    box.grow(tb[b.order[i]]);
    cbox.grow(cent[b.order[i]]);
  }
  b.nodes[index].box = box;
  const int n = end - begin;
  if (n <= kLeafMax) {
    b.nodes[index].begin = begin;
    b.nodes[index].count = n;
    return index;
  }
  // Binned SAH over centroid bounds on every axis.
  double best_cost = std::numeric_limits<double>::infinity();
  int best_axis = -1, best_split = -1;
  for (int axis = 0; axis < 3; ++axis) {
    const double lo = coord(cbox.lo, axis), hi = coord(cbox.hi, axis);
    if (!(hi > lo)) continue;
    std::array<Box, kBins> bins;
    std::array<int, kBins> counts{};
    const double scale = kBins / (hi - lo);
    for (int i = begin; i < end; ++i) {
      int k = static_cast<int>((coord(cent[b.order[i]], axis) - lo) * scale);
      k = std::min(std::max(k, 0), kBins - 1);
      bins[k].grow(tb[b.order[i]]);
      ++counts[k];
    }
    std::array<double, kBins> right_area{};
    std::array<int, kBins> right_count{};
    Box acc;
    int cnt = 0;
    for (int k = kBins - 1; k > 0; --k) {
      acc.grow(bins[k]);
      cnt += counts[k];
      right_area[k] = acc.area();
      right_count[k] = cnt;
    }
    Box lacc;
    int lcnt = 0;
    for (int k = 0; k < kBins - 1; ++k) {
      lacc.grow(bins[k]);
      lcnt += counts[k];
      if (lcnt == 0 || right_count[k + 1] == 0) continue;
      const double cost = lacc.area() * lcnt + right_area[k + 1] * right_count[k + 1];
      if (cost < best_cost) {
        best_cost = cost;
        best_axis = axis;
        best_split = k;
      }
    }
  }
  int mid;
  if (best_axis < 0) {
    mid = begin + n / 2;  // all centroids coincide: split by index
  } else {
    const double lo = coord(cbox.lo, best_axis), hi = coord(cbox.hi, best_axis);
    const double scale = kBins / (hi - lo);
    auto it = std::partition(b.order.begin() + begin, b.order.begin() + end, [&](uint32_t t) {
      int k = static_cast<int>((coord(cent[t], best_axis) - lo) * scale);
      k = std::min(std::max(k, 0), kBins - 1);
      return k <= best_split;
    });
    mid = static_cast<int>(it - b.order.begin());
    if (mid == begin || mid == end) mid = begin + n / 2;
  }
  const int l = build_node(m, tb, cent, begin, mid, depth + 1);
  const int r = build_node(m, tb, cent, mid, end, depth + 1);
  b.nodes[index].left = l;
  b.nodes[index].right = r;
  return index;
}

void build_bvh(Mesh &m) {
  const size_t nf = m.f.size();
  std::vector<Box> tb(nf);
  std::vector<Vec3> cent(nf);
  for (size_t i = 0; i < nf; ++i) {
    Box b;
    b.grow(m.v[m.f[i][0]]);
    b.grow(m.v[m.f[i][1]]);
    b.grow(m.v[m.f[i][2]]);
    tb[i] = b;
    cent[i] = (b.lo + b.hi) * 0.5;
  }
  m.bvh.order.resize(nf);
  std::iota(m.bvh.order.begin(), m.bvh.order.end(), 0u);
  m.bvh.nodes.reserve(2 * nf + 1);
  build_node(m, tb, cent, 0, static_cast<int>(nf), 0);
}

struct QueryStats {
  uint64_t aabb = 0, tri = 0;
};

struct Closest {
  double distance = std::numeric_limits<double>::infinity();
  Vec3 point;
  uint32_t tri = 0xffffffffu;
};

// Exact FP64 closest point; counts box and triangle tests of the canonical
// traversal.  `radius` plays the role of the reference's initial query radius
// (wih_twos.cpp:348, 4.0F): nothing at or beyond it is reported.
Closest closest_point(const Mesh &m, const Vec3 &p, double radius, QueryStats *stats) {
  Closest out;
  double best2 = radius * radius;
  const Bvh &b = m.bvh;
  struct Entry {
    int node;
    double d2;
  };
  Entry stack[128];
  int sp = 0;
  // The root's box is tested like every other box.
  if (stats) ++stats->aabb;
  const double root_d2 = b.nodes[0].box.dist2(p);
  if (root_d2 < best2) stack[sp++] = {0, root_d2};
  while (sp > 0) {
    const Entry e = stack[--sp];
    if (!(e.d2 < best2)) continue;
    const Bvh::Node &n = b.nodes[e.node];
    if (n.left < 0) {
      for (int i = 0; i < n.count; ++i) {
        const uint32_t t = b.order[n.begin + i];
        if (stats) ++stats->tri;
        const auto &f = m.f[t];
        const Vec3 q = closest_point_triangle(p, m.v[f[0]], m.v[f[1]], m.v[f[2]]);
        const Vec3 d = p - q;
        const double d2 = dot(d, d);
        if (d2 < best2) {
          best2 = d2;
          out.point = q;
          out.tri = t;
        }
      }
      continue;
    }
    const Bvh::Node &l = b.nodes[n.left], &r = b.nodes[n.right];
    if (stats) stats->aabb += 2;
    const double dl = l.box.dist2(p), dr = r.box.dist2(p);
    // Push the farther child first so the nearer one is visited next.
    if (dl <= dr) {
      if (dr < best2) stack[sp++] = {n.right, dr};
      if (dl < best2) stack[sp++] = {n.left, dl};
    } else {
      if (dl < best2) stack[sp++] = {n.left, dl};
      if (dr < best2) stack[sp++] = {n.right, dr};
    }
    if (sp > 120) throw std::runtime_error("oracle BVH stack overflow");
  }
  if (out.tri != 0xffffffffu) out.distance = norm(p - out.point);
  return out;
}

Closest closest_point_brute(const Mesh &m, const Vec3 &p) {
  Closest out;
  double best2 = std::numeric_limits<double>::infinity();
  for (uint32_t t = 0; t < m.f.size(); ++t) {
    const auto &f = m.f[t];
    const Vec3 q = closest_point_triangle(p, m.v[f[0]], m.v[f[1]], m.v[f[2]]);
    const Vec3 d = p - q;
    const double d2 = dot(d, d);
    if (d2 < best2) {
      best2 = d2;
      out.point = q;
      out.tri = t;
    }
  }
  out.distance = norm(p - out.point);
  return out;
}

// ---------------------------------------------------------------- sources
// One source term; a source is the ordered sum of its terms.
struct Term {
  int32_t kind;  // 0 const, 1 linear, 2 gauss, 3 bump, 4 box, 5 ball
  int32_t axis;
  double amp, offset, div;
  double c[3], w[3];
};
static_assert(sizeof(Term) == 80, "term layout");

double term_value(const Term &t, const Vec3 &x) {
  switch (t.kind) {
    case 0:
      return t.amp;
    case 1:
      return t.amp * (coord(x, t.axis) + t.offset);
    case 2: {
      // wih_twos.cpp:553-556: exp(-((x-c0)/w0)^2 - ((y-c1)/w1)^2 - ((z-c2)/w2)^2)
      const double a = (x.x - t.c[0]) / t.w[0], b = (x.y - t.c[1]) / t.w[1], c = (x.z - t.c[2]) / t.w[2];
      return t.amp * std::exp(-(a * a) - (b * b) - (c * c));
    }
    case 3: {
      // adjoint.cpp:11-15: (max(0, 1 - |x-c|^2/r^2))^2
      const Vec3 d{x.x - t.c[0], x.y - t.c[1], x.z - t.c[2]};
      const double s = std::max(0.0, 1.0 - dot(d, d) / (t.w[0] * t.w[0]));
      return t.amp * (s * s) / t.div;
    }
    case 4:
      return (x.x >= t.c[0] && x.x <= t.w[0] && x.y >= t.c[1] && x.y <= t.w[1] && x.z >= t.c[2] &&
              x.z <= t.w[2])
                 ? t.amp
                 : 0.0;
    case 5: {
      const Vec3 d{x.x - t.c[0], x.y - t.c[1], x.z - t.c[2]};
      return dot(d, d) <= t.w[0] * t.w[0] ? t.amp : 0.0;
    }
    case 6: {  // amp * sum_k w_k (x_k - c_k)^2
      const double a = x.x - t.c[0], b = x.y - t.c[1], c = x.z - t.c[2];
      return t.amp * (t.w[0] * (a * a) + t.w[1] * (b * b) + t.w[2] * (c * c));
    }
    default:
      return 0.0;
  }
}

double source_value(const Term *terms, int n, const Vec3 &x) {
  if (n <= 0) return 0.0;
  double s = term_value(terms[0], x);
  for (int i = 1; i < n; ++i) s = s + term_value(terms[i], x);
  return s;
}

// ---------------------------------------------------------------- exact ball integral
// exact_bump_green (benchmarks/submission_study/study.cpp:53-77, the
// WIH_ANALYTIC_SOURCE path), restated in long double as the reference
// computes it: the bump's Newton potential N at the ball centre minus its
// mean over the ball's sphere, from the primitive P(x) = int_0^x s N(s) ds.
long double ld_bump_potential(long double d, long double R, long double A) {
  if (d >= R) return A * R * R * R * (8.0L / 105) / d;
  const long double t = d / R;
  return A * R * R * (1.0L / 6 - t * t / 6 + t * t * t * t / 10 - t * t * t * t * t * t / 42);
}

long double ld_potential_primitive(long double d, long double R, long double A) {
  const long double t = std::min(d / R, 1.0L), t2 = t * t, t4 = t2 * t2;
  const long double inner = A * R * R * R * R * (t2 / 12 - t4 / 24 + t4 * t2 / 60 - t4 * t4 / 336);
  return inner + (d > R ? A * R * R * R * (8.0L / 105) * (d - R) : 0.0L);
}

double exact_bump_green(double d_, double r_, double R_, double A_, bool &negative) {
  const long double d = d_, r = r_, R = R_, A = A_;
  if (d >= r + R) return 0.0;
  const long double at_center = ld_bump_potential(d, R, A);
  long double mean;
  if (d + R <= r)
    mean = A * R * R * R * (8.0L / 105) / r;
  else if (d < 1e-12L * R)
    mean = ld_bump_potential(r, R, A);
  else
    mean = (ld_potential_primitive(d + r, R, A) - ld_potential_primitive(std::fabs(d - r), R, A)) / (2 * d * r);
  const long double value = at_center - mean;
  if (value < -1e-11L * std::max(1.0L, std::fabs(at_center))) negative = true;
  return static_cast<double>(std::max(0.0L, value));
}

// One step's exact source integral over B_r(y) (study.cpp:96-104): the
// harmonic (constant and linear) terms as r*r/6 f(y), then every bump term's
// exact integral, in term order.
double exact_source(const Term *terms, int n, const Vec3 &y, double r, double acc, bool &negative) {
  double harmonic = 0.0;
  bool any = false;
  for (int i = 0; i < n; ++i) {
    if (terms[i].kind == 0 || terms[i].kind == 1) {
      harmonic = any ? harmonic + term_value(terms[i], y) : term_value(terms[i], y);
      any = true;
    }
  }
  if (any) acc += r * r / 6 * harmonic;
  for (int i = 0; i < n; ++i) {
    const Term &t = terms[i];
    if (t.kind != 3) continue;
    const Vec3 c{t.c[0], t.c[1], t.c[2]};
    acc += exact_bump_green(norm(y - c), r, t.w[0], t.amp / t.div, negative);
  }
  return acc;
}

// ---------------------------------------------------------------- random streams
uint64_t splitmix64(uint64_t x) {
  // SplitMix64 finaliser (Steele, Lea & Flood 2014), as wih_twos.cpp:529-534 uses it.
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30U)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27U)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31U);
}

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11).
struct Philox {
  static void block(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                    uint32_t out[4]) {
    for (int r = 0; r < 10; ++r) {
      const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
      const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
      const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
      const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
      c0 = hi1 ^ c1 ^ k0;
      c1 = lo1;
      c2 = hi0 ^ c3 ^ k1;
      c3 = lo0;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
  }
};

inline double u53(uint32_t hi, uint32_t lo) {
  const uint64_t v = (static_cast<uint64_t>(hi) << 32) | lo;
  return static_cast<double>(v >> 11) * 0x1.0p-53;
}

// Counter stream of one walk: counter = (step, walk, site, repeat*8 + draw block).
struct CounterStream {
  uint32_t k0, k1, walk, site, repeat;
  // Two FP64 uniforms from block j of step s.
  void uniforms(uint32_t step, uint32_t j, double &a, double &b) const {
    uint32_t o[4];
    Philox::block(k0, k1, step, walk, site, (repeat << 3) | j, o);
    a = u53(o[0], o[1]);
    b = u53(o[2], o[3]);
  }
};

inline void counter_key(uint64_t seed, uint32_t stream, uint32_t &k0, uint32_t &k1) {
  const uint64_t k = splitmix64(seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(stream) + 1));
  k0 = static_cast<uint32_t>(k);
  k1 = static_cast<uint32_t>(k >> 32);
}

// Uniform direction on S^2 from two uniforms: z = 1 - 2a, phi = 2*pi*b.
inline Vec3 direction_from(double a, double b) {
  const double z = 1.0 - 2.0 * a;
  const double phi = 2.0 * 3.141592653589793 * b;
  const double radial = std::sqrt(std::max(0.0, 1.0 - z * z));
  return {radial * std::cos(phi), radial * std::sin(phi), z};
}

inline double median3(double a, double b, double c) {
  return std::max(std::min(a, b), std::min(std::max(a, b), c));
}

// Reference stream pieces (wih_twos.cpp:536-542, 569-575).
Vec3 random_unit_vector(std::mt19937_64 &rng) {
  std::uniform_real_distribution<double> uniform(0.0, 1.0);
  const double z = 1.0 - 2.0 * uniform(rng);
  const double phi = 2.0 * std::acos(-1.0) * uniform(rng);
  const double radial = std::sqrt(std::max(0.0, 1.0 - z * z));
  return {radial * std::cos(phi), radial * std::sin(phi), z};
}

double beta_22(std::mt19937_64 &rng) {
  std::uniform_real_distribution<double> uniform(0.0, 1.0);
  while (true) {
    const double value = uniform(rng);
    if (uniform(rng) <= 4.0 * value * (1.0 - value)) return value;
  }
}

}  // namespace

// ================================================================ C ABI
extern "C" {

struct oracle_params {
  int32_t mode;       // 0 compliance, 1 paired, 2 hot (paired with primal only)
  int32_t rng;        // 0 reference mt19937_64 stream, 1 counter (GPU) stream
  int32_t walks;
  int32_t max_steps;
  uint64_t seed;
  uint32_t repeat;
  uint32_t stream;
  double epsilon;
  double cavity_radius;
  double query_radius;
  int32_t green;       // 0 ball centre, 1 Beta(2,2) Green point, 2 exact ball integral
  int32_t n_source;
  int32_t n_adjoint;
  int32_t skip_cavity_sites;
  int32_t weight_order;  // reference association: 0 (f*r*r)/6 [wih_twos walk], 1 (r*r/6)*f [paired_site]
  int32_t threads;
  Term source[8];
  Term adjoint[8];
  int32_t n_boundary;  // Dirichlet data of u on the mesh (gradient form)
  int32_t pad;
  Term boundary[8];
};

struct oracle_site {
  double u, p, score, score_se, same_index;
  uint64_t steps, caps;
};

struct oracle_mesh {
  Mesh m;
};

static thread_local std::string g_error;

const char *oracle_last_error() { return g_error.c_str(); }

oracle_mesh *oracle_mesh_new(const double *vertices, uint32_t nv, const uint32_t *faces, uint32_t nf) {
  try {
    auto *om = new oracle_mesh;
    om->m.v.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) om->m.v[i] = {vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
    om->m.f.resize(nf);
    for (uint32_t i = 0; i < nf; ++i) {
      for (int k = 0; k < 3; ++k) {
        if (faces[3 * i + k] >= nv) throw std::runtime_error("face index out of range");
        om->m.f[i][k] = faces[3 * i + k];
      }
    }
    if (nf == 0) throw std::runtime_error("empty mesh");
    build_bvh(om->m);
    return om;
  } catch (const std::exception &e) {
    g_error = e.what();
    return nullptr;
  }
}

void oracle_mesh_free(oracle_mesh *om) { delete om; }

int oracle_bvh_info(const oracle_mesh *om, uint64_t *nodes, int *depth) {
  *nodes = om->m.bvh.nodes.size();
  *depth = om->m.bvh.depth;
  return 0;
}

// Batched closest point.  mode 0: BVH traversal (counts box/triangle tests
// into counts[2*i], counts[2*i+1] when counts != null); mode 1: brute force.
int oracle_closest_point(const oracle_mesh *om, const double *pts, uint64_t n, int brute, double radius,
                         double *dist, double *closest, uint32_t *tri, uint64_t *counts, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) {
    const Vec3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    QueryStats st;
    const Closest c = brute ? closest_point_brute(om->m, p) : closest_point(om->m, p, radius, &st);
    dist[i] = c.distance;
    if (closest) {
      closest[3 * i] = c.point.x;
      closest[3 * i + 1] = c.point.y;
      closest[3 * i + 2] = c.point.z;
    }
    if (tri) tri[i] = c.tri;
    if (counts) {
      counts[2 * i] = st.aabb;
      counts[2 * i + 1] = st.tri;
    }
  }
  return 0;
}

}  // extern "C"

namespace {

struct WalkOut {
  double u = 0.0, p = 0.0;
  uint32_t steps = 0;
  bool cap = false;
  bool failed = false;
  uint64_t aabb = 0, tri = 0;
};

inline double domain_distance(const Mesh &m, const Vec3 &x, const double *cav, uint32_t ncav, double cr,
                              double query_radius, QueryStats *st, bool &failed) {
  const Closest c = closest_point(m, x, query_radius, st);
  if (!std::isfinite(c.distance)) failed = true;
  double d = c.distance;
  for (uint32_t i = 0; i < ncav; ++i) {
    const Vec3 cc{cav[3 * i], cav[3 * i + 1], cav[3 * i + 2]};
    d = std::min(d, norm(x - cc) - cr);
  }
  return d;
}

inline bool inside_cavity(const Vec3 &x, const double *cav, uint32_t ncav, double cr) {
  for (uint32_t i = 0; i < ncav; ++i) {
    const Vec3 cc{cav[3 * i], cav[3 * i + 1], cav[3 * i + 2]};
    if (norm(x - cc) <= cr) return true;
  }
  return false;
}

// One walk.  Reference stream: wih_twos.cpp:635-664 (compliance) and
// adjoint.cpp:18-37 (paired).  Counter stream: the GPU kernel's draw layout.
WalkOut walk(const Mesh &m, const oracle_params &o, const double *cav, uint32_t ncav, Vec3 y, uint64_t site,
             uint32_t sample, bool count_tests) {
  WalkOut out;
  QueryStats st;
  QueryStats *stp = count_tests ? &st : nullptr;
  const bool primal_only = (o.mode != 1);  // compliance and hot keep only u
  const bool want_p = (o.mode == 1);
  if (o.rng == 0) {
    std::mt19937_64 rng;
    if (o.mode == 0) {
      // wih_twos.cpp:681-686: XOR of four hashed keys, reseeded through splitmix64.
      const uint64_t key = splitmix64(o.seed + 0x2d358dccaa6c78a5ULL) ^
                           splitmix64(static_cast<uint64_t>(o.repeat) + 0x8bb84b93962eacc9ULL) ^
                           splitmix64(site + 0x4b33a62ed433d4a3ULL) ^
                           splitmix64(static_cast<uint64_t>(sample) + 0x4d5a2da51de1aa47ULL);
      rng.seed(splitmix64(key));
    } else {
      // adjoint.cpp:22
      rng.seed(splitmix64(o.seed) ^ splitmix64(site + 91347) ^ splitmix64(static_cast<uint64_t>(sample) + 571));
    }
    for (int k = 0; k < o.max_steps; ++k) {
      const double r = domain_distance(m, y, cav, ncav, o.cavity_radius, o.query_radius, stp, out.failed);
      if (!(r > o.epsilon)) {
        out.aabb = st.aabb;
        out.tri = st.tri;
        return out;
      }
      Vec3 a = y;
      if (o.green == 2) {
        // The analytic study source (study.cpp:96-104): no Green-point draw.
        bool negative = false;
        out.u = exact_source(o.source, o.n_source, y, r, out.u, negative);
        if (want_p) out.p = exact_source(o.adjoint, o.n_adjoint, y, r, out.p, negative);
        if (negative) out.failed = true;
        y = y + random_unit_vector(rng) * r;
        ++out.steps;
        continue;
      }
      if (o.green) {
        // The scale operand (and so beta_22) is evaluated before the
        // direction, as g++ sequences `operator*(random_unit_vector(rng),
        // radius * beta_22(rng))`; the tracked fixtures pin this order.
        const double scale = r * beta_22(rng);
        const Vec3 dir = random_unit_vector(rng);
        a = y + dir * scale;
      }
      if (o.weight_order == 0) {
        out.u += source_value(o.source, o.n_source, a) * r * r / 6.0;
      } else {
        out.u += r * r / 6 * source_value(o.source, o.n_source, a);
        if (want_p) out.p += r * r / 6 * source_value(o.adjoint, o.n_adjoint, a);
      }
      y = y + random_unit_vector(rng) * r;
      ++out.steps;
    }
    out.cap = true;
  } else {
    CounterStream cs;
    counter_key(o.seed, o.stream, cs.k0, cs.k1);
    cs.walk = sample;
    cs.site = static_cast<uint32_t>(site);
    cs.repeat = o.repeat;
    for (int k = 0; k < o.max_steps; ++k) {
      const double r = domain_distance(m, y, cav, ncav, o.cavity_radius, o.query_radius, stp, out.failed);
      if (!(r > o.epsilon)) {
        out.aabb = st.aabb;
        out.tri = st.tri;
        return out;
      }
      double a0, a1;
      cs.uniforms(static_cast<uint32_t>(k), 0, a0, a1);
      Vec3 a = y;
      if (o.green == 2) {
        bool negative = false;
        out.u = exact_source(o.source, o.n_source, y, r, out.u, negative);
        if (want_p) out.p = exact_source(o.adjoint, o.n_adjoint, y, r, out.p, negative);
        if (negative) out.failed = true;
        y = y + direction_from(a0, a1) * r;
        ++out.steps;
        continue;
      }
      if (o.green) {
        double g0, g1, b0, b1, b2, spare;
        cs.uniforms(static_cast<uint32_t>(k), 1, g0, g1);
        cs.uniforms(static_cast<uint32_t>(k), 2, b0, b1);
        cs.uniforms(static_cast<uint32_t>(k), 3, b2, spare);
        const double beta = median3(b0, b1, b2);
        a = y + direction_from(g0, g1) * (r * beta);
      }
      const double w = r * r / 6.0;
      out.u += w * source_value(o.source, o.n_source, a);
      if (want_p) out.p += w * source_value(o.adjoint, o.n_adjoint, a);
      y = y + direction_from(a0, a1) * r;
      ++out.steps;
    }
    out.cap = true;
  }
  (void)primal_only;
  out.aabb = st.aabb;
  out.tri = st.tri;
  return out;
}

}  // namespace

extern "C" {

// exact_bump_green for cases[4i..4i+3] = (d, r, R, A) (the reader of
// analytic_integral_audit.cpp).  Returns 1 when an integral came out negative.
int oracle_exact_bump_green(const double *cases, uint32_t n, double *out) {
  bool negative = false;
  for (uint32_t i = 0; i < n; ++i)
    out[i] = exact_bump_green(cases[4 * i], cases[4 * i + 1], cases[4 * i + 2], cases[4 * i + 3], negative);
  if (negative) {
    g_error = "negative analytic Green integral";
    return 1;
  }
  return 0;
}

// Per-walk samples for n_sites sites (site ids site_ids[i], or i when null).
// u, p: [n_sites * walks]; steps: [n_sites * walks] with bit 31 set on a cap.
int oracle_walk_samples(const oracle_mesh *om, const oracle_params *o, const double *sites,
                        const uint64_t *site_ids, uint32_t n_sites, const double *cav, uint32_t ncav, double *u,
                        double *p, uint32_t *steps, uint64_t *tests) {
  std::atomic<int> failed{0};
#ifdef _OPENMP
  if (o->threads > 0) omp_set_num_threads(o->threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t i = 0; i < static_cast<int64_t>(n_sites); ++i) {
    const Vec3 x{sites[3 * i], sites[3 * i + 1], sites[3 * i + 2]};
    const uint64_t sid = site_ids ? site_ids[i] : static_cast<uint64_t>(i);
    const bool skip = o->skip_cavity_sites && inside_cavity(x, cav, ncav, o->cavity_radius);
    for (int w = 0; w < o->walks; ++w) {
      const size_t slot = static_cast<size_t>(i) * o->walks + w;
      if (skip) {
        u[slot] = 0.0;
        if (p) p[slot] = 0.0;
        steps[slot] = 0;
        continue;
      }
      const WalkOut r = walk(om->m, *o, cav, ncav, x, sid, static_cast<uint32_t>(w), tests != nullptr);
      if (r.failed) failed = 1;
      u[slot] = r.u;
      if (p) p[slot] = r.p;
      steps[slot] = r.steps | (r.cap ? 0x80000000u : 0u);
      if (tests) {
        tests[2 * slot] = r.aabb;
        tests[2 * slot + 1] = r.tri;
      }
    }
  }
  if (failed) {
    g_error = "closest-point query failed";
    return 1;
  }
  return 0;
}

// Per-site estimates.  Compliance: wih_twos.cpp:691-715 (mean, U-statistic
// (S^2 - S2)/(n(n-1)), leave-one-out jackknife SE).  Paired/hot:
// adjoint.cpp:36-41 (score (SuSp - Sup)/(n(n-1)), same_index Sup/n, hot
// score = mean u) plus the jackknife SE of the cross statistic.
int oracle_estimate(const oracle_mesh *om, const oracle_params *o, const double *sites, const uint64_t *site_ids,
                    uint32_t n_sites, const double *cav, uint32_t ncav, oracle_site *out) {
  const size_t total = static_cast<size_t>(n_sites) * o->walks;
  std::vector<double> u(total), p(total);
  std::vector<uint32_t> st(total);
  const int rc = oracle_walk_samples(om, o, sites, site_ids, n_sites, cav, ncav, u.data(), p.data(), st.data(),
                                     nullptr);
  const double n = o->walks;
  for (uint32_t i = 0; i < n_sites; ++i) {
    const double *U = &u[static_cast<size_t>(i) * o->walks];
    const double *P = &p[static_cast<size_t>(i) * o->walks];
    const uint32_t *S = &st[static_cast<size_t>(i) * o->walks];
    oracle_site r{};
    for (int w = 0; w < o->walks; ++w) {
      r.steps += S[w] & 0x7fffffffu;
      r.caps += (S[w] >> 31) & 1u;
    }
    if (o->mode == 0) {
      double sum = 0.0;
      for (int w = 0; w < o->walks; ++w) sum += U[w];
      double sum2 = 0.0;
      for (int w = 0; w < o->walks; ++w) sum2 += U[w] * U[w];
      r.u = sum / n;
      r.score = (sum * sum - sum2) / (n * (n - 1.0));
      if (o->walks >= 4) {
        std::vector<double> leave(o->walks);
        for (int w = 0; w < o->walks; ++w) {
          const double ls = sum - U[w], ls2 = sum2 - U[w] * U[w];
          leave[w] = (ls * ls - ls2) / ((n - 1.0) * (n - 2.0));
        }
        double lm = 0.0;
        for (double v : leave) lm += v;
        lm /= n;
        double spread = 0.0;
        for (double v : leave) spread += (v - lm) * (v - lm);
        r.score_se = std::sqrt((n - 1.0) / n * spread);
      } else {
        r.score_se = std::numeric_limits<double>::quiet_NaN();
      }
      r.p = r.u;
      r.same_index = sum2 / n;
    } else {
      double su = 0.0, sp = 0.0, same = 0.0;
      for (int w = 0; w < o->walks; ++w) {
        su += U[w];
        sp += P[w];
        same += U[w] * P[w];
      }
      const bool hot = (o->mode == 2);
      r.score = hot ? su / n : (su * sp - same) / (n * (n - 1));
      if (o->walks >= 4) {
        std::vector<double> leave(o->walks);
        for (int w = 0; w < o->walks; ++w) {
          if (hot) {
            leave[w] = (su - U[w]) / (n - 1.0);
          } else {
            leave[w] = ((su - U[w]) * (sp - P[w]) - (same - U[w] * P[w])) / ((n - 1.0) * (n - 2.0));
          }
        }
        double lm = 0.0;
        for (double v : leave) lm += v;
        lm /= n;
        double spread = 0.0;
        for (double v : leave) spread += (v - lm) * (v - lm);
        r.score_se = std::sqrt((n - 1.0) / n * spread);
      } else {
        r.score_se = std::numeric_limits<double>::quiet_NaN();
      }
      r.same_index = same / n;
      r.u = su / n;
      r.p = sp / n;
    }
    out[i] = r;
  }
  return rc;
}

// Reference-identical paired output fields (adjoint.cpp:36-41): the site
// loop skips sites inside a cavity (adjoint.cpp:123-126).
int oracle_sizeof_params() { return static_cast<int>(sizeof(oracle_params)); }
int oracle_sizeof_site() { return static_cast<int>(sizeof(oracle_site)); }

}  // extern "C"

// ================================================================ Differential WoS
// Restates evaluate_differential_site (wih_twos.cpp:839-928) with
// walk_to_boundary (725-740), closest_boundary (602-626),
// classify_offset_safety (765-837, with the WIH_ENCLOSURE_FALLBACK branch of
// benchmarks/submission_study/study.cpp:7) and EmbreeMesh::inside (361-394),
// in the reference's mt19937_64 stream (rng 0) or the GPU's counter stream
// (rng 1).  Distance queries and parity rays are counted as
// note_query(0)/(1)/(2) count them (study.cpp:8-16).

namespace {

struct Counters {
  uint64_t queries = 0, rays = 0, fallbacks = 0;
};

// Closest hit t of a ray in [tnear, tfar] (Moller-Trumbore, FP64), or -1.
double ray_triangle(const Vec3 &o, const Vec3 &d, const Vec3 &a, const Vec3 &b, const Vec3 &c) {
  const Vec3 e1 = b - a, e2 = c - a;
  const Vec3 pv{d.y * e2.z - d.z * e2.y, d.z * e2.x - d.x * e2.z, d.x * e2.y - d.y * e2.x};
  const double det = dot(e1, pv);
  if (det == 0.0) return -1.0;
  const double inv = 1.0 / det;
  const Vec3 tv = o - a;
  const double u = dot(tv, pv) * inv;
  if (u < 0.0 || u > 1.0) return -1.0;
  const Vec3 qv{tv.y * e1.z - tv.z * e1.y, tv.z * e1.x - tv.x * e1.z, tv.x * e1.y - tv.y * e1.x};
  const double w = dot(d, qv) * inv;
  if (w < 0.0 || u + w > 1.0) return -1.0;
  return dot(e2, qv) * inv;
}

bool ray_box(const Box &b, const Vec3 &o, const Vec3 &inv, double tmin, double tmax) {
  for (int a = 0; a < 3; ++a) {
    double t0 = (coord(b.lo, a) - coord(o, a)) * coord(inv, a), t1 = (coord(b.hi, a) - coord(o, a)) * coord(inv, a);
    if (t0 > t1) std::swap(t0, t1);
    tmin = std::max(tmin, t0);
    tmax = std::min(tmax, t1);
    if (tmin > tmax) return false;
  }
  return true;
}

double first_hit(const Mesh &m, const Vec3 &o, const Vec3 &d, double tnear, double tfar) {
  const Vec3 inv{1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
  double best = -1.0, lim = tfar;
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const Bvh::Node &n = m.bvh.nodes[stack[--sp]];
    if (!ray_box(n.box, o, inv, tnear, lim)) continue;
    if (n.left < 0) {
      for (int i = 0; i < n.count; ++i) {
        const auto &f = m.f[m.bvh.order[n.begin + i]];
        const double t = ray_triangle(o, d, m.v[f[0]], m.v[f[1]], m.v[f[2]]);
        if (t >= tnear && t <= lim) {
          lim = t;
          best = t;
        }
      }
    } else {
      stack[sp++] = n.left;
      stack[sp++] = n.right;
    }
  }
  return best;
}

// EmbreeMesh::inside: parity of hits along a fixed oblique ray, re-shot from
// each hit (t + 2e-6), at most 128 hits.
bool inside_parity(const Mesh &m, const Vec3 &p, Counters &cnt) {
  Vec3 dir{1.0, 0.3713906763541037, 0.1570796326794897};
  dir = dir * (1.0 / norm(dir));
  Vec3 origin = p;
  unsigned hits = 0;
  for (; hits < 128; ++hits) {
    ++cnt.rays;
    const double t = first_hit(m, origin, dir, 1.0e-6, 4.0);
    if (t < 0.0) break;
    origin = origin + dir * (t + 2.0e-6);
  }
  if (hits == 128) throw std::runtime_error("ray-parity traversal exceeded 128 intersections");
  return hits % 2U == 1U;
}

struct Hit {
  double distance = std::numeric_limits<double>::infinity();
  Vec3 point, normal;
  int cavity = -1;
};

Hit closest_boundary(const Mesh &m, const Vec3 &x, const std::vector<Vec3> &cav, double R, Counters &cnt) {
  ++cnt.queries;
  const Closest c = closest_point(m, x, 4.0, nullptr);
  if (!std::isfinite(c.distance)) throw std::runtime_error("closest-point query failed");
  Hit h;
  h.distance = c.distance;
  h.point = c.point;
  if (c.distance > 0.0) h.normal = (c.point - x) * (1.0 / c.distance);
  for (size_t i = 0; i < cav.size(); ++i) {
    const Vec3 radial = x - cav[i];
    const double len = norm(radial);
    const double d = len - R;
    if (d < h.distance && len > 0.0) {
      const Vec3 dir = radial * (1.0 / len);
      h.distance = d;
      h.point = cav[i] + dir * R;
      h.normal = dir * -1.0;
      h.cavity = static_cast<int>(i);
    }
  }
  return h;
}

double domain_distance_counted(const Mesh &m, const Vec3 &x, const std::vector<Vec3> &cav, double R, Counters &cnt) {
  ++cnt.queries;
  const Closest c = closest_point(m, x, 4.0, nullptr);
  if (!std::isfinite(c.distance)) throw std::runtime_error("closest-point query failed");
  double d = c.distance;
  for (const Vec3 &cc : cav) d = std::min(d, norm(x - cc) - R);
  return d;
}

struct DiffSite {
  std::vector<double> sums, sq;  // per cavity: cx, cy, cz, r
  uint64_t outer_steps = 0, nested_steps = 0, cav_terms = 0, near_seam = 0, seg_unsafe = 0, unsafe = 0, limits = 0;
};

}  // namespace

extern "C" {

// Per-site results: out[site][cavity][8] = dc (3), dc_se (3), dR, dR_se;
// stats[site][7] = outer_steps, nested_steps, cavity_terminations,
// near_seam, segment_unsafe, unsafe_offset, limits; totals[3] = distance
// queries, parity rays, enclosure fallbacks.
int oracle_diffwos(const oracle_mesh *om, const oracle_params *o, double diff_offset, int enclosure_fallback,
                   const double *sites, const uint64_t *site_ids, uint32_t n_sites, const double *cav_xyz,
                   uint32_t ncav, double *out, uint64_t *stats, uint64_t *totals) {
  const Mesh &m = om->m;
  std::vector<Vec3> cav(ncav);
  for (uint32_t i = 0; i < ncav; ++i) cav[i] = {cav_xyz[3 * i], cav_xyz[3 * i + 1], cav_xyz[3 * i + 2]};
  const double R = o->cavity_radius, eps = o->epsilon;
  std::atomic<uint64_t> tq{0}, tr{0}, tf{0};
  std::atomic<int> failed{0};
#ifdef _OPENMP
  if (o->threads > 0) omp_set_num_threads(o->threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t si = 0; si < static_cast<int64_t>(n_sites); ++si) {
    try {
      Counters cnt;
      const Vec3 x0{sites[3 * si], sites[3 * si + 1], sites[3 * si + 2]};
      const uint64_t site = site_ids ? site_ids[si] : static_cast<uint64_t>(si);
      DiffSite r;
      r.sums.assign(4 * ncav, 0.0);
      r.sq.assign(4 * ncav, 0.0);
      for (int sample = 0; sample < o->walks; ++sample) {
        const uint64_t outer_key = splitmix64(o->seed + 0x6a09e667f3bcc909ULL) ^
                                   splitmix64(static_cast<uint64_t>(o->repeat) + 0xbb67ae8584caa73bULL) ^
                                   splitmix64(site + 0x3c6ef372fe94f82bULL) ^
                                   splitmix64(static_cast<uint64_t>(sample) + 0xa54ff53a5f1d36f1ULL);
        // walk_to_boundary.  Counter stream: the outer walk draws block 0 of
        // (seed, stream); the nested walk is a compliance walk of
        // (seed, stream + 1), both at counter (step, sample, site, repeat).
        std::mt19937_64 rng(splitmix64(outer_key));
        CounterStream cs_outer{}, cs_nested{};
        if (o->rng != 0) {
          counter_key(o->seed, o->stream, cs_outer.k0, cs_outer.k1);
          counter_key(o->seed, o->stream + 1, cs_nested.k0, cs_nested.k1);
          cs_outer.walk = cs_nested.walk = static_cast<uint32_t>(sample);
          cs_outer.site = cs_nested.site = static_cast<uint32_t>(site);
          cs_outer.repeat = cs_nested.repeat = o->repeat;
        }
        Vec3 y = x0;
        Hit hit;
        int steps = 0;
        bool limit = true;
        for (int k = 0; k < o->max_steps; ++k) {
          hit = closest_boundary(m, y, cav, R, cnt);
          if (!(hit.distance > eps)) {
            limit = false;
            break;
          }
          if (o->rng == 0) {
            y = y + random_unit_vector(rng) * hit.distance;
          } else {
            double a0, a1;
            cs_outer.uniforms(static_cast<uint32_t>(k), 0, a0, a1);
            y = y + direction_from(a0, a1) * hit.distance;
          }
          ++steps;
        }
        r.outer_steps += steps;
        if (limit) {
          ++r.limits;
          continue;
        }
        if (hit.cavity < 0) continue;
        ++r.cav_terms;
        const Vec3 offset = hit.point - hit.normal * diff_offset;
        // classify_offset_safety
        bool near_seam = false, seg_unsafe = false;
        const Vec3 segment = offset - hit.point;
        const double seg2 = dot(segment, segment);
        const double tol = 1.0e-10 * std::max(1.0, std::abs(R));
        const double coll2 = (R + tol) * (R + tol);
        const Vec3 &hc = cav[hit.cavity];
        for (size_t i = 0; i < cav.size(); ++i) {
          if (static_cast<int>(i) == hit.cavity) continue;
          const Vec3 cd = cav[i] - hc;
          const double cdist = norm(cd);
          if (cdist > tol && cdist < 2.0 * R) {
            const Vec3 axis = cd * (1.0 / cdist);
            const Vec3 seam_center = (hc + cav[i]) * 0.5;
            const double seam_r = std::sqrt(std::max(0.0, R * R - 0.25 * (cdist * cdist)));
            const Vec3 rel = hit.point - seam_center;
            const double axial = dot(rel, axis);
            const Vec3 radial = rel - axis * axial;
            const double nr = norm(radial) - seam_r;
            const double seam_d = std::sqrt(axial * axial + nr * nr);
            near_seam = near_seam || seam_d <= diff_offset;
          }
          if (seg2 > 0.0) {
            const double par = std::clamp(dot(cav[i] - hit.point, segment) / seg2, 0.0, 1.0);
            const Vec3 cl = hit.point + segment * par;
            if (dot(cl - cav[i], cl - cav[i]) <= coll2) seg_unsafe = true;
          }
        }
        bool inside = inside_parity(m, offset, cnt);
        if (enclosure_fallback && !inside && inside_parity(m, hc, cnt)) {
          ++cnt.queries;
          const Closest cc = closest_point(m, hc, 4.0, nullptr);
          if (cc.distance > R + diff_offset + eps && norm(offset - hc) <= R + diff_offset + eps * 0.5) {
            inside = true;
            ++cnt.fallbacks;
          }
        }
        if (!inside || !(domain_distance_counted(m, offset, cav, R, cnt) > eps)) seg_unsafe = true;
        r.near_seam += near_seam;
        r.seg_unsafe += seg_unsafe;
        if (near_seam || seg_unsafe) {
          ++r.unsafe;
          continue;
        }
        // nested walk (wih_twos.cpp walk, counted queries)
        const uint64_t nested_key = splitmix64(outer_key ^ 0x510e527fade682d1ULL);
        std::mt19937_64 nr(splitmix64(nested_key));
        Vec3 z = offset;
        double value = 0.0;
        int nsteps = 0;
        bool nlimit = true;
        for (int k = 0; k < o->max_steps; ++k) {
          const double rr = domain_distance_counted(m, z, cav, R, cnt);
          if (!(rr > eps)) {
            nlimit = false;
            break;
          }
          if (o->rng == 0) {
            Vec3 a = z;
            if (o->green) {
              const double scale = rr * beta_22(nr);
              const Vec3 dir = random_unit_vector(nr);
              a = z + dir * scale;
            }
            value += source_value(o->source, o->n_source, a) * rr * rr / 6.0;
            z = z + random_unit_vector(nr) * rr;
          } else {
            // The GPU walk's draw layout (see walk()).
            double a0, a1;
            cs_nested.uniforms(static_cast<uint32_t>(k), 0, a0, a1);
            Vec3 a = z;
            if (o->green) {
              double g0, g1, b0, b1, b2, spare;
              cs_nested.uniforms(static_cast<uint32_t>(k), 1, g0, g1);
              cs_nested.uniforms(static_cast<uint32_t>(k), 2, b0, b1);
              cs_nested.uniforms(static_cast<uint32_t>(k), 3, b2, spare);
              a = z + direction_from(g0, g1) * (rr * median3(b0, b1, b2));
            }
            value += rr * rr / 6.0 * source_value(o->source, o->n_source, a);
            z = z + direction_from(a0, a1) * rr;
          }
          ++nsteps;
        }
        r.nested_steps += nsteps;
        r.limits += nlimit ? 1 : 0;
        const double scale = value / diff_offset;
        const double sample_v[4] = {hit.normal.x * scale, hit.normal.y * scale, hit.normal.z * scale, -scale};
        for (int k = 0; k < 4; ++k) {
          r.sums[4 * hit.cavity + k] += sample_v[k];
          r.sq[4 * hit.cavity + k] += sample_v[k] * sample_v[k];
        }
      }
      const double n = o->walks;
      for (uint32_t c = 0; c < ncav; ++c) {
        double *row = out + (static_cast<size_t>(si) * ncav + c) * 8;
        for (int k = 0; k < 3; ++k) row[k] = r.sums[4 * c + k] * (1.0 / n);
        row[6] = r.sums[4 * c + 3] / n;
        const double den = n * (n - 1.0);
        for (int k = 0; k < 4; ++k) {
          const double v = o->walks > 1 ? std::sqrt(std::max(0.0, (r.sq[4 * c + k] - r.sums[4 * c + k] *
                                                                                            r.sums[4 * c + k] / n) /
                                                                        den))
                                        : 0.0;
          if (k < 3)
            row[3 + k] = v;
          else
            row[7] = v;
        }
      }
      uint64_t *st = stats + 7 * static_cast<size_t>(si);
      st[0] = r.outer_steps;
      st[1] = r.nested_steps;
      st[2] = r.cav_terms;
      st[3] = r.near_seam;
      st[4] = r.seg_unsafe;
      st[5] = r.unsafe;
      st[6] = r.limits;
      tq += cnt.queries;
      tr += cnt.rays;
      tf += cnt.fallbacks;
    } catch (const std::exception &) {
      failed = 1;
    }
  }
  totals[0] = tq;
  totals[1] = tr;
  totals[2] = tf;
  if (failed) {
    g_error = "differential walk failed";
    return 1;
  }
  return 0;
}

}  // extern "C"

// ================================================================ certified validation
// Restates the certified fresh-sample validator of
// benchmarks/compiled_bunny/src/minimum_benefit.hpp (run_minimum_benefit,
// cert_walk, CertDistanceTree, cert_source_lower): a walk whose distances are
// rigorous lower bounds (distance to the union of the triangles' bounding
// boxes, every positive operation rounded one ulp down after rounding to
// nearest), whose ball radius is min(radius_cap, 0.95 d), whose payoff is a
// rounded-down lower bound of the source, clipped at value_cap, and which
// fails closed when a sampled point might leave its ball.

namespace {

inline double rdn(double x) { return std::nextafter(x, -std::numeric_limits<double>::infinity()); }
inline double rup(double x) { return std::nextafter(x, std::numeric_limits<double>::infinity()); }
inline double pos_dn(double x) { return std::max(0.0, rdn(x)); }

double cert_box_lower(const Vec3 &lo, const Vec3 &hi, const Vec3 &x) {
  double sum = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double g = std::max({0.0, rdn(coord(lo, a) - coord(x, a)), rdn(coord(x, a) - coord(hi, a))});
    sum = pos_dn(sum + pos_dn(g * g));
  }
  return pos_dn(std::sqrt(sum));
}

double cert_point_distance(const Vec3 &a, const Vec3 &b, bool upper) {
  double sum = 0.0;
  for (int k = 0; k < 3; ++k) {
    double d = std::abs(coord(a, k) - coord(b, k));
    d = upper ? rup(d) : pos_dn(d);
    const double q = upper ? rup(d * d) : pos_dn(d * d);
    sum = upper ? rup(sum + q) : pos_dn(sum + q);
  }
  return upper ? rup(std::sqrt(sum)) : pos_dn(std::sqrt(sum));
}

// Minimum over triangles of the lower distance to each triangle's box; the
// oracle BVH's node boxes (unions of those boxes) prune exactly.
double cert_mesh_distance(const Mesh &m, const Vec3 &x) {
  double best = std::numeric_limits<double>::infinity();
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const Bvh::Node &n = m.bvh.nodes[stack[--sp]];
    if (cert_box_lower(n.box.lo, n.box.hi, x) >= best) continue;
    if (n.left < 0) {
      for (int i = 0; i < n.count; ++i) {
        const auto &f = m.f[m.bvh.order[n.begin + i]];
        Box b;
        b.grow(m.v[f[0]]);
        b.grow(m.v[f[1]]);
        b.grow(m.v[f[2]]);
        best = std::min(best, cert_box_lower(b.lo, b.hi, x));
      }
    } else {
      stack[sp++] = n.left;
      stack[sp++] = n.right;
    }
  }
  return best;
}

double cert_domain_distance(const Mesh &m, const Vec3 &p, const std::vector<Vec3> &holes, double r) {
  double d = cert_mesh_distance(m, p);
  for (const Vec3 &c : holes) d = std::min(d, rdn(cert_point_distance(p, c, false) - r));
  return std::max(0.0, d);
}

// (1 - t/1024)^1024 <= exp(-t), every step rounded down.
double cert_exp_lower(double t_upper) {
  double a = std::max(0.0, rdn(1.0 - rup(t_upper / 1024.0)));
  for (int i = 0; i < 10; ++i) a = pos_dn(a * a);
  return a;
}

// Lower bound of a source given as terms: a leading constant, then linear
// terms (down(value + down(amp down(x + offset)))) and Gaussian terms
// (down(value + pos_dn(amp exp_lower(exponent_up)))); cert_source_lower's
// affine and housing forms are exactly these sequences.
double cert_source_lower(const Term *terms, int n, const Vec3 &p) {
  double value = n > 0 && terms[0].kind == 0 ? terms[0].amp : 0.0;
  for (int i = (n > 0 && terms[0].kind == 0) ? 1 : 0; i < n; ++i) {
    const Term &t = terms[i];
    if (t.kind == 1) {
      value = rdn(value + rdn(t.amp * rdn(coord(p, t.axis) + t.offset)));
    } else if (t.kind == 2) {
      double exponent = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double q = rup(rup(std::abs(coord(p, a) - t.c[a])) / t.w[a]);
        exponent = rup(exponent + rup(q * q));
      }
      value = rdn(value + pos_dn(t.amp * cert_exp_lower(exponent)));
    } else if (t.kind == 0) {
      value = rdn(value + t.amp);
    }
  }
  return std::max(0.0, value);
}

struct CertSample {
  double value = 0.0;
  int steps = 0;
  bool capped = false, clipped = false, contained = true;
};

CertSample cert_walk(const Mesh &m, const std::vector<Vec3> &holes, Vec3 point, const oracle_params &o,
                     double radius_cap, double value_cap, uint64_t site, uint32_t sample) {
  std::mt19937_64 rng;
  CounterStream cs{};
  if (o.rng == 0) {
    rng.seed(splitmix64(splitmix64(o.seed) ^ splitmix64(site + 0xa1224ULL) ^ splitmix64(sample + 0x6242cULL)));
  } else {
    counter_key(o.seed, o.stream, cs.k0, cs.k1);
    cs.walk = sample;
    cs.site = static_cast<uint32_t>(site);
    cs.repeat = o.repeat;
  }
  CertSample out;
  for (int k = 0; k < o.max_steps; ++k) {
    const double d = cert_domain_distance(m, point, holes, o.cavity_radius);
    if (d <= o.epsilon) return out;
    const double s = std::min(radius_cap, pos_dn(0.95 * d));
    Vec3 y = point, next;
    if (o.rng == 0) {
      if (o.green) {
        const double scale = s * beta_22(rng);
        y = point + random_unit_vector(rng) * scale;
      }
      next = point + random_unit_vector(rng) * s;
    } else {
      double a0, a1;
      cs.uniforms(static_cast<uint32_t>(k), 0, a0, a1);
      if (o.green) {
        double g0, g1, b0, b1, b2, spare;
        cs.uniforms(static_cast<uint32_t>(k), 1, g0, g1);
        cs.uniforms(static_cast<uint32_t>(k), 2, b0, b1);
        cs.uniforms(static_cast<uint32_t>(k), 3, b2, spare);
        y = point + direction_from(g0, g1) * (s * median3(b0, b1, b2));
      }
      next = point + direction_from(a0, a1) * s;
    }
    if (!(cert_point_distance(point, next, true) < d) || !(cert_point_distance(point, y, true) < d)) {
      out.contained = false;
      return out;
    }
    const double weight = pos_dn(pos_dn(s * s) / 6.0);
    const double increment = pos_dn(weight * cert_source_lower(o.source, o.n_source, y));
    out.value = pos_dn(out.value + increment);
    ++out.steps;
    if (out.value >= value_cap) {
      out.value = value_cap;
      out.clipped = true;
      return out;
    }
    point = next;
  }
  out.capped = true;
  return out;
}

}  // namespace

extern "C" {

// Certified samples for n_sites sites (site ids site_ids[i] or i):
// value/steps [n_sites * walks], flags bit 0 capped, bit 1 clipped, bit 2
// containment failure; clearance[i] = the certified domain distance at site
// i.  Returns 1 when a site is outside the mesh or inside a cavity.
int oracle_validate(const oracle_mesh *om, const oracle_params *o, double radius_cap, double value_cap,
                    const double *sites, const uint64_t *site_ids, uint32_t n_sites, const double *cav_xyz,
                    uint32_t ncav, double *value, uint32_t *steps, uint8_t *flags, double *clearance) {
  const Mesh &m = om->m;
  std::vector<Vec3> holes(ncav);
  for (uint32_t i = 0; i < ncav; ++i) holes[i] = {cav_xyz[3 * i], cav_xyz[3 * i + 1], cav_xyz[3 * i + 2]};
  for (uint32_t s = 0; s < n_sites; ++s) {
    const Vec3 x{sites[3 * s], sites[3 * s + 1], sites[3 * s + 2]};
    Counters cnt;
    bool in_cav = false;
    for (const Vec3 &c : holes) in_cav = in_cav || norm(x - c) <= o->cavity_radius;
    if (!inside_parity(m, x, cnt) || in_cav) {
      g_error = "candidate classified outside; exact driver predicate is also required";
      return 1;
    }
    clearance[s] = cert_domain_distance(m, x, holes, o->cavity_radius);
    const uint64_t site = site_ids ? site_ids[s] : s;
#ifdef _OPENMP
    if (o->threads > 0) omp_set_num_threads(o->threads);
#pragma omp parallel for schedule(static)
#endif
    for (int j = 0; j < o->walks; ++j) {
      const CertSample c = cert_walk(m, holes, x, *o, radius_cap, value_cap, site, static_cast<uint32_t>(j));
      const size_t slot = static_cast<size_t>(s) * o->walks + j;
      value[slot] = c.value;
      steps[slot] = static_cast<uint32_t>(c.steps);
      flags[slot] = static_cast<uint8_t>((c.capped ? 1 : 0) | (c.clipped ? 2 : 0) | (c.contained ? 0 : 4));
    }
  }
  return 0;
}

}  // extern "C"

// ================================================================ gradient form
// The GPU's gradient form (twos_estimate_gradient) in the counter stream:
// paired walks whose first ball gives the gradient samples
//   grad U = (3/R) (U - u0) w + R (1 - t^3) f(x + t R w') w'
// (likewise grad P with the adjoint source), plus Dirichlet data g of u at
// the exit point on the mesh.  No reference counterpart: this is the plain
// method's Neumann-cavity estimator (unit sphere, harmonic Dirichlet data).

namespace {

struct GradWalk {
  double u = 0.0, p = 0.0, gu[3] = {0, 0, 0}, gp[3] = {0, 0, 0};
  uint32_t steps = 0;
  bool cap = false, failed = false;
};

GradWalk grad_walk(const Mesh &m, const oracle_params &o, const double *cav, uint32_t ncav, Vec3 y, uint64_t site,
                   uint32_t sample) {
  GradWalk out;
  CounterStream cs;
  counter_key(o.seed, o.stream, cs.k0, cs.k1);
  cs.walk = sample;
  cs.site = static_cast<uint32_t>(site);
  cs.repeat = o.repeat;
  double r0 = 0.0, u0 = 0.0, p0 = 0.0;
  Vec3 w0, su, sp;
  for (int k = 0; k < o.max_steps; ++k) {
    const Closest c = closest_point(m, y, o.query_radius, nullptr);
    if (!std::isfinite(c.distance)) out.failed = true;
    double r = c.distance;
    bool cav_nearer = false;
    for (uint32_t i = 0; i < ncav; ++i) {
      const Vec3 cc{cav[3 * i], cav[3 * i + 1], cav[3 * i + 2]};
      const double dc = norm(y - cc) - o.cavity_radius;
      r = std::min(r, dc);
      if (dc < c.distance) cav_nearer = true;
    }
    if (!(r > o.epsilon)) {
      // Exit: Dirichlet data at the nearest mesh point (the walk's position
      // when it stops at its first query, as the device does).
      if (o.n_boundary > 0 && !cav_nearer) out.u += source_value(o.boundary, o.n_boundary, k == 0 ? y : c.point);
      break;
    }
    double a0, a1;
    cs.uniforms(static_cast<uint32_t>(k), 0, a0, a1);
    Vec3 a = y;
    if (o.green) {
      double g0, g1, b0, b1, b2, spare;
      cs.uniforms(static_cast<uint32_t>(k), 1, g0, g1);
      cs.uniforms(static_cast<uint32_t>(k), 2, b0, b1);
      cs.uniforms(static_cast<uint32_t>(k), 3, b2, spare);
      a = y + direction_from(g0, g1) * (r * median3(b0, b1, b2));
    }
    const double w = r * r / 6.0;
    const double du = w * source_value(o.source, o.n_source, a), dp = w * source_value(o.adjoint, o.n_adjoint, a);
    out.u += du;
    out.p += dp;
    const Vec3 dir = direction_from(a0, a1);
    if (k == 0) {
      double t, b0, b1, spare;
      cs.uniforms(0, 4, t, b0);
      cs.uniforms(0, 5, b1, spare);
      const Vec3 wp = direction_from(b0, b1);
      const Vec3 z = y + wp * (t * r);
      const double wt = r * (1.0 - t * t * t);
      const double fs = wt * source_value(o.source, o.n_source, z);
      const double fq = wt * source_value(o.adjoint, o.n_adjoint, z);
      su = wp * fs;
      sp = wp * fq;
      r0 = r;
      u0 = du;
      p0 = dp;
      w0 = dir;
    }
    y = y + dir * r;
    ++out.steps;
    if (k + 1 == o.max_steps) out.cap = true;
  }
  if (r0 > 0.0) {
    const double kf = 3.0 / r0, cu = kf * (out.u - u0), cp = kf * (out.p - p0);
    const Vec3 gu = w0 * cu + su, gp = w0 * cp + sp;
    out.gu[0] = gu.x;
    out.gu[1] = gu.y;
    out.gu[2] = gu.z;
    out.gp[0] = gp.x;
    out.gp[1] = gp.y;
    out.gp[2] = gp.z;
  }
  return out;
}

}  // namespace

extern "C" {

// Per-site gradient rows (u, p, grad_u[3], grad_p[3], cross, cross_se,
// u_se, p_se as doubles; steps, caps as uint64 in a separate array),
// and optionally the per-walk samples (u, p, grad_u, grad_p: 8 doubles).
int oracle_estimate_gradient(const oracle_mesh *om, const oracle_params *o, const double *sites, uint32_t n_sites,
                             const double *cav, uint32_t ncav, double *rows, uint64_t *counts, double *walks) {
  std::atomic<int> failed{0};
  const int N = o->walks;
#ifdef _OPENMP
  if (o->threads > 0) omp_set_num_threads(o->threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t s = 0; s < static_cast<int64_t>(n_sites); ++s) {
    const Vec3 x{sites[3 * s], sites[3 * s + 1], sites[3 * s + 2]};
    std::vector<GradWalk> W(N);
    for (int j = 0; j < N; ++j) {
      W[j] = grad_walk(om->m, *o, cav, ncav, x, static_cast<uint64_t>(s), static_cast<uint32_t>(j));
      if (W[j].failed) failed = 1;
    }
    double su = 0, sp = 0, sgu[3] = {0, 0, 0}, sgp[3] = {0, 0, 0}, sdot = 0;
    uint64_t steps = 0, caps = 0;
    for (const GradWalk &g : W) {
      su += g.u;
      sp += g.p;
      double d = 0;
      for (int k = 0; k < 3; ++k) {
        sgu[k] += g.gu[k];
        sgp[k] += g.gp[k];
        d += g.gu[k] * g.gp[k];
      }
      sdot += d;
      steps += g.steps;
      caps += g.cap;
    }
    const double n = N;
    const double cross = (sgu[0] * sgp[0] + sgu[1] * sgp[1] + sgu[2] * sgp[2] - sdot) / (n * (n - 1.0));
    std::vector<double> leave(N);
    double mean = 0;
    for (int j = 0; j < N; ++j) {
      const GradWalk &g = W[j];
      double d = 0, c = 0;
      for (int k = 0; k < 3; ++k) {
        d += g.gu[k] * g.gp[k];
        c += (sgu[k] - g.gu[k]) * (sgp[k] - g.gp[k]);
      }
      leave[j] = (c - (sdot - d)) / ((n - 1.0) * (n - 2.0));
      mean += leave[j];
    }
    mean /= n;
    double spread = 0;
    for (double v : leave) spread += (v - mean) * (v - mean);
    double vu = 0, vp = 0;
    for (const GradWalk &g : W) {
      vu += (g.u - su / n) * (g.u - su / n);
      vp += (g.p - sp / n) * (g.p - sp / n);
    }
    double *row = rows + 12 * s;
    row[0] = su / n;
    row[1] = sp / n;
    for (int k = 0; k < 3; ++k) {
      row[2 + k] = sgu[k] / n;
      row[5 + k] = sgp[k] / n;
    }
    row[8] = cross;
    row[9] = N > 2 ? std::sqrt((n - 1.0) / n * spread) : 0.0;
    row[10] = N > 1 ? std::sqrt(vu / (n * (n - 1.0))) : 0.0;
    row[11] = N > 1 ? std::sqrt(vp / (n * (n - 1.0))) : 0.0;
    counts[2 * s] = steps;
    counts[2 * s + 1] = caps;
    if (walks)
      for (int j = 0; j < N; ++j) {
        double *w = walks + (static_cast<size_t>(s) * N + j) * 8;
        w[0] = W[j].u;
        w[1] = W[j].p;
        for (int k = 0; k < 3; ++k) {
          w[2 + k] = W[j].gu[k];
          w[5 + k] = W[j].gp[k];
        }
      }
  }
  if (failed) {
    g_error = "closest-point query failed";
    return 1;
  }
  return 0;
}

}  // extern "C"

// ================================================================ Array-RQMC
// The GPU's lockstep Array-RQMC / matched MC walks (twos_rqmc) in FP64 and
// the counter stream: per (site, batch), each step answers every active
// walk's query, stops walks within epsilon (boundary data at the exit),
// orders active walks by the 3D Hilbert key of their position (finished
// walks last, ties by walk index) and gives the walk of rank i the 3D
// Korobov point (i/n, g i/n, g^2 i/n) whose last two coordinates, shifted by
// (U1, U2) mod 1, drive the step -- the 3D form of
// benchmarks/critical_baselines/sampling.py:49-74.  oracle_neighbour_means
// is reused_means (sampling.py:76-88) in 3D.

namespace {

// Skilling's transpose method for the Hilbert index (AIP Conf. Proc. 707,
// 2004), 3 axes x 10 bits, axis 0 most significant.
uint32_t oracle_hilbert3(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t X[3] = {x, y, z};
  for (uint32_t Q = 1u << 9; Q > 1u; Q >>= 1) {
    const uint32_t P = Q - 1u;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; ++i) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Q = 1u << 9; Q > 1u; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1u;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  uint32_t h = 0;
  for (int bit = 9; bit >= 0; --bit)
    for (int i = 0; i < 3; ++i) h = (h << 1) | ((X[i] >> bit) & 1u);
  return h;
}

}  // namespace

namespace {

// Sobol' direction numbers in the fixed-point form of Bratley and Fox (ACM
// TOMS 14, 1988): V_k = m_k 2^(32-k), and beyond the degree s of the
// dimension's polynomial x^s + a_1 x^(s-1) + ... + a_(s-1) x + 1,
// V_k = a_1 V_(k-1) ^ ... ^ a_(s-1) V_(k-s+1) ^ V_(k-s) ^ (V_(k-s) >> s).
// Dimension 0 is van der Corput's; dimension d >= 1 the d-th primitive
// polynomial (by degree, then coefficient bits; primitivity by counting the
// order of x directly), initial odd m_k < 2^k from SplitMix64 of
// 0x536f626f6c2d3344 + 64 d + k.
uint64_t oracle_splitmix(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

bool oracle_primitive(uint32_t p, int deg) {
  // Powers of x modulo p until they return to 1.
  const uint32_t top = 1u << deg, want = top - 1u;
  uint32_t r = 1;
  for (uint32_t e = 1; e <= want; ++e) {
    r <<= 1;
    if (r & top) r ^= p;
    if (r == 1u) return e == want;
  }
  return false;
}

std::vector<uint32_t> oracle_sobol_table(uint32_t dims, uint32_t bits) {
  std::vector<uint32_t> polys;
  for (int deg = 1; polys.size() + 1 < dims; ++deg)
    for (uint32_t p = (1u << deg) | 1u; p < (2u << deg) && polys.size() + 1 < dims; p += 2)
      if (oracle_primitive(p, deg)) polys.push_back(p);
  std::vector<uint32_t> out(static_cast<size_t>(dims) * bits);
  for (uint32_t d = 0; d < dims; ++d) {
    std::vector<uint32_t> V(bits + 1, 0u);
    if (d == 0) {
      for (uint32_t k = 1; k <= bits; ++k) V[k] = 1u << (32 - k);
    } else {
      const uint32_t p = polys[d - 1];
      int s = 0;
      while ((p >> (s + 1)) != 0u) ++s;
      for (uint32_t k = 1; k <= bits; ++k) {
        if (static_cast<int>(k) <= s) {
          const uint64_t m = (oracle_splitmix(0x536f626f6c2d3344ull + 64ull * d + k) & ((1ull << k) - 1)) | 1ull;
          V[k] = static_cast<uint32_t>(m << (32 - k));
        } else {
          uint32_t x = V[k - s] ^ (V[k - s] >> s);
          for (int j = 1; j < s; ++j)
            if ((p >> (s - j)) & 1u) x ^= V[k - j];
          V[k] = x;
        }
      }
    }
    for (uint32_t b = 0; b < bits; ++b) out[static_cast<size_t>(d) * bits + b] = V[b + 1];
  }
  return out;
}

}  // namespace

extern "C" {

uint32_t oracle_hilbert_key(uint32_t x, uint32_t y, uint32_t z) { return oracle_hilbert3(x, y, z); }

// The Sobol' direction numbers twos_rqmc's SOBOL method uses: out [dims][bits].
void oracle_sobol_directions(uint32_t dims, uint32_t bits, uint32_t *out) {
  const std::vector<uint32_t> t = oracle_sobol_table(dims, bits);
  std::copy(t.begin(), t.end(), out);
}

// batch_u, batch_p: [batches][n_sites]; steps, caps summed.  method 0 MC,
// 1 ARRAY, 3 SOBOL (Sobol-over-steps: walk i holds point i of the Sobol'
// sequence scrambled per (site, batch, coordinate) by a lower-triangular
// digit matrix with unit diagonal and a digital shift, drawn per step from
// the counter stream; coordinates 2k, 2k + 1 at step k < 256, the MC stream
// after).
// Optional record (each may be null): walk_first [batches][n_sites][walks][3]
// the point after the first step, walk_u / walk_p [batches][n_sites][walks]
// each walk's payoffs, site_radius [n_sites] the first ball's radius.
int oracle_rqmc(const oracle_mesh *om, const oracle_params *o, int method, uint32_t batches, uint32_t generator,
                const double *bbox_lo, const double *bbox_hi, const Term *ub, int n_ub, const Term *pb, int n_pb,
                const double *sites, uint32_t n_sites, double *batch_u, double *batch_p, uint64_t *totals,
                double *walk_first, double *walk_u, double *walk_p, double *site_radius) {
  const Mesh &m = om->m;
  const uint32_t n = static_cast<uint32_t>(o->walks);
  uint32_t k0, k1;
  counter_key(o->seed, o->stream, k0, k1);
  constexpr uint32_t kSobolSteps = 256, kSobolBits = 10;
  uint32_t sobol_bits = 0;
  while ((1u << sobol_bits) < n) ++sobol_bits;
  const std::vector<uint32_t> sobol = method == 3 ? oracle_sobol_table(2 * kSobolSteps, kSobolBits)
                                                  : std::vector<uint32_t>();
  std::atomic<uint64_t> tsteps{0}, tcaps{0};
  std::atomic<int> failed{0};
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t job = 0; job < static_cast<int64_t>(n_sites) * batches; ++job) {
    const uint32_t site = static_cast<uint32_t>(job % n_sites), batch = static_cast<uint32_t>(job / n_sites);
    const uint32_t ctr3 = (batch << 16) | (o->repeat << 3);
    std::vector<Vec3> pos(n, Vec3{sites[3 * site], sites[3 * site + 1], sites[3 * site + 2]});
    std::vector<char> active(n, 1);
    std::vector<double> r(n, 0.0);
    std::vector<double> vu(n, 0.0), vp(n, 0.0);
    uint64_t steps = 0, caps = 0;
    const size_t wbase = (static_cast<size_t>(batch) * n_sites + site) * n;
    std::vector<uint32_t> stepc(n, 0);
    for (int k = 0; k < o->max_steps; ++k) {
      bool any = false;
      for (uint32_t i = 0; i < n; ++i) {
        if (!active[i]) continue;
        const Closest c = closest_point(m, pos[i], std::numeric_limits<double>::infinity(), nullptr);
        if (!std::isfinite(c.distance)) {
          failed = 1;
          active[i] = 0;
          continue;
        }
        r[i] = c.distance;
        if (!(r[i] > o->epsilon)) {
          if (n_ub) vu[i] += source_value(ub, n_ub, c.point);
          if (n_pb) vp[i] += source_value(pb, n_pb, c.point);
          active[i] = 0;
        }
        any = any || active[i];
      }
      if (!any) break;
      std::vector<double> u1(n), u2(n);
      if (method == 1) {
        std::vector<std::pair<uint64_t, uint32_t>> keys(n);
        for (uint32_t i = 0; i < n; ++i) {
          uint32_t key = 0xffffffffu;
          if (active[i]) {
            uint32_t q[3];
            for (int a = 0; a < 3; ++a) {
              const double f = (coord(pos[i], a) - bbox_lo[a]) * (1.0 / std::max(bbox_hi[a] - bbox_lo[a], 1e-300)) *
                               1024.0;
              q[a] = static_cast<uint32_t>(std::min(std::max(f, 0.0), 1023.0));
            }
            key = oracle_hilbert3(q[0], q[1], q[2]);
          }
          keys[i] = {(static_cast<uint64_t>(key) << 32) | i, i};
        }
        std::sort(keys.begin(), keys.end());
        uint32_t sh[4];
        Philox::block(k0, k1, static_cast<uint32_t>(k), 0xffffffffu, site, ctr3 | 6u, sh);
        const double U1 = u53(sh[0], sh[1]), U2 = u53(sh[2], sh[3]);
        for (uint32_t rank = 0; rank < n; ++rank) {
          const uint32_t i = keys[rank].second;
          // Korobov point (i/n, a i/n, a^2 i/n): the rank orders, the rest step.
          const uint64_t g2 = (static_cast<uint64_t>(generator) * generator) % n;
          double a1 = static_cast<double>((static_cast<uint64_t>(generator) * rank) % n) / n + U1;
          double a2 = static_cast<double>((g2 * rank) % n) / n + U2;
          u1[i] = a1 - std::floor(a1);
          u2[i] = a2 - std::floor(a2);
        }
      } else if (method == 3 && static_cast<uint32_t>(k) < kSobolSteps) {
        uint32_t rows[2][32], shift[2], dir[2][kSobolBits];
        for (uint32_t w = 0; w < 66; ++w) {
          uint32_t q[4];
          Philox::block(k0, k1, static_cast<uint32_t>(k), w, site, ctr3 | 5u, q);
          if (w < 64) {
            // Row r of the lower-triangular digit matrix: digits 0..r, digit r set.
            const uint32_t r = w % 32;
            uint32_t row = 0;
            for (uint32_t j = 0; j <= r; ++j)
              if (j == r || ((q[0] >> (31 - j)) & 1u)) row |= 1u << (31 - j);
            rows[w / 32][r] = row;
          } else {
            shift[w - 64] = q[0];
          }
        }
        for (int c = 0; c < 2; ++c)
          for (uint32_t b = 0; b < sobol_bits; ++b) {
            const uint32_t v = sobol[(2 * static_cast<size_t>(k) + c) * kSobolBits + b];
            uint32_t x = 0;
            for (uint32_t r = 0; r < 32; ++r) {
              uint32_t parity = 0;
              for (uint32_t j = 0; j < 32; ++j) parity ^= ((rows[c][r] & v) >> j) & 1u;
              x |= parity << (31 - r);
            }
            dir[c][b] = x;
          }
        for (uint32_t i = 0; i < n; ++i) {
          uint32_t x1 = shift[0], x2 = shift[1];
          for (uint32_t b = 0; b < sobol_bits; ++b)
            if ((i >> b) & 1u) {
              x1 ^= dir[0][b];
              x2 ^= dir[1][b];
            }
          u1[i] = (static_cast<double>(x1) + 0.5) / 4294967296.0;
          u2[i] = (static_cast<double>(x2) + 0.5) / 4294967296.0;
        }
      } else {
        for (uint32_t i = 0; i < n; ++i) {
          uint32_t q[4];
          Philox::block(k0, k1, static_cast<uint32_t>(k), i, site, ctr3, q);
          u1[i] = u53(q[0], q[1]);
          u2[i] = u53(q[2], q[3]);
        }
      }
      for (uint32_t i = 0; i < n; ++i) {
        if (!active[i]) continue;
        if (o->n_source) vu[i] += r[i] * r[i] / 6.0 * source_value(o->source, o->n_source, pos[i]);
        pos[i] = pos[i] + direction_from(u1[i], u2[i]) * r[i];
        if (k == 0 && walk_first) {
          walk_first[3 * (wbase + i)] = pos[i].x;
          walk_first[3 * (wbase + i) + 1] = pos[i].y;
          walk_first[3 * (wbase + i) + 2] = pos[i].z;
        }
        if (k == 0 && site_radius && batch == 0 && i == 0) site_radius[site] = r[i];
        ++stepc[i];
        if (static_cast<int>(stepc[i]) >= o->max_steps) {
          active[i] = 0;
          ++caps;
        }
      }
    }
    double su = 0.0, sp = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
      steps += stepc[i];
      su += vu[i];
      sp += vp[i];
      if (walk_u) walk_u[wbase + i] = vu[i];
      if (walk_p) walk_p[wbase + i] = vp[i];
    }
    batch_u[static_cast<size_t>(batch) * n_sites + site] = su / n;
    batch_p[static_cast<size_t>(batch) * n_sites + site] = sp / n;
    tsteps += steps;
    tcaps += caps;
  }
  totals[0] = tsteps;
  totals[1] = tcaps;
  if (failed) {
    g_error = "closest-point query failed";
    return 1;
  }
  return 0;
}

// reused_means (sampling.py:76-88) in 3D over the record of oracle_rqmc:
// site x pools the walks started at every site y with a = |x - y| / r_y <
// 1 - 1e-12, walk j weighted by the Poisson kernel ratio of B(y, r_y),
// r_y (r_y^2 - |x - y|^2) / |x - z_j|^3, site y by (1 - a)^4 / (1 + a)^2.
// A site with no such y keeps its plain mean (batch_u/batch_p in, out).
void oracle_neighbour_means(const double *sites, uint32_t n_sites, uint32_t batches, uint32_t walks,
                            const double *walk_first, const double *walk_u, const double *walk_p,
                            const double *site_radius, double *batch_u, double *batch_p) {
  for (uint32_t b = 0; b < batches; ++b)
    for (uint32_t x = 0; x < n_sites; ++x) {
      const Vec3 X{sites[3 * x], sites[3 * x + 1], sites[3 * x + 2]};
      double wsum = 0.0, su = 0.0, sp = 0.0;
      for (uint32_t y = 0; y < n_sites; ++y) {
        const double ry = site_radius[y];
        const Vec3 Y{sites[3 * y], sites[3 * y + 1], sites[3 * y + 2]};
        const double rho2 = dot(X - Y, X - Y);
        const double a = std::sqrt(rho2) / ry;
        if (!(a < 1.0 - 1e-12)) continue;
        const double w = std::pow(1.0 - a, 4) / ((1.0 + a) * (1.0 + a));
        double mu = 0.0, mp = 0.0;
        const size_t base = (static_cast<size_t>(b) * n_sites + y) * walks;
        for (uint32_t j = 0; j < walks; ++j) {
          const Vec3 Z{walk_first[3 * (base + j)], walk_first[3 * (base + j) + 1], walk_first[3 * (base + j) + 2]};
          const double d = std::sqrt(dot(X - Z, X - Z));
          const double K = ry * (ry * ry - rho2) / (d * d * d);
          mu += K * walk_u[base + j];
          mp += K * walk_p[base + j];
        }
        wsum += w;
        su += w * mu / walks;
        sp += w * mp / walks;
      }
      if (wsum > 0.0) {
        batch_u[static_cast<size_t>(b) * n_sites + x] = su / wsum;
        batch_p[static_cast<size_t>(b) * n_sites + x] = sp / wsum;
      }
    }
}

}  // extern "C"

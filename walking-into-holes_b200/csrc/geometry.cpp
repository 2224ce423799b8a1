// Host geometry for libtwos.so: mesh readers, the BVH builder, device layout
// packing and ray-parity membership.
//
// Replaces EmbreeMesh (benchmarks/compiled_bunny/src/wih_twos.cpp:291-506):
// the PLY reader keeps the reference's accept/reject rules and messages
// (437-493), the points reader keeps read_points (508-522), and the BVH
// builder stands in for rtcCommitScene (320-324).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>

#include "twos_internal.h"

namespace twos {

void load_ascii_ply(const std::string &path, std::vector<double> &vertices, std::vector<uint32_t> &faces) {
  std::ifstream input(path);
  if (!input) throw std::runtime_error("cannot open mesh: " + path);
  std::string line;
  size_t vertex_count = 0, face_count = 0;
  bool ascii = false, header_done = false;
  while (std::getline(input, line)) {
    std::istringstream words(line);
    std::string first;
    words >> first;
    if (first == "format") {
      std::string format;
      words >> format;
      ascii = format == "ascii";
    } else if (first == "element") {
      std::string type;
      size_t count = 0;
      words >> type >> count;
      if (type == "vertex") vertex_count = count;
      if (type == "face") face_count = count;
    } else if (first == "end_header") {
      header_done = true;
      break;
    }
  }
  if (!ascii || !header_done || vertex_count == 0 || face_count == 0)
    throw std::runtime_error("expected a nonempty ASCII triangle PLY mesh");
  vertices.resize(3 * vertex_count);
  for (size_t i = 0; i < vertex_count; ++i) {
    if (!(input >> vertices[3 * i] >> vertices[3 * i + 1] >> vertices[3 * i + 2]))
      throw std::runtime_error("truncated PLY vertex section");
    std::getline(input, line);
  }
  faces.resize(3 * face_count);
  for (size_t i = 0; i < face_count; ++i) {
    unsigned count = 0;
    uint64_t a = 0, b = 0, c = 0;
    if (!(input >> count >> a >> b >> c) || count != 3 || a >= vertex_count || b >= vertex_count ||
        c >= vertex_count)
      throw std::runtime_error("expected valid triangular PLY faces");
    faces[3 * i] = static_cast<uint32_t>(a);
    faces[3 * i + 1] = static_cast<uint32_t>(b);
    faces[3 * i + 2] = static_cast<uint32_t>(c);
    std::getline(input, line);
  }
}

std::vector<double> read_points(const std::string &path) {
  std::ifstream input(path);
  if (!input) throw std::runtime_error("cannot open points: " + path);
  std::vector<double> points;
  std::string line;
  while (std::getline(input, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::replace(line.begin(), line.end(), ',', ' ');
    std::istringstream values(line);
    double x, y, z;
    if (values >> x >> y >> z) {
      points.push_back(x);
      points.push_back(y);
      points.push_back(z);
    }
  }
  if (points.empty()) throw std::runtime_error("points file contains no points");
  return points;
}

// ---------------------------------------------------------------- BVH build
namespace {

struct Aabb {
  double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                  std::numeric_limits<double>::infinity()};
  double hi[3] = {-std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
                  -std::numeric_limits<double>::infinity()};
  void grow(const double p[3]) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  void grow(const Aabb &b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  double area() const {
    const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0.0)) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
  }
};

constexpr int kBins = 32;

struct Builder {
  const std::vector<Aabb> &tb;
  const std::vector<std::array<double, 3>> &cent;
  HostBvh &out;
  std::vector<uint32_t> &order;

  // Builds the subtree over order[begin, end) and returns its child code.
  int32_t build(int begin, int end, int depth, Aabb &box_out) {
    Aabb box, cbox;
    for (int i = begin; i < end; ++i) {
      box.grow(tb[order[i]]);
      cbox.grow(cent[order[i]].data());
    }
    box_out = box;
    const int n = end - begin;
    out.depth = std::max(out.depth, depth);
    if (n <= kLeafMax) return ~static_cast<int32_t>((static_cast<uint32_t>(begin) << 3) | static_cast<uint32_t>(n));
    // Depth budget: a subtree at `depth` may use at most kMaxDepth - depth
    // more levels, so split by the median once SAH could overrun it.
    const int budget = kMaxDepth - depth;
    const bool force_median = budget < 31 && (static_cast<double>(n) > kLeafMax * std::ldexp(1.0, budget - 1));
    int mid = begin + n / 2;
    int best_axis = -1, best_split = -1;
    if (!force_median) {
      double best_cost = std::numeric_limits<double>::infinity();
      for (int axis = 0; axis < 3; ++axis) {
        const double lo = cbox.lo[axis], hi = cbox.hi[axis];
        if (!(hi > lo)) continue;
        std::array<Aabb, kBins> bins;
        std::array<int, kBins> counts{};
        const double scale = kBins / (hi - lo);
        for (int i = begin; i < end; ++i) {
          int k = static_cast<int>((cent[order[i]][axis] - lo) * scale);
          k = std::min(std::max(k, 0), kBins - 1);
          bins[k].grow(tb[order[i]]);
          ++counts[k];
        }
        std::array<double, kBins> right_area{};
        std::array<int, kBins> right_count{};
        Aabb acc;
        int cnt = 0;
        for (int k = kBins - 1; k > 0; --k) {
          acc.grow(bins[k]);
          cnt += counts[k];
          right_area[k] = acc.area();
          right_count[k] = cnt;
        }
        Aabb lacc;
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
    }
    if (best_axis >= 0) {
      const double lo = cbox.lo[best_axis], hi = cbox.hi[best_axis];
      const double scale = kBins / (hi - lo);
      auto it = std::partition(order.begin() + begin, order.begin() + end, [&](uint32_t t) {
        int k = static_cast<int>((cent[t][best_axis] - lo) * scale);
        k = std::min(std::max(k, 0), kBins - 1);
        return k <= best_split;
      });
      mid = static_cast<int>(it - order.begin());
      if (mid == begin || mid == end) best_axis = -1;
    }
    if (best_axis < 0) {
      // Median split on the longest centroid axis.
      int axis = 0;
      for (int a = 1; a < 3; ++a)
        if (cbox.hi[a] - cbox.lo[a] > cbox.hi[axis] - cbox.lo[axis]) axis = a;
      mid = begin + n / 2;
      std::nth_element(order.begin() + begin, order.begin() + mid, order.begin() + end,
                       [&](uint32_t a, uint32_t b) { return cent[a][axis] < cent[b][axis]; });
    }
    const int index = static_cast<int>(out.nodes.size());
    out.nodes.emplace_back();
    Aabb lb, rb;
    const int32_t l = build(begin, mid, depth + 1, lb);
    const int32_t r = build(mid, end, depth + 1, rb);
    HostBvh::Node &node = out.nodes[index];
    for (int a = 0; a < 3; ++a) {
      node.lo[0][a] = lb.lo[a];
      node.hi[0][a] = lb.hi[a];
      node.lo[1][a] = rb.lo[a];
      node.hi[1][a] = rb.hi[a];
    }
    node.child[0] = l;
    node.child[1] = r;
    return index;
  }
};

}  // namespace

void build_bvh(const std::vector<double> &v, const std::vector<uint32_t> &f, HostBvh &out) {
  const size_t nf = f.size() / 3;
  if (nf == 0) throw std::runtime_error("empty mesh");
  if (nf >= (1u << 28)) throw std::runtime_error("mesh too large (>= 2^28 triangles)");
  std::vector<Aabb> tb(nf);
  std::vector<std::array<double, 3>> cent(nf);
  for (size_t i = 0; i < nf; ++i) {
    Aabb b;
    for (int k = 0; k < 3; ++k) b.grow(&v[3 * static_cast<size_t>(f[3 * i + k])]);
    tb[i] = b;
    for (int a = 0; a < 3; ++a) cent[i][a] = 0.5 * (b.lo[a] + b.hi[a]);
  }
  out.nodes.clear();
  out.nodes.reserve(nf);
  out.order.resize(nf);
  std::iota(out.order.begin(), out.order.end(), 0u);
  out.depth = 0;
  Builder b{tb, cent, out, out.order};
  if (nf <= static_cast<size_t>(kLeafMax)) {
    // Single leaf: a root with the leaf on the left and an empty right child.
    Aabb box;
    for (size_t i = 0; i < nf; ++i) box.grow(tb[i]);
    HostBvh::Node root{};
    for (int a = 0; a < 3; ++a) {
      root.lo[0][a] = box.lo[a];
      root.hi[0][a] = box.hi[a];
      root.lo[1][a] = std::numeric_limits<double>::infinity();
      root.hi[1][a] = -std::numeric_limits<double>::infinity();
    }
    root.child[0] = ~static_cast<int32_t>(nf);
    root.child[1] = ~static_cast<int32_t>(0);
    out.nodes.push_back(root);
    out.depth = 1;
    return;
  }
  Aabb rootbox;
  const int32_t root = b.build(0, static_cast<int>(nf), 0, rootbox);
  if (root != 0) throw std::runtime_error("BVH root is not node 0");
  if (out.depth > kMaxDepth) throw std::runtime_error("BVH depth bound exceeded");
}

void pack_bvh_f32(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                  const double center[3], std::vector<NodeF> &nodes, std::vector<TriF> &tris) {
  const size_t nf = bvh.order.size();
  tris.resize(nf);
  std::vector<float> tri_lo(3 * nf), tri_hi(3 * nf);
  for (size_t i = 0; i < nf; ++i) {
    const uint32_t t = bvh.order[i];
    float p[3][3];
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a)
        p[k][a] = static_cast<float>(v[3 * static_cast<size_t>(f[3 * t + k]) + a] - center[a]);
    uint32_t id = t;
    float idf;
    std::memcpy(&idf, &id, 4);
    tris[i].a = make_float4(p[0][0], p[0][1], p[0][2], idf);
    tris[i].b = make_float4(p[1][0], p[1][1], p[1][2], 0.f);
    tris[i].c = make_float4(p[2][0], p[2][1], p[2][2], 0.f);
    for (int a = 0; a < 3; ++a) {
      tri_lo[3 * i + a] = std::min({p[0][a], p[1][a], p[2][a]});
      tri_hi[3 * i + a] = std::max({p[0][a], p[1][a], p[2][a]});
    }
  }
  // Child boxes recomputed from the FP32 triangles (exact min/max).
  nodes.resize(bvh.nodes.size());
  struct Box3 {
    float lo[3], hi[3];
  };
  std::vector<Box3> nodebox(bvh.nodes.size());
  auto leafbox = [&](int32_t code) {
    Box3 b;
    for (int a = 0; a < 3; ++a) {
      b.lo[a] = std::numeric_limits<float>::infinity();
      b.hi[a] = -std::numeric_limits<float>::infinity();
    }
    const uint32_t enc = ~static_cast<uint32_t>(code);
    const uint32_t first = enc >> 3, count = enc & 7u;
    for (uint32_t i = first; i < first + count; ++i)
      for (int a = 0; a < 3; ++a) {
        b.lo[a] = std::min(b.lo[a], tri_lo[3 * i + a]);
        b.hi[a] = std::max(b.hi[a], tri_hi[3 * i + a]);
      }
    return b;
  };
  // Children always have larger indices than parents: fill bottom-up.
  for (size_t ni = bvh.nodes.size(); ni-- > 0;) {
    const HostBvh::Node &n = bvh.nodes[ni];
    Box3 cb[2];
    for (int c = 0; c < 2; ++c) cb[c] = n.child[c] < 0 ? leafbox(n.child[c]) : nodebox[n.child[c]];
    Box3 all;
    for (int a = 0; a < 3; ++a) {
      all.lo[a] = std::min(cb[0].lo[a], cb[1].lo[a]);
      all.hi[a] = std::max(cb[0].hi[a], cb[1].hi[a]);
    }
    nodebox[ni] = all;
    NodeF &o = nodes[ni];
    o.x = make_float4(cb[0].lo[0], cb[1].lo[0], cb[0].hi[0], cb[1].hi[0]);
    o.y = make_float4(cb[0].lo[1], cb[1].lo[1], cb[0].hi[1], cb[1].hi[1]);
    o.z = make_float4(cb[0].lo[2], cb[1].lo[2], cb[0].hi[2], cb[1].hi[2]);
    o.child = make_int4(n.child[0], n.child[1], 0, 0);
  }
}

void pack_bvh_f64(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                  std::vector<NodeD> &nodes, std::vector<TriD> &tris) {
  const size_t nf = bvh.order.size();
  tris.resize(nf);
  for (size_t i = 0; i < nf; ++i) {
    const uint32_t t = bvh.order[i];
    const double *a = &v[3 * static_cast<size_t>(f[3 * t])];
    const double *b = &v[3 * static_cast<size_t>(f[3 * t + 1])];
    const double *c = &v[3 * static_cast<size_t>(f[3 * t + 2])];
    TriD &o = tris[i];
    o.axy = make_double2(a[0], a[1]);
    o.azbx = make_double2(a[2], b[0]);
    o.bybz = make_double2(b[1], b[2]);
    o.cxy = make_double2(c[0], c[1]);
    o.czid = make_double2(c[2], static_cast<double>(t));
    o.pad = make_double2(0.0, 0.0);
  }
  nodes.resize(bvh.nodes.size());
  for (size_t ni = 0; ni < bvh.nodes.size(); ++ni) {
    const HostBvh::Node &n = bvh.nodes[ni];
    NodeD &o = nodes[ni];
    o.xlo = make_double2(n.lo[0][0], n.lo[1][0]);
    o.xhi = make_double2(n.hi[0][0], n.hi[1][0]);
    o.ylo = make_double2(n.lo[0][1], n.lo[1][1]);
    o.yhi = make_double2(n.hi[0][1], n.hi[1][1]);
    o.zlo = make_double2(n.lo[0][2], n.lo[1][2]);
    o.zhi = make_double2(n.hi[0][2], n.hi[1][2]);
    o.child = make_int4(n.child[0], n.child[1], 0, 0);
    o.pad = make_int4(0, 0, 0, 0);
  }
}

// ---------------------------------------------------------------- ray parity
namespace {

// Moller-Trumbore ray/triangle intersection (FP64); returns t or -1.
double ray_triangle(const double o[3], const double d[3], const double *a, const double *b, const double *c) {
  const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
  if (det == 0.0) return -1.0;
  const double inv = 1.0 / det;
  const double tv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
  const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
  if (u < 0.0 || u > 1.0) return -1.0;
  const double qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
  const double w = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
  if (w < 0.0 || u + w > 1.0) return -1.0;
  return (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
}

bool ray_box(const double o[3], const double inv[3], const double lo[3], const double hi[3], double tmin,
             double tmax) {
  for (int a = 0; a < 3; ++a) {
    double t0 = (lo[a] - o[a]) * inv[a], t1 = (hi[a] - o[a]) * inv[a];
    if (t0 > t1) std::swap(t0, t1);
    tmin = std::max(tmin, t0);
    tmax = std::min(tmax, t1);
    if (tmin > tmax) return false;
  }
  return true;
}

}  // namespace

int inside_parity(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                  const double p[3], bool &inside, std::string &err) {
  // The reference's fixed oblique ray (wih_twos.cpp:362-363), re-shot from
  // each hit at t_hit + 2e-6 with tnear 1e-6 and tfar 4, at most 128 hits.
  double dir[3] = {1.0, 0.3713906763541037, 0.1570796326794897};
  const double len = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  for (double &d : dir) d *= 1.0 / len;
  const double inv[3] = {1.0 / dir[0], 1.0 / dir[1], 1.0 / dir[2]};
  double origin[3] = {p[0], p[1], p[2]};
  unsigned hits = 0;
  for (; hits < 128; ++hits) {
    const double tnear = 1.0e-6, tfar = 4.0;
    double best = tfar;
    bool found = false;
    int32_t stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int32_t code = stack[--sp];
      if (code < 0) {
        const uint32_t enc = ~static_cast<uint32_t>(code);
        for (uint32_t i = enc >> 3, e = (enc >> 3) + (enc & 7u); i < e; ++i) {
          const uint32_t t = bvh.order[i];
          const double th = ray_triangle(origin, dir, &v[3 * static_cast<size_t>(f[3 * t])],
                                         &v[3 * static_cast<size_t>(f[3 * t + 1])],
                                         &v[3 * static_cast<size_t>(f[3 * t + 2])]);
          if (th >= tnear && th <= best) {
            best = th;
            found = true;
          }
        }
        continue;
      }
      const HostBvh::Node &n = bvh.nodes[code];
      for (int c = 0; c < 2; ++c) {
        if (ray_box(origin, inv, n.lo[c], n.hi[c], tnear, best)) {
          if (sp >= 64) {
            err = "ray traversal stack overflow";
            return 1;
          }
          stack[sp++] = n.child[c];
        }
      }
    }
    if (!found) break;
    for (int a = 0; a < 3; ++a) origin[a] = origin[a] + dir[a] * (best + 2.0e-6);
  }
  if (hits == 128) {
    err = "ray-parity traversal exceeded 128 intersections";
    return 1;
  }
  inside = (hits % 2u) == 1u;
  return 0;
}

}  // namespace twos

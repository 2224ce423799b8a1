// Host geometry for libtwos.so: mesh readers, the BVH builder, device layout
// packing and ray-parity membership.
//
// Replaces EmbreeMesh (benchmarks/compiled_bunny/src/wih_twos.cpp:291-506):
// the PLY reader keeps the reference's accept/reject rules and messages
// (437-493), the points reader keeps read_points (508-522), and the BVH
// builder stands in for rtcCommitScene (320-324).
#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "twos_internal.h"

namespace twos {

namespace {

// What the header of a PLY file declares, as far as the reader needs it:
// the format keyword and the last vertex and face element counts.
struct PlyHeader {
  bool ascii = false;
  bool complete = false;  // "end_header" seen
  size_t vertex_count = 0;
  size_t face_count = 0;
};

PlyHeader read_ply_header(std::istream &in) {
  PlyHeader h;
  for (std::string line; !h.complete && std::getline(in, line);) {
    std::istringstream tokens(line);
    std::string keyword;
    tokens >> keyword;
    if (keyword == "end_header") {
      h.complete = true;
    } else if (keyword == "format") {
      std::string kind;
      tokens >> kind;
      h.ascii = kind == "ascii";
    } else if (keyword == "element") {
      std::string name;
      size_t n = 0;
      tokens >> name >> n;
      if (name == "vertex") h.vertex_count = n;
      else if (name == "face") h.face_count = n;
    }
  }
  return h;
}

// Drops whatever follows the values just read on the current line (extra
// properties of a vertex or face row).
void skip_rest_of_line(std::istream &in) { in.ignore(std::numeric_limits<std::streamsize>::max(), '\n'); }

}  // namespace

// The reference's reader rules (wih_twos.cpp:437-493): an ASCII header with
// nonzero vertex and face counts; each vertex row starts with x y z; each
// face row is "3 a b c" with indices below the vertex count; anything else
// is an error with the reference's message.
void load_ascii_ply(const std::string &path, std::vector<double> &vertices, std::vector<uint32_t> &faces) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open mesh: " + path);
  const PlyHeader h = read_ply_header(in);
  if (!h.ascii || !h.complete || h.vertex_count == 0 || h.face_count == 0)
    throw std::runtime_error("expected a nonempty ASCII triangle PLY mesh");
  vertices.assign(3 * h.vertex_count, 0.0);
  for (double *v = vertices.data(), *end = v + vertices.size(); v != end; v += 3) {
    if (!(in >> v[0] >> v[1] >> v[2])) throw std::runtime_error("truncated PLY vertex section");
    skip_rest_of_line(in);
  }
  faces.assign(3 * h.face_count, 0u);
  for (uint32_t *f = faces.data(), *end = f + faces.size(); f != end; f += 3) {
    unsigned corners = 0;
    uint64_t idx[3] = {0, 0, 0};
    const bool parsed = static_cast<bool>(in >> corners >> idx[0] >> idx[1] >> idx[2]);
    if (!parsed || corners != 3 || std::max({idx[0], idx[1], idx[2]}) >= h.vertex_count)
      throw std::runtime_error("expected valid triangular PLY faces");
    for (int k = 0; k < 3; ++k) f[k] = static_cast<uint32_t>(idx[k]);
    skip_rest_of_line(in);
  }
}

// Points file rules of wih_twos.cpp:508-522: blank lines and lines starting
// with '#' are skipped, commas count as spaces, a line contributes a point
// when it starts with three numbers, and a file without points is an error.
std::vector<double> read_points(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open points: " + path);
  std::vector<double> xyz;
  for (std::string line; std::getline(in, line);) {
    if (line.empty() || line.front() == '#') continue;
    for (char &ch : line)
      if (ch == ',') ch = ' ';
    std::istringstream row(line);
    double p[3];
    if (row >> p[0] >> p[1] >> p[2]) xyz.insert(xyz.end(), p, p + 3);
  }
  if (xyz.empty()) throw std::runtime_error("points file contains no points");
  return xyz;
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
  if (nf > (static_cast<size_t>(kLeafMax) << kMaxDepth)) throw std::runtime_error("mesh too large (> 4 * 2^24 triangles)");
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

namespace {

float round_down(double x) {
  float f = static_cast<float>(x);
  if (static_cast<double>(f) > x) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
  return f;
}
float round_up(double x) {
  float f = static_cast<float>(x);
  if (static_cast<double>(f) < x) f = std::nextafter(f, std::numeric_limits<float>::infinity());
  return f;
}

struct Range {
  uint32_t begin = 0, end = 0;
};

Range code_range(int32_t code, const std::vector<Range> &node_range) {
  if (code >= 0) return node_range[code];
  const uint32_t enc = ~static_cast<uint32_t>(code);
  return {enc >> 3, (enc >> 3) + (enc & 7u)};
}

// Leaf-order ranges of every node (children always follow their parent).
std::vector<Range> node_ranges(const HostBvh &bvh) {
  std::vector<Range> r(bvh.nodes.size());
  for (size_t ni = bvh.nodes.size(); ni-- > 0;) {
    const Range a = code_range(bvh.nodes[ni].child[0], r), b = code_range(bvh.nodes[ni].child[1], r);
    if (a.end == a.begin) {
      r[ni] = b;
    } else if (b.end == b.begin) {
      r[ni] = a;
    } else {
      r[ni] = {std::min(a.begin, b.begin), std::max(a.end, b.end)};
    }
  }
  return r;
}

// Vertex coordinates of leaf-order triangle i in a frame (the FP32 layout
// passes the rounded FP32 coordinates, the FP64 layout the originals).
struct TriCoords {
  std::vector<double> xyz;  // 9 per triangle
  const double *tri(uint32_t i) const { return &xyz[9 * static_cast<size_t>(i)]; }
};

void cross(const double *a, const double *b, const double *c, double out[3]) {
  const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  out[0] = e1[1] * e2[2] - e1[2] * e2[1];
  out[1] = e1[2] * e2[0] - e1[0] * e2[2];
  out[2] = e1[0] * e2[1] - e1[1] * e2[0];
}

// Unit mean normal of a triangle range and the interval of n.v over its
// vertices.  `nq` receives the direction as the kernel stores it (FP32-rounded
// for the FP32 layout), and the interval is computed with that direction.
// Returns false (no slab) when the normals cancel.
bool range_slab(const TriCoords &tc, Range r, bool fp32, double nq[3], double &smin, double &smax) {
  double N[3] = {0, 0, 0}, total = 0.0;
  for (uint32_t i = r.begin; i < r.end; ++i) {
    const double *t = tc.tri(i);
    double c[3];
    cross(t, t + 3, t + 6, c);
    N[0] += c[0];
    N[1] += c[1];
    N[2] += c[2];
    total += std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  }
  const double len = std::sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
  if (!(len > 1e-3 * total) || !(len > 0.0)) return false;
  for (int k = 0; k < 3; ++k) {
    nq[k] = N[k] / len;
    if (fp32) nq[k] = static_cast<double>(static_cast<float>(nq[k]));
  }
  smin = std::numeric_limits<double>::infinity();
  smax = -std::numeric_limits<double>::infinity();
  double mag = 0.0;
  for (uint32_t i = r.begin; i < r.end; ++i) {
    const double *t = tc.tri(i);
    for (int v = 0; v < 3; ++v) {
      const double *x = t + 3 * v;
      const double s = nq[0] * x[0] + nq[1] * x[1] + nq[2] * x[2];
      smin = std::min(smin, s);
      smax = std::max(smax, s);
      mag = std::max(mag, std::fabs(nq[0] * x[0]) + std::fabs(nq[1] * x[1]) + std::fabs(nq[2] * x[2]));
    }
  }
  // Rounding of the three-term dot products above (and in the FP64 kernel).
  const double pad = 8.0 * std::ldexp(1.0, -52) * mag;
  smin -= pad;
  smax += pad;
  return true;
}

TriCoords leaf_coords(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                      const double *center, bool fp32) {
  const size_t nf = bvh.order.size();
  TriCoords tc;
  tc.xyz.resize(9 * nf);
  for (size_t i = 0; i < nf; ++i) {
    const uint32_t t = bvh.order[i];
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) {
        const double x = v[3 * static_cast<size_t>(f[3 * t + k]) + a];
        tc.xyz[9 * i + 3 * k + a] =
            fp32 ? static_cast<double>(static_cast<float>(x - center[a])) : x;
      }
  }
  return tc;
}

}  // namespace

void pack_bvh_f32(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                  const double center[3], std::vector<NodeF> &nodes, std::vector<TriF> &tris) {
  const size_t nf = bvh.order.size();
  const TriCoords tc = leaf_coords(bvh, v, f, center, true);
  tris.resize(nf);
  std::vector<float> tri_lo(3 * nf), tri_hi(3 * nf);
  for (size_t i = 0; i < nf; ++i) {
    const double *t = tc.tri(static_cast<uint32_t>(i));
    float p[3][3];
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) p[k][a] = static_cast<float>(t[3 * k + a]);
    double c[3];
    cross(t, t + 3, t + 6, c);
    const double len = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    float n[3] = {0.f, 0.f, 0.f};
    float dmin = 0.f, dmax = 0.f;
    if (len > 0.0) {
      for (int a = 0; a < 3; ++a) n[a] = static_cast<float>(c[a] / len);
      double lo = std::numeric_limits<double>::infinity(), hi = -lo, mag = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double s = static_cast<double>(n[0]) * t[3 * k] + static_cast<double>(n[1]) * t[3 * k + 1] +
                         static_cast<double>(n[2]) * t[3 * k + 2];
        lo = std::min(lo, s);
        hi = std::max(hi, s);
        mag = std::max(mag, std::fabs(n[0] * t[3 * k]) + std::fabs(n[1] * t[3 * k + 1]) +
                                std::fabs(n[2] * t[3 * k + 2]));
      }
      const double pad = 8.0 * std::ldexp(1.0, -52) * mag;
      dmin = round_down(lo - pad);
      dmax = round_up(hi + pad);
    }
    uint32_t id = bvh.order[i];
    float idf;
    std::memcpy(&idf, &id, 4);
    tris[i].plane = make_float4(n[0], n[1], n[2], dmin);
    tris[i].a = make_float4(p[0][0], p[0][1], p[0][2], dmax);
    tris[i].b = make_float4(p[1][0], p[1][1], p[1][2], idf);
    tris[i].c = make_float4(p[2][0], p[2][1], p[2][2], 0.f);
    for (int a = 0; a < 3; ++a) {
      tri_lo[3 * i + a] = std::min({p[0][a], p[1][a], p[2][a]});
      tri_hi[3 * i + a] = std::max({p[0][a], p[1][a], p[2][a]});
    }
  }
  const std::vector<Range> ranges = node_ranges(bvh);
  nodes.resize(bvh.nodes.size());
  for (size_t ni = 0; ni < bvh.nodes.size(); ++ni) {
    const HostBvh::Node &hn = bvh.nodes[ni];
    float lo[2][3], hi[2][3], nv[2][3], smin[2], smax[2];
    for (int c = 0; c < 2; ++c) {
      const Range r = code_range(hn.child[c], ranges);
      for (int a = 0; a < 3; ++a) {
        lo[c][a] = std::numeric_limits<float>::infinity();
        hi[c][a] = -std::numeric_limits<float>::infinity();
      }
      for (uint32_t i = r.begin; i < r.end; ++i)
        for (int a = 0; a < 3; ++a) {
          lo[c][a] = std::min(lo[c][a], tri_lo[3 * i + a]);
          hi[c][a] = std::max(hi[c][a], tri_hi[3 * i + a]);
        }
      double nq[3], s0, s1;
      if (r.end > r.begin && range_slab(tc, r, true, nq, s0, s1)) {
        for (int a = 0; a < 3; ++a) nv[c][a] = static_cast<float>(nq[a]);
        smin[c] = round_down(s0);
        smax[c] = round_up(s1);
      } else {
        nv[c][0] = nv[c][1] = nv[c][2] = 0.f;
        smin[c] = smax[c] = 0.f;
      }
    }
    NodeF &o = nodes[ni];
    o.x = make_float4(lo[0][0], lo[1][0], hi[0][0], hi[1][0]);
    o.y = make_float4(lo[0][1], lo[1][1], hi[0][1], hi[1][1]);
    o.z = make_float4(lo[0][2], lo[1][2], hi[0][2], hi[1][2]);
    o.nl = make_float4(nv[0][0], nv[0][1], nv[0][2], smin[0]);
    o.nr = make_float4(nv[1][0], nv[1][1], nv[1][2], smin[1]);
    float cl, cr;
    std::memcpy(&cl, &hn.child[0], 4);
    std::memcpy(&cr, &hn.child[1], 4);
    o.tail = make_float4(smax[0], smax[1], cl, cr);
  }
}

void pack_bvh_f64(const HostBvh &bvh, const std::vector<double> &v, const std::vector<uint32_t> &f,
                  std::vector<NodeD> &nodes, std::vector<TriD> &tris) {
  const size_t nf = bvh.order.size();
  const double zero[3] = {0.0, 0.0, 0.0};
  const TriCoords tc = leaf_coords(bvh, v, f, zero, false);
  tris.resize(nf);
  for (size_t i = 0; i < nf; ++i) {
    const double *t = tc.tri(static_cast<uint32_t>(i));
    double c[3];
    cross(t, t + 3, t + 6, c);
    const double len = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    double n[3] = {0.0, 0.0, 0.0}, dmin = 0.0, dmax = 0.0;
    if (len > 0.0) {
      for (int a = 0; a < 3; ++a) n[a] = c[a] / len;
      double lo = std::numeric_limits<double>::infinity(), hi = -lo, mag = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double s = n[0] * t[3 * k] + n[1] * t[3 * k + 1] + n[2] * t[3 * k + 2];
        lo = std::min(lo, s);
        hi = std::max(hi, s);
        mag = std::max(mag, std::fabs(n[0] * t[3 * k]) + std::fabs(n[1] * t[3 * k + 1]) +
                                std::fabs(n[2] * t[3 * k + 2]));
      }
      const double pad = 8.0 * std::ldexp(1.0, -52) * mag;
      dmin = lo - pad;
      dmax = hi + pad;
    }
    TriD &o = tris[i];
    o.nxy = make_double2(n[0], n[1]);
    o.nzmin = make_double2(n[2], dmin);
    o.dmax_id = make_double2(dmax, static_cast<double>(bvh.order[i]));
    o.axy = make_double2(t[0], t[1]);
    o.azbx = make_double2(t[2], t[3]);
    o.bybz = make_double2(t[4], t[5]);
    o.cxy = make_double2(t[6], t[7]);
    o.czpad = make_double2(t[8], 0.0);
  }
  const std::vector<Range> ranges = node_ranges(bvh);
  nodes.resize(bvh.nodes.size());
  for (size_t ni = 0; ni < bvh.nodes.size(); ++ni) {
    const HostBvh::Node &n = bvh.nodes[ni];
    double nv[2][3], smin[2], smax[2];
    for (int c = 0; c < 2; ++c) {
      const Range r = code_range(n.child[c], ranges);
      if (!(r.end > r.begin && range_slab(tc, r, false, nv[c], smin[c], smax[c]))) {
        nv[c][0] = nv[c][1] = nv[c][2] = 0.0;
        smin[c] = smax[c] = 0.0;
      }
    }
    NodeD &o = nodes[ni];
    o.xlo = make_double2(n.lo[0][0], n.lo[1][0]);
    o.xhi = make_double2(n.hi[0][0], n.hi[1][0]);
    o.ylo = make_double2(n.lo[0][1], n.lo[1][1]);
    o.yhi = make_double2(n.hi[0][1], n.hi[1][1]);
    o.zlo = make_double2(n.lo[0][2], n.lo[1][2]);
    o.zhi = make_double2(n.hi[0][2], n.hi[1][2]);
    o.nl_xy = make_double2(nv[0][0], nv[0][1]);
    o.nl_zmin = make_double2(nv[0][2], smin[0]);
    o.nr_xy = make_double2(nv[1][0], nv[1][1]);
    o.nr_zmin = make_double2(nv[1][2], smin[1]);
    o.smax = make_double2(smax[0], smax[1]);
    o.child = make_int4(n.child[0], n.child[1], 0, 0);
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


// Entry nodes of the mixed form's query (see twos_internal.h).  Every cell
// collects the leaf-order range [lo, hi] of the leaves whose box lies within
// `radius` of the cell's box grown by `pad` (box-to-box distance, a lower
// bound of every triangle's distance); the cell's entry is the deepest node
// whose subtree covers that range.  Node subtrees cover contiguous
// leaf-order ranges, so the descent from the root keeps the child that
// contains the whole range.
std::vector<int32_t> build_entry_table(const HostBvh &bvh, const double origin[3], double cell, const uint32_t dims[3],
                                       double radius, double pad) {
  const std::vector<Range> ranges = node_ranges(bvh);
  const size_t count = static_cast<size_t>(dims[0]) * dims[1] * dims[2];
  std::vector<int32_t> entry(count, 0);
  if (bvh.nodes.empty() || count == 0) return entry;
  const double r2 = radius * radius;
  auto box_gap2 = [](const double *alo, const double *ahi, const double *blo, const double *bhi) {
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double g = std::max(std::max(alo[a] - bhi[a], blo[a] - ahi[a]), 0.0);
      s += g * g;
    }
    return s;
  };
  // The deepest node under `start` whose subtree holds every leaf whose box
  // lies within `radius` of [lo, hi]; -1 when no leaf does.
  auto lca = [&](int32_t start, const double *lo, const double *hi, std::vector<int32_t> &stack) {
    uint32_t mn = std::numeric_limits<uint32_t>::max(), mx = 0;
    stack.clear();
    stack.push_back(start);
    while (!stack.empty()) {
      const HostBvh::Node &nd = bvh.nodes[static_cast<size_t>(stack.back())];
      stack.pop_back();
      for (int c = 0; c < 2; ++c) {
        if (!(nd.lo[c][0] <= nd.hi[c][0])) continue;  // empty child
        if (box_gap2(lo, hi, nd.lo[c], nd.hi[c]) > r2) continue;
        if (nd.child[c] >= 0) {
          stack.push_back(nd.child[c]);
        } else {
          const Range rg = code_range(nd.child[c], ranges);
          if (rg.end > rg.begin) {
            mn = std::min(mn, rg.begin);
            mx = std::max(mx, rg.end - 1);
          }
        }
      }
    }
    if (mn > mx) return -1;
    int32_t ni = start;
    for (bool deeper = true; deeper;) {
      deeper = false;
      const HostBvh::Node &nd = bvh.nodes[static_cast<size_t>(ni)];
      for (int c = 0; c < 2; ++c) {
        const int32_t code = nd.child[c];
        if (code >= 0 && ranges[code].begin <= mn && mx < ranges[code].end) {
          ni = code;
          deeper = true;
          break;
        }
      }
    }
    return ni;
  };
  // Coarse to fine: a block of kB^3 cells first.  Every leaf within radius
  // of one of its cells is within radius of the block, so a cell's node lies
  // in the block's subtree and its search starts there; a block with no leaf
  // within radius (most of the volume) keeps the root everywhere.
  constexpr uint32_t kB = 8;
  const uint32_t nb[3] = {(dims[0] + kB - 1) / kB, (dims[1] + kB - 1) / kB, (dims[2] + kB - 1) / kB};
  // Threads take (bi, bj) block columns from a shared counter: the blocks
  // near the surface, which carry the work, are unevenly spread.
  std::atomic<uint64_t> next{0};
  const uint64_t columns = static_cast<uint64_t>(nb[0]) * nb[1];
  auto work = [&]() {
    std::vector<int32_t> stack;
    stack.reserve(256);
    for (uint64_t col = next.fetch_add(1); col < columns; col = next.fetch_add(1)) {
      const uint32_t bi = static_cast<uint32_t>(col / nb[1]), bj = static_cast<uint32_t>(col % nb[1]);
      for (uint32_t bk = 0; bk < nb[2]; ++bk) {
        const uint32_t b0[3] = {bi * kB, bj * kB, bk * kB};
        uint32_t b1[3];
        double blo[3], bhi[3];
        for (int a = 0; a < 3; ++a) {
          b1[a] = std::min(b0[a] + kB, dims[a]);
          blo[a] = origin[a] + cell * b0[a] - pad;
          bhi[a] = origin[a] + cell * b1[a] + pad;
        }
        const int32_t start = lca(0, blo, bhi, stack);
        if (start < 0) continue;
        for (uint32_t i = b0[0]; i < b1[0]; ++i)
          for (uint32_t j = b0[1]; j < b1[1]; ++j)
            for (uint32_t k = b0[2]; k < b1[2]; ++k) {
              const uint32_t ijk[3] = {i, j, k};
              double lo[3], hi[3];
              for (int a = 0; a < 3; ++a) {
                lo[a] = origin[a] + cell * ijk[a] - pad;
                hi[a] = origin[a] + cell * (ijk[a] + 1) + pad;
              }
              const int32_t ni = lca(start, lo, hi, stack);
              entry[(static_cast<size_t>(i) * dims[1] + j) * dims[2] + k] = ni < 0 ? 0 : ni;
            }
      }
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t threads = std::min<uint64_t>(hw, columns);
  std::vector<std::thread> pool;
  for (uint64_t t = 0; t < threads; ++t) pool.emplace_back(work);
  for (auto &th : pool) th.join();
  return entry;
}


// Collapse of the packed binary BVH into four-wide nodes: slot boxes, slabs
// and child codes are copied from the binary nodes (so every bound is the
// same conservative FP32 value), internal slot children become four-wide
// nodes in turn.
void pack_bvh4_f32(const HostBvh &bvh, const std::vector<NodeF> &binary, std::vector<Node4F> &nodes4,
                   std::vector<int32_t> &cover) {
  nodes4.clear();
  cover.assign(bvh.nodes.size(), 0);
  if (bvh.nodes.empty()) return;
  struct Slot {
    float lo[3], hi[3], n[3], smin, smax;
    int32_t code;
  };
  auto slot_of = [&](int32_t ni, int c) {
    const NodeF &b = binary[static_cast<size_t>(ni)];
    const float *x = &b.x.x, *y = &b.y.x, *z = &b.z.x;
    const float4 &nv = c == 0 ? b.nl : b.nr;
    Slot s;
    s.lo[0] = x[c];
    s.lo[1] = y[c];
    s.lo[2] = z[c];
    s.hi[0] = x[2 + c];
    s.hi[1] = y[2 + c];
    s.hi[2] = z[2 + c];
    s.n[0] = nv.x;
    s.n[1] = nv.y;
    s.n[2] = nv.z;
    s.smin = nv.w;
    s.smax = c == 0 ? b.tail.x : b.tail.y;
    s.code = bvh.nodes[static_cast<size_t>(ni)].child[c];
    return s;
  };
  // Iterative build: (binary node, four-wide index) pairs still to fill.
  std::vector<std::pair<int32_t, int32_t>> todo{{0, 0}};
  nodes4.emplace_back();
  cover[0] = 0;
  while (!todo.empty()) {
    const auto [ni, qi] = todo.back();
    todo.pop_back();
    Slot slots[4];
    int ns = 0;
    for (int c = 0; c < 2; ++c) {
      const int32_t code = bvh.nodes[static_cast<size_t>(ni)].child[c];
      if (code >= 0) {
        cover[static_cast<size_t>(code)] = qi;  // absorbed into this node
        slots[ns++] = slot_of(code, 0);
        slots[ns++] = slot_of(code, 1);
      } else {
        slots[ns++] = slot_of(ni, c);
      }
    }
    float *f[11];
    Node4F q{};
    float *base = &q.xlo.x;
    for (int k = 0; k < 11; ++k) f[k] = base + 4 * k;
    int32_t child[4];
    for (int k = 0; k < 4; ++k) {
      if (k < ns) {
        const Slot &s = slots[k];
        for (int a = 0; a < 3; ++a) {
          f[2 * a][k] = s.lo[a];
          f[2 * a + 1][k] = s.hi[a];
          f[6 + a][k] = s.n[a];
        }
        f[9][k] = s.smin;
        f[10][k] = s.smax;
        if (s.code >= 0) {
          const int32_t qc = static_cast<int32_t>(nodes4.size());
          nodes4.emplace_back();
          cover[static_cast<size_t>(s.code)] = qc;
          todo.push_back({s.code, qc});
          child[k] = qc;
        } else {
          child[k] = s.code;
        }
      } else {
        for (int a = 0; a < 3; ++a) {
          f[2 * a][k] = std::numeric_limits<float>::infinity();
          f[2 * a + 1][k] = -std::numeric_limits<float>::infinity();
          f[6 + a][k] = 0.f;
        }
        f[9][k] = f[10][k] = 0.f;
        child[k] = ~static_cast<int32_t>(0);
      }
    }
    q.child = make_int4(child[0], child[1], child[2], child[3]);
    nodes4[static_cast<size_t>(qi)] = q;
  }
}


// ---------------------------------------------------------------- Sobol'
namespace {

// Product a b modulo p over GF(2); deg = degree of p, a and b reduced.
uint32_t gf2_mulmod(uint32_t a, uint32_t b, uint32_t p, int deg) {
  uint32_t r = 0;
  while (b) {
    if (b & 1u) r ^= a;
    b >>= 1;
    a <<= 1;
    if ((a >> deg) & 1u) a ^= p;
  }
  return r;
}

uint32_t gf2_powmod(uint32_t a, uint64_t e, uint32_t p, int deg) {
  uint32_t r = 1;
  while (e) {
    if (e & 1u) r = gf2_mulmod(r, a, p, deg);
    a = gf2_mulmod(a, a, p, deg);
    e >>= 1;
  }
  return r;
}

// p (bit i = coefficient of x^i, degree deg >= 2, constant term 1) is
// primitive iff x has multiplicative order exactly 2^deg - 1 modulo p: x to
// that power is 1 and to no quotient by one of its prime factors.
bool gf2_primitive(uint32_t p, int deg) {
  const uint64_t order = (1ull << deg) - 1;
  if (gf2_powmod(2u, order, p, deg) != 1u) return false;
  uint64_t rest = order;
  for (uint64_t q = 3; q * q <= rest; q += 2) {
    if (rest % q) continue;
    while (rest % q == 0) rest /= q;
    if (gf2_powmod(2u, order / q, p, deg) == 1u) return false;
  }
  return rest == 1 || gf2_powmod(2u, order / rest, p, deg) != 1u;
}

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): one output per state.
uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

}  // namespace

std::vector<uint32_t> sobol_directions(uint32_t dims, uint32_t bits) {
  if (bits == 0 || bits > 32) throw std::runtime_error("Sobol direction bits must be 1..32");
  std::vector<uint32_t> polys;  // primitive polynomials, by degree then value
  if (dims > 1) polys.push_back(3u);  // x + 1
  for (int deg = 2; polys.size() + 1 < dims; ++deg) {
    if (deg > 30) throw std::runtime_error("too many Sobol dimensions");
    for (uint32_t p = (1u << deg) | 1u; p < (2u << deg) && polys.size() + 1 < dims; p += 2)
      if (gf2_primitive(p, deg)) polys.push_back(p);
  }
  std::vector<uint32_t> v(static_cast<size_t>(dims) * bits);
  std::vector<uint64_t> m(bits + 1);
  for (uint32_t d = 0; d < dims; ++d) {
    if (d == 0) {
      for (uint32_t k = 1; k <= bits; ++k) m[k] = 1;
    } else {
      const uint32_t p = polys[d - 1];
      int deg = 31;
      while (!((p >> deg) & 1u)) --deg;
      for (uint32_t k = 1; k <= bits; ++k) {
        if (k <= static_cast<uint32_t>(deg)) {
          // Odd initial value below 2^k.
          const uint64_t h = splitmix64(0x536f626f6c2d3344ull + 64ull * d + k);
          m[k] = (h & ((1ull << k) - 1)) | 1ull;
        } else {
          uint64_t x = m[k - deg] ^ (m[k - deg] << deg);
          for (int j = 1; j < deg; ++j)
            if ((p >> (deg - j)) & 1u) x ^= m[k - j] << j;
          m[k] = x;
        }
      }
    }
    for (uint32_t b = 0; b < bits; ++b) v[static_cast<size_t>(d) * bits + b] = static_cast<uint32_t>(m[b + 1] << (31 - b));
  }
  return v;
}

}  // namespace twos

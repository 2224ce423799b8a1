// TEST INFRASTRUCTURE: a project-written stand-in for the part of the Embree 4
// API that the reference's compiled backend calls
// (benchmarks/compiled_bunny/src/wih_twos.cpp:298-359 and 361-394:
// rtcNewDevice ... rtcCommitScene, rtcPointQuery with a user callback,
// rtcIntersect1).  Embree is not installed here; with this header the
// reference's own source compiles unchanged into oracle/_ref/wih_twos, the
// CPU baseline and a second checker.  Only the names and argument meanings of
// Embree's interface are kept (the reference calls them); the implementation
// is this file's own: a binned-SAH binary BVH over the triangles' FP32 boxes.
//
// Semantics kept from Embree's documentation:
// * rtcPointQuery calls the callback for every triangle whose box meets the
//   query sphere (centre x, y, z; radius), nearest subtrees first; when the
//   callback returns true it has shrunk query->radius, and culling continues
//   with the new radius.  The reference's callback computes the exact FP64
//   distance itself, so the result is the nearest triangle whatever the
//   visiting order, except for ties at the FP32 radius.
// * rtcIntersect1 finds the nearest triangle hit with tnear <= t <= tfar,
//   writes t into ray.tfar and sets hit.geomID / hit.primID (or leaves
//   hit.geomID at RTC_INVALID_GEOMETRY_ID).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#define RTC_INVALID_GEOMETRY_ID (static_cast<unsigned int>(-1))
#define RTC_MAX_INSTANCE_LEVEL_COUNT 1

enum RTCError {
  RTC_ERROR_NONE = 0,
  RTC_ERROR_UNKNOWN = 1,
  RTC_ERROR_INVALID_ARGUMENT = 2,
  RTC_ERROR_INVALID_OPERATION = 3,
  RTC_ERROR_OUT_OF_MEMORY = 4,
};
enum RTCGeometryType { RTC_GEOMETRY_TYPE_TRIANGLE = 0 };
enum RTCBufferType { RTC_BUFFER_TYPE_INDEX = 0, RTC_BUFFER_TYPE_VERTEX = 1 };
enum RTCFormat { RTC_FORMAT_UNDEFINED = 0, RTC_FORMAT_UINT3 = 0x5003, RTC_FORMAT_FLOAT3 = 0x9003 };

typedef void (*RTCErrorFunction)(void *userPtr, RTCError code, const char *str);

struct RTCPointQuery {
  float x, y, z;
  float time;
  float radius;
};

struct RTCPointQueryContext {
  unsigned int instStackSize;
  unsigned int instID[RTC_MAX_INSTANCE_LEVEL_COUNT];
};

struct RTCPointQueryFunctionArguments {
  RTCPointQuery *query;
  void *userPtr;
  unsigned int primID;
  unsigned int geomID;
  RTCPointQueryContext *context;
  float similarityScale;
};
typedef bool (*RTCPointQueryFunction)(RTCPointQueryFunctionArguments *args);

struct RTCRay {
  float org_x, org_y, org_z;
  float tnear;
  float dir_x, dir_y, dir_z;
  float time;
  float tfar;
  unsigned int mask;
  unsigned int id;
  unsigned int flags;
};

struct RTCHit {
  float Ng_x, Ng_y, Ng_z;
  float u, v;
  unsigned int primID;
  unsigned int geomID;
  unsigned int instID[RTC_MAX_INSTANCE_LEVEL_COUNT];
};

struct RTCRayHit {
  RTCRay ray;
  RTCHit hit;
};

struct RTCIntersectArguments {
  unsigned int flags;
};

namespace wih_shim {

struct Box {
  float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                 std::numeric_limits<float>::infinity()};
  float hi[3] = {-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
                 -std::numeric_limits<float>::infinity()};
  void grow(const Box &b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  void grow(const float *p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  double area() const {
    const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx < 0 ? 0.0 : 2.0 * (dx * dy + dy * dz + dz * dx);
  }
};

// Both children's boxes in one node; child >= 0 is a node index, child < 0 a
// leaf ~(first << 3 | count) over prims[first, first + count).
struct Node {
  float lo[2][3], hi[2][3];
  int32_t child[2];
};

inline float box_dist2(const float lo[3], const float hi[3], const float p[3]) {
  float s = 0.f;
  for (int a = 0; a < 3; ++a) {
    const float g = std::max(std::max(lo[a] - p[a], p[a] - hi[a]), 0.f);
    s += g * g;
  }
  return s;
}

class Bvh {
 public:
  std::vector<Node> nodes;
  std::vector<uint32_t> prims;
  std::vector<Box> boxes;  // per primitive (original index)

  void build(const std::vector<Box> &prim_boxes) {
    boxes = prim_boxes;
    const size_t n = boxes.size();
    prims.resize(n);
    for (size_t i = 0; i < n; ++i) prims[i] = static_cast<uint32_t>(i);
    cent_.resize(n);
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) cent_[i][a] = 0.5f * (boxes[i].lo[a] + boxes[i].hi[a]);
    nodes.clear();
    nodes.reserve(n / 2 + 2);
    if (n == 0) return;
    Box all;
    for (size_t i = 0; i < n; ++i) all.grow(boxes[i]);
    if (n <= kLeaf) {
      Node root{};
      set_child(root, 0, all, ~static_cast<int32_t>(n));
      Box empty;
      set_child(root, 1, empty, ~static_cast<int32_t>(0));
      nodes.push_back(root);
      return;
    }
    build_node(0, static_cast<uint32_t>(n));
    cent_.clear();
    cent_.shrink_to_fit();
  }

 private:
  static constexpr uint32_t kLeaf = 4;
  static constexpr int kBins = 16;
  std::vector<std::array<float, 3>> cent_;

  static void set_child(Node &nd, int c, const Box &b, int32_t code) {
    for (int a = 0; a < 3; ++a) {
      nd.lo[c][a] = b.lo[a];
      nd.hi[c][a] = b.hi[a];
    }
    nd.child[c] = code;
  }

  Box range_box(uint32_t b, uint32_t e) const {
    Box box;
    for (uint32_t i = b; i < e; ++i) box.grow(boxes[prims[i]]);
    return box;
  }

  // Splits prims[b, e) by binned SAH over centroids (midpoint split of the
  // index range when every centroid coincides); returns the split index.
  uint32_t split(uint32_t b, uint32_t e) {
    Box cb;
    for (uint32_t i = b; i < e; ++i) cb.grow(cent_[prims[i]].data());
    double best = std::numeric_limits<double>::infinity();
    int best_axis = -1, best_bin = 0;
    for (int a = 0; a < 3; ++a) {
      const float ext = cb.hi[a] - cb.lo[a];
      if (!(ext > 0.f)) continue;
      Box bin_box[kBins];
      uint32_t count[kBins] = {};
      const float scale = kBins / ext;
      for (uint32_t i = b; i < e; ++i) {
        int k = static_cast<int>((cent_[prims[i]][a] - cb.lo[a]) * scale);
        k = std::min(std::max(k, 0), kBins - 1);
        bin_box[k].grow(boxes[prims[i]]);
        ++count[k];
      }
      double right_area[kBins];
      uint32_t right_count[kBins];
      Box acc;
      uint32_t c = 0;
      for (int k = kBins - 1; k > 0; --k) {
        acc.grow(bin_box[k]);
        c += count[k];
        right_area[k] = acc.area();
        right_count[k] = c;
      }
      acc = Box();
      c = 0;
      for (int k = 0; k < kBins - 1; ++k) {
        acc.grow(bin_box[k]);
        c += count[k];
        if (c == 0 || right_count[k + 1] == 0) continue;
        const double cost = acc.area() * c + right_area[k + 1] * right_count[k + 1];
        if (cost < best) {
          best = cost;
          best_axis = a;
          best_bin = k;
        }
      }
    }
    uint32_t mid;
    if (best_axis < 0) {
      mid = b + (e - b) / 2;
    } else {
      const int a = best_axis;
      const float ext = cb.hi[a] - cb.lo[a];
      const float scale = kBins / ext;
      auto left = [&](uint32_t p) {
        int k = static_cast<int>((cent_[p][a] - cb.lo[a]) * scale);
        k = std::min(std::max(k, 0), kBins - 1);
        return k <= best_bin;
      };
      mid = static_cast<uint32_t>(std::partition(prims.begin() + b, prims.begin() + e, left) - prims.begin());
      if (mid == b || mid == e) mid = b + (e - b) / 2;
    }
    return mid;
  }

  // Builds the node over prims[b, e) (more than kLeaf of them).
  int32_t build_node(uint32_t b, uint32_t e) {
    const int32_t idx = static_cast<int32_t>(nodes.size());
    nodes.push_back(Node{});
    const uint32_t m = split(b, e);
    const uint32_t lo[2] = {b, m}, hi[2] = {m, e};
    for (int c = 0; c < 2; ++c) {
      const Box box = range_box(lo[c], hi[c]);
      int32_t code;
      if (hi[c] - lo[c] <= kLeaf)
        code = ~static_cast<int32_t>((lo[c] << 3) | (hi[c] - lo[c]));
      else
        code = build_node(lo[c], hi[c]);
      set_child(nodes[idx], c, box, code);
    }
    return idx;
  }
};

}  // namespace wih_shim

struct RTCDeviceTy {
  RTCErrorFunction error = nullptr;
  void *error_user = nullptr;
};

struct RTCGeometryTy {
  int refs = 1;
  std::vector<unsigned char> vertex, index;
  size_t vertex_stride = 0, vertex_count = 0, index_stride = 0, index_count = 0;
};

struct RTCSceneTy {
  RTCDeviceTy *device = nullptr;
  RTCGeometryTy *geometry = nullptr;
  std::vector<float> v;     // 3 per vertex
  std::vector<uint32_t> f;  // 3 per triangle
  wih_shim::Bvh bvh;
};

typedef RTCDeviceTy *RTCDevice;
typedef RTCGeometryTy *RTCGeometry;
typedef RTCSceneTy *RTCScene;

inline RTCDevice rtcNewDevice(const char *) { return new RTCDeviceTy(); }
inline void rtcReleaseDevice(RTCDevice d) { delete d; }
inline void rtcSetDeviceErrorFunction(RTCDevice d, RTCErrorFunction fn, void *user) {
  d->error = fn;
  d->error_user = user;
}
inline RTCScene rtcNewScene(RTCDevice d) {
  RTCScene s = new RTCSceneTy();
  s->device = d;
  return s;
}
inline RTCGeometry rtcNewGeometry(RTCDevice, RTCGeometryType) { return new RTCGeometryTy(); }
inline void *rtcSetNewGeometryBuffer(RTCGeometry g, RTCBufferType type, unsigned int, RTCFormat, size_t stride,
                                     size_t count) {
  std::vector<unsigned char> &buf = type == RTC_BUFFER_TYPE_VERTEX ? g->vertex : g->index;
  buf.assign(stride * count + 16, 0);
  if (type == RTC_BUFFER_TYPE_VERTEX) {
    g->vertex_stride = stride;
    g->vertex_count = count;
  } else {
    g->index_stride = stride;
    g->index_count = count;
  }
  return buf.data();
}
inline void rtcCommitGeometry(RTCGeometry) {}
inline void rtcReleaseGeometry(RTCGeometry g) {
  if (--g->refs == 0) delete g;
}
inline unsigned int rtcAttachGeometry(RTCScene s, RTCGeometry g) {
  s->geometry = g;
  ++g->refs;
  return 0;
}
inline void rtcCommitScene(RTCScene s) {
  RTCGeometryTy *g = s->geometry;
  if (!g) return;
  s->v.resize(3 * g->vertex_count);
  for (size_t i = 0; i < g->vertex_count; ++i)
    std::memcpy(&s->v[3 * i], g->vertex.data() + i * g->vertex_stride, 3 * sizeof(float));
  s->f.resize(3 * g->index_count);
  for (size_t i = 0; i < g->index_count; ++i)
    std::memcpy(&s->f[3 * i], g->index.data() + i * g->index_stride, 3 * sizeof(uint32_t));
  std::vector<wih_shim::Box> boxes(g->index_count);
  for (size_t i = 0; i < g->index_count; ++i)
    for (int k = 0; k < 3; ++k) boxes[i].grow(&s->v[3 * static_cast<size_t>(s->f[3 * i + k])]);
  s->bvh.build(boxes);
}
inline void rtcReleaseScene(RTCScene s) {
  if (s->geometry) rtcReleaseGeometry(s->geometry);
  delete s;
}

inline void rtcInitPointQueryContext(RTCPointQueryContext *c) {
  c->instStackSize = 0;
  c->instID[0] = RTC_INVALID_GEOMETRY_ID;
}
inline void rtcInitIntersectArguments(RTCIntersectArguments *a) { a->flags = 0; }

inline bool rtcPointQuery(RTCScene s, RTCPointQuery *q, RTCPointQueryContext *ctx, RTCPointQueryFunction fn,
                          void *user) {
  const wih_shim::Bvh &bvh = s->bvh;
  if (bvh.nodes.empty()) return false;
  const float p[3] = {q->x, q->y, q->z};
  float r2 = q->radius * q->radius;
  bool changed = false;
  struct Entry {
    int32_t code;
    float d2;
  };
  Entry stack[64];
  int sp = 0;
  int32_t code = 0;
  RTCPointQueryFunctionArguments args{};
  args.query = q;
  args.userPtr = user;
  args.geomID = 0;
  args.context = ctx;
  args.similarityScale = 1.f;
  for (;;) {
    if (code >= 0) {
      const wih_shim::Node &nd = bvh.nodes[static_cast<size_t>(code)];
      float d[2];
      for (int c = 0; c < 2; ++c) d[c] = wih_shim::box_dist2(nd.lo[c], nd.hi[c], p);
      const bool v0 = d[0] <= r2 && nd.lo[0][0] <= nd.hi[0][0], v1 = d[1] <= r2 && nd.lo[1][0] <= nd.hi[1][0];
      if (v0 && v1) {
        const int near = d[1] < d[0] ? 1 : 0;
        if (sp < 64) stack[sp++] = {nd.child[1 - near], d[1 - near]};
        code = nd.child[near];
        continue;
      }
      if (v0 || v1) {
        code = nd.child[v0 ? 0 : 1];
        continue;
      }
    } else {
      const uint32_t enc = ~static_cast<uint32_t>(code);
      const uint32_t first = enc >> 3, count = enc & 7u;
      for (uint32_t i = first; i < first + count; ++i) {
        const uint32_t prim = bvh.prims[i];
        const wih_shim::Box &b = bvh.boxes[prim];
        if (wih_shim::box_dist2(b.lo, b.hi, p) > r2) continue;
        args.primID = prim;
        if (fn(&args)) {
          r2 = q->radius * q->radius;
          changed = true;
        }
      }
    }
    // Next subtree still within the (possibly shrunk) radius.
    code = INT32_MIN;
    while (sp > 0) {
      const Entry e = stack[--sp];
      if (e.d2 <= r2) {
        code = e.code;
        break;
      }
    }
    if (code == INT32_MIN) break;
  }
  return changed;
}

namespace wih_shim {
// Moller-Trumbore ray/triangle test in double precision; t in [tnear, tfar].
inline bool ray_triangle(const double o[3], const double d[3], const float *a, const float *b, const float *c,
                         double tnear, double tfar, double &t) {
  const double e1[3] = {double(b[0]) - a[0], double(b[1]) - a[1], double(b[2]) - a[2]};
  const double e2[3] = {double(c[0]) - a[0], double(c[1]) - a[1], double(c[2]) - a[2]};
  const double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
  if (det == 0.0) return false;
  const double inv = 1.0 / det;
  const double tv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
  const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
  if (u < 0.0 || u > 1.0) return false;
  const double qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2], tv[0] * e1[1] - tv[1] * e1[0]};
  const double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
  if (v < 0.0 || u + v > 1.0) return false;
  t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
  return t >= tnear && t <= tfar;
}

inline bool ray_box(const double o[3], const double inv[3], const float lo[3], const float hi[3], double tnear,
                    double tfar) {
  double t0 = tnear, t1 = tfar;
  for (int a = 0; a < 3; ++a) {
    double ta = (lo[a] - o[a]) * inv[a], tb = (hi[a] - o[a]) * inv[a];
    if (ta > tb) std::swap(ta, tb);
    t0 = std::max(t0, ta);
    t1 = std::min(t1, tb);
  }
  return t0 <= t1;
}
}  // namespace wih_shim

inline void rtcIntersect1(RTCScene s, RTCRayHit *rh, RTCIntersectArguments * = nullptr) {
  const wih_shim::Bvh &bvh = s->bvh;
  if (bvh.nodes.empty()) return;
  const double o[3] = {rh->ray.org_x, rh->ray.org_y, rh->ray.org_z};
  const double d[3] = {rh->ray.dir_x, rh->ray.dir_y, rh->ray.dir_z};
  const double inv[3] = {1.0 / d[0], 1.0 / d[1], 1.0 / d[2]};
  const double tnear = rh->ray.tnear;
  double tfar = rh->ray.tfar;
  int32_t stack[64];
  int sp = 0;
  int32_t code = 0;
  bool hit = false;
  unsigned int prim_hit = 0;
  for (;;) {
    if (code >= 0) {
      const wih_shim::Node &nd = bvh.nodes[static_cast<size_t>(code)];
      const bool v0 = wih_shim::ray_box(o, inv, nd.lo[0], nd.hi[0], tnear, tfar);
      const bool v1 = wih_shim::ray_box(o, inv, nd.lo[1], nd.hi[1], tnear, tfar);
      if (v0 && v1) {
        if (sp < 64) stack[sp++] = nd.child[1];
        code = nd.child[0];
        continue;
      }
      if (v0 || v1) {
        code = nd.child[v0 ? 0 : 1];
        continue;
      }
    } else {
      const uint32_t enc = ~static_cast<uint32_t>(code);
      for (uint32_t i = enc >> 3; i < (enc >> 3) + (enc & 7u); ++i) {
        const uint32_t prim = bvh.prims[i];
        const uint32_t *tri = &s->f[3 * static_cast<size_t>(prim)];
        double t;
        if (wih_shim::ray_triangle(o, d, &s->v[3 * size_t(tri[0])], &s->v[3 * size_t(tri[1])],
                                   &s->v[3 * size_t(tri[2])], tnear, tfar, t)) {
          tfar = t;
          hit = true;
          prim_hit = prim;
        }
      }
    }
    if (sp == 0) break;
    code = stack[--sp];
  }
  if (hit) {
    rh->ray.tfar = static_cast<float>(tfar);
    rh->hit.geomID = 0;
    rh->hit.primID = prim_hit;
  }
}

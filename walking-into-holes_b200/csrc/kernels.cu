// CUDA kernels of libtwos.so (sm_100a).
//
//   wos_kernel       persistent walk-on-spheres: every lane runs one walk at a
//                    time and refills from a device work queue when its walk
//                    ends on the epsilon shell, so walks of very different
//                    lengths do not idle a warp.  Replaces the OpenMP site loop
//                    + evaluate_site/paired_site + walk of the reference
//                    (wih_twos.cpp:635-717, 1825-1841; adjoint.cpp:18-42).
//   nearest()        BVH closest-point query used by every step: 16-byte node
//                    and triangle loads, nearest-child-first order, a traversal
//                    stack in shared memory, pruning on push and pop.  Replaces
//                    rtcPointQuery + point_query_callback (wih_twos.cpp:339-359,
//                    416-430).
//   finalize_kernel  one warp per site: FP64 U-statistic, means and the
//                    leave-one-out jackknife SE over the per-walk samples with
//                    warp-shuffle reductions in a fixed order (wih_twos.cpp:
//                    691-715; adjoint.cpp:36-41).
//   closest_kernel   batched closest point (tests and the queries/s figure).
//   grid_build_kernel / grid_bound_kernel
//                    the mixed form's distance-bound grid: one FP32 closest-
//                    point query per grid vertex at mesh open, and the bound
//                    a walk step would use at given points.
//   topk kernels     block-local bitonic top-k then a merge block.
//
// Compiled with -fmad=false: FP64 arithmetic is evaluated exactly as written
// (no contraction), so it matches a plain IEEE FP64 evaluation on the host;
// the FP32 path asks for FMAs explicitly where it wants them.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>

#include "twos_internal.h"

namespace twos {

// ================================================================ random stream
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): counter = (step, walk, site, repeat*8 + block).
struct Philox4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ Philox4 philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2,
                                          uint32_t c3) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return {c0, c1, c2, c3};
}

// Uniforms in [0,1): FP64 takes the top 53 bits of (hi:lo); FP32 takes the
// top 24, i.e. the FP64 value truncated, so both forms share samples.
template <typename T> __device__ __forceinline__ T uniform(uint32_t hi, uint32_t lo);
template <> __device__ __forceinline__ double uniform<double>(uint32_t hi, uint32_t lo) {
  const uint64_t v = (static_cast<uint64_t>(hi) << 32) | lo;
  return static_cast<double>(v >> 11) * 0x1.0p-53;
}
template <> __device__ __forceinline__ float uniform<float>(uint32_t hi, uint32_t) {
  return static_cast<float>(hi >> 8) * 0x1.0p-24f;
}

template <typename T> struct Vec {
  T x, y, z;
};

__device__ __forceinline__ void sincos_pi(double a, double *s, double *c) { sincospi(a, s, c); }
__device__ __forceinline__ void sincos_pi(float a, float *s, float *c) { sincospif(a, s, c); }

// Uniform direction on S^2: z = 1 - 2a, phi = 2*pi*b (the parametrisation of
// random_unit_vector, wih_twos.cpp:536-542).
template <typename T> __device__ __forceinline__ Vec<T> direction(T a, T b) {
  const T z = T(1) - T(2) * a;
  const T zz = z * z;
  const T radial = sqrt(fmax(T(0), T(1) - zz));
  T s, c;
  sincos_pi(T(2) * b, &s, &c);
  return {radial * c, radial * s, z};
}

template <typename T> __device__ __forceinline__ T median3(T a, T b, T c) {
  return fmax(fmin(a, b), fmin(fmax(a, b), c));
}

// ================================================================ arithmetic helpers
// madd: FMA in FP32, plain multiply-add in FP64 (bit-identical to host FP64).
__device__ __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double madd(double a, double b, double c) { return a * b + c; }

__device__ __forceinline__ float dot3(const Vec<float> &a, const Vec<float> &b) {
  return __fmaf_rn(a.x, b.x, __fmaf_rn(a.y, b.y, a.z * b.z));
}
__device__ __forceinline__ double dot3(const Vec<double> &a, const Vec<double> &b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T> __device__ __forceinline__ Vec<T> sub(const Vec<T> &a, const Vec<T> &b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
// a*b + c: one fused multiply-add in FP32 (the mixed form's arithmetic);
// separately rounded in FP64, so the plain form keeps the host's operations
// (the library is built without contraction).
template <typename T> __device__ __forceinline__ T mad_t(T a, T b, T c) { return a * b + c; }
template <> __device__ __forceinline__ float mad_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <typename T> __device__ __forceinline__ Vec<T> add_scaled(const Vec<T> &a, const Vec<T> &d, T s) {
  return {mad_t(d.x, s, a.x), mad_t(d.y, s, a.y), mad_t(d.z, s, a.z)};
}

// Squared distance from p to the closest point of triangle (a, b, c):
// Ericson's Voronoi-region case analysis (Real-Time Collision Detection,
// 5.1.5), the algorithm of closest_point_triangle (wih_twos.cpp:247-289).
template <typename T>
__device__ __forceinline__ Vec<T> tri_closest(const Vec<T> &p, const Vec<T> &a, const Vec<T> &b, const Vec<T> &c) {
  const Vec<T> ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const T d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  Vec<T> q;
  if (d1 <= T(0) && d2 <= T(0)) {
    q = a;
  } else {
    const Vec<T> bp = sub(p, b);
    const T d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= T(0) && d4 <= d3) {
      q = b;
    } else {
      const T vc = mad_t(d1, d4, -(d3 * d2));
      if (vc <= T(0) && d1 >= T(0) && d3 <= T(0)) {
        const T v = d1 / (d1 - d3);
        q = add_scaled(a, ab, v);
      } else {
        const Vec<T> cp = sub(p, c);
        const T d5 = dot3(ab, cp), d6 = dot3(ac, cp);
        if (d6 >= T(0) && d5 <= d6) {
          q = c;
        } else {
          const T vb = mad_t(d5, d2, -(d1 * d6));
          if (vb <= T(0) && d2 >= T(0) && d6 <= T(0)) {
            const T w = d2 / (d2 - d6);
            q = add_scaled(a, ac, w);
          } else {
            const T va = mad_t(d3, d6, -(d5 * d4));
            if (va <= T(0) && (d4 - d3) >= T(0) && (d5 - d6) >= T(0)) {
              const T w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
              q = add_scaled(b, sub(c, b), w);
            } else {
              const T denom = T(1) / (va + vb + vc);
              const T v = vb * denom, w = vc * denom;
              const Vec<T> t = add_scaled(a, ab, v);
              q = add_scaled(t, ac, w);
            }
          }
        }
      }
    }
  }
  return q;
}

template <typename T>
__device__ __forceinline__ T tri_dist2(const Vec<T> &p, const Vec<T> &a, const Vec<T> &b, const Vec<T> &c) {
  const Vec<T> d = sub(p, tri_closest(p, a, b, c));
  return dot3(d, d);
}

// ================================================================ BVH traversal
template <typename T> struct Layout;
template <> struct Layout<float> {
  using Node = NodeF;
  using Tri = TriF;
};
template <> struct Layout<double> {
  using Node = NodeD;
  using Tri = TriD;
};

__device__ __forceinline__ float gap(float lo, float hi, float p) { return fmaxf(fmaxf(lo - p, p - hi), 0.f); }
__device__ __forceinline__ double gap(double lo, double hi, double p) { return fmax(fmax(lo - p, p - hi), 0.0); }

// Lower bound on the squared distance from p to each child: the larger of
// the box bound and the normal-slab bound (the child's triangles lie between
// the planes n.x = smin and n.x = smax, so |n.p - [smin, smax]| bounds the
// distance from below; for a nearly flat patch the slab is thin and the
// bound is close to the true distance, where the box bound is off by up to
// the box size).
// 32-byte read-only load (two float4) of 32-byte aligned data: one L1
// request instead of two.
__device__ __forceinline__ void ldg32(const void *p, float4 &a, float4 &b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ void node_dist2(const NodeF *__restrict__ nodes, int idx, const Vec<float> &p,
                                           float &dl, float &dr, int &cl, int &cr) {
  const NodeF *n = nodes + idx;
  float4 x, y, z, nl, nr, t;
  ldg32(&n->x, x, y);
  ldg32(&n->z, z, nl);
  ldg32(&n->nr, nr, t);
  const float lx = gap(x.x, x.z, p.x), rx = gap(x.y, x.w, p.x);
  const float ly = gap(y.x, y.z, p.y), ry = gap(y.y, y.w, p.y);
  const float lz = gap(z.x, z.z, p.z), rz = gap(z.y, z.w, p.z);
  const float sl = __fmaf_rn(nl.x, p.x, __fmaf_rn(nl.y, p.y, nl.z * p.z));
  const float sr = __fmaf_rn(nr.x, p.x, __fmaf_rn(nr.y, p.y, nr.z * p.z));
  const float gl = gap(nl.w, t.x, sl), gr = gap(nr.w, t.y, sr);
  dl = fmaxf(__fmaf_rn(lx, lx, __fmaf_rn(ly, ly, lz * lz)), gl * gl);
  dr = fmaxf(__fmaf_rn(rx, rx, __fmaf_rn(ry, ry, rz * rz)), gr * gr);
  cl = __float_as_int(t.z);
  cr = __float_as_int(t.w);
}

__device__ __forceinline__ void node_dist2(const NodeD *__restrict__ nodes, int idx, const Vec<double> &p,
                                           double &dl, double &dr, int &cl, int &cr) {
  const NodeD *n = nodes + idx;
  const double2 xl = __ldg(&n->xlo), xh = __ldg(&n->xhi);
  const double2 yl = __ldg(&n->ylo), yh = __ldg(&n->yhi);
  const double2 zl = __ldg(&n->zlo), zh = __ldg(&n->zhi);
  const double2 l0 = __ldg(&n->nl_xy), l1 = __ldg(&n->nl_zmin);
  const double2 r0 = __ldg(&n->nr_xy), r1 = __ldg(&n->nr_zmin);
  const double2 smax = __ldg(&n->smax);
  const int4 ch = __ldg(&n->child);
  const double lx = gap(xl.x, xh.x, p.x), rx = gap(xl.y, xh.y, p.x);
  const double ly = gap(yl.x, yh.x, p.y), ry = gap(yl.y, yh.y, p.y);
  const double lz = gap(zl.x, zh.x, p.z), rz = gap(zl.y, zh.y, p.z);
  const double sl = l0.x * p.x + l0.y * p.y + l1.x * p.z;
  const double sr = r0.x * p.x + r0.y * p.y + r1.x * p.z;
  const double gl = gap(l1.y, smax.x, sl), gr = gap(r1.y, smax.y, sr);
  dl = fmax(lx * lx + ly * ly + lz * lz, gl * gl);
  dr = fmax(rx * rx + ry * ry + rz * rz, gr * gr);
  cl = ch.x;
  cr = ch.y;
}

// The same bounds for the four children of a four-wide node (six 32-byte
// loads); slot k's squared lower bound in d[k], its child code in c[k].  An
// empty slot's inverted box gives +inf.
__device__ __forceinline__ void node4_dist2(const Node4F *__restrict__ nodes, int idx, const Vec<float> &p,
                                            float d[4], int c[4]) {
  const Node4F *n = nodes + idx;
  float4 xlo, xhi, ylo, yhi, zlo, zhi, nx, ny, nz, smin, smax, ch;
  ldg32(&n->xlo, xlo, xhi);
  ldg32(&n->ylo, ylo, yhi);
  ldg32(&n->zlo, zlo, zhi);
  ldg32(&n->nx, nx, ny);
  ldg32(&n->nz, nz, smin);
  ldg32(&n->smax, smax, ch);
  auto slot = [&](float xl, float xh, float yl, float yh, float zl, float zh, float a, float b, float e, float s0,
                  float s1) {
    const float gx = gap(xl, xh, p.x), gy = gap(yl, yh, p.y), gz = gap(zl, zh, p.z);
    const float s = __fmaf_rn(a, p.x, __fmaf_rn(b, p.y, e * p.z));
    const float gs = gap(s0, s1, s);
    return fmaxf(__fmaf_rn(gx, gx, __fmaf_rn(gy, gy, gz * gz)), gs * gs);
  };
  d[0] = slot(xlo.x, xhi.x, ylo.x, yhi.x, zlo.x, zhi.x, nx.x, ny.x, nz.x, smin.x, smax.x);
  d[1] = slot(xlo.y, xhi.y, ylo.y, yhi.y, zlo.y, zhi.y, nx.y, ny.y, nz.y, smin.y, smax.y);
  d[2] = slot(xlo.z, xhi.z, ylo.z, yhi.z, zlo.z, zhi.z, nx.z, ny.z, nz.z, smin.z, smax.z);
  d[3] = slot(xlo.w, xhi.w, ylo.w, yhi.w, zlo.w, zhi.w, nx.w, ny.w, nz.w, smin.w, smax.w);
  c[0] = __float_as_int(ch.x);
  c[1] = __float_as_int(ch.y);
  c[2] = __float_as_int(ch.z);
  c[3] = __float_as_int(ch.w);
}

__device__ __forceinline__ void order2(float &da, int &ca, float &db, int &cb) {
  if (db < da) {
    const float t = da;
    da = db;
    db = t;
    const int u = ca;
    ca = cb;
    cb = u;
  }
}

// Plane-slab lower bound of a triangle (one or two 16-byte loads); the full
// closest-point test loads the vertices only when this bound is below best.
__device__ __forceinline__ float tri_plane_gap2(const TriF *__restrict__ tris, uint32_t i, const Vec<float> &p) {
  const float4 P = __ldg(&tris[i].plane);
  const float dmax = __ldg(&tris[i].a.w);
  const float s = __fmaf_rn(P.x, p.x, __fmaf_rn(P.y, p.y, P.z * p.z));
  const float g = gap(P.w, dmax, s);
  return g * g;
}
__device__ __forceinline__ double tri_plane_gap2(const TriD *__restrict__ tris, uint32_t i, const Vec<double> &p) {
  const double2 n = __ldg(&tris[i].nxy), z = __ldg(&tris[i].nzmin);
  const double dmax = __ldg(&tris[i].dmax_id.x);
  const double s = n.x * p.x + n.y * p.y + z.x * p.z;
  const double g = gap(z.y, dmax, s);
  return g * g;
}

__device__ __forceinline__ void load_tri(const TriF *__restrict__ tris, uint32_t i, Vec<float> &a, Vec<float> &b,
                                         Vec<float> &c) {
  const float4 A = __ldg(&tris[i].a), B = __ldg(&tris[i].b), C = __ldg(&tris[i].c);
  a = {A.x, A.y, A.z};
  b = {B.x, B.y, B.z};
  c = {C.x, C.y, C.z};
}
__device__ __forceinline__ void load_tri(const TriD *__restrict__ tris, uint32_t i, Vec<double> &a,
                                         Vec<double> &b, Vec<double> &c) {
  const double2 p0 = __ldg(&tris[i].axy), p1 = __ldg(&tris[i].azbx), p2 = __ldg(&tris[i].bybz);
  const double2 p3 = __ldg(&tris[i].cxy), p4 = __ldg(&tris[i].czpad);
  a = {p0.x, p0.y, p1.x};
  b = {p1.y, p2.x, p2.y};
  c = {p3.x, p3.y, p4.x};
}

// One triangle against the current best: the plane-slab bound first, the
// full closest-point test only when the bound is below best.  Returns true
// when the triangle is strictly closer (best2 updated); `full` counts full tests.
__device__ __forceinline__ bool tri_test(const TriF *__restrict__ tris, uint32_t i, const Vec<float> &p, float &best2,
                                         uint32_t &full) {
  float4 P, A;
  ldg32(&tris[i].plane, P, A);
  const float s = __fmaf_rn(P.x, p.x, __fmaf_rn(P.y, p.y, P.z * p.z));
  const float g = gap(P.w, A.w, s);
  if (!(g * g < best2)) return false;
  ++full;
  float4 B, C;
  ldg32(&tris[i].b, B, C);
  const float d2 = tri_dist2(p, Vec<float>{A.x, A.y, A.z}, Vec<float>{B.x, B.y, B.z}, Vec<float>{C.x, C.y, C.z});
  if (d2 < best2) {
    best2 = d2;
    return true;
  }
  return false;
}
__device__ __forceinline__ bool tri_test(const TriD *__restrict__ tris, uint32_t i, const Vec<double> &p,
                                         double &best2, uint32_t &full) {
  if (!(tri_plane_gap2(tris, i, p) < best2)) return false;
  ++full;
  Vec<double> a, b, c;
  load_tri(tris, i, a, b, c);
  const double d2 = tri_dist2(p, a, b, c);
  if (d2 < best2) {
    best2 = d2;
    return true;
  }
  return false;
}

__device__ __forceinline__ float lower_f(float v) { return v; }
__device__ __forceinline__ float lower_f(double v) { return __double2float_rd(v); }

// Closest-point query: on return best2 holds the squared distance to the
// nearest triangle strictly closer than sqrt(best2) on entry; returns false
// when there is none.  The stack lives in shared memory, `stack` pointing at
// this thread's column (stride `stride` entries).  Bounded: at most kStack
// pushes outstanding and `max_iter` node/leaf visits; overruns set `err`.
template <typename T>
__device__ bool nearest(const typename Layout<T>::Node *__restrict__ nodes,
                        const typename Layout<T>::Tri *__restrict__ tris, uint32_t max_iter, const Vec<T> &p,
                        T &best2, uint32_t &best_tri, uint2 *stack, int stride, uint32_t &err) {
  bool found = false;
  int sp = 0;
  int node = 0;
  bool have = true;
  uint32_t iter = 0;
  while (have) {
    if (++iter > max_iter) {
      err |= TWOS_DEVERR_ITER;
      break;
    }
    if (node >= 0) {
      T dl, dr;
      int cl, cr;
      node_dist2(nodes, node, p, dl, dr, cl, cr);
      const bool vl = dl < best2, vr = dr < best2;
      if (vl && vr) {
        if (dr < dl) {
          const T td = dl;
          dl = dr;
          dr = td;
          const int tc = cl;
          cl = cr;
          cr = tc;
        }
        if (sp >= kStack) {
          err |= TWOS_DEVERR_STACK;
          break;
        }
        stack[sp * stride] = make_uint2(static_cast<uint32_t>(cr), __float_as_uint(lower_f(dr)));
        ++sp;
        node = cl;
        continue;
      }
      if (vl) {
        node = cl;
        continue;
      }
      if (vr) {
        node = cr;
        continue;
      }
    } else {
      const uint32_t enc = ~static_cast<uint32_t>(node);
      const uint32_t first = enc >> 3, count = enc & 7u;
      for (uint32_t i = 0; i < count; ++i) {
        uint32_t full = 0;
        if (tri_test(tris, first + i, p, best2, full)) {
          best_tri = first + i;
          found = true;
        }
      }
    }
    // Pop the next entry still closer than the current best.
    have = false;
    while (sp > 0) {
      --sp;
      const uint2 e = stack[sp * stride];
      if (static_cast<T>(__uint_as_float(e.y)) < best2) {
        node = static_cast<int>(e.x);
        have = true;
        break;
      }
    }
  }
  return found;
}

// ================================================================ sources
template <typename T> struct TermT {
  int kind, axis;
  T amp, offset, div;
  T c[3], w[3];
};

template <typename T> __device__ __forceinline__ T coord(const Vec<T> &v, int a) {
  return a == 0 ? v.x : (a == 1 ? v.y : v.z);
}

template <typename T> __device__ __forceinline__ T term_value(const TermT<T> &t, const Vec<T> &x) {
  switch (t.kind) {
    case TWOS_TERM_CONST:
      return t.amp;
    case TWOS_TERM_LINEAR:
      return t.amp * (coord(x, t.axis) + t.offset);
    case TWOS_TERM_GAUSS: {
      const T a = (x.x - t.c[0]) / t.w[0], b = (x.y - t.c[1]) / t.w[1], c = (x.z - t.c[2]) / t.w[2];
      return t.amp * exp(-(a * a) - (b * b) - (c * c));
    }
    case TWOS_TERM_BUMP: {
      const Vec<T> d{x.x - t.c[0], x.y - t.c[1], x.z - t.c[2]};
      const T dd = d.x * d.x + d.y * d.y + d.z * d.z;
      const T s = fmax(T(0), T(1) - dd / (t.w[0] * t.w[0]));
      return t.amp * (s * s) / t.div;
    }
    case TWOS_TERM_BOX:
      return (x.x >= t.c[0] && x.x <= t.w[0] && x.y >= t.c[1] && x.y <= t.w[1] && x.z >= t.c[2] &&
              x.z <= t.w[2])
                 ? t.amp
                 : T(0);
    case TWOS_TERM_BALL: {
      const Vec<T> d{x.x - t.c[0], x.y - t.c[1], x.z - t.c[2]};
      const T dd = d.x * d.x + d.y * d.y + d.z * d.z;
      return dd <= t.w[0] * t.w[0] ? t.amp : T(0);
    }
    case TWOS_TERM_QUAD: {
      const T a = x.x - t.c[0], b = x.y - t.c[1], c = x.z - t.c[2];
      return t.amp * (t.w[0] * (a * a) + t.w[1] * (b * b) + t.w[2] * (c * c));
    }
    default:
      return T(0);
  }
}

template <typename T>
__device__ __forceinline__ T source_value(const TermT<T> *terms, uint32_t begin, uint32_t n, const Vec<T> &x) {
  if (n == 0) return T(0);
  T s = term_value(terms[begin], x);
  for (uint32_t i = 1; i < n; ++i) s = s + term_value(terms[begin + i], x);
  return s;
}

}  // namespace twos
#include "ball_green.cuh"
namespace twos {

// One step's EXACT source integral over B_r(x), accumulated into acc as the
// analytic study backend does (study.cpp:96-104): the harmonic (CONST and
// LINEAR) terms as r^2/6 f(x) in one product, then each bump's closed-form
// ball integral added in term order.  Bumps are evaluated in FP64 (double-
// double inside) from the frame coordinates.
template <typename T>
__device__ __forceinline__ T exact_source(T acc, const TermT<T> *terms, uint32_t begin, uint32_t n,
                                          const Vec<T> &x, T r, uint32_t &err) {
  T harmonic = T(0);
  bool any = false;
  for (uint32_t i = 0; i < n; ++i) {
    const TermT<T> &t = terms[begin + i];
    if (t.kind == TWOS_TERM_CONST || t.kind == TWOS_TERM_LINEAR) {
      harmonic = any ? harmonic + term_value(t, x) : term_value(t, x);
      any = true;
    }
  }
  if (any) acc = acc + r * r / T(6) * harmonic;
  for (uint32_t i = 0; i < n; ++i) {
    const TermT<T> &t = terms[begin + i];
    if (t.kind != TWOS_TERM_BUMP) continue;
    const double dx = static_cast<double>(x.x) - static_cast<double>(t.c[0]);
    const double dy = static_cast<double>(x.y) - static_cast<double>(t.c[1]);
    const double dz = static_cast<double>(x.z) - static_cast<double>(t.c[2]);
    bool negative = false;
    const double v = exact_bump_green(sqrt(dx * dx + dy * dy + dz * dz), static_cast<double>(r),
                                      static_cast<double>(t.w[0]),
                                      static_cast<double>(t.amp) / static_cast<double>(t.div), negative);
    if (negative) err |= TWOS_DEVERR_SOURCE;
    acc = acc + static_cast<T>(v);
  }
  return acc;
}

// ================================================================ WoS kernel
constexpr int kWosBlock = 128;

template <typename T> __device__ __forceinline__ T to_T(double v);
template <> __device__ __forceinline__ double to_T<double>(double v) { return v; }
template <> __device__ __forceinline__ float to_T<float>(double v) { return static_cast<float>(v); }

// Position of a site/cavity in the geometry frame: FP64 keeps the original
// coordinates; FP32 is taken about the geometry centre.
template <typename T> __device__ __forceinline__ Vec<T> to_frame(const double *xyz, const GeoDesc &g);
template <> __device__ __forceinline__ Vec<double> to_frame<double>(const double *xyz, const GeoDesc &) {
  return {xyz[0], xyz[1], xyz[2]};
}
template <> __device__ __forceinline__ Vec<float> to_frame<float>(const double *xyz, const GeoDesc &g) {
  return {static_cast<float>(xyz[0] - g.center[0]), static_cast<float>(xyz[1] - g.center[1]),
          static_cast<float>(xyz[2] - g.center[2])};
}

template <typename T> __device__ __forceinline__ const typename Layout<T>::Node *geo_nodes(const GeoDesc &g);
template <> __device__ __forceinline__ const NodeF *geo_nodes<float>(const GeoDesc &g) { return g.nodes_f; }
template <> __device__ __forceinline__ const NodeD *geo_nodes<double>(const GeoDesc &g) { return g.nodes_d; }
template <typename T> __device__ __forceinline__ const typename Layout<T>::Tri *geo_tris(const GeoDesc &g);
template <> __device__ __forceinline__ const TriF *geo_tris<float>(const GeoDesc &g) { return g.tris_f; }
template <> __device__ __forceinline__ const TriD *geo_tris<double>(const GeoDesc &g) { return g.tris_d; }

// An upper bound on sqrtf(x) for x > 0 from rsqrtf, whose stated maximum
// error is 2 ulp: x rsqrtf(x) is within 1.25 * 2^-22 of sqrt(x) (relative),
// so raising it by 2^-20 puts it above the correctly rounded sqrtf(x).  The
// grid bounds only need |p - v| from above (a larger distance lowers the
// lower bound and raises the upper one), and this takes fewer instructions
// than the correctly rounded square root.  x = 0 gives NaN, which the
// bounds' fmaxf / fminf skip: that corner is left out, which only loosens
// them.
__device__ __forceinline__ float sqrt_up(float x) { return x * rsqrtf(x) * (1.0f + 0x1.0p-20f); }

// Distance-grid vertex (i, j, k) in the FP32 frame, rounded the same way in
// the grid build and in the walk step.
__device__ __forceinline__ Vec<float> grid_vertex(const GeoDesc &g, uint32_t i, uint32_t j, uint32_t k) {
  return {__fadd_rn(g.grid_lo[0], __fmul_rn(static_cast<float>(i), g.grid_h)),
          __fadd_rn(g.grid_lo[1], __fmul_rn(static_cast<float>(j), g.grid_h)),
          __fadd_rn(g.grid_lo[2], __fmul_rn(static_cast<float>(k), g.grid_h))};
}

// The grid's bounds of the mesh distance at `p` (FP32 frame).  Lower: the
// largest D(v) - |p - v| over the eight corners v of p's cell (the distance
// is 1-Lipschitz, so each is a bound).  Upper (before the FP32 allowance
// the caller adds): the smallest (D(v) + 1) q + |p - v| over the corners
// whose value is held exactly -- a vertex stores floor((d_FP32 - 2 delta)/q),
// so its distance is below (D + 1) q + 3 delta.  `entry_node` is the cell's
// entry node (-1: none).  False when p lies outside the grid (or is NaN).
// One 16-byte record per cell (GeoDesc::grid).
__device__ __forceinline__ bool grid_bounds(const GeoDesc &g, const Vec<float> &p, float &bound, float &upper,
                                            int &entry_node) {
  const float fx = (p.x - g.grid_lo[0]) * g.grid_inv_h;
  const float fy = (p.y - g.grid_lo[1]) * g.grid_inv_h;
  const float fz = (p.z - g.grid_lo[2]) * g.grid_inv_h;
  if (!(fx >= 0.f && fy >= 0.f && fz >= 0.f && fx <= static_cast<float>(g.grid_n[0] - 1) &&
        fy <= static_cast<float>(g.grid_n[1] - 1) && fz <= static_cast<float>(g.grid_n[2] - 1)))
    return false;
  // The cell's lower corner (clamped so the cell lies inside the grid), then
  // the best of its eight corners' bounds.
  const uint32_t i0 = min(static_cast<uint32_t>(fx), g.grid_n[0] - 2);
  const uint32_t j0 = min(static_cast<uint32_t>(fy), g.grid_n[1] - 2);
  const uint32_t k0 = min(static_cast<uint32_t>(fz), g.grid_n[2] - 2);
  float best = -CUDART_INF_F, up = CUDART_INF_F;
  const uint4 rec = __ldg(g.grid + (static_cast<size_t>(i0) * (g.grid_n[1] - 1) + j0) * (g.grid_n[2] - 1) + k0);
  const uint32_t base = rec.z & 0xffffu;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const uint32_t i = i0 + (c >> 2), j = j0 + ((c >> 1) & 1), k = k0 + (c & 1);
    const Vec<float> v = grid_vertex(g, i, j, k);
    const Vec<float> dv = sub(p, v);
    const uint32_t off = ((c < 4 ? rec.x : rec.y) >> (8 * (c & 3))) & 0xffu;
    const float dist = sqrt_up(dot3(dv, dv));
    const float dq = static_cast<float>(off == 0xffu ? base : base + off) * g.grid_q;
    best = fmaxf(best, dq - dist);
    if (off != 0xffu) up = fminf(up, dq + g.grid_q + dist);
  }
  bound = best;
  upper = up;
  entry_node = static_cast<int>(rec.w);
  return true;
}

__device__ __forceinline__ bool grid_bound(const GeoDesc &g, const Vec<float> &p, float &bound) {
  float upper;
  int entry_node;
  return grid_bounds(g, p, bound, upper, entry_node);
}

__device__ __forceinline__ uint32_t find_job(const JobDesc *jobs, uint32_t n, uint64_t wid) {
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (jobs[mid].walk_begin <= wid)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Dynamic shared memory: the launch's job, geometry and term tables.
// Job and geometry descriptors are copied to shared memory when they take at
// most kTableSmem bytes, which keeps 8 blocks of 128 threads (with their
// traversal stacks) resident per SM; a launch with more jobs reads them from
// global memory (through L1) instead of giving up resident blocks.
constexpr uint32_t kTableSmem = 2048;
struct SmemPlan {
  uint32_t geo_offset, term_offset, bytes;
  bool tables;  // jobs and geometries in shared memory
};
template <typename T> __host__ __device__ inline SmemPlan smem_plan(uint32_t n_jobs, uint32_t n_geos, uint32_t n_terms) {
  SmemPlan p;
  const uint32_t jobs = n_jobs * static_cast<uint32_t>(sizeof(JobDesc));
  const uint32_t geo_offset = (jobs + 15u) & ~15u;
  const uint32_t geos = geo_offset + n_geos * static_cast<uint32_t>(sizeof(GeoDesc));
  p.tables = geos <= kTableSmem;
  p.geo_offset = p.tables ? geo_offset : 0u;
  p.term_offset = p.tables ? (geos + 15u) & ~15u : 0u;
  p.bytes = p.term_offset + n_terms * static_cast<uint32_t>(sizeof(TermT<T>));
  return p;
}

bool launch_tables_in_smem(int precision, uint32_t n_jobs, uint32_t n_geos, uint32_t n_terms) {
  return precision == TWOS_PREC_MIXED ? smem_plan<float>(n_jobs, n_geos, n_terms).tables
                                      : smem_plan<double>(n_jobs, n_geos, n_terms).tables;
}

enum : int { kIdle = 0, kTraverse = 1, kStep = 2 };

// Persistent walk-on-spheres kernel as a per-lane state machine.  Each loop
// iteration every traversing lane runs up to `units` units of work back to
// back -- BVH node tests or triangle tests of its current closest-point query
// -- and stops early when its query ends.  A lane whose query
// has finished waits in kStep until at least `step_threshold` lanes of its
// warp are ready (or no lane is still traversing); those lanes then take
// their walk step together and start their next query, and lanes whose walk
// ended refill from the work queue once `refill` lanes are idle.  So lanes
// never wait for the slowest traversal of the warp, only for the batched
// step.  In the mixed form a step first tries the geometry's distance-bound
// grid and skips the query when the grid's bound is large enough.  MODE:
// TWOS_MODE_*; the per-walk value type is T (FP32 accumulation in the mixed
// form, FP64 in the plain form).  SRC: TWOS_SOURCE_* (a
// template argument, so the exact-integral code of TWOS_SOURCE_EXACT adds no
// registers to the other forms).
// Residency: the FP32 form with the centre-point source fits 64 registers, so
// 1024 threads (8 blocks of 128) stay resident per SM; the others take up to
// 80 (768 threads, 6 blocks of 128).
template <typename T, int MODE, int SRC>
constexpr int wos_min_blocks(int block) {
  return sizeof(T) == 4 && SRC == TWOS_SOURCE_CENTER && MODE != kModeGradient ? 1024 / block
         : block >= 768                                                      ? 1
                                                                              : 768 / block;
}

// Walks a lane claims from the work queue at once.
__device__ __forceinline__ uint32_t lane_walks_of(const WosLaunch &L) {
  return L.lane_walks > 1 ? static_cast<uint32_t>(L.lane_walks) : 1u;
}

template <typename T, int MODE, int SRC, int BLOCK, bool TRACE = false, bool GRID64 = false, bool WIDE = false,
          bool CLAIM = false>
__global__ void __launch_bounds__(BLOCK, wos_min_blocks<T, MODE, SRC>(BLOCK)) wos_kernel(const WosLaunch L) {
  constexpr bool GREEN = SRC == TWOS_SOURCE_GREEN;
  constexpr bool EXACT = SRC == TWOS_SOURCE_EXACT && MODE != kModeBoundary;
  constexpr bool GRAD = MODE == kModeGradient;
  constexpr bool PAIRED = MODE == TWOS_MODE_PAIRED || GRAD;
  // Dynamic shared memory: the traversal stacks (kStack entries per thread,
  // column-major so a warp's accesses hit distinct banks), then the tables.
  extern __shared__ __align__(16) unsigned char s_dyn[];
  uint2 *s_stack = reinterpret_cast<uint2 *>(s_dyn);
  unsigned char *s_tab = s_dyn + kStack * BLOCK * sizeof(uint2);
  const SmemPlan plan = smem_plan<T>(L.n_jobs, L.n_geos, L.n_terms);
  const JobDesc *s_jobs = plan.tables ? reinterpret_cast<const JobDesc *>(s_tab) : L.jobs;
  const GeoDesc *s_geos = plan.tables ? reinterpret_cast<const GeoDesc *>(s_tab + plan.geo_offset) : L.geos;
  TermT<T> *s_terms = reinterpret_cast<TermT<T> *>(s_tab + plan.term_offset);

  if (plan.tables) {
    JobDesc *tj = reinterpret_cast<JobDesc *>(s_tab);
    GeoDesc *tg = reinterpret_cast<GeoDesc *>(s_tab + plan.geo_offset);
    for (uint32_t i = threadIdx.x; i < L.n_jobs; i += blockDim.x) tj[i] = L.jobs[i];
    for (uint32_t i = threadIdx.x; i < L.n_geos; i += blockDim.x) tg[i] = L.geos[i];
  }
  for (uint32_t i = threadIdx.x; i < L.n_terms; i += blockDim.x) {
    const TermDev &d = L.terms[i];
    TermT<T> t;
    t.kind = d.kind;
    t.axis = d.axis;
    t.amp = to_T<T>(d.amp);
    t.offset = to_T<T>(d.offset);
    t.div = to_T<T>(d.div);
    for (int k = 0; k < 3; ++k) {
      t.c[k] = to_T<T>(d.c[k]);
      t.w[k] = to_T<T>(d.w[k]);
    }
    s_terms[i] = t;
  }
  __syncthreads();

  const unsigned lane = threadIdx.x & 31u;
  const unsigned full = 0xffffffffu;
  uint2 *stack = s_stack + threadIdx.x;
  uint32_t err = 0;
  // Per-thread traversal counters (32-bit: a thread's share of one launch
  // stays far below 2^32), summed in 64 bits at the end.
  uint32_t c_nodes = 0, c_planes = 0, c_tris = 0, c_grid = 0;

  int phase = kIdle;
  bool exhausted = false;  // warp-uniform
  const int units = L.units > 0 ? L.units : 1;
  // Walk state.
  uint64_t wid = 0;
  uint32_t job = 0, site = 0, walk = 0, steps = 0;
  Vec<T> pos{T(0), T(0), T(0)};
  T u = T(0), pv = T(0);
  // Gradient mode: first-ball radius, direction and payoff increments, and
  // the ball source terms of grad U / grad P.
  T g_r0 = T(0), g_u0 = T(0), g_p0 = T(0);
  Vec<T> g_w0{T(0), T(0), T(0)}, g_su{T(0), T(0), T(0)}, g_sp{T(0), T(0), T(0)};
  // Query state.
  T best2 = T(0);
  int node = 0, sp = 0;
  bool have = false, found = false;
  // Four-wide form: this query continues on the binary BVH (set when a
  // four-wide visit would overflow the stack).
  bool narrow = false;
  uint32_t best_tri = 0;  // leaf-order index of the nearest triangle found for this walk
  bool tri_ok = false;    // best_tri belongs to this walk
  uint32_t tri_cur = 0, tri_end = 0, iter = 0;
  // CLAIM: walks a lane claims from the queue at once, run one after
  // another: s_claim[thread] of them, wid + 1 onwards, are not yet started
  // (shared memory, read only at refills).  A compile-time variant, so the
  // default kernel's refill stays one atomic per warp and one start per lane.
  __shared__ uint32_t s_claim[CLAIM ? BLOCK : 1];
  if (CLAIM) s_claim[threadIdx.x] = 0u;

  for (;;) {
    // Starts walk `wid` on this lane (its first radius from the per-site
    // pre-pass when there is one).
    auto start_walk = [&]() {
      const uint64_t id = wid;
      job = find_job(s_jobs, L.n_jobs, id);
      const JobDesc &J = s_jobs[job];
      const uint64_t local = id - J.walk_begin;
      site = static_cast<uint32_t>(local / J.walks);
      walk = static_cast<uint32_t>(local - static_cast<uint64_t>(site) * J.walks);
      const GeoDesc &G = s_geos[J.geo];
      bool skip = false;
      if (L.walk_start) {
        const double *st = L.walk_start + 3ull * wid;
        skip = isnan(st[0]);
        pos = to_frame<T>(st, G);
      } else {
        pos = to_frame<T>(L.sites + 3ull * (J.site_begin + site), G);
      }
      u = T(0);
      pv = T(0);
      steps = 0;
      tri_ok = false;
      if (GRAD) g_r0 = T(0);
      if (!skip && (J.flags & kJobSkipCavitySites)) {
        const T R = to_T<T>(J.cavity_radius);
        for (uint32_t c = 0; c < J.n_cav; ++c) {
          const Vec<T> cc = to_frame<T>(L.cavities + 3ull * (J.cav_begin + c), G);
          const Vec<T> dv = sub(pos, cc);
          if (sqrt(dot3(dv, dv)) <= R) skip = true;
        }
      }
      if (skip) {
        if (MODE != kModeBoundary) static_cast<T *>(L.u_out)[wid] = T(0);
        if (PAIRED) static_cast<T *>(L.p_out)[wid] = T(0);
        if (GRAD)
          for (int k = 0; k < 6; ++k) static_cast<T *>(L.grad_out)[6ull * wid + k] = T(0);
        if (MODE == kModeBoundary) L.hits[wid].cavity = -2;
        L.steps_out[wid] = 0u;
      } else if (L.site_best2 && MODE != kModeBoundary) {
        // First query answered by the per-site pre-pass.
        best2 = static_cast<const T *>(L.site_best2)[J.site_rank + site];
        found = best2 >= T(0);
        phase = kStep;
      } else {
        best2 = static_cast<T>(J.query_radius2);
        node = 0;
        sp = 0;
        have = true;
        narrow = false;
        found = false;
        tri_cur = tri_end = 0;
        iter = 0;
        phase = kTraverse;
      }
    };

    // ---- refill idle lanes from the work queue (CLAIM: from their own
    // claims first)
    const unsigned idle = __ballot_sync(full, phase == kIdle);
    if constexpr (CLAIM) {
      if (idle != 0u) {
        const unsigned pending = __ballot_sync(full, s_claim[threadIdx.x] != 0u);
        if ((!exhausted || pending != 0u) && (__popc(idle) >= L.refill || idle == full)) {
          uint32_t claim_left = s_claim[threadIdx.x];
          const unsigned claim = __ballot_sync(full, phase == kIdle && claim_left == 0u);
          if (!exhausted && claim != 0u) {
            const uint64_t span = static_cast<uint64_t>(lane_walks_of(L)) * __popc(claim);
            unsigned long long base = 0;
            const int leader = __ffs(claim) - 1;
            if (static_cast<int>(lane) == leader) base = atomicAdd(L.counter, static_cast<unsigned long long>(span));
            base = __shfl_sync(full, base, leader);
            if (base + span >= L.total_walks) exhausted = true;
            if (phase == kIdle && claim_left == 0u) {
              const uint64_t first =
                  base + static_cast<uint64_t>(lane_walks_of(L)) * __popc(claim & ((1u << lane) - 1u));
              if (first < L.total_walks) {
                wid = first - 1;  // wraps for the first walk of the queue; wid + 1 is exact
                const uint64_t left = L.total_walks - first;
                claim_left = left < lane_walks_of(L) ? static_cast<uint32_t>(left) : lane_walks_of(L);
              }
            }
          }
          if (phase == kIdle && claim_left != 0u) {
            ++wid;
            --claim_left;
            start_walk();
          }
          s_claim[threadIdx.x] = claim_left;
        }
      }
    } else if (!exhausted && idle != 0u && (__popc(idle) >= L.refill || idle == full)) {
      unsigned long long base = 0;
      const int leader = __ffs(idle) - 1;
      if (static_cast<int>(lane) == leader)
        base = atomicAdd(L.counter, static_cast<unsigned long long>(__popc(idle)));
      base = __shfl_sync(full, base, leader);
      if (base + __popc(idle) >= L.total_walks) exhausted = true;
      if (phase == kIdle) {
        const uint64_t id = base + __popc(idle & ((1u << lane) - 1u));
        if (id < L.total_walks) {
          wid = id;
          start_walk();
        }
      }
    }

    // ---- batched walk step for lanes whose query has finished
    const unsigned ready = __ballot_sync(full, phase == kStep);
    const unsigned trav = __ballot_sync(full, phase == kTraverse);
    if (ready != 0u && (__popc(ready) >= L.step_threshold || trav == 0u) && phase == kStep) {
      const JobDesc &J = s_jobs[job];
      const GeoDesc &G = s_geos[J.geo];
      // One pass; `break` leaves it once the lane's next phase is set.
      do {
        T d = sqrt(best2);
        if (!found) {
          err |= TWOS_DEVERR_QUERY;
          d = T(0);  // ends the walk; the call reports the failure
        }
        const T R = to_T<T>(J.cavity_radius);
        const T dmesh = d;
        int hit_cav = -1;
        bool cav_nearer = false;  // gradient mode: the exit is on a cavity
        for (uint32_t c = 0; c < J.n_cav; ++c) {
          const Vec<T> cc = to_frame<T>(L.cavities + 3ull * (J.cav_begin + c), G);
          const Vec<T> dv = sub(pos, cc);
          const T len = sqrt(dot3(dv, dv));
          const T dc = len - R;
          if (MODE == kModeBoundary) {
            // closest_boundary (wih_twos.cpp:612-624): the first strictly nearer cavity.
            if (dc < d && len > T(0)) {
              d = dc;
              hit_cav = static_cast<int>(c);
            }
          } else {
            d = dc < d ? dc : d;
            if (GRAD && dc < dmesh) cav_nearer = true;
          }
        }
        // The mixed form shrinks the radius by the FP32 distance error bound;
        // the FP64 form uses the distance itself (wih_twos.cpp:645-647).
        const T r = sizeof(T) == 4 ? d - static_cast<T>(G.delta) : d;
        bool done = !(r > to_T<T>(J.epsilon));
        bool cap = false;
        if (!done) {
          const uint32_t ctr3 = J.repeat << 3;
          const Philox4 q0 = philox(J.k0, J.k1, steps, walk, J.site_offset + site, ctr3 | 0u);
          Vec<T> a = pos;
          if (GREEN) {
            const Philox4 q1 = philox(J.k0, J.k1, steps, walk, J.site_offset + site, ctr3 | 1u);
            const Philox4 q2 = philox(J.k0, J.k1, steps, walk, J.site_offset + site, ctr3 | 2u);
            const Philox4 q3 = philox(J.k0, J.k1, steps, walk, J.site_offset + site, ctr3 | 3u);
            const T beta = median3(uniform<T>(q2.x, q2.y), uniform<T>(q2.z, q2.w), uniform<T>(q3.x, q3.y));
            const Vec<T> g = direction<T>(uniform<T>(q1.x, q1.y), uniform<T>(q1.z, q1.w));
            a = add_scaled(pos, g, r * beta);
          }
          if (EXACT) {
            u = exact_source(u, s_terms, J.src_begin, J.n_src, pos, r, err);
            if (PAIRED) pv = exact_source(pv, s_terms, J.adj_begin, J.n_adj, pos, r, err);
          } else {
            const T w = r * r / T(6);
            if (MODE != kModeBoundary) {
              const T du = w * source_value(s_terms, J.src_begin, J.n_src, a);
              u = u + du;
              if (GRAD && steps == 0) g_u0 = du;
            }
            if (PAIRED) {
              const T dp = w * source_value(s_terms, J.adj_begin, J.n_adj, a);
              pv = pv + dp;
              if (GRAD && steps == 0) g_p0 = dp;
            }
          }
          const Vec<T> dir = direction<T>(uniform<T>(q0.x, q0.y), uniform<T>(q0.z, q0.w));
          if (GRAD && steps == 0) {
            // First ball: the sphere term's radius and direction, and one draw
            // (blocks 4-5) for the ball source term of the gradient,
            // R (1 - t^3) f(x + t R w') w' with t ~ U(0,1), w' uniform.
            const Philox4 q4 = philox(J.k0, J.k1, 0u, walk, J.site_offset + site, ctr3 | 4u);
            const Philox4 q5 = philox(J.k0, J.k1, 0u, walk, J.site_offset + site, ctr3 | 5u);
            const T t = uniform<T>(q4.x, q4.y);
            const Vec<T> wp = direction<T>(uniform<T>(q4.z, q4.w), uniform<T>(q5.x, q5.y));
            const Vec<T> z = add_scaled(pos, wp, t * r);
            const T wt = r * (T(1) - t * t * t);
            const T fs = wt * source_value(s_terms, J.src_begin, J.n_src, z);
            const T fq = wt * source_value(s_terms, J.adj_begin, J.n_adj, z);
            g_su = {wp.x * fs, wp.y * fs, wp.z * fs};
            g_sp = {wp.x * fq, wp.y * fq, wp.z * fq};
            g_r0 = r;
            g_w0 = dir;
          }
          pos = add_scaled(pos, dir, r);
          ++steps;
          if (static_cast<int>(steps) >= J.max_steps) {
            done = true;
            cap = true;
          }
        }
        if (done) {
          if (MODE == kModeBoundary) {
            HitRec h;
            h.pad = 0;
            Vec<T> q{T(0), T(0), T(0)}, nrm{T(0), T(0), T(0)};
            if (cap || !found) {
              h.cavity = -2;
            } else if (hit_cav >= 0) {
              // Point on the sphere along the radial direction; the domain
              // excludes the sphere, so the outward normal points into it.
              const Vec<T> cc = to_frame<T>(L.cavities + 3ull * (J.cav_begin + hit_cav), G);
              const Vec<T> dv = sub(pos, cc);
              const T inv = T(1) / sqrt(dot3(dv, dv));
              const Vec<T> dir{dv.x * inv, dv.y * inv, dv.z * inv};
              q = add_scaled(cc, dir, R);
              nrm = {dir.x * T(-1), dir.y * T(-1), dir.z * T(-1)};
              h.cavity = hit_cav;
            } else {
              Vec<T> ta, tb, tc;
              load_tri(geo_tris<T>(G), best_tri, ta, tb, tc);
              q = tri_closest(pos, ta, tb, tc);
              if (dmesh > T(0)) {
                const T inv = T(1) / dmesh;
                const Vec<T> dq = sub(q, pos);
                nrm = {dq.x * inv, dq.y * inv, dq.z * inv};
              }
              h.cavity = -1;
            }
            const bool f32 = sizeof(T) == 4;
            h.point[0] = static_cast<double>(q.x) + (f32 ? G.center[0] : 0.0);
            h.point[1] = static_cast<double>(q.y) + (f32 ? G.center[1] : 0.0);
            h.point[2] = static_cast<double>(q.z) + (f32 ? G.center[2] : 0.0);
            h.normal[0] = static_cast<double>(nrm.x);
            h.normal[1] = static_cast<double>(nrm.y);
            h.normal[2] = static_cast<double>(nrm.z);
            L.hits[wid] = h;
          } else {
            if (GRAD) {
              // Dirichlet data of u at the exit point on the mesh.
              if (!cap && found && J.n_bnd > 0 && !cav_nearer) {
                Vec<T> q = pos;
                if (tri_ok) {
                  Vec<T> ta, tb, tc;
                  load_tri(geo_tris<T>(G), best_tri, ta, tb, tc);
                  q = tri_closest(pos, ta, tb, tc);
                }
                u = u + source_value(s_terms, J.bnd_begin, J.n_bnd, q);
              }
              T *go = static_cast<T *>(L.grad_out) + 6ull * wid;
              if (g_r0 > T(0)) {
                const T k = T(3) / g_r0;
                const T cu = k * (u - g_u0), cp = k * (pv - g_p0);
                go[0] = g_w0.x * cu + g_su.x;
                go[1] = g_w0.y * cu + g_su.y;
                go[2] = g_w0.z * cu + g_su.z;
                go[3] = g_w0.x * cp + g_sp.x;
                go[4] = g_w0.y * cp + g_sp.y;
                go[5] = g_w0.z * cp + g_sp.z;
              } else {
                for (int k = 0; k < 6; ++k) go[k] = T(0);
              }
            }
            static_cast<T *>(L.u_out)[wid] = u;
          }
          if (PAIRED) static_cast<T *>(L.p_out)[wid] = pv;
          L.steps_out[wid] = steps | (cap ? 0x80000000u : 0u);
          phase = kIdle;
          break;
        }
        best2 = static_cast<T>(J.query_radius2);
        found = false;
        node = 0;
        if constexpr (sizeof(T) == 4) {
          // Distance-bound grid: D(v) - |x - v| over the corners v of x's cell
          // bounds the mesh distance from below; a bound of at least grid_tau
          // spacings is the next ball's radius and no query is needed.  A grid
          // step never ends a walk: the bound must clear the termination
          // shell with room to spare.
          float bound, upper = CUDART_INF_F;
          int entry_node = -1;
          const bool in_grid = (L.grid_tau > 0.f || L.entry) && G.grid && grid_bounds(G, pos, bound, upper, entry_node);
          if (in_grid && L.grid_tau > 0.f && bound >= L.grid_tau * G.grid_h &&
              bound > 2.f * (static_cast<float>(J.epsilon) + G.delta) && bound * bound < best2) {
            best2 = bound * bound;
            found = true;
            ++c_grid;
            if constexpr (TRACE) {
              const unsigned long long slot = atomicAdd(L.trace_count, 1ull);
              if (slot < L.trace_cap) L.trace[slot] = make_float4(pos.x, pos.y, pos.z, bound);
            }
            // The step itself comes with the warp's next batch.
            break;
          }
          if (!(in_grid && L.entry)) entry_node = -1;
          if (L.warm && tri_ok) {
            Vec<T> ta, tb, tc;
            load_tri(geo_tris<T>(G), best_tri, ta, tb, tc);
            ++c_tris;
            const T w2 = tri_dist2(pos, ta, tb, tc);
            if (w2 < best2) {
              best2 = w2;
              found = true;
            }
          }
          // Entry node: with an initial bound b below one entry cell, every
          // triangle outside the cell's entry subtree is farther than b (the
          // table keeps every triangle within a cell size plus 4 delta), so
          // the traversal starts there.  The grid's upper bound plus 6 delta
          // (its 3 delta and the FP32 query's delta, with room) may serve as
          // b before any triangle is found.  (The four-wide form keeps the
          // bound but starts at its root: the table holds binary nodes.)
          if (entry_node >= 0) {
            const float ubs = upper + 6.f * G.delta;
            if (fminf(sqrtf(best2), ubs) < G.entry_radius) {
              if (!WIDE) node = entry_node;
              if (ubs * ubs < best2) best2 = ubs * ubs;
            }
          }
        } else {
          // FP64 form.  With GRID64 it takes the same grid steps and entry
          // nodes as the mixed form (a comparison of precision alone): the
          // bound is evaluated at the FP32 image p32 of the position, within
          // a few 1e-8 of it, and bound <= d(p32) - delta covers that.
          float bound = 0.f, upper = CUDART_INF_F;
          int entry_node = -1;
          bool in_grid = false;
          if constexpr (GRID64) {
            const double p3[3] = {pos.x, pos.y, pos.z};
            in_grid = L.grid_tau > 0.f && G.grid && grid_bounds(G, to_frame<float>(p3, G), bound, upper, entry_node);
            const double b = static_cast<double>(bound);
            if (in_grid && bound >= L.grid_tau * G.grid_h && bound > 2.f * (static_cast<float>(J.epsilon) + G.delta) &&
                b * b < best2) {
              best2 = b * b;
              found = true;
              ++c_grid;
              break;
            }
          }
          if (L.warm && tri_ok) {
            Vec<T> ta, tb, tc;
            load_tri(geo_tris<T>(G), best_tri, ta, tb, tc);
            ++c_tris;
            const T w2 = tri_dist2(pos, ta, tb, tc);
            if (w2 < best2) {
              best2 = w2;
              found = true;
            }
          }
          if constexpr (GRID64) {
            if (in_grid && L.entry && entry_node >= 0) {
              const double ubs = static_cast<double>(upper) + 6.0 * G.delta;
              if (fmin(sqrt(best2), ubs) < static_cast<double>(G.entry_radius)) {
                node = entry_node;
                if (ubs * ubs < best2) best2 = ubs * ubs;
              }
            }
          }
        }
        sp = 0;
        have = true;
        narrow = false;
        tri_cur = tri_end = 0;
        iter = 0;
        phase = kTraverse;
        break;
      } while (false);
    }

    if (__ballot_sync(full, phase != kIdle) == 0u) {
      if (exhausted && (!CLAIM || __ballot_sync(full, s_claim[threadIdx.x] != 0u) == 0u)) break;
      continue;
    }

    // ---- one unit of closest-point traversal.  The warp runs one kind of
    // unit per iteration -- triangle tests or node tests/pops -- whichever
    // more of its traversing lanes need, so each iteration executes one code
    // path instead of the union of both.
    bool take = phase == kTraverse;
    if (L.vote) {  // warp-uniform; the ballots cost nothing when it is off
      const bool want_tri = phase == kTraverse && tri_cur < tri_end;
      const unsigned vt = __ballot_sync(full, want_tri);
      const unsigned vn = __ballot_sync(full, phase == kTraverse && !want_tri);
      const bool tri_turn = __popc(vt) >= __popc(vn);
      take = take && want_tri == tri_turn;
    }
    if (take) {
      const GeoDesc &G = s_geos[s_jobs[job].geo];
      // Up to `units` units back to back before the warp returns to the
      // refill and step ballots: the loop overhead is paid once per batch.
#pragma unroll 1
      for (int unit = 0; unit < units && phase == kTraverse; ++unit) {
        if (++iter > G.max_iter) {
          err |= TWOS_DEVERR_ITER;
          found = false;
          phase = kStep;
        } else if (tri_cur < tri_end) {
          const typename Layout<T>::Tri *tris = geo_tris<T>(G);
          ++c_planes;
          if (tri_test(tris, tri_cur, pos, best2, c_tris)) {
            found = true;
            best_tri = tri_cur;
            tri_ok = true;
          }
          ++tri_cur;
        } else {
          // Pop the next entry still closer than the current best.
          while (!have && sp > 0) {
            --sp;
            const uint2 e = stack[sp * BLOCK];
            if (static_cast<T>(__uint_as_float(e.y)) < best2) {
              node = static_cast<int>(e.x);
              have = true;
            }
          }
          if (!have) {
            phase = kStep;
          } else {
            if constexpr (WIDE) {
              if (node >= 0 && !narrow) {
                // Four-wide node: its valid children sorted nearest first (a
                // five-comparator network); the nearest is next, the others
                // are pushed farthest first.
                ++c_nodes;
                float d[4];
                int c[4];
                node4_dist2(G.nodes4_f, node, pos, d, c);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                  if (!(d[k] < best2)) d[k] = CUDART_INF_F;
                order2(d[0], c[0], d[1], c[1]);
                order2(d[2], c[2], d[3], c[3]);
                order2(d[0], c[0], d[2], c[2]);
                order2(d[1], c[1], d[3], c[3]);
                order2(d[1], c[1], d[2], c[2]);
                const int nv = (d[0] < CUDART_INF_F) + (d[1] < CUDART_INF_F) + (d[2] < CUDART_INF_F) +
                               (d[3] < CUDART_INF_F);
                if (nv == 0) {
                  have = false;
                } else if (sp + nv - 1 > kStack) {
                  // Up to three pushes per level can outgrow the stack on a
                  // root-started query with a loose bound.  The query goes
                  // on from the binary root with the bound found so far
                  // (one push per level there): every triangle nearer than
                  // best2 is still reached.
                  narrow = true;
                  sp = 0;
                  node = 0;
                } else {
                  if (nv > 3) stack[(sp++) * BLOCK] = make_uint2(static_cast<uint32_t>(c[3]), __float_as_uint(d[3]));
                  if (nv > 2) stack[(sp++) * BLOCK] = make_uint2(static_cast<uint32_t>(c[2]), __float_as_uint(d[2]));
                  if (nv > 1) stack[(sp++) * BLOCK] = make_uint2(static_cast<uint32_t>(c[1]), __float_as_uint(d[1]));
                  node = c[0];
                }
              }
            }
            if (!WIDE || narrow) {
              if (node >= 0) {
                ++c_nodes;
                T dl, dr;
                int cl, cr;
                node_dist2(geo_nodes<T>(G), node, pos, dl, dr, cl, cr);
                const bool vl = dl < best2, vr = dr < best2;
                if (vl && vr) {
                  if (dr < dl) {
                    const T td = dl;
                    dl = dr;
                    dr = td;
                    const int tc = cl;
                    cl = cr;
                    cr = tc;
                  }
                  if (sp >= kStack) {
                    err |= TWOS_DEVERR_STACK;
                    found = false;
                    phase = kStep;
                  } else {
                    stack[sp * BLOCK] = make_uint2(static_cast<uint32_t>(cr), __float_as_uint(lower_f(dr)));
                    ++sp;
                    node = cl;
                  }
                } else if (vl) {
                  node = cl;
                } else if (vr) {
                  node = cr;
                } else {
                  have = false;
                }
              }
            }
            // A leaf reached by this unit's visit or pop: its triangle range
            // is taken in the same unit, so the next unit tests a triangle.
            if (have && node < 0 && phase == kTraverse) {
              const uint32_t enc = ~static_cast<uint32_t>(node);
              tri_cur = enc >> 3;
              tri_end = tri_cur + (enc & 7u);
              have = false;
            }
          }
        }
      }
    }
  }
  if (err) atomicOr(L.error, err);
  if (L.counters) {
    unsigned long long n_nodes = c_nodes, n_planes = c_planes, n_tris = c_tris, n_grid = c_grid;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      n_nodes += __shfl_xor_sync(full, n_nodes, o);
      n_planes += __shfl_xor_sync(full, n_planes, o);
      n_tris += __shfl_xor_sync(full, n_tris, o);
      n_grid += __shfl_xor_sync(full, n_grid, o);
    }
    if (lane == 0) {
      atomicAdd(&L.counters[0], n_nodes);
      atomicAdd(&L.counters[1], n_planes);
      atomicAdd(&L.counters[2], n_tris);
      if (n_grid) atomicAdd(&L.counters[3], n_grid);
    }
  }
}

// Per-site first query: one closest-point traversal per site of the launch
// (the N walks of a site all start there), written as the squared mesh
// distance, or -1 when no surface point lies within the query radius.
template <typename T>
__global__ void __launch_bounds__(kWosBlock) site_prepass_kernel(const WosLaunch L) {
  __shared__ uint2 s_stack[kStack * kWosBlock];
  uint2 *stack = s_stack + threadIdx.x;
  uint32_t err = 0;
  T *out = static_cast<T *>(L.site_best2);
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < L.total_sites; g += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = L.n_jobs - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (L.jobs[mid].site_rank <= g)
        lo = mid;
      else
        hi = mid - 1;
    }
    const JobDesc &J = L.jobs[lo];
    const GeoDesc &G = L.geos[J.geo];
    const Vec<T> p = to_frame<T>(L.sites + 3ull * (J.site_begin + (g - J.site_rank)), G);
    T best2 = static_cast<T>(J.query_radius2);
    uint32_t tri = 0;
    const bool found = nearest<T>(geo_nodes<T>(G), geo_tris<T>(G), G.max_iter, p, best2, tri, stack, kWosBlock, err);
    out[g] = found ? best2 : T(-1);
  }
  if (err) atomicOr(L.error, err);
}

cudaError_t launch_site_prepass(int precision, const WosLaunch &L, cudaStream_t s) {
  if (!L.site_best2 || L.total_sites == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint32_t>((L.total_sites + kWosBlock - 1) / kWosBlock, 148u * 16));
  if (precision == TWOS_PREC_MIXED)
    site_prepass_kernel<float><<<grid, kWosBlock, 0, s>>>(L);
  else
    site_prepass_kernel<double><<<grid, kWosBlock, 0, s>>>(L);
  return cudaGetLastError();
}

template <typename T, int MODE, int SRC, int BLOCK> static const void *wos_fn() {
  return reinterpret_cast<const void *>(&wos_kernel<T, MODE, SRC, BLOCK>);
}

template <typename T, int MODE, int BLOCK> static const void *select_src(int src) {
  if (src == TWOS_SOURCE_GREEN) return wos_fn<T, MODE, TWOS_SOURCE_GREEN, BLOCK>();
  if (src == TWOS_SOURCE_EXACT) return wos_fn<T, MODE, TWOS_SOURCE_EXACT, BLOCK>();
  return wos_fn<T, MODE, TWOS_SOURCE_CENTER, BLOCK>();
}

template <int MODE, int BLOCK> static const void *select_wide_src(int src) {
  if (src == TWOS_SOURCE_GREEN)
    return reinterpret_cast<const void *>(&wos_kernel<float, MODE, TWOS_SOURCE_GREEN, BLOCK, false, false, true>);
  return reinterpret_cast<const void *>(&wos_kernel<float, MODE, TWOS_SOURCE_CENTER, BLOCK, false, false, true>);
}

template <int MODE, int BLOCK> static const void *claim_fn() {
  return reinterpret_cast<const void *>(
      &wos_kernel<float, MODE, TWOS_SOURCE_CENTER, BLOCK, false, false, false, true>);
}

template <int BLOCK>
static const void *select_wos_block(int precision, int mode, int src, int grid64, int wide, int claim) {
  // Walk claims (lane_walks > 1): the mixed centre-source modes on the binary BVH.
  if (claim && !wide && precision == TWOS_PREC_MIXED && src == TWOS_SOURCE_CENTER) {
    if (mode == TWOS_MODE_COMPLIANCE) return claim_fn<TWOS_MODE_COMPLIANCE, BLOCK>();
    if (mode == TWOS_MODE_PAIRED) return claim_fn<TWOS_MODE_PAIRED, BLOCK>();
    if (mode == TWOS_MODE_HOT) return claim_fn<TWOS_MODE_HOT, BLOCK>();
  }
  if (wide && precision == TWOS_PREC_MIXED && (src == TWOS_SOURCE_CENTER || src == TWOS_SOURCE_GREEN)) {
    if (mode == TWOS_MODE_COMPLIANCE) return select_wide_src<TWOS_MODE_COMPLIANCE, BLOCK>(src);
    if (mode == TWOS_MODE_PAIRED) return select_wide_src<TWOS_MODE_PAIRED, BLOCK>(src);
    if (mode == TWOS_MODE_HOT) return select_wide_src<TWOS_MODE_HOT, BLOCK>(src);
  }
  if (grid64 && precision == TWOS_PREC_FP64 && mode == TWOS_MODE_COMPLIANCE && src == TWOS_SOURCE_CENTER)
    return reinterpret_cast<const void *>(
        &wos_kernel<double, TWOS_MODE_COMPLIANCE, TWOS_SOURCE_CENTER, BLOCK, false, true>);
  if (mode == kModeBoundary)
    return precision == TWOS_PREC_MIXED ? wos_fn<float, kModeBoundary, TWOS_SOURCE_CENTER, BLOCK>()
                                        : wos_fn<double, kModeBoundary, TWOS_SOURCE_CENTER, BLOCK>();
#define TWOS_PICK(T)                                                                 \
  if (mode == TWOS_MODE_COMPLIANCE) return select_src<T, TWOS_MODE_COMPLIANCE, BLOCK>(src); \
  if (mode == TWOS_MODE_PAIRED) return select_src<T, TWOS_MODE_PAIRED, BLOCK>(src);         \
  if (mode == kModeGradient) return select_src<T, kModeGradient, BLOCK>(src);               \
  return select_src<T, TWOS_MODE_HOT, BLOCK>(src);
  if (precision == TWOS_PREC_MIXED) {
    TWOS_PICK(float)
  }
  TWOS_PICK(double)
#undef TWOS_PICK
}

// Walk kernel instantiations: block sizes 128, 256 and 512 threads.
static const void *select_wos(int precision, int mode, int src, int block, int grid64, int wide, int claim) {
  switch (block) {
    case 128:
      return select_wos_block<128>(precision, mode, src, grid64, wide, claim);
    case 256:
      return select_wos_block<256>(precision, mode, src, grid64, wide, claim);
    case 512:
      return select_wos_block<512>(precision, mode, src, grid64, wide, claim);
    default:
      return nullptr;
  }
}

static uint32_t wos_dyn_smem(int precision, const WosLaunch &L, int block) {
  const uint32_t stack = static_cast<uint32_t>(kStack * block * sizeof(uint2));
  return stack + (precision == TWOS_PREC_MIXED ? smem_plan<float>(L.n_jobs, L.n_geos, L.n_terms).bytes
                                               : smem_plan<double>(L.n_jobs, L.n_geos, L.n_terms).bytes);
}

// The mixed compliance walk kernel (centre source, 128 threads) with a
// record of every grid step's position and bound (L.trace): used by tests to
// check each bound against the FP64 distance.
cudaError_t launch_wos_traced(const WosLaunch &L, int grid, cudaStream_t s) {
  if (L.n_jobs == 0 || L.n_geos == 0 || !L.trace || !L.trace_count) return cudaErrorInvalidValue;
  const uint32_t dyn = wos_dyn_smem(TWOS_PREC_MIXED, L, kWosBlock);
  const void *fn = reinterpret_cast<const void *>(&wos_kernel<float, TWOS_MODE_COMPLIANCE, TWOS_SOURCE_CENTER,
                                                              kWosBlock, true>);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn));
  if (e != cudaSuccess) return e;
  WosLaunch copy = L;
  void *args[] = {&copy};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kWosBlock), args, dyn, s);
}

cudaError_t launch_wos(int precision, int mode, int src, const WosLaunch &L, int grid, int block,
                       cudaStream_t s) {
  if (L.n_jobs == 0 || L.n_geos == 0) return cudaErrorInvalidValue;
  const uint32_t dyn = wos_dyn_smem(precision, L, block);
  if (dyn > 200 * 1024) return cudaErrorInvalidValue;
  const void *fn = select_wos(precision, mode, src, block, L.grid64, L.wide, L.lane_walks > 1);
  if (!fn) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn));
  if (e != cudaSuccess) return e;
  WosLaunch copy = L;
  void *args[] = {&copy};
  return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, dyn, s);
}

int wos_max_blocks_per_sm(int precision, int mode, int src, int block, const WosLaunch &L) {
  const uint32_t dyn = wos_dyn_smem(precision, L, block);
  const void *fn = select_wos(precision, mode, src, block, L.grid64, L.wide, L.lane_walks > 1);
  if (!fn || dyn > 200 * 1024) return 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn)) != cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block, dyn) != cudaSuccess) return 0;
  return n;
}

// ================================================================ finalize
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename V, int MODE>
__global__ void __launch_bounds__(256) finalize_kernel(const FinalizeLaunch F) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t g = warp; g < F.total_sites; g += nwarps) {
    // Job of launch site g (jobs ordered by site_rank).
    uint32_t lo = 0, hi = F.n_jobs - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (F.jobs[mid].site_rank <= g)
        lo = mid;
      else
        hi = mid - 1;
    }
    const JobDesc &J = F.jobs[lo];
    const uint32_t s = g - J.site_rank;
    const uint64_t base = J.walk_begin + static_cast<uint64_t>(s) * J.walks;
    const V *U = static_cast<const V *>(F.u) + base;
    const V *P = static_cast<const V *>(F.p) + base;
    const uint32_t *S = F.steps + base;
    const uint32_t n = J.walks;
    const double nd = static_cast<double>(n);
    double a = 0.0, b = 0.0, c = 0.0;
    unsigned long long st = 0, caps = 0;
    for (uint32_t w = lane; w < n; w += 32) {
      const double x = static_cast<double>(U[w]);
      const uint32_t sw = S[w];
      st += sw & 0x7fffffffu;
      caps += sw >> 31;
      if (MODE == TWOS_MODE_PAIRED) {
        const double y = static_cast<double>(P[w]);
        a += x;
        b += y;
        c += x * y;
      } else {
        a += x;
        b += x * x;
      }
    }
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    st = warp_sum_u64(st);
    caps = warp_sum_u64(caps);
    twos_site_result r;
    r.steps = st;
    r.caps = caps;
    // Leave-one-out values, their mean and spread (two more passes over the
    // samples, which are L2-resident at this point).
    double lsum = 0.0;
    for (uint32_t w = lane; w < n; w += 32) {
      const double x = static_cast<double>(U[w]);
      double leave;
      if (MODE == TWOS_MODE_COMPLIANCE) {
        const double ls = a - x, ls2 = b - x * x;
        leave = (ls * ls - ls2) / ((nd - 1.0) * (nd - 2.0));
      } else if (MODE == TWOS_MODE_PAIRED) {
        const double y = static_cast<double>(P[w]);
        leave = ((a - x) * (b - y) - (c - x * y)) / ((nd - 1.0) * (nd - 2.0));
      } else {
        leave = (a - x) / (nd - 1.0);
      }
      lsum += leave;
    }
    const double lmean = warp_sum(lsum) / nd;
    double spread = 0.0;
    for (uint32_t w = lane; w < n; w += 32) {
      const double x = static_cast<double>(U[w]);
      double leave;
      if (MODE == TWOS_MODE_COMPLIANCE) {
        const double ls = a - x, ls2 = b - x * x;
        leave = (ls * ls - ls2) / ((nd - 1.0) * (nd - 2.0));
      } else if (MODE == TWOS_MODE_PAIRED) {
        const double y = static_cast<double>(P[w]);
        leave = ((a - x) * (b - y) - (c - x * y)) / ((nd - 1.0) * (nd - 2.0));
      } else {
        leave = (a - x) / (nd - 1.0);
      }
      const double dv = leave - lmean;
      spread += dv * dv;
    }
    spread = warp_sum(spread);
    const double se = n >= 4 ? sqrt((nd - 1.0) / nd * spread) : CUDART_NAN;
    if (MODE == TWOS_MODE_COMPLIANCE) {
      r.u = a / nd;
      r.p = r.u;
      r.score = (a * a - b) / (nd * (nd - 1.0));
      r.same_index = b / nd;
    } else if (MODE == TWOS_MODE_PAIRED) {
      r.u = a / nd;
      r.p = b / nd;
      r.score = (a * b - c) / (nd * (nd - 1.0));
      r.same_index = c / nd;
    } else {
      r.u = a / nd;
      r.p = 0.0;
      r.score = a / nd;
      r.same_index = 0.0;
    }
    r.score_se = se;
    if (lane == 0) {
      F.out[J.site_begin + s] = r;
      if (F.totals) {
        atomicAdd(&F.totals[0], st);
        atomicAdd(&F.totals[1], caps);
      }
    }
  }
}

// Gradient mode: one warp per site (warp_sum: a fixed xor-tree order).  Pass 1: sums of u, p, grad u, grad p
// and grad u . grad p; pass 2: the leave-one-out cross statistics and their
// mean; pass 3: the jackknife variance.  FP64 throughout.
template <typename V> __global__ void __launch_bounds__(256) grad_finalize_kernel(const GradFinalizeLaunch F) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  const V *u = static_cast<const V *>(F.u), *p = static_cast<const V *>(F.p), *g = static_cast<const V *>(F.grad);
  const uint32_t N = F.walks;
  const double n = static_cast<double>(N);
  for (uint64_t site = warp; site < F.n_sites; site += nwarps) {
    const uint64_t base = site * N;
    double su = 0, sp = 0, sgu[3] = {0, 0, 0}, sgp[3] = {0, 0, 0}, sdot = 0;
    unsigned long long steps = 0, caps = 0;
    for (uint32_t w = lane; w < N; w += 32) {
      const uint64_t i = base + w;
      su += static_cast<double>(u[i]);
      sp += static_cast<double>(p[i]);
      double d = 0;
      for (int k = 0; k < 3; ++k) {
        const double a = static_cast<double>(g[6 * i + k]), b = static_cast<double>(g[6 * i + 3 + k]);
        sgu[k] += a;
        sgp[k] += b;
        d += a * b;
      }
      sdot += d;
      const uint32_t st = F.steps[i];
      steps += st & 0x7fffffffu;
      caps += st >> 31;
    }
    su = warp_sum(su);
    sp = warp_sum(sp);
    for (int k = 0; k < 3; ++k) {
      sgu[k] = warp_sum(sgu[k]);
      sgp[k] = warp_sum(sgp[k]);
    }
    sdot = warp_sum(sdot);
    const double den = n * (n - 1.0);
    const double cross = (sgu[0] * sgp[0] + sgu[1] * sgp[1] + sgu[2] * sgp[2] - sdot) / den;
    // Leave-one-out: ((S_u - g_i).(S_p - h_i) - (S_dot - g_i.h_i)) / ((N-1)(N-2)).
    const double den1 = (n - 1.0) * (n - 2.0);
    double s1 = 0, s2 = 0;
    if (N > 2) {
      for (uint32_t w = lane; w < N; w += 32) {
        const uint64_t i = base + w;
        double a[3], b[3], d = 0;
        for (int k = 0; k < 3; ++k) {
          a[k] = static_cast<double>(g[6 * i + k]);
          b[k] = static_cast<double>(g[6 * i + 3 + k]);
          d += a[k] * b[k];
        }
        const double c = ((sgu[0] - a[0]) * (sgp[0] - b[0]) + (sgu[1] - a[1]) * (sgp[1] - b[1]) +
                          (sgu[2] - a[2]) * (sgp[2] - b[2]) - (sdot - d)) / den1;
        s1 += c;
      }
      s1 = warp_sum(s1);
      const double mean = s1 / n;
      for (uint32_t w = lane; w < N; w += 32) {
        const uint64_t i = base + w;
        double a[3], b[3], d = 0;
        for (int k = 0; k < 3; ++k) {
          a[k] = static_cast<double>(g[6 * i + k]);
          b[k] = static_cast<double>(g[6 * i + 3 + k]);
          d += a[k] * b[k];
        }
        const double c = ((sgu[0] - a[0]) * (sgp[0] - b[0]) + (sgu[1] - a[1]) * (sgp[1] - b[1]) +
                          (sgu[2] - a[2]) * (sgp[2] - b[2]) - (sdot - d)) / den1;
        s2 += (c - mean) * (c - mean);
      }
      s2 = warp_sum(s2);
    }
    // Standard errors of the means of u and p (two-pass sample variance).
    const double mu = su / n, mp = sp / n;
    double vu = 0, vp = 0;
    for (uint32_t w = lane; w < N; w += 32) {
      const double du = static_cast<double>(u[base + w]) - mu, dp = static_cast<double>(p[base + w]) - mp;
      vu += du * du;
      vp += dp * dp;
    }
    vu = warp_sum(vu);
    vp = warp_sum(vp);
    for (int o = 16; o > 0; o >>= 1) {
      steps += __shfl_xor_sync(0xffffffffu, steps, o);
      caps += __shfl_xor_sync(0xffffffffu, caps, o);
    }
    if (lane == 0) {
      twos_gradient_result r;
      r.u = su / n;
      r.p = sp / n;
      for (int k = 0; k < 3; ++k) {
        r.grad_u[k] = sgu[k] / n;
        r.grad_p[k] = sgp[k] / n;
      }
      r.cross = cross;
      r.cross_se = N > 2 ? sqrt((n - 1.0) / n * s2) : 0.0;
      r.steps = steps;
      r.caps = caps;
      r.u_se = N > 1 ? sqrt(vu / (n * (n - 1.0))) : 0.0;
      r.p_se = N > 1 ? sqrt(vp / (n * (n - 1.0))) : 0.0;
      F.out[site] = r;
      atomicAdd(&F.totals[0], steps);
      atomicAdd(&F.totals[1], caps);
    }
  }
}

cudaError_t launch_grad_finalize(int precision, const GradFinalizeLaunch &F, cudaStream_t s) {
  if (F.n_sites == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint64_t>((static_cast<uint64_t>(F.n_sites) * 32 + 255) / 256,
                                                       148ull * 16));
  if (precision == TWOS_PREC_MIXED)
    grad_finalize_kernel<float><<<grid, 256, 0, s>>>(F);
  else
    grad_finalize_kernel<double><<<grid, 256, 0, s>>>(F);
  return cudaGetLastError();
}

cudaError_t launch_finalize(int precision, int mode, const FinalizeLaunch &F, cudaStream_t s) {
  if (F.total_sites == 0) return cudaSuccess;
  const int block = 256;
  const uint64_t warps = F.total_sites;
  int grid = static_cast<int>(std::min<uint64_t>((warps * 32 + block - 1) / block, 148ull * 16));
  FinalizeLaunch copy = F;
  void *args[] = {&copy};
  const void *fn;
  if (precision == TWOS_PREC_MIXED) {
    fn = mode == TWOS_MODE_COMPLIANCE ? reinterpret_cast<const void *>(&finalize_kernel<float, 0>)
         : mode == TWOS_MODE_PAIRED   ? reinterpret_cast<const void *>(&finalize_kernel<float, 1>)
                                      : reinterpret_cast<const void *>(&finalize_kernel<float, 2>);
  } else {
    fn = mode == TWOS_MODE_COMPLIANCE ? reinterpret_cast<const void *>(&finalize_kernel<double, 0>)
         : mode == TWOS_MODE_PAIRED   ? reinterpret_cast<const void *>(&finalize_kernel<double, 1>)
                                      : reinterpret_cast<const void *>(&finalize_kernel<double, 2>);
  }
  return cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, s);
}

// ================================================================ L2 read probe
// Streams an L2-resident buffer with the walk kernel's load form (32-byte
// read-only vector loads, one per lane, consecutive lanes on consecutive
// sectors), `passes` times over.  The measured rate is the L2 read roof for a
// working set that fits the L2 (the distance grid and the BVH of one mesh).
__global__ void __launch_bounds__(256) l2_read_kernel(const float4 *__restrict__ buf, uint64_t n32, int passes,
                                                      uint32_t *sink) {
  float acc = 0.f;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (int p = 0; p < passes; ++p) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n32; i += stride) {
      float4 a, b;
      ldg32(buf + 2 * i, a, b);
      acc += (a.x + a.y + a.z + a.w) + (b.x + b.y + b.z + b.w);
    }
  }
  // The buffer holds zeros, so this store never happens; the compiler cannot
  // know that and keeps every load.
  if (acc != 0.f) sink[0] = __float_as_uint(acc);
}

cudaError_t launch_l2_read(const void *buf, uint64_t bytes, int passes, uint32_t *sink, int blocks, cudaStream_t s) {
  l2_read_kernel<<<blocks, 256, 0, s>>>(static_cast<const float4 *>(buf), bytes / 32, passes, sink);
  return cudaGetLastError();
}

// ================================================================ batched closest point
template <typename T>
__global__ void __launch_bounds__(kWosBlock) closest_kernel(const GeoDesc *geo, const double *pts, uint64_t n,
                                                            double query_radius2, double *dist, double *closest,
                                                            uint32_t *error) {
  __shared__ uint2 s_stack[kStack * kWosBlock];
  __shared__ GeoDesc G;
  if (threadIdx.x == 0) G = *geo;
  __syncthreads();
  uint32_t err = 0;
  uint2 *stack = s_stack + threadIdx.x;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const Vec<T> p = to_frame<T>(pts + 3 * i, G);
    T best2 = static_cast<T>(query_radius2);
    uint32_t best_tri = 0;
    const bool found =
        nearest<T>(geo_nodes<T>(G), geo_tris<T>(G), G.max_iter, p, best2, best_tri, stack, kWosBlock, err);
    dist[i] = found ? static_cast<double>(sqrt(best2)) : CUDART_INF;
    if (closest) {
      double q[3] = {CUDART_NAN, CUDART_NAN, CUDART_NAN};
      if (found) {
        Vec<T> a, b, c;
        load_tri(geo_tris<T>(G), best_tri, a, b, c);
        const Vec<T> cp = tri_closest(p, a, b, c);
        const bool f32 = sizeof(T) == 4;
        q[0] = static_cast<double>(cp.x) + (f32 ? G.center[0] : 0.0);
        q[1] = static_cast<double>(cp.y) + (f32 ? G.center[1] : 0.0);
        q[2] = static_cast<double>(cp.z) + (f32 ? G.center[2] : 0.0);
      }
      closest[3 * i] = q[0];
      closest[3 * i + 1] = q[1];
      closest[3 * i + 2] = q[2];
    }
  }
  if (err) atomicOr(error, err);
}

__global__ void ball_green_kernel(const double *__restrict__ cases, uint32_t n, double *__restrict__ out,
                                  uint32_t *error) {
  uint32_t err = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    bool negative = false;
    out[i] = exact_bump_green(cases[4ull * i], cases[4ull * i + 1], cases[4ull * i + 2], cases[4ull * i + 3],
                              negative);
    if (negative) err |= TWOS_DEVERR_SOURCE;
  }
  if (err) atomicOr(error, err);
}

cudaError_t launch_ball_green(const double *cases, uint32_t n, double *out, uint32_t *error, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint32_t>((n + 127) / 128, 148u * 8));
  ball_green_kernel<<<grid, 128, 0, s>>>(cases, n, out, error);
  return cudaGetLastError();
}

cudaError_t launch_closest(int precision, const GeoDesc *geo_dev, const double *pts, uint64_t n,
                           double query_radius2, double *dist, double *closest, uint32_t *error, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int block = kWosBlock;
  const int grid = static_cast<int>(std::min<uint64_t>((n + block - 1) / block, 148ull * 32));
  if (precision == TWOS_PREC_MIXED)
    closest_kernel<float><<<grid, block, 0, s>>>(geo_dev, pts, n, query_radius2, dist, closest, error);
  else
    closest_kernel<double><<<grid, block, 0, s>>>(geo_dev, pts, n, query_radius2, dist, closest, error);
  return cudaGetLastError();
}

// ================================================================ distance-bound grid
// One thread per grid vertex: its FP32 closest-point distance, less `margin`,
// rounded down to a multiple of grid_q and saturated at 65535 multiples.  A
// vertex whose query fails keeps 0 (a bound no step uses).
__global__ void __launch_bounds__(kWosBlock) grid_build_kernel(const GeoDesc *geo, double margin, uint16_t *out,
                                                               uint32_t *error) {
  __shared__ uint2 s_stack[kStack * kWosBlock];
  __shared__ GeoDesc G;
  if (threadIdx.x == 0) G = *geo;
  __syncthreads();
  uint32_t err = 0;
  uint2 *stack = s_stack + threadIdx.x;
  const uint64_t n = static_cast<uint64_t>(G.grid_n[0]) * G.grid_n[1] * G.grid_n[2];
  for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < n;
       v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t gk = static_cast<uint32_t>(v % G.grid_n[2]);
    const uint64_t ij = v / G.grid_n[2];
    const uint32_t gj = static_cast<uint32_t>(ij % G.grid_n[1]), gi = static_cast<uint32_t>(ij / G.grid_n[1]);
    const Vec<float> p = grid_vertex(G, gi, gj, gk);
    float best2 = CUDART_INF_F;
    uint32_t tri = 0;
    uint16_t q = 0;
    if (nearest<float>(geo_nodes<float>(G), geo_tris<float>(G), G.max_iter, p, best2, tri, stack, kWosBlock, err)) {
      const double m = floor((static_cast<double>(sqrtf(best2)) - margin) / static_cast<double>(G.grid_q));
      q = m <= 0.0 ? 0 : m >= 65535.0 ? 65535 : static_cast<uint16_t>(m);
    }
    out[v] = q;
  }
  if (err) atomicOr(error, err);
}

// The grid's lower bound at each point (original coordinates), NaN where the
// point lies outside the grid or the geometry has none.
__global__ void __launch_bounds__(256) grid_bound_kernel(const GeoDesc *geo, const double *pts, uint64_t n,
                                                         double *out) {
  const GeoDesc G = *geo;
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    float b = 0.f;
    out[i] = G.grid && grid_bound(G, to_frame<float>(pts + 3 * i, G), b) ? static_cast<double>(b) : CUDART_NAN;
  }
}

cudaError_t launch_grid_bound(const GeoDesc *geo_dev, const double *pts, uint64_t n, double *out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint64_t>((n + 255) / 256, 148ull * 16));
  grid_bound_kernel<<<grid, 256, 0, s>>>(geo_dev, pts, n, out);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) grid_pack_kernel(const uint16_t *__restrict__ v, uint32_t n0, uint32_t n1,
                                                         uint32_t n2, const int32_t *__restrict__ table,
                                                         uint32_t shift, uint32_t e1, uint32_t e2,
                                                         uint4 *__restrict__ cells) {
  const uint64_t m1 = n1 - 1, m2 = n2 - 1, count = static_cast<uint64_t>(n0 - 1) * m1 * m2;
  for (uint64_t cell = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; cell < count;
       cell += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t k = static_cast<uint32_t>(cell % m2);
    const uint64_t ij = cell / m2;
    const uint32_t j = static_cast<uint32_t>(ij % m1), i = static_cast<uint32_t>(ij / m1);
    uint32_t d[8], base = 0xffffu;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      d[c] = v[(static_cast<uint64_t>(i + (c >> 2)) * n1 + (j + ((c >> 1) & 1))) * n2 + (k + (c & 1))];
      base = min(base, d[c]);
    }
    // Byte offsets above the base; 255 for a saturated corner or one too far
    // above the base (the reader then uses the base: a lower bound still).
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const uint32_t off = d[c] == 0xffffu || d[c] - base > 254u ? 0xffu : d[c] - base;
      if (c < 4)
        lo |= off << (8 * c);
      else
        hi |= off << (8 * (c - 4));
    }
    const int32_t entry = table ? table[(static_cast<uint64_t>(i >> shift) * e1 + (j >> shift)) * e2 + (k >> shift)]
                                : -1;
    cells[cell] = make_uint4(lo, hi, base, static_cast<uint32_t>(entry));
  }
}

cudaError_t launch_grid_pack(const uint16_t *vertices, const uint32_t n[3], const int32_t *table, uint32_t shift,
                             const uint32_t entry_n[3], uint4 *cells, cudaStream_t s) {
  if (n[0] < 2 || n[1] < 2 || n[2] < 2) return cudaErrorInvalidValue;
  if (table && (((n[0] - 2) >> shift) >= entry_n[0] || ((n[1] - 2) >> shift) >= entry_n[1] ||
                ((n[2] - 2) >> shift) >= entry_n[2]))
    return cudaErrorInvalidValue;
  const uint64_t count = static_cast<uint64_t>(n[0] - 1) * (n[1] - 1) * (n[2] - 1);
  const int grid = static_cast<int>(std::min<uint64_t>((count + 255) / 256, 148ull * 64));
  grid_pack_kernel<<<grid, 256, 0, s>>>(vertices, n[0], n[1], n[2], table, shift, table ? entry_n[1] : 0,
                                        table ? entry_n[2] : 0, cells);
  return cudaGetLastError();
}

cudaError_t launch_grid_build(const GeoDesc *geo_dev, uint64_t n, double margin, uint16_t *out, uint32_t *error,
                              cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int block = kWosBlock;
  const int grid = static_cast<int>(std::min<uint64_t>((n + block - 1) / block, 148ull * 32));
  grid_build_kernel<<<grid, block, 0, s>>>(geo_dev, margin, out, error);
  return cudaGetLastError();
}

// ================================================================ top-k
// Keys compare by (value desc, index asc); NaN sorts last.
struct KeyIdx {
  double v;
  uint32_t i;
};
__device__ __forceinline__ bool before(const KeyIdx &a, const KeyIdx &b) {
  const bool an = isnan(a.v), bn = isnan(b.v);
  if (an != bn) return bn;
  if (a.v != b.v) return a.v > b.v;
  return a.i < b.i;
}

constexpr int kTopkTile = 2048;

// Sorts one tile of kTopkTile keys in shared memory (bitonic) and writes its
// first k entries.
__global__ void __launch_bounds__(1024) topk_tile_kernel(const double *keys, uint32_t n, uint32_t k,
                                                         KeyIdx *partial) {
  __shared__ double sv[kTopkTile];
  __shared__ uint32_t si[kTopkTile];
  const uint32_t base = blockIdx.x * kTopkTile;
  for (uint32_t t = threadIdx.x; t < kTopkTile; t += blockDim.x) {
    const uint32_t g = base + t;
    sv[t] = g < n ? keys[g] : -CUDART_INF;
    si[t] = g < n ? g : 0xffffffffu;
  }
  __syncthreads();
  for (uint32_t size = 2; size <= kTopkTile; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t t = threadIdx.x; t < kTopkTile / 2; t += blockDim.x) {
        const uint32_t pos = 2 * t - (t & (stride - 1));
        const uint32_t a = pos, b = pos + stride;
        const bool up = ((pos & size) == 0);
        const KeyIdx ka{sv[a], si[a]}, kb{sv[b], si[b]};
        const bool swap = up ? before(kb, ka) : before(ka, kb);
        if (swap) {
          sv[a] = kb.v;
          si[a] = kb.i;
          sv[b] = ka.v;
          si[b] = ka.i;
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t t = threadIdx.x; t < k; t += blockDim.x) partial[blockIdx.x * k + t] = {sv[t], si[t]};
}

// Merges the per-tile candidates by repeated selection of the best remaining
// (k <= 1024, candidates <= a few hundred thousand).
__global__ void __launch_bounds__(1024) topk_merge_kernel(const KeyIdx *partial, uint32_t m, uint32_t k,
                                                          uint32_t *index) {
  __shared__ KeyIdx red[32];
  __shared__ KeyIdx last;
  if (threadIdx.x == 0) last = {CUDART_INF, 0u};
  __syncthreads();
  for (uint32_t r = 0; r < k; ++r) {
    KeyIdx best{-CUDART_INF, 0xffffffffu};
    bool have = false;
    for (uint32_t t = threadIdx.x; t < m; t += blockDim.x) {
      const KeyIdx c = partial[t];
      if (c.i == 0xffffffffu) continue;
      if (r > 0 && !before(last, c)) continue;  // already taken
      if (!have || before(c, best)) {
        best = c;
        have = true;
      }
    }
    // Block reduction.
    for (int o = 16; o > 0; o >>= 1) {
      KeyIdx other{__shfl_xor_sync(0xffffffffu, best.v, o), __shfl_xor_sync(0xffffffffu, best.i, o)};
      if (other.i != 0xffffffffu && (best.i == 0xffffffffu || before(other, best))) best = other;
    }
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
      KeyIdx b2 = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : KeyIdx{-CUDART_INF, 0xffffffffu};
      for (int o = 16; o > 0; o >>= 1) {
        KeyIdx other{__shfl_xor_sync(0xffffffffu, b2.v, o), __shfl_xor_sync(0xffffffffu, b2.i, o)};
        if (other.i != 0xffffffffu && (b2.i == 0xffffffffu || before(other, b2))) b2 = other;
      }
      if (threadIdx.x == 0) {
        index[r] = b2.i;
        last = b2;
      }
    }
    __syncthreads();
  }
}

size_t topk_scratch_bytes(uint32_t n, uint32_t k) {
  const uint32_t tiles = (n + kTopkTile - 1) / kTopkTile;
  return static_cast<size_t>(tiles) * k * sizeof(KeyIdx);
}

cudaError_t launch_topk(const double *keys, uint32_t n, uint32_t k, uint32_t *index, void *scratch,
                        size_t scratch_bytes, cudaStream_t s) {
  if (n == 0 || k == 0) return cudaSuccess;
  if (k > 1024 || k > static_cast<uint32_t>(kTopkTile)) return cudaErrorInvalidValue;
  if (scratch_bytes < topk_scratch_bytes(n, k)) return cudaErrorInvalidValue;
  const uint32_t tiles = (n + kTopkTile - 1) / kTopkTile;
  KeyIdx *partial = static_cast<KeyIdx *>(scratch);
  topk_tile_kernel<<<tiles, 1024, 0, s>>>(keys, n, k, partial);
  topk_merge_kernel<<<1, 1024, 0, s>>>(partial, tiles * k, k, index);
  return cudaGetLastError();
}

}  // namespace twos

// Differential WoS kernels (use nearest<double> above).
#include "diffwos.cuh"

// Certified validation kernels (use the stream, direction and nearest<double> above).
#include "validate.cuh"

// Array-RQMC / matched MC lockstep walks (use nearest<T>, the stream and warp sums above).
#include "rqmc.cuh"

#include "wavefront.cuh"

// Differential WoS on the device: derivatives of u at probe sites with respect
// to each spherical cavity's centre and radius (evaluate_differential_site,
// benchmarks/compiled_bunny/src/wih_twos.cpp:839-928).
//
//   1. outer walks to the boundary   wos_kernel<T, kModeBoundary>  (kernels.cu)
//   2. diff_classify_kernel          per walk that ended on a cavity: the
//                                    offset point x - l n, its seam and
//                                    segment safety and ray-parity membership
//                                    (classify_offset_safety, 765-837), and
//                                    the nested walk's start point
//   3. nested walks                  wos_kernel<T, compliance> from those points
//   4. diff_reduce_kernel            per site, in walk order: samples
//                                    n u/l (centre) and -u/l (radius) per
//                                    cavity, means and standard errors
//                                    (891-926)
//
// Ray parity and the classification run in FP64 on the FP64 BVH in both
// precision forms; they touch only walks that end on a cavity.
//
// Included at the end of kernels.cu (one translation unit, so these kernels
// call its traversal functions without relocatable device code).
#pragma once

namespace twos {

namespace {

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double normd(D3 a) { return sqrt(dotd(a, a)); }
__device__ __forceinline__ double comp(D3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// Moller-Trumbore ray/triangle intersection (Moller & Trumbore 1997), FP64;
// returns the hit parameter or -1.
__device__ double ray_triangle(D3 o, D3 d, D3 a, D3 b, D3 c) {
  const D3 e1 = b - a, e2 = c - a;
  const D3 pv{d.y * e2.z - d.z * e2.y, d.z * e2.x - d.x * e2.z, d.x * e2.y - d.y * e2.x};
  const double det = dotd(e1, pv);
  if (det == 0.0) return -1.0;
  const double inv = 1.0 / det;
  const D3 tv = o - a;
  const double u = dotd(tv, pv) * inv;
  if (u < 0.0 || u > 1.0) return -1.0;
  const D3 qv{tv.y * e1.z - tv.z * e1.y, tv.z * e1.x - tv.x * e1.z, tv.x * e1.y - tv.y * e1.x};
  const double w = dotd(d, qv) * inv;
  if (w < 0.0 || u + w > 1.0) return -1.0;
  return dotd(e2, qv) * inv;
}

__device__ bool ray_box(D3 o, D3 inv, double lox, double loy, double loz, double hix, double hiy, double hiz,
                        double tmin, double tmax) {
  const double lo[3] = {lox, loy, loz}, hi[3] = {hix, hiy, hiz};
  for (int a = 0; a < 3; ++a) {
    double t0 = (lo[a] - comp(o, a)) * comp(inv, a), t1 = (hi[a] - comp(o, a)) * comp(inv, a);
    if (t0 > t1) {
      const double t = t0;
      t0 = t1;
      t1 = t;
    }
    tmin = fmax(tmin, t0);
    tmax = fmin(tmax, t1);
    if (tmin > tmax) return false;
  }
  return true;
}

// Nearest hit parameter of a ray in [tnear, tfar], or -1.  Bounded stack and
// visit count; overruns set `err`.
__device__ double first_hit(const NodeD *nodes, const TriD *tris, uint32_t max_iter, D3 o, D3 d, double tnear,
                            double tfar, uint32_t &err) {
  const D3 inv{1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
  double best = -1.0, lim = tfar;
  int32_t stack[64];
  int sp = 0;
  stack[sp++] = 0;
  uint32_t iter = 0;
  while (sp > 0) {
    if (++iter > max_iter) {
      err |= TWOS_DEVERR_ITER;
      break;
    }
    const int32_t code = stack[--sp];
    if (code < 0) {
      const uint32_t enc = ~static_cast<uint32_t>(code);
      for (uint32_t i = enc >> 3, e = (enc >> 3) + (enc & 7u); i < e; ++i) {
        const TriD &t = tris[i];
        const D3 a{t.axy.x, t.axy.y, t.azbx.x}, b{t.azbx.y, t.bybz.x, t.bybz.y}, c{t.cxy.x, t.cxy.y, t.czpad.x};
        const double th = ray_triangle(o, d, a, b, c);
        if (th >= tnear && th <= lim) {
          lim = th;
          best = th;
        }
      }
      continue;
    }
    const NodeD &n = nodes[code];
    for (int c = 0; c < 2; ++c) {
      const bool hit = c == 0 ? ray_box(o, inv, n.xlo.x, n.ylo.x, n.zlo.x, n.xhi.x, n.yhi.x, n.zhi.x, tnear, lim)
                              : ray_box(o, inv, n.xlo.y, n.ylo.y, n.zlo.y, n.xhi.y, n.yhi.y, n.zhi.y, tnear, lim);
      if (hit) {
        if (sp >= 64) {
          err |= TWOS_DEVERR_STACK;
          return best;
        }
        stack[sp++] = c == 0 ? n.child.x : n.child.y;
      }
    }
  }
  return best;
}

// EmbreeMesh::inside (wih_twos.cpp:361-394): parity of the hits of a fixed
// oblique ray re-shot from each hit (t + 2e-6), tnear 1e-6, tfar 4, at most
// 128 hits (more is an error).  Counts rays.
__device__ bool inside_parity(const GeoDesc &G, D3 p, uint32_t &rays, uint32_t &err) {
  D3 dir{1.0, 0.3713906763541037, 0.1570796326794897};
  dir = dir * (1.0 / normd(dir));
  D3 origin = p;
  unsigned hits = 0;
  for (; hits < 128; ++hits) {
    ++rays;
    const double t = first_hit(G.nodes_d, G.tris_d, G.max_iter, origin, dir, 1.0e-6, 4.0, err);
    if (t < 0.0) break;
    origin = origin + dir * (t + 2.0e-6);
  }
  if (hits == 128) err |= TWOS_DEVERR_QUERY;
  return hits % 2u == 1u;
}

// FP64 closest-point distance on the FP64 BVH; infinity when no surface
// point lies within sqrt(radius2), which is an error only when `required`.
__device__ double closest_distance_fp64(const GeoDesc &G, double x, double y, double z, double radius2,
                                        bool required, uint2 *stack, int stride, uint32_t &err) {
  double best2 = radius2;
  uint32_t tri = 0;
  const bool found = nearest<double>(G.nodes_d, G.tris_d, G.max_iter, Vec<double>{x, y, z}, best2, tri, stack,
                                     stride, err);
  if (!found) {
    if (required) err |= TWOS_DEVERR_QUERY;
    return CUDART_INF;
  }
  return sqrt(best2);
}

}  // namespace

__global__ void __launch_bounds__(128) diff_classify_kernel(const DiffLaunch D) {
  __shared__ uint2 s_stack[kStack * 128];
  uint2 *stack = s_stack + threadIdx.x;
  const GeoDesc G = *D.geo;
  uint32_t err = 0;
  unsigned long long q = 0, rays_total = 0, falls = 0;
  const double R = D.cavity_radius, ell = D.diff_offset, eps = D.epsilon;
  for (uint64_t wid = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; wid < D.total_walks;
       wid += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const HitRec h = D.hits[wid];
    uint32_t flags = 0;
    D3 start{CUDART_NAN, CUDART_NAN, CUDART_NAN};
    const bool capped = (D.outer_steps[wid] >> 31) != 0;
    if (!capped && h.cavity >= 0 && static_cast<uint32_t>(h.cavity) < D.n_cav) {
      flags |= kDiffCavity;
      const D3 point{h.point[0], h.point[1], h.point[2]}, nrm{h.normal[0], h.normal[1], h.normal[2]};
      const D3 offset = point - nrm * ell;
      const D3 hc{D.cavities[3 * h.cavity], D.cavities[3 * h.cavity + 1], D.cavities[3 * h.cavity + 2]};
      bool near_seam = false, seg_unsafe = false;
      const D3 segment = offset - point;
      const double seg2 = dotd(segment, segment);
      const double tol = 1.0e-10 * fmax(1.0, fabs(R));
      const double coll2 = (R + tol) * (R + tol);
      for (uint32_t i = 0; i < D.n_cav; ++i) {
        if (static_cast<int>(i) == h.cavity) continue;
        const D3 ci{D.cavities[3 * i], D.cavities[3 * i + 1], D.cavities[3 * i + 2]};
        const D3 cd = ci - hc;
        const double cdist = normd(cd);
        if (cdist > tol && cdist < 2.0 * R) {
          // Distance from the hit point to the seam circle of two equal spheres.
          const D3 axis = cd * (1.0 / cdist);
          const D3 seam_center = (hc + ci) * 0.5;
          const double seam_r = sqrt(fmax(0.0, R * R - 0.25 * (cdist * cdist)));
          const D3 rel = point - seam_center;
          const double axial = dotd(rel, axis);
          const D3 radial = rel - axis * axial;
          const double nr = normd(radial) - seam_r;
          const double seam_d = sqrt(axial * axial + nr * nr);
          near_seam = near_seam || seam_d <= ell;
        }
        if (seg2 > 0.0) {
          const double par = fmin(fmax(dotd(ci - point, segment) / seg2, 0.0), 1.0);
          const D3 cl = point + segment * par;
          if (dotd(cl - ci, cl - ci) <= coll2) seg_unsafe = true;
        }
      }
      uint32_t rays = 0;
      bool inside = inside_parity(G, offset, rays, err);
      if (D.enclosure_fallback && !inside && inside_parity(G, hc, rays, err)) {
        ++q;
        const double dc = closest_distance_fp64(G, hc.x, hc.y, hc.z, 16.0, false, stack, 128, err);
        if (dc > R + ell + eps && normd(offset - hc) <= R + ell + eps * 0.5) {
          inside = true;
          ++falls;
        }
      }
      bool ok_dist = false;
      if (inside) {
        ++q;
        double dd = closest_distance_fp64(G, offset.x, offset.y, offset.z, 16.0, true, stack, 128, err);
        for (uint32_t i = 0; i < D.n_cav; ++i) {
          const D3 ci{D.cavities[3 * i], D.cavities[3 * i + 1], D.cavities[3 * i + 2]};
          const double v = normd(offset - ci) - R;
          dd = v < dd ? v : dd;
        }
        ok_dist = dd > eps;
      }
      if (!inside || !ok_dist) seg_unsafe = true;
      rays_total += rays;
      if (near_seam) flags |= kDiffNearSeam;
      if (seg_unsafe) flags |= kDiffSegmentUnsafe;
      if (near_seam || seg_unsafe)
        flags |= kDiffUnsafe;
      else
        start = offset;
    }
    D.flags[wid] = flags;
    D.start[3 * wid] = start.x;
    D.start[3 * wid + 1] = start.y;
    D.start[3 * wid + 2] = start.z;
  }
  if (err) atomicOr(D.error, err);
  atomicAdd(&D.totals[0], q);
  atomicAdd(&D.totals[1], rays_total);
  atomicAdd(&D.totals[2], falls);
}

// One thread per site, walks in order (the reference's accumulation order).
template <typename V>
__global__ void diff_reduce_kernel(const DiffLaunch D) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < D.n_sites; s += gridDim.x * blockDim.x) {
    twos_diff_result *rows = D.out + static_cast<size_t>(D.site_begin + s) * D.n_cav;
    for (uint32_t c = 0; c < D.n_cav; ++c) {
      twos_diff_result &r = rows[c];
      r.dc[0] = r.dc[1] = r.dc[2] = 0.0;
      r.dc_se[0] = r.dc_se[1] = r.dc_se[2] = 0.0;
      r.dR = r.dR_se = 0.0;
    }
    twos_diff_stats st{};
    uint64_t outer_caps = 0, nested_caps = 0;
    const uint64_t base = static_cast<uint64_t>(s) * D.walks;
    for (uint32_t w = 0; w < D.walks; ++w) {
      const uint64_t wid = base + w;
      const uint32_t so = D.outer_steps[wid];
      st.outer_steps += so & 0x7fffffffu;
      if (so >> 31) {
        ++st.limits;
        ++outer_caps;
        continue;
      }
      const HitRec &h = D.hits[wid];
      if (h.cavity < 0 || static_cast<uint32_t>(h.cavity) >= D.n_cav) continue;
      ++st.cavity_terminations;
      const uint32_t fl = D.flags[wid];
      st.near_seam += (fl & kDiffNearSeam) ? 1 : 0;
      st.segment_unsafe += (fl & kDiffSegmentUnsafe) ? 1 : 0;
      if (fl & kDiffUnsafe) {
        ++st.unsafe_offset;
        continue;
      }
      const uint32_t sn = D.nested_steps[wid];
      st.nested_steps += sn & 0x7fffffffu;
      st.limits += sn >> 31;
      nested_caps += sn >> 31;
      const double value = static_cast<double>(static_cast<const V *>(D.nested_u)[wid]);
      // dot(u) = V_n u(x - l n)/l: centre V_n = n . dot(c), radius V_n = -dot(R).
      const double scale = value / D.diff_offset;
      const double sample[4] = {h.normal[0] * scale, h.normal[1] * scale, h.normal[2] * scale, -scale};
      twos_diff_result &r = rows[h.cavity];
      // Running sums in dc (centre) / dR, squares in dc_se / dR_se.
      r.dc[0] = r.dc[0] + sample[0];
      r.dc[1] = r.dc[1] + sample[1];
      r.dc[2] = r.dc[2] + sample[2];
      r.dR += sample[3];
      r.dc_se[0] += sample[0] * sample[0];
      r.dc_se[1] += sample[1] * sample[1];
      r.dc_se[2] += sample[2] * sample[2];
      r.dR_se += sample[3] * sample[3];
    }
    const double n = static_cast<double>(D.walks);
    const double den = n * (n - 1.0);
    for (uint32_t c = 0; c < D.n_cav; ++c) {
      twos_diff_result &r = rows[c];
      for (int k = 0; k < 3; ++k) {
        const double sum = r.dc[k], sq = r.dc_se[k];
        r.dc[k] = sum * (1.0 / n);
        r.dc_se[k] = D.walks > 1 ? sqrt(fmax(0.0, (sq - sum * sum / n) / den)) : 0.0;
      }
      const double sum = r.dR, sq = r.dR_se;
      r.dR = sum / n;
      r.dR_se = D.walks > 1 ? sqrt(fmax(0.0, (sq - sum * sum / n) / den)) : 0.0;
    }
    if (D.stats) D.stats[D.site_begin + s] = st;
    atomicAdd(&D.totals[3], static_cast<unsigned long long>(st.outer_steps));
    atomicAdd(&D.totals[4], static_cast<unsigned long long>(st.nested_steps));
    atomicAdd(&D.totals[5], static_cast<unsigned long long>(st.limits));
    atomicAdd(&D.totals[6], static_cast<unsigned long long>(st.unsafe_offset));
    atomicAdd(&D.totals[7], static_cast<unsigned long long>(st.cavity_terminations));
    atomicAdd(&D.totals[8], static_cast<unsigned long long>(outer_caps));
    atomicAdd(&D.totals[9], static_cast<unsigned long long>(nested_caps));
  }
}

cudaError_t launch_diff_classify(const DiffLaunch &D, cudaStream_t s) {
  if (D.total_walks == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint64_t>((D.total_walks + 127) / 128, 148ull * 16));
  diff_classify_kernel<<<grid, 128, 0, s>>>(D);
  return cudaGetLastError();
}

cudaError_t launch_diff_reduce(int precision, const DiffLaunch &D, cudaStream_t s) {
  if (D.n_sites == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint32_t>((D.n_sites + 127) / 128, 148u * 16));
  if (precision == TWOS_PREC_MIXED)
    diff_reduce_kernel<float><<<grid, 128, 0, s>>>(D);
  else
    diff_reduce_kernel<double><<<grid, 128, 0, s>>>(D);
  return cudaGetLastError();
}

}  // namespace twos

// Certified fresh-sample validation on the device (run_minimum_benefit and
// cert_walk, benchmarks/compiled_bunny/src/minimum_benefit.hpp:13-188).
//
// Every quantity the certificate relies on is a rigorous bound computed the
// way the reference computes it: round to nearest, then step one ulp toward
// the safe side (nextafter), in FP64 without contraction (the library is
// built with -fmad=false).  The mesh distance is the distance to the union
// of the triangles' bounding boxes -- the minimum over triangles of a
// rounded-down box distance, which does not depend on traversal order, so it
// equals the reference's CertDistanceTree value bit for bit.  The FP64 BVH's
// node boxes (padded outward at build) contain those triangle boxes, so
// their rounded-down distances are lower bounds that prune exactly.
//
// One thread per walk; the traversal stack is per thread (64 entries,
// bounded by the BVH depth limit), and every loop is bounded by the
// session's iteration limit or max_steps.
//
// Included at the end of kernels.cu (one translation unit with the random
// stream, direction and closest-point helpers).
#pragma once

namespace twos {

namespace {

__device__ __forceinline__ double cv_dn(double x) { return nextafter(x, -CUDART_INF); }
__device__ __forceinline__ double cv_up(double x) { return nextafter(x, CUDART_INF); }
__device__ __forceinline__ double cv_pdn(double x) { return fmax(0.0, cv_dn(x)); }

__device__ __forceinline__ double cv_box_lower(double lx, double ly, double lz, double hx, double hy, double hz,
                                               double x, double y, double z) {
  const double lo[3] = {lx, ly, lz}, hi[3] = {hx, hy, hz}, p[3] = {x, y, z};
  double sum = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double g = fmax(fmax(0.0, cv_dn(lo[a] - p[a])), cv_dn(p[a] - hi[a]));
    sum = cv_pdn(sum + cv_pdn(g * g));
  }
  return cv_pdn(sqrt(sum));
}

// point_distance_bound: rounded up (upper) or down.
__device__ __forceinline__ double cv_point_distance(const double *a, const double *b, bool upper) {
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double d = fabs(a[k] - b[k]);
    d = upper ? cv_up(d) : cv_pdn(d);
    const double q = upper ? cv_up(d * d) : cv_pdn(d * d);
    sum = upper ? cv_up(sum + q) : cv_pdn(sum + q);
  }
  return upper ? cv_up(sqrt(sum)) : cv_pdn(sqrt(sum));
}

// Minimum over triangles of the rounded-down distance to the triangle's box.
__device__ double cv_mesh_distance(const GeoDesc &G, const double *p, uint32_t &err) {
  double best = CUDART_INF;
  int32_t stack[64];
  int sp = 0;
  stack[sp++] = 0;
  uint32_t iter = 0;
  while (sp > 0) {
    if (++iter > G.max_iter) {
      err |= TWOS_DEVERR_ITER;
      return 0.0;  // fail closed: a zero distance ends the walk
    }
    const int32_t code = stack[--sp];
    if (code < 0) {
      const uint32_t enc = ~static_cast<uint32_t>(code);
      for (uint32_t i = enc >> 3, e = (enc >> 3) + (enc & 7u); i < e; ++i) {
        Vec<double> a, b, c;
        load_tri(G.tris_d, i, a, b, c);
        const double v = cv_box_lower(fmin(fmin(a.x, b.x), c.x), fmin(fmin(a.y, b.y), c.y), fmin(fmin(a.z, b.z), c.z),
                                      fmax(fmax(a.x, b.x), c.x), fmax(fmax(a.y, b.y), c.y), fmax(fmax(a.z, b.z), c.z),
                                      p[0], p[1], p[2]);
        best = fmin(best, v);
      }
      continue;
    }
    const NodeD &n = G.nodes_d[code];
    const double2 xl = __ldg(&n.xlo), xh = __ldg(&n.xhi), yl = __ldg(&n.ylo), yh = __ldg(&n.yhi);
    const double2 zl = __ldg(&n.zlo), zh = __ldg(&n.zhi);
    const int4 ch = __ldg(&n.child);
    const double dl = cv_box_lower(xl.x, yl.x, zl.x, xh.x, yh.x, zh.x, p[0], p[1], p[2]);
    const double dr = cv_box_lower(xl.y, yl.y, zl.y, xh.y, yh.y, zh.y, p[0], p[1], p[2]);
    // Nearer child on top of the stack; a child whose bound is >= best
    // cannot hold a smaller triangle bound.
    const bool left_first = dl < dr;
    const double d_far = left_first ? dr : dl, d_near = left_first ? dl : dr;
    const int32_t c_far = left_first ? ch.y : ch.x, c_near = left_first ? ch.x : ch.y;
    if (d_far < best) {
      if (sp >= 64) {
        err |= TWOS_DEVERR_STACK;
        return 0.0;
      }
      stack[sp++] = c_far;
    }
    if (d_near < best) {
      if (sp >= 64) {
        err |= TWOS_DEVERR_STACK;
        return 0.0;
      }
      stack[sp++] = c_near;
    }
  }
  return best;
}

__device__ double cv_domain_distance(const ValidateLaunch &V, const GeoDesc &G, const double *p, uint32_t &err) {
  double d = cv_mesh_distance(G, p, err);
  for (uint32_t i = 0; i < V.n_cav; ++i) d = fmin(d, cv_dn(cv_point_distance(p, V.cavities + 3 * i, false) - V.cavity_radius));
  return fmax(0.0, d);
}

// (1 - t/1024)^1024 <= exp(-t), every step rounded down.
__device__ double cv_exp_lower(double t_upper) {
  double a = fmax(0.0, cv_dn(1.0 - cv_up(t_upper / 1024.0)));
  for (int i = 0; i < 10; ++i) a = cv_pdn(a * a);
  return a;
}

// Rounded-down source: a leading constant, then linear and Gaussian terms
// in order (cert_source_lower's affine and housing sequences).
__device__ double cv_source_lower(const ValidateLaunch &V, const double *p) {
  uint32_t i = 0;
  double value = 0.0;
  if (V.n_terms > 0 && V.terms[0].kind == TWOS_TERM_CONST) value = V.terms[i++].amp;
  for (; i < V.n_terms; ++i) {
    const TermDev &t = V.terms[i];
    if (t.kind == TWOS_TERM_LINEAR) {
      value = cv_dn(value + cv_dn(t.amp * cv_dn(p[t.axis] + t.offset)));
    } else if (t.kind == TWOS_TERM_GAUSS) {
      double exponent = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double q = cv_up(cv_up(fabs(p[a] - t.c[a])) / t.w[a]);
        exponent = cv_up(exponent + cv_up(q * q));
      }
      value = cv_dn(value + cv_pdn(t.amp * cv_exp_lower(exponent)));
    } else if (t.kind == TWOS_TERM_CONST) {
      value = cv_dn(value + t.amp);
    }
  }
  return fmax(0.0, value);
}

}  // namespace

__global__ void __launch_bounds__(128) validate_kernel(const ValidateLaunch V) {
  const GeoDesc G = *V.geo;
  uint32_t err = 0;
  unsigned long long failures = 0, total_steps = 0;
  const uint64_t total = static_cast<uint64_t>(V.n_sites) * V.walks;
  for (uint64_t wid = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; wid < total;
       wid += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t site = static_cast<uint32_t>(wid / V.walks);
    const uint32_t walk = static_cast<uint32_t>(wid - static_cast<uint64_t>(site) * V.walks);
    double pt[3] = {V.sites[3ull * site], V.sites[3ull * site + 1], V.sites[3ull * site + 2]};
    twos_cert_sample out{};
    out.contained = 1;
    bool done = false;
    for (int k = 0; k < V.max_steps && !done; ++k) {
      const double d = cv_domain_distance(V, G, pt, err);
      if (d <= V.epsilon) {
        done = true;
        break;
      }
      const double s = fmin(V.radius_cap, cv_pdn(0.95 * d));
      const uint32_t ctr3 = V.repeat << 3;
      const Philox4 q0 = philox(V.k0, V.k1, static_cast<uint32_t>(k), walk, V.site_offset + site, ctr3 | 0u);
      double y[3] = {pt[0], pt[1], pt[2]};
      if (V.green) {
        const Philox4 q1 = philox(V.k0, V.k1, static_cast<uint32_t>(k), walk, V.site_offset + site, ctr3 | 1u);
        const Philox4 q2 = philox(V.k0, V.k1, static_cast<uint32_t>(k), walk, V.site_offset + site, ctr3 | 2u);
        const Philox4 q3 = philox(V.k0, V.k1, static_cast<uint32_t>(k), walk, V.site_offset + site, ctr3 | 3u);
        const double beta = median3(uniform<double>(q2.x, q2.y), uniform<double>(q2.z, q2.w),
                                    uniform<double>(q3.x, q3.y));
        const Vec<double> g = direction<double>(uniform<double>(q1.x, q1.y), uniform<double>(q1.z, q1.w));
        const double sc = s * beta;
        y[0] = pt[0] + g.x * sc;
        y[1] = pt[1] + g.y * sc;
        y[2] = pt[2] + g.z * sc;
      }
      const Vec<double> dir = direction<double>(uniform<double>(q0.x, q0.y), uniform<double>(q0.z, q0.w));
      const double next[3] = {pt[0] + dir.x * s, pt[1] + dir.y * s, pt[2] + dir.z * s};
      if (!(cv_point_distance(pt, next, true) < d) || !(cv_point_distance(pt, y, true) < d)) {
        out.contained = 0;  // fail closed: this record must not be used
        ++failures;
        done = true;
        break;
      }
      const double weight = cv_pdn(cv_pdn(s * s) / 6.0);
      const double increment = cv_pdn(weight * cv_source_lower(V, y));
      out.value = cv_pdn(out.value + increment);
      ++out.steps;
      if (out.value >= V.value_cap) {
        out.value = V.value_cap;
        out.clipped = 1;
        done = true;
        break;
      }
      pt[0] = next[0];
      pt[1] = next[1];
      pt[2] = next[2];
    }
    if (!done) out.capped = 1;
    total_steps += out.steps;
    V.samples[wid] = out;
  }
  // Per-site clearances (certified and exact FP64) at the start points.
  for (uint32_t site = blockIdx.x * blockDim.x + threadIdx.x; site < V.n_sites; site += gridDim.x * blockDim.x) {
    const double *p = V.sites + 3ull * site;
    V.clearance[site] = cv_domain_distance(V, G, p, err);
  }
  if (err) atomicOr(V.error, err);
  if (failures) atomicAdd(&V.totals[0], failures);
  if (total_steps) atomicAdd(&V.totals[1], total_steps);
}

__global__ void __launch_bounds__(kWosBlock) validate_center_kernel(const ValidateLaunch V) {
  __shared__ uint2 s_stack[kStack * kWosBlock];
  const GeoDesc G = *V.geo;
  uint32_t err = 0;
  for (uint32_t site = blockIdx.x * blockDim.x + threadIdx.x; site < V.n_sites; site += gridDim.x * blockDim.x) {
    const double *p = V.sites + 3ull * site;
    double best2 = CUDART_INF;
    uint32_t tri = 0;
    double d = CUDART_INF;
    if (nearest<double>(G.nodes_d, G.tris_d, G.max_iter, Vec<double>{p[0], p[1], p[2]}, best2, tri,
                        s_stack + threadIdx.x, kWosBlock, err))
      d = sqrt(best2);
    for (uint32_t i = 0; i < V.n_cav; ++i) {
      const double dx = p[0] - V.cavities[3 * i], dy = p[1] - V.cavities[3 * i + 1], dz = p[2] - V.cavities[3 * i + 2];
      d = fmin(d, sqrt(dx * dx + dy * dy + dz * dz) - V.cavity_radius);
    }
    V.center_distance[site] = d;
  }
  if (err) atomicOr(V.error, err);
}

cudaError_t launch_validate(const ValidateLaunch &V, cudaStream_t s) {
  const uint64_t total = static_cast<uint64_t>(V.n_sites) * V.walks;
  if (total == 0) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint64_t>((total + 127) / 128, 148ull * 16));
  validate_kernel<<<grid, 128, 0, s>>>(V);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int grid_c = static_cast<int>(std::min<uint32_t>((V.n_sites + kWosBlock - 1) / kWosBlock, 148u * 4));
  validate_center_kernel<<<grid_c, kWosBlock, 0, s>>>(V);
  return cudaGetLastError();
}

}  // namespace twos

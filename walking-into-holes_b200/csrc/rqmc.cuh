// Array-RQMC and matched Monte Carlo walks (twos_rqmc): the 3D counterpart
// of the reference's sampling study (benchmarks/critical_baselines/
// sampling.py:49-88: Ho and Owen's Array-RQMC, shifted Korobov lattice,
// Hilbert ordering, converged paths last).
//
// One block per (site, batch), one thread per walk; all walks of the block
// take their steps together.  At each step a thread answers its walk's
// closest-point query (nearest<T>, stack in local memory); walks within
// epsilon stop and add the boundary data at their exit point; then, in
// ARRAY mode, the block sorts (Hilbert key, thread) pairs with a bitonic
// network in shared memory and the walk of rank i takes the Korobov lattice
// point (i/n, a i/n, a^2 i/n) mod 1 -- the first coordinate is consumed by
// the ordering, the other two, shifted by one random (U1, U2) per (site,
// batch, step), give the direction as in the walk kernel; in MC mode every
// walk draws its own uniforms.  NEIGHBOUR mode runs the MC walks with the
// per-walk record on (first step point, payoffs, first radius) and then
// rqmc_reuse_kernel pools the neighbours' walks into each site's batch mean.
// SOBOL mode gives walk i point i of a scrambled Sobol' sequence, two
// coordinates per step (the reference's Sobol-over-steps method).
//
// Included at the end of kernels.cu.
#pragma once

namespace twos {

namespace {

// Hilbert index of a point of the 1024^3 grid: Skilling's transpose method
// ("Programming the Hilbert curve", AIP Conf. Proc. 707, 2004): undo the
// excess work of the reflected Gray code per bit plane, Gray-encode, then
// interleave the transposed bits (axis 0 most significant).
__host__ __device__ inline uint32_t hilbert3(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t X[3] = {x, y, z};
  constexpr int kBits = 10;
  for (uint32_t Q = 1u << (kBits - 1); Q > 1u; Q >>= 1) {
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
  for (uint32_t Q = 1u << (kBits - 1); Q > 1u; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1u;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  uint32_t h = 0;
  for (int bit = kBits - 1; bit >= 0; --bit)
    for (int i = 0; i < 3; ++i) h = (h << 1) | ((X[i] >> bit) & 1u);
  return h;
}

template <typename T> __device__ __forceinline__ TermT<T> to_termT(const TermDev &d) {
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
  return t;
}

}  // namespace

template <typename T> __global__ void __launch_bounds__(1024) rqmc_kernel(const RqmcLaunch R) {
  extern __shared__ unsigned long long s_keys[];  // [walks] (key << 32 | thread), then ranks
  uint32_t *s_rank = reinterpret_cast<uint32_t *>(s_keys + R.walks);
  __shared__ TermT<T> s_terms[3 * TWOS_MAX_TERMS];
  __shared__ double s_red[32][2];
  // SOBOL: one step's scrambling (lower-triangular matrix rows and digital
  // shift per coordinate) and scrambled direction numbers.
  __shared__ uint32_t s_lms[2][32], s_shift[2], s_dir[2][kSobolBits];
  const uint32_t n_terms = R.n_src + R.n_ub + R.n_pb;
  for (uint32_t i = threadIdx.x; i < n_terms; i += blockDim.x) s_terms[i] = to_termT<T>(R.terms[i]);
  __syncthreads();
  const uint32_t site = blockIdx.x % R.n_sites, batch = blockIdx.x / R.n_sites;
  const uint32_t tid = threadIdx.x, n = R.walks;
  const GeoDesc G = *R.geo;
  Vec<T> pos = to_frame<T>(R.sites + 3ull * site, G);
  bool active = true, cap = false;
  uint32_t steps = 0, err = 0;
  double vu = 0.0, vp = 0.0;
  uint2 lstack[kStack];
  const uint32_t ctr3 = (batch << 16) | (R.repeat << 3);
  for (int k = 0; k < R.max_steps; ++k) {
    T r = T(0);
    if (active) {
      T best2 = static_cast<T>(CUDART_INF);
      uint32_t tri = 0;
      if (!nearest<T>(geo_nodes<T>(G), geo_tris<T>(G), G.max_iter, pos, best2, tri, lstack, 1, err)) {
        err |= TWOS_DEVERR_QUERY;
        active = false;
      } else {
        const T d = sqrt(best2);
        r = sizeof(T) == 4 ? d - static_cast<T>(G.delta) : d;
        if (!(r > static_cast<T>(R.epsilon))) {
          Vec<T> a, b, c;
          load_tri(geo_tris<T>(G), tri, a, b, c);
          const Vec<T> q = tri_closest(pos, a, b, c);
          if (R.n_ub) vu += static_cast<double>(source_value(s_terms, R.n_src, R.n_ub, q));
          if (R.n_pb) vp += static_cast<double>(source_value(s_terms, R.n_src + R.n_ub, R.n_pb, q));
          active = false;
        }
      }
    }
    if (!__syncthreads_or(active)) break;
    T u1, u2;
    if (R.method == TWOS_RQMC_ARRAY) {
      uint32_t key = 0xffffffffu;
      if (active) {
        uint32_t qc[3];
        const T pc[3] = {pos.x, pos.y, pos.z};
        for (int a = 0; a < 3; ++a) {
          const double f = (static_cast<double>(pc[a]) - R.lo[a]) * R.inv_extent[a] * 1024.0;
          qc[a] = static_cast<uint32_t>(fmin(fmax(f, 0.0), 1023.0));
        }
        key = hilbert3(qc[0], qc[1], qc[2]);
      }
      s_keys[tid] = (static_cast<unsigned long long>(key) << 32) | tid;
      __syncthreads();
      for (uint32_t kk = 2; kk <= n; kk <<= 1) {
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
          const uint32_t ixj = tid ^ j;
          if (ixj > tid) {
            const unsigned long long a = s_keys[tid], b = s_keys[ixj];
            const bool ascending = (tid & kk) == 0;
            if ((a > b) == ascending) {
              s_keys[tid] = b;
              s_keys[ixj] = a;
            }
          }
          __syncthreads();
        }
      }
      s_rank[static_cast<uint32_t>(s_keys[tid] & 0xffffffffu)] = tid;
      __syncthreads();
      const uint32_t rank = s_rank[tid];
      const Philox4 sh = philox(R.k0, R.k1, static_cast<uint32_t>(k), 0xffffffffu, site, ctr3 | 6u);
      const double U1 = uniform<double>(sh.x, sh.y), U2 = uniform<double>(sh.z, sh.w);
      // Korobov point (i/n, a i/n, a^2 i/n) mod 1: its first coordinate is
      // the sorted rank itself; the other two drive the step.
      double a1 = static_cast<double>((static_cast<uint64_t>(R.generator) * rank) % n) / n + U1;
      double a2 = static_cast<double>((static_cast<uint64_t>(R.generator2) * rank) % n) / n + U2;
      a1 -= floor(a1);
      a2 -= floor(a2);
      u1 = static_cast<T>(a1);
      u2 = static_cast<T>(a2);
    } else if (R.method == TWOS_RQMC_SOBOL && static_cast<uint32_t>(k) < kSobolSteps) {
      // Sobol-over-steps (sampling.py:49-60 in 3D): walk i holds point i of
      // a Sobol' sequence scrambled once per (site, batch) -- a random
      // lower-triangular matrix with unit diagonal applied to the digits
      // (LMS) and a digital shift, per coordinate -- and step k takes its
      // coordinates 2k and 2k + 1.  Words 0..63 are matrix rows, 64..65 the
      // shifts; all are keyed by (step, word, site, batch).
      for (uint32_t w = tid; w < 66u; w += n) {
        const uint32_t word = philox(R.k0, R.k1, static_cast<uint32_t>(k), w, site, ctr3 | 5u).x;
        if (w < 64u) {
          const uint32_t row = w & 31u;
          s_lms[w >> 5][row] = (word & (~0u << (31u - row))) | (1u << (31u - row));
        } else {
          s_shift[w - 64u] = word;
        }
      }
      __syncthreads();
      if (tid < 2u * R.sobol_bits) {
        const uint32_t c = tid / R.sobol_bits, b = tid % R.sobol_bits;
        const uint32_t v = R.sobol_v[(2u * static_cast<uint32_t>(k) + c) * kSobolBits + b];
        uint32_t out = 0;
        for (uint32_t row = 0; row < 32u; ++row) out |= (__popc(s_lms[c][row] & v) & 1u) << (31u - row);
        s_dir[c][b] = out;
      }
      __syncthreads();
      uint32_t x1 = s_shift[0], x2 = s_shift[1];
      for (uint32_t b = 0; b < R.sobol_bits; ++b)
        if ((tid >> b) & 1u) {
          x1 ^= s_dir[0][b];
          x2 ^= s_dir[1][b];
        }
      // Cell midpoints: exact in double, never 0 or 1.
      u1 = static_cast<T>((static_cast<double>(x1) + 0.5) * 0x1p-32);
      u2 = static_cast<T>((static_cast<double>(x2) + 0.5) * 0x1p-32);
      // (The barrier at the end of the step orders these reads before the
      // next step's writes.)
    } else {
      const Philox4 q = philox(R.k0, R.k1, static_cast<uint32_t>(k), tid, site, ctr3);
      u1 = uniform<T>(q.x, q.y);
      u2 = uniform<T>(q.z, q.w);
    }
    if (active) {
      if (R.n_src) vu += static_cast<double>(r * r / T(6) * source_value(s_terms, 0, R.n_src, pos));
      const Vec<T> dir = direction<T>(u1, u2);
      pos = add_scaled(pos, dir, r);
      if (k == 0 && R.walk_first) {
        const size_t w = (static_cast<size_t>(batch) * R.n_sites + site) * n + tid;
        const bool f32 = sizeof(T) == 4;
        R.walk_first[3 * w] = static_cast<double>(pos.x) + (f32 ? G.center[0] : 0.0);
        R.walk_first[3 * w + 1] = static_cast<double>(pos.y) + (f32 ? G.center[1] : 0.0);
        R.walk_first[3 * w + 2] = static_cast<double>(pos.z) + (f32 ? G.center[2] : 0.0);
        if (tid == 0 && batch == 0 && R.site_radius) R.site_radius[site] = static_cast<double>(r);
      }
      ++steps;
      if (static_cast<int>(steps) >= R.max_steps) {
        cap = true;
        active = false;
      }
    }
    __syncthreads();
  }
  if (R.walk_u) {
    const size_t w = (static_cast<size_t>(batch) * R.n_sites + site) * n + tid;
    R.walk_u[w] = vu;
    R.walk_p[w] = vp;
  }
  // Block sums in a fixed order: warp xor trees, then warp 0 over the warps.
  double su = warp_sum(vu), sp = warp_sum(vp);
  const uint32_t warp = tid >> 5, lane = tid & 31u;
  if (lane == 0) {
    s_red[warp][0] = su;
    s_red[warp][1] = sp;
  }
  __syncthreads();
  if (tid == 0) {
    double tu = 0.0, tp = 0.0;
    for (uint32_t w = 0; w < (n + 31) / 32; ++w) {
      tu += s_red[w][0];
      tp += s_red[w][1];
    }
    R.batch_u[static_cast<size_t>(batch) * R.n_sites + site] = tu / n;
    R.batch_p[static_cast<size_t>(batch) * R.n_sites + site] = tp / n;
  }
  const unsigned long long st = warp_sum_u64(steps), cp = warp_sum_u64(cap ? 1ull : 0ull);
  if (lane == 0) {
    if (st) atomicAdd(&R.totals[0], st);
    if (cp) atomicAdd(&R.totals[1], cp);
  }
  if (err) atomicOr(R.error, err);
}

// Neighbour reuse (reused_means, sampling.py:76-88, in 3D): block (site x,
// batch b) pools the walks of batch b started at every site y whose first
// ball B(y, r_y) holds x, a = |x - y| / r_y < 1 - 1e-12.  A walk whose first
// step landed at z carries the Poisson kernel ratio of the ball,
// P(x, z) / P(y, z) = r_y (r_y^2 - |x - y|^2) / |x - z|^3, and site y the
// weight (1 - a)^4 / (1 + a)^2 -- the inverse square of that ratio's bound
// (1 + a) / (1 - a)^2, as the reference's 2D weight (1 - a)^4 / (1 - a^2)^2
// is for the 2D ratio's bound (1 + a) / (1 - a).  The batch mean of x becomes
// sum_y w_y mean_j(K_yj v_yj) / sum_y w_y; a site with no such y (its walks
// stopped at once, r = 0) keeps its plain mean.  Each thread sums its walks
// over all y in a fixed order, then the block sums in a fixed order.
__global__ void __launch_bounds__(256) rqmc_reuse_kernel(const RqmcLaunch R) {
  __shared__ double s_red[8][2];
  const uint32_t x = blockIdx.x % R.n_sites, b = blockIdx.x / R.n_sites;
  const uint32_t tid = threadIdx.x, n = R.walks;
  const double x0 = R.sites[3ull * x], x1 = R.sites[3ull * x + 1], x2 = R.sites[3ull * x + 2];
  double au = 0.0, ap = 0.0, wsum = 0.0;
  for (uint32_t y = 0; y < R.n_sites; ++y) {
    const double ry = R.site_radius[y];
    const double e0 = x0 - R.sites[3ull * y], e1 = x1 - R.sites[3ull * y + 1], e2 = x2 - R.sites[3ull * y + 2];
    const double rho2 = e0 * e0 + e1 * e1 + e2 * e2;
    const double a = sqrt(rho2) / ry;
    if (!(a < 1.0 - 1e-12)) continue;
    const double w = (1.0 - a) * (1.0 - a) * (1.0 - a) * (1.0 - a) / ((1.0 + a) * (1.0 + a));
    wsum += w;
    const double c = w * ry * (ry * ry - rho2) / n;
    const size_t base = (static_cast<size_t>(b) * R.n_sites + y) * n;
    for (uint32_t j = tid; j < n; j += blockDim.x) {
      const double *z = R.walk_first + 3 * (base + j);
      const double d0 = x0 - z[0], d1 = x1 - z[1], d2 = x2 - z[2];
      const double dist2 = d0 * d0 + d1 * d1 + d2 * d2;
      const double K = c / (dist2 * sqrt(dist2));
      au += K * R.walk_u[base + j];
      ap += K * R.walk_p[base + j];
    }
  }
  double su = warp_sum(au), sp = warp_sum(ap);
  const uint32_t warp = tid >> 5, lane = tid & 31u;
  if (lane == 0) {
    s_red[warp][0] = su;
    s_red[warp][1] = sp;
  }
  __syncthreads();
  if (tid == 0 && wsum > 0.0) {
    double tu = 0.0, tp = 0.0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
      tu += s_red[w][0];
      tp += s_red[w][1];
    }
    R.batch_u[static_cast<size_t>(b) * R.n_sites + x] = tu / wsum;
    R.batch_p[static_cast<size_t>(b) * R.n_sites + x] = tp / wsum;
  }
}

cudaError_t launch_rqmc(int precision, const RqmcLaunch &R, cudaStream_t s) {
  const uint64_t blocks = static_cast<uint64_t>(R.n_sites) * R.batches;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffull || R.walks < 32 || R.walks > 1024 || (R.walks & (R.walks - 1)))
    return cudaErrorInvalidValue;
  if ((R.walk_u == nullptr) != (R.walk_p == nullptr)) return cudaErrorInvalidValue;
  if (R.method == TWOS_RQMC_SOBOL && (!R.sobol_v || (1u << R.sobol_bits) != R.walks || R.sobol_bits > kSobolBits))
    return cudaErrorInvalidValue;
  const size_t dyn = R.walks * (sizeof(unsigned long long) + sizeof(uint32_t));
  if (precision == TWOS_PREC_MIXED)
    rqmc_kernel<float><<<static_cast<unsigned>(blocks), R.walks, dyn, s>>>(R);
  else
    rqmc_kernel<double><<<static_cast<unsigned>(blocks), R.walks, dyn, s>>>(R);
  return cudaGetLastError();
}

cudaError_t launch_rqmc_reuse(const RqmcLaunch &R, cudaStream_t s) {
  const uint64_t blocks = static_cast<uint64_t>(R.n_sites) * R.batches;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffull || !R.walk_first || !R.walk_u || !R.walk_p || !R.site_radius)
    return cudaErrorInvalidValue;
  rqmc_reuse_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(R);
  return cudaGetLastError();
}

}  // namespace twos

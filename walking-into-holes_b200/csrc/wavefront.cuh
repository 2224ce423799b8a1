// Wavefront form of the mixed-precision walk (FP32 compliance, paired and
// hot modes with the centre-point source): the same walks as wos_kernel --
// same counter stream, distance grid, warm start and entry nodes, so the
// same per-walk samples -- reorganised so that each kernel runs one kind of
// work over many walks at once, instead of one warp interleaving walk steps,
// grid steps and traversal units of different walks (a per-lane state
// machine whose warps issue at about a quarter of their width).
//
// The walks in flight live in slot arrays in device memory.  Each iteration:
//   wf_step_kernel  -- one thread per slot: the walk's step with the radius
//                      found last iteration (termination, source term, move),
//                      the grid bound at the new point (a grid step needs no
//                      query), else the query's initial bound and start node
//                      and a place in the query list; a slot whose walk ended
//                      takes the next walk of the work queue (its first radius
//                      comes from the per-site pre-pass);
//   wf_query_kernel -- persistent over the query list: each lane runs one
//                      closest-point traversal after another (shared-memory
//                      stack), `units` traversal units per loop iteration.
// Every live slot steps once per iteration, so a walk of k steps spends k
// iterations in flight.  The host keeps launching iterations, a chunk at a
// time, until a chunk ends with no live slot (the queue is then empty).
//
// Included at the end of kernels.cu.
#pragma once

namespace twos {

constexpr uint32_t kWfLive = 1u, kWfFound = 2u, kWfTriOk = 4u;  // slot flags (meta.w low byte; job << 8)
constexpr int kWfStepBlock = 256, kWfQueryBlock = 128;

template <int MODE>
__global__ void __launch_bounds__(kWfStepBlock) wf_step_kernel(const WosLaunch L, const WfSlots S) {
  constexpr bool PAIRED = MODE == TWOS_MODE_PAIRED;
  extern __shared__ __align__(16) unsigned char s_dyn[];
  TermT<float> *s_terms = reinterpret_cast<TermT<float> *>(s_dyn);
  for (uint32_t i = threadIdx.x; i < L.n_terms; i += blockDim.x) {
    const TermDev &d = L.terms[i];
    TermT<float> t;
    t.kind = d.kind;
    t.axis = d.axis;
    t.amp = static_cast<float>(d.amp);
    t.offset = static_cast<float>(d.offset);
    t.div = static_cast<float>(d.div);
    for (int k = 0; k < 3; ++k) {
      t.c[k] = static_cast<float>(d.c[k]);
      t.w[k] = static_cast<float>(d.w[k]);
    }
    s_terms[i] = t;
  }
  __syncthreads();

  const unsigned full = 0xffffffffu;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t slot = blockIdx.x * kWfStepBlock + threadIdx.x;
  const bool mine = slot < S.slots;
  uint32_t err = 0, c_grid = 0, c_tris = 0;
  uint4 M = mine ? S.meta[slot] : make_uint4(0u, 0u, 0u, 0u);
  bool live = (M.w & kWfLive) != 0u;
  bool queued = false;
  int node = 0;
  Vec<float> pos{0.f, 0.f, 0.f};
  float best2 = 0.f, u = 0.f, pv = 0.f;
  uint32_t wid = M.x, steps = M.y, best_tri = M.z, job = M.w >> 8;
  bool found = (M.w & kWfFound) != 0u, tri_ok = (M.w & kWfTriOk) != 0u;

  if (live) {
    const float4 P = S.pos[slot];
    const float2 V = S.val[slot];
    pos = {P.x, P.y, P.z};
    best2 = P.w;
    u = V.x;
    pv = V.y;
    const JobDesc &J = L.jobs[job];
    const GeoDesc &G = L.geos[J.geo];
    const uint64_t local = static_cast<uint64_t>(wid) - J.walk_begin;
    const uint32_t site = static_cast<uint32_t>(local / J.walks);
    const uint32_t walk = static_cast<uint32_t>(local - static_cast<uint64_t>(site) * J.walks);
    // The step (wos_kernel's step block for the centre-point source).
    float d = sqrtf(best2);
    if (!found) {
      err |= TWOS_DEVERR_QUERY;
      d = 0.f;
    }
    const float R = static_cast<float>(J.cavity_radius);
    for (uint32_t c = 0; c < J.n_cav; ++c) {
      const Vec<float> cc = to_frame<float>(L.cavities + 3ull * (J.cav_begin + c), G);
      const Vec<float> dv = sub(pos, cc);
      const float dc = sqrtf(dot3(dv, dv)) - R;
      d = dc < d ? dc : d;
    }
    const float r = d - static_cast<float>(G.delta);
    const float eps = static_cast<float>(J.epsilon);
    bool done = !(r > eps), cap = false;
    if (!done) {
      const uint32_t ctr3 = J.repeat << 3;
      const Philox4 q0 = philox(J.k0, J.k1, steps, walk, J.site_offset + site, ctr3);
      const float w = r * r / 6.f;
      u = u + w * source_value(s_terms, J.src_begin, J.n_src, pos);
      if (PAIRED) pv = pv + w * source_value(s_terms, J.adj_begin, J.n_adj, pos);
      const Vec<float> dir = direction<float>(uniform<float>(q0.x, q0.y), uniform<float>(q0.z, q0.w));
      pos = add_scaled(pos, dir, r);
      ++steps;
      if (static_cast<int>(steps) >= J.max_steps) {
        done = true;
        cap = true;
      }
    }
    if (done) {
      static_cast<float *>(L.u_out)[wid] = u;
      if (PAIRED) static_cast<float *>(L.p_out)[wid] = pv;
      L.steps_out[wid] = steps | (cap ? 0x80000000u : 0u);
      live = false;
    } else {
      // The next radius: a grid step, or the query's initial bound and start.
      best2 = static_cast<float>(J.query_radius2);
      found = false;
      float bound, upper = CUDART_INF_F;
      int entry_node = -1;
      const bool in_grid = (L.grid_tau > 0.f || L.entry) && G.grid && grid_bounds(G, pos, bound, upper, entry_node);
      if (in_grid && L.grid_tau > 0.f && bound >= L.grid_tau * G.grid_h && bound > 2.f * (eps + G.delta) &&
          bound * bound < best2) {
        best2 = bound * bound;
        found = true;
        ++c_grid;
      } else {
        if (!(in_grid && L.entry)) entry_node = -1;
        if (L.warm && tri_ok) {
          Vec<float> ta, tb, tc;
          load_tri(G.tris_f, best_tri, ta, tb, tc);
          ++c_tris;
          const float w2 = tri_dist2(pos, ta, tb, tc);
          if (w2 < best2) {
            best2 = w2;
            found = true;
          }
        }
        if (entry_node >= 0) {
          const float ubs = upper + 6.f * G.delta;
          if (fminf(sqrtf(best2), ubs) < G.entry_radius) {
            node = entry_node;
            if (ubs * ubs < best2) best2 = ubs * ubs;
          }
        }
        queued = true;
      }
    }
  }

  // A slot without a walk takes the next one from the work queue.
  const bool want = mine && !live;
  const unsigned need = __ballot_sync(full, want);
  if (need != 0u) {
    unsigned long long base = L.total_walks;
    const int leader = __ffs(need) - 1;
    if (static_cast<int>(lane) == leader && *reinterpret_cast<volatile unsigned long long *>(L.counter) < L.total_walks)
      base = atomicAdd(L.counter, static_cast<unsigned long long>(__popc(need)));
    base = __shfl_sync(full, base, leader);
    const uint64_t id = base + __popc(need & ((1u << lane) - 1u));
    if (want && id < L.total_walks) {
      job = find_job(L.jobs, L.n_jobs, id);
      const JobDesc &J = L.jobs[job];
      const GeoDesc &G = L.geos[J.geo];
      const uint64_t local = id - J.walk_begin;
      const uint32_t site = static_cast<uint32_t>(local / J.walks);
      wid = static_cast<uint32_t>(id);
      pos = to_frame<float>(L.sites + 3ull * (J.site_begin + site), G);
      bool skip = false;
      if (J.flags & kJobSkipCavitySites) {
        const float R = static_cast<float>(J.cavity_radius);
        for (uint32_t c = 0; c < J.n_cav; ++c) {
          const Vec<float> cc = to_frame<float>(L.cavities + 3ull * (J.cav_begin + c), G);
          const Vec<float> dv = sub(pos, cc);
          if (sqrtf(dot3(dv, dv)) <= R) skip = true;
        }
      }
      if (skip) {
        static_cast<float *>(L.u_out)[wid] = 0.f;
        if (PAIRED) static_cast<float *>(L.p_out)[wid] = 0.f;
        L.steps_out[wid] = 0u;
      } else {
        live = true;
        u = pv = 0.f;
        steps = 0;
        tri_ok = false;
        best_tri = 0;
        if (L.site_best2) {
          // First radius from the per-site pre-pass.
          best2 = static_cast<const float *>(L.site_best2)[J.site_rank + site];
          found = best2 >= 0.f;
        } else {
          best2 = static_cast<float>(J.query_radius2);
          found = false;
          node = 0;
          queued = true;
        }
      }
    }
  }

  if (mine && (live || (M.w & kWfLive))) {
    S.pos[slot] = make_float4(pos.x, pos.y, pos.z, best2);
    S.val[slot] = make_float2(u, pv);
    S.meta[slot] = make_uint4(wid, steps, best_tri,
                              (live ? kWfLive : 0u) | (found ? kWfFound : 0u) | (tri_ok ? kWfTriOk : 0u) | (job << 8));
    if (queued) S.node[slot] = node;
  }
  // Queue the slots whose next radius needs a query; count the live ones.
  const unsigned qv = __ballot_sync(full, queued);
  if (qv != 0u) {
    uint32_t qbase = 0;
    const int leader = __ffs(qv) - 1;
    if (static_cast<int>(lane) == leader) qbase = atomicAdd(&S.counts[0], static_cast<uint32_t>(__popc(qv)));
    qbase = __shfl_sync(full, qbase, leader);
    if (queued) S.queue[qbase + __popc(qv & ((1u << lane) - 1u))] = slot;
  }
  const unsigned lv = __ballot_sync(full, live);
  if (lane == 0 && lv != 0u) atomicAdd(&S.counts[1], static_cast<uint32_t>(__popc(lv)));
  if (err) atomicOr(L.error, err);
  if (L.counters) {
    uint32_t g = c_grid, t = c_tris;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      g += __shfl_xor_sync(full, g, o);
      t += __shfl_xor_sync(full, t, o);
    }
    if (lane == 0) {
      if (t) atomicAdd(&L.counters[2], static_cast<unsigned long long>(t));
      if (g) atomicAdd(&L.counters[3], static_cast<unsigned long long>(g));
    }
  }
}

// The queued closest-point queries, one traversal per lane at a time: a lane
// whose query ends writes its radius and takes the next queued slot, so
// lanes do not wait for the warp's longest traversal.  The traversal is
// wos_kernel's (same initial bound and start node, same pruning), so it
// returns the same minimum.
__global__ void __launch_bounds__(kWfQueryBlock, 8) wf_query_kernel(const WosLaunch L, const WfSlots S) {
  __shared__ uint2 s_stack[kStack * kWfQueryBlock];
  uint2 *stack = s_stack + threadIdx.x;
  const unsigned full = 0xffffffffu;
  const uint32_t n = *reinterpret_cast<volatile uint32_t *>(&S.counts[0]);
  const uint32_t stride = gridDim.x * blockDim.x;
  const int units = L.units > 0 ? L.units : 1;
  uint32_t err = 0, c_nodes = 0, c_planes = 0, c_tris = 0;
  uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
  // Query state of this lane.
  uint32_t slot = 0, flags = 0, best_tri = 0, tri_cur = 0, tri_end = 0, iter = 0;
  Vec<float> pos{0.f, 0.f, 0.f};
  float best2 = 0.f;
  int node = 0, sp = 0;
  bool have = false, found = false, active = false;
  const GeoDesc *G = nullptr;

  auto load = [&](uint32_t q) {
    slot = S.queue[q];
    const float4 P = S.pos[slot];
    const uint4 M = S.meta[slot];
    pos = {P.x, P.y, P.z};
    best2 = P.w;
    best_tri = M.z;
    flags = M.w;
    found = (flags & kWfFound) != 0u;
    G = &L.geos[L.jobs[flags >> 8].geo];
    node = S.node[slot];
    sp = 0;
    have = true;
    tri_cur = tri_end = 0;
    iter = 0;
  };
  if (qi < n) {
    load(qi);
    active = true;
  }
  while (__any_sync(full, active)) {
    if (active) {
      for (int unit = 0; unit < units && active; ++unit) {
        bool end = false;
        if (++iter > G->max_iter) {
          err |= TWOS_DEVERR_ITER;
          found = false;
          end = true;
        } else if (tri_cur < tri_end) {
          ++c_planes;
          if (tri_test(G->tris_f, tri_cur, pos, best2, c_tris)) {
            found = true;
            best_tri = tri_cur;
            flags |= kWfTriOk;
          }
          ++tri_cur;
        } else {
          while (!have && sp > 0) {
            --sp;
            const uint2 e = stack[sp * kWfQueryBlock];
            if (__uint_as_float(e.y) < best2) {
              node = static_cast<int>(e.x);
              have = true;
            }
          }
          if (!have) {
            end = true;
          } else {
            if (node >= 0) {
              ++c_nodes;
              float dl, dr;
              int cl, cr;
              node_dist2(G->nodes_f, node, pos, dl, dr, cl, cr);
              const bool vl = dl < best2, vr = dr < best2;
              if (vl && vr) {
                if (dr < dl) {
                  const float td = dl;
                  dl = dr;
                  dr = td;
                  const int tc = cl;
                  cl = cr;
                  cr = tc;
                }
                if (sp >= kStack) {
                  err |= TWOS_DEVERR_STACK;
                  found = false;
                  end = true;
                } else {
                  stack[sp * kWfQueryBlock] = make_uint2(static_cast<uint32_t>(cr), __float_as_uint(dr));
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
            if (!end && have && node < 0) {
              const uint32_t enc = ~static_cast<uint32_t>(node);
              tri_cur = enc >> 3;
              tri_end = tri_cur + (enc & 7u);
              have = false;
            }
          }
        }
        if (end) {
          // The radius for the next step kernel.
          reinterpret_cast<float *>(S.pos)[4ull * slot + 3] = best2;
          S.meta[slot].z = best_tri;
          S.meta[slot].w = (flags & ~kWfFound) | (found ? kWfFound : 0u);
          qi += stride;
          active = qi < n;
          if (active) load(qi);
        }
      }
    }
  }
  if (err) atomicOr(L.error, err);
  if (L.counters) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      c_nodes += __shfl_xor_sync(full, c_nodes, o);
      c_planes += __shfl_xor_sync(full, c_planes, o);
      c_tris += __shfl_xor_sync(full, c_tris, o);
    }
    if ((threadIdx.x & 31u) == 0) {
      if (c_nodes) atomicAdd(&L.counters[0], static_cast<unsigned long long>(c_nodes));
      if (c_planes) atomicAdd(&L.counters[1], static_cast<unsigned long long>(c_planes));
      if (c_tris) atomicAdd(&L.counters[2], static_cast<unsigned long long>(c_tris));
    }
  }
}

// Bytes of slot storage for `slots` walks in flight.
size_t wf_slot_bytes(uint32_t slots) {
  return static_cast<size_t>(slots) * (sizeof(float4) + sizeof(uint4) + sizeof(float2) + 2 * sizeof(uint32_t)) + 64;
}

WfSlots wf_slots_at(void *base, uint32_t slots) {
  WfSlots S{};
  unsigned char *p = static_cast<unsigned char *>(base);
  S.pos = reinterpret_cast<float4 *>(p);
  p += static_cast<size_t>(slots) * sizeof(float4);
  S.meta = reinterpret_cast<uint4 *>(p);
  p += static_cast<size_t>(slots) * sizeof(uint4);
  S.val = reinterpret_cast<float2 *>(p);
  p += static_cast<size_t>(slots) * sizeof(float2);
  S.node = reinterpret_cast<int *>(p);
  p += static_cast<size_t>(slots) * sizeof(int);
  S.queue = reinterpret_cast<uint32_t *>(p);
  p += static_cast<size_t>(slots) * sizeof(uint32_t);
  S.counts = reinterpret_cast<uint32_t *>(p);
  S.slots = slots;
  return S;
}

cudaError_t launch_wos_wavefront(int mode, const WosLaunch &L, void *slot_mem, uint32_t slots, int num_sms,
                                 uint64_t max_iterations, cudaStream_t s) {
  if (slots == 0 || slots % kWfStepBlock || L.total_walks >= (1ull << 32) || num_sms <= 0)
    return cudaErrorInvalidValue;
  int per_sm = 0;
  cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wf_query_kernel, kWfQueryBlock, 0);
  if (oe != cudaSuccess) return oe;
  if (per_sm <= 0) return cudaErrorInvalidConfiguration;
  const int query_grid = per_sm * num_sms;
  const WfSlots S = wf_slots_at(slot_mem, slots);
  const size_t smem = static_cast<size_t>(L.n_terms) * sizeof(TermT<float>);
  const unsigned step_blocks = slots / kWfStepBlock;
  void (*step)(const WosLaunch, const WfSlots) = mode == TWOS_MODE_PAIRED ? wf_step_kernel<TWOS_MODE_PAIRED>
                                                 : mode == TWOS_MODE_HOT  ? wf_step_kernel<TWOS_MODE_HOT>
                                                                          : wf_step_kernel<TWOS_MODE_COMPLIANCE>;
  cudaError_t e = cudaMemsetAsync(S.meta, 0, static_cast<size_t>(slots) * sizeof(uint4), s);
  if (e != cudaSuccess) return e;
  // Chunks of iterations; the live count of a chunk's last iteration is read
  // back while the next chunk runs (double-buffered), so the device does not
  // wait for the host.
  constexpr int kChunk = 16;
  uint32_t *h_live = nullptr;
  if ((e = cudaMallocHost(&h_live, 2 * sizeof(uint32_t))) != cudaSuccess) return e;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  for (auto &x : ev)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
  uint64_t it = 0;
  int chunk = 0;
  bool finished = false;
  while (e == cudaSuccess && !finished) {
    for (int k = 0; k < kChunk && e == cudaSuccess; ++k, ++it) {
      if ((e = cudaMemsetAsync(S.counts, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) break;
      step<<<step_blocks, kWfStepBlock, smem, s>>>(L, S);
      wf_query_kernel<<<query_grid, kWfQueryBlock, 0, s>>>(L, S);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) break;
    const int b = chunk & 1;
    if ((e = cudaMemcpyAsync(h_live + b, S.counts + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      break;
    if ((e = cudaEventRecord(ev[b], s)) != cudaSuccess) break;
    if (chunk > 0) {
      // The previous chunk's count (its copy is done once its event is).
      if ((e = cudaEventSynchronize(ev[b ^ 1])) != cudaSuccess) break;
      if (h_live[b ^ 1] == 0u) finished = true;
    }
    ++chunk;
    if (!finished && it > max_iterations) {
      e = cudaErrorLaunchTimeout;  // reported as a launch failure; never expected
      break;
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  for (auto &x : ev)
    if (x) cudaEventDestroy(x);
  cudaFreeHost(h_live);
  return e;
}

}  // namespace twos

// rm_batch.cu - many plain-path images rendered together by one pool of path
// slots (wavefront stages over compacted queues, persistent grid-stride
// kernels whose grids do not depend on queue lengths, so a sequence of waves
// can be captured in a CUDA graph once and replayed).
//
// Each image follows the reference's plain chain: render_paths (K1,
// pathtrace.metal:739-769) with one lane per pixel, or render_paths_simd (K2,
// :773-815) with 8 or 32 lanes per pixel that take one sample each per round,
// are summed with a butterfly reduction, and stop early when the adaptive test
// (:759-764) passes at the end of a round.  Here every lane is a slot of the
// pool with its own random stream; a lane that finishes its sample of the
// round publishes it, and the last lane of the pixel to finish queues the
// pixel; a combine pass then gives each queued pixel L lanes of a warp, which
// sum the round with the same shuffles as K2, run the adaptive test and either
// queue the next round's lane slots or write the pixel.  So the images, random
// streams and sample counts equal those of the one-image lane kernels bit for
// bit, whatever the mix of images in the pool.
//
// Per wave:  refill  chunks that finished their tile take the batch's next tile;
//            start   lane slots start their sample of the round (camera ray);
//            trace   closest hit of every extension ray (stochastic alpha
//                    crossings in partially transparent scenes, with the
//                    slot's random stream, as pathtrace.metal:536-550),
//                    then any hit of every deferred shadow ray;
//            shade   one vertex per path (rm_wf_common.cuh), by surface type;
//            combine the pixels whose round is complete, one warp lane per
//                    pixel lane, with K2's own shuffles.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"
#include "rm_wf_common.cuh"

namespace rmd {

namespace {

using namespace wf;

__device__ __forceinline__ void tile_pixel(const BtJob& J, int tile, int g, int& x, int& y) {
  const int tx = tile % J.tiles_x, ty = tile / J.tiles_x;
  x = tx * J.tile_w + g % J.tile_w;
  y = ty * J.tile_h + g / J.tile_w;
}

__device__ __forceinline__ void bload(const BtState& w, int i, PathRegs& r, uint32_t& rng) {
  const uint4 u = w.u[i];
  rng = u.x; r.meta = u.y; r.v = int(u.z);
  const float4 acc = w.acc[i], thr = w.thr[i], pb = w.pb[i], o = w.o[i], d = w.d[i];
  r.ax = acc.x; r.ay = acc.y; r.az = acc.z; r.psumW = acc.w;
  r.tx = thr.x; r.ty = thr.y; r.tz = thr.z; r.pbcos = thr.w;
  r.pbr = pb.x; r.pbg = pb.y; r.pbb = pb.z; r.pM = uint32_t(__float_as_int(pb.w));
  r.ox = o.x; r.oy = o.y; r.oz = o.z; r.last_pdf = o.w;
  r.dx = d.x; r.dy = d.y; r.dz = d.z;
}

__device__ __forceinline__ void bstore(const BtState& w, int i, const PathRegs& r, uint32_t rng) {
  w.u[i] = make_uint4(rng, r.meta, uint32_t(r.v), 0u);
  w.acc[i] = make_float4(r.ax, r.ay, r.az, r.psumW);
  w.thr[i] = make_float4(r.tx, r.ty, r.tz, r.pbcos);
  w.pb[i] = make_float4(r.pbr, r.pbg, r.pbb, __int_as_float(int(r.pM)));
  w.o[i] = make_float4(r.ox, r.oy, r.oz, r.last_pdf);
  w.d[i] = make_float4(r.dx, r.dy, r.dz, 0.f);
}

// A lane's sample of the round is done (value already clamped): publish it.
// Returns true for the pixel's last lane of the round, which queues the pixel
// for k_bt_combine.  The slot's RNG state must be stored before this (the
// pixel's output XORs the lanes' states).
__device__ __forceinline__ bool arrive(const BtState& w, const BtJob& J, int i, float fr, float fg, float fb,
                                       int& g0) {
  const int chunk = i >> 5, k = i & 31;
  const int L = J.lanes, g = k / L;
  g0 = (chunk << 5) + g * L;
  w.val[i] = make_float4(fr, fg, fb, 0.f);
  const int takers = min(L, J.p.spp - w.gbase[g0]);
  __threadfence();
  const int old = atomicAdd(&w.garr[g0], 1);
  if (old + 1 != takers) return false;
  __threadfence();
  return true;
}

// Queue a pixel whose round is complete by its lane count; every thread of the
// warp must reach this.
__device__ __forceinline__ void queue_round(const BtQueues& q, int lanes, int g0) {
  append(q.cm1, q.counts + kBtCm1, lanes == 1, g0);
  append(q.cm8, q.counts + kBtCm8, lanes == 8, g0);
  append(q.cm32, q.counts + kBtCm32, lanes == 32, g0);
}

__global__ void k_bt_init(BtState w, BtQueues q0, int chunks, int* next_tile) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < chunks) {
    q0.rf[i] = i;
    w.cjob[i] = -1;
  }
  if (i < kBtCounts) q0.counts[i] = i == kBtRf ? chunks : 0;
  if (i == 0) *next_tile = 0;
}

// Chunks whose tile is done take the next tile of the batch (one warp per
// chunk) and queue their lane slots to start round 0.
__global__ void __launch_bounds__(256) k_bt_refill(BtBatch b, BtState w, BtQueues q) {
  const int n = q.counts[kBtRf];
  const int k = int(threadIdx.x & 31);
  const int stride = int(gridDim.x * blockDim.x);
  for (int base = int(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); base < n * kBtChunk; base += stride) {
    const int chunk = q.rf[base >> 5];
    int t = 0;
    if (k == 0) t = atomicAdd(b.next_tile, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= b.total_tiles) {
      if (k == 0) w.cjob[chunk] = -1;
      continue;
    }
    int lo = 0, hi = b.n_jobs - 1;  // last job whose first tile is <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b.tile_begin[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const BtJob& J = b.jobs[lo];
    const int tile = t - J.tile_begin;
    const int L = J.lanes, g = k / L, lane = k % L;
    int x, y;
    tile_pixel(J, tile, g, x, y);
    const bool present = x < J.p.width && y < J.p.height;
    const int slot = (chunk << 5) + k;
    if (present && lane == 0) {
      w.gsum[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
      w.gsl2[slot] = 0.f;
      w.gbase[slot] = 0;
      w.garr[slot] = 0;
    }
    const unsigned groups = __ballot_sync(0xffffffffu, present && lane == 0);
    if (k == 0) {
      w.cjob[chunk] = lo;
      w.ctile[chunk] = tile;
      w.cleft[chunk] = __popc(groups);
    }
    append(q.st, q.counts + kBtSt, present, slot);
  }
}

// Start the round's sample of each queued lane slot: the jitter and camera ray
// of K1 / K2 (pathtrace.metal:754-756, :792-794; sample_sensor :729-737).
__global__ void __launch_bounds__(256) k_bt_start(BtBatch b, BtState w, BtQueues q, unsigned long long* ctr,
                                                  uint32_t* err) {
  const int n = q.counts[kBtSt];
  const int stride = int(gridDim.x * blockDim.x);
  uint32_t samples = 0;
  for (int base = int(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); base < n; base += stride) {
    const int qi = base + int(threadIdx.x & 31);
    bool ext = false;
    int i = 0, g0 = 0, round_lanes = 0;
    if (qi < n) {
      i = q.st[qi];
      const int chunk = i >> 5, k = i & 31;
      const BtJob& J = b.jobs[w.cjob[chunk]];
      const int L = J.lanes, g = k / L, lane = k % L;
      g0 = (chunk << 5) + g * L;
      int x, y;
      tile_pixel(J, w.ctile[chunk], g, x, y);
      Tracer pt(J.s, J.p, err);
      if (w.gbase[g0] == 0) {
        uint64_t sd = seed_pixel(J.seed, uint32_t(x), uint32_t(y));
        if (L > 1) sd ^= uint64_t(lane) * 0x94D049BB133111EBull;
        pt.rng.seed(sd);
      } else {
        pt.rng.state = w.u[i].x;
      }
      float sx, sy;
      pt.jitter(uint32_t(x), uint32_t(y), sx, sy);
      const rm_camera& cam = J.p.camera;
      const float focal2 = cam.focal * cam.focal;
      const float dist = 1.0f / sqrtf(sx * sx + (sy * sy + focal2));
      const float tx = sx * dist, ty = sy * dist, tz = cam.focal * dist;
      PathRegs r;
      r.dx = tx * cam.m0 + (ty * cam.m1 + tz * cam.m2);
      r.dy = tx * cam.m3 + (ty * cam.m4 + tz * cam.m5);
      r.dz = tx * cam.m6 + (ty * cam.m7 + tz * cam.m8);
      r.ox = cam.x; r.oy = cam.y; r.oz = cam.z;
      r.ax = r.ay = r.az = 0.0f;
      r.tx = r.ty = r.tz = 1.0f;
      r.v = 0;
      r.meta = kDelta;
      r.last_pdf = 0.0f; r.psumW = 0.0f; r.pM = 0;
      r.pbr = r.pbg = r.pbb = r.pbcos = 0.0f;
      if (J.p.bounces > 0) {
        r.meta |= kExt;
        bstore(w, i, r, pt.rng.state);
        ext = true;
      } else {  // no bounce: the sample is zero
        w.u[i] = make_uint4(pt.rng.state, 0u, 0u, 0u);
        float fr = 0.f, fg = 0.f, fb = 0.f;
        clamp3(J.p, fr, fg, fb);
        ++samples;
        if (arrive(w, J, i, fr, fg, fb, g0)) round_lanes = L;
      }
    }
    append(q.ext, q.counts + kBtExt, ext, i);
    queue_round(q, round_lanes, g0);
  }
  __syncwarp();
  warp_add(ctr + 0, samples);
}

// Traversal of a queue of rays, one thread per ray (closest hit for extension
// rays, pathtrace.metal:119-163 and :536-550; any hit for shadow rays, :164).
// Finished extension rays are sorted into the shading queue of their surface
// type.
// One ray of a batch job: through the 8-wide BVH (kWide, when the job's scene
// has one) or the binary BVH; both give the same hit.
template <bool kAnyHit, bool kWide>
__device__ __forceinline__ TraceResult bt_traverse(const Scene& s, float ox, float oy, float oz, float dx, float dy,
                                                   float dz, float tmax, uint32_t* err, uint32_t& nodes,
                                                   uint32_t& tests) {
  if (kWide) return traverse_any<kAnyHit>(s, ox, oy, oz, dx, dy, dz, tmax, err, nodes, tests);
  return traverse<kAnyHit>(s, ox, oy, oz, dx, dy, dz, tmax, err, nodes, tests);
}

// Ten 128-thread blocks per SM (48 registers, ~100 bytes of spills; nine at
// 55), and three 256-thread k_bt_shade blocks (80 registers, against two at
// 113): batched config-3 rendering 914 against 866 M path samples/s.
template <bool kShadowRays, bool kWide>
__global__ void __launch_bounds__(128, 10) k_bt_trace(BtBatch b, BtState w, BtQueues q, unsigned long long* ctr,
                                                  uint32_t* err) {
  const int n = q.counts[kShadowRays ? kBtShd : kBtExt];
  const int* queue = kShadowRays ? q.shd : q.ext;
  const int stride = int(gridDim.x * blockDim.x);
  uint32_t nodes = 0, tests = 0, rays = 0;
  for (int base = int(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); base < n; base += stride) {
    const int qi = base + int(threadIdx.x & 31);
    int cls = -1;  // the shading queue: 0 a, 1 b (dielectric), 2 c (miss), 3 d
    int i = 0;
    if (qi < n) {
      i = queue[qi];
      const BtJob& J = b.jobs[w.cjob[i >> 5]];
      const Scene& s = J.s;
      if (kShadowRays) {
        const float4 o = w.so[i], d = w.sd[i];
        const TraceResult r = bt_traverse<true, kWide>(s, o.x, o.y, o.z, d.x, d.y, d.z, o.w, err, nodes, tests);
        ++rays;
        w.occ[i] = r.tri >= 0 ? 1u : 0u;
      } else {
        const float4 o = w.o[i], d = w.d[i];
        TraceResult r;
        if (J.p.opaque) {
          r = bt_traverse<false, kWide>(s, o.x, o.y, o.z, d.x, d.y, d.z, kFar, err, nodes, tests);
          ++rays;
        } else {
          // stochastic coverage: step through transparent crossings
          Rng rng;
          rng.state = w.u[i].x;
          r.tri = -1;
          r.t = kFar;
          float traveled = 0.0f;
          float hx = o.x, hy = o.y, hz = o.z;
          for (int it = 0; it < kMaxAlphaCrossings && traveled < kFar; ++it) {
            const float qx = o.x + d.x * traveled, qy = o.y + d.y * traveled, qz = o.z + d.z * traveled;
            const TraceResult h =
                bt_traverse<false, kWide>(s, qx, qy, qz, d.x, d.y, d.z, kFar - traveled, err, nodes, tests);
            ++rays;
            if (h.tri < 0) break;
            const float opacity = s.tris[h.tri].alpha;
            if (opacity >= 1.0f || (opacity > 0.0f && rng.uniform01() < opacity)) {
              r = h;
              hx = qx; hy = qy; hz = qz;
              break;
            }
            traveled += h.t + 0.0001f;
          }
          w.u[i].x = rng.state;
          w.hoff[i] = make_float4(hx, hy, hz, 0.f);
        }
        w.hit[i] = make_float4(r.t, r.u, r.v, __int_as_float(r.tri));
        cls = 2;
        if (r.tri >= 0)
          cls = __ldg(&s.tris[r.tri].ior) > 1.0001f ? 1 : ((J.p.opaque && J.p.restir_candidates <= 1) ? 0 : 3);
      }
    }
    if (!kShadowRays) {
      append(q.qa, q.counts + kBtA, cls == 0, i);
      append(q.qb, q.counts + kBtB, cls == 1, i);
      append(q.qc, q.counts + kBtC, cls == 2, i);
      append(q.qd, q.counts + kBtD, cls == 3, i);
    }
  }
  __syncwarp();
  warp_add(ctr + 1, rays);
  warp_add(ctr + 2, nodes);
  warp_add(ctr + 3, tests);
}

// Shade the paths of one queue: VK 0 opaque hits in opaque scenes with
// single-candidate NEE, 1 dielectric hits, 2 paths without a vertex (the ray
// missed, or the path ended and waited for its last shadow ray), 3 other
// opaque hits.  A path that ends finishes its lane's sample of the round.
template <int VK>
__global__ void __launch_bounds__(256, 3) k_bt_shade(BtBatch b, BtState w, BtQueues cq, BtQueues nq,
                                                  unsigned long long* ctr, uint32_t* err) {
  const int count = cq.counts[VK == 0 ? kBtA : VK == 1 ? kBtB : VK == 2 ? kBtC : kBtD];
  const int* queue = VK == 0 ? cq.qa : VK == 1 ? cq.qb : VK == 2 ? cq.qc : cq.qd;
  const int stride = int(gridDim.x * blockDim.x);
  uint32_t samples = 0, rays = 0, nodes = 0, tests = 0;
  for (int base = int(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); base < count; base += stride) {
    const int qi = base + int(threadIdx.x & 31);
    bool ext = false, shd = false, fin = false;
    int i = 0, g0 = 0, round_lanes = 0;
    if (qi < count) {
      i = queue[qi];
      const BtJob& J = b.jobs[w.cjob[i >> 5]];
      Tracer pt(J.s, J.p, err);
      PathRegs r;
      bload(w, i, r, pt.rng.state);
      if (r.meta & kShadow) {
        r.meta &= ~kShadow;
        if (w.occ[i] == 0u) {
          const float4 c = w.c[i];
          r.ax += c.x; r.ay += c.y; r.az += c.z;
        }
      }
      bool ended;
      if (VK == 2) {
        ended = true;  // a miss ends the path; a finishing path has now folded in its last shadow ray
        r.meta &= ~(kExt | kFinish);
      } else {
        r.meta &= ~kExt;
        const float4 hh = w.hit[i];
        const TraceResult tr{hh.x, __float_as_int(hh.w), hh.y, hh.z};
        Hit hit;
        if (J.p.opaque) {
          hit = pt.attributes(tr, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz);
        } else {
          const float4 ho = w.hoff[i];
          hit = pt.attributes(tr, ho.x, ho.y, ho.z, r.dx, r.dy, r.dz);
        }
        bool has_shadow = false;
        float4 so, sd, c;
        const bool go = VK == 3 ? vertex<0, 1>(pt, J.p, r, hit, has_shadow, so, sd, c)
                                : vertex<VK == 1 ? 1 : 0, VK == 0 ? 0 : 1>(pt, J.p, r, hit, has_shadow, so, sd, c);
        if (has_shadow) {
          w.so[i] = so; w.sd[i] = sd; w.c[i] = c;
          r.meta |= kShadow;
          shd = true;
        }
        if (go) { r.meta |= kExt; ext = true; }
        ended = !go;
        if (ended && has_shadow) { r.meta |= kFinish; ended = false; fin = true; }  // wait for the shadow ray
      }
      bstore(w, i, r, pt.rng.state);
      if (ended) {
        float fr = r.ax, fg = r.ay, fb = r.az;
        clamp3(J.p, fr, fg, fb);
        ++samples;
        if (arrive(w, J, i, fr, fg, fb, g0)) round_lanes = J.lanes;
      }
      rays += pt.rays; nodes += pt.nodes; tests += pt.tests;
    }
    append(nq.ext, nq.counts + kBtExt, ext, i);
    append(nq.shd, nq.counts + kBtShd, shd, i);
    append(nq.qc, nq.counts + kBtC, fin, i);
    queue_round(cq, round_lanes, g0);
  }
  __syncwarp();
  warp_add(ctr + 0, samples);
  warp_add(ctr + 1, rays);
  warp_add(ctr + 2, nodes);
  warp_add(ctr + 3, tests);
}

// Pixels whose round is complete, `L` lanes each, L lanes of a warp per pixel:
// the round's butterfly sum exactly as K2 does it (pathtrace.metal:797-805,
// shuffles of width L), then the adaptive test (:806-810) and either the next
// round's lane slots queued to start or the pixel's output (:811-814; K1
// :759-768 is the one-lane case).
template <int L>
__global__ void __launch_bounds__(256) k_bt_combine(BtBatch b, BtState w, BtQueues q, BtQueues nq) {
  const int n = q.counts[L == 1 ? kBtCm1 : L == 8 ? kBtCm8 : kBtCm32];
  const int* queue = L == 1 ? q.cm1 : L == 8 ? q.cm8 : q.cm32;
  const int lane = int(threadIdx.x & 31), k = lane % L;
  const int stride = int(gridDim.x * blockDim.x) / L;  // pixels per sweep of the grid
  for (int base = int(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)) / L; base < n; base += stride) {
    const int e = base + lane / L;
    const bool valid = e < n;
    int g0 = 0, m = 0;
    float cr = 0.f, cg = 0.f, cb = 0.f;
    uint32_t st = 0;
    const BtJob* J = nullptr;
    int rbase = 0;
    if (valid) {
      g0 = queue[e];
      J = &b.jobs[w.cjob[g0 >> 5]];
      rbase = w.gbase[g0];
      if (k < J->p.spp - rbase) {
        const float4 a = w.val[g0 + k];
        cr = a.x; cg = a.y; cb = a.z;
      }
      st = w.u[g0 + k].x;
    }
    float lum = cr * 0.2126f + cg * 0.7152f + cb * 0.0722f;
    float lum2 = lum * lum;
#pragma unroll
    for (int mm = 1; mm < L; mm <<= 1) {
      cr += __shfl_xor_sync(0xffffffffu, cr, mm, L);
      cg += __shfl_xor_sync(0xffffffffu, cg, mm, L);
      cb += __shfl_xor_sync(0xffffffffu, cb, mm, L);
      lum += __shfl_xor_sync(0xffffffffu, lum, mm, L);
      lum2 += __shfl_xor_sync(0xffffffffu, lum2, mm, L);
      st ^= __shfl_xor_sync(0xffffffffu, st, mm, L);
    }
    if (valid) {
      // every lane of the pixel holds the same sums and takes the same decision
      const Params& p = J->p;
      float4 gs = w.gsum[g0];
      float sl2 = w.gsl2[g0];
      gs.x += cr; gs.y += cg; gs.z += cb; gs.w += lum;
      sl2 += lum2;
      const int nn = min(rbase + L, p.spp);
      bool stop = nn >= p.spp;
      if (!stop && p.adapt_min > 0 && nn >= p.adapt_min && nn > 1 && nn % p.adapt_step == 0) {
        float mean = gs.w / float(nn);
        float var = fmaxf(0.0f, (sl2 - gs.w * mean) / float(nn - 1));
        float thr = p.adapt_rel * mean + p.adapt_abs;
        if (var < thr * thr) stop = true;
      }
      if (stop) {
        if (k == 0) {
          const int chunk = g0 >> 5;
          int x, y;
          tile_pixel(*J, w.ctile[chunk], (g0 & 31) / L, x, y);
          const size_t pix = size_t(y) * size_t(p.width) + size_t(x);
          const float fr = gs.x / float(nn), fg = gs.y / float(nn), fb = gs.z / float(nn);
          if (J->hdr) { J->hdr[pix * 3] = fr; J->hdr[pix * 3 + 1] = fg; J->hdr[pix * 3 + 2] = fb; }
          if (J->rgb) {
            J->rgb[pix * 3] = tonemap8(fr); J->rgb[pix * 3 + 1] = tonemap8(fg); J->rgb[pix * 3 + 2] = tonemap8(fb);
          }
          if (J->dbg) { J->dbg[pix * 2] = st; J->dbg[pix * 2 + 1] = uint32_t(nn); }
          if (atomicSub(&w.cleft[chunk], 1) == 1) {
            const int pos = atomicAdd(nq.counts + kBtRf, 1);
            nq.rf[pos] = chunk;
          }
        }
      } else {
        __syncwarp(0xffffffffu >> (32 - L) << (lane & ~(L - 1)));  // the group's reads of the old sums are done
        if (k == 0) {
          w.gsum[g0] = gs;
          w.gsl2[g0] = sl2;
          w.gbase[g0] = rbase + L;
          w.garr[g0] = 0;
        }
        m = min(L, p.spp - (rbase + L));
      }
    }
    append(nq.st, nq.counts + kBtSt, k < m, g0 + k);
  }
}

}  // namespace

cudaError_t launch_batch_init(const BtState& w, const BtQueues& q0, int chunks, int* next_tile, cudaStream_t st) {
  const int n = chunks > kBtCounts ? chunks : kBtCounts;
  k_bt_init<<<(n + 255) / 256, 256, 0, st>>>(w, q0, chunks, next_tile);
  return cudaGetLastError();
}

cudaError_t launch_batch_refill(const BtBatch& b, const BtState& w, const BtQueues& q, int grid, cudaStream_t st) {
  k_bt_refill<<<grid, 256, 0, st>>>(b, w, q);
  return cudaGetLastError();
}

cudaError_t launch_batch_start(const BtBatch& b, const BtState& w, const BtQueues& q, const BtQueues& nq, int grid,
                               unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  (void)nq;
  k_bt_start<<<grid, 256, 0, st>>>(b, w, q, ctr, err);
  return cudaGetLastError();
}

cudaError_t launch_batch_combine(int lanes, const BtBatch& b, const BtState& w, const BtQueues& q,
                                 const BtQueues& nq, int grid, cudaStream_t st) {
  if (lanes == 1) k_bt_combine<1><<<grid, 256, 0, st>>>(b, w, q, nq);
  else if (lanes == 8) k_bt_combine<8><<<grid, 256, 0, st>>>(b, w, q, nq);
  else k_bt_combine<32><<<grid, 256, 0, st>>>(b, w, q, nq);
  return cudaGetLastError();
}

cudaError_t launch_batch_trace(const BtBatch& b, const BtState& w, const BtQueues& q, bool shadow, bool wide,
                               int grid, unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  if (wide) {
    if (shadow) k_bt_trace<true, true><<<grid, 128, 0, st>>>(b, w, q, ctr, err);
    else k_bt_trace<false, true><<<grid, 128, 0, st>>>(b, w, q, ctr, err);
  } else {
    if (shadow) k_bt_trace<true, false><<<grid, 128, 0, st>>>(b, w, q, ctr, err);
    else k_bt_trace<false, false><<<grid, 128, 0, st>>>(b, w, q, ctr, err);
  }
  return cudaGetLastError();
}

cudaError_t launch_batch_shade(int vk, const BtBatch& b, const BtState& w, const BtQueues& q, const BtQueues& nq,
                               int grid, unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  if (vk == 0) k_bt_shade<0><<<grid, 256, 0, st>>>(b, w, q, nq, ctr, err);
  else if (vk == 1) k_bt_shade<1><<<grid, 256, 0, st>>>(b, w, q, nq, ctr, err);
  else if (vk == 2) k_bt_shade<2><<<grid, 256, 0, st>>>(b, w, q, nq, ctr, err);
  else k_bt_shade<3><<<grid, 256, 0, st>>>(b, w, q, nq, ctr, err);
  return cudaGetLastError();
}

void batch_occupancy(int& aux, int& trace, int& shade) {
  aux = trace = shade = 1;
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_bt_start, 256, 0) == cudaSuccess && v > 0) aux = v;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_bt_trace<false, false>, 128, 0) == cudaSuccess && v > 0)
    trace = v;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_bt_shade<0>, 256, 0) == cudaSuccess && v > 0) shade = v;
}

}  // namespace rmd

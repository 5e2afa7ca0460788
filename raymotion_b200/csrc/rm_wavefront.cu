// rm_wavefront.cu - ReSTIR shading (reference restir_shade, pathtrace.metal:1056-1258)
// as wavefront stages over compacted queues.
//
// The reference shades with one thread per pixel that loops over all samples
// of its pixel; on a GPU the 32 threads of a warp are then almost never in the
// same phase (traversal, RIS candidates, BSDF sampling, next sample).  Here a
// frame runs in waves of three kernels:
//   k_wf_extend  closest-hit traversal of every queued extension ray,
//   k_wf_shadow  any-hit traversal of every queued shadow ray,
//   k_wf_shade   for every path touched this wave: fold in its shadow result,
//                shade its hit, sample the next direction, and queue its next
//                rays (or finish the sample and start the next one),
// with warp-aggregated atomic appends building the next wave's queues.
//
// Results stay bit-identical to the one-thread-per-pixel kernel because
// (i) each pixel has at most one path in flight, so its random stream is
// consumed in the same order; (ii) the scene is opaque (ReSTIR requires it,
// metal.mm:237), so a shadow test consumes no random numbers and only gates
// the light contribution, which is computed at the vertex and added to the
// path sum at the start of the next shade, before anything else is added;
// (iii) every expression keeps the reference's operand order.
#include <cuda_runtime.h>

#include "rm_device.cuh"
#include "rm_launch.h"
#include "rm_wf_common.cuh"

namespace rmd {

namespace {

using namespace wf;

__device__ __forceinline__ void load(const WfState& w, uint32_t i, PathRegs& r, uint32_t& rng, uint32_t& n,
                                     float& sr, float& sg, float& sb) {
  const uint4 u = w.u[i];
  rng = u.x; r.meta = u.y; n = u.z; r.v = int(u.w);
  const float4 sum = w.sum[i], acc = w.acc[i], thr = w.thr[i], pb = w.pb[i], o = w.o[i], d = w.d[i];
  sr = sum.x; sg = sum.y; sb = sum.z; r.last_pdf = sum.w;
  r.ax = acc.x; r.ay = acc.y; r.az = acc.z; r.psumW = acc.w;
  r.tx = thr.x; r.ty = thr.y; r.tz = thr.z; r.pbcos = thr.w;
  r.pbr = pb.x; r.pbg = pb.y; r.pbb = pb.z; r.pM = uint32_t(__float_as_int(pb.w));
  r.ox = o.x; r.oy = o.y; r.oz = o.z; r.dx = d.x; r.dy = d.y; r.dz = d.z;
}

__device__ __forceinline__ void store(const WfState& w, uint32_t i, const PathRegs& r, uint32_t rng, uint32_t n,
                                      float sr, float sg, float sb) {
  w.u[i] = make_uint4(rng, r.meta, n, uint32_t(r.v));
  w.sum[i] = make_float4(sr, sg, sb, r.last_pdf);
  w.acc[i] = make_float4(r.ax, r.ay, r.az, r.psumW);
  w.thr[i] = make_float4(r.tx, r.ty, r.tz, r.pbcos);
  w.pb[i] = make_float4(r.pbr, r.pbg, r.pbb, __int_as_float(int(r.pM)));
  w.o[i] = make_float4(r.ox, r.oy, r.oz, 0.f);
  w.d[i] = make_float4(r.dx, r.dy, r.dz, 0.f);
}

// Pixel constants of a kind-1 pixel (pathtrace.metal:1086-1128): the primary
// direct light from the merged reservoir.
struct Pixel1 {
  float gpx, gpy, gpz, gnx, gny, gnz, wox, woy, woz, ar, ag, ab, rough, metallic, alpha2, spec_prob;
};

__device__ __forceinline__ Pixel1 pixel1(const GBufSoA& gb, uint32_t id) {
  const float4 PK = gb.pos_kind[id], NR = gb.nor_rough[id], AM = gb.alb_met[id], WO = gb.wo_ior[id];
  Pixel1 q;
  q.gpx = PK.x; q.gpy = PK.y; q.gpz = PK.z; q.gnx = NR.x; q.gny = NR.y; q.gnz = NR.z;
  q.wox = WO.x; q.woy = WO.y; q.woz = WO.z; q.ar = AM.x; q.ag = AM.y; q.ab = AM.z;
  float rough = NR.w; if (rough < 0.0f) rough = 0.0f; if (rough > 1.0f) rough = 1.0f;
  float metallic = AM.w; if (metallic < 0.0f) metallic = 0.0f; if (metallic > 1.0f) metallic = 1.0f;
  float r2 = rough; if (r2 < 0.02f) r2 = 0.02f;
  q.alpha2 = (r2 * r2) * (r2 * r2);
  float sp = 0.05f + 0.95f * metallic; if (sp > 0.98f) sp = 0.98f;
  if (metallic >= 0.999f) sp = 1.0f;
  q.rough = rough; q.metallic = metallic; q.spec_prob = sp;
  return q;
}

// Start samples of a pixel until one has a ray to trace or all spp are done.
// Returns true when an extension ray was produced.
__device__ bool start_samples(Tracer& pt, const Params& p, const GBufSoA& gb, const WfState& w, uint32_t id,
                              uint32_t x, uint32_t y, PathRegs& r, uint32_t& n, float& sr, float& sg, float& sb) {
  const bool ind = (r.meta & kInd) != 0;
  if (ind) {
    const Pixel1 q = pixel1(gb, id);
    const float4 base = w.base[id];
    const uint32_t m_M = w.mM[id];
    while (n < uint32_t(p.spp)) {
      float nx2 = 0, ny2 = 0, nz2 = 0;
      int pdelta = 0;
      bool early = false;
      if (pt.U() < q.spec_prob) {
        float hx, hy, hz;
        pt.sample_ggx_half(q.alpha2, q.gnx, q.gny, q.gnz, hx, hy, hz);
        float md = q.wox * hx + (q.woy * hy + q.woz * hz);
        if (!(md > 1e-8f)) early = true;
        else {
          nx2 = 2.0f * md * hx - q.wox; ny2 = 2.0f * md * hy - q.woy; nz2 = 2.0f * md * hz - q.woz;
          pdelta = (q.rough <= 0.0201f) ? 1 : 0;
        }
      } else {
        pt.sample_cosine(q.gnx, q.gny, q.gnz, nx2, ny2, nz2);
        pdelta = 0;
      }
      Bsdf e0{0.f, 0.f, 0.f, 0.f};
      if (!early) {
        float ncos = nx2 * q.gnx + (ny2 * q.gny + nz2 * q.gnz);
        if (!(ncos > 1e-8f)) early = true;
        else {
          float d = 1.0f / sqrtf(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
          nx2 *= d; ny2 *= d; nz2 *= d;
          e0 = Tracer::eval_bsdf(nx2, ny2, nz2, q.wox, q.woy, q.woz, q.gnx, q.gny, q.gnz, q.alpha2, q.metallic,
                                 q.spec_prob, q.ar, q.ag, q.ab);
          if (!(e0.pdf > 1e-12f)) early = true;
        }
      }
      if (early) {
        float fr = base.x, fg = base.y, fb = base.z;
        clamp3(p, fr, fg, fb);
        sr += fr; sg += fg; sb += fb;
        ++n;
        continue;
      }
      float cos0 = nx2 * q.gnx + (ny2 * q.gny + nz2 * q.gnz);
      r.tx = e0.r * cos0 / e0.pdf; r.ty = e0.g * cos0 / e0.pdf; r.tz = e0.b * cos0 / e0.pdf;
      r.ox = q.gpx + q.gnx * 0.001f; r.oy = q.gpy + q.gny * 0.001f; r.oz = q.gpz + q.gnz * 0.001f;
      r.dx = nx2; r.dy = ny2; r.dz = nz2;
      r.last_pdf = e0.pdf;
      r.pbr = e0.r; r.pbg = e0.g; r.pbb = e0.b; r.pbcos = cos0;
      r.psumW = base.w;
      r.pM = m_M;
      r.meta = (r.meta & ~kDelta) | (pdelta ? kDelta : 0u);
      r.ax = r.ay = r.az = 0.0f;
      r.v = 1;
      return true;
    }
    return false;
  }
  // camera path (kind 3): pathtrace.metal:1073-1079 and sample_sensor :729-737
  while (n < uint32_t(p.spp)) {
    float sx, sy;
    pt.jitter(x, y, sx, sy);
    const rm_camera& cam = p.camera;
    float focal2 = cam.focal * cam.focal;
    float dist = 1.0f / sqrtf(sx * sx + (sy * sy + focal2));
    float tx = sx * dist, ty = sy * dist, tz = cam.focal * dist;
    r.dx = tx * cam.m0 + (ty * cam.m1 + tz * cam.m2);
    r.dy = tx * cam.m3 + (ty * cam.m4 + tz * cam.m5);
    r.dz = tx * cam.m6 + (ty * cam.m7 + tz * cam.m8);
    r.ox = cam.x; r.oy = cam.y; r.oz = cam.z;
    r.ax = r.ay = r.az = 0.0f;
    r.tx = r.ty = r.tz = 1.0f;
    r.v = 0;
    r.meta |= kDelta;
    r.last_pdf = 0.0f; r.psumW = 0.0f; r.pM = 0;
    r.pbr = r.pbg = r.pbb = r.pbcos = 0.0f;
    if (p.bounces > 0) return true;
    float cr = 0.0f, cg = 0.0f, cb = 0.0f;  // no bounce: the path adds nothing
    clamp3(p, cr, cg, cb);
    sr += cr; sg += cg; sb += cb;
    ++n;
  }
  return false;
}

// Finish the current sample (pathtrace.metal:1077-1078 camera, :1252-1254 kind 1).
__device__ __forceinline__ void finish_sample(const Params& p, const WfState& w, uint32_t id, const PathRegs& r,
                                              uint32_t& n, float& sr, float& sg, float& sb) {
  float fr, fg, fb;
  if (r.meta & kInd) {
    const float4 base = w.base[id];
    fr = base.x + r.ax; fg = base.y + r.ay; fb = base.z + r.az;
  } else {
    fr = r.ax; fg = r.ay; fb = r.az;
  }
  clamp3(p, fr, fg, fb);
  sr += fr; sg += fg; sb += fb;
  ++n;
}

__device__ __forceinline__ void write_pixel(const Params& p, uint32_t id, bool ind, uint32_t n, float sr, float sg,
                                            float sb, uint32_t rng, float* hdr, uint32_t* dbg) {
  float fn = float(max(int(n), 1));
  float cr = sr / fn, cg = sg / fn, cb = sb / fn;
  if (!ind) clamp3(p, cr, cg, cb);
  hdr[size_t(id) * 3] = cr; hdr[size_t(id) * 3 + 1] = cg; hdr[size_t(id) * 3 + 2] = cb;
  if (dbg) { dbg[size_t(id) * 2] = rng; dbg[size_t(id) * 2 + 1] = n; }
}

// Wave 0: per pixel, the kind-1 primary direct light (pathtrace.metal:1097-1128)
// and the first samples.
// A pixel of row y queues its first ray in part y mod parts (the parts of a
// frame that run on their own streams).
__global__ void __launch_bounds__(256) k_wf_init(Scene s, Params p, uint64_t seed, GBufSoA gb, ResSoA rm,
                                                 WfState w, WfParts parts, float* __restrict__ hdr,
                                                 uint32_t* __restrict__ dbg, unsigned long long* ctr, uint32_t* err) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  const int part = id < npix ? int((id / uint32_t(p.width)) % uint32_t(parts.parts)) : 0;
  bool push = false, ext = false;
  uint32_t samples = 0;
  if (id < npix) {
    const int kind = __float_as_int(gb.pos_kind[id].w);
    if (kind == 0) {
      hdr[size_t(id) * 3] = 0.f; hdr[size_t(id) * 3 + 1] = 0.f; hdr[size_t(id) * 3 + 2] = 0.f;
      if (dbg) { dbg[size_t(id) * 2] = 0; dbg[size_t(id) * 2 + 1] = 0; }
    } else {
      const uint32_t x = id % uint32_t(p.width), y = id / uint32_t(p.width);
      Tracer pt(s, p, err);
      pt.rng.seed(seed ^ (uint64_t(id + 1) * 0xBF58476D1CE4E5B9ull) ^ 0x94D049BB133111EBull);
      PathRegs r{};
      uint32_t n = 0;
      float sr = 0, sg = 0, sb = 0;
      r.meta = kind == 1 ? kInd : 0u;
      bool done = false;
      if (kind == 1) {
        const Pixel1 g = pixel1(gb, id);
        const float4 EM = gb.emi[id];
        float pdr = 0, pdg = 0, pdb = 0, m_sumWu = 0;
        uint32_t m_M = 0;
        const float4 R3 = rm.sumwu_m_valid[id];
        const float4 R0 = rm.lp_alpha[id], R1 = rm.ln_phat[id], R2 = rm.le_sumws[id];
        if (__float_as_int(R3.z) != 0 && __float_as_int(R3.y) != 0 && R3.x > 0.0f && R2.w > 0.0f && R1.w > 0.0f) {
          m_sumWu = R3.x; m_M = uint32_t(__float_as_int(R3.y));
          float m_sumWs = R2.w;
          float ldx = R0.x - g.gpx, ldy = R0.y - g.gpy, ldz = R0.z - g.gpz;
          float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
          if (dist > 0.003f) {
            float inv = 1.0f / dist;
            float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
            float lcos = -(R1.x * dxn + (R1.y * dyn + R1.z * dzn));
            float scos = g.gnx * dxn + (g.gny * dyn + g.gnz * dzn);
            if (lcos > 1e-8f && scos > 1e-8f) {
              Bsdf e = Tracer::eval_bsdf(dxn, dyn, dzn, g.wox, g.woy, g.woz, g.gnx, g.gny, g.gnz, g.alpha2,
                                         g.metallic, g.spec_prob, g.ar, g.ag, g.ab);
              float Fr = R2.x * e.r * scos * R0.w, Fg = R2.y * e.g * scos * R0.w, Fb = R2.z * e.b * scos * R0.w;
              float ph = lum3(Fr, Fg, Fb);
              if (ph > 0.0f) {
                float pdf_ris = float(m_M) * ph / m_sumWu;
                float wnee = 1.0f;
                if (!p.nomis && e.pdf > 1e-20f) wnee = pdf_ris / (pdf_ris + e.pdf);
                float Wt = m_sumWs / (float(m_M) * ph);
                pdr = Fr * Wt * wnee; pdg = Fg * Wt * wnee; pdb = Fb * Wt * wnee;
              }
            }
          }
        }
        const float bsr = EM.x + pdr, bsg = EM.y + pdg, bsb = EM.z + pdb;
        w.base[id] = make_float4(bsr, bsg, bsb, m_sumWu);
        w.mM[id] = m_M;
        if (p.bounces <= 1 || p.spp <= 0) {
          float cr = bsr, cg = bsg, cb = bsb;
          clamp3(p, cr, cg, cb);
          hdr[size_t(id) * 3] = cr; hdr[size_t(id) * 3 + 1] = cg; hdr[size_t(id) * 3 + 2] = cb;
          if (dbg) { dbg[size_t(id) * 2] = pt.rng.state; dbg[size_t(id) * 2 + 1] = 0; }
          done = true;
        }
      }
      if (!done) {
        ext = start_samples(pt, p, gb, w, id, x, y, r, n, sr, sg, sb);
        if (ext) r.meta |= kExt;
        else write_pixel(p, id, kind == 1, n, sr, sg, sb, pt.rng.state, hdr, dbg);
        store(w, id, r, pt.rng.state, n, sr, sg, sb);
        push = ext;
        samples = n;
      }
    }
  }
  (void)push;
  for (int k = 0; k < parts.parts; ++k) append(parts.q[k].ext, parts.q[k].counts + kCntExt, ext && part == k, int(id));
  warp_add(ctr + 0, samples);
}

// Traversal of a queue of rays, one thread per ray (closest hit for extension
// rays, pathtrace.metal:119-163; any hit for shadow rays, :164).  T is the
// traversal (Trav: binary BVH, WTrav: wide BVH) and E / kDepth its stack.
// Finished extension rays are sorted into the shading queue of their surface
// type.  (Persistent grids whose idle lanes claim new rays, per leaf-to-leaf
// step or per node / triangle, measured 7-70 % slower on the 720p frame.)
template <bool kShadowRays, class T, class E, int kDepth>
__global__ void __launch_bounds__(128) k_wf_trace(Scene s, WfState w, WfQueues q, unsigned long long* ctr,
                                                  uint32_t* err) {
  const int n = q.counts[kShadowRays ? kCntShd : kCntExt];
  const int* queue = kShadowRays ? q.shd : q.ext;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nodes = 0, tests = 0, rays = 0;
  int cls = -1;
  int id = 0;
  if (i < n) {
    id = queue[i];
    const float4 o = kShadowRays ? w.so[id] : w.o[id];
    const float4 d = kShadowRays ? w.sd[id] : w.d[id];
    T t;
    E stack[kDepth];
    t.init(o.x, o.y, o.z, d.x, d.y, d.z, kShadowRays ? o.w : kFar);
    while (!t.template step<kShadowRays>(s, stack, err, nodes, tests)) {
    }
    rays = 1;
    if (kShadowRays) {
      w.occ[id] = t.r.tri >= 0 ? 1u : 0u;
    } else {
      w.hit[id] = make_float4(t.r.t, t.r.u, t.r.v, __int_as_float(t.r.tri));
      cls = 2;
      if (t.r.tri >= 0) cls = __ldg(&s.tris[t.r.tri].ior) > 1.0001f ? 1 : 0;
    }
  }
  if (!kShadowRays) {
    append(q.qa, q.counts + kCntA, cls == 0, id);
    append(q.qb, q.counts + kCntB, cls == 1, id);
    append(q.qc, q.counts + kCntC, cls == 2, id);
  }
  __syncwarp();
  warp_add(ctr + 1, rays);
  warp_add(ctr + 2, nodes);
  warp_add(ctr + 3, tests);
}

// Both traversals of a wave in one launch (binary BVH): thread i < n_ext
// takes extension ray i (closest hit), the next n_shd threads the shadow rays
// (any hit), with the any-hit rule as a per-thread flag so that the two kinds
// run one instruction stream.  Each launch's time is set by its slowest rays
// while most of the GPU idles; in one launch the shadow rays fill that time.
// ctr_ext / ctr_shd: the counters of each kind.  40 warps per SM (48
// registers, no spills; 36 at 55 by default): 51.5 against 53.1 ms of
// traversal a frame and 320.9 / 325.2 against 318.7 / 317.4 M path
// samples/s on the 720p frame; 44 or 48 warps (40 registers) spill and lose
// 6 %.  64-thread blocks (20 per SM) fit beside the other parts' launches
// more easily than 128-thread ones (~1 %).
__global__ void __launch_bounds__(64, 20) k_wf_trace2(Scene s, WfState w, WfQueues q, unsigned long long* ctr_ext,
                                                   unsigned long long* ctr_shd, uint32_t* err,
                                                   int* __restrict__ next_counts) {
  // the next wave's queue lengths start at zero: no launch reads or appends
  // to them until the shading launch after this one
  if (blockIdx.x == 0 && threadIdx.x < kCntSlots) next_counts[threadIdx.x] = 0;
  const int n_ext = q.counts[kCntExt], n_shd = q.counts[kCntShd];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nodes = 0, tests = 0;
  int cls = -1;
  int id = 0;
  const bool shadow = i >= n_ext;
  const bool live = i < n_ext + n_shd;
  if (live) {
    id = shadow ? q.shd[i - n_ext] : q.ext[i];
    const float4 o = shadow ? w.so[id] : w.o[id];
    const float4 d = shadow ? w.sd[id] : w.d[id];
    const TraceResult r = traverse_rt(s, o.x, o.y, o.z, d.x, d.y, d.z, shadow ? o.w : kFar, shadow, err, nodes,
                                      tests);
    if (shadow) {
      w.occ[id] = r.tri >= 0 ? 1u : 0u;
    } else {
      w.hit[id] = make_float4(r.t, r.u, r.v, __int_as_float(r.tri));
      cls = 2;
      if (r.tri >= 0) cls = __ldg(&s.tris[r.tri].ior) > 1.0001f ? 1 : 0;
    }
  }
  append(q.qa, q.counts + kCntA, cls == 0, id);
  append(q.qb, q.counts + kCntB, cls == 1, id);
  append(q.qc, q.counts + kCntC, cls == 2, id);
  __syncwarp();
  warp_add(ctr_ext + 1, live && !shadow ? 1u : 0u);
  warp_add(ctr_ext + 2, shadow ? 0u : nodes);
  warp_add(ctr_ext + 3, shadow ? 0u : tests);
  warp_add(ctr_shd + 1, live && shadow ? 1u : 0u);
  warp_add(ctr_shd + 2, shadow ? nodes : 0u);
  warp_add(ctr_shd + 3, shadow ? tests : 0u);
}

// One path of a shading queue: fold in its shadow ray, shade the vertex its
// extension ray found (VK 0 opaque, 1 dielectric) or end it (VK 2), finish and
// restart samples; ext / shd / fin tell which queues of the next wave take it.
// NEE: the NEE variant of vertex() (2 in opaque scenes, 1 otherwise).
template <int VK, int NEE>
__device__ __forceinline__ void shade_path(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w, int id,
                                           float* __restrict__ hdr, uint32_t* __restrict__ dbg, uint32_t* err,
                                           bool& ext, bool& shd, bool& fin, uint32_t& samples) {
  const uint32_t x = uint32_t(id) % uint32_t(p.width), y = uint32_t(id) / uint32_t(p.width);
  Tracer pt(s, p, err);
  PathRegs r;
  uint32_t n;
  float sr, sg, sb;
  load(w, uint32_t(id), r, pt.rng.state, n, sr, sg, sb);
  const uint32_t n0 = n;
  if (r.meta & kShadow) {
    r.meta &= ~kShadow;
    if (w.occ[id] == 0u) {
      const float4 c = w.c[id];
      r.ax += c.x; r.ay += c.y; r.az += c.z;
    }
  }
  bool ended;
  if (VK == 2) {
    ended = true;  // a miss ends the path; a finishing path has now folded in its last shadow ray
    r.meta &= ~(kExt | kFinish);
  } else {
    r.meta &= ~kExt;
    const float4 hh = w.hit[id];
    const TraceResult tr{hh.x, __float_as_int(hh.w), hh.y, hh.z};
    const Hit hit = pt.attributes(tr, r.ox, r.oy, r.oz, r.dx, r.dy, r.dz);
    bool has_shadow = false;
    float4 so, sd, c;
    const bool go = vertex<VK, NEE>(pt, p, r, hit, has_shadow, so, sd, c);
    if (has_shadow) {
      w.so[id] = so; w.sd[id] = sd; w.c[id] = c;
      r.meta |= kShadow;
      shd = true;
    }
    if (go) { r.meta |= kExt; ext = true; }
    ended = !go;
    if (ended && has_shadow) { r.meta |= kFinish; ended = false; fin = true; }  // wait for the shadow ray
  }
  if (ended) {
    finish_sample(p, w, uint32_t(id), r, n, sr, sg, sb);
    if (start_samples(pt, p, gb, w, uint32_t(id), x, y, r, n, sr, sg, sb)) {
      r.meta |= kExt;
      ext = true;
    } else {
      write_pixel(p, uint32_t(id), (r.meta & kInd) != 0, n, sr, sg, sb, pt.rng.state, hdr, dbg);
    }
  }
  samples += n - n0;
  store(w, uint32_t(id), r, pt.rng.state, n, sr, sg, sb);
}

// Shade the paths of one queue: VK 0 opaque hits, 1 dielectric hits, 2 paths
// without a vertex (the ray missed, or the path ended and waited for its last
// shadow ray).  Specialising on the vertex type keeps the warps' lanes on the
// same branch.
template <int VK, int NEE>
__global__ void __launch_bounds__(256) k_wf_shade(Scene s, Params p, GBufSoA gb, WfState w, WfQueues cq,
                                                  WfQueues nq, float* __restrict__ hdr, uint32_t* __restrict__ dbg,
                                                  unsigned long long* ctr, uint32_t* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int count = cq.counts[VK == 0 ? kCntA : (VK == 1 ? kCntB : kCntC)];
  const int* queue = VK == 0 ? cq.qa : (VK == 1 ? cq.qb : cq.qc);
  bool ext = false, shd = false, fin = false;
  int id = 0;
  uint32_t samples = 0;
  if (i < count) {
    id = queue[i];
    shade_path<VK, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
  }
  append(nq.ext, nq.counts + kCntExt, ext, id);
  append(nq.shd, nq.counts + kCntShd, shd, id);
  append(nq.qc, nq.counts + kCntC, fin, id);
  warp_add(ctr + 0, samples);
}

// The three shading queues of a wave in one launch: block b serves queue
// b % 3 (0 opaque hits, 1 dielectric hits, 2 no vertex), so a block's
// warps take one branch as in k_wf_shade while the three queues' work
// overlaps instead of running in three launches one after another.  The
// opaque variant runs 24 warps per SM (80 registers, ~250 bytes of spills,
// against 16 at 128): a launch alone runs 8 % slower, but beside the other
// parts' traversal launches its blocks fit where fewer did, and the frame is
// faster (on the 720p frame 318.1 / 319.7 against 314.3 / 312.6 M path
// samples/s with 256-thread blocks; 128-thread blocks, which fit into smaller
// gaps, another ~1 %).  The variant with in-place shadow traversal would
// spill 600 bytes at 80 registers and keeps 16 warps.
template <int NEE>
__global__ void __launch_bounds__(128, NEE == 2 ? 6 : 4) k_wf_shade3(Scene s, Params p, GBufSoA gb, WfState w, WfQueues cq,
                                                   WfQueues nq, float* __restrict__ hdr, uint32_t* __restrict__ dbg,
                                                   unsigned long long* ctr, uint32_t* err) {
  const int vk = int(blockIdx.x % 3u);
  const int i = int(blockIdx.x / 3u) * 128 + int(threadIdx.x);
  const int count = cq.counts[vk == 0 ? kCntA : (vk == 1 ? kCntB : kCntC)];
  const int* queue = vk == 0 ? cq.qa : (vk == 1 ? cq.qb : cq.qc);
  bool ext = false, shd = false, fin = false;
  int id = 0;
  uint32_t samples = 0;
  if (i < count) {
    id = queue[i];
    if (bad_index(id, (long long)p.width * p.height, err, kSiteQueue)) id = -1;
  }
  if (id >= 0 && i < count) {
    if (vk == 0) shade_path<0, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
    else if (vk == 1) shade_path<1, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
    else shade_path<2, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
  }
  append(nq.ext, nq.counts + kCntExt, ext, id);
  append(nq.shd, nq.counts + kCntShd, shd, id);
  append(nq.qc, nq.counts + kCntC, fin, id);
  warp_add(ctr + 0, samples);
}

// One vertex step of a tail pixel, one thread per pixel: its extension ray,
// its pending shadow ray and shade_path of the vertex type, in the waves'
// order.  Returns true while the pixel has work left (ext: its next step
// starts with an extension ray).  cnt: extension rays, nodes, tests; shadow
// rays, nodes, tests.
template <int NEE>
__device__ __forceinline__ bool tail_step(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w, int id,
                                          bool& ext, float* __restrict__ hdr, uint32_t* __restrict__ dbg,
                                          uint32_t* err, uint32_t& samples, uint32_t* cnt) {
  int vk = 2;
  if (ext) {
    const float4 o = w.o[id];
    const float4 d = w.d[id];
    const TraceResult r = traverse<false>(s, o.x, o.y, o.z, d.x, d.y, d.z, kFar, err, cnt[1], cnt[2]);
    ++cnt[0];
    w.hit[id] = make_float4(r.t, r.u, r.v, __int_as_float(r.tri));
    if (r.tri >= 0) vk = __ldg(&s.tris[r.tri].ior) > 1.0001f ? 1 : 0;
  }
  if (w.u[id].y & kShadow) {
    const float4 o = w.so[id];
    const float4 d = w.sd[id];
    const TraceResult r = traverse<true>(s, o.x, o.y, o.z, d.x, d.y, d.z, o.w, err, cnt[4], cnt[5]);
    ++cnt[3];
    w.occ[id] = r.tri >= 0 ? 1u : 0u;
  }
  bool shd = false, fin = false;
  ext = false;
  if (vk == 0) shade_path<0, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
  else if (vk == 1) shade_path<1, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
  else shade_path<2, NEE>(s, p, gb, w, id, hdr, dbg, err, ext, shd, fin, samples);
  return ext || fin;
}

// The end of the wavefront loop, once few paths remain: each thread takes an
// unfinished pixel and runs it to the end with the waves' steps, in their
// order (extension ray, pending shadow ray, shade_path of the vertex type), so
// the pixel comes out the same, without a launch and a queue round trip per
// vertex.  ctr: the stage counter of the tail's samples; ctr_ext / ctr_shd:
// its traversals'.  Eight 64-thread blocks per SM (128 registers, ~200
// bytes of spills): the tail is latency-bound and its path count is capped
// to one wave of resident blocks, so more resident blocks can take the paths
// over earlier (a capacity of 75.8 k instead of 56.8 k paths on 148 SMs; on
// the 720p frame a tenth of the first wave, ~60.6 k, now sets the hand-off,
// against 56.8 k before).  On the 720p frame:
// six 64-thread blocks (168 registers) 330.5 against 327.3 M path samples/s
// for three of 128 threads, and eight 334.1 against 331.2 M for six: a
// point each, inside the run-to-run spread.
template <int NEE>
__global__ void __launch_bounds__(64, 8) k_wf_tail(Scene s, Params p, GBufSoA gb, WfState w, WfQueues q,
                                                 float* __restrict__ hdr, uint32_t* __restrict__ dbg,
                                                 unsigned long long* ctr, unsigned long long* ctr_ext,
                                                 unsigned long long* ctr_shd, uint32_t* err) {
  const int n_ext = q.counts[kCntExt], n_c = q.counts[kCntC];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t samples = 0;
  uint32_t cnt[6] = {0, 0, 0, 0, 0, 0};
  bool active = i < n_ext + n_c;
  int id = 0;
  bool ext = false;
  if (active) {
    id = i < n_ext ? q.ext[i] : q.qc[i - n_ext];
    ext = i < n_ext;
    if (bad_index(id, (long long)p.width * p.height, err, kSiteTailQueue)) active = false;
  }
  // each pass of the loop advances the pixel by one vertex, and a pixel has
  // at most spp x (depth + 2) vertices left: past that, flag and stop
  const uint32_t max_steps = uint32_t(p.spp) * uint32_t(p.bounces + 2) * 4u + 64u;
  for (uint32_t step = 0; active; ++step) {
    if (step > max_steps) {
      atomicOr(err, kErrSteps);
      break;
    }
    active = tail_step<NEE>(s, p, gb, w, id, ext, hdr, dbg, err, samples, cnt);
  }
  __syncwarp();
  warp_add(ctr + 0, samples);
  warp_add(ctr_ext + 1, cnt[0]);
  warp_add(ctr_ext + 2, cnt[1]);
  warp_add(ctr_ext + 3, cnt[2]);
  warp_add(ctr_shd + 1, cnt[3]);
  warp_add(ctr_shd + 2, cnt[4]);
  warp_add(ctr_shd + 3, cnt[5]);
}

}  // namespace

cudaError_t launch_wavefront_init(const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb, const ResSoA& rm,
                                  const WfState& w, const WfParts& parts, float* hdr, uint32_t* dbg,
                                  unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  const uint32_t npix = uint32_t(p.width) * uint32_t(p.height);
  k_wf_init<<<(npix + 255) / 256, 256, 0, st>>>(s, p, seed, gb, rm, w, parts, hdr, dbg, ctr, err);
  return cudaGetLastError();
}

template <bool kShadowRays, class T, class E, int kDepth>
static cudaError_t trace_grid(const Scene& s, const WfState& w, const WfQueues& q, int bound, unsigned long long* ctr,
                              uint32_t* err, cudaStream_t st) {
  k_wf_trace<kShadowRays, T, E, kDepth><<<unsigned((bound + 127) / 128), 128, 0, st>>>(s, w, q, ctr, err);
  return cudaGetLastError();
}

cudaError_t launch_wavefront_trace(const Scene& s, const WfState& w, const WfQueues& q, int bound, bool shadow,
                                   unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  if (bound <= 0) return cudaSuccess;
  if (s.wnodes) {
    if (shadow) return trace_grid<true, WTrav, uint2, kWideStack>(s, w, q, bound, ctr, err, st);
    return trace_grid<false, WTrav, uint2, kWideStack>(s, w, q, bound, ctr, err, st);
  }
  if (shadow) return trace_grid<true, Trav, int, kStack>(s, w, q, bound, ctr, err, st);
  return trace_grid<false, Trav, int, kStack>(s, w, q, bound, ctr, err, st);
}

cudaError_t launch_wavefront_trace2(const Scene& s, const WfState& w, const WfQueues& q, int bound,
                                    unsigned long long* ctr_ext, unsigned long long* ctr_shd, uint32_t* err,
                                    int* next_counts, cudaStream_t st) {
  if (bound <= 0) return cudaMemsetAsync(next_counts, 0, kCntSlots * sizeof(int), st);
  k_wf_trace2<<<unsigned((2 * bound + 63) / 64), 64, 0, st>>>(s, w, q, ctr_ext, ctr_shd, err, next_counts);
  return cudaGetLastError();
}

cudaError_t launch_wavefront_shade3(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                    const WfQueues& cq, int bound, const WfQueues& nq, float* hdr, uint32_t* dbg,
                                    unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  if (bound <= 0) return cudaSuccess;
  const unsigned g = unsigned(3 * ((bound + 127) / 128));
  if (p.opaque) k_wf_shade3<2><<<g, 128, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
  else k_wf_shade3<1><<<g, 128, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
  return cudaGetLastError();
}

int wavefront_tail_capacity(bool opaque) {
  static int cap[2] = {0, 0};
  int& c = cap[opaque ? 1 : 0];
  if (c == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, opaque ? k_wf_tail<2> : k_wf_tail<1>, 64, 0) !=
            cudaSuccess)
      return 0;
    c = sms * per_sm * 64;
  }
  return c;
}

cudaError_t launch_wavefront_tail(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                  const WfQueues& q, int bound, float* hdr, uint32_t* dbg, unsigned long long* ctr,
                                  unsigned long long* ctr_ext, unsigned long long* ctr_shd, uint32_t* err,
                                  cudaStream_t st) {
  if (bound <= 0) return cudaSuccess;
  const unsigned g = unsigned((bound + 63) / 64);
  if (p.opaque) k_wf_tail<2><<<g, 64, 0, st>>>(s, p, gb, w, q, hdr, dbg, ctr, ctr_ext, ctr_shd, err);
  else k_wf_tail<1><<<g, 64, 0, st>>>(s, p, gb, w, q, hdr, dbg, ctr, ctr_ext, ctr_shd, err);
  return cudaGetLastError();
}

cudaError_t launch_wavefront_shade(int vk, const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                   const WfQueues& cq, int bound, const WfQueues& nq, float* hdr, uint32_t* dbg,
                                   unsigned long long* ctr, uint32_t* err, cudaStream_t st) {
  if (bound <= 0) return cudaSuccess;
  const unsigned g = unsigned((bound + 255) / 256);
  if (p.opaque) {
    if (vk == 0) k_wf_shade<0, 2><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
    else if (vk == 1) k_wf_shade<1, 2><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
    else k_wf_shade<2, 2><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
  } else {
    if (vk == 0) k_wf_shade<0, 1><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
    else if (vk == 1) k_wf_shade<1, 1><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
    else k_wf_shade<2, 1><<<g, 256, 0, st>>>(s, p, gb, w, cq, nq, hdr, dbg, ctr, err);
  }
  return cudaGetLastError();
}

}  // namespace rmd

// rm_device.cuh - device-side scene layout, traversal and shading for sm_100a.
//
// One path tracer, written for the GPU, that reproduces the reference Metal
// shader's arithmetic (reference src/engine/pathtrace.metal) operation for
// operation: this file is compiled with -fmad=false and IEEE div/sqrt so that,
// on identical RNG streams, radiance matches the CPU oracle bit for bit.
//
// Scene layout in HBM (built by rm_bvh.cu):
//  * tgeo: 3 x float4 per triangle, in BVH leaf order: (v0, original index),
//    (v1 - v0, 0), (v2 - v0, 0).  One 48-byte, 16-byte-aligned record is all a
//    Moller-Trumbore test reads (the reference fetches a 176-byte AoS record).
//  * nodes: binary BVH in the child-pair layout of Aila & Laine ("Understanding
//    the Efficiency of Ray Traversal on GPUs", HPG 2009): each internal node
//    holds both children's boxes, 64 bytes = four 128-bit loads; a ray tests
//    both children at once and descends into the nearer one first with a
//    per-thread stack.
//  * tris: the caller's packed 176-byte triangles, read only for the surface
//    attributes of a confirmed hit and for light sampling.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rm_detmath.h"
#include "rmcuda.h"

namespace rmd {

constexpr float kFar = 1e30f;
constexpr float kPi = 3.141592653589793f;
constexpr float kBoxSlack = 1.0000152587890625f;  // 1 + 2^-16, see traverse()
constexpr int kStack = 64;                         // max BVH depth accepted at build time
constexpr int kMaxLeaf = 255;                      // 8-bit leaf count in a stack entry
constexpr int kMaxLink = 1 << 24;                  // 24-bit node / triangle link
constexpr int kMaxAlphaCrossings = 1024;
constexpr uint64_t kSpatialSeedXor = 0x1B54A35A6F31B458ull;  // low 64 bits of pathtrace.metal:937

// device error word bits
constexpr uint32_t kErrStack = 1u;
constexpr uint32_t kErrAlpha = 2u;
constexpr uint32_t kErrBounds = 4u;
constexpr uint32_t kErrSteps = 8u;  // a loop ran past its bound on the steps a pixel can take

// The checked build (RMCUDA_CHECKED defined; raymotion_b200/build.py
// `checked`, librmcuda_checked.so): every index read from a device structure
// (a BVH node or leaf range, a hit's triangle, a light, a texel, a queue
// entry) is compared with its array before the access; a bad one sets
// kErrBounds in the error word and the access is skipped (a node as an empty
// subtree, a leaf or hit as a miss, a light as the first light, a texel as
// white, a queue entry as no work).  The call then fails with RM_ERR_DEVICE
// instead of reading out of bounds; valid inputs give the same results as
// the unchecked build.
#ifdef RMCUDA_CHECKED
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif

// Which check fired is recorded as bit 8 + site of the error word.
enum CheckSite : uint32_t {
  kSiteNode = 0, kSiteLeaf, kSiteWideLeaf, kSiteHit, kSiteTexel, kSiteLight, kSiteQueue, kSiteTailQueue, kSiteVertex
};
__device__ __forceinline__ bool bad_index(long long i, long long n, uint32_t* err, uint32_t site) {
  if (!kChecked || (i >= 0 && i < n)) return false;
  if (err) atomicOr(err, kErrBounds | (1u << (8u + site)));
  return true;
}

struct Scene {
  const rm_triangle* __restrict__ tris;
  const float4* __restrict__ tgeo;
  const float4* __restrict__ nodes;
  int n_nodes;  // internal child-pair records; 0 = empty scene
  const int32_t* __restrict__ lights;
  const float* __restrict__ cdf;
  int n_lights;
  float light_total;
  const rm_vec3* __restrict__ texels;
  // Light sampling accelerators (built at upload, rm_bvh.cu k_light_prep):
  // lrec: 4 x float4 per light, in light-list order: (v0, er), (v1, eg),
  // (v2, eb), (nn, alpha) of triangle lights[i];  guide: guide_n + 1 entries,
  // guide[g] = first light index whose CDF value is >= g * guide_step.
  const float4* __restrict__ lrec;
  const int32_t* __restrict__ guide;
  int guide_n;
  float guide_inv;  // guide_n / light_total
  // 8-wide compressed BVH (rm_wide.cu), used instead of `nodes` when set:
  // 5 x float4 per node, and the triangle records (as tgeo) in its leaf order
  const float4* __restrict__ wnodes = nullptr;
  const float4* __restrict__ wtgeo = nullptr;
  int n_tris = 0;          // triangles (and triangle records)
  long long n_texels = 0;  // texels
};

// One emissive triangle as light sampling reads it (the fields of
// rm_triangle that NEE uses, with the same names).
struct LightRec {
  rm_vec3 v0, v1, v2, nn;
  float er, eg, eb, alpha;
};

__device__ __forceinline__ LightRec load_light(const Scene& s, int i) {
  const float4* r = s.lrec + size_t(i) * 4;
  const float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3);
  LightRec t;
  t.v0 = rm_vec3{a.x, a.y, a.z}; t.er = a.w;
  t.v1 = rm_vec3{b.x, b.y, b.z}; t.eg = b.w;
  t.v2 = rm_vec3{c.x, c.y, c.z}; t.eb = c.w;
  t.nn = rm_vec3{d.x, d.y, d.z}; t.alpha = d.w;
  return t;
}

// metal_types.h:21-30 plus this build's switches.
struct Params {
  rm_camera camera;
  int width, height, spp, bounces, nodes, lights, adapt_min, adapt_step, nomis, opaque;
  float light_total, resolution, clamp_value, adapt_rel, adapt_abs;
  int restir_candidates, restir_spatial, restir_mcap;
  float restir_radius;
  rm_camera prevCamera;
  int hasHistory;
  int rr;
};

// SoA G-buffer: pos|kind, normal|rough, albedo|metallic, wo|ior, emission.
struct GBufSoA {
  float4* pos_kind;
  float4* nor_rough;
  float4* alb_met;
  float4* wo_ior;
  float4* emi;
};
// SoA reservoir: lightPos|alpha, lightNormal|p_hat, emission|sumWs, (sumWu, M, valid,
// the selected light index as int bits; 0 for no sample).
struct ResSoA {
  float4* lp_alpha;
  float4* ln_phat;
  float4* le_sumws;
  float4* sumwu_m_valid;
};

struct Rng {
  uint32_t state;
  __device__ __forceinline__ void seed(uint64_t s) {
    uint64_t z = s + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    state = uint32_t(z ^ (z >> 31));
  }
  __device__ __forceinline__ float uniform01() {
    state = state * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return float(((word >> 22u) ^ word) >> 8u) * 0x1p-24f;
  }
};

__device__ __forceinline__ uint64_t seed_pixel(uint64_t seed, uint32_t x, uint32_t y) {
  return seed ^ (uint64_t(y + 1) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(x + 1) * 0xBF58476D1CE4E5B9ull);
}

__device__ __forceinline__ float lum3(float r, float g, float b) {
  return 0.2126f * r + 0.7152f * g + 0.0722f * b;
}

struct Hit {
  float t;
  int tri;
  float u, v;
  float px, py, pz;
  float nix, niy, niz;
  float ar, ag, ab, er, eg, eb, ior, rough;
  int shader;
  float ngx, ngy, ngz;
  float txr, txg, txb;  // texel colour the albedo was multiplied by (1 untextured)
};

struct Bsdf { float r, g, b, pdf; };

// ---------------------------------------------------------------- traversal
//
// Closest hit = smallest t, ties to the smaller original triangle index; a
// candidate is accepted under the reference's Moller-Trumbore rules
// (pathtrace.metal:150-158).  A box is culled only when its entry exceeds
// its exit by more than a relative 2^-16, so that no BVH culls a triangle that
// the Moller-Trumbore test would accept: the hit is independent of the BVH.
struct TraceResult { float t; int tri; float u, v; };

// Moller-Trumbore against one triangle record (pathtrace.metal:150-158) with
// the (t, triangle index) order of the header; true when it became the hit.
__device__ __forceinline__ bool test_triangle(const float4* __restrict__ g, float ox, float oy, float oz, float dx,
                                              float dy, float dz, TraceResult& r) {
  const float4 q0 = __ldg(g + 0);
  const float4 q1 = __ldg(g + 1);
  const float4 q2 = __ldg(g + 2);
  const int j = __float_as_int(q0.w);
  float px = dy * q2.z - dz * q2.y;
  float py = dz * q2.x - dx * q2.z;
  float pz = dx * q2.y - dy * q2.x;
  float det = q1.x * px + q1.y * py + q1.z * pz;
  if (fabsf(det) < 1e-12f) return false;
  float tx = ox - q0.x, ty = oy - q0.y, tz = oz - q0.z;
  float u = (tx * px + ty * py + tz * pz) / det;
  if (u < 0.0f || u > 1.0f) return false;
  float qx = ty * q1.z - tz * q1.y;
  float qy = tz * q1.x - tx * q1.z;
  float qz = tx * q1.y - ty * q1.x;
  float v = (dx * qx + dy * qy + dz * qz) / det;
  if (v < 0.0f || u + v > 1.0f) return false;
  float dd = (q2.x * qx + q2.y * qy + q2.z * qz) / det;
  if (dd > 1e-8f && (dd < r.t || (dd == r.t && r.tri >= 0 && j < r.tri))) {
    r.t = dd; r.tri = j; r.u = u; r.v = v;
    return true;
  }
  return false;
}

// Resumable traversal of one ray: init() then step() until it returns true.
// A step visits child-pair records until a leaf is pending (descending into
// the nearer child, pushing the farther one as an 8-bit count / 24-bit link
// word), tests that leaf, and pops the next subtree.  The persistent kernels
// interleave steps of different rays on one thread; traverse() below runs
// one ray to the end.
//
// Box test.  The base test is the reference's slab form: per axis the bounds
// A = (L - o) * i with two roundings, entry = max(0, max A_near), exit =
// min(t, min A_far), the box culled when entry > exit (1 + 2^-16).  The
// traversal evaluates each bound as one fma, B = fma(L, i, c), with the
// per-ray addend c = -(o i) lowered by m = |o i| 2^-21 for the bound that is
// near for the sign of i and raised by m for the far one.  m exceeds the
// rounding of o i and of c, so as real numbers L i + c_near <= (L - o) i <=
// L i + c_far, and the rounded B_near <= RN((L - o) i) <= B_far.  Each RN
// differs from A by at most 2^-23 relative, so B_entry <= A_entry (1 + 2^-22)
// and B_exit >= A_exit (1 - 2^-22) for A_exit >= 0 (a box with A_exit < 0 is
// culled by the base test), and with the slack 1 + 2^-15 every box the base
// test accepts is accepted: the hits stay those of the base test.
constexpr float kFmaBoxSlack = 1.000030517578125f;  // 1 + 2^-15

// three-input min / max of sm_100 (PTX ISA 8.8); like fminf / fmaxf, a NaN
// operand is ignored
__device__ __forceinline__ float fmin3(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// The addends of one axis: lo is the near bound for i >= 0, hi for i < 0.
// If o i overflows (|o| near FLT_MAX / |i|) the axis culls nothing.
__device__ __forceinline__ void slab_addends(float o, float i, float& c_lo, float& c_hi) {
  const float oi = o * i;
  const float m = fabsf(oi) * 0x1p-21f;
  const float lowered = -oi - m, raised = -oi + m;
  const bool finite = fabsf(oi) <= 3.4028234663852886e38f;
  const float inf = __int_as_float(0x7f800000);
  c_lo = finite ? (i >= 0.0f ? lowered : raised) : (i >= 0.0f ? -inf : inf);
  c_hi = finite ? (i >= 0.0f ? raised : lowered) : (i >= 0.0f ? inf : -inf);
}

struct Trav {
  float ox, oy, oz, dx, dy, dz, ix, iy, iz;
  float cxl, cxh, cyl, cyh, czl, czh;  // slab addends of the lo / hi bound per axis
  TraceResult r;
  int sp, node, leaf_first, leaf_count;

  __device__ __forceinline__ void init(float ox_, float oy_, float oz_, float dx_, float dy_, float dz_, float tmax) {
    ox = ox_; oy = oy_; oz = oz_; dx = dx_; dy = dy_; dz = dz_;
    ix = 1.0f / (dx == 0.0f ? 1e-30f : dx);
    iy = 1.0f / (dy == 0.0f ? 1e-30f : dy);
    iz = 1.0f / (dz == 0.0f ? 1e-30f : dz);
    slab_addends(ox, ix, cxl, cxh);
    slab_addends(oy, iy, cyl, cyh);
    slab_addends(oz, iz, czl, czh);
    r = TraceResult{tmax, -1, 0.f, 0.f};
    sp = 0;
    node = 0;
    leaf_first = 0;
    leaf_count = 0;
  }

  // Pop the next pending subtree (8-bit leaf count / 24-bit link word); true
  // when none is left.
  __device__ __forceinline__ bool pop(const int* stack) {
    if (sp == 0) return true;
    const int e = stack[--sp];
    const int cnt = int(uint32_t(e) >> 24), link = e & 0xFFFFFF;
    if (cnt > 0) { leaf_first = link; leaf_count = cnt; node = -1; }
    else node = link;
    return false;
  }

  // Box-test the two children of record `node` and move on: into the nearer
  // hit child (pushing the farther one), else to the next pending subtree.
  // True when nothing is left (or the stack overflowed, flagged in err).
  __device__ __forceinline__ bool visit(const Scene& s, int* stack, uint32_t* err, uint32_t& n_nodes) {
    if (bad_index(node, s.n_nodes, err, kSiteNode)) return pop(stack);
    ++n_nodes;
    const float4* n = s.nodes + size_t(node) * 4;
    const float4 a = __ldg(n + 0);
    const float4 b = __ldg(n + 1);
    const float4 c = __ldg(n + 2);
    const int4 d = __ldg(reinterpret_cast<const int4*>(n + 3));
    // child 0
    const float l0x = __fmaf_rn(a.x, ix, cxl), h0x = __fmaf_rn(a.y, ix, cxh);
    const float l0y = __fmaf_rn(a.z, iy, cyl), h0y = __fmaf_rn(a.w, iy, cyh);
    const float l0z = __fmaf_rn(c.x, iz, czl), h0z = __fmaf_rn(c.y, iz, czh);
    const float n0 = fmax3(fminf(l0x, h0x), fminf(l0y, h0y), fmaxf(fminf(l0z, h0z), 0.0f));
    const float f0 = fmin3(fmaxf(l0x, h0x), fmaxf(l0y, h0y), fminf(fmaxf(l0z, h0z), r.t));
    // child 1
    const float l1x = __fmaf_rn(b.x, ix, cxl), h1x = __fmaf_rn(b.y, ix, cxh);
    const float l1y = __fmaf_rn(b.z, iy, cyl), h1y = __fmaf_rn(b.w, iy, cyh);
    const float l1z = __fmaf_rn(c.z, iz, czl), h1z = __fmaf_rn(c.w, iz, czh);
    const float n1 = fmax3(fminf(l1x, h1x), fminf(l1y, h1y), fmaxf(fminf(l1z, h1z), 0.0f));
    const float f1 = fmin3(fmaxf(l1x, h1x), fmaxf(l1y, h1y), fminf(fmaxf(l1z, h1z), r.t));
    bool hit0 = d.z >= 0 && !(n0 > f0 * kFmaBoxSlack);
    bool hit1 = d.w >= 0 && !(n1 > f1 * kFmaBoxSlack);
    // a child record: link d.x/d.y, count d.z/d.w (>0 leaf, 0 internal, <0 empty)
    if (hit0 && hit1) {
      int first = d.x, firstc = d.z, second = d.y, secondc = d.w;
      if (n1 < n0) { first = d.y; firstc = d.w; second = d.x; secondc = d.z; }
      if (sp >= kStack) { atomicOr(err, kErrStack); return true; }
      stack[sp++] = int((uint32_t(secondc) << 24) | uint32_t(second));  // far child: 8-bit count, 24-bit link
      if (firstc > 0) { leaf_first = first; leaf_count = firstc; node = -1; }
      else node = first;
    } else if (hit0 || hit1) {
      int link = hit0 ? d.x : d.y, cnt = hit0 ? d.z : d.w;
      if (cnt > 0) { leaf_first = link; leaf_count = cnt; node = -1; }
      else node = link;
    } else {
      return pop(stack);
    }
    return false;
  }

  // Returns true when the ray is finished (r holds the result).  `stack` is
  // the caller's kStack-entry array (kept out of the struct so that the scalar
  // state stays in registers).
  template <bool kAnyHit>
  __device__ __forceinline__ bool step(const Scene& s, int* stack, uint32_t* err, uint32_t& n_nodes,
                                       uint32_t& n_tests) {
    return step_rt(s, stack, err, n_nodes, n_tests, kAnyHit);
  }

  // step() with the any-hit rule as a run-time flag: lanes of one warp that
  // trace closest-hit and any-hit rays then run the same instructions.
  __device__ __forceinline__ bool step_rt(const Scene& s, int* stack, uint32_t* err, uint32_t& n_nodes,
                                          uint32_t& n_tests, bool any_hit) {
    if (s.n_nodes == 0) return true;
    while (node >= 0 && leaf_count == 0)
      if (visit(s, stack, err, n_nodes)) return true;
    // leaf: Moller-Trumbore, pathtrace.metal:150-158
    if (kChecked && (bad_index(leaf_first, s.n_tris, err, kSiteLeaf) ||
                     bad_index(leaf_first + leaf_count - 1, s.n_tris, err, kSiteLeaf)))
      leaf_count = 0;
    n_tests += uint32_t(leaf_count);
    for (int k = 0; k < leaf_count; ++k)
      if (test_triangle(s.tgeo + size_t(leaf_first + k) * 3, ox, oy, oz, dx, dy, dz, r) && any_hit) return true;
    leaf_count = 0;
    return pop(stack);
  }
};

// Traversal of the 8-wide compressed BVH built by rm_wide.cu.  A node is 5 x
// float4: origin p (3 floats), the three scale exponents and the mask of
// internal children (4 bytes), the index of its first internal child node and
// of its first triangle record, one byte per child slot (0xFF empty, 0xFE
// internal, else a leaf: bits 5-6 triangle count - 1, bits 0-4 offset from the
// node's first triangle), and each child's box as 8-bit lo / hi per axis on the
// grid p + q 2^e.  Boxes are dequantized with the same float expression the
// builder checked to contain the true boxes, and culled with the slack rule of
// the binary traversal, so the hits are the same as with any other BVH.
// Child slots follow the octant of the child's centre in its parent: visiting
// keys slot ^ octant(ray) in increasing order is near to far.  The stack holds
// groups (first child node, remaining keys | internal mask << 8).
constexpr int kWideStack = 32;

// p + float(q) * scale for an 8-bit q, computed as one fused multiply-add: the
// product of an integer below 256 and a power of two is exact, so the single
// rounding of the fma equals the rounding of the separate add.  float(q) is
// formed without a conversion instruction: 0x4B000000 | q is the float 2^23 + q.
__device__ __forceinline__ float dequant(float p, uint32_t q, float scale) {
  return __fmaf_rn(__uint_as_float(0x4B000000u | q) - 8388608.0f, scale, p);
}

// Byte b of `word` as a float (exact): 0x4B000000 | q is the float 2^23 + q.
template <int b>
__device__ __forceinline__ float byte_float(uint32_t word) {
  return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u | b)) - 8388608.0f;
}

// Resumable traversal of the wide BVH: init() then step() until it returns
// true.  A step visits one node (boxes of its 8 child slots) and tests the
// triangles of the leaves it hit, popping a group first when the current one
// is exhausted.
struct WTrav {
  float ox, oy, oz, dx, dy, dz, ix, iy, iz;
  TraceResult r;
  uint32_t oct, gbase, gbits;
  int sp;

  __device__ __forceinline__ void init(float ox_, float oy_, float oz_, float dx_, float dy_, float dz_, float tmax) {
    ox = ox_; oy = oy_; oz = oz_; dx = dx_; dy = dy_; dz = dz_;
    ix = 1.0f / (dx == 0.0f ? 1e-30f : dx);
    iy = 1.0f / (dy == 0.0f ? 1e-30f : dy);
    iz = 1.0f / (dz == 0.0f ? 1e-30f : dz);
    r = TraceResult{tmax, -1, 0.f, 0.f};
    oct = (dx < 0.0f ? 1u : 0u) | (dy < 0.0f ? 2u : 0u) | (dz < 0.0f ? 4u : 0u);
    gbase = 0;
    gbits = (1u << oct) | (1u << 8);  // the root: slot 0 of a virtual parent
    sp = 0;
  }

  template <bool kAnyHit>
  __device__ __forceinline__ bool step(const Scene& s, uint2* stack, uint32_t* err, uint32_t& n_nodes,
                                       uint32_t& n_tests) {
    if (s.n_nodes == 0) return true;
    while (!(gbits & 0xFFu)) {
      if (sp == 0) return true;
      const uint2 e = stack[--sp];
      gbase = e.x;
      gbits = e.y;
    }
    const uint32_t k = __ffs(gbits & 0xFFu) - 1;
    gbits &= ~(1u << k);
    const uint32_t slot = k ^ oct;
    const uint32_t node = gbase + __popc((gbits >> 8) & ((1u << slot) - 1u));
    ++n_nodes;
    const float4* nd = s.wnodes + size_t(node) * 5;
    const float4 n0 = __ldg(nd + 0);
    const uint4 n1 = __ldg(reinterpret_cast<const uint4*>(nd + 1));
    const uint4 n2 = __ldg(reinterpret_cast<const uint4*>(nd + 2));
    const uint4 n3 = __ldg(reinterpret_cast<const uint4*>(nd + 3));
    const uint4 n4 = __ldg(reinterpret_cast<const uint4*>(nd + 4));
    const uint32_t ew = __float_as_uint(n0.w);
    const float sx = __uint_as_float((ew & 0xFFu) << 23);
    const float sy = __uint_as_float(((ew >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((ew >> 16) & 0xFFu) << 23);
    // n1: child_base, tri_base, meta 0-3, meta 4-7; n2: qlo_x (8), qlo_y (8);
    // n3: qlo_z (8), qhi_x (8); n4: qhi_y (8), qhi_z (8).
    // A child's slab on axis a is t = q s_a i_a + (p_a - o_a) i_a, one fma per
    // bound from the per-node base (p_a - o_a) i_a and the exact product
    // s_a i_a (s_a is a power of two).  Its rounding differs from the base
    // test's (L - o) i (Trav), so the near bound's base is lowered and the far
    // bound's raised by m_a = |i_a| 2^-20 (|p_a - o_a| + 256 s_a + |p_a|),
    // rounded outward: m_a exceeds the sum of both forms' rounding errors and
    // of the decoded bound's half ulp, so every box the base test accepts
    // is accepted here and the hits stay the base test's.  Which
    // stored bound is near follows the sign of i_a (the decoded lo <= hi).
    const float six = sx * ix, siy = sy * iy, siz = sz * iz;
    const float bx = (n0.x - ox) * ix, by = (n0.y - oy) * iy, bz = (n0.z - oz) * iz;
    const float mx = fabsf(ix) * 0x1p-20f * (fabsf(n0.x - ox) + 256.0f * sx + fabsf(n0.x));
    const float my = fabsf(iy) * 0x1p-20f * (fabsf(n0.y - oy) + 256.0f * sy + fabsf(n0.y));
    const float mz = fabsf(iz) * 0x1p-20f * (fabsf(n0.z - oz) + 256.0f * sz + fabsf(n0.z));
    const float bnx = __fsub_rd(bx, mx), bfx = __fadd_ru(bx, mx);
    const float bny = __fsub_rd(by, my), bfy = __fadd_ru(by, my);
    const float bnz = __fsub_rd(bz, mz), bfz = __fadd_ru(bz, mz);
    const bool sxp = ix >= 0.0f, syp = iy >= 0.0f, szp = iz >= 0.0f;
    const uint32_t nx0 = sxp ? n2.x : n3.z, nx1 = sxp ? n2.y : n3.w, fx0 = sxp ? n3.z : n2.x, fx1 = sxp ? n3.w : n2.y;
    const uint32_t ny0 = syp ? n2.z : n4.x, ny1 = syp ? n2.w : n4.y, fy0 = syp ? n4.x : n2.z, fy1 = syp ? n4.y : n2.w;
    const uint32_t nz0 = szp ? n3.x : n4.z, nz1 = szp ? n3.y : n4.w, fz0 = szp ? n4.z : n3.x, fz1 = szp ? n4.w : n3.y;
    uint32_t ikeys = 0, tmask = 0;
#define RM_WIDE_SLOT(J, H, B)                                                                              \
  {                                                                                                        \
    const uint32_t meta = (n1.H >> (8 * B)) & 0xFFu;                                                       \
    if (meta != 0xFFu) {                                                                                   \
      const float tnx = __fmaf_rn(byte_float<B>(J < 4 ? nx0 : nx1), six, bnx);                             \
      const float tny = __fmaf_rn(byte_float<B>(J < 4 ? ny0 : ny1), siy, bny);                             \
      const float tnz = __fmaf_rn(byte_float<B>(J < 4 ? nz0 : nz1), siz, bnz);                             \
      const float tfx = __fmaf_rn(byte_float<B>(J < 4 ? fx0 : fx1), six, bfx);                             \
      const float tfy = __fmaf_rn(byte_float<B>(J < 4 ? fy0 : fy1), siy, bfy);                             \
      const float tfz = __fmaf_rn(byte_float<B>(J < 4 ? fz0 : fz1), siz, bfz);                             \
      const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));                                           \
      const float tf = fminf(fminf(tfx, tfy), fminf(tfz, r.t));                                            \
      if (!(tn > tf * kBoxSlack)) {                                                                        \
        if (meta == 0xFEu) ikeys |= 1u << (uint32_t(J) ^ oct);                                             \
        else tmask |= ((1u << ((meta >> 5) + 1u)) - 1u) << (meta & 31u);                                   \
      }                                                                                                    \
    }                                                                                                      \
  }
    RM_WIDE_SLOT(0, z, 0) RM_WIDE_SLOT(1, z, 1) RM_WIDE_SLOT(2, z, 2) RM_WIDE_SLOT(3, z, 3)
    RM_WIDE_SLOT(4, w, 0) RM_WIDE_SLOT(5, w, 1) RM_WIDE_SLOT(6, w, 2) RM_WIDE_SLOT(7, w, 3)
#undef RM_WIDE_SLOT
    if (ikeys) {
      // descend; the node's remaining siblings wait on the stack
      if (gbits & 0xFFu) {
        if (sp >= kWideStack) { atomicOr(err, kErrStack); return true; }
        stack[sp++] = make_uint2(gbase, gbits);
      }
      gbase = n1.x;
      gbits = ikeys | ((ew >> 24) << 8);
    }
    if (tmask) {
      n_tests += uint32_t(__popc(tmask));
      const float4* tg = s.wtgeo + size_t(n1.y) * 3;
      do {
        const uint32_t i = __ffs(tmask) - 1;
        tmask &= tmask - 1u;
        if (bad_index((long long)n1.y + i, s.n_tris, err, kSiteWideLeaf)) continue;
        if (test_triangle(tg + size_t(i) * 3, ox, oy, oz, dx, dy, dz, r) && kAnyHit) return true;
      } while (tmask);
    }
    return false;
  }
};

// One ray through the binary BVH (always built; the megakernels trace here,
// so that the wide traversal's registers never count against them).
template <bool kAnyHit>
__device__ __forceinline__ TraceResult traverse(const Scene& s, float ox, float oy, float oz, float dx, float dy,
                                                float dz, float tmax, uint32_t* err, uint32_t& n_nodes,
                                                uint32_t& n_tests) {
  Trav t;
  int stack[kStack];
  t.init(ox, oy, oz, dx, dy, dz, tmax);
  while (!t.step<kAnyHit>(s, stack, err, n_nodes, n_tests)) {
  }
  return t.r;
}

// traverse() with the any-hit rule as a run-time flag (one instruction stream
// for the closest-hit and any-hit rays of a warp).
__device__ __forceinline__ TraceResult traverse_rt(const Scene& s, float ox, float oy, float oz, float dx, float dy,
                                                   float dz, float tmax, bool any_hit, uint32_t* err,
                                                   uint32_t& n_nodes, uint32_t& n_tests) {
  Trav t;
  int stack[kStack];
  t.init(ox, oy, oz, dx, dy, dz, tmax);
  while (!t.step_rt(s, stack, err, n_nodes, n_tests, any_hit)) {
  }
  return t.r;
}

// One ray through the 8-wide BVH when the scene has one, else the binary BVH
// (the ray-query entry point; the wavefront trace kernels pick WTrav or Trav
// per launch instead).  Both give the same hits.
template <bool kAnyHit>
__device__ __forceinline__ TraceResult traverse_any(const Scene& s, float ox, float oy, float oz, float dx, float dy,
                                                    float dz, float tmax, uint32_t* err, uint32_t& n_nodes,
                                                    uint32_t& n_tests) {
  if (s.wnodes) {
    WTrav t;
    uint2 stack[kWideStack];
    t.init(ox, oy, oz, dx, dy, dz, tmax);
    while (!t.step<kAnyHit>(s, stack, err, n_nodes, n_tests)) {
    }
    return t.r;
  }
  return traverse<kAnyHit>(s, ox, oy, oz, dx, dy, dz, tmax, err, n_nodes, n_tests);
}

// ---------------------------------------------------------------- tracer
struct Tracer {
  const Scene& s;
  const Params& p;
  Rng rng;
  uint32_t rays, nodes, tests;
  uint32_t* err;

  __device__ __forceinline__ Tracer(const Scene& s_, const Params& p_, uint32_t* e)
      : s(s_), p(p_), rays(0), nodes(0), tests(0), err(e) {}

  __device__ __forceinline__ float U() { return rng.uniform01(); }

  __device__ __forceinline__ bool shadow(float ox, float oy, float oz, float dx, float dy, float dz, float dist) {
    ++rays;
    return traverse<true>(s, ox, oy, oz, dx, dy, dz, dist, err, nodes, tests).tri >= 0;
  }

  __device__ static void hsv2rgb(float h, float sat, float val, float& r, float& g, float& b) {
    float c = sat * val;
    float hm = h / 60.0f;
    float md = hm - floorf(hm / 2.0f) * 2.0f;
    float x = c * (1.0f - fabsf(md - 1.0f));
    float m = val - c;
    float cr = 0, cg = 0, cb = 0;
    if (h < 60.0f) { cr = c; cg = x; }
    else if (h < 120.0f) { cr = x; cg = c; }
    else if (h < 180.0f) { cg = c; cb = x; }
    else if (h < 240.0f) { cg = x; cb = c; }
    else if (h < 300.0f) { cr = x; cb = c; }
    else if (h < 360.0f) { cr = c; cb = x; }
    cr += m; cg += m; cb += m;
    r = cr * 255.0f; g = cg * 255.0f; b = cb * 255.0f;
  }

  // pathtrace.metal:165-204
  __device__ __noinline__ Hit cast_ray(float ox, float oy, float oz, float dx, float dy, float dz, float dist) {
    ++rays;
    TraceResult tr = traverse<false>(s, ox, oy, oz, dx, dy, dz, dist, err, nodes, tests);
    return attributes(tr, ox, oy, oz, dx, dy, dz);
  }

  // Surface attributes of a traversal result (the second half of cast_ray).
  __device__ __forceinline__ Hit attributes(const TraceResult& tr, float ox, float oy, float oz, float dx, float dy,
                                            float dz) const {
    Hit h;
    h.t = tr.t; h.tri = tr.tri; h.u = tr.u; h.v = tr.v;
    h.px = ox + dx * h.t; h.py = oy + dy * h.t; h.pz = oz + dz * h.t;
    h.shader = 0;
    if (h.tri >= 0 && bad_index(h.tri, s.n_tris, err, kSiteHit)) h.tri = -1;
    if (h.tri >= 0) {
      const rm_triangle& t = s.tris[h.tri];
      float w = 1.0f - (h.u + h.v);
      float nx = w * t.n0.x + (h.u * t.n1.x + h.v * t.n2.x);
      float ny = w * t.n0.y + (h.u * t.n1.y + h.v * t.n2.y);
      float nz = w * t.n0.z + (h.u * t.n1.z + h.v * t.n2.z);
      float d = 1.0f / sqrtf(nx * nx + (ny * ny + nz * nz));
      h.nix = nx * d; h.niy = ny * d; h.niz = nz * d;
      h.ar = t.ar; h.ag = t.ag; h.ab = t.ab;
      h.txr = h.txg = h.txb = 1.0f;
      if (t.texture_offset >= 0) {
        float tu = w * t.tu0 + h.u * t.tu1 + h.v * t.tu2;
        float tv = w * t.tv0 + h.u * t.tv1 + h.v * t.tv2;
        tu = fminf(tu - floorf(tu), 0.99999994f);
        tv = fminf(tv - floorf(tv), 0.99999994f);
        int x = min(int(tu * float(t.texture_width)), t.texture_width - 1);
        int y = t.texture_height - 1 - min(int(tv * float(t.texture_height)), t.texture_height - 1);
        const size_t ti = size_t(t.texture_offset) + size_t(y) * size_t(t.texture_width) + size_t(x);
        const rm_vec3 c = bad_index((long long)ti, s.n_texels, err, kSiteTexel) ? rm_vec3{1.0f, 1.0f, 1.0f} : s.texels[ti];
        h.ar *= c.x; h.ag *= c.y; h.ab *= c.z;
        h.txr = c.x; h.txg = c.y; h.txb = c.z;
      }
      h.er = t.er; h.eg = t.eg; h.eb = t.eb;
      h.ior = t.ior; h.rough = t.rough; h.shader = t.shader;
      h.ngx = t.n.x; h.ngy = t.n.y; h.ngz = t.n.z;
      if (h.shader == 1) {
        float az = rm_atanf(h.px / h.pz) * 180.0f / kPi + ((h.pz > 0.0f) ? 0.0f : 180.0f);
        float hh = (az - floorf(az / 360.0f) * 360.0f) / 360.0f;
        hsv2rgb(hh, 0.8f, 1.0f, h.ar, h.ag, h.ab);
      }
    }
    return h;
  }

  // pathtrace.metal:536-550, crossings capped at kMaxAlphaCrossings.
  __device__ __forceinline__ Hit cast_alpha_ray(float ox, float oy, float oz, float dx, float dy, float dz, float dist) {
    if (p.opaque) return cast_ray(ox, oy, oz, dx, dy, dz, dist);
    float traveled = 0.0f;
    for (int it = 0; it < kMaxAlphaCrossings && traveled < dist; ++it) {
      Hit h = cast_ray(ox + dx * traveled, oy + dy * traveled, oz + dz * traveled, dx, dy, dz, dist - traveled);
      if (h.tri < 0) return h;
      float opacity = s.tris[h.tri].alpha;
      if (opacity >= 1.0f || (opacity > 0.0f && U() < opacity)) {
        h.t += traveled;
        return h;
      }
      traveled += h.t + 0.0001f;
    }
    Hit miss;
    miss.t = kFar; miss.tri = -1;
    return miss;
  }

  __device__ __forceinline__ bool occluded(float ox, float oy, float oz, float dx, float dy, float dz, float dist) {
    return p.opaque ? shadow(ox, oy, oz, dx, dy, dz, dist) : cast_alpha_ray(ox, oy, oz, dx, dy, dz, dist).tri >= 0;
  }

  __device__ static __forceinline__ void tangent(float nx, float ny, float nz, float& tx, float& ty, float& tz,
                                                 float& bx, float& by, float& bz) {
    if (fabsf(nx) > 0.1f) { tx = nz; ty = 0.0f; tz = -nx; }
    else { tx = 0.0f; ty = -nz; tz = ny; }
    float l = 1.0f / sqrtf(tx * tx + ty * ty + tz * tz);
    tx *= l; ty *= l; tz *= l;
    bx = ny * tz - nz * ty;
    by = nz * tx - nx * tz;
    bz = nx * ty - ny * tx;
  }

  __device__ __forceinline__ void sample_cosine(float nx, float ny, float nz, float& ox, float& oy, float& oz) {
    float ru = U();
    float phi = U() * (2.0f * kPi);
    float sp, c;
    rm_sincosf(phi, &sp, &c);
    float rr = sqrtf(ru);
    float lx = rr * c, ly = rr * sp, lz = sqrtf(fmaxf(0.0f, 1.0f - ru));
    float tx, ty, tz, bx, by, bz;
    tangent(nx, ny, nz, tx, ty, tz, bx, by, bz);
    ox = tx * lx + (bx * ly + nx * lz);
    oy = ty * lx + (by * ly + ny * lz);
    oz = tz * lx + (bz * ly + nz * lz);
  }

  __device__ __forceinline__ void sample_ggx_half(float alpha2, float nx, float ny, float nz, float& hx, float& hy,
                                                  float& hz) {
    (void)U();
    float rv = U();
    float phi = U() * (2.0f * kPi);
    float sp, c;
    rm_sincosf(phi, &sp, &c);
    float cs = sqrtf((1.0f - rv) / (1.0f + (alpha2 - 1.0f) * rv));
    float sn = sqrtf(fmaxf(0.0f, 1.0f - cs * cs));
    float lx = sn * c, ly = sn * sp, lz = cs;
    float tx, ty, tz, bx, by, bz;
    tangent(nx, ny, nz, tx, ty, tz, bx, by, bz);
    hx = tx * lx + (bx * ly + nx * lz);
    hy = ty * lx + (by * ly + ny * lz);
    hz = tz * lx + (bz * ly + nz * lz);
    float d = 1.0f / sqrtf(hx * hx + hy * hy + hz * hz);
    hx *= d; hy *= d; hz *= d;
  }

  // pathtrace.metal:243-295
  // The factors of eval_bsdf that do not depend on wi, computed once for a
  // vertex whose candidate loop evaluates many wi (same expressions, so the
  // same values as eval_bsdf computes per call).
  struct BsdfPrep {
    float cos_o, g1, di, f0r, f0g, f0b, adr, adg, adb;
  };
  __device__ static __forceinline__ BsdfPrep prep_bsdf(float wox, float woy, float woz, float nx, float ny, float nz,
                                                       float alpha2, float metallic, float ar, float ag, float ab) {
    BsdfPrep q;
    q.cos_o = wox * nx + (woy * ny + woz * nz);
    q.g1 = 2.0f * q.cos_o / (q.cos_o + sqrtf(q.cos_o * q.cos_o + alpha2 * (1.0f - q.cos_o * q.cos_o)));
    q.di = 1.0f - metallic;
    q.f0r = 0.04f * q.di + ar * metallic;
    q.f0g = 0.04f * q.di + ag * metallic;
    q.f0b = 0.04f * q.di + ab * metallic;
    q.adr = ar * q.di;
    q.adg = ag * q.di;
    q.adb = ab * q.di;
    return q;
  }

  // eval_bsdf with the wi-independent factors of prep_bsdf.
  __device__ static __forceinline__ Bsdf eval_bsdf_prep(const BsdfPrep& q, float wix, float wiy, float wiz, float wox,
                                                        float woy, float woz, float nx, float ny, float nz,
                                                        float alpha2, float spec_prob) {
    Bsdf out{0.f, 0.f, 0.f, 0.f};
    float cos_i = wix * nx + (wiy * ny + wiz * nz);
    const float cos_o = q.cos_o;
    if (!(cos_i > 1e-8f && cos_o > 1e-8f)) return out;
    float hx = wix + wox, hy = wiy + woy, hz = wiz + woz;
    float hl = sqrtf(hx * hx + hy * hy + hz * hz);
    if (!(hl > 1e-8f)) return out;
    float inv = 1.0f / hl;
    hx *= inv; hy *= inv; hz *= inv;
    float cos_h = hx * nx + (hy * ny + hz * nz);
    float vo_h = wox * hx + (woy * hy + woz * hz);
    if (cos_h < 0.0f) { hx = -hx; hy = -hy; hz = -hz; cos_h = -cos_h; vo_h = -vo_h; }
    if (!(vo_h > 1e-8f)) return out;
    float dd = cos_h * cos_h * (alpha2 - 1.0f) + 1.0f;
    float D = alpha2 / (kPi * dd * dd);
    float g2 = 2.0f * cos_i / (cos_i + sqrtf(cos_i * cos_i + alpha2 * (1.0f - cos_i * cos_i)));
    float G = q.g1 * g2;
    float om = 1.0f - vo_h;
    om *= om; om *= om; om *= 1.0f - vo_h;
    float fr = q.f0r + (1.0f - q.f0r) * om, fg = q.f0g + (1.0f - q.f0g) * om, fb = q.f0b + (1.0f - q.f0b) * om;
    float kdr = q.adr * (1.0f - fr), kdg = q.adg * (1.0f - fg), kdb = q.adb * (1.0f - fb);
    float base = D * G / (4.0f * cos_i * cos_o);
    out.r = kdr / kPi + base * fr;
    out.g = kdg / kPi + base * fg;
    out.b = kdb / kPi + base * fb;
    float pdf_d = cos_i / kPi;
    float pdf_s = D * cos_h / (4.0f * vo_h);
    out.pdf = (1.0f - spec_prob) * pdf_d + spec_prob * pdf_s;
    return out;
  }

  __device__ static __forceinline__ Bsdf eval_bsdf(float wix, float wiy, float wiz, float wox, float woy, float woz,
                                                   float nx, float ny, float nz, float alpha2, float metallic,
                                                   float spec_prob, float ar, float ag, float ab) {
    Bsdf out{0.f, 0.f, 0.f, 0.f};
    float cos_i = wix * nx + (wiy * ny + wiz * nz);
    float cos_o = wox * nx + (woy * ny + woz * nz);
    if (!(cos_i > 1e-8f && cos_o > 1e-8f)) return out;
    float hx = wix + wox, hy = wiy + woy, hz = wiz + woz;
    float hl = sqrtf(hx * hx + hy * hy + hz * hz);
    if (!(hl > 1e-8f)) return out;
    float inv = 1.0f / hl;
    hx *= inv; hy *= inv; hz *= inv;
    float cos_h = hx * nx + (hy * ny + hz * nz);
    float vo_h = wox * hx + (woy * hy + woz * hz);
    if (cos_h < 0.0f) { hx = -hx; hy = -hy; hz = -hz; cos_h = -cos_h; vo_h = -vo_h; }
    if (!(vo_h > 1e-8f)) return out;
    float dd = cos_h * cos_h * (alpha2 - 1.0f) + 1.0f;
    float D = alpha2 / (kPi * dd * dd);
    float g1 = 2.0f * cos_o / (cos_o + sqrtf(cos_o * cos_o + alpha2 * (1.0f - cos_o * cos_o)));
    float g2 = 2.0f * cos_i / (cos_i + sqrtf(cos_i * cos_i + alpha2 * (1.0f - cos_i * cos_i)));
    float G = g1 * g2;
    float om = 1.0f - vo_h;
    om *= om; om *= om; om *= 1.0f - vo_h;
    float di = 1.0f - metallic;
    float f0r = 0.04f * di + ar * metallic, f0g = 0.04f * di + ag * metallic, f0b = 0.04f * di + ab * metallic;
    float fr = f0r + (1.0f - f0r) * om, fg = f0g + (1.0f - f0g) * om, fb = f0b + (1.0f - f0b) * om;
    float kdr = ar * di * (1.0f - fr), kdg = ag * di * (1.0f - fg), kdb = ab * di * (1.0f - fb);
    float base = D * G / (4.0f * cos_i * cos_o);
    out.r = kdr / kPi + base * fr;
    out.g = kdg / kPi + base * fg;
    out.b = kdb / kPi + base * fb;
    float pdf_d = cos_i / kPi;
    float pdf_s = D * cos_h / (4.0f * vo_h);
    out.pdf = (1.0f - spec_prob) * pdf_d + spec_prob * pdf_s;
    return out;
  }

  // Index into the light list of the first CDF entry >= pick, or the last
  // entry (pathtrace.metal:323-331).  The guide table narrows the binary
  // search to the entries between guide[g-1] and guide[g+2] around the
  // pick's bucket g; the one-bucket margins absorb the rounding of the bucket
  // index, so the result is the same index the full search returns.
  __device__ __forceinline__ int pick_light(float pick) const {
    int lo = 0, hi = p.lights - 1;
    if (s.guide_n > 0) {
      int g = int(pick * s.guide_inv);
      g = g < 0 ? 0 : (g >= s.guide_n ? s.guide_n - 1 : g);
      lo = __ldg(s.guide + (g > 0 ? g - 1 : 0));
      hi = __ldg(s.guide + (g + 2 < s.guide_n ? g + 2 : s.guide_n));
    }
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (__ldg(s.cdf + mid) >= pick) hi = mid; else lo = mid + 1;
    }
    if (bad_index(lo, p.lights, err, kSiteLight)) lo = 0;
    return lo;
  }

  // pathtrace.metal:299-469
  __device__ __noinline__ void direct_lighting(float px, float py, float pz, float nx, float ny, float nz, float wox,
                                               float woy, float woz, float rough, float metallic, float spec_prob,
                                               float ar, float ag, float ab, float& o_r, float& o_g, float& o_b,
                                               float& out_sumW, uint32_t& out_M) {
    o_r = o_g = o_b = 0.0f;
    out_sumW = 0.0f;
    out_M = 0;
    if (p.lights == 0 || !(p.light_total > 1e-12f)) return;
    int Mc = p.restir_candidates;
    if (Mc < 1) Mc = 1;
    if (Mc > 32) Mc = 32;
    float r2 = rough;
    if (r2 < 0.0f) r2 = 0.0f;
    if (r2 > 1.0f) r2 = 1.0f;
    if (r2 < 0.02f) r2 = 0.02f;
    float alpha2 = (r2 * r2) * (r2 * r2);
    const float LT = p.light_total;
    if (Mc <= 1) {
      float pick = U() * LT;
      const LightRec t = load_light(s, pick_light(pick));
      float lu = U(), lv = U();
      if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
      float lw = 1.0f - lu - lv;
      float ldx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x) - px;
      float ldy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y) - py;
      float ldz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z) - pz;
      float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
      if (!(dist > 0.003f)) { out_M = 1; return; }
      float inv = 1.0f / dist;
      ldx *= inv; ldy *= inv; ldz *= inv;
      float lcos = -(t.nn.x * ldx + (t.nn.y * ldy + t.nn.z * ldz));
      float scos = nx * ldx + (ny * ldy + nz * ldz);
      if (!(lcos > 1e-8f && scos > 1e-8f)) { out_M = 1; return; }
      float lt_lum = lum3(t.er, t.eg, t.eb);
      if (lt_lum < 1e-6f) lt_lum = 1e-6f;
      float pdf = dist * dist * lt_lum / (lcos * LT);
      float sox = px + nx * 0.002f, soy = py + ny * 0.002f, soz = pz + nz * 0.002f;
      if (occluded(sox, soy, soz, ldx, ldy, ldz, dist - 0.003f)) {
        Bsdf eo = eval_bsdf(ldx, ldy, ldz, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
        float Fr0 = t.er * eo.r * scos * t.alpha;
        float Fg0 = t.eg * eo.g * scos * t.alpha;
        float Fb0 = t.eb * eo.b * scos * t.alpha;
        float ph0 = lum3(Fr0, Fg0, Fb0);
        out_sumW = (ph0 > 0.0f && pdf > 1e-12f) ? ph0 / pdf : 0.0f;
        out_M = 1;
        return;
      }
      Bsdf e = eval_bsdf(ldx, ldy, ldz, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
      if (!(pdf > 1e-12f)) { out_M = 1; return; }
      float Fr = t.er * e.r * scos * t.alpha;
      float Fg = t.eg * e.g * scos * t.alpha;
      float Fb = t.eb * e.b * scos * t.alpha;
      float ph = lum3(Fr, Fg, Fb);
      out_sumW = (ph > 0.0f) ? ph / pdf : 0.0f;
      out_M = 1;
      float wnee = 1.0f;
      if (!p.nomis && e.pdf > 1e-20f) wnee = pdf / (pdf + e.pdf);
      float k = scos * wnee * t.alpha / pdf;
      o_r = t.er * e.r * k;
      o_g = t.eg * e.g * k;
      o_b = t.eb * e.b * k;
      return;
    }
    float sumW = 0.0f;
    float sel_lx = 0, sel_ly = 0, sel_lz = 0, sel_Fr = 0, sel_Fg = 0, sel_Fb = 0, sel_phat = 0, sel_epdf = 0;
    bool have = false;
    for (int j = 0; j < Mc; ++j) {
      float pick = U() * LT;
      const LightRec t = load_light(s, pick_light(pick));
      float lu = U(), lv = U();
      if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
      float lw = 1.0f - lu - lv;
      float qx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x);
      float qy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y);
      float qz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z);
      float ldx = qx - px, ldy = qy - py, ldz = qz - pz;
      float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
      float w = 0, ph = 0, epdf = 0, Fr = 0, Fg = 0, Fb = 0;
      if (dist > 0.003f) {
        float inv = 1.0f / dist;
        float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
        float lcos = -(t.nn.x * dxn + (t.nn.y * dyn + t.nn.z * dzn));
        float scos = nx * dxn + (ny * dyn + nz * dzn);
        if (lcos > 1e-8f && scos > 1e-8f) {
          float lt_lum = lum3(t.er, t.eg, t.eb);
          if (lt_lum < 1e-6f) lt_lum = 1e-6f;
          float q = dist * dist * lt_lum / (lcos * LT);
          if (q > 1e-12f) {
            Bsdf e = eval_bsdf(dxn, dyn, dzn, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
            epdf = e.pdf;
            Fr = t.er * e.r * scos * t.alpha;
            Fg = t.eg * e.g * scos * t.alpha;
            Fb = t.eb * e.b * scos * t.alpha;
            ph = lum3(Fr, Fg, Fb);
            if (ph > 0.0f) w = ph / q;
          }
        }
      }
      sumW += w;
      float r = U();
      if (w > 0.0f && r * sumW < w) {
        have = true;
        sel_lx = qx; sel_ly = qy; sel_lz = qz;
        sel_Fr = Fr; sel_Fg = Fg; sel_Fb = Fb;
        sel_phat = ph; sel_epdf = epdf;
      }
    }
    out_sumW = sumW;
    out_M = uint32_t(Mc);
    if (!have || !(sumW > 0.0f) || !(sel_phat > 0.0f)) return;
    float pdf_ris = float(Mc) * sel_phat / sumW;
    float wnee = 1.0f;
    if (!p.nomis && sel_epdf > 1e-20f) wnee = pdf_ris / (pdf_ris + sel_epdf);
    float vdx = sel_lx - px, vdy = sel_ly - py, vdz = sel_lz - pz;
    float vdist = sqrtf(vdx * vdx + vdy * vdy + vdz * vdz);
    if (!(vdist > 0.003f)) return;
    float vinv = 1.0f / vdist;
    vdx *= vinv; vdy *= vinv; vdz *= vinv;
    float sox = px + nx * 0.002f, soy = py + ny * 0.002f, soz = pz + nz * 0.002f;
    if (occluded(sox, soy, soz, vdx, vdy, vdz, vdist - 0.003f)) return;
    float W = sumW / (float(Mc) * sel_phat);
    o_r = sel_Fr * W * wnee;
    o_g = sel_Fg * W * wnee;
    o_b = sel_Fb * W * wnee;
  }

  // The single-candidate branch (Mc <= 1, pathtrace.metal:319-384) of
  // direct_lighting_deferred, inlined where a caller knows Mc <= 1.
  // `parts`, when given, receives the light's list index and the factor k of
  // the contribution o = emission * bsdf * k (the adjoint differentiates it).
  __device__ __forceinline__ void nee_single_deferred(float px, float py, float pz, float nx, float ny, float nz,
                                                      float wox, float woy, float woz, float rough, float metallic,
                                                      float spec_prob, float ar, float ag, float ab, float& o_r,
                                                      float& o_g, float& o_b, float& out_sumW, uint32_t& out_M,
                                                      bool& has_ray, float& sox, float& soy, float& soz,
                                                      float& sdx, float& sdy, float& sdz, float& sdist,
                                                      float* parts = nullptr) {
    o_r = o_g = o_b = 0.0f;
    out_sumW = 0.0f;
    out_M = 0;
    has_ray = false;
    if (p.lights == 0 || !(p.light_total > 1e-12f)) return;
    float r2 = rough;
    if (r2 < 0.0f) r2 = 0.0f;
    if (r2 > 1.0f) r2 = 1.0f;
    if (r2 < 0.02f) r2 = 0.02f;
    float alpha2 = (r2 * r2) * (r2 * r2);
    const float LT = p.light_total;
    float pick = U() * LT;
    const int li = pick_light(pick);
    const LightRec t = load_light(s, li);
    if (parts) { parts[0] = __int_as_float(li); parts[1] = 0.0f; }
    float lu = U(), lv = U();
    if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
    float lw = 1.0f - lu - lv;
    float ldx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x) - px;
    float ldy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y) - py;
    float ldz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z) - pz;
    float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
    if (!(dist > 0.003f)) { out_M = 1; return; }
    float inv = 1.0f / dist;
    ldx *= inv; ldy *= inv; ldz *= inv;
    float lcos = -(t.nn.x * ldx + (t.nn.y * ldy + t.nn.z * ldz));
    float scos = nx * ldx + (ny * ldy + nz * ldz);
    if (!(lcos > 1e-8f && scos > 1e-8f)) { out_M = 1; return; }
    float lt_lum = lum3(t.er, t.eg, t.eb);
    if (lt_lum < 1e-6f) lt_lum = 1e-6f;
    float pdf = dist * dist * lt_lum / (lcos * LT);
    has_ray = true;
    sox = px + nx * 0.002f; soy = py + ny * 0.002f; soz = pz + nz * 0.002f;
    sdx = ldx; sdy = ldy; sdz = ldz; sdist = dist - 0.003f;
    Bsdf e = eval_bsdf(ldx, ldy, ldz, wox, woy, woz, nx, ny, nz, alpha2, metallic, spec_prob, ar, ag, ab);
    out_M = 1;
    if (!(pdf > 1e-12f)) return;
    float Fr = t.er * e.r * scos * t.alpha;
    float Fg = t.eg * e.g * scos * t.alpha;
    float Fb = t.eb * e.b * scos * t.alpha;
    float ph = lum3(Fr, Fg, Fb);
    out_sumW = (ph > 0.0f) ? ph / pdf : 0.0f;
    float wnee = 1.0f;
    if (!p.nomis && e.pdf > 1e-20f) wnee = pdf / (pdf + e.pdf);
    float k = scos * wnee * t.alpha / pdf;
    o_r = t.er * e.r * k;
    o_g = t.eg * e.g * k;
    o_b = t.eb * e.b * k;
    if (parts) parts[1] = k;
  }

  // direct_lighting for opaque scenes with the visibility test left to the
  // caller: the same draws and arithmetic, returning the contribution a
  // visible light would add (o_*) and the shadow ray to test (has_ray).  In an
  // opaque scene the visibility test consumes no random numbers and changes
  // nothing but the contribution (out_sumW is the same either way), so testing
  // the ray later in a separate pass gives the same result.
  __device__ __noinline__ void direct_lighting_deferred(float px, float py, float pz, float nx, float ny, float nz,
                                                        float wox, float woy, float woz, float rough, float metallic,
                                                        float spec_prob, float ar, float ag, float ab, float& o_r,
                                                        float& o_g, float& o_b, float& out_sumW, uint32_t& out_M,
                                                        bool& has_ray, float& sox, float& soy, float& soz,
                                                        float& sdx, float& sdy, float& sdz, float& sdist,
                                                        float* parts = nullptr) {
    o_r = o_g = o_b = 0.0f;
    out_sumW = 0.0f;
    out_M = 0;
    has_ray = false;
    if (parts) { parts[0] = __int_as_float(0); parts[1] = 0.0f; }
    if (p.lights == 0 || !(p.light_total > 1e-12f)) return;
    int Mc = p.restir_candidates;
    if (Mc < 1) Mc = 1;
    if (Mc > 32) Mc = 32;
    float r2 = rough;
    if (r2 < 0.0f) r2 = 0.0f;
    if (r2 > 1.0f) r2 = 1.0f;
    if (r2 < 0.02f) r2 = 0.02f;
    float alpha2 = (r2 * r2) * (r2 * r2);
    const float LT = p.light_total;
    if (Mc <= 1) {
      nee_single_deferred(px, py, pz, nx, ny, nz, wox, woy, woz, rough, metallic, spec_prob, ar, ag, ab, o_r, o_g,
                          o_b, out_sumW, out_M, has_ray, sox, soy, soz, sdx, sdy, sdz, sdist, parts);
      return;
    }
    float sumW = 0.0f;
    float sel_lx = 0, sel_ly = 0, sel_lz = 0, sel_Fr = 0, sel_Fg = 0, sel_Fb = 0, sel_phat = 0, sel_epdf = 0;
    float sel_sa = 0;  // scos * alpha of the selected candidate (for `parts`)
    int sel_li = 0;
    bool have = false;
    const BsdfPrep bp = prep_bsdf(wox, woy, woz, nx, ny, nz, alpha2, metallic, ar, ag, ab);
    for (int j = 0; j < Mc; ++j) {
      float pick = U() * LT;
      const int li = pick_light(pick);
      const LightRec t = load_light(s, li);
      float lu = U(), lv = U();
      if (lu + lv > 1.0f) { lu = 1.0f - lu; lv = 1.0f - lv; }
      float lw = 1.0f - lu - lv;
      float qx = lw * t.v0.x + (lu * t.v1.x + lv * t.v2.x);
      float qy = lw * t.v0.y + (lu * t.v1.y + lv * t.v2.y);
      float qz = lw * t.v0.z + (lu * t.v1.z + lv * t.v2.z);
      float ldx = qx - px, ldy = qy - py, ldz = qz - pz;
      float dist = sqrtf(ldx * ldx + ldy * ldy + ldz * ldz);
      float w = 0, ph = 0, epdf = 0, Fr = 0, Fg = 0, Fb = 0, sa = 0;
      if (dist > 0.003f) {
        float inv = 1.0f / dist;
        float dxn = ldx * inv, dyn = ldy * inv, dzn = ldz * inv;
        float lcos = -(t.nn.x * dxn + (t.nn.y * dyn + t.nn.z * dzn));
        float scos = nx * dxn + (ny * dyn + nz * dzn);
        if (lcos > 1e-8f && scos > 1e-8f) {
          float lt_lum = lum3(t.er, t.eg, t.eb);
          if (lt_lum < 1e-6f) lt_lum = 1e-6f;
          float q = dist * dist * lt_lum / (lcos * LT);
          if (q > 1e-12f) {
            Bsdf e = eval_bsdf_prep(bp, dxn, dyn, dzn, wox, woy, woz, nx, ny, nz, alpha2, spec_prob);
            epdf = e.pdf;
            Fr = t.er * e.r * scos * t.alpha;
            Fg = t.eg * e.g * scos * t.alpha;
            Fb = t.eb * e.b * scos * t.alpha;
            ph = lum3(Fr, Fg, Fb);
            if (ph > 0.0f) w = ph / q;
            sa = scos * t.alpha;
          }
        }
      }
      sumW += w;
      float r = U();
      if (w > 0.0f && r * sumW < w) {
        have = true;
        sel_lx = qx; sel_ly = qy; sel_lz = qz;
        sel_Fr = Fr; sel_Fg = Fg; sel_Fb = Fb;
        sel_phat = ph; sel_epdf = epdf;
        sel_sa = sa; sel_li = li;
      }
    }
    out_sumW = sumW;
    out_M = uint32_t(Mc);
    if (!have || !(sumW > 0.0f) || !(sel_phat > 0.0f)) return;
    float pdf_ris = float(Mc) * sel_phat / sumW;
    float wnee = 1.0f;
    if (!p.nomis && sel_epdf > 1e-20f) wnee = pdf_ris / (pdf_ris + sel_epdf);
    float vdx = sel_lx - px, vdy = sel_ly - py, vdz = sel_lz - pz;
    float vdist = sqrtf(vdx * vdx + vdy * vdy + vdz * vdz);
    if (!(vdist > 0.003f)) return;
    float vinv = 1.0f / vdist;
    vdx *= vinv; vdy *= vinv; vdz *= vinv;
    has_ray = true;
    sox = px + nx * 0.002f; soy = py + ny * 0.002f; soz = pz + nz * 0.002f;
    sdx = vdx; sdy = vdy; sdz = vdz; sdist = vdist - 0.003f;
    float W = sumW / (float(Mc) * sel_phat);
    o_r = sel_Fr * W * wnee;
    o_g = sel_Fg * W * wnee;
    o_b = sel_Fb * W * wnee;
    // the selected light and the factor k of o = Le * f * k (held by the adjoint)
    if (parts) { parts[0] = __int_as_float(sel_li); parts[1] = sel_sa * W * wnee; }
  }

  __device__ static __forceinline__ float fresnel(float ci_in, float eta_in, float eta_out) {
    float ci = ci_in;
    if (ci < 0.0f) ci = 0.0f;
    if (ci > 1.0f) ci = 1.0f;
    float eta = eta_in / eta_out;
    float s2 = eta * eta * (1.0f - ci * ci);
    if (s2 >= 1.0f) return 1.0f;
    float ct = sqrtf(1.0f - s2);
    float rp = (eta_out * ci - eta_in * ct) / (eta_out * ci + eta_in * ct);
    float rs = (eta_in * ci - eta_out * ct) / (eta_in * ci + eta_out * ct);
    return 0.5f * (rp * rp + rs * rs);
  }

  // pathtrace.metal:470-534; returns valid, writes direction and eta scale.
  // `parts`, when given, receives what the adjoint differentiates: the event
  // (0 reflection, 1 refraction, 2 total internal reflection), cos_m, for a
  // rough surface cos_i, cos_o, cos_h and whether the weight was clamped, and
  // |h x n|^2.
  __device__ __noinline__ bool sample_dielectric(float wox, float woy, float woz, float nx, float ny, float nz,
                                                 float cdx, float cdy, float cdz, float ior, bool front, float rough,
                                                 float alpha2, float& o_x, float& o_y, float& o_z, float& eta_scale,
                                                 float* parts = nullptr) {
    bool valid = true;
    float eta_i = 1.0f, eta_t = ior;
    if (!front) { eta_i = ior; eta_t = 1.0f; }
    float hx, hy, hz;
    if (rough <= 0.0201f) { hx = nx; hy = ny; hz = nz; }
    else {
      sample_ggx_half(alpha2, nx, ny, nz, hx, hy, hz);
      float md = wox * hx + (woy * hy + woz * hz);
      if (!(md > 1e-8f)) valid = false;
    }
    float cos_m = wox * hx + (woy * hy + woz * hz);
    if (cos_m < 0.0f) { hx = -hx; hy = -hy; hz = -hz; cos_m = -cos_m; }
    if (cos_m > 1.0f) cos_m = 1.0f;
    float fres = fresnel(cos_m, eta_i, eta_t);
    float eta = eta_i / eta_t;
    float s2 = eta * eta * (1.0f - cos_m * cos_m);
    if (s2 >= 1.0f || U() < fres) {
      o_x = 2.0f * cos_m * hx - wox;
      o_y = 2.0f * cos_m * hy - woy;
      o_z = 2.0f * cos_m * hz - woz;
      eta_scale = 1.0f;
      if (parts) parts[0] = s2 >= 1.0f ? 2.0f : 0.0f;
    } else {
      float cos_t = sqrtf(1.0f - s2);
      o_x = eta * cdx + hx * (eta * cos_m - cos_t);
      o_y = eta * cdy + hy * (eta * cos_m - cos_t);
      o_z = eta * cdz + hz * (eta * cos_m - cos_t);
      eta_scale = eta * eta;
      if (parts) parts[0] = 1.0f;
    }
    if (parts) {
      parts[1] = cos_m;
      parts[2] = parts[3] = parts[4] = parts[5] = 0.0f;
      const float cx = hy * nz - hz * ny, cy = hz * nx - hx * nz, cz = hx * ny - hy * nx;
      parts[6] = cx * cx + cy * cy + cz * cz;  // |h x n|^2
    }
    {
      float d = 1.0f / sqrtf(o_x * o_x + o_y * o_y + o_z * o_z);
      o_x *= d; o_y *= d; o_z *= d;
    }
    if (rough > 0.0201f) {
      float cos_i = fabsf(o_x * nx + (o_y * ny + o_z * nz));
      float cos_o = fabsf(wox * nx + (woy * ny + woz * nz));
      float cos_h = fabsf(hx * nx + (hy * ny + hz * nz));
      float vo_h = fabsf(wox * hx + (woy * hy + woz * hz));
      if (cos_i > 1e-8f && cos_o > 1e-8f && cos_h > 1e-8f && vo_h > 1e-8f) {
        float g1 = 2.0f * cos_o / (cos_o + sqrtf(cos_o * cos_o + alpha2 * (1.0f - cos_o * cos_o)));
        float g2 = 2.0f * cos_i / (cos_i + sqrtf(cos_i * cos_i + alpha2 * (1.0f - cos_i * cos_i)));
        float w = g1 * g2 * vo_h / (cos_o * cos_h);
        if (parts) { parts[2] = cos_i; parts[3] = cos_o; parts[4] = cos_h; parts[5] = w > 10.0f ? 1.0f : 0.0f; }
        if (w > 10.0f) w = 10.0f;
        eta_scale *= w;
      } else {
        valid = false;
      }
    }
    return valid;
  }

  // pathtrace.metal:552-728
  __device__ __noinline__ void pathtrace(float ox, float oy, float oz, float dx, float dy, float dz, int max_bounces,
                                         float& out_r, float& out_g, float& out_b) {
    float accr = 0, accg = 0, accb = 0, thr_r = 1, thr_g = 1, thr_b = 1;
    int bounce = 0, prev_delta = 1;
    float last_pdf = 0, prev_sumW = 0;
    uint32_t prev_M = 0;
    float prev_br = 0, prev_bg = 0, prev_bb = 0, prev_cos = 0;
    const float LT = p.light_total;
    for (int b = 0; b < max_bounces; ++b) {
      Hit hit = cast_alpha_ray(ox, oy, oz, dx, dy, dz, kFar);
      if (hit.tri < 0) break;
      float pnx = hit.nix, pny = hit.niy, pnz = hit.niz;
      float geom = hit.ngx * pnx + (hit.ngy * pny + hit.ngz * pnz);
      if (geom < 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; }
      float ndot = dx * pnx + (dy * pny + dz * pnz);
      bool front = true;
      if (ndot > 0.0f) { pnx = -pnx; pny = -pny; pnz = -pnz; front = false; }
      float wox = -dx, woy = -dy, woz = -dz;
      float rough = hit.rough;
      if (rough < 0.0f) rough = 0.0f;
      if (rough > 1.0f) rough = 1.0f;
      if (rough < 0.02f) rough = 0.02f;
      float alpha = rough * rough;
      float alpha2 = alpha * alpha;
      const rm_triangle& lt = s.tris[hit.tri];
      float metallic = lt.metallic;
      if (metallic < 0.0f) metallic = 0.0f;
      if (metallic > 1.0f) metallic = 1.0f;
      if (bounce == 0 || prev_delta == 1) {
        accr += hit.er * thr_r; accg += hit.eg * thr_g; accb += hit.eb * thr_b;
      } else {
        float lx = hit.px - ox, ly = hit.py - oy, lz = hit.pz - oz;
        float dist2 = lx * lx + ly * ly + lz * lz;
        float dist = sqrtf(dist2);
        float pl = 1e30f;
        float lta = lt.alpha;
        if (dist > 1e-20f && last_pdf > 1e-20f && prev_M > 0 && prev_sumW > 1e-20f) {
          float ph = lum3(hit.er * prev_br * prev_cos * lta, hit.eg * prev_bg * prev_cos * lta,
                          hit.eb * prev_bb * prev_cos * lta);
          if (ph > 1e-20f) pl = float(prev_M) * ph / prev_sumW;
          else {
            float inv = 1.0f / dist;
            float lxn = lx * inv, lyn = ly * inv, lzn = lz * inv;
            float cos_l = -(lt.nn.x * lxn + (lt.nn.y * lyn + lt.nn.z * lzn));
            if (cos_l > 1e-8f) {
              float lum = lum3(lt.er, lt.eg, lt.eb);
              if (lum < 1e-6f) lum = 1e-6f;
              pl = dist2 * lum / (cos_l * LT);
            }
          }
        } else if (dist > 1e-20f && last_pdf > 1e-20f) {
          float inv = 1.0f / dist;
          lx *= inv; ly *= inv; lz *= inv;
          float cos_l = -(lt.nn.x * lx + (lt.nn.y * ly + lt.nn.z * lz));
          if (cos_l > 1e-8f) {
            float lum = lum3(lt.er, lt.eg, lt.eb);
            if (lum < 1e-6f) lum = 1e-6f;
            pl = dist2 * lum / (cos_l * LT);
          }
        }
        float w = p.nomis ? 0.0f : ((last_pdf + pl > 1e-20f) ? last_pdf / (last_pdf + pl) : 0.0f);
        accr += hit.er * thr_r * w; accg += hit.eg * thr_g * w; accb += hit.eb * thr_b * w;
      }
      if (hit.ior > 1.0001f) {
        float nx2, ny2, nz2, eta_scale;
        bool valid = sample_dielectric(wox, woy, woz, pnx, pny, pnz, dx, dy, dz, hit.ior, front, rough, alpha2, nx2,
                                       ny2, nz2, eta_scale);
        if (!valid) break;
        thr_r *= eta_scale; thr_g *= eta_scale; thr_b *= eta_scale;
        float sg = 1.0f;
        if (nx2 * pnx + (ny2 * pny + nz2 * pnz) < 0.0f) sg = -1.0f;
        ox = hit.px + pnx * 0.001f * sg;
        oy = hit.py + pny * 0.001f * sg;
        oz = hit.pz + pnz * 0.001f * sg;
        dx = nx2; dy = ny2; dz = nz2;
        prev_delta = 1;
        prev_sumW = 0; prev_M = 0;
      } else {
        float spec_prob = 0.05f + 0.95f * metallic;
        if (spec_prob > 0.98f) spec_prob = 0.98f;
        if (metallic >= 0.999f) spec_prob = 1.0f;
        float cur_sumW = 0;
        uint32_t cur_M = 0;
        {
          float dlr, dlg, dlb;
          direct_lighting(hit.px, hit.py, hit.pz, pnx, pny, pnz, wox, woy, woz, rough, metallic, spec_prob, hit.ar,
                          hit.ag, hit.ab, dlr, dlg, dlb, cur_sumW, cur_M);
          accr += dlr * thr_r; accg += dlg * thr_g; accb += dlb * thr_b;
        }
        float nx2, ny2, nz2;
        if (U() < spec_prob) {
          float hx, hy, hz;
          sample_ggx_half(alpha2, pnx, pny, pnz, hx, hy, hz);
          float md = wox * hx + (woy * hy + woz * hz);
          if (!(md > 1e-8f)) break;
          nx2 = 2.0f * md * hx - wox;
          ny2 = 2.0f * md * hy - woy;
          nz2 = 2.0f * md * hz - woz;
          prev_delta = (rough <= 0.0201f) ? 1 : 0;
        } else {
          sample_cosine(pnx, pny, pnz, nx2, ny2, nz2);
          prev_delta = 0;
        }
        float ncos = nx2 * pnx + (ny2 * pny + nz2 * pnz);
        if (!(ncos > 1e-8f)) break;
        {
          float d = 1.0f / sqrtf(nx2 * nx2 + ny2 * ny2 + nz2 * nz2);
          nx2 *= d; ny2 *= d; nz2 *= d;
        }
        Bsdf e = eval_bsdf(nx2, ny2, nz2, wox, woy, woz, pnx, pny, pnz, alpha2, metallic, spec_prob, hit.ar, hit.ag,
                           hit.ab);
        if (!(e.pdf > 1e-12f)) break;
        last_pdf = e.pdf;
        float cos_i = nx2 * pnx + (ny2 * pny + nz2 * pnz);
        thr_r *= e.r * cos_i / e.pdf;
        thr_g *= e.g * cos_i / e.pdf;
        thr_b *= e.b * cos_i / e.pdf;
        prev_sumW = cur_sumW; prev_M = cur_M;
        prev_br = e.r; prev_bg = e.g; prev_bb = e.b; prev_cos = cos_i;
        ox = hit.px + pnx * 0.001f;
        oy = hit.py + pny * 0.001f;
        oz = hit.pz + pnz * 0.001f;
        dx = nx2; dy = ny2; dz = nz2;
      }
      if (thr_r < 0.0f) thr_r = 0.0f;
      if (thr_g < 0.0f) thr_g = 0.0f;
      if (thr_b < 0.0f) thr_b = 0.0f;
      float mx = fmaxf(thr_r, thr_g);
      mx = fmaxf(mx, thr_b);
      if (!(mx >= 1e-12f)) break;
      if (p.rr && bounce >= 1) {
        float rr = mx;
        if (rr < 0.05f) rr = 0.05f;
        if (rr > 0.9f) rr = 0.9f;
        if (!(U() <= rr)) break;
        float ir = 1.0f / rr;
        thr_r *= ir; thr_g *= ir; thr_b *= ir;
      }
      bounce++;
    }
    out_r = accr; out_g = accg; out_b = accb;
  }

  // pathtrace.metal:729-737
  __device__ __forceinline__ void sample_sensor(float sx, float sy, int max_bounces, float& r, float& g, float& b) {
    const rm_camera& cam = p.camera;
    float focal2 = cam.focal * cam.focal;
    float dist = 1.0f / sqrtf(sx * sx + (sy * sy + focal2));
    float tx = sx * dist, ty = sy * dist, tz = cam.focal * dist;
    float dx = tx * cam.m0 + (ty * cam.m1 + tz * cam.m2);
    float dy = tx * cam.m3 + (ty * cam.m4 + tz * cam.m5);
    float dz = tx * cam.m6 + (ty * cam.m7 + tz * cam.m8);
    pathtrace(cam.x, cam.y, cam.z, dx, dy, dz, max_bounces, r, g, b);
  }

  // pathtrace.metal:754-755
  __device__ __forceinline__ void jitter(uint32_t x, uint32_t y, float& sx, float& sy) {
    const float res = p.resolution;
    sx = float(x) + 1e-12f + (res - 2e-12f) * U() - float(p.width) * 0.5f;
    sy = float(p.height) * 0.5f - (float(y) + 1e-12f + (res - 2e-12f) * U());
  }
};

__device__ __forceinline__ uint8_t tonemap8(float c) {
  float v = floorf(c / (c + 1.0f) * 255.0f);
  v = fminf(fmaxf(v, 0.0f), 255.0f);
  return uint8_t(v);
}

}  // namespace rmd

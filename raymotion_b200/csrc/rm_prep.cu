// rm_prep.cu - world triangles of instanced models, built on the device.
//
// The reference builds its world on the host before every frame
// (include/raymotion/runtime.hpp:121-131): Objects::append transforms each
// model triangle of each pushed instance (runtime.hpp:86-113) and
// Scene::add_triangle precomputes, rejects degenerate triangles and extends the
// emissive CDF (src/engine/scene.cpp:16-87); metal.mm then packs the fp64
// Scene to fp32 records.  Here the same fp64 expressions, in the same
// operation order (the library is compiled without FMA contraction), run one
// thread per (instance, model triangle) slot:
//   pass 1 (k_prep_flags): keep / light flags of every slot;
//   exclusive scans of both flag arrays give each kept triangle its world
//   index and each light its light-list index, in push order;
//   pass 2 (k_prep_write): the packed rm_triangle, the light list and the
//   light weights area x luminance;
//   k_prep_cdf: the running sum of the weights, left to right in double as
//   light_total += w does, and the counts.
// Textures are not carried (models have none: texture_offset -1).
#include <cuda_runtime.h>


#include "rm_launch.h"
#include "rm_sort.h"

static_assert(sizeof(rm_model_tri) == 280, "rm_model_tri layout");
static_assert(sizeof(rm_instance) == 184, "rm_instance layout");

namespace rmd {
namespace {

struct D3 { double x, y, z; };

__device__ __forceinline__ D3 ld3(const double* v) { return D3{v[0], v[1], v[2]}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// normalize (math.hpp:58-62): zero below length 1e-30, else a division by the length
__device__ __forceinline__ D3 normalize3(D3 v) {
  const double l = sqrt(dot3(v, v));
  if (l < 1e-30) return D3{0.0, 0.0, 0.0};
  return D3{v.x / l, v.y / l, v.z / l};
}

// rotate about x, then y, then z with the instance's cosines and sines (runtime.hpp:94-101)
__device__ __forceinline__ D3 rotate3(const rm_instance& in, D3 v) {
  double c = in.cos_rot[0], s = in.sin_rot[0];
  v = D3{v.x, c * v.y - s * v.z, s * v.y + c * v.z};
  c = in.cos_rot[1];
  s = in.sin_rot[1];
  v = D3{c * v.x + s * v.z, v.y, -s * v.x + c * v.z};
  c = in.cos_rot[2];
  s = in.sin_rot[2];
  return D3{c * v.x - s * v.y, s * v.x + c * v.y, v.z};
}

__device__ __forceinline__ D3 point3(const rm_instance& in, D3 v) {
  const D3 r = rotate3(in, D3{v.x * in.scale[0], v.y * in.scale[1], v.z * in.scale[2]});
  return D3{r.x + in.position[0], r.y + in.position[1], r.z + in.position[2]};
}

__device__ __forceinline__ D3 normal3(const rm_instance& in, D3 v) {
  return normalize3(rotate3(in, D3{v.x / in.scale[0], v.y / in.scale[1], v.z / in.scale[2]}));
}

__device__ __forceinline__ rm_vec3 f3(D3 v) { return rm_vec3{float(v.x), float(v.y), float(v.z)}; }

// The instance and model triangle of world slot g (start: n_inst + 1 prefix sums).
__device__ __forceinline__ int slot_instance(const int* __restrict__ start, int n_inst, int g) {
  int lo = 0, hi = n_inst - 1;
  while (lo < hi) {  // last instance whose start <= g
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct World {
  D3 p0, p1, p2, e1, e2;
  double d00, d01, d11, denom;
  double er, eg, eb;
};

__device__ __forceinline__ World world_of(const rm_instance& in, const rm_model_tri& t) {
  World w;
  w.p0 = point3(in, ld3(t.v0));
  w.p1 = point3(in, ld3(t.v1));
  w.p2 = point3(in, ld3(t.v2));
  w.e1 = D3{w.p1.x - w.p0.x, w.p1.y - w.p0.y, w.p1.z - w.p0.z};
  w.e2 = D3{w.p2.x - w.p0.x, w.p2.y - w.p0.y, w.p2.z - w.p0.z};
  w.d00 = dot3(w.e1, w.e1);
  w.d01 = dot3(w.e1, w.e2);
  w.d11 = dot3(w.e2, w.e2);
  w.denom = w.d00 * w.d11 - w.d01 * w.d01;
  w.er = in.emission[0] < 0 ? t.er : in.emission[0];
  w.eg = in.emission[1] < 0 ? t.eg : in.emission[1];
  w.eb = in.emission[2] < 0 ? t.eb : in.emission[2];
  return w;
}

__device__ __forceinline__ bool kept(const World& w) { return !(fabs(w.denom) <= 1e-12); }

// emissive with a positive area (scene.cpp:73-84): its CDF weight, else 0
__device__ __forceinline__ double light_weight(const World& w) {
  if (!(w.er + (w.eg + w.eb) > 0)) return 0.0;
  double area2 = w.d00 * w.d11 - w.d01 * w.d01;
  if (area2 < 0) area2 = 0;
  const double area = 0.5 * sqrt(area2);
  if (!(area > 1e-12)) return 0.0;
  double lum = 0.2126 * w.er + 0.7152 * w.eg + 0.0722 * w.eb;
  if (lum < 1e-6) lum = 1e-6;
  return area * lum;
}

__device__ __forceinline__ double keep_or(double v, double model) { return isnan(v) ? model : v; }

__global__ void __launch_bounds__(256) k_prep_flags(const rm_instance* __restrict__ inst,
                                                    const rm_model_tri* const* __restrict__ mptr,
                                                    const int* __restrict__ start, int n_inst, int total,
                                                    int* __restrict__ keep, int* __restrict__ light) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int i = slot_instance(start, n_inst, g);
  const rm_instance in = inst[i];
  const World w = world_of(in, mptr[i][g - start[i]]);
  const bool k = kept(w);
  keep[g] = k ? 1 : 0;
  light[g] = (k && light_weight(w) > 0.0) ? 1 : 0;
}

__global__ void __launch_bounds__(256) k_prep_write(const rm_instance* __restrict__ inst,
                                                    const rm_model_tri* const* __restrict__ mptr,
                                                    const int* __restrict__ start, int n_inst, int total,
                                                    const int* __restrict__ keep, const int* __restrict__ kscan,
                                                    const int* __restrict__ light, const int* __restrict__ lscan,
                                                    rm_triangle* __restrict__ out, int32_t* __restrict__ light_tri,
                                                    double* __restrict__ weight, int* __restrict__ flags) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total || !keep[g]) return;
  const int i = slot_instance(start, n_inst, g);
  const rm_instance in = inst[i];
  const rm_model_tri& t = mptr[i][g - start[i]];
  const World w = world_of(in, t);
  const int o = kscan[g];
  rm_triangle r;
  r.v0 = f3(w.p0);
  r.v1 = f3(w.p1);
  r.v2 = f3(w.p2);
  const D3 n = cross3(w.e1, w.e2);
  r.n = f3(n);
  r.nn = f3(normalize3(n));
  r.n0 = f3(normal3(in, ld3(t.n0)));
  r.n1 = f3(normal3(in, ld3(t.n1)));
  r.n2 = f3(normal3(in, ld3(t.n2)));
  r.ar = float(in.albedo[0] < 0 ? t.ar : in.albedo[0]);
  r.ag = float(in.albedo[1] < 0 ? t.ag : in.albedo[1]);
  r.ab = float(in.albedo[2] < 0 ? t.ab : in.albedo[2]);
  r.er = float(w.er);
  r.eg = float(w.eg);
  r.eb = float(w.eb);
  r.ior = float(keep_or(in.refract, t.ior));
  r.rough = float(keep_or(in.rough, t.rough));
  r.metallic = float(keep_or(in.metallic, t.metallic));
  const double a = keep_or(in.alpha, t.alpha);
  r.alpha = float(isfinite(a) ? (a < 0.0 ? 0.0 : (1.0 < a ? 1.0 : a)) : 1.0);  // std::clamp(a, 0, 1)
  r.shader = t.shader;
  r.tu0 = float(t.tu0); r.tv0 = float(t.tv0);
  r.tu1 = float(t.tu1); r.tv1 = float(t.tv1);
  r.tu2 = float(t.tu2); r.tv2 = float(t.tv2);
  r.texture_offset = -1;
  r.texture_width = 0;
  r.texture_height = 0;
  out[o] = r;
  if (!(r.alpha >= 1.0f)) atomicAnd(flags, 0);  // flags[0]: 1 while every triangle is opaque
  if (light[g]) {
    const int j = lscan[g];
    light_tri[j] = o;
    weight[j] = light_weight(w);
  }
}

// counts[0..1] = triangles, lights (from the scans); total[0] = the emissive
// total, cdf its running values, summed left to right in double.
__global__ void k_prep_cdf(const int* __restrict__ keep, const int* __restrict__ kscan,
                           const int* __restrict__ light, const int* __restrict__ lscan, int total,
                           const double* __restrict__ weight, float* __restrict__ cdf, int* __restrict__ counts,
                           double* __restrict__ light_total) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int n_tris = total > 0 ? kscan[total - 1] + keep[total - 1] : 0;
  const int n_lights = total > 0 ? lscan[total - 1] + light[total - 1] : 0;
  double acc = 0.0;
  for (int j = 0; j < n_lights; ++j) {
    acc += weight[j];
    cdf[j] = float(acc);
  }
  counts[0] = n_tris;
  counts[1] = n_lights;
  light_total[0] = acc;
}

}  // namespace

cudaError_t prep_scan_bytes(int total, size_t& bytes) {
  bytes = exclusive_scan_temp_bytes(total > 0 ? total : 1);
  return cudaSuccess;
}

cudaError_t prep_world(const PrepArgs& a, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.flags, 0xFF, sizeof(int), st)) != cudaSuccess) return e;
  if (a.total > 0) {
    const unsigned g = unsigned((a.total + 255) / 256);
    k_prep_flags<<<g, 256, 0, st>>>(a.inst, a.mptr, a.start, a.n_inst, a.total, a.keep, a.light);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = exclusive_scan(a.keep, a.kscan, a.total, a.scan_temp, a.scan_bytes, st)) != cudaSuccess) return e;
    if ((e = exclusive_scan(a.light, a.lscan, a.total, a.scan_temp, a.scan_bytes, st)) != cudaSuccess) return e;
    k_prep_write<<<g, 256, 0, st>>>(a.inst, a.mptr, a.start, a.n_inst, a.total, a.keep, a.kscan, a.light, a.lscan,
                                    a.out, a.light_tri, a.weight, a.flags);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  k_prep_cdf<<<1, 1, 0, st>>>(a.keep, a.kscan, a.light, a.lscan, a.total, a.weight, a.cdf, a.counts, a.light_total);
  return cudaGetLastError();
}

}  // namespace rmd

// rm_bvh.cu - device BVH: caller-BVH conversion, LBVH build, refit, packing.
//
// The reference builds a binned-SAH binary BVH on the CPU in fp64
// (src/engine/bvh.cpp:29-248), refits it in reverse node order (:250-272),
// and its Metal backend flattens it to preorder escape-link nodes every frame
// (src/engine/metal.mm:129-144).  Here:
//  * a caller BVH in the reference layout is validated, converted to the
//    child-pair layout of rm_device.cuh on the host in O(nodes), and uploaded;
//  * without a caller BVH the device builds a linear BVH (Karras, "Maximizing
//    Parallelism in the Construction of BVHs, Octrees, and k-d Trees", HPG
//    2012): 30-bit Morton codes of the centroids, a radix sort (rm_sort.cu), one
//    thread per internal node to find its range and split, bottom-up boxes
//    with arrival counters; subtrees of at most `leaf_max` triangles collapse
//    into leaves;
//  * refit runs bottom-up on the device over the child-pair records with the
//    same arrival-counter scheme (one pass, no per-level launches).
// Triangle boxes come from the caller's fp32 vertices, so every box bounds its
// float triangle exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "rm_launch.h"
#include "rm_sort.h"

namespace rmd {

#define RM_TRY_(x)                         \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return e_;      \
  } while (0)


cudaError_t DevBuf::reserve(size_t bytes) {
  if (bytes <= cap && ptr) return cudaSuccess;
  if (ptr) { cudaFree(ptr); ptr = nullptr; cap = 0; }
  size_t want = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) { ptr = nullptr; return e; }
  cap = want;
  return cudaSuccess;
}
void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}

namespace {

struct Box { float mn[3], mx[3]; };

__device__ __forceinline__ Box tri_box(const rm_triangle& t) {
  Box b;
  b.mn[0] = fminf(t.v0.x, fminf(t.v1.x, t.v2.x)); b.mx[0] = fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x));
  b.mn[1] = fminf(t.v0.y, fminf(t.v1.y, t.v2.y)); b.mx[1] = fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y));
  b.mn[2] = fminf(t.v0.z, fminf(t.v1.z, t.v2.z)); b.mx[2] = fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z));
  return b;
}
__device__ __forceinline__ void grow(Box& a, const Box& b) {
  for (int k = 0; k < 3; ++k) { a.mn[k] = fminf(a.mn[k], b.mn[k]); a.mx[k] = fmaxf(a.mx[k], b.mx[k]); }
}
__device__ __forceinline__ Box empty_box() {
  Box b;
  for (int k = 0; k < 3; ++k) { b.mn[k] = __int_as_float(0x7f800000); b.mx[k] = -__int_as_float(0x7f800000); }
  return b;
}

// Slot boxes live in the first three float4 of a record (see rm_device.cuh).
__device__ __forceinline__ void write_slot(float4* rec, int slot, const Box& b) {
  float* f = reinterpret_cast<float*>(rec);
  if (slot == 0) { f[0] = b.mn[0]; f[1] = b.mx[0]; f[2] = b.mn[1]; f[3] = b.mx[1]; f[8] = b.mn[2]; f[9] = b.mx[2]; }
  else { f[4] = b.mn[0]; f[5] = b.mx[0]; f[6] = b.mn[1]; f[7] = b.mx[1]; f[10] = b.mn[2]; f[11] = b.mx[2]; }
}
__device__ __forceinline__ Box read_slot_cg(const float4* rec, int slot) {
  const float4 a = __ldcg(rec + slot), c = __ldcg(rec + 2);
  Box b;
  b.mn[0] = a.x; b.mx[0] = a.y; b.mn[1] = a.z; b.mx[1] = a.w;
  if (slot == 0) { b.mn[2] = c.x; b.mx[2] = c.y; } else { b.mn[2] = c.z; b.mx[2] = c.w; }
  return b;
}

__global__ void k_pack_tgeo(const rm_triangle* __restrict__ tris, const int32_t* __restrict__ order, int n,
                            float4* __restrict__ tgeo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = order[i];
  const rm_triangle& t = tris[j];
  tgeo[size_t(i) * 3 + 0] = make_float4(t.v0.x, t.v0.y, t.v0.z, __int_as_float(j));
  tgeo[size_t(i) * 3 + 1] = make_float4(t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z, 0.f);
  tgeo[size_t(i) * 3 + 2] = make_float4(t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z, 0.f);
}

// Refit: one thread per record; leaf slots are boxed from their triangles,
// then the last child to arrive at a record carries the union upward.
__global__ void k_refit(const rm_triangle* __restrict__ tris, const int32_t* __restrict__ order, float4* recs,
                        const int32_t* __restrict__ parents, int* counters, int n_records) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_records) return;
  float4* rec = recs + size_t(i) * 4;
  const int4 d = *reinterpret_cast<const int4*>(rec + 3);
  int ready = 0;
  for (int slot = 0; slot < 2; ++slot) {
    const int cnt = slot ? d.w : d.z, link = slot ? d.y : d.x;
    if (cnt < 0) { ++ready; continue; }
    if (cnt == 0) continue;
    Box b = empty_box();
    for (int k = 0; k < cnt; ++k) grow(b, tri_box(tris[order[link + k]]));
    write_slot(rec, slot, b);
    ++ready;
  }
  if (ready == 0) return;
  __threadfence();
  int node = i;
  int add = ready;
  for (;;) {
    const int old = atomicAdd(counters + node, add);
    if (old + add < 2) return;  // the other child is still on its way
    __threadfence();
    const int pr = parents[node];
    if (pr < 0) return;
    float4* nrec = recs + size_t(node) * 4;
    const int4 nd = __ldcg(reinterpret_cast<const int4*>(nrec + 3));
    Box b = empty_box();
    if (nd.z >= 0) grow(b, read_slot_cg(nrec, 0));
    if (nd.w >= 0) grow(b, read_slot_cg(nrec, 1));
    write_slot(recs + size_t(pr >> 1) * 4, pr & 1, b);
    __threadfence();
    node = pr >> 1;
    add = 1;
  }
}

// ---- LBVH -------------------------------------------------------------------

__device__ __forceinline__ unsigned int ordered(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned int u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_centroid_bounds(const rm_triangle* __restrict__ tris, int n, unsigned int* bounds) {
  unsigned int mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const rm_triangle& t = tris[i];
    const float c[3] = {t.v0.x + t.v1.x + t.v2.x, t.v0.y + t.v1.y + t.v2.y, t.v0.z + t.v1.z + t.v2.z};
    for (int k = 0; k < 3; ++k) { mn[k] = min(mn[k], ordered(c[k])); mx[k] = max(mx[k], ordered(c[k])); }
  }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o; o >>= 1) {
      mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) { atomicMin(bounds + k, mn[k]); atomicMax(bounds + 3 + k, mx[k]); }
}

__device__ __forceinline__ unsigned int expand_bits(unsigned int v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(const rm_triangle* __restrict__ tris, int n, const unsigned int* __restrict__ bounds,
                         unsigned int* __restrict__ keys, int* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rm_triangle& t = tris[i];
  const float c[3] = {t.v0.x + t.v1.x + t.v2.x, t.v0.y + t.v1.y + t.v2.y, t.v0.z + t.v1.z + t.v2.z};
  unsigned int q[3];
  for (int k = 0; k < 3; ++k) {
    const float lo = unordered(bounds[k]), hi = unordered(bounds[3 + k]);
    const float span = hi - lo;
    float f = span > 0.0f ? (c[k] - lo) / span : 0.5f;
    f = fminf(fmaxf(f, 0.0f), 1.0f);
    q[k] = min(unsigned(f * 1024.0f), 1023u);
  }
  keys[i] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
  vals[i] = i;
}

// Common-prefix length of keys i and j, with the sorted position breaking
// ties between equal codes (Karras 2012, section 4).
__device__ __forceinline__ int delta(const unsigned int* keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const unsigned int a = keys[i], b = keys[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz(unsigned(i) ^ unsigned(j));
}

// Internal node i of n-1: children encoded as (index << 1) | is_leaf; ranges.
__global__ void k_karras(const unsigned int* __restrict__ keys, int n, int2* __restrict__ children,
                         int2* __restrict__ ranges, int* __restrict__ parent_int, int* __restrict__ parent_leaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, n, i, j);
  int s = 0;
  for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if (t == 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int first = min(i, j), last = max(i, j);
  const int left = gamma, right = gamma + 1;
  const bool left_leaf = (first == gamma), right_leaf = (last == gamma + 1);
  children[i] = make_int2((left << 1) | int(left_leaf), (right << 1) | int(right_leaf));
  ranges[i] = make_int2(first, last);
  if (left_leaf) parent_leaf[left] = i; else parent_int[left] = i;
  if (right_leaf) parent_leaf[right] = i; else parent_int[right] = i;
}

// Boxes of the Karras tree, bottom-up from the leaves; the sorted triangle
// order is vals[].  kbox: (n-1) internal boxes.
__global__ void k_karras_boxes(const rm_triangle* __restrict__ tris, const int* __restrict__ order, int n,
                               const int2* __restrict__ children, const int* __restrict__ parent_int,
                               const int* __restrict__ parent_leaf, Box* kbox, int* kcount) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int node = parent_leaf[i];
  while (node >= 0) {
    __threadfence();
    if (atomicAdd(kcount + node, 1) == 0) return;  // first arrival waits for the sibling
    __threadfence();
    const int2 ch = children[node];
    Box b = empty_box();
    for (int k = 0; k < 2; ++k) {
      const int c = k ? ch.y : ch.x;
      if (c & 1) grow(b, tri_box(tris[order[c >> 1]]));
      else {
        const Box* src = kbox + (c >> 1);
        Box cb;
        for (int q = 0; q < 3; ++q) { cb.mn[q] = __ldcg(&src->mn[q]); cb.mx[q] = __ldcg(&src->mx[q]); }
        grow(b, cb);
      }
    }
    kbox[node] = b;
    node = node == 0 ? -1 : parent_int[node];
  }
}

// Child-pair records from the Karras tree: record index = Karras index;
// children with at most leaf_max triangles become leaves.
__global__ void k_emit_records(const rm_triangle* __restrict__ tris, const int* __restrict__ order, int n,
                               int leaf_max, const int2* __restrict__ children, const int2* __restrict__ ranges,
                               const Box* __restrict__ kbox, float4* recs, int* parents) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  float4* rec = recs + size_t(i) * 4;
  const int2 ch = children[i];
  int links[2], counts[2];
  for (int k = 0; k < 2; ++k) {
    const int c = k ? ch.y : ch.x;
    Box b;
    if (c & 1) {
      b = tri_box(tris[order[c >> 1]]);
      links[k] = c >> 1; counts[k] = 1;
    } else {
      const int2 r = ranges[c >> 1];
      b = kbox[c >> 1];
      const int size = r.y - r.x + 1;
      if (size <= leaf_max) { links[k] = r.x; counts[k] = size; }
      else { links[k] = c >> 1; counts[k] = 0; parents[c >> 1] = (i << 1) | k; }
    }
    write_slot(rec, k, b);
  }
  rec[3] = make_float4(__int_as_float(links[0]), __int_as_float(links[1]), __int_as_float(counts[0]),
                       __int_as_float(counts[1]));
  if (i == 0) parents[0] = -1;
}

// Depth of each leaf slot (for the traversal stack bound).
__global__ void k_depth(const float4* __restrict__ recs, const int* __restrict__ parents, int n_records, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_records) return;
  const int4 d = *reinterpret_cast<const int4*>(recs + size_t(i) * 4 + 3);
  if (d.z <= 0 && d.w <= 0) return;
  int depth = 1, node = i, guard = 0;
  while (parents[node] >= 0 && guard < 4096) { node = parents[node] >> 1; ++depth; ++guard; }
  atomicMax(out, depth);
}

__global__ void k_single_leaf(const rm_triangle* __restrict__ tris, int n, float4* rec, int* parents, int* order) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Box b = empty_box();
  for (int i = 0; i < n; ++i) { grow(b, tri_box(tris[i])); order[i] = i; }
  write_slot(rec, 0, b);
  write_slot(rec, 1, empty_box());
  rec[3] = make_float4(__int_as_float(0), __int_as_float(0), __int_as_float(n), __int_as_float(-1));
  parents[0] = -1;
}

__global__ void k_hash(const unsigned long long* __restrict__ w, size_t n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    unsigned long long z = w[i] ^ (0x9E3779B97F4A7C15ull * (i + 1));
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    acc += z ^ (z >> 31);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// flag[0] |= 1 where the two word arrays differ.
__global__ void k_differ(const uint4* __restrict__ a, const uint4* __restrict__ b, size_t n, int* flag) {
  bool d = false;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const uint4 x = a[i], y = b[i];
    d |= (x.x != y.x) | (x.y != y.y) | (x.z != y.z) | (x.w != y.w);
  }
  if (__any_sync(0xffffffffu, d) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

__global__ void k_light_records(const rm_triangle* __restrict__ tris, const int32_t* __restrict__ lights, int n,
                                float4* __restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const rm_triangle& t = tris[lights[i]];
  rec[size_t(i) * 4 + 0] = make_float4(t.v0.x, t.v0.y, t.v0.z, t.er);
  rec[size_t(i) * 4 + 1] = make_float4(t.v1.x, t.v1.y, t.v1.z, t.eg);
  rec[size_t(i) * 4 + 2] = make_float4(t.v2.x, t.v2.y, t.v2.z, t.eb);
  rec[size_t(i) * 4 + 3] = make_float4(t.nn.x, t.nn.y, t.nn.z, t.alpha);
}

// guide[g] = first index with cdf >= g * step (the last index if none);
// guide[G] = L - 1.
__global__ void k_light_guide(const float* __restrict__ cdf, int L, int G, float step, int32_t* __restrict__ guide) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > G) return;
  if (g == G) { guide[g] = L - 1; return; }
  const float th = float(g) * step;
  int lo = 0, hi = L - 1;
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (cdf[mid] >= th) hi = mid; else lo = mid + 1;
  }
  guide[g] = lo;
}

}  // namespace

cudaError_t prepare_lights(const rm_triangle* d_tris, const int32_t* d_lights, const float* d_cdf, int n_lights,
                           float light_total, DevBuf& rec, DevBuf& guide, int& guide_n, float& guide_inv,
                           cudaStream_t st) {
  guide_n = 0;
  guide_inv = 0.0f;
  if (n_lights <= 0 || !(light_total > 1e-12f)) return cudaSuccess;
  RM_TRY_(rec.reserve(size_t(n_lights) * 4 * sizeof(float4)));
  k_light_records<<<(n_lights + 255) / 256, 256, 0, st>>>(d_tris, d_lights, n_lights, rec.as<float4>());
  int G = 1;
  while (G < n_lights && G < 65536) G <<= 1;
  RM_TRY_(guide.reserve(size_t(G + 1) * sizeof(int32_t)));
  const float step = light_total / float(G);
  k_light_guide<<<(G + 1 + 255) / 256, 256, 0, st>>>(d_cdf, n_lights, G, step, guide.as<int32_t>());
  guide_n = G;
  guide_inv = float(G) / light_total;
  return cudaGetLastError();
}

namespace {

}  // namespace

cudaError_t pack_tgeo(const rm_triangle* d_tris, DevBvh& bvh, cudaStream_t st) {
  if (bvh.n_tris <= 0) return cudaSuccess;
  cudaError_t e = bvh.tgeo.reserve(size_t(bvh.n_tris) * 3 * sizeof(float4));
  if (e != cudaSuccess) return e;
  k_pack_tgeo<<<(bvh.n_tris + 255) / 256, 256, 0, st>>>(d_tris, bvh.order.as<int32_t>(), bvh.n_tris,
                                                       bvh.tgeo.as<float4>());
  return cudaGetLastError();
}

cudaError_t refit_bvh(const rm_triangle* d_tris, DevBvh& bvh, cudaStream_t st) {
  if (bvh.n_records <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(bvh.counters.ptr, 0, size_t(bvh.n_records) * sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_refit<<<(bvh.n_records + 255) / 256, 256, 0, st>>>(d_tris, bvh.order.as<int32_t>(), bvh.records.as<float4>(),
                                                       bvh.parents.as<int32_t>(), bvh.counters.as<int>(),
                                                       bvh.n_records);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return pack_tgeo(d_tris, bvh, st);
}

cudaError_t device_differ(const void* a, const void* b, size_t n_bytes, int* d_flag, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_flag, 0, sizeof(int), st);
  if (e != cudaSuccess || n_bytes == 0) return e;
  if (n_bytes % 16) return cudaErrorInvalidValue;
  k_differ<<<148 * 4, 256, 0, st>>>(static_cast<const uint4*>(a), static_cast<const uint4*>(b), n_bytes / 16, d_flag);
  return cudaGetLastError();
}

cudaError_t device_hash(const void* d_bytes, size_t n_bytes, unsigned long long* d_out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  size_t words = n_bytes / 8;
  if (words == 0) return cudaSuccess;
  k_hash<<<148 * 4, 256, 0, st>>>(static_cast<const unsigned long long*>(d_bytes), words, d_out);
  return cudaGetLastError();
}

#define RM_TRY(x)                          \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return e_;      \
  } while (0)

cudaError_t build_lbvh(const rm_triangle* d_tris, int n, int leaf_max, DevBvh& b, cudaStream_t st, std::string& err) {
  b.n_tris = n;
  b.max_depth = 0;
  if (n <= 0) { b.n_records = 0; return cudaSuccess; }
  leaf_max = std::max(1, std::min(leaf_max, kMaxLeaf));
  if (n >= kMaxLink) { err = "scene exceeds 16777215 triangles"; return cudaErrorInvalidValue; }
  RM_TRY(b.order.reserve(size_t(n) * sizeof(int)));
  if (n <= leaf_max) {
    b.n_records = 1;
    RM_TRY(b.records.reserve(4 * sizeof(float4)));
    RM_TRY(b.parents.reserve(sizeof(int)));
    RM_TRY(b.counters.reserve(sizeof(int)));
    k_single_leaf<<<1, 1, 0, st>>>(d_tris, n, b.records.as<float4>(), b.parents.as<int>(), b.order.as<int>());
    RM_TRY(cudaGetLastError());
    b.max_depth = 1;
    return pack_tgeo(d_tris, b, st);
  }
  const int ni = n - 1;
  RM_TRY(b.bounds.reserve(6 * sizeof(unsigned int)));
  RM_TRY(b.keys.reserve(size_t(n) * 4 * 2));
  RM_TRY(b.keys_alt.reserve(size_t(n) * 4));
  RM_TRY(b.vals_alt.reserve(size_t(n) * 4));
  RM_TRY(b.knodes.reserve(size_t(ni) * sizeof(int2) * 2));  // children + ranges
  RM_TRY(b.ranges.reserve(size_t(ni) * sizeof(int) + size_t(n) * sizeof(int)));  // parent_int + parent_leaf
  RM_TRY(b.kbox.reserve(size_t(ni) * sizeof(Box)));
  RM_TRY(b.kcount.reserve(size_t(ni) * sizeof(int)));
  RM_TRY(b.records.reserve(size_t(ni) * 4 * sizeof(float4)));
  RM_TRY(b.parents.reserve(size_t(ni) * sizeof(int)));
  RM_TRY(b.counters.reserve(size_t(ni) * sizeof(int)));
  RM_TRY(b.depth.reserve(sizeof(int)));
  unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  RM_TRY(cudaMemcpyAsync(b.bounds.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_centroid_bounds<<<148 * 4, 256, 0, st>>>(d_tris, n, b.bounds.as<unsigned int>());
  unsigned int* keys = b.keys.as<unsigned int>();
  int* vals = reinterpret_cast<int*>(keys + n);
  k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_tris, n, b.bounds.as<unsigned int>(), keys, vals);
  RM_TRY(cudaGetLastError());
  const size_t temp_bytes = radix_sort_temp_bytes(n);
  RM_TRY(b.temp.reserve(temp_bytes));
  bool in_alt = false;
  RM_TRY(radix_sort_pairs(keys, b.keys_alt.as<unsigned int>(), vals, b.vals_alt.as<int>(), n, 30, b.temp.ptr,
                          temp_bytes, in_alt, st));
  const unsigned int* skeys = in_alt ? b.keys_alt.as<unsigned int>() : keys;
  const int* sorder = in_alt ? b.vals_alt.as<int>() : vals;
  RM_TRY(cudaMemcpyAsync(b.order.ptr, sorder, size_t(n) * sizeof(int), cudaMemcpyDeviceToDevice, st));
  int2* children = b.knodes.as<int2>();
  int2* ranges = children + ni;
  int* parent_int = b.ranges.as<int>();
  int* parent_leaf = parent_int + ni;
  RM_TRY(cudaMemsetAsync(parent_int, 0xff, size_t(ni) * sizeof(int), st));
  k_karras<<<(ni + 255) / 256, 256, 0, st>>>(skeys, n, children, ranges, parent_int, parent_leaf);
  RM_TRY(cudaMemsetAsync(b.kcount.ptr, 0, size_t(ni) * sizeof(int), st));
  k_karras_boxes<<<(n + 255) / 256, 256, 0, st>>>(d_tris, b.order.as<int>(), n, children, parent_int, parent_leaf,
                                                  b.kbox.as<Box>(), b.kcount.as<int>());
  RM_TRY(cudaMemsetAsync(b.parents.ptr, 0xff, size_t(ni) * sizeof(int), st));
  k_emit_records<<<(ni + 255) / 256, 256, 0, st>>>(d_tris, b.order.as<int>(), n, leaf_max, children, ranges,
                                                   b.kbox.as<Box>(), b.records.as<float4>(), b.parents.as<int>());
  RM_TRY(cudaGetLastError());
  b.n_records = ni;
  // Records of subtrees that collapsed into a leaf are never reached from the
  // root; they keep parent -1, so refit ends at them and depth counts them as 1.
  RM_TRY(cudaMemsetAsync(b.depth.ptr, 0, sizeof(int), st));
  k_depth<<<(ni + 255) / 256, 256, 0, st>>>(b.records.as<float4>(), b.parents.as<int>(), ni, b.depth.as<int>());
  RM_TRY(cudaMemcpyAsync(&b.max_depth, b.depth.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  RM_TRY(cudaStreamSynchronize(st));
  if (b.max_depth > kStack) { err = "device BVH deeper than the traversal stack"; return cudaErrorInvalidValue; }
  return pack_tgeo(d_tris, b, st);
}

cudaError_t build_lbvh_into(const rm_triangle* d_tris, int n, int leaf_max, const LbvhScratch& w, DevBvhView& out,
                            cudaStream_t st, std::string& err) {
  out.n_records = 0;
  // The error word lives in scratch shared by every call: clear it before any
  // early return, or an empty scene would report the last call's overflow.
  RM_TRY(cudaMemsetAsync(w.err_word, 0, sizeof(uint32_t), st));
  if (n <= 0) return cudaSuccess;
  leaf_max = std::max(1, std::min(leaf_max, kMaxLeaf));
  if (n <= leaf_max) {
    k_single_leaf<<<1, 1, 0, st>>>(d_tris, n, w.records, w.parents, w.order);
    RM_TRY(cudaGetLastError());
    out.n_records = 1;
  } else {
    const int ni = n - 1;
    // centroid bounds start at (+max ordered, 0): min slots all ones, max slots zero
    RM_TRY(cudaMemsetAsync(w.bounds, 0xff, 3 * sizeof(unsigned int), st));
    RM_TRY(cudaMemsetAsync(w.bounds + 3, 0, 3 * sizeof(unsigned int), st));
    k_centroid_bounds<<<148 * 4, 256, 0, st>>>(d_tris, n, w.bounds);
    k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_tris, n, w.bounds, w.keys, w.vals);
    RM_TRY(cudaGetLastError());
    if (radix_sort_temp_bytes(n) > w.sort_temp_bytes) { err = "sort scratch too small"; return cudaErrorInvalidValue; }
    bool in_alt = false;
    RM_TRY(radix_sort_pairs(w.keys, w.keys_alt, w.vals, w.vals_alt, n, 30, w.sort_temp, w.sort_temp_bytes, in_alt,
                            st));
    RM_TRY(cudaMemcpyAsync(w.order, in_alt ? w.vals_alt : w.vals, size_t(n) * sizeof(int), cudaMemcpyDeviceToDevice,
                           st));
    RM_TRY(cudaMemsetAsync(w.parent_int, 0xff, size_t(ni) * sizeof(int), st));
    k_karras<<<(ni + 255) / 256, 256, 0, st>>>(in_alt ? w.keys_alt : w.keys, n, w.children, w.ranges, w.parent_int,
                                               w.parent_leaf);
    RM_TRY(cudaMemsetAsync(w.kcount, 0, size_t(ni) * sizeof(int), st));
    k_karras_boxes<<<(n + 255) / 256, 256, 0, st>>>(d_tris, w.order, n, w.children, w.parent_int, w.parent_leaf,
                                                    reinterpret_cast<Box*>(w.kbox), w.kcount);
    RM_TRY(cudaMemsetAsync(w.parents, 0xff, size_t(ni) * sizeof(int), st));
    k_emit_records<<<(ni + 255) / 256, 256, 0, st>>>(d_tris, w.order, n, leaf_max, w.children, w.ranges,
                                                     reinterpret_cast<const Box*>(w.kbox), w.records, w.parents);
    RM_TRY(cudaGetLastError());
    out.n_records = ni;
  }
  k_pack_tgeo<<<(n + 255) / 256, 256, 0, st>>>(d_tris, w.order, n, w.tgeo);
  RM_TRY(cudaGetLastError());
  out.records = w.records;
  out.tgeo = w.tgeo;
  return cudaSuccess;
}

size_t lbvh_box_bytes() { return sizeof(Box); }

// ---- PLOC ---------------------------------------------------------------------
//
// Meister & Bittner, "Parallel Locally-Ordered Clustering for Bounding Volume
// Hierarchy Construction" (IEEE TVCG 2018).  Clusters start as the triangles in
// Morton order; every iteration each cluster finds, within a window of
// +-kPlocRadius neighbours in that order, the cluster whose union box has the
// smallest surface area; mutual nearest neighbours merge into a new node, and
// the survivors are compacted in order.  Node ids: leaves 0..n-1 (Morton
// position), internal nodes n.. in creation order, so a parent's id is larger
// than its children's.  The tree is then laid out like the LBVH: leaves in
// depth-first order, subtrees of at most `leaf_max` triangles as leaves, one
// child-pair record per remaining internal node (record of node k is
// 2n-2-k, the root is record 0).

namespace {

constexpr int kPlocRadius = 16;

__device__ __forceinline__ float half_area(const float4& lo, const float4& hi) {
  const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  return dx * dy + dy * dz + dz * dx;
}

__global__ void k_ploc_leaves(const rm_triangle* __restrict__ tris, const int* __restrict__ order, int n,
                              float4* __restrict__ blo, float4* __restrict__ bhi, int* __restrict__ cl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Box b = tri_box(tris[order[i]]);
  blo[i] = make_float4(b.mn[0], b.mn[1], b.mn[2], __int_as_float(1));
  bhi[i] = make_float4(b.mx[0], b.mx[1], b.mx[2], __int_as_float(-1));
  cl[i] = i;
}

__global__ void k_ploc_nn(const int* __restrict__ cl, int C, const float4* __restrict__ blo,
                          const float4* __restrict__ bhi, int* __restrict__ nn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C) return;
  const int a = cl[i];
  const float4 alo = blo[a], ahi = bhi[a];
  float best = __int_as_float(0x7f800000);
  int bj = -1;
  const int j0 = max(0, i - kPlocRadius), j1 = min(C - 1, i + kPlocRadius);
  for (int j = j0; j <= j1; ++j) {
    if (j == i) continue;
    const int b = cl[j];
    const float4 l = blo[b], h = bhi[b];
    const float4 ulo = make_float4(fminf(alo.x, l.x), fminf(alo.y, l.y), fminf(alo.z, l.z), 0.f);
    const float4 uhi = make_float4(fmaxf(ahi.x, h.x), fmaxf(ahi.y, h.y), fmaxf(ahi.z, h.z), 0.f);
    const float area = half_area(ulo, uhi);
    if (area < best) { best = area; bj = j; }  // ties keep the smaller index (scanned in order)
  }
  nn[i] = bj;
}

// flags: x = this cluster creates a node, y = this cluster survives
__global__ void k_ploc_flags(const int* __restrict__ nn, int C, int force, int* __restrict__ mflag,
                             int* __restrict__ kflag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C) return;
  int j = nn[i];
  bool mutual = j >= 0 && nn[j] == i;
  if (force) {  // no mutual pair anywhere: merge neighbours (0,1), (2,3), ...
    j = (i & 1) ? i - 1 : i + 1;
    mutual = j < C;
  }
  mflag[i] = (mutual && i < j) ? 1 : 0;
  kflag[i] = (!mutual || i < j) ? 1 : 0;
}

__global__ void k_ploc_apply(const int* __restrict__ cl, const int* __restrict__ nn, int C, int force,
                             const int* __restrict__ mflag, const int* __restrict__ mscan,
                             const int* __restrict__ kflag, const int* __restrict__ kscan, int next_node,
                             float4* __restrict__ blo, float4* __restrict__ bhi, int2* __restrict__ child,
                             int* __restrict__ ncl, int n_leaves) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= C) return;
  if (!kflag[i]) return;
  int out = cl[i];
  if (mflag[i]) {
    const int j = force ? i + 1 : nn[i];
    const int a = cl[i], b = cl[j];
    const int id = next_node + mscan[i];
    const float4 al = blo[a], ah = bhi[a], bl = blo[b], bh = bhi[b];
    const int size = __float_as_int(al.w) + __float_as_int(bl.w);
    blo[id] = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), __int_as_float(size));
    bhi[id] = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), __int_as_float(-1));
    child[id - n_leaves] = make_int2(a, b);
    bhi[a].w = __int_as_float(id);  // parent links
    bhi[b].w = __int_as_float(id);
    out = id;
  }
  ncl[kscan[i]] = out;
}

__global__ void k_ploc_totals(const int* __restrict__ mflag, const int* __restrict__ mscan,
                              const int* __restrict__ kflag, const int* __restrict__ kscan, int C,
                              int* __restrict__ totals) {
  totals[0] = mscan[C - 1] + mflag[C - 1];
  totals[1] = kscan[C - 1] + kflag[C - 1];
}

// Leaf position in depth-first order and depth: walk to the root adding the
// sizes of left siblings.  Only the n leaves walk; max depth -> *depth.
__global__ void k_ploc_layout(int n, int root, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                              const int2* __restrict__ child, const int* __restrict__ order, int* __restrict__ pos,
                              int* __restrict__ out_order, int* __restrict__ depth) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int off = 0, d = 1, cur = i;
  while (cur != root) {
    const int p = __float_as_int(bhi[cur].w);
    const int2 c = child[p - n];
    if (c.y == cur) off += __float_as_int(blo[c.x].w);
    cur = p;
    ++d;
    if (d > 4 * kStack) break;  // a corrupt tree cannot loop forever
  }
  pos[i] = off;
  out_order[off] = order[i];
  atomicMax(depth, d);
}

// Depth-first (pre-order) record index of each internal node among the
// internal nodes: one slot per ancestor, plus the internal nodes of every left
// sibling's subtree on the way up (a subtree of s leaves has s - 1).  The
// nearer child of a descent then usually sits in the next record.
__global__ void k_ploc_preorder(int n, int root, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                const int2* __restrict__ child, int* __restrict__ pre) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;  // internal node n + k
  if (k >= n - 1) return;
  int off = 0, d = 0, cur = n + k;
  while (cur != root) {
    const int p = __float_as_int(bhi[cur].w);
    const int2 c = child[p - n];
    off += 1;
    if (c.y == cur) off += __float_as_int(blo[c.x].w) - 1;
    cur = p;
    if (++d > 4 * kStack) break;  // a corrupt tree cannot loop forever
  }
  pre[k] = off;
}

__device__ __forceinline__ int ploc_first(int node, int n, const int2* __restrict__ child,
                                          const int* __restrict__ pos) {
  while (node >= n) node = child[node - n].x;
  return pos[node];
}

__global__ void k_ploc_emit(int n, int leaf_max, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                            const int2* __restrict__ child, const int* __restrict__ pos, const int* __restrict__ pre,
                            float4* recs, int* parents) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;  // internal node n + k
  if (k >= n - 1) return;
  const int node = n + k;
  const int rec_id = pre[k];
  float4* rec = recs + size_t(rec_id) * 4;
  if (__float_as_int(blo[node].w) <= leaf_max) {
    // collapsed into an ancestor's leaf: an unreachable record
    write_slot(rec, 0, empty_box());
    write_slot(rec, 1, empty_box());
    rec[3] = make_float4(__int_as_float(0), __int_as_float(0), __int_as_float(-1), __int_as_float(-1));
    parents[rec_id] = -1;
    return;
  }
  const int2 ch = child[k];
  int links[2], counts[2];
  for (int s = 0; s < 2; ++s) {
    const int c = s ? ch.y : ch.x;
    const float4 l = blo[c], h = bhi[c];
    Box b;
    b.mn[0] = l.x; b.mn[1] = l.y; b.mn[2] = l.z;
    b.mx[0] = h.x; b.mx[1] = h.y; b.mx[2] = h.z;
    write_slot(rec, s, b);
    const int size = __float_as_int(l.w);
    if (size <= leaf_max) {
      links[s] = ploc_first(c, n, child, pos);
      counts[s] = size;
    } else {
      links[s] = pre[c - n];
      counts[s] = 0;
      parents[links[s]] = (rec_id << 1) | s;
    }
  }
  rec[3] = make_float4(__int_as_float(links[0]), __int_as_float(links[1]), __int_as_float(counts[0]),
                       __int_as_float(counts[1]));
  if (rec_id == 0) parents[0] = -1;
}

}  // namespace

cudaError_t build_ploc(const rm_triangle* d_tris, int n, int leaf_max, DevBvh& b, cudaStream_t st, std::string& err) {
  b.n_tris = n;
  b.max_depth = 0;
  if (n <= 0) { b.n_records = 0; return cudaSuccess; }
  leaf_max = std::max(1, std::min(leaf_max, kMaxLeaf));
  if (n <= leaf_max) return build_lbvh(d_tris, n, leaf_max, b, st, err);  // one leaf
  if (n >= kMaxLink / 2) { err = "scene exceeds 8388607 triangles for the clustering build"; return cudaErrorInvalidValue; }
  const int total = 2 * n - 1;
  // Morton order (shared with the LBVH build)
  RM_TRY(b.order.reserve(size_t(n) * sizeof(int)));
  RM_TRY(b.bounds.reserve(6 * sizeof(unsigned int)));
  RM_TRY(b.keys.reserve(size_t(n) * 4 * 2));
  RM_TRY(b.keys_alt.reserve(size_t(n) * 4));
  RM_TRY(b.vals_alt.reserve(size_t(n) * 4));
  unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  RM_TRY(cudaMemcpyAsync(b.bounds.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_centroid_bounds<<<148 * 4, 256, 0, st>>>(d_tris, n, b.bounds.as<unsigned int>());
  unsigned int* keys = b.keys.as<unsigned int>();
  int* vals = reinterpret_cast<int*>(keys + n);
  k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_tris, n, b.bounds.as<unsigned int>(), keys, vals);
  RM_TRY(cudaGetLastError());
  const size_t sort_bytes = radix_sort_temp_bytes(n), scan_bytes = exclusive_scan_temp_bytes(n);
  RM_TRY(b.temp.reserve(std::max(sort_bytes, scan_bytes)));
  bool in_alt = false;
  RM_TRY(radix_sort_pairs(keys, b.keys_alt.as<unsigned int>(), vals, b.vals_alt.as<int>(), n, 30, b.temp.ptr,
                          sort_bytes, in_alt, st));
  const int* sorted = in_alt ? b.vals_alt.as<int>() : vals;
  // node and cluster arrays (kbox: box lo/hi; knodes: children; ranges: 2 cluster lists + nn + 4 flag arrays)
  RM_TRY(b.kbox.reserve(size_t(total) * 2 * sizeof(float4)));
  RM_TRY(b.knodes.reserve(size_t(n) * sizeof(int2)));
  RM_TRY(b.ranges.reserve(size_t(n) * 7 * sizeof(int) + 2 * sizeof(int)));
  RM_TRY(b.kcount.reserve(size_t(n) * sizeof(int)));
  float4* blo = b.kbox.as<float4>();
  float4* bhi = blo + total;
  int2* child = b.knodes.as<int2>();
  int* cl0 = b.ranges.as<int>();
  int* cl1 = cl0 + n;
  int* nn = cl1 + n;
  int* mflag = nn + n;
  int* mscan = mflag + n;
  int* kflag = mscan + n;
  int* kscan = kflag + n;
  int* totals = kscan + n;
  k_ploc_leaves<<<(n + 255) / 256, 256, 0, st>>>(d_tris, sorted, n, blo, bhi, cl0);
  RM_TRY(cudaGetLastError());
  int C = n, next_node = n, iters = 0;
  int* cl = cl0;
  int* ncl = cl1;
  int h_tot[2];
  while (C > 1) {
    if (++iters > 4 * n + 64) { err = "clustering build did not converge"; return cudaErrorInvalidValue; }
    const unsigned g = unsigned((C + 255) / 256);
    int force = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      if (!force) k_ploc_nn<<<g, 256, 0, st>>>(cl, C, blo, bhi, nn);
      k_ploc_flags<<<g, 256, 0, st>>>(nn, C, force, mflag, kflag);
      RM_TRY(exclusive_scan(mflag, mscan, C, b.temp.ptr, scan_bytes, st));
      RM_TRY(exclusive_scan(kflag, kscan, C, b.temp.ptr, scan_bytes, st));
      k_ploc_totals<<<1, 1, 0, st>>>(mflag, mscan, kflag, kscan, C, totals);
      RM_TRY(cudaMemcpyAsync(h_tot, totals, sizeof(h_tot), cudaMemcpyDeviceToHost, st));
      RM_TRY(cudaStreamSynchronize(st));
      if (h_tot[0] > 0) break;
      force = 1;  // degenerate input: pair up neighbours
    }
    k_ploc_apply<<<g, 256, 0, st>>>(cl, nn, C, force, mflag, mscan, kflag, kscan, next_node, blo, bhi, child, ncl, n);
    RM_TRY(cudaGetLastError());
    next_node += h_tot[0];
    C = h_tot[1];
    std::swap(cl, ncl);
  }
  const int root = next_node - 1;
  if (root != total - 1) { err = "clustering build produced a malformed tree"; return cudaErrorInvalidValue; }
  // layout
  int* pos = b.kcount.as<int>();
  RM_TRY(b.depth.reserve(sizeof(int)));
  RM_TRY(cudaMemsetAsync(b.depth.ptr, 0, sizeof(int), st));
  k_ploc_layout<<<(n + 255) / 256, 256, 0, st>>>(n, root, blo, bhi, child, sorted, pos, b.order.as<int>(),
                                                 b.depth.as<int>());
  int* pre = nn;  // the cluster arrays are free once the tree is built
  k_ploc_preorder<<<(n - 1 + 255) / 256, 256, 0, st>>>(n, root, blo, bhi, child, pre);
  RM_TRY(b.records.reserve(size_t(n - 1) * 4 * sizeof(float4)));
  RM_TRY(b.parents.reserve(size_t(n - 1) * sizeof(int)));
  RM_TRY(b.counters.reserve(size_t(n - 1) * sizeof(int)));
  k_ploc_emit<<<(n - 1 + 255) / 256, 256, 0, st>>>(n, leaf_max, blo, bhi, child, pos, pre, b.records.as<float4>(),
                                                   b.parents.as<int>());
  RM_TRY(cudaGetLastError());
  RM_TRY(cudaMemcpyAsync(&b.max_depth, b.depth.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  RM_TRY(cudaStreamSynchronize(st));
  if (b.max_depth > kStack) { err = "device BVH deeper than the traversal stack"; return cudaErrorInvalidValue; }
  b.n_records = n - 1;
  return pack_tgeo(d_tris, b, st);
}

bool convert_caller_bvh(const rm_bvh_node* nodes, int M, const int32_t* bvh_tri, int n_tris, DevBvh& out,
                        cudaStream_t st, std::string& err) {
  out.n_tris = n_tris;
  if (M <= 0 || n_tris <= 0) { out.n_records = 0; return true; }
  if (!nodes || !bvh_tri) { err = "BVH nodes without bvh_tri"; return false; }
  if (n_tris >= kMaxLink || M >= kMaxLink) { err = "BVH exceeds 16777215 nodes or triangles"; return false; }
  for (int i = 0; i < n_tris; ++i)
    if (bvh_tri[i] < 0 || bvh_tri[i] >= n_tris) { err = "bvh_tri index out of range"; return false; }
  // record index of each internal node, in node order (parents precede children)
  std::vector<int> rec(size_t(M), -1);
  int n_rec = 0;
  for (int i = 0; i < M; ++i) {
    const rm_bvh_node& s = nodes[i];
    if (s.count > 0) {
      if (s.count > kMaxLeaf || s.offset < 0 || int64_t(s.offset) + s.count > n_tris) {
        err = "BVH leaf range invalid (or more than 255 triangles)";
        return false;
      }
    } else {
      if (s.left <= i || s.right <= i || s.left >= M || s.right >= M) {
        err = "BVH child index invalid (children must follow their parent)";
        return false;
      }
      rec[size_t(i)] = n_rec++;
    }
  }
  const bool root_leaf = nodes[0].count > 0;
  if (root_leaf) n_rec = 1;
  std::vector<float> recs(size_t(n_rec) * 16, 0.0f);
  std::vector<int> parents(size_t(n_rec), -1);
  std::vector<int> depth(size_t(M), 0);
  auto put = [&](int r, int slot, const rm_bvh_node* c, int link, int count) {
    float* f = recs.data() + size_t(r) * 16;
    const float inf = __builtin_inff();
    float mn[3] = {inf, inf, inf}, mx[3] = {-inf, -inf, -inf};
    if (c) { mn[0] = c->mn.x; mn[1] = c->mn.y; mn[2] = c->mn.z; mx[0] = c->mx.x; mx[1] = c->mx.y; mx[2] = c->mx.z; }
    int base = slot ? 4 : 0;
    f[base] = mn[0]; f[base + 1] = mx[0]; f[base + 2] = mn[1]; f[base + 3] = mx[1];
    f[8 + slot * 2] = mn[2]; f[9 + slot * 2] = mx[2];
    int* iv = reinterpret_cast<int*>(f + 12);
    iv[slot] = link;
    iv[2 + slot] = count;
  };
  int max_depth = 1;
  if (root_leaf) {
    put(0, 0, &nodes[0], nodes[0].offset, nodes[0].count);
    put(0, 1, nullptr, 0, -1);
  } else {
    depth[0] = 1;
    for (int i = 0; i < M; ++i) {
      if (nodes[i].count > 0 || rec[size_t(i)] < 0) continue;
      const int r = rec[size_t(i)];
      if (depth[size_t(i)] == 0) continue;  // unreachable from the root
      for (int slot = 0; slot < 2; ++slot) {
        const int c = slot ? nodes[i].right : nodes[i].left;
        const rm_bvh_node& cn = nodes[c];
        depth[size_t(c)] = depth[size_t(i)] + 1;
        max_depth = std::max(max_depth, depth[size_t(c)]);
        if (cn.count > 0) put(r, slot, &cn, cn.offset, cn.count);
        else {
          put(r, slot, &cn, rec[size_t(c)], 0);
          parents[size_t(rec[size_t(c)])] = (r << 1) | slot;
        }
      }
    }
    // an unreachable internal node keeps an all-empty record
    for (int i = 0; i < M; ++i)
      if (rec[size_t(i)] >= 0 && depth[size_t(i)] == 0) {
        put(rec[size_t(i)], 0, nullptr, 0, -1);
        put(rec[size_t(i)], 1, nullptr, 0, -1);
      }
  }
  if (max_depth > kStack) { err = "BVH deeper than 64 levels"; return false; }
  out.max_depth = max_depth;
  out.n_records = n_rec;
  cudaError_t e;
  if ((e = out.records.reserve(recs.size() * sizeof(float))) != cudaSuccess ||
      (e = out.parents.reserve(parents.size() * sizeof(int))) != cudaSuccess ||
      (e = out.counters.reserve(parents.size() * sizeof(int))) != cudaSuccess ||
      (e = out.order.reserve(size_t(n_tris) * sizeof(int))) != cudaSuccess) {
    err = std::string("BVH allocation failed: ") + cudaGetErrorString(e);
    return false;
  }
  if ((e = cudaMemcpyAsync(out.records.ptr, recs.data(), recs.size() * sizeof(float), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaMemcpyAsync(out.parents.ptr, parents.data(), parents.size() * sizeof(int), cudaMemcpyHostToDevice,
                           st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(out.order.ptr, bvh_tri, size_t(n_tris) * sizeof(int), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess) {
    err = std::string("BVH upload failed: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

}  // namespace rmd

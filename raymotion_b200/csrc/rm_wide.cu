// rm_wide.cu - 8-wide compressed BVH from the binary child-pair BVH.
//
// The reference traverses a binary BVH (pathtrace.metal:137-161).  On a GPU
// without ray-tracing cores, traversal is bound by the latency of dependent
// node fetches, so fewer, wider nodes per ray pay: this pass collapses the
// device-built binary BVH (rm_bvh.cu) into nodes of up to 8 children with
// 8-bit quantized boxes, 80 bytes each (the node format and traversal are in
// rm_device.cuh, WTrav; the scheme follows Ylitie, Karras and Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs",
// HPG 2017).
//
// Top-down, one frontier level per launch: a wide node starts from the two
// children of a binary node and repeatedly opens the internal child with the
// largest surface area until it has 8 children or only leaves (leaves hold at
// most 4 triangles, the count field's range).  Its internal children get
// consecutive node indices, its leaves' triangles consecutive records
// (copied from the binary order), and its children take slots by the octant of
// their centre around the node's centre (a greedy assignment), so that a ray
// visits slots in near-to-far order by XOR with its direction's octant.
// Quantized boxes are rounded outward and then checked with the traversal's
// own dequantization expression, so every dequantized box contains its true
// box: hits stay bit for bit those of the binary BVH.
#include <cuda_runtime.h>

#include <utility>

#include "rm_device.cuh"
#include "rm_launch.h"

namespace rmd {

namespace {

struct Child {
  float lo[3], hi[3];
  int link, cnt;  // cnt > 0: leaf of cnt triangles from record link; 0: binary node link
};

__device__ __forceinline__ void read_children(const float4* __restrict__ rec, int r, Child* out, int& n) {
  const float4* q = rec + size_t(r) * 4;
  const float4 a = q[0], b = q[1], c = q[2];
  const int4 d = *reinterpret_cast<const int4*>(q + 3);
  if (d.z >= 0) {
    Child& ch = out[n++];
    ch.lo[0] = a.x; ch.hi[0] = a.y; ch.lo[1] = a.z; ch.hi[1] = a.w; ch.lo[2] = c.x; ch.hi[2] = c.y;
    ch.link = d.x; ch.cnt = d.z;
  }
  if (d.w >= 0) {
    Child& ch = out[n++];
    ch.lo[0] = b.x; ch.hi[0] = b.y; ch.lo[1] = b.z; ch.hi[1] = b.w; ch.lo[2] = c.z; ch.hi[2] = c.w;
    ch.link = d.y; ch.cnt = d.w;
  }
}

__device__ __forceinline__ float half_area(const Child& c) {
  const float ex = c.hi[0] - c.lo[0], ey = c.hi[1] - c.lo[1], ez = c.hi[2] - c.lo[2];
  return ex * ey + ey * ez + ez * ex;
}

// Smallest power of two s (as a float) with 255 s >= hi - lo (rounded up);
// never below 2^-100.
__device__ __forceinline__ float grid_scale(float lo, float hi) {
  const float extent = __fsub_ru(hi, lo);
  float sc = 0x1p-100f;
  for (int k = 0; k < 256 && sc * 255.0f < extent; ++k) sc *= 2.0f;
  return sc;
}

// Quantize [lo, hi] on the grid p + q * scale, outward; false if it cannot be held.
__device__ bool quantize(float p, float scale, float lo, float hi, uint32_t& qlo, uint32_t& qhi) {
  float fl = floorf(__fsub_rd(lo, p) / scale);
  float fh = ceilf(__fsub_ru(hi, p) / scale);
  int il = int(fminf(fmaxf(fl, 0.0f), 255.0f));
  int ih = int(fminf(fmaxf(fh, 0.0f), 255.0f));
  while (il > 0 && dequant(p, uint32_t(il), scale) > lo) --il;
  while (ih < 255 && dequant(p, uint32_t(ih), scale) < hi) ++ih;
  if (dequant(p, uint32_t(il), scale) > lo || dequant(p, uint32_t(ih), scale) < hi) return false;
  qlo = uint32_t(il);
  qhi = uint32_t(ih);
  return true;
}

struct WItem {
  int w;    // wide node to write
  int rec;  // binary record whose children it collapses
};

// counters: [0] items of the next level, [1] wide nodes allocated, [2] triangle
// records allocated, [3] nonzero when a node cannot be encoded (a leaf of more
// than 4 triangles, a box the grid cannot hold): the caller keeps the binary BVH
__global__ void k_wide_level(const float4* __restrict__ rec, const float4* __restrict__ tgeo,
                             const WItem* __restrict__ in, int n_in, WItem* __restrict__ out, int* counters,
                             float4* __restrict__ wnodes, float4* __restrict__ wtgeo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_in) return;
  const WItem it = in[i];
  Child ch[9];
  int n = 0;
  read_children(rec, it.rec, ch, n);
  // open the largest internal child while the node has room
  while (n < 8) {
    int best = -1;
    float ba = -1.0f;
    for (int j = 0; j < n; ++j)
      if (ch[j].cnt == 0) {
        const float a = half_area(ch[j]);
        if (a > ba) { ba = a; best = j; }
      }
    if (best < 0) break;
    Child two[2];
    int m = 0;
    read_children(rec, ch[best].link, two, m);
    if (m == 0) { ch[best] = ch[--n]; continue; }
    ch[best] = two[0];
    if (m == 2) ch[n++] = two[1];
  }
  // the node's box and centre
  float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  int n_int = 0, n_tri = 0;
  for (int j = 0; j < n; ++j) {
    for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], ch[j].lo[a]); hi[a] = fmaxf(hi[a], ch[j].hi[a]); }
    if (ch[j].cnt == 0) ++n_int;
    else {
      if (ch[j].cnt > 4) { atomicOr(counters + 3, 1); return; }
      n_tri += ch[j].cnt;
    }
  }
  // slots: greedy assignment of children to the octants around the centre
  float cx = 0.5f * (lo[0] + hi[0]), cy = 0.5f * (lo[1] + hi[1]), cz = 0.5f * (lo[2] + hi[2]);
  int slot_of[8];
  uint32_t used = 0, placed = 0;
  for (int round = 0; round < n; ++round) {
    float bc = 3.4e38f;
    int bj = 0, bs = 0;
    for (int j = 0; j < n; ++j) {
      if (placed & (1u << j)) continue;
      const float ox = 0.5f * (ch[j].lo[0] + ch[j].hi[0]) - cx;
      const float oy = 0.5f * (ch[j].lo[1] + ch[j].hi[1]) - cy;
      const float oz = 0.5f * (ch[j].lo[2] + ch[j].hi[2]) - cz;
      for (int sl = 0; sl < 8; ++sl) {
        if (used & (1u << sl)) continue;
        const float c = -((sl & 1 ? ox : -ox) + (sl & 2 ? oy : -oy) + (sl & 4 ? oz : -oz));
        if (c < bc) { bc = c; bj = j; bs = sl; }
      }
    }
    slot_of[bj] = bs;
    placed |= 1u << bj;
    used |= 1u << bs;
  }
  int by_slot[8];
  for (int sl = 0; sl < 8; ++sl) by_slot[sl] = -1;
  for (int j = 0; j < n; ++j) by_slot[slot_of[j]] = j;
  const int child_base = n_int ? atomicAdd(counters + 1, n_int) : 0;
  const int tri_base = n_tri ? atomicAdd(counters + 2, n_tri) : 0;
  // quantization grid
  const float sc[3] = {grid_scale(lo[0], hi[0]), grid_scale(lo[1], hi[1]), grid_scale(lo[2], hi[2])};
  uint32_t ql[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qh[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  uint32_t meta[2] = {0, 0}, imask = 0;
  int rank = 0, toff = 0;
  const int next = n_int ? atomicAdd(counters + 0, n_int) : 0;
  for (int sl = 0; sl < 8; ++sl) {
    const int word = sl >> 2, sh = 8 * (sl & 3);
    const int j = by_slot[sl];
    uint32_t mb = 0xFFu;
    uint32_t bl[3] = {255u, 255u, 255u}, bh[3] = {0u, 0u, 0u};
    if (j >= 0) {
      for (int a = 0; a < 3; ++a)
        if (!quantize(lo[a], sc[a], ch[j].lo[a], ch[j].hi[a], bl[a], bh[a])) { atomicOr(counters + 3, 2); return; }
      if (ch[j].cnt == 0) {
        mb = 0xFEu;
        imask |= 1u << sl;
        out[next + rank] = WItem{child_base + rank, ch[j].link};
        ++rank;
      } else {
        mb = (uint32_t(ch[j].cnt - 1) << 5) | uint32_t(toff);
        for (int k = 0; k < ch[j].cnt; ++k)
          for (int q = 0; q < 3; ++q)
            wtgeo[size_t(tri_base + toff + k) * 3 + q] = tgeo[size_t(ch[j].link + k) * 3 + q];
        toff += ch[j].cnt;
      }
    }
    meta[word] |= mb << sh;
    for (int a = 0; a < 3; ++a) { ql[a][word] |= bl[a] << sh; qh[a][word] |= bh[a] << sh; }
  }
  const uint32_t ew = (__float_as_uint(sc[0]) >> 23) | ((__float_as_uint(sc[1]) >> 23) << 8) |
                      ((__float_as_uint(sc[2]) >> 23) << 16) | (imask << 24);
  float4* nd = wnodes + size_t(it.w) * 5;
  nd[0] = make_float4(lo[0], lo[1], lo[2], __uint_as_float(ew));
  reinterpret_cast<uint4*>(nd)[1] = make_uint4(uint32_t(child_base), uint32_t(tri_base), meta[0], meta[1]);
  reinterpret_cast<uint4*>(nd)[2] = make_uint4(ql[0][0], ql[0][1], ql[1][0], ql[1][1]);
  reinterpret_cast<uint4*>(nd)[3] = make_uint4(ql[2][0], ql[2][1], qh[0][0], qh[0][1]);
  reinterpret_cast<uint4*>(nd)[4] = make_uint4(qh[1][0], qh[1][1], qh[2][0], qh[2][1]);
}

__global__ void k_wide_root(WItem* in, int* counters) {
  in[0] = WItem{0, 0};
  counters[0] = 0;
  counters[1] = 1;  // node 0 is the root
  counters[2] = 0;
  counters[3] = 0;
}

}  // namespace

cudaError_t build_wide(DevBvh& b, cudaStream_t st) {
  b.n_wide = 0;
  if (b.n_records <= 0 || b.n_tris <= 0) return cudaSuccess;
  const int n = b.n_tris;
  // at most one wide node per binary record, one frontier item per wide node
  cudaError_t e;
  if ((e = b.wnodes.reserve(size_t(b.n_records) * 5 * sizeof(float4))) != cudaSuccess) return e;
  if ((e = b.wtgeo.reserve(size_t(n) * 3 * sizeof(float4))) != cudaSuccess) return e;
  if ((e = b.wq.reserve(size_t(b.n_records + 1) * 2 * sizeof(WItem) + 4 * sizeof(int))) != cudaSuccess) return e;
  if (!b.h_wcnt && (e = cudaMallocHost(reinterpret_cast<void**>(&b.h_wcnt), 4 * sizeof(int))) != cudaSuccess)
    return e;
  WItem* qa = b.wq.as<WItem>();
  WItem* qb = qa + (b.n_records + 1);
  int* counters = reinterpret_cast<int*>(qb + (b.n_records + 1));
  k_wide_root<<<1, 1, 0, st>>>(qa, counters);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  int level_n = 1, levels = 0;
  while (level_n > 0) {
    // the traversal keeps one stack entry per level below the root
    if (++levels >= kWideStack) return cudaSuccess;  // too deep: keep the binary BVH
    if ((e = cudaMemsetAsync(counters, 0, sizeof(int), st)) != cudaSuccess) return e;
    k_wide_level<<<(level_n + 127) / 128, 128, 0, st>>>(b.records.as<float4>(), b.tgeo.as<float4>(), qa, level_n,
                                                        qb, counters, b.wnodes.as<float4>(), b.wtgeo.as<float4>());
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(b.h_wcnt, counters, 4 * sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return e;
    if (b.h_wcnt[3]) return cudaSuccess;  // not encodable: keep the binary BVH
    level_n = b.h_wcnt[0];
    std::swap(qa, qb);
  }
  if (b.h_wcnt[2] != n) return cudaSuccess;
  b.n_wide = b.h_wcnt[1];
  b.wide_levels = levels;
  return cudaSuccess;
}

}  // namespace rmd

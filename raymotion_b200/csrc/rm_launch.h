// rm_launch.h - host-side launch wrappers shared by the .cu translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rm_device.cuh"

namespace rmd {

// rm_kernels.cu
cudaError_t launch_render_paths(int lanes, const Scene& s, const Params& p, uint64_t seed, float* hdr, uint8_t* rgb,
                                uint32_t* dbg, unsigned long long* ctr, uint32_t* err, cudaStream_t st);
// stage 0 generate, 1 spatial (temporal + spatial reuse), 2 shade
cudaError_t launch_restir_stage(int stage, const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb,
                                const ResSoA& ri, const ResSoA& rm, const GBufSoA& hg, const ResSoA& hr, float* hdr,
                                uint32_t* dbg, unsigned long long* ctr, uint32_t* err, cudaStream_t st);
cudaError_t launch_trace(const Scene& s, const float* rays, int n, int any_hit, int32_t* tri, float* t, float* u,
                         float* v, uint32_t* err, cudaStream_t st);

// rm_wavefront.cu: ReSTIR shading as wavefront stages.  Path slots are SoA
// arrays indexed by pixel id.
struct WfState {
  uint4* u;      // rng, meta, samples done, vertex index
  float4* sum;   // sample sum, last_pdf
  float4* acc;   // path radiance, psumW
  float4* thr;   // throughput, previous BSDF cosine
  float4* pb;    // previous BSDF value, previous reservoir M
  float4* o;     // extension ray origin
  float4* d;     // extension ray direction
  float4* c;     // contribution of the pending shadow ray if visible
  float4* so;    // shadow ray origin, length
  float4* sd;    // shadow ray direction
  float4* hit;   // t, u, v, triangle
  float4* base;  // kind 1: emission + primary direct light, reservoir sumWu
  uint32_t* occ;
  uint32_t* mM;  // kind 1: reservoir M
};
// Queue slots of one wave: extension rays, shadow rays, then the paths to
// shade sorted by vertex type (a: opaque hit, b: dielectric hit, c: no vertex).
constexpr int kCntExt = 0, kCntShd = 1, kCntA = 2, kCntB = 3, kCntC = 4;
constexpr int kCntSlots = 8;
struct WfQueues {
  int* ext;
  int* shd;
  int* qa;
  int* qb;
  int* qc;
  int* counts;  // kCntSlots ints
};
// The frame's pixels in up to kWfParts parts by row (row y in part y mod
// parts), each with its own queues.
constexpr int kWfParts = 4;
struct WfParts {
  WfQueues q[kWfParts];
  int parts;
};
// The first wave: each pixel queues its first ray in its part's queue.
cudaError_t launch_wavefront_init(const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb, const ResSoA& rm,
                                  const WfState& w, const WfParts& parts, float* hdr, uint32_t* dbg,
                                  unsigned long long* ctr, uint32_t* err, cudaStream_t st);
cudaError_t launch_wavefront_trace(const Scene& s, const WfState& w, const WfQueues& q, int bound, bool shadow,
                                   unsigned long long* ctr, uint32_t* err, cudaStream_t st);
cudaError_t launch_wavefront_shade(int vk, const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                   const WfQueues& cq, int bound, const WfQueues& nq, float* hdr, uint32_t* dbg,
                                   unsigned long long* ctr, uint32_t* err, cudaStream_t st);
// One launch per wave for both traversals (binary BVH) and for the three
// shading queues; the counters of extension and shadow rays stay apart.
// next_counts: the next wave's queue lengths, zeroed by this launch.
cudaError_t launch_wavefront_trace2(const Scene& s, const WfState& w, const WfQueues& q, int bound,
                                    unsigned long long* ctr_ext, unsigned long long* ctr_shd, uint32_t* err,
                                    int* next_counts, cudaStream_t st);
cudaError_t launch_wavefront_shade3(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                    const WfQueues& cq, int bound, const WfQueues& nq, float* hdr, uint32_t* dbg,
                                    unsigned long long* ctr, uint32_t* err, cudaStream_t st);
// Run every path left in q (extension queue + queue c) to the end of its pixel.
// wavefront_tail_capacity: the paths one wave of resident tail blocks holds.
int wavefront_tail_capacity(bool opaque);
cudaError_t launch_wavefront_tail(const Scene& s, const Params& p, const GBufSoA& gb, const WfState& w,
                                  const WfQueues& q, int bound, float* hdr, uint32_t* dbg, unsigned long long* ctr,
                                  unsigned long long* ctr_ext, unsigned long long* ctr_shd, uint32_t* err,
                                  cudaStream_t st);

// rm_batch.cu: many plain-path images (reference K1 / K2) rendered together
// by one pool of path slots.  A pixel owns `lanes` consecutive lane slots (its
// K2 lanes); 32 lane slots form a chunk, which renders one tile of one image
// (tile_w x tile_h pixels, tile_w * tile_h * lanes == 32) and is refilled with
// the next tile of the batch when all its pixels are done.
constexpr int kBtChunk = 32;
struct BtJob {
  Scene s;
  Params p;
  uint64_t seed;
  float* hdr;      // W*H*3 floats, or null
  uint8_t* rgb;    // W*H*3 bytes, or null
  uint32_t* dbg;   // W*H*2 words (xor of the lanes' final RNG states, samples), or null
  int lanes;       // 1, 8 or 32
  int tile_w, tile_h, tiles_x, tiles;
  int tile_begin;  // first tile of the job in the batch's tile sequence
};
struct BtBatch {
  const BtJob* jobs;
  const int* tile_begin;  // per job, ascending
  int n_jobs, total_tiles;
  int* next_tile;         // device counter: next tile to hand out
};
struct BtState {
  // per lane slot
  uint4* u;      // rng, meta, vertex index, -
  float4* acc;   // path radiance, psumW
  float4* thr;   // throughput, previous BSDF cosine
  float4* pb;    // previous BSDF value, previous M
  float4* o;     // extension ray origin, last_pdf
  float4* d;     // extension ray direction
  float4* c;     // contribution of the pending shadow ray if visible
  float4* so;    // shadow ray origin, length
  float4* sd;    // shadow ray direction
  float4* hit;   // t, u, v, triangle (t from hoff's origin in partially transparent scenes)
  float4* hoff;  // partially transparent scenes: origin of the ray that made the hit
  float4* val;   // the slot's sample of the current round
  uint32_t* occ;
  // per pixel group, at the index of its first lane slot
  float4* gsum;  // radiance sums, luminance sum
  float* gsl2;   // squared-luminance sum
  int* gbase;    // first sample index of the current round
  int* garr;     // lanes of the round that have finished their sample
  // per chunk
  int* cjob;     // job, or -1 when idle
  int* ctile;    // tile within the job
  int* cleft;    // pixels of the tile still rendering
};
// Queues of one wave: extension rays, shadow rays, paths to shade by vertex
// type (a opaque surface of an opaque scene with single-candidate NEE, b
// dielectric, c none, d any other opaque surface), lane slots to start a
// sample, chunks to refill, and pixels whose round is complete by lane count
// (1, 8, 32).
constexpr int kBtExt = 0, kBtShd = 1, kBtA = 2, kBtB = 3, kBtC = 4, kBtD = 5, kBtSt = 6, kBtRf = 7;
constexpr int kBtCm1 = 8, kBtCm8 = 9, kBtCm32 = 10;
constexpr int kBtQueues = 11, kBtCounts = 16;
struct BtQueues {
  int *ext, *shd, *qa, *qb, *qc, *qd, *st, *rf, *cm1, *cm8, *cm32;
  int* counts;  // kBtCounts ints
};
cudaError_t launch_batch_init(const BtState& w, const BtQueues& q0, int chunks, int* next_tile, cudaStream_t st);
cudaError_t launch_batch_refill(const BtBatch& b, const BtState& w, const BtQueues& q, int grid, cudaStream_t st);
cudaError_t launch_batch_start(const BtBatch& b, const BtState& w, const BtQueues& q, const BtQueues& nq, int grid,
                               unsigned long long* ctr, uint32_t* err, cudaStream_t st);
cudaError_t launch_batch_trace(const BtBatch& b, const BtState& w, const BtQueues& q, bool shadow, bool wide, int grid,
                               unsigned long long* ctr, uint32_t* err, cudaStream_t st);
cudaError_t launch_batch_shade(int vk, const BtBatch& b, const BtState& w, const BtQueues& q, const BtQueues& nq,
                               int grid, unsigned long long* ctr, uint32_t* err, cudaStream_t st);
// Sum the completed rounds of the pixels with `lanes` lanes (1, 8, 32).
cudaError_t launch_batch_combine(int lanes, const BtBatch& b, const BtState& w, const BtQueues& q,
                                 const BtQueues& nq, int grid, cudaStream_t st);
// Resident blocks per SM of each batch kernel (aux, trace, shade).
void batch_occupancy(int& aux, int& trace, int& shade);

// rm_adjoint.cu: path-replay adjoint of the plain frame (adds g . dC/dparams
// into grad, n_mat x 8 floats: albedo rgb, rough, emission rgb, ior).
cudaError_t launch_adjoint(int lanes, const Scene& s, const Params& p, uint64_t seed, const int32_t* tri_mat,
                           int n_mat, const float* dLdI, float* grad, unsigned long long* ctr, uint32_t* err,
                           cudaStream_t st);
// The adjoint of the ReSTIR shade from the frame's G-buffer and merged
// reservoirs (one thread per pixel).
cudaError_t launch_adjoint_restir(const Scene& s, const Params& p, uint64_t seed, const GBufSoA& gb, const ResSoA& rm,
                                  const int32_t* tri_mat, int n_mat, const float* dLdI, const float* dLdalb,
                                  float* grad, unsigned long long* ctr, uint32_t* err, cudaStream_t st);
// rm_denoise_adjoint.cu: dL/d(ReSTIR shade HDR) and dL/d(G-buffer albedo) from
// dL/d(denoised image), the G-buffer geometry and history colour of the frame
// held; scratch holds 14 floats per pixel.
cudaError_t launch_denoise_backward(const Params& p, const GBufSoA& gb, const GBufSoA& hg, const float* hdr,
                                    const float* hist_col, const float* dLdout, float* scratch, float* dLdhdr,
                                    float* dLdalb, cudaStream_t st);
// Write per-material parameters (8 floats each) into the triangles with tri_mat >= 0.
cudaError_t apply_materials(rm_triangle* tris, const int32_t* tri_mat, const float* mats, int n_tris,
                            cudaStream_t st);

// rm_denoise.cu
// stage 0 temporal (in + hist_in -> out), 1 / 2 a-trous step 0 / 1 (in -> out, + RGB8 when rgb != nullptr)
cudaError_t launch_denoise_stage(int stage, const Params& p, const GBufSoA& gb, const GBufSoA& hg, const float* in,
                                 const float* hist_in, float* out, uint8_t* rgb, cudaStream_t st);
cudaError_t launch_tonemap(const float* hdr, uint8_t* rgb, uint32_t npix, cudaStream_t st);
// rm_atrous.cu: a-trous pass `step` (stride 1 << step), RGB8 written when rgb != nullptr.
cudaError_t launch_atrous_tiled(int step, const Params& p, const GBufSoA& gb, const float* in, float* out,
                                uint8_t* rgb, cudaStream_t st);

// rm_bvh.cu ------------------------------------------------------------------

// Growable device allocation.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t bytes);
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Device-resident BVH + triangle geometry of one scene.
struct DevBvh {
  DevBuf records;   // float4 x 4 per internal record
  DevBuf parents;   // int per record: (parent << 1) | slot, -1 for the root
  DevBuf counters;  // int per record, refit arrival counts
  DevBuf order;     // int per leaf slot: original triangle index (leaf order)
  DevBuf tgeo;      // float4 x 3 per triangle in leaf order
  // LBVH temporaries
  DevBuf keys, keys_alt, vals_alt, knodes, kbox, kcount, ranges, temp, bounds, depth;
  int n_records = 0;
  int n_tris = 0;
  int max_depth = 0;
  // 8-wide compressed BVH collapsed from the records (rm_wide.cu): 5 float4 per
  // node, triangle records in its leaf order, frontier queues; n_wide 0: none
  DevBuf wnodes, wtgeo, wq;
  int* h_wcnt = nullptr;  // pinned counters read back per level
  int n_wide = 0;
  int wide_levels = 0;
};

// Convert and validate a caller BVH (reference Scene::nodes layout) on the
// host, then upload it.  Returns false with a message on invalid input.
bool convert_caller_bvh(const rm_bvh_node* nodes, int n_nodes, const int32_t* bvh_tri, int n_tris, DevBvh& out,
                        cudaStream_t st, std::string& err);
// Build an LBVH on the device from the device triangle array.
cudaError_t build_lbvh(const rm_triangle* d_tris, int n_tris, int leaf_max, DevBvh& out, cudaStream_t st,
                       std::string& err);
// Build a clustering BVH (PLOC) on the device from the device triangle array.
cudaError_t build_ploc(const rm_triangle* d_tris, int n_tris, int leaf_max, DevBvh& out, cudaStream_t st,
                       std::string& err);
// Write the leaf-ordered Moller-Trumbore records from the triangles.
cudaError_t pack_tgeo(const rm_triangle* d_tris, DevBvh& bvh, cudaStream_t st);
// Refit all boxes bottom-up from the current triangle positions.
cudaError_t refit_bvh(const rm_triangle* d_tris, DevBvh& bvh, cudaStream_t st);
// Collapse the binary records into the 8-wide compressed BVH (rm_wide.cu).
// Leaves n_wide at 0 (the binary BVH stays in use) when a node cannot be
// encoded or the wide tree would be deeper than the traversal stack.
cudaError_t build_wide(DevBvh& bvh, cudaStream_t st);
// Caller-provided scratch of an LBVH build (device pointers; see rm_noalloc.cu).
struct LbvhScratch {
  float4* records;        // (n-1) x 4 float4
  int* parents;           // n ints
  int* order;             // n ints
  float4* tgeo;           // n x 3 float4
  unsigned int* keys;     // n
  int* vals;              // n
  unsigned int* keys_alt; // n
  int* vals_alt;          // n
  int2* children;         // n - 1
  int2* ranges;           // n - 1
  int* parent_int;        // n - 1
  int* parent_leaf;       // n
  void* kbox;             // (n - 1) x lbvh_box_bytes()
  int* kcount;            // n - 1
  unsigned int* bounds;   // 6
  uint32_t* err_word;     // 1
  void* sort_temp;
  size_t sort_temp_bytes;
};
struct DevBvhView {
  const float4* records = nullptr;
  const float4* tgeo = nullptr;
  int n_records = 0;
};
// Build an LBVH into caller scratch without allocating (no depth check: the
// traversal's stack guard reports overflow through err_word).
cudaError_t build_lbvh_into(const rm_triangle* d_tris, int n, int leaf_max, const LbvhScratch& w, DevBvhView& out,
                            cudaStream_t st, std::string& err);
size_t lbvh_box_bytes();
// Light records and CDF guide table for light sampling (see Scene in rm_device.cuh).
cudaError_t prepare_lights(const rm_triangle* d_tris, const int32_t* d_lights, const float* d_cdf, int n_lights,
                           float light_total, DevBuf& rec, DevBuf& guide, int& guide_n, float& guide_inv,
                           cudaStream_t st);
// d_flag[0] = 1 when the two device byte ranges differ, else 0 (n_bytes a multiple of 16).
cudaError_t device_differ(const void* a, const void* b, size_t n_bytes, int* d_flag, cudaStream_t st);
// 64-bit content hash of a device byte range (order-sensitive per 8-byte word).
cudaError_t device_hash(const void* d_bytes, size_t n_bytes, unsigned long long* d_out, cudaStream_t st);

// rm_prep.cu: the world triangles of instanced models (Objects::append +
// Scene::add_triangle on the device).  Device pointers; `total` slots = the
// sum of the instances' model triangle counts, start[n_inst + 1] their
// prefix sums.  Outputs: out (world triangles in push order), light_tri /
// cdf (the light list), counts[0..1] (triangles, lights), light_total[0]
// (double), flags[0] (nonzero when every triangle is opaque).
struct PrepArgs {
  const rm_instance* inst;
  const rm_model_tri* const* mptr;  // per instance: its model's triangles
  const int* start;
  int n_inst, total;
  int *keep, *kscan, *light, *lscan;  // total each
  void* scan_temp;
  size_t scan_bytes;
  rm_triangle* out;
  int32_t* light_tri;
  double* weight;
  float* cdf;
  int* counts;
  double* light_total;
  int* flags;
};
cudaError_t prep_scan_bytes(int total, size_t& bytes);
cudaError_t prep_world(const PrepArgs& a, cudaStream_t st);

}  // namespace rmd

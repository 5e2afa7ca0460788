// rm_ctx.h - the library context and device-resident scenes, shared by the
// translation units of the C ABI (rmcuda_api.cu, rmcuda_batch.cu).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <mutex>
#include <string>
#include <vector>

#include "rm_launch.h"
#include "rmcuda.h"

namespace rmapi {

using rmd::DevBuf;
using rmd::DevBvh;
using rmd::GBufSoA;
using rmd::ResSoA;

struct GBufSet {
  DevBuf pos_kind, nor_rough, alb_met, wo_ior, emi;
  cudaError_t reserve(size_t npix) {
    cudaError_t e;
    for (DevBuf* b : {&pos_kind, &nor_rough, &alb_met, &wo_ior, &emi})
      if ((e = b->reserve(npix * sizeof(float4))) != cudaSuccess) return e;
    return cudaSuccess;
  }
  GBufSoA view() const {
    return GBufSoA{pos_kind.as<float4>(), nor_rough.as<float4>(), alb_met.as<float4>(), wo_ior.as<float4>(),
                   emi.as<float4>()};
  }
  void release() { for (DevBuf* b : {&pos_kind, &nor_rough, &alb_met, &wo_ior, &emi}) b->release(); }
};
struct ResSet {
  DevBuf lp, ln, le, wm;
  cudaError_t reserve(size_t npix) {
    cudaError_t e;
    for (DevBuf* b : {&lp, &ln, &le, &wm})
      if ((e = b->reserve(npix * sizeof(float4))) != cudaSuccess) return e;
    return cudaSuccess;
  }
  ResSoA view() const { return ResSoA{lp.as<float4>(), ln.as<float4>(), le.as<float4>(), wm.as<float4>()}; }
  void release() { for (DevBuf* b : {&lp, &ln, &le, &wm}) b->release(); }
};

// One device-resident scene: the uploaded triangles, lights, textures, the
// light-sampling tables and the BVH.
struct DevScene {
  DevBuf tris, lights, cdf, texels, lrec, guide;
  DevBuf tris_in;  // staging of an upload compared with `tris` before the BVH is rebuilt
  uint64_t reuses = 0;  // uploads whose triangles equalled the resident ones (BVH kept)
  std::string build_key;  // the BVH build settings the resident BVH was built with
  int guide_n = 0;
  float guide_inv = 0.0f;
  DevBvh bvh;
  int n_tris = 0, n_lights = 0;
  float light_total = 0;
  bool opaque = true;
  bool have_scene = false;
  int refits = 0;
  bool device_built = false;
  // the texel count the resident triangles were last checked against by
  // upload_scene (texture ranges, opacity); -1 after any other write
  long long validated_texels = -1;
  long long n_texels = 0;  // texels of the last upload
  // host copies of the last upload's light list, CDF, light total and texels,
  // and whether that upload's triangles equalled the resident ones: what a
  // speculative frame (rmcuda_render) needs to know the next upload's small
  // arrays unchanged without sending them
  std::vector<int32_t> h_lights;
  std::vector<float> h_cdf;
  std::vector<rm_vec3> h_texels;
  float h_light_total = 0;
  bool h_valid = false;
  bool last_upload_equal = false;
  // per-triangle materials (rmcuda_scene_set_materials): index per triangle,
  // 8 parameters per material
  DevBuf tri_mat, mats;
  int n_materials = 0;
  void release() {
    for (DevBuf* b : {&tri_mat, &mats, &tris, &tris_in, &lights, &cdf, &texels, &lrec, &guide, &bvh.records, &bvh.parents, &bvh.counters,
                      &bvh.order, &bvh.tgeo, &bvh.keys, &bvh.keys_alt, &bvh.vals_alt, &bvh.knodes, &bvh.kbox,
                      &bvh.kcount, &bvh.ranges, &bvh.temp, &bvh.bounds, &bvh.depth, &bvh.wnodes, &bvh.wtgeo,
                      &bvh.wq})
      b->release();
    if (bvh.h_wcnt) cudaFreeHost(bvh.h_wcnt);
    bvh.h_wcnt = nullptr;
  }
};

// Buffers of batched rendering: the pool of lane slots (rmd::BtState), the
// queues of two waves, the job table and the captured wave graph.
struct BatchPool {
  DevBuf slot[17];   // per lane slot and per group arrays of BtState
  DevBuf chunk[3];   // per chunk arrays of BtState
  DevBuf queue[2 * rmd::kBtQueues + 1];  // the queues of two waves + the counts of both
  DevBuf jobs, tile_begin, next_tile;
  rm_batch_tuning tuning{65536, 0, 1, 8, 2};
  int chunks = 0;    // pool size the buffers hold, in chunks of 32 lane slots
  int occ[3] = {0, 0, 0};  // resident blocks per SM of the batch kernels
  int* h_counts = nullptr;  // pinned: queue lengths read back between graph launches (2 x kBtCounts)
  cudaGraphExec_t exec = nullptr;
  uint64_t waves = 0;
  std::vector<int> wave_log;  // last batch: (live slots, extension rays) per check
  void release();
};

// Frame policy of one image (metal.mm:146-170, :236-237, :390-394).
struct Plan {
  rmd::Params p;
  int lanes = 1;
  bool use_spatial = false;
  bool denoise = true;
  bool temporal_off = false;
};

}  // namespace rmapi

struct rmcuda_scene {
  rmapi::DevScene d;
  int device = 0;
};

struct rmcuda_ctx {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  std::mutex mu;
  rmapi::DevScene sc;  // the resident scene
  // frame buffers
  rmapi::GBufSet gb, hg;
  rmapi::ResSet rinit, rmerged, hres;
  rmd::DevBuf hdr, tmp_a, tmp_b, hist_col, rgb, dbg, hash_out;
  rmd::DevBuf ctr, err;
  // speculative frames of rmcuda_render: the copy stream that uploads and
  // compares the triangles while the frame renders, its pinned result, a copy
  // of the counters to restore, and the configuration of the last frame
  cudaStream_t copy_stream = nullptr;
  rmd::DevBuf differ, ctr_save;
  int* h_differ = nullptr;
  rm_config last_cfg{};
  bool have_last_cfg = false;
  // temporal history (metal.mm:35-40)
  rm_camera hist_cam{};
  int hist_w = 0, hist_h = 0;
  uint64_t hist_seed = 0;
  unsigned long long hist_hash = 0;
  bool hist_valid = false, have_hist_bufs = false;
  // the frame the history buffers hold (the ReSTIR adjoint's checkpoint)
  const void* hist_scene = nullptr;
  rm_config hist_cfg{};
  bool hist_denoised = false;
  bool hist_had_history = false;  // the frame's temporal passes used the history before it
  rm_camera hist_prev_cam{};       // and this camera for reprojection
  rmd::DevBuf adj_scratch;         // the denoiser backward's intermediate images
  uint8_t* h_preview = nullptr;    // pinned RGB8 read-back of rmcuda_preview_last
  size_t h_preview_cap = 0;
  // last frame
  int last_chain = 0;
  uint64_t frames = 0;
  uint64_t launches = 0;
  float* last_final = nullptr;  // device pointer of the last frame's tonemap input
  int last_w = 0, last_h = 0;
  // wavefront shading state (rm_wavefront.cu)
  rmd::DevBuf wf[14];
  // queues of the parts of a frame (rows y mod parts), two wave sets each (5
  // arrays per set), then their counts; the streams of the parts after the first
  rmd::DevBuf wq[10 * rmd::kWfParts + 1];
  int* h_counts = nullptr;  // pinned: two reads of the parts' queue lengths (2 x kWfParts x kCntSlots)
  cudaEvent_t ev_counts[2][rmd::kWfParts] = {};  // the end of each of those reads
  cudaStream_t side_stream[rmd::kWfParts - 1] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[rmd::kWfParts - 1] = {};
  size_t wf_cap = 0;
  uint64_t waves = 0;
  std::vector<int> wave_log;  // last frame: (act, ext, shd, us) per count read
  // batched rendering (rmcuda_batch.cu)
  rmapi::BatchPool batch;
  // device-side scene preparation (rm_prep.cu): models, the last commit's
  // model list (its topology), scratch, pinned read-back
  struct Model { rmd::DevBuf tris; int n = 0; };
  std::vector<Model> models;
  std::vector<int> prep_topology;
  uint64_t prep_commits = 0;
  rmd::DevBuf prep_inst, prep_mptr, prep_start, prep_keep, prep_kscan, prep_light, prep_lscan, prep_temp,
      prep_weight, prep_small;
  void* h_prep = nullptr;  // pinned: counts[2], flags, pad, light total (double)
  uint32_t bvh_builds = 0, bvh_refits = 0;
  // per-stage CUDA-event timing (rmcuda_profile)
  int profiling = 0;
  struct Pending { int stage; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  double stage_ms[RM_STAGE_COUNT] = {};
  uint64_t stage_n[RM_STAGE_COUNT] = {};
};

namespace rmapi {

extern const char* const kUnavailable;
extern const char* const kInvalidDims;

void set_err(char* err, size_t cap, const std::string& m);
std::string cuda_msg(const char* what, cudaError_t e);

// A named NVTX range over a host scope (API calls, frame stages): profilers
// (ncu --nvtx, Nsight) attribute the kernels launched inside it to that name.
// Without a tool attached, a push and a pop cost a few nanoseconds.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// NVTX names of the RM_STAGE_* stages
const char* stage_name(int stage);

// Launch through `fn`, bracketed by events on the context stream when profiling.
template <class Fn> cudaError_t staged(rmcuda_ctx* c, int stage, Fn&& fn) {
  NvtxRange range(stage_name(stage));
  cudaEvent_t a = nullptr, b = nullptr;
  if (c->profiling > 0 && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
    cudaEventRecord(a, c->stream);
  cudaError_t e = fn();
  if (a && b) {
    cudaEventRecord(b, c->stream);
    c->pending.push_back({stage, a, b});
  }
  c->launches += 1;
  return e;
}

// As staged2(), on another stream of the context.
template <class Fn> cudaError_t staged2_on(rmcuda_ctx* c, int stage, cudaStream_t st, Fn&& fn) {
  c->launches += 1;
  if (c->profiling < 2) return fn();
  NvtxRange range(stage_name(stage));
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess) cudaEventRecord(a, st);
  cudaError_t e = fn();
  if (a && b) {
    cudaEventRecord(b, st);
    c->pending.push_back({stage, a, b});
  }
  return e;
}

// As staged(), but timed only at profiling level 2 (per-launch breakdown).
template <class Fn> cudaError_t staged2(rmcuda_ctx* c, int stage, Fn&& fn) {
  if (c->profiling >= 2) return staged(c, stage, fn);
  c->launches += 1;
  return fn();
}

void resolve_pending(rmcuda_ctx* c);
rmd::Scene scene_view(const DevScene& sc);
// Validate and upload one scene into `sc`; build or convert its BVH.
int upload_scene(rmcuda_ctx* c, DevScene& sc, const rm_scene_view* sv, std::string& msg);
Plan make_plan(const DevScene& sc, const rm_camera& cam, const rm_config& cfg);
// Enqueue one frame of `sc` with the single-frame policy.
int enqueue_frame(rmcuda_ctx* c, DevScene& sc, const rm_camera& cam, const rm_config& cfg, uint64_t seed,
                  uint8_t* d_rgb, std::string& msg);
int check_device_error(rmcuda_ctx* c, std::string& msg);

}  // namespace rmapi

// rmcuda_api.cu - the C ABI of include/rmcuda.h: context, scene upload, and
// the per-frame policy of the reference's render_image_metal
// (src/engine/metal.mm:95-414), re-expressed for CUDA streams.
//
// Differences in mechanism, not in results:
//  * the scene is uploaded once per call into grow-only device buffers (the
//    reference re-packs into Metal shared buffers, metal.mm:171-186); the
//    BVH is either the caller's (validated and converted, rm_bvh.cu) or built
//    on the device;
//  * the scene hash that guards temporal reuse (metal.mm:241-248) is computed
//    on the device over the uploaded bytes;
//  * the plain path runs the lane kernels (metal.mm:390-394) and the ReSTIR
//    path runs generate / spatial / shade / denoise (metal.mm:287-366) as
//    kernels on one stream, then one device-to-host copy of the RGB8 image.
#include <cuda_runtime.h>

#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "rm_ctx.h"
#include "rm_launch.h"
#include "rmcuda.h"

using namespace rmd;
using namespace rmapi;

namespace rmapi {

const char* const kUnavailable = "Metal backend is not available in this build";
const char* const kInvalidDims = "Invalid Metal render dimensions or sample count";

void set_err(char* err, size_t cap, const std::string& m) {
  if (err && cap) std::snprintf(err, cap, "%s", m.c_str());
}

std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

}  // namespace rmapi

namespace {

constexpr int kLbvhLeaf = 4;

// The 8-wide compressed BVH, collapsed from the binary one (rm_wide.cu), when
// RAYMOTION_CUDA_WIDE=1: traversal then uses it instead of the binary BVH.  It
// visits a third of the nodes, but its exact box decoding costs more per ray
// than the binary BVH's fetches on the bench scene, so the binary BVH is the
// default.
cudaError_t finish_wide(rmd::DevBvh& bvh, cudaStream_t st) {
  const char* v = std::getenv("RAYMOTION_CUDA_WIDE");
  if (!v || std::string(v) != "1") { bvh.n_wide = 0; return cudaSuccess; }
  return rmd::build_wide(bvh, st);
}

// Device BVH builder: PLOC clustering (default) or LBVH (RAYMOTION_CUDA_BVH=lbvh);
// RAYMOTION_CUDA_BVH_LEAF sets the maximum triangles per leaf (default 4).
cudaError_t build_device_bvh(const rm_triangle* d_tris, int n, rmd::DevBvh& bvh, cudaStream_t st, std::string& err) {
  int leaf = kLbvhLeaf;
  if (const char* v = std::getenv("RAYMOTION_CUDA_BVH_LEAF")) leaf = std::max(1, std::min(255, std::atoi(v)));
  const char* kind = std::getenv("RAYMOTION_CUDA_BVH");
  if (kind && std::string(kind) == "lbvh") return rmd::build_lbvh(d_tris, n, leaf, bvh, st, err);
  cudaError_t e = rmd::build_ploc(d_tris, n, leaf, bvh, st, err);
  if (e != cudaSuccess && err.find("deeper") != std::string::npos) {
    err.clear();
    return rmd::build_lbvh(d_tris, n, leaf, bvh, st, err);  // depth fallback
  }
  return e;
}

struct Env {
  bool noadapt = false, nomis = false, restir_off = false, denoise_off = false, temporal_off = false;
  bool have_cand = false, have_spatial = false;
  int cand = 0, spatial = 0;
};

Env read_env(uint32_t flags) {
  Env e;
  if (flags & RM_FLAG_NO_ENV) {
    e.noadapt = flags & RM_FLAG_NOADAPT;
    e.nomis = flags & RM_FLAG_NOMIS;
    e.restir_off = flags & RM_FLAG_RESTIR_OFF;
    e.denoise_off = flags & RM_FLAG_DENOISE_OFF;
    e.temporal_off = flags & RM_FLAG_TEMPORAL_OFF;
    return e;
  }
  auto eq0 = [](const char* v) { return v && std::string(v) == "0"; };
  e.noadapt = std::getenv("UOW2_NOADAPT") != nullptr;
  e.nomis = std::getenv("UOW2_NOMIS") != nullptr;
  e.restir_off = eq0(std::getenv("RAYMOTION_RESTIR"));
  e.denoise_off = eq0(std::getenv("RAYMOTION_DENOISE"));
  e.temporal_off = eq0(std::getenv("RAYMOTION_RESTIR_TEMPORAL"));
  if (const char* v = std::getenv("RAYMOTION_RESTIR_CANDIDATES")) { e.have_cand = true; e.cand = std::atoi(v); }
  if (const char* v = std::getenv("RAYMOTION_RESTIR_SPATIAL")) { e.have_spatial = true; e.spatial = std::atoi(v); }
  return e;
}

}  // namespace

namespace rmapi {

const char* stage_name(int stage) {
  static const char* const names[RM_STAGE_COUNT] = {
      "rm plain paths", "rm scene hash", "rm restir generate", "rm restir spatial", "rm restir shade",
      "rm denoise temporal", "rm denoise atrous 1", "rm denoise atrous 2", "rm tonemap", "rm wavefront traversal",
      "rm wavefront shadow", "rm wavefront shade", "rm batch start", "rm batch extend", "rm batch shadow",
      "rm batch shade", "rm batch", "rm adjoint", "rm wavefront tail", "rm scene preparation"};
  return stage >= 0 && stage < RM_STAGE_COUNT ? names[stage] : "rm stage";
}

void resolve_pending(rmcuda_ctx* c) {
  for (auto& pe : c->pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(pe.b) == cudaSuccess && cudaEventElapsedTime(&ms, pe.a, pe.b) == cudaSuccess) {
      c->stage_ms[pe.stage] += ms;
      c->stage_n[pe.stage] += 1;
    }
    cudaEventDestroy(pe.a);
    cudaEventDestroy(pe.b);
  }
  c->pending.clear();
}

Scene scene_view(const DevScene& sc) {
  Scene s;
  s.tris = sc.tris.as<rm_triangle>();
  s.tgeo = sc.bvh.tgeo.as<float4>();
  s.nodes = sc.bvh.records.as<float4>();
  s.n_nodes = sc.n_tris > 0 ? sc.bvh.n_records : 0;
  s.lights = sc.lights.as<int32_t>();
  s.cdf = sc.cdf.as<float>();
  s.n_lights = sc.n_lights;
  s.light_total = sc.light_total;
  s.texels = sc.texels.as<rm_vec3>();
  s.lrec = sc.lrec.as<float4>();
  s.guide = sc.guide.as<int32_t>();
  s.guide_n = sc.guide_n;
  s.guide_inv = sc.guide_inv;
  s.n_tris = sc.n_tris;
  s.n_texels = sc.n_texels;
  if (sc.n_tris > 0 && sc.bvh.n_wide > 0) {
    s.wnodes = sc.bvh.wnodes.as<float4>();
    s.wtgeo = sc.bvh.wtgeo.as<float4>();
  }
  return s;
}

// Validate and upload one scene; build or convert its BVH.
int upload_scene(rmcuda_ctx* c, DevScene& sc, const rm_scene_view* sv, std::string& msg) {
  NvtxRange range("rm scene upload");
  if (!sv || sv->n_tris < 0 || sv->n_lights < 0 || sv->n_texels < 0 || (sv->n_tris > 0 && !sv->tris) ||
      (sv->n_lights > 0 && (!sv->light_tri || !sv->light_cdf)) || (sv->n_texels > 0 && !sv->texels)) {
    msg = "invalid scene view";
    return RM_ERR_INVALID;
  }
  for (int i = 0; i < sv->n_lights; ++i)
    if (sv->light_tri[i] < 0 || sv->light_tri[i] >= sv->n_tris) { msg = "light index out of range"; return RM_ERR_INVALID; }
  // Texture ranges and opacity, from the host triangles (a pass over all of
  // them); skipped below for triangles equal to resident ones that passed it
  // against the same texel count.
  bool opaque = true;
  auto check_tris = [&]() {
    opaque = true;
    for (int i = 0; i < sv->n_tris; ++i) {
      const rm_triangle& t = sv->tris[i];
      if (!(t.alpha >= 1.0f)) opaque = false;
      if (t.texture_offset >= 0) {
        if (t.texture_width <= 0 || t.texture_height <= 0 ||
            int64_t(t.texture_offset) + int64_t(t.texture_width) * t.texture_height > sv->n_texels) {
          msg = "triangle texture outside the texel array";
          return false;
        }
      }
    }
    return true;
  };
  cudaStream_t st = c->stream;
  cudaError_t e;
  const size_t tb = size_t(sv->n_tris) * sizeof(rm_triangle);
  if ((e = sc.tris.reserve(tb)) != cudaSuccess || (e = sc.lights.reserve(size_t(sv->n_lights) * 4)) != cudaSuccess ||
      (e = sc.cdf.reserve(size_t(sv->n_lights) * 4)) != cudaSuccess ||
      (e = sc.texels.reserve(size_t(sv->n_texels) * sizeof(rm_vec3))) != cudaSuccess) {
    msg = cuda_msg("Metal scene buffer allocation failed", e);
    return RM_ERR_ALLOC;
  }
  // The reference re-uploads the scene every frame (metal.mm:171-186).  When a
  // device-built scene is uploaded again with the same triangle count, the new
  // triangles go to a staging buffer and are compared with the resident ones
  // on the device: equal bytes keep the BVH (the build is deterministic, so
  // it would come out the same), different bytes swap in and rebuild.
  std::string key;
  for (const char* k : {"RAYMOTION_CUDA_BVH", "RAYMOTION_CUDA_BVH_LEAF", "RAYMOTION_CUDA_WIDE"}) {
    const char* v = std::getenv(k);
    key += v ? v : "-";
    key += '|';
  }
  const bool may_reuse = sc.have_scene && sc.device_built && !sv->nodes && sv->n_tris > 0 &&
                         sv->n_tris == sc.n_tris && sc.bvh.n_records > 0 && key == sc.build_key;
  bool reuse = false;
  if (may_reuse) {
    int differ = 1;
    if ((e = sc.tris_in.reserve(tb)) != cudaSuccess || (e = c->hash_out.reserve(8)) != cudaSuccess ||
        (e = cudaMemcpyAsync(sc.tris_in.ptr, sv->tris, tb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = device_differ(sc.tris_in.ptr, sc.tris.ptr, tb, c->hash_out.as<int>(), st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&differ, c->hash_out.ptr, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
      msg = cuda_msg("scene upload failed", e);
      return RM_ERR_CUDA;
    }
    reuse = differ == 0;
  }
  if (reuse && sc.validated_texels == int64_t(sv->n_texels)) opaque = sc.opaque;
  else if (!check_tris()) return RM_ERR_INVALID;  // the resident scene is untouched
  if (may_reuse && !reuse) std::swap(sc.tris, sc.tris_in);
  if (&sc == &c->sc) c->prep_topology.clear();  // an uploaded scene is not an instance commit
  sc.validated_texels = -1;
  if ((!may_reuse && tb && (e = cudaMemcpyAsync(sc.tris.ptr, sv->tris, tb, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
      (sv->n_lights &&
       (e = cudaMemcpyAsync(sc.lights.ptr, sv->light_tri, size_t(sv->n_lights) * 4, cudaMemcpyHostToDevice, st)) !=
           cudaSuccess) ||
      (sv->n_lights &&
       (e = cudaMemcpyAsync(sc.cdf.ptr, sv->light_cdf, size_t(sv->n_lights) * 4, cudaMemcpyHostToDevice, st)) !=
           cudaSuccess) ||
      (sv->n_texels && (e = cudaMemcpyAsync(sc.texels.ptr, sv->texels, size_t(sv->n_texels) * sizeof(rm_vec3),
                                            cudaMemcpyHostToDevice, st)) != cudaSuccess)) {
    msg = cuda_msg("scene upload failed", e);
    return RM_ERR_CUDA;
  }
  sc.n_tris = sv->n_tris;
  sc.n_lights = sv->n_lights;
  sc.light_total = sv->light_total;
  sc.opaque = opaque;
  sc.validated_texels = sv->n_texels;
  sc.n_texels = sv->n_texels;
  if (&sc == &c->sc) {
    sc.h_lights.assign(sv->light_tri, sv->light_tri + sv->n_lights);
    sc.h_cdf.assign(sv->light_cdf, sv->light_cdf + sv->n_lights);
    sc.h_texels.assign(sv->texels, sv->texels + sv->n_texels);
    sc.h_light_total = sv->light_total;
    sc.h_valid = true;
    sc.last_upload_equal = reuse;
  }
  if ((e = prepare_lights(sc.tris.as<rm_triangle>(), sc.lights.as<int32_t>(), sc.cdf.as<float>(), sc.n_lights,
                          sc.light_total, sc.lrec, sc.guide, sc.guide_n, sc.guide_inv, st)) != cudaSuccess) {
    msg = cuda_msg("light preparation failed", e);
    return RM_ERR_CUDA;
  }
  if (reuse) {
    sc.reuses++;
    return RM_OK;  // BVH (and wide nodes) of these very triangles kept
  }
  sc.refits = 0;
  sc.have_scene = false;
  if (sv->n_tris > 0 && sv->nodes && sv->n_nodes == 0) {
    // caller passed an empty BVH: every ray misses, as with params.nodes == 0
    // in the reference (pathtrace.metal:121)
    sc.bvh.n_records = 0;
    sc.bvh.n_tris = 0;
    sc.device_built = false;
  } else if (sv->n_tris > 0) {
    bool converted = false;
    if (sv->nodes && sv->n_nodes > 0) {
      std::string berr;
      if (convert_caller_bvh(sv->nodes, sv->n_nodes, sv->bvh_tri, sv->n_tris, sc.bvh, st, berr)) {
        converted = true;
      } else if (berr.find("deeper") == std::string::npos) {
        msg = berr;
        return RM_ERR_BVH;
      }
      if (converted && (e = pack_tgeo(sc.tris.as<rm_triangle>(), sc.bvh, st)) != cudaSuccess) {
        msg = cuda_msg("BVH packing failed", e);
        return RM_ERR_CUDA;
      }
    }
    sc.device_built = !converted;
    if (!converted) {
      if (&sc == &c->sc) c->bvh_builds++;  // the resident scene's builds are counted
      std::string berr;
      if ((e = build_device_bvh(sc.tris.as<rm_triangle>(), sv->n_tris, sc.bvh, st, berr)) != cudaSuccess) {
        msg = berr.empty() ? cuda_msg("device BVH build failed", e) : berr;
        return RM_ERR_CUDA;
      }
    }
  } else {
    sc.bvh.n_records = 0;
    sc.bvh.n_tris = 0;
  }
  if ((e = finish_wide(sc.bvh, st)) != cudaSuccess) {
    msg = cuda_msg("wide BVH build failed", e);
    return RM_ERR_CUDA;
  }
  sc.build_key = key;
  sc.have_scene = true;
  return RM_OK;
}

// metal.mm:146-170, :236-237, :390-394
Plan make_plan(const DevScene& sc, const rm_camera& cam, const rm_config& cfg) {
  Env env = read_env(cfg.flags);
  Plan pl;
  Params& p = pl.p;
  std::memset(&p, 0, sizeof(p));
  p.camera = cam;
  p.width = cfg.width; p.height = cfg.height; p.spp = cfg.spp; p.bounces = cfg.max_bounces;
  p.nodes = sc.n_tris > 0 ? sc.bvh.n_records : 0;
  p.lights = sc.n_lights; p.light_total = sc.light_total;
  p.resolution = cfg.resolution; p.clamp_value = cfg.clamp; p.adapt_rel = cfg.adapt_rel; p.adapt_abs = cfg.adapt_abs;
  p.adapt_min = env.noadapt ? 0 : cfg.adapt_min;
  p.adapt_step = cfg.adapt_step > 0 ? cfg.adapt_step : 8;
  p.opaque = sc.opaque ? 1 : 0;
  p.nomis = env.nomis ? 1 : 0;
  p.restir_candidates = env.restir_off ? 1 : (cfg.restir_candidates > 0 ? cfg.restir_candidates : 1);
  p.restir_candidates = std::min(32, std::max(1, p.restir_candidates));
  p.restir_spatial = env.restir_off ? 0 : (cfg.restir_spatial > 0 ? cfg.restir_spatial : 0);
  p.restir_spatial = std::min(8, std::max(0, p.restir_spatial));
  p.restir_mcap = cfg.restir_mcap > 0 ? cfg.restir_mcap : 128;
  p.restir_radius = cfg.restir_radius > 0 ? cfg.restir_radius : 16.0f;
  if (env.have_cand) p.restir_candidates = std::max(1, env.cand);
  if (env.have_spatial) p.restir_spatial = std::max(0, env.spatial);
  p.rr = (cfg.flags & RM_FLAG_NO_RR) ? 0 : 1;
  const size_t pixels = size_t(cfg.width) * size_t(cfg.height);
  const size_t restir_bytes = pixels * (76 + 2 * 60);  // reference record sizes, metal.mm:236
  pl.use_spatial = p.restir_spatial > 0 && p.lights > 0 && p.bounces > 0 && p.opaque &&
                   restir_bytes <= size_t(512) * 1024 * 1024;
  pl.denoise = !env.denoise_off;
  pl.temporal_off = env.temporal_off;
  if (cfg.spp >= 8 && (p.adapt_min <= 0 || p.adapt_step % 8 == 0)) pl.lanes = 8;
  if (cfg.spp >= 32 && (p.adapt_min <= 0 || p.adapt_step % 32 == 0)) pl.lanes = 32;
  return pl;
}

bool use_megakernel() {
  const char* v = std::getenv("RAYMOTION_CUDA_MEGAKERNEL");
  return v && std::string(v) == "1";
}

cudaError_t ensure_wavefront(rmcuda_ctx* c, size_t npix) {
  if (c->wf_cap >= npix && c->h_counts) return cudaSuccess;
  cudaError_t e;
  for (int i = 0; i < 14; ++i)
    if ((e = c->wf[i].reserve(npix * (i < 12 ? sizeof(float4) : sizeof(uint32_t)))) != cudaSuccess) return e;
  for (int i = 0; i < 10 * kWfParts; ++i)
    if ((e = c->wq[i].reserve(npix * sizeof(int))) != cudaSuccess) return e;
  if ((e = c->wq[10 * kWfParts].reserve(2 * kWfParts * kCntSlots * sizeof(int))) != cudaSuccess) return e;
  if (!c->h_counts &&
      (e = cudaMallocHost(reinterpret_cast<void**>(&c->h_counts), 2 * kWfParts * kCntSlots * sizeof(int))) !=
          cudaSuccess)
    return e;
  for (auto& row : c->ev_counts)
    for (cudaEvent_t& ev : row)
      if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
  c->wf_cap = npix;
  return cudaSuccess;
}

// ReSTIR shading as wavefront stages (rm_wavefront.cu): init, then waves of
// extend / shadow / shade until no path is left.
// Unfinished paths at or below which the wavefront loop hands its last paths
// to one tail launch: a tenth of the paths of the first wave (on the 720p bench
// frame a tenth to a twentieth measured best; below it the waves run with
// the GPU mostly idle, above it the tail's one-thread-per-pixel loop is slower
// than the waves), and no more than one wave of resident tail blocks holds (a
// second wave of blocks would run after the first, doubling the tail).
// RAYMOTION_CUDA_TAIL sets a fixed count; 0 keeps the waves to the end.
static int tail_paths(int first_bound, bool opaque) {
  const char* v = std::getenv("RAYMOTION_CUDA_TAIL");
  if (v) return std::max(0, std::atoi(v));
  return std::min(first_bound / 10, rmd::wavefront_tail_capacity(opaque));
}

cudaError_t run_wavefront_shade(rmcuda_ctx* c, const Scene& s, const Params& p, uint64_t seed, std::string& msg) {
  NvtxRange range("rm wavefront shading loop");
  const size_t npix = size_t(p.width) * size_t(p.height);
  cudaError_t e = ensure_wavefront(c, npix);
  if (e != cudaSuccess) { msg = cuda_msg("wavefront allocation failed", e); return e; }
  WfState w{c->wf[0].as<uint4>(), c->wf[1].as<float4>(), c->wf[2].as<float4>(), c->wf[3].as<float4>(),
            c->wf[4].as<float4>(), c->wf[5].as<float4>(), c->wf[6].as<float4>(), c->wf[7].as<float4>(),
            c->wf[8].as<float4>(), c->wf[9].as<float4>(), c->wf[10].as<float4>(), c->wf[11].as<float4>(),
            c->wf[12].as<uint32_t>(), c->wf[13].as<uint32_t>()};
  // One launch per wave for the traversals and one for the shading queues
  // (each launch's slowest warps then overlap the others' work);
  // RAYMOTION_CUDA_SPLIT_WAVES=1 launches each traversal and queue alone.
  const char* split_env = std::getenv("RAYMOTION_CUDA_SPLIT_WAVES");
  const bool merged = !(split_env && split_env[0] == '1');
  // The frame's pixels in parts (row y in part y mod parts) with their own
  // queues, waves and tail, on their own streams: every launch ends with its
  // slowest warps while the GPU idles, and the other parts' launches fill that
  // time.  A pixel's steps are the same either way.  RAYMOTION_CUDA_STREAMS
  // sets the number of parts (1-4, default 3; on the 720p bench frame 2, 3
  // and 4 parts measured 310, 314 and 311 M path samples/s, one part 292 M).
  int parts = 3;
  if (const char* v = std::getenv("RAYMOTION_CUDA_STREAMS")) parts = std::max(1, std::min(kWfParts, std::atoi(v)));
  if (!merged || p.height < parts) parts = 1;
  if (parts > 1 && !c->ev_fork && cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    parts = 1;
  }
  for (int h = 1; h < parts; ++h)
    if (!c->side_stream[h - 1] &&
        (cudaStreamCreateWithFlags(&c->side_stream[h - 1], cudaStreamNonBlocking) != cudaSuccess ||
         cudaEventCreateWithFlags(&c->ev_join[h - 1], cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      parts = h;
      break;
    }
  cudaStream_t sts[kWfParts];
  for (int h = 0; h < kWfParts; ++h) sts[h] = h == 0 || h >= parts ? c->stream : c->side_stream[h - 1];
  // on an early return (an error), the other parts' queued work finishes
  // before the next frame can reuse the path state
  struct SideSync {
    cudaStream_t* st;
    int n;
    ~SideSync() { for (int h = 1; h < n; ++h) cudaStreamSynchronize(st[h]); }
  } side_sync{sts, parts};
  int* counts = c->wq[10 * kWfParts].as<int>();
  WfQueues q[kWfParts][2];
  WfParts first{};
  first.parts = parts;
  for (int h = 0; h < kWfParts; ++h) {
    for (int k = 0; k < 2; ++k) {
      DevBuf* b = c->wq + 10 * h + 5 * k;
      q[h][k] = WfQueues{b[0].as<int>(), b[1].as<int>(), b[2].as<int>(), b[3].as<int>(), b[4].as<int>(),
                         counts + kCntSlots * (2 * h + k)};
    }
    first.q[h] = q[h][0];
  }
  unsigned long long* ctr = c->ctr.as<unsigned long long>();
  uint32_t* err = c->err.as<uint32_t>();
  if ((e = cudaMemsetAsync(counts, 0, 2 * kWfParts * kCntSlots * sizeof(int), c->stream)) != cudaSuccess) {
    msg = cuda_msg("memset", e);
    return e;
  }
  e = staged2(c, RM_STAGE_WF_SHADE, [&] {
    return launch_wavefront_init(s, p, seed, c->gb.view(), c->rmerged.view(), w, first, c->hdr.as<float>(),
                                 c->dbg.as<uint32_t>(), ctr + 4 * RM_STAGE_WF_SHADE, err, c->stream);
  });
  if (e != cudaSuccess) { msg = cuda_msg("wavefront init failed", e); return e; }
  if (parts > 1 && (e = cudaEventRecord(c->ev_fork, c->stream)) != cudaSuccess) {
    msg = cuda_msg("stream fork failed", e);
    return e;
  }
  for (int h = 1; h < parts; ++h)
    if ((e = cudaStreamWaitEvent(sts[h], c->ev_fork, 0)) != cudaSuccess) {
      msg = cuda_msg("stream fork failed", e);
      return e;
    }
  c->wave_log.clear();
  // Every unfinished pixel of a part has its path either in the part's
  // extension queue or (if it only waits for a shadow ray) in its queue c,
  // and the number of unfinished pixels only shrinks: ext + c read every
  // kBatch waves bounds all queues of the part's later waves, which size their
  // grids; kernels read exact lengths on the device.  RAYMOTION_CUDA_WAVE_BATCH
  // sets kBatch (default 4).  Each batch's waves are sized by the read taken
  // one batch earlier (its copy has finished while the previous batch's
  // waves run), so the host never waits for the GPU to drain; the bound is at
  // most kBatch waves older, the tail starts up to kBatch waves later, and
  // the pixels come out the same.  RAYMOTION_CUDA_COUNT_LAG=0 sizes each
  // batch by a read of its own queues, waiting for them.
  int kBatch = 4;
  if (const char* v = std::getenv("RAYMOTION_CUDA_WAVE_BATCH")) kBatch = std::max(1, std::min(64, std::atoi(v)));
  const char* lag_env = std::getenv("RAYMOTION_CUDA_COUNT_LAG");
  const bool lag = !(lag_env && lag_env[0] == '0');
  int slot = 0;
  const uint64_t max_waves = uint64_t(p.spp) * uint64_t(p.bounces + 2) * 4 + 64;
  int cur[kWfParts] = {};
  bool done[kWfParts];
  for (int h = 0; h < kWfParts; ++h) done[h] = h >= parts;
  int bound[kWfParts] = {};
  std::chrono::steady_clock::time_point t0;
  int tail = 0;
  for (uint64_t wave = 0;; wave += kBatch) {
    if (wave > max_waves) { msg = "wavefront did not drain"; return cudaErrorLaunchFailure; }
    for (int h = 0; h < parts; ++h)
      if (!done[h] &&
          ((e = cudaMemcpyAsync(c->h_counts + kCntSlots * (kWfParts * slot + h), q[h][cur[h]].counts,
                                kCntSlots * sizeof(int), cudaMemcpyDeviceToHost, sts[h])) != cudaSuccess ||
           (e = cudaEventRecord(c->ev_counts[slot][h], sts[h])) != cudaSuccess)) {
        msg = cuda_msg("wavefront count read failed", e);
        return e;
      }
    // the first batch has nothing queued behind its read: it waits for it
    const int use = lag && wave > 0 ? slot ^ 1 : slot;
    slot ^= 1;
    for (int h = 0; h < parts; ++h)
      if (!done[h] && (e = cudaEventSynchronize(c->ev_counts[use][h])) != cudaSuccess) {
        msg = cuda_msg("wavefront count read failed", e);
        return e;
      }
    int b_all = 0, ext_all = 0, shd_all = 0;
    for (int h = 0; h < parts; ++h) {
      if (done[h]) continue;
      const int* hc = c->h_counts + kCntSlots * (kWfParts * use + h);
      bound[h] = hc[kCntExt] + hc[kCntC];
      b_all += bound[h]; ext_all += hc[kCntExt]; shd_all += hc[kCntShd];
    }
    const auto now = std::chrono::steady_clock::now();
    if (wave == 0) {
      t0 = now;
      tail = tail_paths(b_all, p.opaque != 0) / parts;
    }
    c->wave_log.insert(c->wave_log.end(), {b_all, ext_all, shd_all,
                                           int(std::chrono::duration_cast<std::chrono::microseconds>(now - t0).count())});
    bool all_done = true;
    for (int h = 0; h < parts; ++h) {
      if (done[h]) continue;
      if (bound[h] == 0) { done[h] = true; continue; }
      if (bound[h] <= tail) {
        NvtxRange tail_range(stage_name(RM_STAGE_WF_TAIL));
        e = staged2_on(c, RM_STAGE_WF_TAIL, sts[h], [&] {
          // the tail's traversals are counted with the tail (both kinds in its slot)
          return launch_wavefront_tail(s, p, c->gb.view(), w, q[h][cur[h]], bound[h], c->hdr.as<float>(),
                                       c->dbg.as<uint32_t>(), ctr + 4 * RM_STAGE_WF_SHADE, ctr + 4 * RM_STAGE_WF_TAIL,
                                       ctr + 4 * RM_STAGE_WF_TAIL, err, sts[h]);
        });
        if (e != cudaSuccess) { msg = cuda_msg("wavefront tail failed", e); return e; }
        done[h] = true;
      }
      all_done = all_done && done[h];
    }
    if (all_done) break;
    for (int k = 0; k < kBatch; ++k) {
      c->waves++;
      for (int h = 0; h < parts; ++h) {
        if (done[h]) continue;
        const WfQueues& Q = q[h][cur[h]];
        const WfQueues& N = q[h][cur[h] ^ 1];
        const cudaStream_t st = sts[h];
        const int bd = bound[h];
        if (merged && !s.wnodes) {
          // both traversals in one launch (timed as the extension stage)
          e = staged2_on(c, RM_STAGE_WF_EXTEND, st, [&] {
            return launch_wavefront_trace2(s, w, Q, bd, ctr + 4 * RM_STAGE_WF_EXTEND, ctr + 4 * RM_STAGE_WF_SHADOW,
                                           err, N.counts, st);
          });
        } else {
          e = staged2_on(c, RM_STAGE_WF_EXTEND, st, [&] {
            return launch_wavefront_trace(s, w, Q, bd, false, ctr + 4 * RM_STAGE_WF_EXTEND, err, st);
          });
          if (e == cudaSuccess)
            e = staged2_on(c, RM_STAGE_WF_SHADOW, st, [&] {
              return launch_wavefront_trace(s, w, Q, bd, true, ctr + 4 * RM_STAGE_WF_SHADOW, err, st);
            });
        }
        // (k_wf_trace2 zeroes the next wave's queue lengths itself)
        if (e == cudaSuccess && !(merged && !s.wnodes)) e = cudaMemsetAsync(N.counts, 0, kCntSlots * sizeof(int), st);
        if (merged) {
          if (e == cudaSuccess)
            e = staged2_on(c, RM_STAGE_WF_SHADE, st, [&] {
              return launch_wavefront_shade3(s, p, c->gb.view(), w, Q, bd, N, c->hdr.as<float>(),
                                             c->dbg.as<uint32_t>(), ctr + 4 * RM_STAGE_WF_SHADE, err, st);
            });
        } else {
          for (int vk = 0; vk < 3 && e == cudaSuccess; ++vk)
            e = staged2_on(c, RM_STAGE_WF_SHADE, st, [&] {
              return launch_wavefront_shade(vk, s, p, c->gb.view(), w, Q, bd, N, c->hdr.as<float>(),
                                            c->dbg.as<uint32_t>(), ctr + 4 * RM_STAGE_WF_SHADE, err, st);
            });
        }
        if (e != cudaSuccess) { msg = cuda_msg("wavefront launch failed", e); return e; }
        cur[h] ^= 1;
      }
    }
  }
  // join: the frame's later stages on the context stream wait for every part
  for (int h = 1; h < parts; ++h)
    if ((e = cudaEventRecord(c->ev_join[h - 1], sts[h])) != cudaSuccess ||
        (e = cudaStreamWaitEvent(c->stream, c->ev_join[h - 1], 0)) != cudaSuccess) {
      msg = cuda_msg("stream join failed", e);
      return e;
    }
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) { msg = cuda_msg("wavefront tail failed", e); return e; }
  // the end of the loop (the tails included), as a last record with empty queues
  c->wave_log.insert(c->wave_log.end(), {0, 0, 0, int(std::chrono::duration_cast<std::chrono::microseconds>(
                                                          std::chrono::steady_clock::now() - t0).count())});
  return cudaSuccess;
}

cudaError_t ensure_frame(rmcuda_ctx* c, size_t npix, bool restir) {
  cudaError_t e;
  if ((e = c->hdr.reserve(npix * 12)) != cudaSuccess || (e = c->rgb.reserve(npix * 3)) != cudaSuccess ||
      (e = c->dbg.reserve(npix * 8)) != cudaSuccess)
    return e;
  if (restir) {
    if ((e = c->gb.reserve(npix)) != cudaSuccess || (e = c->rinit.reserve(npix)) != cudaSuccess ||
        (e = c->rmerged.reserve(npix)) != cudaSuccess || (e = c->tmp_a.reserve(npix * 12)) != cudaSuccess ||
        (e = c->tmp_b.reserve(npix * 12)) != cudaSuccess ||
        (e = c->hist_col.reserve(npix * 12)) != cudaSuccess || (e = c->hg.reserve(npix)) != cudaSuccess ||
        (e = c->hres.reserve(npix)) != cudaSuccess)
      return e;
  }
  return cudaSuccess;
}

// Enqueue one frame of the resident scene.  d_rgb (device) receives the
// image; the final linear radiance stays in c->last_final.
int enqueue_frame(rmcuda_ctx* c, DevScene& sc, const rm_camera& cam, const rm_config& cfg, uint64_t seed, uint8_t* d_rgb,
                  std::string& msg) {
  NvtxRange range("rm frame");
  if (cfg.width <= 0 || cfg.height <= 0 || cfg.spp <= 0 || cfg.max_bounces < 0 ||
      size_t(cfg.width) * size_t(cfg.height) > 100000000) {
    msg = kInvalidDims;
    return RM_ERR_INVALID;
  }
  if (!sc.have_scene) { msg = "no resident scene"; return RM_ERR_INVALID; }
  Plan pl = make_plan(sc, cam, cfg);
  Params& p = pl.p;
  const size_t npix = size_t(cfg.width) * size_t(cfg.height);
  cudaStream_t st = c->stream;
  cudaError_t e = ensure_frame(c, npix, pl.use_spatial);
  if (e != cudaSuccess) {
    msg = cuda_msg(pl.use_spatial ? "Metal ReSTIR buffer allocation failed" : "Metal image buffer allocation failed", e);
    return RM_ERR_ALLOC;
  }
  Scene s = scene_view(sc);
  unsigned long long* ctr = c->ctr.as<unsigned long long>();
  uint32_t* err = c->err.as<uint32_t>();
  if (!pl.use_spatial) {
    c->last_chain = pl.lanes;
    e = staged(c, RM_STAGE_PLAIN, [&] {
      return launch_render_paths(pl.lanes, s, p, seed, c->hdr.as<float>(), d_rgb, c->dbg.as<uint32_t>(),
                                 ctr + 4 * RM_STAGE_PLAIN, err, st);
    });
    if (e != cudaSuccess) { msg = cuda_msg("render_paths launch failed", e); return RM_ERR_CUDA; }
    c->last_final = c->hdr.as<float>();
  } else {
    c->last_chain = 2;
    // scene hash over the uploaded triangle bytes (metal.mm:241-248)
    if ((e = c->hash_out.reserve(8)) != cudaSuccess) { msg = cuda_msg("hash buffer", e); return RM_ERR_ALLOC; }
    e = staged(c, RM_STAGE_HASH, [&] {
      return device_hash(sc.tris.ptr, size_t(sc.n_tris) * sizeof(rm_triangle), c->hash_out.as<unsigned long long>(), st);
    });
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, c->hash_out.ptr, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { msg = cuda_msg("scene hash failed", e); return RM_ERR_CUDA; }
    uint32_t lt_bits;
    std::memcpy(&lt_bits, &sc.light_total, 4);
    h ^= uint64_t(sc.n_tris) * 0x9E3779B97F4A7C15ull ^ uint64_t(sc.n_lights) * 0xBF58476D1CE4E5B9ull ^
         uint64_t(lt_bits) * 0x94D049BB133111EBull;
    const bool animated = (cfg.flags & RM_FLAG_ANIMATED_HISTORY) != 0;
    bool have_hist = c->hist_valid && c->hist_w == cfg.width && c->hist_h == cfg.height && c->have_hist_bufs &&
                     seed != c->hist_seed && (animated || h == c->hist_hash);
    if (pl.temporal_off) have_hist = false;
    p.hasHistory = have_hist ? 1 : 0;
    p.prevCamera = c->hist_cam;
    const bool wavefront = !use_megakernel();  // ReSTIR scenes are opaque (make_plan)
    for (int stage = 0; stage < 3 && e == cudaSuccess; ++stage) {
      if (stage == 2 && wavefront) {
        std::string wmsg;
        cudaEvent_t a = nullptr, b = nullptr;
        if (c->profiling == 1 && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
          cudaEventRecord(a, st);
        e = run_wavefront_shade(c, s, p, seed, wmsg);
        if (a && b) {
          cudaEventRecord(b, st);
          c->pending.push_back({RM_STAGE_SHADE, a, b});
        }
        if (e != cudaSuccess) { msg = wmsg; return RM_ERR_CUDA; }
        continue;
      }
      e = staged(c, RM_STAGE_GENERATE + stage, [&] {
        return launch_restir_stage(stage, s, p, seed, c->gb.view(), c->rinit.view(), c->rmerged.view(), c->hg.view(),
                                   c->hres.view(), c->hdr.as<float>(), c->dbg.as<uint32_t>(),
                                   ctr + 4 * (RM_STAGE_GENERATE + stage), err, st);
      });
    }
    if (e != cudaSuccess) { msg = cuda_msg("ReSTIR launch failed", e); return RM_ERR_CUDA; }
    if (pl.denoise) {
      // temporal(hdr, hist_col) -> tmp_a -> a-trous -> tmp_b -> a-trous + tonemap -> tmp_a
      float* ins[3] = {c->hdr.as<float>(), c->tmp_a.as<float>(), c->tmp_b.as<float>()};
      float* outs[3] = {c->tmp_a.as<float>(), c->tmp_b.as<float>(), c->tmp_a.as<float>()};
      for (int stage = 0; stage < 3 && e == cudaSuccess; ++stage)
        e = staged(c, RM_STAGE_TEMPORAL + stage, [&] {
          return launch_denoise_stage(stage, p, c->gb.view(), c->hg.view(), ins[stage], c->hist_col.as<float>(),
                                      outs[stage], stage == 2 ? d_rgb : nullptr, st);
        });
      if (e != cudaSuccess) { msg = cuda_msg("denoise launch failed", e); return RM_ERR_CUDA; }
      c->last_final = c->tmp_a.as<float>();
    } else {
      if (d_rgb) {
        e = staged(c, RM_STAGE_TONEMAP, [&] { return launch_tonemap(c->hdr.as<float>(), d_rgb, uint32_t(npix), st); });
        if (e != cudaSuccess) { msg = cuda_msg("tonemap launch failed", e); return RM_ERR_CUDA; }
      }
      c->last_final = c->hdr.as<float>();
    }
    // publish history (metal.mm:374-385); buffers swap by ownership
    std::swap(c->gb, c->hg);
    std::swap(c->rmerged, c->hres);
    if (pl.denoise) { std::swap(c->tmp_a, c->hist_col); c->last_final = c->hist_col.as<float>(); }
    c->have_hist_bufs = true;
    c->hist_cam = cam;
    c->hist_w = cfg.width; c->hist_h = cfg.height;
    c->hist_seed = seed; c->hist_hash = h;
    c->hist_valid = true;
    c->hist_scene = &sc; c->hist_cfg = cfg; c->hist_denoised = pl.denoise;
    c->hist_had_history = p.hasHistory != 0; c->hist_prev_cam = p.prevCamera;
  }
  c->last_w = cfg.width;
  c->last_h = cfg.height;
  c->frames++;
  return RM_OK;
}

int check_device_error(rmcuda_ctx* c, std::string& msg) {
  uint32_t dev_err = 0;
  cudaError_t e = cudaMemcpyAsync(&dev_err, c->err.ptr, 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { msg = cuda_msg("Metal command buffer failed", e); return RM_ERR_CUDA; }
  if (dev_err) {
    cudaMemsetAsync(c->err.ptr, 0, 4, c->stream);
    msg = "device error word " + std::to_string(dev_err) +
          " (1: traversal stack exceeded, 2: transparent crossings exceeded, 8: a pixel's step bound exceeded, "
          "4: index out of bounds in the checked "
          "build, with bit 8 + n for the check that fired: 0 BVH node, 1 leaf range, 2 wide leaf, 3 hit triangle, "
          "4 texel, 5 light, 6 shading queue, 7 tail queue, 8 vertex triangle)";
    return RM_ERR_DEVICE;
  }
  return RM_OK;
}

}  // namespace rmapi

extern "C" {

const char* rmcuda_version(void) { return "rmcuda 0.1 (sm_100a)"; }

int rmcuda_create(rmcuda_ctx** out, int device, char* err, size_t errcap) {
  if (!out) { set_err(err, errcap, "null output pointer"); return RM_ERR_INVALID; }
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
    cudaGetLastError();
    set_err(err, errcap, kUnavailable);
    return RM_ERR_UNAVAILABLE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    set_err(err, errcap, kUnavailable);
    return RM_ERR_UNAVAILABLE;
  }
  auto* c = new rmcuda_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = c->ctr.reserve(RM_STAGE_COUNT * 32);
  if (e == cudaSuccess) e = c->err.reserve(4);
  if (e == cudaSuccess) e = cudaMemset(c->ctr.ptr, 0, RM_STAGE_COUNT * 32);
  if (e == cudaSuccess) e = cudaMemset(c->err.ptr, 0, 4);
  if (e != cudaSuccess) {
    set_err(err, errcap, cuda_msg("context creation failed", e));
    delete c;
    return RM_ERR_CUDA;
  }
  c->stream = c->own;
  *out = c;
  return RM_OK;
}

void rmcuda_destroy(rmcuda_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->sc.release();
  c->batch.release();
  for (DevBuf* b : {&c->hdr, &c->tmp_a, &c->tmp_b, &c->hist_col, &c->rgb, &c->dbg, &c->hash_out, &c->ctr, &c->err,
                    &c->adj_scratch, &c->differ, &c->ctr_save})
    b->release();
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  for (int h = 0; h < kWfParts - 1; ++h) {
    if (c->side_stream[h]) cudaStreamDestroy(c->side_stream[h]);
    if (c->ev_join[h]) cudaEventDestroy(c->ev_join[h]);
  }
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->h_differ) cudaFreeHost(c->h_differ);
  for (DevBuf& b : c->wf) b.release();
  for (DevBuf& b : c->wq) b.release();
  if (c->h_counts) cudaFreeHost(c->h_counts);
  for (auto& row : c->ev_counts)
    for (cudaEvent_t ev : row)
      if (ev) cudaEventDestroy(ev);
  for (auto& m : c->models) m.tris.release();
  for (DevBuf* b : {&c->prep_inst, &c->prep_mptr, &c->prep_start, &c->prep_keep, &c->prep_kscan, &c->prep_light,
                    &c->prep_lscan, &c->prep_temp, &c->prep_weight, &c->prep_small})
    b->release();
  if (c->h_prep) cudaFreeHost(c->h_prep);
  if (c->h_preview) cudaFreeHost(c->h_preview);
  c->gb.release(); c->hg.release();
  c->rinit.release(); c->rmerged.release(); c->hres.release();
  resolve_pending(c);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

int rmcuda_set_stream(rmcuda_ctx* c, void* s, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStreamSynchronize(c->stream);
  c->stream = s ? static_cast<cudaStream_t>(s) : c->own;
  return RM_OK;
}

int rmcuda_scene_upload(rmcuda_ctx* c, const rm_scene_view* sv, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::string msg;
  int rc = upload_scene(c, c->sc, sv, msg);
  if (rc == RM_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { msg = cuda_msg("scene upload failed", e); rc = RM_ERR_CUDA; }
  }
  if (rc != RM_OK) { c->hist_valid = false; set_err(err, errcap, msg); }
  return rc;
}

int rmcuda_scene_update(rmcuda_ctx* c, const rm_triangle* tris, int32_t n, int32_t rebuild_every, char* err,
                        size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->sc.have_scene || n != c->sc.n_tris || (n > 0 && !tris)) {
    set_err(err, errcap, "scene update needs a resident scene with the same triangle count");
    return RM_ERR_INVALID;
  }
  c->sc.validated_texels = -1;
  cudaError_t e = cudaMemcpyAsync(c->sc.tris.ptr, tris, size_t(n) * sizeof(rm_triangle), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("scene update upload failed", e)); return RM_ERR_CUDA; }
  bool opaque = true;
  for (int i = 0; i < n; ++i)
    if (!(tris[i].alpha >= 1.0f)) { opaque = false; break; }
  c->sc.opaque = opaque;
  if (n == 0) return RM_OK;
  e = prepare_lights(c->sc.tris.as<rm_triangle>(), c->sc.lights.as<int32_t>(), c->sc.cdf.as<float>(), c->sc.n_lights,
                     c->sc.light_total, c->sc.lrec, c->sc.guide, c->sc.guide_n, c->sc.guide_inv, c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("light preparation failed", e)); return RM_ERR_CUDA; }
  if (rebuild_every > 0 && c->sc.refits + 1 >= rebuild_every) {
    std::string berr;
    e = build_device_bvh(c->sc.tris.as<rm_triangle>(), n, c->sc.bvh, c->stream, berr);
    c->sc.refits = 0;
    c->sc.device_built = true;
    c->bvh_builds++;
    if (e != cudaSuccess) { set_err(err, errcap, berr.empty() ? cuda_msg("rebuild failed", e) : berr); return RM_ERR_CUDA; }
  } else {
    e = refit_bvh(c->sc.tris.as<rm_triangle>(), c->sc.bvh, c->stream);
    c->sc.refits++;
    c->bvh_refits++;
    if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("refit failed", e)); return RM_ERR_CUDA; }
  }
  // the wide nodes are collapsed again from the refitted or rebuilt records
  if ((e = finish_wide(c->sc.bvh, c->stream)) != cudaSuccess) {
    set_err(err, errcap, cuda_msg("wide BVH build failed", e));
    return RM_ERR_CUDA;
  }
  return RM_OK;
}

int rmcuda_model_create(rmcuda_ctx* c, const rm_model_tri* tris, int32_t n, int32_t* model_id, char* err,
                        size_t errcap) {
  if (!c || !model_id || n < 0 || (n > 0 && !tris)) { set_err(err, errcap, "invalid model"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  rmcuda_ctx::Model m;
  cudaError_t e = m.tris.reserve(size_t(std::max(n, 1)) * sizeof(rm_model_tri));
  if (e == cudaSuccess && n > 0)
    e = cudaMemcpyAsync(m.tris.ptr, tris, size_t(n) * sizeof(rm_model_tri), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // the caller may free `tris` on return
  if (e != cudaSuccess) {
    m.tris.release();
    set_err(err, errcap, cuda_msg("model upload failed", e));
    return RM_ERR_CUDA;
  }
  m.n = n;
  c->models.push_back(std::move(m));
  *model_id = int32_t(c->models.size() - 1);
  return RM_OK;
}

int rmcuda_model_update(rmcuda_ctx* c, int32_t id, const rm_model_tri* tris, int32_t n, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (id < 0 || size_t(id) >= c->models.size() || n != c->models[size_t(id)].n || (n > 0 && !tris)) {
    set_err(err, errcap, "model update needs an existing model and the same triangle count");
    return RM_ERR_INVALID;
  }
  cudaError_t e = n > 0 ? cudaMemcpyAsync(c->models[size_t(id)].tris.ptr, tris, size_t(n) * sizeof(rm_model_tri),
                                          cudaMemcpyHostToDevice, c->stream)
                        : cudaSuccess;
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("model update failed", e)); return RM_ERR_CUDA; }
  return RM_OK;
}

// Objects::render's scene step (runtime.hpp:121-131) on the device: the world
// of the instances (rm_prep.cu), then refit or build (bvh.cpp:250-272 falls
// back to a build when the triangle count changed).
int rmcuda_instances_commit(rmcuda_ctx* c, const rm_instance* inst, int32_t n, int32_t rebuild_every, char* err,
                            size_t errcap) {
  if (!c || n < 0 || (n > 0 && !inst)) { set_err(err, errcap, "invalid instance list"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::vector<int> start(static_cast<size_t>(n) + 1, 0), topo(static_cast<size_t>(n));
  std::vector<const rm_model_tri*> mptr(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    const rm_instance& in = inst[i];
    if (in.model < 0 || size_t(in.model) >= c->models.size()) { set_err(err, errcap, "null object"); return RM_ERR_INVALID; }
    if (in.scale[0] == 0 || in.scale[1] == 0 || in.scale[2] == 0) {
      set_err(err, errcap, "scale must be nonzero");  // Objects::push, runtime.hpp:80
      return RM_ERR_INVALID;
    }
    const auto& m = c->models[size_t(in.model)];
    if (int64_t(start[size_t(i)]) + m.n > int64_t(1) << 30) { set_err(err, errcap, "too many triangles"); return RM_ERR_INVALID; }
    start[size_t(i) + 1] = start[size_t(i)] + m.n;
    topo[size_t(i)] = in.model;
    mptr[size_t(i)] = m.tris.as<rm_model_tri>();
  }
  const int total = start[size_t(n)];
  cudaStream_t st = c->stream;
  cudaError_t e;
  size_t scan_bytes = 0;
  c->sc.validated_texels = -1;  // the world triangles are rewritten below
  const size_t slots = size_t(std::max(total, 1));
  if ((e = prep_scan_bytes(total, scan_bytes)) != cudaSuccess ||
      (e = c->prep_inst.reserve(size_t(std::max(n, 1)) * sizeof(rm_instance))) != cudaSuccess ||
      (e = c->prep_mptr.reserve(size_t(std::max(n, 1)) * sizeof(void*))) != cudaSuccess ||
      (e = c->prep_start.reserve((size_t(n) + 1) * sizeof(int))) != cudaSuccess ||
      (e = c->prep_keep.reserve(slots * 4)) != cudaSuccess || (e = c->prep_kscan.reserve(slots * 4)) != cudaSuccess ||
      (e = c->prep_light.reserve(slots * 4)) != cudaSuccess || (e = c->prep_lscan.reserve(slots * 4)) != cudaSuccess ||
      (e = c->prep_temp.reserve(std::max<size_t>(scan_bytes, 16))) != cudaSuccess ||
      (e = c->prep_weight.reserve(slots * 8)) != cudaSuccess || (e = c->prep_small.reserve(64)) != cudaSuccess ||
      (e = c->sc.tris.reserve(slots * sizeof(rm_triangle))) != cudaSuccess ||
      (e = c->sc.lights.reserve(slots * 4)) != cudaSuccess || (e = c->sc.cdf.reserve(slots * 4)) != cudaSuccess ||
      (!c->h_prep && (e = cudaMallocHost(&c->h_prep, 64)) != cudaSuccess)) {
    set_err(err, errcap, cuda_msg("scene preparation allocation failed", e));
    return RM_ERR_ALLOC;
  }
  // the previous commit's kernels may still read these buffers: stream order keeps them apart
  if ((n > 0 && ((e = cudaMemcpyAsync(c->prep_inst.ptr, inst, size_t(n) * sizeof(rm_instance), cudaMemcpyHostToDevice,
                                      st)) != cudaSuccess ||
                 (e = cudaMemcpyAsync(c->prep_mptr.ptr, mptr.data(), size_t(n) * sizeof(void*), cudaMemcpyHostToDevice,
                                      st)) != cudaSuccess)) ||
      (e = cudaMemcpyAsync(c->prep_start.ptr, start.data(), (size_t(n) + 1) * sizeof(int), cudaMemcpyHostToDevice,
                           st)) != cudaSuccess) {
    set_err(err, errcap, cuda_msg("instance upload failed", e));
    return RM_ERR_CUDA;
  }
  int* small = c->prep_small.as<int>();
  rmd::PrepArgs a{c->prep_inst.as<rm_instance>(), c->prep_mptr.as<const rm_model_tri* const>(), c->prep_start.as<int>(),
                  n, total, c->prep_keep.as<int>(), c->prep_kscan.as<int>(), c->prep_light.as<int>(),
                  c->prep_lscan.as<int>(), c->prep_temp.ptr, scan_bytes, c->sc.tris.as<rm_triangle>(),
                  c->sc.lights.as<int32_t>(), c->prep_weight.as<double>(), c->sc.cdf.as<float>(), small,
                  reinterpret_cast<double*>(small + 4), small + 2};
  if ((e = staged(c, RM_STAGE_PREP, [&] { return rmd::prep_world(a, st); })) != cudaSuccess ||
      (e = cudaMemcpyAsync(c->h_prep, small, 32, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess) {
    set_err(err, errcap, cuda_msg("scene preparation failed", e));
    return RM_ERR_CUDA;
  }
  const int* hc = static_cast<const int*>(c->h_prep);
  double total_w = 0;
  std::memcpy(&total_w, static_cast<const char*>(c->h_prep) + 16, 8);
  const int n_tris = hc[0];
  const bool same = c->sc.have_scene && topo == c->prep_topology && n_tris == c->sc.n_tris && c->sc.device_built;
  c->sc.n_tris = n_tris;
  c->sc.n_lights = hc[1];
  c->sc.light_total = float(total_w);
  c->sc.opaque = hc[2] != 0;
  c->sc.have_scene = false;
  if ((e = prepare_lights(c->sc.tris.as<rm_triangle>(), c->sc.lights.as<int32_t>(), c->sc.cdf.as<float>(),
                          c->sc.n_lights, c->sc.light_total, c->sc.lrec, c->sc.guide, c->sc.guide_n, c->sc.guide_inv,
                          st)) != cudaSuccess) {
    set_err(err, errcap, cuda_msg("light preparation failed", e));
    return RM_ERR_CUDA;
  }
  const bool refit = same && n_tris > 0 && !(rebuild_every > 0 && c->prep_commits % uint64_t(rebuild_every) == 0);
  if (n_tris == 0) {
    c->sc.bvh.n_records = 0;
    c->sc.bvh.n_tris = 0;
  } else if (refit) {
    e = staged(c, RM_STAGE_PREP, [&] { return refit_bvh(c->sc.tris.as<rm_triangle>(), c->sc.bvh, st); });
    c->sc.refits++;
    c->bvh_refits++;
    if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("refit failed", e)); return RM_ERR_CUDA; }
  } else {
    std::string berr;
    e = staged(c, RM_STAGE_PREP,
               [&] { return build_device_bvh(c->sc.tris.as<rm_triangle>(), n_tris, c->sc.bvh, st, berr); });
    c->sc.refits = 0;
    c->bvh_builds++;
    if (e != cudaSuccess) { set_err(err, errcap, berr.empty() ? cuda_msg("BVH build failed", e) : berr); return RM_ERR_CUDA; }
  }
  if ((e = finish_wide(c->sc.bvh, st)) != cudaSuccess) {
    set_err(err, errcap, cuda_msg("wide BVH build failed", e));
    return RM_ERR_CUDA;
  }
  c->sc.device_built = true;
  c->sc.have_scene = true;
  c->prep_topology = std::move(topo);
  c->prep_commits++;
  return RM_OK;
}

int rmcuda_scene_read(rmcuda_ctx* c, rm_triangle* tris, int32_t tri_cap, int32_t* light_tri, float* light_cdf,
                      int32_t light_cap, int32_t* counts, float* light_total, char* err, size_t errcap) {
  if (!c || tri_cap < 0 || light_cap < 0) { set_err(err, errcap, "invalid arguments"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->sc.have_scene) { set_err(err, errcap, "no resident scene"); return RM_ERR_INVALID; }
  const size_t nt = size_t(std::min(tri_cap, int32_t(c->sc.n_tris)));
  const size_t nl = size_t(std::min(light_cap, int32_t(c->sc.n_lights)));
  cudaError_t e = cudaSuccess;
  if (tris && nt) e = cudaMemcpyAsync(tris, c->sc.tris.ptr, nt * sizeof(rm_triangle), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && light_tri && nl)
    e = cudaMemcpyAsync(light_tri, c->sc.lights.ptr, nl * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && light_cdf && nl)
    e = cudaMemcpyAsync(light_cdf, c->sc.cdf.ptr, nl * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("scene read failed", e)); return RM_ERR_CUDA; }
  if (counts) { counts[0] = c->sc.n_tris; counts[1] = c->sc.n_lights; }
  if (light_total) *light_total = c->sc.light_total;
  return RM_OK;
}

int rmcuda_render_resident_async(rmcuda_ctx* c, const rm_camera* cam, const rm_config* cfg, uint64_t seed,
                                 uint8_t* d_rgb, float* d_hdr, char* err, size_t errcap) {
  if (!c || !cam || !cfg) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::string msg;
  int rc = enqueue_frame(c, c->sc, *cam, *cfg, seed, d_rgb, msg);
  if (rc == RM_OK && d_hdr) {
    const size_t bytes = size_t(cfg->width) * size_t(cfg->height) * 12;
    cudaError_t e = cudaMemcpyAsync(d_hdr, c->last_final, bytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) { msg = cuda_msg("hdr copy failed", e); rc = RM_ERR_CUDA; }
  }
  if (rc != RM_OK) { c->hist_valid = false; set_err(err, errcap, msg); }
  return rc;
}

int rmcuda_sync(rmcuda_ctx* c, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::string msg;
  int rc = check_device_error(c, msg);
  if (rc != RM_OK) { c->hist_valid = false; set_err(err, errcap, msg); }
  return rc;
}

}  // extern "C"

namespace {

// What a frame changes on the host side of the context, and the buffers its
// history swap exchanges: enough to undo a speculative frame.
struct FrameSnap {
  rmapi::GBufSet gb, hg;
  rmapi::ResSet rmerged, hres;
  rmd::DevBuf tmp_a, hist_col;
  rm_camera hist_cam, hist_prev_cam;
  int hist_w, hist_h, last_chain, last_w, last_h;
  uint64_t hist_seed, frames, launches, waves;
  unsigned long long hist_hash;
  bool hist_valid, have_hist_bufs, hist_denoised, hist_had_history;
  const void* hist_scene;
  rm_config hist_cfg;
  float* last_final;
  size_t pending;
  std::vector<int> wave_log;
};

FrameSnap take_snap(rmcuda_ctx* c) {
  return FrameSnap{c->gb, c->hg, c->rmerged, c->hres, c->tmp_a, c->hist_col, c->hist_cam, c->hist_prev_cam,
                   c->hist_w, c->hist_h, c->last_chain, c->last_w, c->last_h, c->hist_seed, c->frames, c->launches,
                   c->waves, c->hist_hash, c->hist_valid, c->have_hist_bufs, c->hist_denoised, c->hist_had_history,
                   c->hist_scene, c->hist_cfg, c->last_final, c->pending.size(), c->wave_log};
}

void restore_snap(rmcuda_ctx* c, const FrameSnap& s) {
  c->gb = s.gb; c->hg = s.hg; c->rmerged = s.rmerged; c->hres = s.hres; c->tmp_a = s.tmp_a; c->hist_col = s.hist_col;
  c->hist_cam = s.hist_cam; c->hist_prev_cam = s.hist_prev_cam; c->hist_w = s.hist_w; c->hist_h = s.hist_h;
  c->last_chain = s.last_chain; c->last_w = s.last_w; c->last_h = s.last_h; c->hist_seed = s.hist_seed;
  c->frames = s.frames; c->launches = s.launches; c->waves = s.waves; c->hist_hash = s.hist_hash;
  c->hist_valid = s.hist_valid; c->have_hist_bufs = s.have_hist_bufs; c->hist_denoised = s.hist_denoised;
  c->hist_had_history = s.hist_had_history; c->hist_scene = s.hist_scene; c->hist_cfg = s.hist_cfg;
  c->last_final = s.last_final;
  for (size_t i = s.pending; i < c->pending.size(); ++i) {
    cudaEventDestroy(c->pending[i].a);
    cudaEventDestroy(c->pending[i].b);
  }
  c->pending.resize(s.pending);
  c->wave_log = s.wave_log;
}

// A re-upload of the resident scene is rendered speculatively when nothing but
// its triangles could have changed since the last frame: the same device-built
// BVH settings and triangle count, light list, CDF, light total and texels
// equal to the host copies of the last upload (the small arrays are compared
// on the host and not sent), triangles that equalled the resident ones on the
// last upload, and the same configuration as the last frame (so that no frame
// buffer is reallocated and the frame can be undone by restoring the host
// state).  RAYMOTION_CUDA_SPECULATE=0 turns it off.
bool may_speculate(rmcuda_ctx* c, const rm_scene_view* sv, const rm_config& cfg) {
  const char* v = std::getenv("RAYMOTION_CUDA_SPECULATE");
  if (v && v[0] == '0') return false;
  const rmapi::DevScene& sc = c->sc;
  if (!sv || !sv->tris || !sc.have_scene || !sc.device_built || sv->nodes || sv->n_tris <= 0 ||
      sv->n_tris != sc.n_tris || sc.bvh.n_records <= 0 || !sc.h_valid || !sc.last_upload_equal ||
      sc.validated_texels != int64_t(sv->n_texels) || !c->have_last_cfg ||
      std::memcmp(&c->last_cfg, &cfg, sizeof(cfg)) != 0)
    return false;
  std::string key;
  for (const char* k : {"RAYMOTION_CUDA_BVH", "RAYMOTION_CUDA_BVH_LEAF", "RAYMOTION_CUDA_WIDE"}) {
    const char* e = std::getenv(k);
    key += e ? e : "-";
    key += '|';
  }
  if (key != sc.build_key) return false;
  if (sv->n_lights < 0 || sv->n_texels < 0 || size_t(sv->n_lights) != sc.h_lights.size() ||
      size_t(sv->n_texels) != sc.h_texels.size())
    return false;
  if (std::memcmp(&sv->light_total, &sc.h_light_total, sizeof(float)) != 0) return false;
  if (sv->n_lights && (!sv->light_tri || !sv->light_cdf ||
                       std::memcmp(sv->light_tri, sc.h_lights.data(), size_t(sv->n_lights) * 4) != 0 ||
                       std::memcmp(sv->light_cdf, sc.h_cdf.data(), size_t(sv->n_lights) * 4) != 0))
    return false;
  if (sv->n_texels && (!sv->texels ||
                       std::memcmp(sv->texels, sc.h_texels.data(), size_t(sv->n_texels) * sizeof(rm_vec3)) != 0))
    return false;
  return true;
}

// The speculative frame: the triangles go to the staging buffer on the copy
// stream (from a helper thread, so that a pageable host array does not hold
// up the launches) and are compared with the resident ones there, while the
// frame renders the resident scene.  Equal bytes: the frame stands (true).
// Different bytes, or any failure: the frame is undone (history, counters,
// host state) and false is returned, and the caller renders the upload the
// ordinary way.
bool speculative_frame(rmcuda_ctx* c, const rm_scene_view* sv, const rm_camera& cam, const rm_config& cfg,
                       uint64_t seed) {
  NvtxRange range("rm speculative frame");
  rmapi::DevScene& sc = c->sc;
  const size_t tb = size_t(sv->n_tris) * sizeof(rm_triangle);
  if (!c->copy_stream && cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    c->copy_stream = nullptr;
    return false;
  }
  if (!c->h_differ && cudaMallocHost(reinterpret_cast<void**>(&c->h_differ), sizeof(int)) != cudaSuccess) {
    c->h_differ = nullptr;
    return false;
  }
  if (sc.tris_in.reserve(tb) != cudaSuccess || c->differ.reserve(16) != cudaSuccess ||
      c->ctr_save.reserve(RM_STAGE_COUNT * 32) != cudaSuccess)
    return false;
  if (cudaMemcpyAsync(c->ctr_save.ptr, c->ctr.ptr, RM_STAGE_COUNT * 32, cudaMemcpyDeviceToDevice, c->stream) !=
      cudaSuccess)
    return false;
  const FrameSnap snap = take_snap(c);
  *c->h_differ = 1;
  cudaError_t ce = cudaSuccess;
  std::thread copier([&] {
    ce = cudaSetDevice(c->device);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(sc.tris_in.ptr, sv->tris, tb, cudaMemcpyHostToDevice, c->copy_stream);
    if (ce == cudaSuccess) ce = rmd::device_differ(sc.tris_in.ptr, sc.tris.ptr, tb, c->differ.as<int>(), c->copy_stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(c->h_differ, c->differ.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->copy_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(c->copy_stream);
  });
  std::string msg;
  const int rc = rmapi::enqueue_frame(c, sc, cam, cfg, seed, c->rgb.as<uint8_t>(), msg);
  copier.join();
  if (rc == RM_OK && ce == cudaSuccess && *c->h_differ == 0) {
    sc.reuses++;
    return true;
  }
  // undo: the frame's work is discarded once it has finished
  cudaStreamSynchronize(c->stream);
  cudaGetLastError();
  restore_snap(c, snap);
  cudaMemcpyAsync(c->ctr.ptr, c->ctr_save.ptr, RM_STAGE_COUNT * 32, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemsetAsync(c->err.ptr, 0, 4, c->stream);
  return false;
}

}  // namespace

extern "C" {

int rmcuda_render(rmcuda_ctx* c, const rm_scene_view* sv, const rm_camera* cam, const rm_config* cfg, uint64_t seed,
                  uint8_t* rgb, size_t rgb_cap, float* hdr, char* err, size_t errcap) {
  if (!cfg || cfg->width <= 0 || cfg->height <= 0 || cfg->spp <= 0 || cfg->max_bounces < 0 ||
      size_t(cfg->width) * size_t(cfg->height) > 100000000) {
    set_err(err, errcap, kInvalidDims);
    return RM_ERR_INVALID;
  }
  if (!c || !sv || !cam) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  const size_t npix = size_t(cfg->width) * size_t(cfg->height);
  if (rgb && rgb_cap < npix * 3) { set_err(err, errcap, "rgb buffer too small"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  NvtxRange range("rmcuda_render");
  std::string msg;
  int rc = RM_OK;
  // an unchanged re-upload (the reference re-uploads every frame,
  // metal.mm:171-186) renders while its triangles are sent and compared
  const bool done = c->rgb.cap >= npix * 3 && may_speculate(c, sv, *cfg) && speculative_frame(c, sv, *cam, *cfg, seed);
  if (!done) {
    rc = upload_scene(c, c->sc, sv, msg);
    if (rc == RM_OK) {
      cudaError_t e = c->rgb.reserve(npix * 3);
      if (e != cudaSuccess) { msg = cuda_msg("Metal image buffer allocation failed", e); rc = RM_ERR_ALLOC; }
    }
    if (rc == RM_OK) rc = enqueue_frame(c, c->sc, *cam, *cfg, seed, c->rgb.as<uint8_t>(), msg);
  }
  if (rc == RM_OK) { c->last_cfg = *cfg; c->have_last_cfg = true; }
  if (rc == RM_OK) {
    cudaError_t e = cudaSuccess;
    if (rgb) e = cudaMemcpyAsync(rgb, c->rgb.ptr, npix * 3, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && hdr) e = cudaMemcpyAsync(hdr, c->last_final, npix * 12, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) { msg = cuda_msg("image readback failed", e); rc = RM_ERR_CUDA; }
  }
  if (rc == RM_OK) rc = check_device_error(c, msg);
  if (rc != RM_OK) {
    c->hist_valid = false;  // CacheGuard, metal.mm:105-108
    cudaGetLastError();
    set_err(err, errcap, msg);
  }
  return rc;
}

// include/raymotion/preview.hpp:17-23: the frame line, the bytes, then one
// byte granted for the next frame (end of file: rendering is complete)
int rmcuda_preview_frame(int32_t fd, const uint8_t* rgb, int32_t width, int32_t height, int32_t frame,
                         int32_t grant_fd, char* err, size_t errcap) {
  if (fd < 0 || !rgb || width <= 0 || height <= 0) { set_err(err, errcap, "invalid preview frame"); return RM_ERR_INVALID; }
  const size_t bytes = size_t(width) * size_t(height) * 3;
  char head[96];
  const int n = std::snprintf(head, sizeof(head), "RAY1 %d %d %d %zu\n", width, height, frame, bytes);
  auto write_all = [fd](const void* data, size_t len) {
    const char* q = static_cast<const char*>(data);
    while (len > 0) {
      const ssize_t k = ::write(fd, q, len);
      if (k < 0 && errno == EINTR) continue;
      if (k <= 0) return false;
      q += k;
      len -= size_t(k);
    }
    return true;
  };
  if (n <= 0 || !write_all(head, size_t(n)) || !write_all(rgb, bytes)) {
    set_err(err, errcap, "preview channel closed");
    return RM_ERR_INVALID;
  }
  if (grant_fd >= 0) {
    char b;
    ssize_t k;
    do k = ::read(grant_fd, &b, 1);
    while (k < 0 && errno == EINTR);
    if (k <= 0) return RM_PREVIEW_DONE;
  }
  return RM_OK;
}

int rmcuda_preview_last(rmcuda_ctx* c, int32_t fd, int32_t frame, int32_t grant_fd, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  {
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (c->frames == 0 || !c->last_final || c->last_w <= 0 || c->last_h <= 0) {
      set_err(err, errcap, "no frame rendered");
      return RM_ERR_INVALID;
    }
    const size_t npix = size_t(c->last_w) * size_t(c->last_h);
    cudaError_t e = c->rgb.reserve(npix * 3);
    if (e == cudaSuccess && c->h_preview_cap < npix * 3) {
      if (c->h_preview) cudaFreeHost(c->h_preview);
      c->h_preview = nullptr;
      c->h_preview_cap = 0;
      if ((e = cudaMallocHost(reinterpret_cast<void**>(&c->h_preview), npix * 3)) == cudaSuccess)
        c->h_preview_cap = npix * 3;
    }
    // the device tonemap of the last linear image (pathtrace.metal:1355-1363)
    if (e == cudaSuccess) e = launch_tonemap(c->last_final, c->rgb.as<uint8_t>(), uint32_t(npix), c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c->h_preview, c->rgb.ptr, npix * 3, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("preview read-back failed", e)); return RM_ERR_CUDA; }
    // written under the context's lock: the pinned image is the context's
    return rmcuda_preview_frame(fd, c->h_preview, c->last_w, c->last_h, frame, grant_fd, err, errcap);
  }
}

int rmcuda_trace(rmcuda_ctx* c, const float* d_rays, int32_t n, int32_t any_hit, int32_t* d_tri, float* d_t,
                 float* d_u, float* d_v, char* err, size_t errcap) {
  if (!c || (n > 0 && (!d_rays || !d_tri)) || n < 0) { set_err(err, errcap, "invalid trace arguments"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->sc.have_scene) { set_err(err, errcap, "no resident scene"); return RM_ERR_INVALID; }
  cudaError_t e = launch_trace(scene_view(c->sc), d_rays, n, any_hit, d_tri, d_t, d_u, d_v, c->err.as<uint32_t>(), c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("trace launch failed", e)); return RM_ERR_CUDA; }
  std::string msg;
  int rc = check_device_error(c, msg);
  if (rc != RM_OK) set_err(err, errcap, msg);
  return rc;
}

int rmcuda_debug_read(rmcuda_ctx* c, int32_t which, void* host, size_t cap, char* err, size_t errcap) {
  if (!c || !host) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const size_t npix = size_t(c->last_w) * size_t(c->last_h);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("sync failed", e)); return RM_ERR_CUDA; }
  auto fetch = [&](const DevBuf& b, std::vector<float4>& v) {
    v.resize(npix);
    return cudaMemcpy(v.data(), b.ptr, npix * sizeof(float4), cudaMemcpyDeviceToHost);
  };
  if (which == 0 || which == 1 || which == 2) {
    // after a ReSTIR frame the just-written buffers were swapped into the history slots
    const size_t rec = which == 0 ? 76 : 60;
    if (cap < npix * rec) { set_err(err, errcap, "buffer too small"); return RM_ERR_INVALID; }
    unsigned char* out = static_cast<unsigned char*>(host);
    std::vector<float4> a, b, cc, d, f;
    if (which == 0) {
      const GBufSet& g = c->hg;
      if ((e = fetch(g.pos_kind, a)) != cudaSuccess || (e = fetch(g.nor_rough, b)) != cudaSuccess ||
          (e = fetch(g.alb_met, cc)) != cudaSuccess || (e = fetch(g.wo_ior, d)) != cudaSuccess ||
          (e = fetch(g.emi, f)) != cudaSuccess) {
        set_err(err, errcap, cuda_msg("read failed", e));
        return RM_ERR_CUDA;
      }
      for (size_t i = 0; i < npix; ++i) {
        float r[19] = {a[i].x, a[i].y, a[i].z, b[i].x, b[i].y, b[i].z, cc[i].x, cc[i].y, cc[i].z, d[i].x,
                       d[i].y, d[i].z, f[i].x, f[i].y, f[i].z, b[i].w, cc[i].w, d[i].w, a[i].w};
        std::memcpy(out + i * 76, r, 76);
      }
    } else {
      const ResSet& r = which == 1 ? c->rinit : c->hres;
      if ((e = fetch(r.lp, a)) != cudaSuccess || (e = fetch(r.ln, b)) != cudaSuccess ||
          (e = fetch(r.le, cc)) != cudaSuccess || (e = fetch(r.wm, d)) != cudaSuccess) {
        set_err(err, errcap, cuda_msg("read failed", e));
        return RM_ERR_CUDA;
      }
      for (size_t i = 0; i < npix; ++i) {
        float rr[15] = {a[i].x, a[i].y, a[i].z, b[i].x, b[i].y, b[i].z, cc[i].x, cc[i].y, cc[i].z,
                        a[i].w, b[i].w, cc[i].w, d[i].x, d[i].y, d[i].z};
        std::memcpy(out + i * 60, rr, 60);
      }
    }
    return RM_OK;
  }
  if (which == 3 || which == 4) {
    const size_t bytes = npix * (which == 3 ? 12 : 8);
    if (cap < bytes) { set_err(err, errcap, "buffer too small"); return RM_ERR_INVALID; }
    // 3: the shaded radiance before the denoiser (the final image is the
    // frame's hdr output); the denoiser reads it without writing it
    const void* src = which == 3 ? static_cast<const void*>(c->last_final ? c->hdr.ptr : nullptr) : c->dbg.ptr;
    if (!src) { set_err(err, errcap, "no frame rendered"); return RM_ERR_INVALID; }
    e = cudaMemcpy(host, src, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("read failed", e)); return RM_ERR_CUDA; }
    return RM_OK;
  }
  set_err(err, errcap, "unknown buffer");
  return RM_ERR_INVALID;
}

int rmcuda_reset_history(rmcuda_ctx* c) {
  if (!c) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  c->hist_valid = false;
  return RM_OK;
}

int rmcuda_stats_get(rmcuda_ctx* c, rm_stats* out) {
  if (!c || !out) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  unsigned long long all[RM_STAGE_COUNT * 4] = {};
  uint32_t e32 = 0;
  if (cudaMemcpyAsync(all, c->ctr.ptr, sizeof(all), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(&e32, c->err.ptr, 4, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return RM_ERR_CUDA;
  unsigned long long v[4] = {0, 0, 0, 0};
  for (int i = 0; i < RM_STAGE_COUNT * 4; ++i) v[i % 4] += all[i];
  out->path_samples = v[0];
  out->rays = v[1];
  out->nodes_visited = v[2];
  out->tris_tested = v[3];
  out->frames = c->frames;
  out->kernel_launches = c->launches;
  out->device_error = e32;
  out->kernel_chain = uint32_t(c->last_chain);
  out->bvh_node_bytes = c->sc.bvh.n_wide > 0 ? 80u : 64u;
  out->bvh_builds = c->bvh_builds;
  out->bvh_refits = c->bvh_refits;
  out->bvh_kept = uint32_t(c->sc.reuses);
  return RM_OK;
}

int rmcuda_profile(rmcuda_ctx* c, int level) {
  if (!c) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  c->profiling = level < 0 ? 0 : level;
  return RM_OK;
}

int rmcuda_wave_log(rmcuda_ctx* c, int32_t* out, int32_t cap) {
  if (!c || cap < 0) return -1;
  std::lock_guard<std::mutex> lk(c->mu);
  const int waves = int(c->wave_log.size() / 4);
  for (int i = 0; i < waves * 4 && i < cap * 4; ++i) out[i] = c->wave_log[size_t(i)];
  return waves;
}

int rmcuda_stage_counters(rmcuda_ctx* c, uint64_t* out, int32_t n) {
  if (!c || !out || n < 0) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  unsigned long long all[RM_STAGE_COUNT * 4] = {};
  if (cudaMemcpyAsync(all, c->ctr.ptr, sizeof(all), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return RM_ERR_CUDA;
  for (int i = 0; i < n * 4 && i < RM_STAGE_COUNT * 4; ++i) out[i] = all[i];
  return RM_OK;
}

int rmcuda_stage_times(rmcuda_ctx* c, double* ms, uint64_t* launches, int32_t n) {
  if (!c || n < 0) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  resolve_pending(c);
  for (int i = 0; i < n && i < RM_STAGE_COUNT; ++i) {
    if (ms) ms[i] = c->stage_ms[i];
    if (launches) launches[i] = c->stage_n[i];
  }
  return RM_OK;
}

int rmcuda_stats_reset(rmcuda_ctx* c) {
  if (!c) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  resolve_pending(c);
  for (int i = 0; i < RM_STAGE_COUNT; ++i) { c->stage_ms[i] = 0; c->stage_n[i] = 0; }
  c->frames = 0;
  c->launches = 0;
  return cudaMemsetAsync(c->ctr.ptr, 0, RM_STAGE_COUNT * 32, c->stream) == cudaSuccess ? RM_OK : RM_ERR_CUDA;
}

}  // extern "C"

// rmcuda_adjoint.cu - the C ABI of differentiable rendering (include/rmcuda.h):
// per-triangle materials on scene objects and the path-replay adjoint of the
// plain frame (rm_adjoint.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "rm_ctx.h"
#include "rm_launch.h"
#include "rmcuda.h"

using namespace rmd;
using namespace rmapi;

static_assert(sizeof(rm_material) == RM_MATERIAL_PARAMS * sizeof(float), "rm_material is 8 floats");

extern "C" {

int rmcuda_scene_set_materials(rmcuda_ctx* c, rmcuda_scene* scene, const int32_t* tri_material,
                               const rm_material* mats, int32_t n_materials, const float* light_cdf,
                               float light_total, char* err, size_t errcap) {
  if (!c || !scene || !mats || n_materials <= 0) { set_err(err, errcap, "invalid materials"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  if (scene->device != c->device) { set_err(err, errcap, "scene of another device"); return RM_ERR_INVALID; }
  cudaSetDevice(c->device);
  DevScene& sc = scene->d;
  if (!sc.have_scene) { set_err(err, errcap, "no scene"); return RM_ERR_INVALID; }
  // a frame rendered with the old materials is no longer the ReSTIR adjoint's checkpoint
  if (c->hist_scene == static_cast<const void*>(&sc)) c->hist_scene = nullptr;
  if (!tri_material && (sc.n_materials == 0 || sc.n_materials != n_materials)) {
    set_err(err, errcap, "the first call needs tri_material, and later calls the same material count");
    return RM_ERR_INVALID;
  }
  if (tri_material)
    for (int i = 0; i < sc.n_tris; ++i)
      if (tri_material[i] < -1 || tri_material[i] >= n_materials) {
        set_err(err, errcap, "material index out of range");
        return RM_ERR_INVALID;
      }
  if (light_cdf && !(light_total > 0.0f) && sc.n_lights > 0) {
    set_err(err, errcap, "light_total must be positive");
    return RM_ERR_INVALID;
  }
  cudaStream_t st = c->stream;
  cudaError_t e = cudaSuccess;
  const size_t mbytes = size_t(n_materials) * sizeof(rm_material);
  if (tri_material) e = sc.tri_mat.reserve(std::max<size_t>(4, size_t(sc.n_tris) * 4));
  if (e == cudaSuccess) e = sc.mats.reserve(mbytes);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("material buffer allocation failed", e)); return RM_ERR_ALLOC; }
  if (tri_material && sc.n_tris > 0)
    e = cudaMemcpyAsync(sc.tri_mat.ptr, tri_material, size_t(sc.n_tris) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sc.mats.ptr, mats, mbytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && light_cdf && sc.n_lights > 0)
    e = cudaMemcpyAsync(sc.cdf.ptr, light_cdf, size_t(sc.n_lights) * 4, cudaMemcpyHostToDevice, st);
  sc.validated_texels = -1;  // the triangles' material fields are rewritten
  if (e == cudaSuccess)
    e = apply_materials(sc.tris.as<rm_triangle>(), sc.tri_mat.as<int32_t>(), sc.mats.as<float>(), sc.n_tris, st);
  if (e == cudaSuccess && light_cdf) sc.light_total = light_total;
  if (e == cudaSuccess)
    e = prepare_lights(sc.tris.as<rm_triangle>(), sc.lights.as<int32_t>(), sc.cdf.as<float>(), sc.n_lights,
                       sc.light_total, sc.lrec, sc.guide, sc.guide_n, sc.guide_inv, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("material update failed", e)); return RM_ERR_CUDA; }
  sc.n_materials = n_materials;
  return RM_OK;
}

int rmcuda_backward(rmcuda_ctx* c, const rmcuda_scene* scene, const rm_camera* cam, const rm_config* cfg,
                    uint64_t seed, const float* d_dL_dimage, float* d_grad, char* err, size_t errcap) {
  if (!c || !scene || !cam || !cfg || !d_dL_dimage || !d_grad) {
    set_err(err, errcap, "null argument");
    return RM_ERR_INVALID;
  }
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->spp <= 0 || cfg->max_bounces < 0 ||
      size_t(cfg->width) * size_t(cfg->height) > 100000000) {
    set_err(err, errcap, kInvalidDims);
    return RM_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  if (scene->device != c->device) { set_err(err, errcap, "scene of another device"); return RM_ERR_INVALID; }
  cudaSetDevice(c->device);
  const DevScene& sc = scene->d;
  if (sc.n_materials <= 0) { set_err(err, errcap, "scene has no materials (rmcuda_scene_set_materials)"); return RM_ERR_INVALID; }
  Plan pl = make_plan(sc, *cam, *cfg);
  if (pl.use_spatial) {
    // the ReSTIR chain: K5 replayed from the checkpoint the frame left in the
    // history slots (its G-buffer and merged reservoirs)
    if (pl.p.bounces - 1 > 24) {
      set_err(err, errcap, "the adjoint of the ReSTIR chain takes at most 25 bounces");
      return RM_ERR_INVALID;
    }
    if (!c->hist_valid || !c->have_hist_bufs || c->hist_scene != static_cast<const void*>(&sc) ||
        c->hist_seed != seed || c->hist_denoised != pl.denoise ||
        std::memcmp(&c->hist_cam, cam, sizeof(rm_camera)) != 0 ||
        std::memcmp(&c->hist_cfg, cfg, sizeof(rm_config)) != 0) {
      set_err(err, errcap,
              "the adjoint of the ReSTIR chain replays the last frame rendered on this context: render it first "
              "with the same scene, camera, config and seed");
      return RM_ERR_INVALID;
    }
    const float* dl_hdr = d_dL_dimage;
    const float* dl_alb = nullptr;  // dL/d(G-buffer albedo), through the denoiser's weights
    cudaError_t e = cudaSuccess;
    if (pl.denoise) {
      // through the denoiser first: its inputs are the frame's shaded HDR, its
      // G-buffer and the history it blended (the previous final colour and
      // G-buffer, in the slots the frame's swap left them in)
      const size_t npix = size_t(cfg->width) * size_t(cfg->height);
      if ((e = c->adj_scratch.reserve(npix * 20 * sizeof(float))) != cudaSuccess) {
        set_err(err, errcap, cuda_msg("adjoint buffer allocation failed", e));
        return RM_ERR_ALLOC;
      }
      Params dp = pl.p;
      dp.hasHistory = c->hist_had_history ? 1 : 0;
      dp.prevCamera = c->hist_prev_cam;
      float* scratch = c->adj_scratch.as<float>();
      float* g_hdr = scratch + npix * 14;
      float* g_alb = scratch + npix * 17;
      e = staged(c, RM_STAGE_ADJOINT, [&] {
        return launch_denoise_backward(dp, c->hg.view(), c->gb.view(), c->hdr.as<float>(), c->tmp_a.as<float>(),
                                       d_dL_dimage, scratch, g_hdr, g_alb, c->stream);
      });
      if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("denoiser adjoint launch failed", e)); return RM_ERR_CUDA; }
      dl_hdr = g_hdr;
      dl_alb = g_alb;
    }
    pl.p.hasHistory = 0;
    e = staged(c, RM_STAGE_ADJOINT, [&] {
      return launch_adjoint_restir(scene_view(sc), pl.p, seed, c->hg.view(), c->hres.view(), sc.tri_mat.as<int32_t>(),
                                   sc.n_materials, dl_hdr, dl_alb, d_grad,
                                   c->ctr.as<unsigned long long>() + 4 * RM_STAGE_ADJOINT, c->err.as<uint32_t>(),
                                   c->stream);
    });
    if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("adjoint launch failed", e)); return RM_ERR_CUDA; }
    return RM_OK;
  }
  if (pl.p.adapt_min > 0) {
    set_err(err, errcap, "the adjoint needs a fixed sample count (adapt_min 0 or RM_FLAG_NOADAPT)");
    return RM_ERR_INVALID;
  }
  cudaError_t e = staged(c, RM_STAGE_ADJOINT, [&] {
    return launch_adjoint(pl.lanes, scene_view(sc), pl.p, seed, sc.tri_mat.as<int32_t>(), sc.n_materials,
                          d_dL_dimage, d_grad, c->ctr.as<unsigned long long>() + 4 * RM_STAGE_ADJOINT,
                          c->err.as<uint32_t>(), c->stream);
  });
  if (e != cudaSuccess) { set_err(err, errcap, cuda_msg("adjoint launch failed", e)); return RM_ERR_CUDA; }
  return RM_OK;
}

}  // extern "C"

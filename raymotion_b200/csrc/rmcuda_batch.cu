// rmcuda_batch.cu - the C ABI of scene objects and batched rendering
// (include/rmcuda.h): many images, each the reference's plain single-frame
// chain (pathtrace.metal:739-815 with the policy of metal.mm:146-170,
// :390-394), rendered together by the persistent wavefront of rm_batch.cu.
//
// Host side of a batch: build the job table (one entry per image, largest
// first so the pool drains on small images), reset the pool, then launch
// waves, captured once into a CUDA graph of `graph_waves` waves and replayed
// until the queue lengths read back after a replay show no work left.  The
// read-back of replay i is checked after replay i+1 is already queued, so
// the GPU never waits for the host; the waves of a replay that runs after the
// work is done find empty queues and return at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "rm_ctx.h"
#include "rm_launch.h"
#include "rmcuda.h"

using namespace rmd;
using namespace rmapi;

void rmapi::BatchPool::release() {
  for (DevBuf& b : slot) b.release();
  for (DevBuf& b : chunk) b.release();
  for (DevBuf& b : queue) b.release();
  jobs.release();
  tile_begin.release();
  next_tile.release();
  if (exec) cudaGraphExecDestroy(exec);
  exec = nullptr;
  if (h_counts) cudaFreeHost(h_counts);
  h_counts = nullptr;
  chunks = 0;
}

namespace {

constexpr int kSlotBytes[17] = {16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 16, 4, 16, 4, 4, 4};

cudaError_t ensure_pool(BatchPool& bp, int chunks) {
  if (bp.chunks >= chunks && bp.h_counts) return cudaSuccess;
  const size_t slots = size_t(chunks) * kBtChunk;
  cudaError_t e;
  for (int i = 0; i < 17; ++i)
    if ((e = bp.slot[i].reserve(slots * size_t(kSlotBytes[i]))) != cudaSuccess) return e;
  for (DevBuf& b : bp.chunk)
    if ((e = b.reserve(size_t(chunks) * sizeof(int))) != cudaSuccess) return e;
  for (int k = 0; k < 2; ++k)
    for (int i = 0; i < kBtQueues; ++i)  // the refill queue holds chunks, the others lane slots or pixels
      if ((e = bp.queue[kBtQueues * k + i].reserve((i == kBtRf ? size_t(chunks) : slots) * sizeof(int))) !=
          cudaSuccess)
        return e;
  if ((e = bp.queue[2 * kBtQueues].reserve(2 * kBtCounts * sizeof(int))) != cudaSuccess) return e;
  if ((e = bp.next_tile.reserve(sizeof(int))) != cudaSuccess) return e;
  if (!bp.h_counts &&
      (e = cudaMallocHost(reinterpret_cast<void**>(&bp.h_counts), 2 * kBtCounts * sizeof(int))) != cudaSuccess)
    return e;
  bp.chunks = chunks;
  return cudaSuccess;
}

BtState state_view(const BatchPool& bp) {
  BtState w;
  w.u = bp.slot[0].as<uint4>();
  float4** f4[] = {&w.acc, &w.thr, &w.pb, &w.o, &w.d, &w.c, &w.so, &w.sd, &w.hit, &w.hoff, &w.val};
  for (int i = 0; i < 11; ++i) *f4[i] = bp.slot[1 + i].as<float4>();
  w.occ = bp.slot[12].as<uint32_t>();
  w.gsum = bp.slot[13].as<float4>();
  w.gsl2 = bp.slot[14].as<float>();
  w.gbase = bp.slot[15].as<int>();
  w.garr = bp.slot[16].as<int>();
  w.cjob = bp.chunk[0].as<int>();
  w.ctile = bp.chunk[1].as<int>();
  w.cleft = bp.chunk[2].as<int>();
  return w;
}

BtQueues queue_view(const BatchPool& bp, int k) {
  BtQueues q;
  int** qs[kBtQueues] = {&q.ext, &q.shd, &q.qa, &q.qb, &q.qc, &q.qd, &q.st, &q.rf, &q.cm1, &q.cm8, &q.cm32};
  for (int i = 0; i < kBtQueues; ++i) *qs[i] = bp.queue[kBtQueues * k + i].as<int>();
  q.counts = bp.queue[2 * kBtQueues].as<int>() + kBtCounts * k;
  return q;
}

bool valid_tuning(const rm_batch_tuning& t) {
  return t.pool_chunks >= 1 && t.pool_chunks <= (1 << 22) && (t.tile_shape == 0 || t.tile_shape == 1) &&
         t.grid_scale >= 1 && t.grid_scale <= 4 &&
         (t.graph_waves == 0 || (t.graph_waves >= 2 && t.graph_waves <= 64 && t.graph_waves % 2 == 0)) &&
         (t.bvh_width == 2 || t.bvh_width == 8);
}

// Tile of a chunk: tile_w x tile_h pixels of `lanes` lane slots each.
void tile_shape(int lanes, int shape, int& tw, int& th) {
  const int px = kBtChunk / lanes;
  tw = px;
  th = 1;
  if (shape == 1) {
    if (px == 32) { tw = 8; th = 4; }
    else if (px == 4) { tw = 2; th = 2; }
  }
}

struct Prepared {
  std::vector<BtJob> jobs;  // largest first
  std::vector<int> tile_begin;
  int total_tiles = 0;
  uint64_t max_waves = 0;
};

int prepare(rmcuda_ctx* c, const rm_batch_item* items, int n, int shape, int width, Prepared& out,
            std::string& msg) {
  if (n < 0 || (n > 0 && !items)) { msg = "invalid batch"; return RM_ERR_INVALID; }
  std::vector<std::pair<double, int>> order;
  std::vector<BtJob> jobs(static_cast<size_t>(n));
  int max_rounds = 1, max_bounces = 0;
  for (int i = 0; i < n; ++i) {
    const rm_batch_item& it = items[i];
    const rm_config& cfg = it.config;
    if (cfg.width <= 0 || cfg.height <= 0 || cfg.spp <= 0 || cfg.max_bounces < 0 ||
        size_t(cfg.width) * size_t(cfg.height) > 100000000) {
      msg = kInvalidDims;
      return RM_ERR_INVALID;
    }
    if (!it.scene || it.scene->device != c->device || !it.scene->d.have_scene) {
      msg = "batch item " + std::to_string(i) + ": no scene of this context's device";
      return RM_ERR_INVALID;
    }
    Plan pl = make_plan(it.scene->d, it.camera, cfg);
    if (pl.use_spatial) {
      msg = "batch item " + std::to_string(i) +
            ": the single-frame policy picks the ReSTIR chain; batches render the plain chain "
            "(set RM_FLAG_RESTIR_OFF or restir_spatial 0)";
      return RM_ERR_INVALID;
    }
    BtJob& J = jobs[size_t(i)];
    std::memset(&J, 0, sizeof(J));
    // the collapse is a cache of the scene object, built once under the context lock
    rmd::DevBvh& bvh = const_cast<rmcuda_scene*>(it.scene)->d.bvh;
    if (width == 8 && bvh.n_wide == 0 && bvh.n_records > 0) {
      // collapse this scene's binary BVH on first use (none if too deep: the
      // job then traverses the binary BVH, which gives the same hits)
      const cudaError_t e = rmd::build_wide(bvh, c->stream);
      if (e != cudaSuccess) { msg = cuda_msg("wide BVH build failed", e); return RM_ERR_CUDA; }
    }
    J.s = scene_view(it.scene->d);
    if (width != 8) {
      J.s.wnodes = nullptr;
      J.s.wtgeo = nullptr;
    }
    J.p = pl.p;
    J.seed = it.seed;
    J.hdr = it.d_hdr;
    J.rgb = it.d_rgb;
    J.dbg = it.d_aux;
    J.lanes = pl.lanes;
    tile_shape(pl.lanes, shape, J.tile_w, J.tile_h);
    J.tiles_x = (cfg.width + J.tile_w - 1) / J.tile_w;
    J.tiles = J.tiles_x * ((cfg.height + J.tile_h - 1) / J.tile_h);
    const int rounds = (cfg.spp + pl.lanes - 1) / pl.lanes;
    max_rounds = std::max(max_rounds, rounds);
    max_bounces = std::max(max_bounces, cfg.max_bounces);
    const double cost = double(cfg.width) * double(cfg.height) * double(cfg.spp) * double(cfg.max_bounces + 1);
    order.push_back({-cost, i});
  }
  std::stable_sort(order.begin(), order.end());
  out.jobs.clear();
  out.tile_begin.clear();
  int64_t t = 0;
  for (auto& o : order) {
    BtJob J = jobs[size_t(o.second)];
    J.tile_begin = int(t);
    out.jobs.push_back(J);
    out.tile_begin.push_back(int(t));
    t += J.tiles;
    if (t > (int64_t(1) << 30)) { msg = "batch too large"; return RM_ERR_INVALID; }
  }
  out.total_tiles = int(t);
  // A chunk finishes its tile within rounds x (bounces + 2) waves and is
  // refilled in the next; the bound only guards against a stalled pool.
  const uint64_t per_tile = uint64_t(max_rounds) * uint64_t(max_bounces + 2) + 2;
  out.max_waves = 2 * (uint64_t(t) / uint64_t(std::max(1, c->batch.tuning.pool_chunks)) + 2) * per_tile + 1000;
  return RM_OK;
}

struct Grids {
  int aux, trace, shade;
  bool wide;  // traverse the 8-wide BVHs
};

Grids grids(rmcuda_ctx* c, int scale) {
  int* occ = c->batch.occ;
  if (!occ[0]) batch_occupancy(occ[0], occ[1], occ[2]);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  return Grids{sms * occ[0] * scale, sms * occ[1] * scale, sms * occ[2] * scale, false};
}

// Kernels of a wave: refill, start, 2 traversals, 4 shades, 3 round sums.
constexpr int kWaveKernels = 11;

// Enqueue one wave on the context stream (cur: this wave's queues).
cudaError_t enqueue_wave(rmcuda_ctx* c, const BtBatch& b, const BtState& w, const BtQueues* q, int cur,
                         const Grids& g) {
  const BtQueues& Q = q[cur];
  const BtQueues& N = q[cur ^ 1];
  unsigned long long* ctr = c->ctr.as<unsigned long long>();
  uint32_t* err = c->err.as<uint32_t>();
  cudaStream_t st = c->stream;
  cudaError_t e = cudaMemsetAsync(N.counts, 0, kBtCounts * sizeof(int), st);
  if (e == cudaSuccess)
    e = staged2(c, RM_STAGE_BT_START, [&] { return launch_batch_refill(b, w, Q, g.aux, st); });
  if (e == cudaSuccess)
    e = staged2(c, RM_STAGE_BT_START,
                [&] { return launch_batch_start(b, w, Q, N, g.aux, ctr + 4 * RM_STAGE_BT_START, err, st); });
  if (e == cudaSuccess)
    e = staged2(c, RM_STAGE_BT_EXTEND,
                [&] { return launch_batch_trace(b, w, Q, false, g.wide, g.trace, ctr + 4 * RM_STAGE_BT_EXTEND, err, st); });
  if (e == cudaSuccess)
    e = staged2(c, RM_STAGE_BT_SHADOW,
                [&] { return launch_batch_trace(b, w, Q, true, g.wide, g.trace, ctr + 4 * RM_STAGE_BT_SHADOW, err, st); });
  for (int vk = 0; vk < 4 && e == cudaSuccess; ++vk)
    e = staged2(c, RM_STAGE_BT_SHADE,
                [&] { return launch_batch_shade(vk, b, w, Q, N, g.shade, ctr + 4 * RM_STAGE_BT_SHADE, err, st); });
  for (int lanes : {1, 8, 32})
    if (e == cudaSuccess)
      e = staged2(c, RM_STAGE_BT_START, [&] { return launch_batch_combine(lanes, b, w, Q, N, g.aux, st); });
  return e;
}

// A timing window over waves [start, stop) of a batch (tuning): events and
// the device counters at both ends.  A batch that drains before `start` is
// timed from its first wave.
struct Window {
  uint64_t start = 0, stop = 0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  unsigned long long before[RM_STAGE_COUNT * 4] = {}, after[RM_STAGE_COUNT * 4] = {};
};

// Run a prepared batch; with a window it ends after the window's last wave.
int run_batch(rmcuda_ctx* c, const Prepared& P, const rm_batch_tuning& tune, Window* win, std::string& msg) {
  BatchPool& bp = c->batch;
  cudaStream_t st = c->stream;
  cudaError_t e = ensure_pool(bp, tune.pool_chunks);
  if (e == cudaSuccess) e = bp.jobs.reserve(std::max<size_t>(1, P.jobs.size()) * sizeof(BtJob));
  if (e == cudaSuccess) e = bp.tile_begin.reserve(std::max<size_t>(1, P.tile_begin.size()) * sizeof(int));
  if (e != cudaSuccess) { msg = cuda_msg("batch buffer allocation failed", e); return RM_ERR_ALLOC; }
  if (P.jobs.empty()) return RM_OK;
  if ((e = cudaMemcpyAsync(bp.jobs.ptr, P.jobs.data(), P.jobs.size() * sizeof(BtJob), cudaMemcpyHostToDevice,
                           st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(bp.tile_begin.ptr, P.tile_begin.data(), P.tile_begin.size() * sizeof(int),
                           cudaMemcpyHostToDevice, st)) != cudaSuccess) {
    msg = cuda_msg("batch upload failed", e);
    return RM_ERR_CUDA;
  }
  const int chunks = tune.pool_chunks;
  BtBatch b{bp.jobs.as<BtJob>(), bp.tile_begin.as<int>(), int(P.jobs.size()), P.total_tiles, bp.next_tile.as<int>()};
  BtState w = state_view(bp);
  BtQueues q[2] = {queue_view(bp, 0), queue_view(bp, 1)};
  // chunks beyond the tuning's pool size are never handed out: queue_view
  // sizes are the allocation's, the init kernel only queues `chunks`
  if ((e = launch_batch_init(w, q[0], chunks, b.next_tile, st)) != cudaSuccess) {
    msg = cuda_msg("batch init failed", e);
    return RM_ERR_CUDA;
  }
  c->launches += 1;
  Grids g = grids(c, tune.grid_scale);
  g.wide = tune.bvh_width == 8;
  // (the legacy default stream cannot be captured)
  const bool use_graph = tune.graph_waves > 0 && c->profiling < 2 && c->stream != nullptr;
  const int per_launch = use_graph ? tune.graph_waves : 8;
  if (bp.exec) { cudaGraphExecDestroy(bp.exec); bp.exec = nullptr; }
  if (use_graph) {
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    const uint64_t launches0 = c->launches;
    for (int k = 0; k < per_launch && e == cudaSuccess; ++k) e = enqueue_wave(c, b, w, q, k & 1, g);
    cudaError_t e2 = cudaStreamEndCapture(st, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&bp.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    c->launches = launches0;  // counted per replay below
    if (e != cudaSuccess) { msg = cuda_msg("batch graph capture failed", e); return RM_ERR_CUDA; }
  }
  const uint64_t graph_kernels = uint64_t(per_launch) * kWaveKernels;
  bp.wave_log.clear();
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if ((e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming)) != cudaSuccess) {
    msg = cuda_msg("event creation failed", e);
    if (ev[0]) cudaEventDestroy(ev[0]);
    return RM_ERR_CUDA;
  }
  int rc = RM_OK;
  uint64_t waves = 0;
  const size_t ctr_bytes = sizeof(unsigned long long) * RM_STAGE_COUNT * 4;
  auto mark = [&](cudaEvent_t ev, unsigned long long* dst) {
    cudaEventRecord(ev, st);
    cudaMemcpyAsync(dst, c->ctr.ptr, ctr_bytes, cudaMemcpyDeviceToHost, st);
  };
  if (win) mark(win->t0, win->before);
  for (uint64_t i = 0;; ++i) {
    if (win && waves == win->start && waves > 0) mark(win->t0, win->before);
    if (use_graph) {
      e = cudaGraphLaunch(bp.exec, st);
      c->launches += graph_kernels;
    } else {
      for (int k = 0; k < per_launch && e == cudaSuccess; ++k) e = enqueue_wave(c, b, w, q, k & 1, g);
    }
    waves += uint64_t(per_launch);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(bp.h_counts + kBtCounts * (i & 1), q[0].counts, kBtCounts * sizeof(int),
                          cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[i & 1], st);
    if (e != cudaSuccess) { msg = cuda_msg("batch wave launch failed", e); rc = RM_ERR_CUDA; break; }
    if (i == 0) continue;
    if ((e = cudaEventSynchronize(ev[(i - 1) & 1])) != cudaSuccess) {
      msg = cuda_msg("batch wave failed", e);
      rc = RM_ERR_CUDA;
      break;
    }
    const int* h = bp.h_counts + kBtCounts * ((i - 1) & 1);
    const int live = h[kBtExt] + h[kBtC] + h[kBtSt] + h[kBtRf];
    bp.wave_log.push_back(live);
    bp.wave_log.push_back(h[kBtExt]);
    if (live == 0) break;
    if (win && waves >= win->stop) break;
    if (waves > P.max_waves) { msg = "batch did not drain"; rc = RM_ERR_DEVICE; break; }
  }
  bp.waves += waves;
  if (win) mark(win->t1, win->after);
  cudaStreamSynchronize(st);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return rc;
}

}  // namespace

extern "C" {

int rmcuda_scene_create(rmcuda_ctx* c, const rm_scene_view* sv, rmcuda_scene** out, char* err, size_t errcap) {
  if (!c || !out) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  *out = nullptr;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  auto* s = new rmcuda_scene();
  s->device = c->device;
  std::string msg;
  int rc = upload_scene(c, s->d, sv, msg);
  if (rc == RM_OK) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { msg = cuda_msg("scene upload failed", e); rc = RM_ERR_CUDA; }
  }
  if (rc != RM_OK) {
    cudaStreamSynchronize(c->stream);
    s->d.release();
    delete s;
    set_err(err, errcap, msg);
    return rc;
  }
  *out = s;
  return RM_OK;
}

void rmcuda_scene_destroy(rmcuda_ctx* c, rmcuda_scene* s) {
  if (!s) return;
  if (c) {
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    // a checkpoint of this scene's last frame must not match a later scene
    // allocated at the same address
    if (c->hist_scene == static_cast<const void*>(&s->d)) c->hist_scene = nullptr;
  }
  s->d.release();
  delete s;
}

int rmcuda_render_scene_async(rmcuda_ctx* c, const rmcuda_scene* scene, const rm_camera* cam, const rm_config* cfg,
                              uint64_t seed, uint8_t* d_rgb, float* d_hdr, char* err, size_t errcap) {
  if (!c || !scene || !cam || !cfg) { set_err(err, errcap, "null argument"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  if (scene->device != c->device) { set_err(err, errcap, "scene of another device"); return RM_ERR_INVALID; }
  cudaSetDevice(c->device);
  std::string msg;
  int rc = enqueue_frame(c, const_cast<DevScene&>(scene->d), *cam, *cfg, seed, d_rgb, msg);
  if (rc == RM_OK && d_hdr) {
    const size_t bytes = size_t(cfg->width) * size_t(cfg->height) * 12;
    cudaError_t e = cudaMemcpyAsync(d_hdr, c->last_final, bytes, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) { msg = cuda_msg("hdr copy failed", e); rc = RM_ERR_CUDA; }
  }
  if (rc != RM_OK) { c->hist_valid = false; set_err(err, errcap, msg); }
  return rc;
}

int rmcuda_render_batch(rmcuda_ctx* c, const rm_batch_item* items, int32_t n, char* err, size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::string msg;
  Prepared P;
  int rc = prepare(c, items, n, c->batch.tuning.tile_shape, c->batch.tuning.bvh_width, P, msg);
  cudaEvent_t a = nullptr, b = nullptr;
  if (rc == RM_OK && c->profiling > 0 && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
    cudaEventRecord(a, c->stream);
  if (rc == RM_OK) rc = run_batch(c, P, c->batch.tuning, nullptr, msg);
  if (a && b) {
    cudaEventRecord(b, c->stream);
    c->pending.push_back({RM_STAGE_BATCH, a, b});
  }
  if (rc == RM_OK) rc = check_device_error(c, msg);
  if (rc == RM_OK) c->frames += uint64_t(n);
  if (rc != RM_OK) { cudaGetLastError(); set_err(err, errcap, msg); }
  return rc;
}

int rmcuda_batch_tune(rmcuda_ctx* c, const rm_batch_item* items, int32_t n, rm_batch_tuning* out, char* err,
                      size_t errcap) {
  if (!c) { set_err(err, errcap, "null context"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  std::string msg;
  const rm_batch_tuning keep = c->batch.tuning;
  rm_batch_tuning best = keep;
  double best_rate = -1.0;
  const int pools[3] = {32768, 65536, 131072};
  Window win;
  win.start = 16;  // the first waves fill the pool
  win.stop = 64;
  if (cudaEventCreate(&win.t0) != cudaSuccess || cudaEventCreate(&win.t1) != cudaSuccess) {
    set_err(err, errcap, "event creation failed");
    return RM_ERR_CUDA;
  }
  int rc = RM_OK;
  const int saved_profiling = c->profiling;
  c->profiling = 0;
  for (int pool : pools) {
    for (int width : {2, 8}) {
    for (int shape = 0; shape < 2 && rc == RM_OK; ++shape) {
      for (int scale = 1; scale <= 2 && rc == RM_OK; ++scale) {
        const rm_batch_tuning t{pool, shape, scale, keep.graph_waves > 0 ? keep.graph_waves : 8, width};
        c->batch.tuning = t;
        Prepared P;
        if ((rc = prepare(c, items, n, shape, width, P, msg)) != RM_OK) break;
        if ((rc = run_batch(c, P, t, &win, msg)) != RM_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, win.t0, win.t1);
        const double samples = double(win.after[4 * RM_STAGE_BT_SHADE] + win.after[4 * RM_STAGE_BT_START]) -
                               double(win.before[4 * RM_STAGE_BT_SHADE] + win.before[4 * RM_STAGE_BT_START]);
        const double rate = ms > 0.f ? samples / double(ms) : 0.0;
        if (rate > best_rate) { best_rate = rate; best = t; }
      }
    }
    }
    if (rc != RM_OK) break;
  }
  c->profiling = saved_profiling;
  cudaEventDestroy(win.t0);
  cudaEventDestroy(win.t1);
  if (rc == RM_OK) rc = check_device_error(c, msg);
  c->batch.tuning = rc == RM_OK ? best : keep;
  if (rc != RM_OK) { set_err(err, errcap, msg); return rc; }
  if (out) *out = best;
  return RM_OK;
}

int rmcuda_batch_log(rmcuda_ctx* c, int32_t* out, int32_t cap) {
  if (!c || cap < 0 || (cap > 0 && !out)) return -1;
  std::lock_guard<std::mutex> lk(c->mu);
  const int recs = int(c->batch.wave_log.size() / 2);
  for (int i = 0; i < recs * 2 && i < cap * 2; ++i) out[i] = c->batch.wave_log[size_t(i)];
  return recs;
}

int rmcuda_batch_get_tuning(rmcuda_ctx* c, rm_batch_tuning* out) {
  if (!c || !out) return RM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(c->mu);
  *out = c->batch.tuning;
  return RM_OK;
}

int rmcuda_batch_set_tuning(rmcuda_ctx* c, const rm_batch_tuning* t, char* err, size_t errcap) {
  if (!c || !t || !valid_tuning(*t)) { set_err(err, errcap, "invalid batch tuning"); return RM_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(c->mu);
  c->batch.tuning = *t;
  return RM_OK;
}

}  // extern "C"

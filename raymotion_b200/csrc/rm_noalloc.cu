// rm_noalloc.cu - rmcuda_trace_noalloc: ray queries that allocate no memory.
//
// Some callers cannot allocate device memory at all once they are running:
// an engine whose memory manager owns every byte of the GPU and forbids
// allocations outside it, a real-time loop with a fixed memory budget, or a
// stack certified to run without runtime allocation.  For them this entry
// point builds the BVH of the caller's device triangles and traces the
// caller's device rays using only caller buffers plus one file-scope device
// array, g_noalloc_scratch, whose size is fixed at compile time.
//
// Costs and rules of that design:
//  * every GPU that loads the library holds the array (kNoallocScratchBytes)
//    until the process exits;
//  * all calls share the array and it keeps the last call's contents; calls
//    that overlap on the GPU (two streams, two threads) race on it, so callers
//    must serialise them;
//  * in host code the array's name is only a host-side stand-in for the
//    symbol, so its device address is looked up once per device with
//    cudaGetSymbolAddress (with that device current) on the first call on
//    that device; that first call should come before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "rm_launch.h"
#include "rmcuda.h"

namespace {

// Scratch for RMCUDA_NOALLOC_MAX_TRIS triangles: BVH records, leaf-ordered
// triangle records, the build's sort keys / tree / boxes, the radix sort's
// temporary storage and the error word.
constexpr size_t kNoallocScratchBytes = size_t(24) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

void set_err(char* err, size_t cap, const std::string& m) {
  if (err && cap) std::snprintf(err, cap, "%s", m.c_str());
}

// Carve the scratch array for n triangles; false if it does not fit.
bool carve(unsigned char* base, int n, rmd::LbvhScratch& w) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> void* {
    off = (off + 255) & ~size_t(255);
    void* p = base + off;
    off += bytes;
    return p;
  };
  const size_t N = size_t(n > 0 ? n : 1), I = N > 1 ? N - 1 : 1;
  w.records = static_cast<float4*>(take(I * 4 * sizeof(float4)));
  w.parents = static_cast<int*>(take(N * sizeof(int)));
  w.order = static_cast<int*>(take(N * sizeof(int)));
  w.tgeo = static_cast<float4*>(take(N * 3 * sizeof(float4)));
  w.keys = static_cast<unsigned int*>(take(N * 4));
  w.vals = static_cast<int*>(take(N * 4));
  w.keys_alt = static_cast<unsigned int*>(take(N * 4));
  w.vals_alt = static_cast<int*>(take(N * 4));
  w.children = static_cast<int2*>(take(I * sizeof(int2)));
  w.ranges = static_cast<int2*>(take(I * sizeof(int2)));
  w.parent_int = static_cast<int*>(take(I * sizeof(int)));
  w.parent_leaf = static_cast<int*>(take(N * sizeof(int)));
  w.kbox = take(I * rmd::lbvh_box_bytes());
  w.kcount = static_cast<int*>(take(I * sizeof(int)));
  w.bounds = static_cast<unsigned int*>(take(6 * sizeof(unsigned int)));
  w.err_word = static_cast<uint32_t*>(take(sizeof(uint32_t)));
  off = (off + 255) & ~size_t(255);
  if (off > kNoallocScratchBytes) return false;
  w.sort_temp = base + off;
  w.sort_temp_bytes = kNoallocScratchBytes - off;
  return true;
}

}  // namespace

extern "C" int rmcuda_trace_noalloc(const rm_triangle* d_tris, int32_t n_tris, const float* d_rays, int32_t n_rays,
                                    int32_t any_hit, int32_t* d_tri, float* d_t, float* d_u, float* d_v,
                                    void* cuda_stream, char* err, size_t errcap) {
  if (n_tris < 0 || n_rays < 0 || (n_tris > 0 && !d_tris) || (n_rays > 0 && (!d_rays || !d_tri))) {
    set_err(err, errcap, "invalid arguments");
    return RM_ERR_INVALID;
  }
  if (n_tris > RMCUDA_NOALLOC_MAX_TRIS) {
    set_err(err, errcap, "rmcuda_trace_noalloc: " + std::to_string(n_tris) + " triangles exceed the maximum of " +
                             std::to_string(RMCUDA_NOALLOC_MAX_TRIS) + " (fixed scratch array)");
    return RM_ERR_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    set_err(err, errcap, "no current CUDA device");
    return RM_ERR_UNAVAILABLE;
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      // first call on this device: resolve the array's device address (the device is current)
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_err(err, errcap, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return RM_ERR_CUDA;
      }
      g_addr[dev] = p;
    }
    base = g_addr[dev];
  }
  rmd::LbvhScratch w;
  if (!carve(static_cast<unsigned char*>(base), n_tris, w)) {
    set_err(err, errcap, "rmcuda_trace_noalloc: scratch layout exceeds the fixed array");
    return RM_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  std::string msg;
  rmd::DevBvhView bvh;
  cudaError_t e = rmd::build_lbvh_into(d_tris, n_tris, 4, w, bvh, st, msg);
  if (e != cudaSuccess) {
    set_err(err, errcap, msg.empty() ? std::string("BVH build failed: ") + cudaGetErrorString(e) : msg);
    return RM_ERR_CUDA;
  }
  rmd::Scene s{};
  s.tris = d_tris;
  s.tgeo = bvh.tgeo;
  s.nodes = bvh.records;
  s.n_nodes = n_tris > 0 ? bvh.n_records : 0;
  s.n_tris = n_tris;
  e = rmd::launch_trace(s, d_rays, n_rays, any_hit, d_tri, d_t, d_u, d_v, w.err_word, st);
  uint32_t word = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&word, w.err_word, sizeof(word), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_err(err, errcap, std::string("trace failed: ") + cudaGetErrorString(e));
    return RM_ERR_CUDA;
  }
  if (word) {
    set_err(err, errcap, "traversal stack exceeded (BVH deeper than 64 levels)");
    return RM_ERR_DEVICE;
  }
  return RM_OK;
}

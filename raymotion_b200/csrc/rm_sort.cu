// rm_sort.cu - the device BVH builders' and the world preparation's radix
// sort and prefix sums, written for this library (no library kernels on the
// build path).
//
// exclusive_scan: reduce-then-scan in three launches per level (tile sums,
// a scan of the tile sums, each tile's scan from its prefix), recursing on
// the tile sums when they exceed one tile.  Within a tile the 256 threads
// take 16 rounds of 256 consecutive items (coalesced), each round a warp
// scan by shuffles and a scan of the eight warp totals.
//
// radix_sort_pairs: least-significant-digit radix sort with 8-bit digits of
// (key, value) pairs, one pass per digit, each pass three steps: the digit
// histogram of every tile of 2048 pairs, an exclusive scan of the histograms
// in (digit, tile) order (every pair's destination base), and the scatter,
// which ranks a tile's pairs by digit in their input order (per warp by
// __match_any_sync, across the warps and rounds of the tile by running counts
// in shared memory), so each pass is stable and the sort is.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "rm_sort.h"

namespace rmd {

namespace {

constexpr int kScanThreads = 256, kScanRounds = 16, kScanTile = kScanThreads * kScanRounds;  // 4096 items
constexpr int kSortThreads = 256, kSortRounds = 8, kSortTile = kSortThreads * kSortRounds;   // 2048 pairs
constexpr int kDigits = 256;

// Exclusive scan of v over the block (kScanThreads threads); *total receives
// the block's sum.  s: 8 + 1 ints of shared memory.
__device__ __forceinline__ int block_exclusive(int v, int* s, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
      const int c = s[w];
      s[w] = run;
      run += c;
    }
    s[kScanThreads / 32] = run;
  }
  __syncthreads();
  const int ex = s[warp] + x - v;
  total = s[kScanThreads / 32];
  __syncthreads();  // s is reused by the next call
  return ex;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const int* __restrict__ in, int n,
                                                             int* __restrict__ sums) {
  __shared__ int s[kScanThreads / 32 + 1];
  const long long base = (long long)blockIdx.x * kScanTile;
  int acc = 0;
  for (int r = 0; r < kScanRounds; ++r) {
    const long long i = base + r * kScanThreads + threadIdx.x;
    acc += i < n ? in[i] : 0;
  }
  int total;
  block_exclusive(acc, s, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// out[i] = prefix[tile] + the exclusive scan of the tile up to i (prefix null: 0).
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const int* __restrict__ in, int n,
                                                             const int* __restrict__ prefix, int* __restrict__ out) {
  __shared__ int s[kScanThreads / 32 + 1];
  const long long base = (long long)blockIdx.x * kScanTile;
  int carry = prefix ? prefix[blockIdx.x] : 0;
  for (int r = 0; r < kScanRounds; ++r) {
    const long long i = base + r * kScanThreads + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int total;
    const int ex = block_exclusive(v, s, total);
    if (i < n) out[i] = carry + ex;
    carry += total;
  }
}

int scan_tiles(int n) { return (n + kScanTile - 1) / kScanTile; }

// Tile histograms of one digit: hist[d * tiles + t].
__global__ void __launch_bounds__(kSortThreads) k_digit_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                              int tiles, int* __restrict__ hist) {
  __shared__ int h[kDigits];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r) {
    const long long i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kDigits - 1)], 1);
  }
  __syncthreads();
  hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one digit: pair i of tile t goes to offset[d * tiles + t]
// + (pairs of digit d before it in the tile).
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const uint32_t* __restrict__ keys,
                                                                 const int* __restrict__ vals, int n, int shift,
                                                                 int tiles, const int* __restrict__ offset,
                                                                 uint32_t* __restrict__ keys_out,
                                                                 int* __restrict__ vals_out) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ int run[kDigits];          // pairs of each digit in the tile's earlier rounds
  __shared__ int wcnt[kWarps][kDigits];  // this round: per warp count, then its base
  __shared__ int base_of[kDigits];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = 0;
  base_of[threadIdx.x] = offset[threadIdx.x * tiles + blockIdx.x];
  const long long tile0 = (long long)blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const long long i = tile0 + r * kSortThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0u;
    const int d = valid ? int((key >> shift) & (kDigits - 1)) : kDigits;  // kDigits: no pair
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    const int in_warp = __popc(peers & ((1u << lane) - 1u));
    if (valid && lane == leader) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {  // per digit (thread = digit): each warp's base after the earlier warps and rounds
      int acc = run[threadIdx.x];
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const int c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = acc;
        acc += c;
      }
      run[threadIdx.x] = acc;
    }
    __syncthreads();
    if (valid) {
      const int pos = base_of[d] + wcnt[warp][d] + in_warp;
      keys_out[pos] = key;
      vals_out[pos] = vals[i];
    }
    __syncthreads();  // wcnt is cleared for the next round
  }
}

int sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

// Scratch of every level of exclusive_scan (0 for one tile).
size_t scan_levels_bytes(int n) {
  size_t bytes = 0;
  for (int m = std::max(n, 1); m > kScanTile;) {
    const int t = scan_tiles(m);
    bytes += 2 * size_t(t) * sizeof(int);  // tile sums and their scan
    m = t;
  }
  return bytes;
}

}  // namespace

size_t exclusive_scan_temp_bytes(int n) { return std::max<size_t>(scan_levels_bytes(n), 16); }

cudaError_t exclusive_scan(const int* in, int* out, int n, void* temp, size_t temp_bytes, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (temp_bytes < scan_levels_bytes(n)) return cudaErrorInvalidValue;
  const int tiles = scan_tiles(n);
  if (tiles == 1) {
    k_tile_scan<<<1, kScanThreads, 0, st>>>(in, n, nullptr, out);
    return cudaGetLastError();
  }
  int* sums = static_cast<int*>(temp);
  int* prefix = sums + tiles;
  k_tile_sums<<<tiles, kScanThreads, 0, st>>>(in, n, sums);
  cudaError_t e = exclusive_scan(sums, prefix, tiles, prefix + tiles, temp_bytes - 2 * size_t(tiles) * sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_tile_scan<<<tiles, kScanThreads, 0, st>>>(in, n, prefix, out);
  return cudaGetLastError();
}

size_t radix_sort_temp_bytes(int n) {
  const size_t hist = size_t(kDigits) * size_t(sort_tiles(std::max(n, 1)));
  return 2 * hist * sizeof(int) + exclusive_scan_temp_bytes(int(hist));
}

cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* keys_alt, int* vals, int* vals_alt, int n, int bits,
                             void* temp, size_t temp_bytes, bool& in_alt, cudaStream_t st) {
  in_alt = false;
  if (n <= 1 || bits <= 0) return cudaSuccess;
  if (temp_bytes < radix_sort_temp_bytes(n)) return cudaErrorInvalidValue;
  const int tiles = sort_tiles(n);
  const int hn = kDigits * tiles;
  int* hist = static_cast<int*>(temp);
  int* offset = hist + hn;
  void* scan_temp = offset + hn;
  const size_t scan_bytes = temp_bytes - 2 * size_t(hn) * sizeof(int);
  uint32_t* kin = keys;
  uint32_t* kout = keys_alt;
  int* vin = vals;
  int* vout = vals_alt;
  for (int shift = 0; shift < bits; shift += 8) {
    k_digit_hist<<<tiles, kSortThreads, 0, st>>>(kin, n, shift, tiles, hist);
    cudaError_t e = exclusive_scan(hist, offset, hn, scan_temp, scan_bytes, st);
    if (e != cudaSuccess) return e;
    k_digit_scatter<<<tiles, kSortThreads, 0, st>>>(kin, vin, n, shift, tiles, offset, kout, vout);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    std::swap(kin, kout);
    std::swap(vin, vout);
    in_alt = !in_alt;
  }
  return cudaSuccess;
}

}  // namespace rmd

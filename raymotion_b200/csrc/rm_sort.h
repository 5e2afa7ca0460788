// rm_sort.h - radix sort and exclusive prefix sum of the device BVH builds
// and the world preparation (rm_sort.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rmd {

// Scratch bytes exclusive_scan needs for n items.
size_t exclusive_scan_temp_bytes(int n);
// out[i] = in[0] + ... + in[i-1] (out[0] = 0) for n ints, on stream st; in and
// out must not overlap.  cudaErrorInvalidValue if temp is smaller than
// exclusive_scan_temp_bytes(n).
cudaError_t exclusive_scan(const int* in, int* out, int n, void* temp, size_t temp_bytes, cudaStream_t st);

// Scratch bytes radix_sort_pairs needs for n pairs.
size_t radix_sort_temp_bytes(int n);
// Stable sort of n (key, value) pairs by the low `bits` bits of the keys
// (higher bits zero), ping-ponging between (keys, vals) and (keys_alt,
// vals_alt), 8 bits a pass; in_alt tells which pair of arrays holds the
// result.  cudaErrorInvalidValue if temp is smaller than
// radix_sort_temp_bytes(n).
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* keys_alt, int* vals, int* vals_alt, int n, int bits,
                             void* temp, size_t temp_bytes, bool& in_alt, cudaStream_t st);

}  // namespace rmd

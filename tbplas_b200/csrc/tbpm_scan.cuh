// Exclusive scan of int32 counts into int64 offsets on the device (one tile
// pass, one pass over the tile sums, one add pass).  Used by the CSR builders:
// the supercell assembly and the device-side split of uploaded CSR matrices.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tbpm_engine.cuh"

namespace tbpm {
namespace {


constexpr int kScanTile = 1024;

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* warp_sums,
                                                        int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t x = v;
  for (int d = 1; d < 32; d <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int64_t w = lane < nw ? warp_sums[lane] : 0;
    for (int d = 1; d < 32; d <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= d) w += y;
    }
    if (lane < nw) warp_sums[lane] = w;
  }
  __syncthreads();
  const int64_t before = warp ? warp_sums[warp - 1] : 0;
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  return before + x - v;
}

__global__ void __launch_bounds__(kScanTile) scan_tiles_kernel(const int32_t* count, int64_t n,
                                                                int64_t* off, int64_t* tsum) {
  __shared__ int64_t ws[32];
  const int64_t i = (int64_t)blockIdx.x * kScanTile + threadIdx.x;
  const int64_t v = i < n ? count[i] : 0;
  int64_t tot;
  const int64_t ex = block_exclusive_scan(v, ws, &tot);
  if (i < n) off[i] = ex;
  if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanTile) scan_sums_kernel(int64_t* tsum, int64_t n_tiles,
                                                               int64_t* off_end) {
  __shared__ int64_t ws[32];
  int64_t carry = 0;
  for (int64_t b = 0; b < n_tiles; b += kScanTile) {
    const int64_t i = b + threadIdx.x;
    const int64_t v = i < n_tiles ? tsum[i] : 0;
    int64_t tot;
    const int64_t ex = block_exclusive_scan(v, ws, &tot);
    __syncthreads();
    if (i < n_tiles) tsum[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *off_end = carry;
}

__global__ void scan_add_kernel(int64_t* off, int64_t n, const int64_t* tsum) {
  const int64_t i = (int64_t)blockIdx.x * kScanTile + threadIdx.x;
  if (i < n) off[i] += tsum[blockIdx.x];
}

// exclusive scan of count[0..n) into off[0..n] (off[n] = total); returns total
int64_t scan_counts(const int32_t* count, int64_t n, int64_t* off, cudaStream_t st) {
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  DevMem tsum;
  tsum.ensure((size_t)std::max<int64_t>(tiles, 1) * 8);
  scan_tiles_kernel<<<(unsigned)tiles, kScanTile, 0, st>>>(count, n, off, tsum.as<int64_t>());
  scan_sums_kernel<<<1, kScanTile, 0, st>>>(tsum.as<int64_t>(), tiles, off + n);
  scan_add_kernel<<<(unsigned)tiles, kScanTile, 0, st>>>(off, n, tsum.as<int64_t>());
  TBPM_CK(cudaGetLastError());
  int64_t total = 0;
  TBPM_CK(cudaMemcpyAsync(&total, off + n, 8, cudaMemcpyDeviceToHost, st));
  TBPM_CK(cudaStreamSynchronize(st));
  return total;
}

}  // namespace
}  // namespace tbpm

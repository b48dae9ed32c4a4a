// warp.cuh -- warp- and block-level integer scans and reductions.
#pragma once

#include "common.cuh"

namespace gpulda {

__device__ __forceinline__ u64 warp_incl_scan_u64(u64 x, u32 lane) {
#pragma unroll
  for (u32 o = 1; o < 32; o <<= 1) {
    const u64 y = __shfl_up_sync(kFullMask, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ u64 warp_sum_u64(u64 x) {
#pragma unroll
  for (u32 o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
  return x;
}

__device__ __forceinline__ double warp_sum_f64(double x) {
#pragma unroll
  for (u32 o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
  return x;
}

// Block-wide exclusive scan of one u64 per thread; `sh` holds 33 entries.
__device__ __forceinline__ u64 block_excl_scan_u64(u64 v, u64* sh, u64* total) {
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const u64 incl = warp_incl_scan_u64(v, lane);
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    u64 x = lane < nw ? sh[lane] : 0;
    x = warp_incl_scan_u64(x, lane);
    sh[lane] = x;
  }
  __syncthreads();
  const u64 off = warp ? sh[warp - 1] : 0;
  *total = sh[nw - 1];
  __syncthreads();
  return off + incl - v;
}

__device__ __forceinline__ u64 block_sum_u64(u64 v, u64* sh) {
  const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum_u64(v);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  u64 t = 0;
  for (u32 i = 0; i < nw; ++i) t += sh[i];
  __syncthreads();
  return t;
}

}  // namespace gpulda

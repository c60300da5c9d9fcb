// ckd_scan.cuh -- warp / block reductions and scans (shuffle based).
#pragma once
#include <cuda_runtime.h>

namespace ckd {

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; result valid in every thread.  `red` holds NT/32 entries.
template <typename T, int NT>
__device__ __forceinline__ T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[w] = v;
  __syncthreads();
  T s = 0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) s += red[i];
  __syncthreads();
  return s;
}

// Exclusive scan over the block of one value per thread; `total` receives the
// block sum.  `tmp` holds NT/32 entries.
template <typename T, int NT>
__device__ __forceinline__ T block_exclusive_scan(T v, T* tmp, T& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) tmp[w] = inc;
  __syncthreads();
  T wpre = 0, tot = 0;
#pragma unroll
  for (int i = 0; i < NT / 32; ++i) {
    T x = tmp[i];
    wpre += (i < w) ? x : (T)0;
    tot += x;
  }
  __syncthreads();
  total = tot;
  return wpre + inc - v;
}

}  // namespace ckd

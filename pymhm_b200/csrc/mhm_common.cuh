// Shared device helpers for the B200 MHM kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mhm_b200.h"

namespace mhm {

// Error-free transformations (Knuth TwoSum, FMA TwoProd) for accurate sums.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// (hi, lo) += a * b, keeping the product's rounding error.
__device__ __forceinline__ void dd_fma(double& hi, double& lo, double a, double b) {
  double p = a * b;
  double pe = fma(a, b, -p);
  double s, e;
  two_sum(hi, p, s, e);
  hi = s;
  lo += e + pe;
}

__device__ __forceinline__ void dd_add(double& hi, double& lo, double a) {
  double s, e;
  two_sum(hi, a, s, e);
  hi = s;
  lo += e;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reductions through `scratch` (>= 32 doubles); result broadcast to all threads.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double r = 0.0;
  for (int i = 0; i < nw; ++i) r += scratch[i];  // fixed order: deterministic
  return r;
}

__device__ __forceinline__ double block_max(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double r = scratch[0];
  for (int i = 1; i < nw; ++i) r = fmax(r, scratch[i]);
  return r;
}

__device__ __forceinline__ double block_min(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_min(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double r = scratch[0];
  for (int i = 1; i < nw; ++i) r = fmin(r, scratch[i]);
  return r;
}

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

}  // namespace mhm

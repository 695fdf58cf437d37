// Shared device helpers for libtspb (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tspb.h"

#define TSPB_CUDA_CHECK(expr)                                   \
  do {                                                          \
    cudaError_t _e = (expr);                                    \
    if (_e != cudaSuccess) return TSPB_ERR_CUDA;                \
  } while (0)

static inline int tspb_launch_status() {
  return cudaGetLastError() == cudaSuccess ? TSPB_OK : TSPB_ERR_CUDA;
}

namespace tspb {

constexpr unsigned FULL = 0xffffffffu;

// TSPLIB EUC_2D from FP64 coordinates with one IEEE rounding per operation, in the
// order NumPy evaluates `(sqrt(sum(diff * diff)) + 0.5).astype(int64)`: two products,
// one sum, a correctly rounded square root, +0.5, truncation. No contraction to FMA.
__device__ __forceinline__ int euc2d(const double2 p, const double2 q) {
  const double dx = __dsub_rn(p.x, q.x);
  const double dy = __dsub_rn(p.y, q.y);
  const double s = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
  return (int)(long long)__dadd_rn(__dsqrt_rn(s), 0.5);
}

// Distance source: a dense int32 matrix or on-the-fly FP64 coordinates. Matrix reads
// are random gathers with no reuse inside an SM, so they bypass L1 (ld.global.cg) and
// leave L1 to the per-instance k-NN tables.
struct DistSrc {
  const int32_t* dist;
  long long stride;
  const double2* coords;
  __device__ __forceinline__ int operator()(int a, int b) const {
    if (dist != nullptr) return __ldcg(dist + (long long)a * stride + b);
    return euc2d(__ldg(coords + a), __ldg(coords + b));
  }
};

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(FULL, v, o);
    v = w < v ? w : v;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Block-wide min; `scratch` holds >= 32 T. Every thread gets the result.
template <typename T>
__device__ __forceinline__ T block_min(T v, T* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_min(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  T r = scratch[0];
  for (int w = 1; w < nw; ++w) r = scratch[w] < r ? scratch[w] : r;
  return r;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  T r = 0;
  for (int w = 0; w < nw; ++w) r += scratch[w];
  return r;
}

}  // namespace tspb

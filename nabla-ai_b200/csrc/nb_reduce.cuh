// nb_reduce.cuh — deterministic block and grid reductions.
//
// Grid reductions write one partial per block, take a ticket with atomicAdd on
// a counter, and the block that draws the last ticket sums all partials in a
// fixed order and runs a finaliser on the totals. No block ever waits for
// another (no spin), and the result is bitwise reproducible run to run.
#pragma once
#include <cuda_runtime.h>

#include "nb_internal.h"

namespace nb {

enum class RedOp { Sum, Max };

template <RedOp OP>
__device__ __forceinline__ double red_combine(double a, double b) {
  if constexpr (OP == RedOp::Sum) return a + b;
  else return a > b ? a : b;
}
// Per-component operator: bit k of MAXMASK selects max for component k.
template <unsigned MAXMASK>
__device__ __forceinline__ double red_k(int k, double a, double b) {
  return ((MAXMASK >> k) & 1u) ? (a > b ? a : b) : a + b;
}
template <unsigned MAXMASK>
__device__ __forceinline__ double red_id(int k) {
  return ((MAXMASK >> k) & 1u) ? -1.0e308 : 0.0;
}

// Reduce K values across the block; the result is valid in thread 0.
template <int K, unsigned MAXMASK = 0u>
__device__ __forceinline__ void block_reduce(double (&v)[K], double* sh /* K*32 */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarp = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] = red_k<MAXMASK>(k, v[k], __shfl_down_sync(0xffffffffu, v[k], off));
  __syncthreads();  // sh may still be in use by a previous reduction
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = lane < nwarp ? sh[k * 32 + lane] : red_id<MAXMASK>(k);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) t = red_k<MAXMASK>(k, t, __shfl_down_sync(0xffffffffu, t, off));
      v[k] = t;
    }
  }
}

// Grid-wide reduction of K values; `fin(tot)` runs once (one thread of the
// last block) with the totals. Must be called by every thread of every block.
template <int K, unsigned MAXMASK = 0u, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[K], const RedBuf& rb, Fin fin) {
  __shared__ double sh[K * 32];
  __shared__ int is_last;
  block_reduce<K, MAXMASK>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) rb.partials[k * rb.max_blocks + blockIdx.x] = v[k];
    __threadfence();
    const unsigned t = atomicAdd(rb.counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = red_id<MAXMASK>(k);
  for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = red_k<MAXMASK>(k, acc[k], __ldcg(&rb.partials[k * rb.max_blocks + i]));
  block_reduce<K, MAXMASK>(acc, sh);
  if (threadIdx.x == 0) {
    fin(acc);
    *rb.counter = 0u;
  }
}

}  // namespace nb

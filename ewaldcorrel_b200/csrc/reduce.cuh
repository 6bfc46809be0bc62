// Deterministic FP64 reductions: fixed shuffle trees and fixed block order,
// so repeated runs give bit-identical sums (no floating-point atomics).
#pragma once

#include "spme_common.cuh"

namespace spme {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum of NC per-thread values: a fixed shuffle tree per warp, then the
// warps in order.  `red` is shared scratch of (blockDim/32) x NC doubles;
// threads c < NC write the block totals to out[c].  All threads must call.
template <int NC>
__device__ __forceinline__ void block_reduce_n(const double (&acc)[NC], double (*red)[NC], double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NC; c++) {
    const double v = warp_sum(acc[c]);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < NC) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// Sum over nblocks partial vectors (stride `stride` doubles) of component
// c = warp index: lanes take blocks in a fixed stride, then a fixed tree.
// Needs >= NC warps; the totals land in tot[0..NC).
template <int NC>
__device__ __forceinline__ void sum_partials(const double *__restrict__ partials, int nblocks, int stride,
                                             double *tot) {
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c < NC) {
    double v = 0.0;
    for (int b = lane; b < nblocks; b += 32) v += partials[(long)b * stride + c];
    v = warp_sum(v);
    if (lane == 0) tot[c] = v;
  }
  __syncthreads();
}

}  // namespace spme

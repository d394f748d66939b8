// Deterministic grid-wide reductions without spin-waiting: every block
// publishes its partial sums, the last block to arrive (ticket counter) adds
// all partials in block-index order and writes the result.
#pragma once

#include "common.cuh"

namespace fpls {

// vals: k block-level sums in shared memory (valid in every thread).
// partial: gridDim.x * k doubles of global scratch; counter: zero-initialised
// unsigned in global memory (reset to 0 by the last block). out: k doubles.
// Returns true in the block that wrote `out`.
__device__ inline bool last_block_reduce(const double* vals, int k,
                                         double* partial, unsigned* counter,
                                         double* out) {
  __shared__ bool am_last;
  for (int i = threadIdx.x; i < k; i += blockDim.x)
    partial[(long)blockIdx.x * k + i] = vals[i];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(counter, 1u);
    am_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    double s = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(&partial[(long)b * k + i]);
    out[i] = s;
  }
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// Block-level sums of `k` per-thread values laid out as v[i] for i < k,
// written to smem out[0..k). scratch must hold 32 * k doubles.
template <int K>
__device__ inline void block_sums(const double (&v)[K], int k, double* scratch,
                                  double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    if (i < k) {
      const double s = warp_sum(v[i]);
      if (lane == 0) scratch[warp * K + i] = s;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < warps; ++w) s += scratch[w * K + i];
    out[i] = s;
  }
  __syncthreads();
}

}  // namespace fpls

// reduce.cuh -- device helper shared by the kernels that end in a scalar reduction.
#pragma once

#include "common.cuh"

namespace edg {

// Fused reduction tail. Thread 0 of every block has written partial[blockIdx.x]; the last
// block to arrive (counter at partial[kRedBlocks]) sums partial[0..nblk) with its first
// kRedThreads threads in exactly the order of the one-block finishing pass (strided sums,
// then the warp-shuffle tree), writes *out and resets the counter. One launch per reduction
// instead of two, with bit-identical results. Every thread of the block must call it.
__device__ __forceinline__ void finish_in_last_block(double* __restrict__ partial, int nblk, double* __restrict__ out,
                                                     int do_sqrt) {
  __shared__ int s_last;
  __shared__ double s_fin[kRedThreads / 32];
  unsigned int* ctr = reinterpret_cast<unsigned int*>(partial + kRedBlocks);
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial is visible before it is counted
    s_last = atomicAdd(ctr, 1u) == unsigned(nblk) - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  if (threadIdx.x < kRedThreads)
    for (int i = threadIdx.x; i < nblk; i += kRedThreads) v += __ldcg(partial + i);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x < kRedThreads) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_fin[wid] = v;
  }
  __syncthreads();
  if (wid == 0) {
    double r = lane < kRedThreads / 32 ? s_fin[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    if (lane == 0) {
      out[0] = do_sqrt ? sqrt(r) : r;
      *ctr = 0u;
    }
  }
}

}  // namespace edg

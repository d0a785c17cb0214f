// Deterministic grid reductions of complex FP64 partials.
//
// Every block writes its k partial sums (re, im) to ws->partials[j][block];
// the block that takes the last ticket adds the partials in block order
// (one warp per output, lanes striding over blocks, then a fixed shuffle
// tree) and resets the ticket.  The result only depends on n and k, never on
// scheduling, so repeated runs are bit-identical.
#pragma once

#include "common.cuh"

struct qk_workspace {
  int device;
  int nsm;
  double* partials;      // kMaxK * kMaxG * 2 doubles
  unsigned int* ticket;  // one counter
  double* result;        // kMaxK * 2 + 16 doubles of scratch results
};

namespace qkd {

constexpr int kMaxK = 512;  // outputs per reduction
constexpr int kMaxG = 1024; // blocks per reduction

__device__ __forceinline__ double warp_sum(double v) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Called by all threads of every block after the block's partials for
// outputs [0, k) are in global memory.  The last block writes out[2j..2j+1].
__device__ __forceinline__ void grid_finish(double* partials, unsigned int* ticket, int k,
                                            double* out) {
  __shared__ unsigned int s_ticket;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket = atomicAdd(ticket, 1u);
  __syncthreads();
  if (s_ticket != gridDim.x - 1) return;
  __threadfence();
  const int G = gridDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = warp; j < k; j += nw) {
    double re = 0.0, im = 0.0;
    const double* pj = partials + size_t(j) * G * 2;
    for (int g = lane; g < G; g += 32) {
      re += __ldcg(pj + 2 * g);
      im += __ldcg(pj + 2 * g + 1);
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) { out[2 * j] = re; out[2 * j + 1] = im; }
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// grid_finish over n partials per output (work items such as chunks of
// tiles) instead of one per block.
__device__ __forceinline__ void grid_finish_n(double* partials, unsigned int* ticket, int k, double* out,
                                              uint32_t n) {
  __shared__ unsigned int s_ticket;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket = atomicAdd(ticket, 1u);
  __syncthreads();
  if (s_ticket != gridDim.x - 1) return;
  __threadfence();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = warp; j < k; j += nw) {
    double re = 0.0, im = 0.0;
    const double* pj = partials + size_t(j) * n * 2;
    for (uint32_t g = lane; g < n; g += 32) {
      re += __ldcg(pj + 2 * size_t(g));
      im += __ldcg(pj + 2 * size_t(g) + 1);
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) { out[2 * j] = re; out[2 * j + 1] = im; }
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// As grid_finish for one output, with the partials indexed by work item
// (n of them, e.g. sector blocks) instead of by block: the sum then does not
// depend on which block processed which item (dynamic work queues).
__device__ __forceinline__ void grid_finish_items(double* partials, unsigned int* ticket, uint32_t n, double* out) {
  __shared__ unsigned int s_ticket;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_ticket = atomicAdd(ticket, 1u);
  __syncthreads();
  if (s_ticket != gridDim.x - 1) return;
  __threadfence();
  if (threadIdx.x < 32) {
    double re = 0.0, im = 0.0;
    for (uint32_t g = threadIdx.x; g < n; g += 32) {
      re += __ldcg(partials + 2 * size_t(g));
      im += __ldcg(partials + 2 * size_t(g) + 1);
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (threadIdx.x == 0) { out[0] = re; out[1] = im; *ticket = 0u; }
  }
}

// Block-level sum of (re, im) over all threads; result valid in thread 0.
__device__ __forceinline__ void block_sum2(double& re, double& im, double* sbuf /*2*nwarps*/) {
  re = warp_sum(re);
  im = warp_sum(im);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (lane == 0) { sbuf[2 * warp] = re; sbuf[2 * warp + 1] = im; }
  __syncthreads();
  if (threadIdx.x == 0) {
    re = 0.0; im = 0.0;
    for (int w = 0; w < nw; ++w) { re += sbuf[2 * w]; im += sbuf[2 * w + 1]; }
  }
  __syncthreads();
}

}  // namespace qkd

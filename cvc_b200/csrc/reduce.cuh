// Deterministic single-launch reductions.
//
// Every thread accumulates a fixed, grid-stride subset of the elements in a
// fixed order; each block reduces its threads with warp shuffles and a fixed
// shared-memory tree and writes one partial per output; the last block to
// finish (found with a completion counter) sums the partials in block order
// and runs an epilogue on the totals.  Grid and block sizes are functions of
// n only, so the same inputs give the same bits on every call -- the
// property the reference's serial left-to-right sums have, with a different
// (tree) summation order.
#pragma once

#include <cuda_runtime.h>

#include "cvcb_internal.h"

namespace cvcb {

constexpr int kRedThreads = 256;

inline int red_blocks(size_t n) {
  size_t b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
  if (b < 1) b = 1;
  if (b > (size_t)kMaxRedBlocks) b = kMaxRedBlocks;
  return (int)b;
}

template <int NOUT>
__device__ __forceinline__ void block_sum(double (&v)[NOUT], double (*sh)[kRedThreads / 32]) {
#pragma unroll
  for (int q = 0; q < NOUT; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NOUT; ++q) sh[q][warp] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NOUT; ++q) {
      double x = lane < kRedThreads / 32 ? sh[q][lane] : 0.0;
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[q] = x;
    }
  }
  __syncthreads();
}

// F: __device__ void operator()(size_t k, double (&acc)[NOUT]) -- adds element k
// E: __device__ void operator()(const double (&tot)[NOUT])     -- runs once
template <int NOUT, class F, class E>
__global__ void __launch_bounds__(kRedThreads)
    k_reduce(F f, E e, size_t n, double *__restrict__ partials, unsigned *__restrict__ counter,
             const int *__restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double sh[NOUT][kRedThreads / 32];
  __shared__ bool last;
  double v[NOUT];
#pragma unroll
  for (int q = 0; q < NOUT; ++q) v[q] = 0.0;
  for (size_t k = (size_t)blockIdx.x * kRedThreads + threadIdx.x; k < n;
       k += (size_t)gridDim.x * kRedThreads)
    f(k, v);
  block_sum<NOUT>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NOUT; ++q) partials[(size_t)blockIdx.x * NOUT + q] = v[q];
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NOUT; ++q) v[q] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kRedThreads)
#pragma unroll
    for (int q = 0; q < NOUT; ++q) v[q] += __ldcg(partials + (size_t)b * NOUT + q);
  block_sum<NOUT>(v, sh);
  if (threadIdx.x == 0) {
    *counter = 0;
    e(v);
  }
}

template <int NOUT, class F, class E>
int launch_reduce(cvcb_lattice *L, F f, E e, size_t n, const int *skip = nullptr) {
  const int blocks = red_blocks(n);
  k_reduce<NOUT><<<blocks, kRedThreads, 0, L->stream>>>(f, e, n, L->partials, L->red_counter, skip);
  CVCB_LAUNCHED(L);
  return CVCB_OK;
}

// Stores the totals into a device array.
template <int NOUT>
struct StoreTotals {
  double *out;
  __device__ void operator()(const double (&t)[NOUT]) const {
#pragma unroll
    for (int q = 0; q < NOUT; ++q) out[q] = t[q];
  }
};

}  // namespace cvcb

// Deterministic FP64 reductions shared by the density, Jacobi and grid-utility paths.
#pragma once

#include "qmt_common.cuh"

namespace qmt {

constexpr int RED_CHUNK = 8192;     // elements per block in the first pass
constexpr int RED_THREADS = 256;

// Block-wide FP64 sum in a fixed order; result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; ++i) r += sh[i];
  __syncthreads();
  return r;
}

// Sums n doubles into *out with one block of 1024 threads in a fixed order.
__global__ void reduce_partials_kernel(const double* __restrict__ in, int64_t n, double* __restrict__ out,
                                       int nvals, int64_t stride);

qmt_status reduce_partials(const double* in, int64_t n, double* out, int nvals, int64_t stride,
                           cudaStream_t s);

}  // namespace qmt

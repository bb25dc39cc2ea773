// kernel_common.cuh -- device helpers shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kernels.h"

namespace vpfft {

constexpr int kVoxelBlock = 128;
constexpr int kFinishThreads = 256;

// Fixed-order block reduction of W doubles per thread; thread 0 of the block
// writes the W sums to out.
template <int W, int BLOCK>
__device__ __forceinline__ void block_reduce_store(double (&acc)[W], double* out) {
  __shared__ double sm[BLOCK / 32][W];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    double v = acc[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) sm[warp][k] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      double v = lane < BLOCK / 32 ? sm[lane][k] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) out[k] = v;
    }
  }
}

template <typename S>
__device__ __forceinline__ void load_R(const S* __restrict__ R, long long n, long long v,
                                       double r[9]) {
#pragma unroll
  for (int k = 0; k < 9; ++k) r[k] = (double)R[k * n + v];
}
template <typename S>
__device__ __forceinline__ void load_tau(const S* __restrict__ crss, const double* uni,
                                         long long n, long long v, double tau[kNS]) {
  if (crss) {
#pragma unroll
    for (int k = 0; k < kNS; ++k) tau[k] = (double)crss[k * n + v];
  } else {
#pragma unroll
    for (int k = 0; k < kNS; ++k) tau[k] = uni[k];
  }
}
template <typename S>
__device__ __forceinline__ void load5(const S* __restrict__ f, long long n, long long v,
                                      double x[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) x[c] = (double)f[c * n + v];
}
template <typename S>
__device__ __forceinline__ void store5(S* __restrict__ f, long long n, long long v,
                                       const double x[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) f[c * n + v] = (S)x[c];
}


// Slot of block b of a batched launch and the block's index within the slot.
__device__ __forceinline__ int batch_slot(const BatchLaunch& bl, int b, int* local) {
  if (bl.per > 0) {  // equal counts (the passes of a size class): no search
    const int k = b / bl.per;
    *local = b - k * bl.per;
    return bl.slot[k];
  }
  int lo = 0, hi = bl.m - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bl.prefix[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  *local = b - bl.prefix[lo];
  return bl.slot[lo];
}

// Block-cooperative copy of a trivially copyable struct (8-byte multiple) into
// shared memory; the caller synchronises.
template <typename T>
__device__ __forceinline__ void copy_struct(T* dst, const T* src) {
  static_assert(sizeof(T) % 8 == 0, "8-byte multiple");
  auto* d = reinterpret_cast<unsigned long long*>(dst);
  auto* s = reinterpret_cast<const unsigned long long*>(src);
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x) d[i] = s[i];
}

// Reductions and convergence test of one iteration (defined in kernels.cu).
__global__ void k_iter_finish(const double* partials, int nparts, IterCtrl* ctrl, double* hist);
template <typename S>
__global__ void k_iter_finish_batch(const SlotDesc<S>* desc, BatchLaunch bl);
// Compensated fixed-order column sums of partials[nparts][width] (kernels.cu).
__global__ void k_column_sums(const double* partials, int nparts, int width, double* out);

}  // namespace vpfft

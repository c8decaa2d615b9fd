// Device helpers shared by the kernel headers: fixed-order block reductions
// and vector loads/stores of R consecutive elements.
#pragma once

#include <cstring>

#include "common.cuh"

namespace hb {

constexpr int kThreads = 256;

// Sum of v over the block (any whole number of warps up to 1024 threads), valid
// in thread 0. Fixed shuffle tree: deterministic.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_part[32];  // up to 1024 threads
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_part[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = lane < (int)(blockDim.x >> 5) ? warp_part[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double warp_part[32];  // up to 1024 threads
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_part[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = lane < (int)(blockDim.x >> 5) ? warp_part[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
  }
  __syncthreads();
  return s;
}

// R consecutive elements through one or two vector loads (p aligned to R elements).
template <typename T, int R>
__device__ __forceinline__ void load_vec(const T* __restrict__ p, T (&out)[R]) {
  static_assert(sizeof(T) * R == 4 || sizeof(T) * R == 8 || sizeof(T) * R == 16 || sizeof(T) * R == 32, "");
  if constexpr (sizeof(T) * R == 4) {
    out[0] = *p;
  } else if constexpr (sizeof(T) * R == 8) {
    const uint2 u = *reinterpret_cast<const uint2*>(p);
    memcpy(out, &u, 8);
  } else if constexpr (sizeof(T) * R == 16) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    memcpy(out, &u, 16);
  } else {
    const uint4 u0 = reinterpret_cast<const uint4*>(p)[0];
    const uint4 u1 = reinterpret_cast<const uint4*>(p)[1];
    memcpy(out, &u0, 16);
    memcpy(reinterpret_cast<char*>(out) + 16, &u1, 16);
  }
}

template <typename T, int R>
__device__ __forceinline__ void store_vec(T* __restrict__ p, const T (&in)[R]) {
  if constexpr (sizeof(T) * R == 4) {
    *p = in[0];
  } else if constexpr (sizeof(T) * R == 8) {
    uint2 u;
    memcpy(&u, in, 8);
    *reinterpret_cast<uint2*>(p) = u;
  } else if constexpr (sizeof(T) * R == 16) {
    uint4 u;
    memcpy(&u, in, 16);
    *reinterpret_cast<uint4*>(p) = u;
  } else {
    uint4 u0, u1;
    memcpy(&u0, in, 16);
    memcpy(&u1, reinterpret_cast<const char*>(in) + 16, 16);
    reinterpret_cast<uint4*>(p)[0] = u0;
    reinterpret_cast<uint4*>(p)[1] = u1;
  }
}

}  // namespace hb

// Host shim under which the reference's CUDA kernels compile as plain C++.
// TEST INFRASTRUCTURE (oracle/_ref only).
//
// Every kernel in the reference uses a grid-stride loop over
// tid = blockDim.x*blockIdx.x + threadIdx.x with stride blockDim.x*gridDim.x,
// so a "grid" of one thread runs each loop over every item, in order.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <functional>
#include <string>
#include <vector>

#include "types.h"

#define __global__
#define __device__
#define __constant__
#define __host__
#define __forceinline__ inline

struct ref_shim_dim3 {
  unsigned x, y, z;
};
static const ref_shim_dim3 blockDim = {1, 1, 1};
static const ref_shim_dim3 gridDim = {1, 1, 1};
static const ref_shim_dim3 blockIdx = {0, 0, 0};
static const ref_shim_dim3 threadIdx = {0, 0, 0};
static inline void __syncthreads() {}

// Host shim used ONLY to compile the reference's unmodified projector sources
// (src/cpp/tf_custom_ops/tor.cu.cc, siddon.cu.cc) as serial C++ on the CPU.
// Test infrastructure: the result is a checker and a CPU baseline, never shipped.
//
// Every CUDA launch becomes a plain call with one block of one thread, so each
// grid-stride loop (tor.cu.cc:255, siddon.cu.cc:443) visits all events in order,
// and atomicAdd becomes an ordinary read-modify-write.
#pragma once
#include <cmath>
#include <cstring>
#include <limits>

#define __device__
#define __global__
#define __host__

struct SrfShimDim3 {
    unsigned int x, y, z;
};
static const SrfShimDim3 threadIdx = {0u, 0u, 0u};
static const SrfShimDim3 blockIdx = {0u, 0u, 0u};
static const SrfShimDim3 blockDim = {1u, 1u, 1u};
static const SrfShimDim3 gridDim = {1u, 1u, 1u};

static inline float atomicAdd(float *address, float value) {
    float old = *address;
    *address = old + value;
    return old;
}

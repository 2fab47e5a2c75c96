// Stand-in for the CUDA runtime header when the reference projector sources are
// compiled for the host CPU (see host_shim.h). Device pointers are host pointers.
#pragma once
#include <cstddef>
#include <cstring>

enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
};

static inline int cudaMemcpy(void *dst, const void *src, size_t bytes, cudaMemcpyKind) {
    std::memcpy(dst, src, bytes);
    return 0;
}

static inline int cudaMemset(void *dst, int value, size_t bytes) {
    std::memset(dst, value, bytes);
    return 0;
}

// Shared pieces of the srf_b200 CUDA library: status handling, launch sizing and the
// float helpers that pin the rounding of every geometric quantity.
//
// Rounding discipline. The projectors make discrete choices from float values —
// which slices a LOR crosses, where a TOR patch starts (a truncating float->int
// conversion), which voxel a Siddon ray enters and in which order it leaves them.
// A one-ulp difference there moves a whole patch column or a voxel boundary, so these
// quantities are computed with explicit round-to-nearest intrinsics (__fadd_rn,
// __fmul_rn, __fdiv_rn, __fsqrt_rn, __fmaf_rn), which the compiler never re-associates
// or fuses. Where the reference source has `a*b + c` in device code, nvcc's default
// contraction turns it into one fused multiply-add, and the code here writes
// __fmaf_rn(a, b, c) for it. Continuous weights (Gaussians, TOF factors, sums) only
// need to stay within float accuracy and use the fast paths.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/srf_b200.h"

namespace srf {

constexpr float kTofThreshold = 405758.0f;  // tor.cu.cc:20, siddon.cu.cc:15
constexpr float kLog2e = 1.4426950408889634f;

void set_cuda_error(cudaError_t e);

// Records and maps the last CUDA error of a launch sequence.
inline int check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    return SRF_OK;
}

int num_sms();

// Stream-ordered scratch from the library's own memory pool on the current device. The
// pool keeps what it has reserved across calls (release threshold: never), so repeated
// calls of the same size neither map nor unmap device memory; srf_release_scratch()
// returns it. Allocation and free are capturable in CUDA graphs.
cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream);

// Process-wide count of kernels this library has launched (srf_launch_count); every
// launch site adds its launches.
void count_launches(int n);

// Grid for a grid-stride kernel: enough blocks to fill every SM `per_sm` times, but
// no more than the work needs.
inline int stride_grid(int64_t work_items, int items_per_block, int per_sm) {
    int64_t need = (work_items + items_per_block - 1) / items_per_block;
    int64_t cap = (int64_t)num_sms() * per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

inline bool finite3(const float *v) {
    for (int i = 0; i < 3; i++)
        if (!(v[i] == v[i]) || v[i] > 3.0e38f || v[i] < -3.0e38f) return false;
    return true;
}

}  // namespace srf

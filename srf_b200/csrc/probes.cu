// Peak probes for the roofline denominators that are not a plain HBM copy: the L2 read
// bandwidth seen by all SMs (a buffer that stays L2-resident, read repeatedly with
// 16-byte loads), the SFU ex2 throughput (independent chains of ex2.approx), the
// shared-memory read bandwidth and the shared-memory float atomicAdd rate (the TOR slab
// kernels serve their voxel samples from shared memory). They
// have no counterpart in the reference; the bench runs them once per invocation and
// times them with CUDA events on the caller's stream.

#include "srf_common.cuh"

namespace srf {
namespace {

constexpr int kProbeThreads = 512;

__global__ void __launch_bounds__(kProbeThreads) l2_read_kernel(const float4 *buf, int64_t n,
                                                                  int reps, float *sink) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    float acc = 0.0f;
    for (int r = 0; r < reps; r++) {
        for (int64_t i = tid; i < n; i += nt) {
            const float4 v = __ldcg(buf + i);  // cache in L2 only
            acc += (v.x + v.y) + (v.z + v.w);
        }
    }
    sink[tid] = acc;
}

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__global__ void __launch_bounds__(kProbeThreads) ex2_kernel(int iters, float *sink) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = -0.001f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = -ex2_approx(x[k]);  // stays in [-1, 0)
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    sink[tid] = s;
}

// Shared-memory read bandwidth: every CTA reads a 32 KB shared buffer with 16-byte loads,
// a warp's lanes on consecutive addresses (no bank conflict), four independent sums.
constexpr int kSmemProbeThreads = 1024;
constexpr int kSmemVec = 2048;  // float4 elements = 32 KB

__global__ void __launch_bounds__(kSmemProbeThreads) smem_read_kernel(int iters, float *sink) {
    __shared__ float4 buf[kSmemVec];
    for (int i = threadIdx.x; i < kSmemVec; i += kSmemProbeThreads)
        buf[i] = make_float4(1e-3f * i, 2e-3f, 3e-3f, 4e-3f);
    __syncthreads();
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int it = 0; it < iters; it++) {
        const float4 v = buf[(threadIdx.x + it * 32) & (kSmemVec - 1)];
        a.x += v.x;
        a.y += v.y;
        a.z += v.z;
        a.w += v.w;
    }
    sink[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = (a.x + a.y) + (a.z + a.w);
}

// Shared-memory float atomicAdd throughput: every thread adds into a 32 KB shared buffer.
// random = 0: a warp's lanes hit 32 consecutive floats (distinct banks); random = 1: a
// hashed address per lane and step (bank conflicts as random scatter meets them).
constexpr int kSmemAtomFloats = 8192;

__global__ void __launch_bounds__(kSmemProbeThreads) smem_atomic_kernel(int iters, int random,
                                                                        float *sink) {
    __shared__ float buf[kSmemAtomFloats];
    for (int i = threadIdx.x; i < kSmemAtomFloats; i += kSmemProbeThreads) buf[i] = 0.0f;
    __syncthreads();
    const unsigned tid = threadIdx.x;
    for (int it = 0; it < iters; it++) {
        unsigned idx;
        if (random) {
            unsigned h = tid * 0x9E3779B1u + (unsigned)it * 0x85EBCA77u;
            h ^= h >> 15;
            h *= 0x2C1B3C6Du;
            h ^= h >> 13;
            idx = h;
        } else {
            idx = tid + (unsigned)it * 1024u;
        }
        atomicAdd(&buf[idx & (kSmemAtomFloats - 1)], 1.0f);
    }
    __syncthreads();
    sink[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = buf[tid * 8];
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int srf_probe_threads(int64_t *n_threads) {
    if (!n_threads) return SRF_ERR_INVALID_ARGUMENT;
    *n_threads = (int64_t)num_sms() * 4 * kProbeThreads;
    return SRF_OK;
}

extern "C" int srf_probe_l2_read(const float *buf, int64_t n_floats, int reps, float *sink,
                                 void *stream) {
    if (!buf || !sink || n_floats < 4 || reps < 1) return SRF_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(buf) & 15u) != 0) return SRF_ERR_INVALID_ARGUMENT;
    l2_read_kernel<<<num_sms() * 4, kProbeThreads, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<const float4 *>(buf), n_floats / 4, reps, sink);
    count_launches(1);
    return check_launch();
}

extern "C" int srf_probe_ex2(int iters, float *sink, void *stream) {
    if (!sink || iters < 1) return SRF_ERR_INVALID_ARGUMENT;
    ex2_kernel<<<num_sms() * 4, kProbeThreads, 0, (cudaStream_t)stream>>>(iters, sink);
    count_launches(1);
    return check_launch();
}

extern "C" int srf_probe_smem_threads(int64_t *n_threads) {
    if (!n_threads) return SRF_ERR_INVALID_ARGUMENT;
    *n_threads = (int64_t)num_sms() * 2 * kSmemProbeThreads;
    return SRF_OK;
}

extern "C" int srf_probe_smem_read(int iters, float *sink, void *stream) {
    if (!sink || iters < 1) return SRF_ERR_INVALID_ARGUMENT;
    smem_read_kernel<<<num_sms() * 2, kSmemProbeThreads, 0, (cudaStream_t)stream>>>(iters, sink);
    count_launches(1);
    return check_launch();
}

extern "C" int srf_probe_smem_atomic(int iters, int random, float *sink, void *stream) {
    if (!sink || iters < 1 || (random != 0 && random != 1)) return SRF_ERR_INVALID_ARGUMENT;
    smem_atomic_kernel<<<num_sms() * 2, kSmemProbeThreads, 0, (cudaStream_t)stream>>>(
        iters, random, sink);
    count_launches(1);
    return check_launch();
}

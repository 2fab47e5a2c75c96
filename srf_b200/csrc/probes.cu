// Peak probes for the roofline denominators that are not a plain HBM copy: the L2 read
// bandwidth seen by all SMs (a buffer that stays L2-resident, read repeatedly with
// 16-byte loads) and the SFU ex2 throughput (independent chains of ex2.approx). They
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

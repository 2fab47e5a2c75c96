// Library-wide runtime pieces: status strings, the per-thread last CUDA error, the
// SM-count cache used for grid sizing, and the image-algebra kernels of the MLEM/OSEM
// update (src/python/srf/model/recon_step.py:48-49).

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "srf_common.cuh"

namespace srf {

namespace {
thread_local int g_last_cuda_error = 0;
constexpr int kMaxDevices = 64;
std::atomic<int> g_sms[kMaxDevices];
std::atomic<long long> g_launches{0};
}  // namespace

void set_cuda_error(cudaError_t e) { g_last_cuda_error = (int)e; }

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};
}  // namespace

cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaMallocAsync(ptr, bytes, stream);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (!g_pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&g_pools[dev], &props);
            if (e != cudaSuccess) {
                g_pools[dev] = nullptr;
                return e;
            }
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
}

int num_sms() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
    int v = g_sms[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
        v = 148;
    g_sms[dev].store(v, std::memory_order_relaxed);
    return v;
}

namespace {

__global__ void mlem_update_kernel(float *__restrict__ image, const float *__restrict__ effinv,
                                   const float *__restrict__ bp, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // 16-byte vectors for the bulk, scalars for the tail and for unaligned pointers.
    const bool vec = ((reinterpret_cast<uintptr_t>(image) | reinterpret_cast<uintptr_t>(effinv) |
                       reinterpret_cast<uintptr_t>(bp)) & 15u) == 0;
    int64_t done = 0;
    if (vec) {
        const int64_t n4 = n / 4;
        float4 *im4 = reinterpret_cast<float4 *>(image);
        const float4 *e4 = reinterpret_cast<const float4 *>(effinv);
        const float4 *b4 = reinterpret_cast<const float4 *>(bp);
        for (int64_t k = i; k < n4; k += stride) {
            float4 x = im4[k], e = __ldg(e4 + k), b = __ldg(b4 + k);
            x.x = x.x * e.x * b.x;
            x.y = x.y * e.y * b.y;
            x.z = x.z * e.z * b.z;
            x.w = x.w * e.w * b.w;
            im4[k] = x;
        }
        done = n4 * 4;
    }
    for (int64_t k = done + i; k < n; k += stride) image[k] = image[k] * effinv[k] * bp[k];
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" const char *srf_status_string(int status) {
    switch (status) {
        case SRF_OK: return "ok";
        case SRF_ERR_INVALID_ARGUMENT: return "invalid argument";
        case SRF_ERR_CUDA: return "CUDA error";
        case SRF_ERR_UNSUPPORTED: return "unsupported parameters";
        default: return "unknown status";
    }
}

extern "C" int srf_last_cuda_error(void) { return g_last_cuda_error; }

extern "C" int srf_version(void) { return 1; }

extern "C" int srf_release_scratch(void) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    for (int d = 0; d < kMaxDevices; d++) {
        if (!g_pools[d]) continue;
        cudaError_t e = cudaMemPoolTrimTo(g_pools[d], 0);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return SRF_ERR_CUDA;
        }
    }
    return SRF_OK;
}

extern "C" int64_t srf_launch_count(void) {
    return (int64_t)g_launches.load(std::memory_order_relaxed);
}

extern "C" int srf_mlem_update(float *image, const float *effinv, const float *bp,
                               int64_t num_voxels, void *stream) {
    if (num_voxels < 0) return SRF_ERR_INVALID_ARGUMENT;
    if (num_voxels == 0) return SRF_OK;
    if (!image || !effinv || !bp) return SRF_ERR_INVALID_ARGUMENT;
    const int block = 256;
    const int grid = stride_grid((num_voxels + 3) / 4, block, 4);
    mlem_update_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(image, effinv, bp, num_voxels);
    count_launches(1);
    return check_launch();
}

// Reordering of preprocessed LOR records by the shape of their tube's section, inside
// blocks of 4096 consecutive records (no counterpart in the reference; an optional step
// between preprocessing and the projectors).
//
// A record's section box spans sqrt((1 - uy^2)/q) by sqrt((1 - ux^2)/q), q = 1 - ux^2 - uy^2,
// with (ux, uy) the in-slice components of its unit direction. The slab kernels hand a
// warp 32 consecutive LORs of a slab and walk the largest box among them, so records of
// similar direction side by side walk fewer voxel slots. Sorting only inside blocks keeps
// every stretch of the per-slab lists a mix of directions, so the persistent grid's equal
// shares stay equal work. The class key quantises both extents to 16 levels over [1, 2)
// (dominant-axis groups have extents in [1, sqrt(3)]); inside a class, records are ordered
// by where the LOR starts along the slice axis (8 mm bins), so a warp's segments cover
// similar slice counts. Records with NaN sort last. The sort is a stable block radix sort,
// so the order is deterministic.

#include <atomic>

#include <cub/block/block_radix_sort.cuh>

#include "srf_common.cuh"

namespace srf {
namespace {

constexpr int kOrderThreads = 512;
constexpr int kOrderItems = 8;
constexpr int kOrderBlock = kOrderThreads * kOrderItems;  // 4096 records

__device__ __forceinline__ int direction_class(const float *r) {
    const float dx = r[3] - r[0], dy = r[4] - r[1], dz = r[5] - r[2];
    const float inv = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
    const float ux2 = dx * dx * inv * inv, uy2 = dy * dy * inv * inv;
    const float q = fmaxf(1.0f - ux2 - uy2, 1e-6f);
    const float bx = sqrtf((1.0f - uy2) / q), by = sqrtf((1.0f - ux2) / q);
    if (!(bx == bx) || !(by == by)) return 255 << 8;
    const int kx = min(15, max(0, (int)((bx - 1.0f) * 16.0f)));
    const int ky = min(15, max(0, (int)((by - 1.0f) * 16.0f)));
    // secondary: where the LOR starts along the slice axis (8 mm bins over +-1 m)
    const float zs = fminf(r[2], r[5]);
    const int kz = (zs == zs) ? min(255, max(0, (int)((zs + 1024.0f) * 0.125f))) : 255;
    return ((kx * 16 + ky) << 8) | kz;
}

// Records of up to kStageCols columns: the block's records pass through shared memory, so
// both the loads and the stores are contiguous runs (records are 28-40 bytes, so one
// thread per record would touch a new sector per lane and column). Same keys, same
// stable sort, same output as order_kernel.
constexpr int kStageCols = 10;
constexpr size_t kStageBytes = sizeof(float) * kOrderBlock * kStageCols;  // 160 KB

__global__ void __launch_bounds__(kOrderThreads)
order_staged_kernel(const float *__restrict__ in, float *__restrict__ out, int64_t n, int ncols,
                    int64_t stride) {
    using Sort = cub::BlockRadixSort<int, kOrderThreads, kOrderItems, int>;
    __shared__ typename Sort::TempStorage tmp;
    __shared__ int key_perm[kOrderBlock];  // keys by record, then source record by position
    extern __shared__ float stage[];       // [kOrderBlock][ncols]
    const int64_t base = (int64_t)blockIdx.x * kOrderBlock;
    const int cnt = (int)min((int64_t)kOrderBlock, n - base);
    const int total = cnt * ncols;
    if (stride == ncols) {
        const float *src = in + base * stride;
        for (int e = threadIdx.x; e < total; e += kOrderThreads) stage[e] = src[e];
    } else {
        for (int e = threadIdx.x; e < total; e += kOrderThreads) {
            const int r = e / ncols;
            stage[e] = in[(base + r) * stride + (e - r * ncols)];
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < kOrderBlock; j += kOrderThreads)
        key_perm[j] = j < cnt ? direction_class(stage + j * ncols) : (256 << 8);
    __syncthreads();
    int key[kOrderItems], idx[kOrderItems];
#pragma unroll
    for (int k = 0; k < kOrderItems; k++) {
        const int j = threadIdx.x * kOrderItems + k;  // blocked arrangement: stable order
        key[k] = key_perm[j];
        idx[k] = j;
    }
    Sort(tmp).Sort(key, idx, 0, 17);  // synchronises: every key is read before the writes below
#pragma unroll
    for (int k = 0; k < kOrderItems; k++) key_perm[threadIdx.x * kOrderItems + k] = idx[k];
    __syncthreads();
    if (stride == ncols) {
        float *dst = out + base * stride;
        for (int e = threadIdx.x; e < total; e += kOrderThreads) {
            const int r = e / ncols;
            dst[e] = stage[key_perm[r] * ncols + (e - r * ncols)];
        }
    } else {
        for (int e = threadIdx.x; e < total; e += kOrderThreads) {
            const int r = e / ncols, c = e - r * ncols;
            out[(base + r) * stride + c] = stage[key_perm[r] * ncols + c];
        }
    }
}

__global__ void __launch_bounds__(kOrderThreads)
order_kernel(const float *__restrict__ in, float *__restrict__ out, int64_t n, int ncols,
             int64_t stride) {
    using Sort = cub::BlockRadixSort<int, kOrderThreads, kOrderItems, int>;
    __shared__ typename Sort::TempStorage tmp;
    const int64_t base = (int64_t)blockIdx.x * kOrderBlock;
    int key[kOrderItems], idx[kOrderItems];
#pragma unroll
    for (int k = 0; k < kOrderItems; k++) {
        const int j = threadIdx.x * kOrderItems + k;  // blocked arrangement: stable order
        const int64_t t = base + j;
        idx[k] = j;
        key[k] = t < n ? direction_class(in + t * stride) : (256 << 8);  // padding sorts last
    }
    Sort(tmp).Sort(key, idx, 0, 17);
#pragma unroll
    for (int k = 0; k < kOrderItems; k++) {
        const int j = threadIdx.x * kOrderItems + k;
        const int64_t dst = base + j;
        if (dst >= n) continue;
        const float *src = in + (base + idx[k]) * stride;
        float *d = out + dst * stride;
        for (int c = 0; c < ncols; c++) d[c] = src[c];
    }
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int srf_order_by_direction(const float *records, int64_t num_records, int ncols,
                                      int64_t record_stride, float *out, void *stream) {
    if (num_records < 0 || ncols < 6 || record_stride < ncols) return SRF_ERR_INVALID_ARGUMENT;
    if (num_records == 0) return SRF_OK;
    if (!records || !out || records == out) return SRF_ERR_INVALID_ARGUMENT;
    const int64_t blocks = (num_records + kOrderBlock - 1) / kOrderBlock;
    if (blocks > INT32_MAX) return SRF_ERR_UNSUPPORTED;
    if (ncols <= kStageCols) {
        static std::atomic<unsigned long long> attr_set{0};  // per device
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
        if (!(attr_set.load() & (1ull << dev))) {
            const cudaError_t e = cudaFuncSetAttribute(
                order_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)kStageBytes);
            if (e != cudaSuccess) {
                set_cuda_error(e);
                return SRF_ERR_CUDA;
            }
            attr_set.fetch_or(1ull << dev);
        }
        order_staged_kernel<<<(int)blocks, kOrderThreads,
                              sizeof(float) * kOrderBlock * (size_t)ncols,
                              (cudaStream_t)stream>>>(records, out, num_records, ncols,
                                                      record_stride);
    } else {
        order_kernel<<<(int)blocks, kOrderThreads, 0, (cudaStream_t)stream>>>(
            records, out, num_records, ncols, record_stride);
    }
    count_launches(1);
    return check_launch();
}

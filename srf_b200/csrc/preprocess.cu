// LOR preprocessing on the GPU: the reference's host numpy pass
// src/python/srf/preprocess/function/on_tor_lors.py (recon_process :251-262,
// map_process :243-248) as three kernels.
//
// Per event (float32 arithmetic in numpy's operation order; numpy never fuses a*b+c,
// so every product and sum here is a separately rounded __fmul_rn/__fadd_rn):
//   f  = (dx^2+dy^2)^2 / (x1^2+x2^2+y1^2+y2^2) / L^2 / 2          (:137-166)
//   dominant axis with the reference tie rules                      (:70-77)
//   swap endpoints so the dominant coordinate grows, negating TOF    (:175-193)
//   recon only: TOF centre C and the cut to C -/+ 3 sigma            (:196-229)
//   column permutation that puts the dominant axis last              (:246-247, :259-260)
//
// Output order is the reference's: the x group, then y, then z; inside a group the
// events that kept their orientation (ascending index), then the swapped ones
// (ascending index) — np.intersect1d sorts, SwapPointsOrder vstacks positive/negative.
// That is a stable partition into six buckets (axis, swapped), done with a per-tile
// count, a scan over tiles and a stable scatter (ballot ranks inside each warp).

#include <mutex>

#include "lor_prep.cuh"
#include "srf_common.cuh"

namespace srf {
namespace {

constexpr int kThreads = 512;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

struct PreParams {
    const float *events;
    int64_t n, stride;
    int recon, cut;
    float limit;
    unsigned char *bucket;   // [n]
    int *tile_counts;        // [ntiles * kBuckets]
    int64_t *tile_offsets;   // [ntiles * kBuckets]
    int64_t *bucket_base;    // [kBuckets + 1]
    int64_t *group_counts;   // [3] output
    float *out;
    int ntiles;
};

template <bool RECON>
__global__ void __launch_bounds__(kThreads) classify_kernel(const PreParams p) {
    __shared__ int counts[kBuckets];
    if (threadIdx.x < kBuckets) counts[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
    int local[kBuckets] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
        if (i < p.n) {
            const Rec r = process<RECON>(p.events + i * p.stride, p.cut, p.limit);
            p.bucket[i] = (unsigned char)r.bucket;
#pragma unroll
            for (int b = 0; b < kBuckets; b++) local[b] += (r.bucket == b);
        }
    }
#pragma unroll
    for (int b = 0; b < kBuckets; b++) {
        int v = local[b];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&counts[b], v);
    }
    __syncthreads();
    if (threadIdx.x < kBuckets) p.tile_counts[blockIdx.x * kBuckets + threadIdx.x] = counts[threadIdx.x];
}

// One block: exclusive scan of the tile counts of each bucket, then of the bucket
// totals; bucket_base[b] is where bucket b starts in the output.
__global__ void __launch_bounds__(1024) scan_kernel(const PreParams p) {
    __shared__ int64_t totals[kBuckets];
    __shared__ int64_t warp_sums[32];
    for (int b = 0; b < kBuckets; b++) {
        int64_t carry = 0;
        for (int start = 0; start < p.ntiles; start += blockDim.x) {
            const int i = start + threadIdx.x;
            int64_t v = i < p.ntiles ? p.tile_counts[i * kBuckets + b] : 0;
            // inclusive scan inside the warp
            int64_t x = v;
            for (int o = 1; o < 32; o <<= 1) {
                int64_t y = __shfl_up_sync(0xffffffffu, x, o);
                if ((threadIdx.x & 31) >= o) x += y;
            }
            if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
            __syncthreads();
            if (threadIdx.x < 32) {
                int64_t w = threadIdx.x < (blockDim.x >> 5) ? warp_sums[threadIdx.x] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                    if (threadIdx.x >= o) w += y;
                }
                warp_sums[threadIdx.x] = w;
            }
            __syncthreads();
            const int wid = threadIdx.x >> 5;
            const int64_t before = (wid ? warp_sums[wid - 1] : 0) + carry;
            if (i < p.ntiles) p.tile_offsets[i * kBuckets + b] = before + x - v;
            const int64_t chunk = warp_sums[(blockDim.x >> 5) - 1];
            __syncthreads();
            carry += chunk;
        }
        if (threadIdx.x == 0) totals[b] = carry;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (int b = 0; b < kBuckets; b++) {
            p.bucket_base[b] = acc;
            acc += totals[b];
        }
        p.bucket_base[kBuckets] = acc;
        for (int a = 0; a < 3; a++) p.group_counts[a] = totals[2 * a] + totals[2 * a + 1];
    }
}

// Per step of kThreads events: each event's rank inside its bucket (warp ballots in index
// order), its record written to a shared staging buffer compacted by bucket, then each
// bucket's run copied to its place in the output as one contiguous stretch (a record
// is 28-40 bytes, so one thread per record would touch a new sector per lane and column).
template <bool RECON>
__global__ void __launch_bounds__(kThreads) scatter_kernel(const PreParams p) {
    constexpr int ncols = RECON ? 10 : 7;
    __shared__ int warp_counts[kThreads / 32][kBuckets];
    __shared__ int64_t running[kBuckets];
    __shared__ int step_start[kBuckets + 1];  // bucket runs in the staging buffer
    __shared__ float stage[kThreads * ncols];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x < kBuckets)
        running[threadIdx.x] =
            p.bucket_base[threadIdx.x] + p.tile_offsets[blockIdx.x * kBuckets + threadIdx.x];
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
    for (int k = 0; k < kItems; k++) {
        const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
        const int b = i < p.n ? (int)p.bucket[i] : kBuckets;
        // rank among equal buckets inside the warp, in index order
        int my_rank = 0;
#pragma unroll
        for (int q = 0; q < kBuckets; q++) {
            const unsigned m = __ballot_sync(0xffffffffu, b == q);
            if (b == q) my_rank = __popc(m & ((1u << lane) - 1u));
            if (lane == 0) warp_counts[wid][q] = __popc(m);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int q = 0; q < kBuckets; q++) {
                step_start[q] = acc;
                for (int w = 0; w < kThreads / 32; w++) acc += warp_counts[w][q];
            }
            step_start[kBuckets] = acc;
        }
        __syncthreads();
        if (b < kBuckets) {
            int pos = step_start[b] + my_rank;
            for (int w = 0; w < wid; w++) pos += warp_counts[w][b];
            const Rec r = process<RECON>(p.events + i * p.stride, p.cut, p.limit);
#pragma unroll
            for (int c = 0; c < ncols; c++) stage[pos * ncols + c] = r.v[c];
        }
        __syncthreads();
        const int total = step_start[kBuckets] * ncols;
        for (int e = threadIdx.x; e < total; e += kThreads) {
            const int rec = e / ncols;
            int q = 0;
            while (rec >= step_start[q + 1]) q++;
            p.out[(running[q] + (rec - step_start[q])) * ncols + (e - rec * ncols)] = stage[e];
        }
        __syncthreads();
        if (threadIdx.x < kBuckets)
            running[threadIdx.x] += step_start[threadIdx.x + 1] - step_start[threadIdx.x];
        __syncthreads();
    }
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int64_t srf_preprocess_workspace_size(int64_t num_events) {
    if (num_events < 0) return -1;
    const int64_t ntiles = (num_events + kTile - 1) / kTile;
    return (int64_t)(align256((size_t)num_events) + align256(sizeof(int) * ntiles * kBuckets) +
                     align256(sizeof(int64_t) * ntiles * kBuckets) +
                     align256(sizeof(int64_t) * (kBuckets + 1)));
}

namespace {
int preprocess(const float *events, int64_t n, int64_t stride, int recon, double tof_res,
               float *out, int64_t *group_counts, void *workspace, int64_t workspace_bytes,
               cudaStream_t stream) {
    if (n < 0 || !group_counts) return SRF_ERR_INVALID_ARGUMENT;
    if (stride < (recon ? 7 : 6)) return SRF_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!events || !out || !workspace)) return SRF_ERR_INVALID_ARGUMENT;
    if (workspace_bytes < srf_preprocess_workspace_size(n)) return SRF_ERR_INVALID_ARGUMENT;
    if (!(tof_res == tof_res)) return SRF_ERR_INVALID_ARGUMENT;
    PreParams p{};
    p.events = events;
    p.n = n;
    p.stride = stride;
    p.recon = recon;
    p.cut = recon && tof_res < 10000.0;
    p.limit = (float)(tof_res * 0.15 / 2.35482005 * 3);
    p.ntiles = (int)((n + kTile - 1) / kTile);
    char *w = static_cast<char *>(workspace);
    p.bucket = reinterpret_cast<unsigned char *>(w);
    w += align256((size_t)n);
    p.tile_counts = reinterpret_cast<int *>(w);
    w += align256(sizeof(int) * p.ntiles * kBuckets);
    p.tile_offsets = reinterpret_cast<int64_t *>(w);
    w += align256(sizeof(int64_t) * p.ntiles * kBuckets);
    p.bucket_base = reinterpret_cast<int64_t *>(w);
    p.group_counts = group_counts;
    p.out = out;
    if (n == 0) {
        cudaError_t e = cudaMemsetAsync(group_counts, 0, 3 * sizeof(int64_t), stream);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return SRF_ERR_CUDA;
        }
        return SRF_OK;
    }
    if (recon) {
        classify_kernel<true><<<p.ntiles, kThreads, 0, stream>>>(p);
        scan_kernel<<<1, 1024, 0, stream>>>(p);
        scatter_kernel<true><<<p.ntiles, kThreads, 0, stream>>>(p);
        count_launches(3);
    } else {
        classify_kernel<false><<<p.ntiles, kThreads, 0, stream>>>(p);
        scan_kernel<<<1, 1024, 0, stream>>>(p);
        scatter_kernel<false><<<p.ntiles, kThreads, 0, stream>>>(p);
        count_launches(3);
    }
    return check_launch();
}
}  // namespace

extern "C" int srf_recon_process(const float *events, int64_t num_events, int64_t event_stride,
                                 double tof_res, float *out, int64_t *group_counts,
                                 void *workspace, int64_t workspace_bytes, void *stream) {
    return preprocess(events, num_events, event_stride, 1, tof_res, out, group_counts, workspace,
                      workspace_bytes, (cudaStream_t)stream);
}

extern "C" int srf_map_process(const float *lors, int64_t num_lors, int64_t lor_stride,
                               float *out, int64_t *group_counts, void *workspace,
                               int64_t workspace_bytes, void *stream) {
    return preprocess(lors, num_lors, lor_stride, 0, 1.0e4, out, group_counts, workspace,
                      workspace_bytes, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------------
// recon_process without any allocation.
//
// Some callers cannot allocate device memory at the time they preprocess events: an
// acquisition-side reconstruction service that owns a fixed memory budget and forbids
// allocations after start-up, or code on a latency-critical path where cudaMalloc's
// implicit device synchronisation is not acceptable. srf_recon_process needs a scratch
// workspace for its stable partition; this variant takes that scratch from a buffer
// that is part of the library itself, a file-scope __device__ array of fixed size.
//
// * The buffer holds the workspace for up to SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS events
//   (8.1 MiB); every GPU that loads the library keeps it until the process exits.
//   Larger calls are rejected with SRF_ERR_UNSUPPORTED before anything is launched.
// * Host code cannot use the array's name as a device address, so the first call on
//   each device (with that device current) asks the runtime for the address with
//   cudaGetSymbolAddress and caches it; that first call should therefore happen before
//   any stream capture. The cache lives as long as the process: after cudaDeviceReset
//   the address is stale, and the library must not be called on that device again.
// * All calls on a device share the one buffer and it keeps the last call's contents.
//   Nothing in it needs to start at zero: every byte a call reads was written earlier
//   in the same call. Calls whose kernels overlap on the GPU (concurrent streams, or
//   several host threads) race on the buffer; serialise them on one stream.
// * No cudaMalloc, cudaFree or allocating library routine is called.

namespace srf {
namespace {

constexpr int64_t kNoAllocMaxEvents = SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS;
constexpr size_t align256c(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr int64_t kNoAllocTiles = (kNoAllocMaxEvents + kTile - 1) / kTile;
constexpr size_t kNoAllocScratchBytes =
    align256c((size_t)kNoAllocMaxEvents) + align256c(sizeof(int) * kNoAllocTiles * kBuckets) +
    align256c(sizeof(int64_t) * kNoAllocTiles * kBuckets) +
    align256c(sizeof(int64_t) * (kBuckets + 1));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once).
int noalloc_scratch(void **ptr) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) return SRF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess && !p) e = cudaErrorInvalidSymbol;  // never a null address
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return SRF_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *ptr = g_noalloc_ptr[dev];
    return SRF_OK;
}

}  // namespace
}  // namespace srf

extern "C" int srf_recon_process_noalloc(const float *events, int64_t num_events,
                                         int64_t event_stride, double tof_res, float *out,
                                         int64_t *group_counts, void *stream) {
    if (num_events < 0) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > kNoAllocMaxEvents) return SRF_ERR_UNSUPPORTED;
    void *scratch = nullptr;
    const int st = noalloc_scratch(&scratch);
    if (st != SRF_OK) return st;
    return preprocess(events, num_events, event_stride, 1, tof_res, out, group_counts, scratch,
                      (int64_t)kNoAllocScratchBytes, (cudaStream_t)stream);
}

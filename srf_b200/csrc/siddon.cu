// Siddon ray-tracing listmode projector for sm_100a.
//
// Operator (reference: src/cpp/tf_custom_ops/siddon.cu.cc): clip the LOR to the image
// box (:118-183), walk the voxels it crosses in order of the next boundary along each
// axis (:196-331), and weight each voxel by w * l with w = 1/L^2 (:459) and l the
// chord length inside it; with TOF on, by the Gaussian of the chord midpoint's offset
// from the TOF position with variance tof_sigma2 + (l^2 + tof_bin^2)/12, cut at 3 sigma
// (:308-317).
//
// One thread per ray, one launch per call (the reference uses a fixed 32x1024 grid
// and copies the geometry device-to-host first). The walk state (next boundary,
// step, voxel counters) is evaluated with the same float operations as the reference,
// so each ray visits the same voxels with the same chord lengths; the TOF weight of a
// voxel uses float arithmetic for the Gaussian itself.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>

#include "srf_common.cuh"

namespace srf {
namespace {

enum SiddonOp { kProj = 0, kBack = 1, kMap = 2, kAdj = 3, kCount = 4 };

struct SiddonParams {
    const float *x1, *y1, *z1, *x2, *y2, *z2, *tof;
    int64_t stride, n;
    int g[3];
    float top[3], bot[3];  // center +/- size/2 (siddon.cu.cc:174)
    float corner[3];       // center - size/2 (siddon.cu.cc:267)
    float v_res[3];        // size/grid (siddon.cu.cc:211)
    int tof_on;
    float tof_sigma2, tof_bin, bin2;
    const float *image_in;
    const float *values;
    float *image_out;
    float *proj_out;
    int *count_out;  // kCount: voxels the walk visits per ray
};

// ClipRay (siddon.cu.cc:118-153) for one axis.
__device__ __forceinline__ bool clip(float top, float bot, float p0, float dp, float &tmin,
                                     float &tmax) {
    float t;
    if (dp > 0.0f) {
        t = __fdiv_rn(__fsub_rn(top, p0), dp);
        if (t < tmax) tmax = t;
        t = __fdiv_rn(__fsub_rn(bot, p0), dp);
        if (t > tmin) tmin = t;
    } else if (dp < 0.0f) {
        t = __fdiv_rn(__fsub_rn(bot, p0), dp);
        if (t < tmax) tmax = t;
        t = __fdiv_rn(__fsub_rn(top, p0), dp);
        if (t > tmin) tmin = t;
    } else {
        if ((p0 < bot) || (p0 > top)) return false;
    }
    return tmin < tmax;
}

// SetupRayCastComponent (siddon.cu.cc:196-250) for one axis; `p0` is already shifted
// to the box corner.
__device__ __forceinline__ void setup_axis(float p0, float dir, float min_t, float v_res,
                                           int count, int &pos, float &next_t, float &delta_t,
                                           int &step, int &in_buf) {
    const float pt = __fmaf_rn(min_t, dir, p0);
    if (dir > 0.0f) {
        pos = __float2int_rz(__fdiv_rn(pt, v_res));
        next_t = __fdiv_rn(__fmaf_rn((float)(pos + 1), v_res, -pt), dir);
        delta_t = __fdiv_rn(v_res, dir);
        step = 1;
        in_buf = count - pos;
    } else if (dir < 0.0f) {
        pos = count - 1 - __float2int_rz(__fsub_rn((float)count, __fdiv_rn(pt, v_res)));
        next_t = __fdiv_rn(__fmaf_rn((float)pos, v_res, -pt), dir);
        delta_t = __fdiv_rn(-v_res, dir);
        step = -1;
        in_buf = pos + 1;
    } else {
        pos = __float2int_rz(__fdiv_rn(pt, v_res));
        next_t = FLT_MAX;
        delta_t = FLT_MAX;
        step = 0;
        in_buf = 1;
    }
}

// One ray's walk state after SetupRayCast (siddon.cu.cc:261-284) and its weights.
struct Ray {
    int pos[3], step[3], in_buf[3];
    float next_t[3], delta_t[3];
    int boffs, stillin;
    int zdir;             // +1 / -1 / 0: direction of the walk along z
    float weight, t_tof;  // 1/L^2 (siddon.cu.cc:459), TOF position (:460)
    float tmin, tmax, z0, dirz;
    float oscale;         // back-projection / map: 1/value; adjoint: value
};

// CreateRay, IsThroughImage and SetupRayCast of ray t. Returns false when the ray
// contributes nothing (misses the box, value at/below 0 for back-projection and map,
// start voxel off the grid).
template <int OP>
__device__ __forceinline__ bool ray_setup(const SiddonParams &p, int64_t t, Ray &R) {
    const int64_t o = t * p.stride;
    const float x1 = __ldg(p.x1 + o), y1 = __ldg(p.y1 + o), z1 = __ldg(p.z1 + o);
    const float x2 = __ldg(p.x2 + o), y2 = __ldg(p.y2 + o), z2 = __ldg(p.z2 + o);

    float vscale = 1.0f;
    if (OP == kBack || OP == kMap) {
        const float v = __ldg(p.values + t);
        if (!(v > 0.0f)) return false;  // siddon.cu.cc:363,370,412
        vscale = v;
    } else if (OP == kAdj) {
        vscale = __ldg(p.values + t);
    }

    // CreateRay (siddon.cu.cc:61-81).
    const float dx = __fsub_rn(x2, x1), dy = __fsub_rn(y2, y1), dz = __fsub_rn(z2, z1);
    const float length = __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy))));
    const float dir[3] = {__fdiv_rn(dx, length), __fdiv_rn(dy, length), __fdiv_rn(dz, length)};
    const float start[3] = {x1, y1, z1};

    // IsThroughImage (siddon.cu.cc:163-183).
    float tmin = 0.0f, tmax = length;
    bool through = true;
#pragma unroll
    for (int k = 0; k < 3; k++)
        through = through && clip(p.top[k], p.bot[k], start[k], dir[k], tmin, tmax);
    if (!(through && tmin < tmax)) return false;

    // SetupRayCast (siddon.cu.cc:261-284).
#pragma unroll
    for (int k = 0; k < 3; k++)
        setup_axis(__fsub_rn(start[k], p.corner[k]), dir[k], tmin, p.v_res[k], p.g[k], R.pos[k],
                   R.next_t[k], R.delta_t[k], R.step[k], R.in_buf[k]);
    R.zdir = R.step[2];
    R.step[1] *= p.g[0];
    R.step[2] *= p.g[0] * p.g[1];
    R.boffs = R.pos[0] + p.g[0] * (R.pos[1] + p.g[1] * R.pos[2]);
    R.stillin = R.in_buf[0] * R.in_buf[1] * R.in_buf[2];
    // A start voxel off the grid would make the reference read outside the image; such
    // a ray contributes nothing here.
    if (!(R.pos[0] >= 0 && R.pos[0] < p.g[0] && R.pos[1] >= 0 && R.pos[1] < p.g[1] &&
          R.pos[2] >= 0 && R.pos[2] < p.g[2]))
        return false;

    // weight (siddon.cu.cc:459, :514 and :557) and TOF position (:460).
    R.weight = (OP == kMap) ? __fdiv_rn(1.0f, __fmul_rn(length, length))
                            : __fdiv_rn(__fdiv_rn(1.0f, length), length);
    R.t_tof = 0.0f;
    if ((OP != kMap && OP != kCount) && p.tof_on)
        R.t_tof = __double2float_rn((double)length * 0.5 - (double)tmin -
                                    (double)__ldg(p.tof + o));
    R.oscale = (OP == kBack || OP == kMap) ? __fdiv_rn(1.0f, vscale) : vscale;
    R.tmin = tmin;
    R.tmax = tmax;
    R.z0 = __fsub_rn(z1, p.corner[2]);
    R.dirz = dir[2];
    return R.stillin != 0;
}

// RayTracing / BackRayTracing / Map (siddon.cu.cc:293-415): visits the ray's voxels in
// order; f(mi, iz, val, use) gets the voxel index, its z index, the weight * chord length
// [* TOF] and the reference's TOF cut decision, and returns false to end the walk early.
// Returns the number of voxels visited.
template <int OP, typename F>
__device__ __forceinline__ int ray_walk(const SiddonParams &p, Ray &R, F &&f) {
    const float sqrt2pi = 2.5066282746310002f;
    const bool tof = (OP != kMap && OP != kCount) && p.tof_on;
    float last_t = 0.0f;
    int iz = R.pos[2];
    int n_visits = 0;
    int stillin = R.stillin;
    while (stillin) {
        // argmin with the reference's tie order (siddon.cu.cc:305)
        const int i = (R.next_t[0] <= R.next_t[1]) ? ((R.next_t[0] <= R.next_t[2]) ? 0 : 2)
                                                   : ((R.next_t[1] <= R.next_t[2]) ? 1 : 2);
        const float nt = i == 0 ? R.next_t[0] : (i == 1 ? R.next_t[1] : R.next_t[2]);
        const float l_len = __fsub_rn(nt, last_t);
        float val;  // weight * l_len * [TOF] for this voxel
        bool use = true;
        if (tof) {
            const float tt = __fmaf_rn(-0.5f, __fadd_rn(nt, last_t), R.t_tof);
            const float s2 =
                __double2float_rn((double)p.tof_sigma2 + (double)__fmaf_rn(l_len, l_len, p.bin2) / 12.0);
            const float r = __fdiv_rn(__fmul_rn(tt, tt), s2);
            use = r < 9.0f;
            val = __fmul_rn(__fmul_rn(R.weight, l_len), p.tof_bin) *
                  (__expf(-0.5f * r) * rsqrtf(s2) * (1.0f / sqrt2pi));
        } else {
            val = __fmul_rn(R.weight, l_len);
        }
        n_visits++;
        if (!f(R.boffs, iz, val, use)) break;
        last_t = nt;
        if (i == 0) {
            R.next_t[0] = __fadd_rn(R.next_t[0], R.delta_t[0]);
            R.boffs += R.step[0];
            stillin = --R.in_buf[0];
        } else if (i == 1) {
            R.next_t[1] = __fadd_rn(R.next_t[1], R.delta_t[1]);
            R.boffs += R.step[1];
            stillin = --R.in_buf[1];
        } else {
            R.next_t[2] = __fadd_rn(R.next_t[2], R.delta_t[2]);
            R.boffs += R.step[2];
            iz += R.zdir;
            stillin = --R.in_buf[2];
        }
    }
    return n_visits;
}

// One thread per ray over the whole image: projection gathers from the image (L2), the
// scatter ops add with global atomics; kCount counts the visits.
template <int OP>
__global__ void __launch_bounds__(256) siddon_kernel(const SiddonParams p) {
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = tid0; t < p.n; t += nthreads) {
        Ray R;
        float acc = 0.0f;
        int n_visits = 0;
        if (ray_setup<OP>(p, t, R)) {
            n_visits = ray_walk<OP>(p, R, [&](int mi, int, float val, bool use) {
                if (OP == kCount || !use) return true;
                if (OP == kProj)
                    acc = fmaf(__ldg(p.image_in + mi), val, acc);
                else
                    atomicAdd(p.image_out + mi, val * R.oscale);
                return true;
            });
        }
        if (OP == kProj) p.proj_out[t] = acc;
        if (OP == kCount) p.count_out[t] = n_visits;
    }
}

// ---------------------------------------------------------------------------------
// Slab path (projection, back-projection, map, adjoint).
//
// The [gz][gy][gx] image is cut into slabs of whole z-slices that fit in shared memory.
// A binning pass gives every ray the range of slabs its walk can reach (the z indices of
// its entry voxel and of its exit point, two voxels of margin) and appends it to those
// slabs' lists. A persistent kernel then gives every CTA an equal share of the slab-major
// list: per slab it loads the slab (projection) or zeroes it (scatter ops), and each
// thread replays its ray's exact walk from the entry voxel, touching memory only for the
// voxels inside the slab and stopping where the walk leaves it (z is monotonic along a
// ray). Scatter ops add into the slab with shared-memory atomics (3-4x the rate of the
// L2 atomics the one-thread-per-ray kernel issues) and add the slab to the image once per
// CTA; the projection adds each ray's per-slab partial sum to its output.

constexpr int kSidThreads = 1024;
constexpr size_t kSidSlabBytes = 216 * 1024;
constexpr int kSidMaxSlabs = 32;
std::atomic<int> g_sid_path{0};  // 0 automatic, 1 slab path, 2 one thread per ray

struct SidPlan {
    int nz_s, n_slabs;
    int *count;  // [n_slabs] rays per slab list
    int *list;   // [n_slabs][n] ray indices
};

// Slices per slab (balanced over the slabs) and the slab count; false when the slab path
// does not apply (a slice does not fit, or too many slabs).
bool sid_geometry(const SiddonParams &p, SidPlan &sp) {
    const size_t slice = sizeof(float) * (size_t)p.g[0] * p.g[1];
    const int max_nz = (int)std::min<size_t>((size_t)p.g[2], kSidSlabBytes / slice);
    if (max_nz < 1) return false;
    sp.n_slabs = (p.g[2] + max_nz - 1) / max_nz;
    if (sp.n_slabs > kSidMaxSlabs) return false;
    sp.nz_s = (p.g[2] + sp.n_slabs - 1) / sp.n_slabs;
    sp.n_slabs = (p.g[2] + sp.nz_s - 1) / sp.nz_s;
    return p.n < (int64_t)INT32_MAX;
}

template <int OP>
__global__ void __launch_bounds__(256) sid_bin_kernel(const SiddonParams p, SidPlan sp) {
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    // whole warps iterate together (the list appends are warp-aggregated)
    for (int64_t base = tid0 - lane; base < p.n; base += nthreads) {
        const int64_t t = base + lane;
        int k_lo = 0, k_hi = -1;
        Ray R;
        if (t < p.n && ray_setup<OP>(p, t, R)) {
            // The walk runs to the grid's edge, not to the ray's end point (it stops only
            // when a voxel counter runs out, siddon.cu.cc:302), so its last z is where
            // the first axis leaves the grid: t_end (from the entry point) = min over the
            // moving axes of next_t + (in_buf - 1) delta_t; z in the box-corner frame.
            float t_end = INFINITY;
#pragma unroll
            for (int a = 0; a < 3; a++)
                if (R.step[a] != 0)
                    t_end = fminf(t_end, fmaf((float)(R.in_buf[a] - 1), R.delta_t[a], R.next_t[a]));
            const float zt = fmaf(R.tmin + t_end, R.dirz, R.z0);
            const float fz = fminf(fmaxf(floorf(zt / p.v_res[2]), -4.0f), (float)p.g[2] + 4.0f);
            const int izt = (int)fz;
            const int lo = max(0, min(R.pos[2], izt) - 2);
            const int hi = min(p.g[2] - 1, max(R.pos[2], izt) + 2);
            k_lo = lo / sp.nz_s;
            k_hi = hi / sp.nz_s;
        }
        for (int k = 0; k < sp.n_slabs; k++) {
            const bool in = k >= k_lo && k <= k_hi;
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (!m) continue;
            int first = 0;
            if (lane == __ffs(m) - 1) first = atomicAdd(sp.count + k, __popc(m));
            first = __shfl_sync(0xffffffffu, first, __ffs(m) - 1);
            if (in) sp.list[(int64_t)k * p.n + first + __popc(m & ((1u << lane) - 1u))] = (int)t;
        }
    }
}

template <int OP>
__global__ void __launch_bounds__(kSidThreads, 1) siddon_slab_kernel(const SiddonParams p,
                                                                    SidPlan sp) {
    extern __shared__ float slab[];
    __shared__ int64_t offs[kSidMaxSlabs + 1];
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (int k = 0; k < sp.n_slabs; k++) {
            offs[k] = acc;
            acc += sp.count[k];
        }
        offs[sp.n_slabs] = acc;
    }
    __syncthreads();
    const int64_t total = offs[sp.n_slabs];
    const int64_t g = blockIdx.x, G = gridDim.x;
    const int64_t lo = total * g / G, hi = total * (g + 1) / G;
    const int slice = p.g[0] * p.g[1];
    int k = 0;
    for (int64_t pos = lo; pos < hi;) {
        while (offs[k + 1] <= pos) k++;
        const int64_t end = min(hi, offs[k + 1]);
        const int Z0 = k * sp.nz_s, Z1 = min(Z0 + sp.nz_s, p.g[2]);
        const int nvox = (Z1 - Z0) * slice;
        const int64_t base = (int64_t)Z0 * slice;
        if (OP == kProj) {
            for (int i = threadIdx.x; i < nvox; i += kSidThreads) slab[i] = __ldg(p.image_in + base + i);
        } else {
            for (int i = threadIdx.x; i < nvox; i += kSidThreads) slab[i] = 0.0f;
        }
        __syncthreads();
        for (int64_t q = pos + threadIdx.x; q < end; q += kSidThreads) {
            const int t = sp.list[(int64_t)k * p.n + (q - offs[k])];
            Ray R;
            if (!ray_setup<OP>(p, t, R)) continue;
            float acc = 0.0f;
            ray_walk<OP>(p, R, [&](int mi, int iz, float val, bool use) {
                if (iz < Z0 || iz >= Z1) {
                    // not in the slab: keep walking only towards it (z is monotonic)
                    return (R.zdir > 0 && iz < Z0) || (R.zdir < 0 && iz >= Z1);
                }
                // a visited voxel is in the grid, so iz in [Z0, Z1) puts mi - base in
                // [0, (Z1 - Z0) gx gy)
                if (!use) return true;
                if (OP == kProj)
                    acc = fmaf(slab[mi - base], val, acc);
                else
                    atomicAdd(&slab[mi - base], val * R.oscale);
                return true;
            });
            if (OP == kProj && acc != 0.0f) atomicAdd(p.proj_out + t, acc);
        }
        __syncthreads();
        if (OP != kProj) {
            for (int i = threadIdx.x; i < nvox; i += kSidThreads) {
                const float v = slab[i];
                if (v != 0.0f) atomicAdd(p.image_out + base + i, v);
            }
            __syncthreads();
        }
        pos = end;
    }
}

int siddon_setup(SiddonParams &p, const int *grid, const float *center, const float *size,
                 float tof_bin, float tof_sigma2, int64_t n, int64_t lor_stride) {
    if (!grid || !center || !size) return SRF_ERR_INVALID_ARGUMENT;
    if (n < 0 || lor_stride < 1) return SRF_ERR_INVALID_ARGUMENT;
    if (grid[0] <= 0 || grid[1] <= 0 || grid[2] <= 0) return SRF_ERR_INVALID_ARGUMENT;
    if (!finite3(center) || !finite3(size)) return SRF_ERR_INVALID_ARGUMENT;
    if (size[0] <= 0.f || size[1] <= 0.f || size[2] <= 0.f) return SRF_ERR_INVALID_ARGUMENT;
    if (!(tof_sigma2 == tof_sigma2) || !(tof_bin == tof_bin)) return SRF_ERR_INVALID_ARGUMENT;
    if ((int64_t)grid[0] * grid[1] * grid[2] > ((int64_t)1 << 31) - 1)
        return SRF_ERR_UNSUPPORTED;
    for (int k = 0; k < 3; k++) {
        p.g[k] = grid[k];
        p.top[k] = center[k] + size[k] / 2;
        p.bot[k] = center[k] - size[k] / 2;
        p.corner[k] = center[k] - size[k] / 2;
        p.v_res[k] = size[k] / grid[k];
    }
    p.tof_on = tof_sigma2 < kTofThreshold ? 1 : 0;
    p.tof_sigma2 = tof_sigma2;
    p.tof_bin = tof_bin;
    p.bin2 = tof_bin * tof_bin;
    p.n = n;
    p.stride = lor_stride;
    return SRF_OK;
}

// The slab path for p's op: bins the rays, then one persistent launch. Returns -1 when
// it does not apply.
template <int OP>
int siddon_launch_slab(const SiddonParams &p, cudaStream_t stream) {
    SidPlan sp{};
    if (!sid_geometry(p, sp)) return -1;
    const size_t b_count = 256;
    const size_t b_list = sizeof(int) * (size_t)sp.n_slabs * (size_t)p.n;
    char *ws = nullptr;
    cudaError_t e = scratch_alloc((void **)&ws, b_count + b_list, stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    sp.count = reinterpret_cast<int *>(ws);
    sp.list = reinterpret_cast<int *>(ws + b_count);
    static std::atomic<unsigned long long> attr_set{0};  // per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    e = cudaSuccess;
    if (!(attr_set.load() & (1ull << dev))) {
        e = cudaFuncSetAttribute(siddon_slab_kernel<OP>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSidSlabBytes);
        if (e == cudaSuccess) attr_set.fetch_or(1ull << dev);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(sp.count, 0, b_count, stream);
    if (e == cudaSuccess && OP == kProj)
        e = cudaMemsetAsync(p.proj_out, 0, sizeof(float) * (size_t)p.n, stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        cudaFreeAsync(ws, stream);
        return SRF_ERR_CUDA;
    }
    sid_bin_kernel<OP><<<stride_grid(p.n, 256, 8), 256, 0, stream>>>(p, sp);
    const size_t smem = sizeof(float) * (size_t)sp.nz_s * p.g[0] * p.g[1];
    siddon_slab_kernel<OP><<<num_sms(), kSidThreads, smem, stream>>>(p, sp);
    count_launches(2);
    int st = check_launch();
    e = cudaFreeAsync(ws, stream);
    if (st == SRF_OK && e != cudaSuccess) {
        set_cuda_error(e);
        st = SRF_ERR_CUDA;
    }
    return st;
}

template <int OP>
int siddon_launch(const SiddonParams &p, cudaStream_t stream) {
    if (p.n == 0) return SRF_OK;
    if (OP != kCount && g_sid_path.load(std::memory_order_relaxed) != 2) {
        const int st = siddon_launch_slab<OP>(p, stream);
        if (st >= 0) return st;
    }
    const int block = 256;
    const int grid = stride_grid(p.n, block, 8);
    siddon_kernel<OP><<<grid, block, 0, stream>>>(p);
    count_launches(1);
    return check_launch();
}

int zero_out(float *image, const int *grid, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(
        image, 0, sizeof(float) * (size_t)grid[0] * grid[1] * grid[2], stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    return SRF_OK;
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int srf_siddon_projection(const float *x1, const float *y1, const float *z1,
                                     const float *x2, const float *y2, const float *z2,
                                     const float *tof_t, float *projection_value,
                                     const int *grid, const float *center, const float *size,
                                     float tof_bin, float tof_sigma2, const float *image,
                                     int64_t num_events, int64_t lor_stride, void *stream) {
    SiddonParams p{};
    int st = siddon_setup(p, grid, center, size, tof_bin, tof_sigma2, num_events, lor_stride);
    if (st != SRF_OK) return st;
    if (num_events > 0 && (!x1 || !y1 || !z1 || !x2 || !y2 || !z2 || !projection_value ||
                           !image || (p.tof_on && !tof_t)))
        return SRF_ERR_INVALID_ARGUMENT;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2; p.tof = tof_t;
    p.image_in = image;
    p.proj_out = projection_value;
    return siddon_launch<kProj>(p, (cudaStream_t)stream);
}

extern "C" int srf_siddon_backprojection(const float *x1, const float *y1, const float *z1,
                                         const float *x2, const float *y2, const float *z2,
                                         const float *tof_t, const float *projection_value,
                                         const int *grid, const float *center,
                                         const float *size, float tof_bin, float tof_sigma2,
                                         float *image, int64_t num_events, int64_t lor_stride,
                                         int accumulate, void *stream) {
    SiddonParams p{};
    int st = siddon_setup(p, grid, center, size, tof_bin, tof_sigma2, num_events, lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && (!x1 || !y1 || !z1 || !x2 || !y2 || !z2 || !projection_value ||
                           (p.tof_on && !tof_t)))
        return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_out(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2; p.tof = tof_t;
    p.values = projection_value;
    p.image_out = image;
    return siddon_launch<kBack>(p, (cudaStream_t)stream);
}

extern "C" int srf_siddon_maplors(const float *x1, const float *y1, const float *z1,
                                  const float *x2, const float *y2, const float *z2,
                                  const float *projection_value, const int *grid,
                                  const float *center, const float *size, float *image,
                                  int64_t num_events, int64_t lor_stride, int accumulate,
                                  void *stream) {
    SiddonParams p{};
    int st = siddon_setup(p, grid, center, size, 0.0f, 1.0e30f, num_events, lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && (!x1 || !y1 || !z1 || !x2 || !y2 || !z2 || !projection_value))
        return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_out(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.values = projection_value;
    p.image_out = image;
    return siddon_launch<kMap>(p, (cudaStream_t)stream);
}

extern "C" int srf_siddon_backproject_adjoint(const float *x1, const float *y1,
                                              const float *z1, const float *x2,
                                              const float *y2, const float *z2,
                                              const float *tof_t, const float *values,
                                              const int *grid, const float *center,
                                              const float *size, float tof_bin,
                                              float tof_sigma2, float *image,
                                              int64_t num_events, int64_t lor_stride,
                                              int accumulate, void *stream) {
    SiddonParams p{};
    int st = siddon_setup(p, grid, center, size, tof_bin, tof_sigma2, num_events, lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 &&
        (!x1 || !y1 || !z1 || !x2 || !y2 || !z2 || !values || (p.tof_on && !tof_t)))
        return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_out(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2; p.tof = tof_t;
    p.values = values;
    p.image_out = image;
    return siddon_launch<kAdj>(p, (cudaStream_t)stream);
}

extern "C" int srf_siddon_count_samples(const float *x1, const float *y1, const float *z1,
                                        const float *x2, const float *y2, const float *z2,
                                        const int *grid, const float *center, const float *size,
                                        int *counts, int64_t num_events, int64_t lor_stride,
                                        void *stream) {
    SiddonParams p{};
    int st = siddon_setup(p, grid, center, size, 1.0f, 1.0e6f, num_events, lor_stride);
    if (st != SRF_OK) return st;
    if (num_events > 0 && (!x1 || !y1 || !z1 || !x2 || !y2 || !z2 || !counts))
        return SRF_ERR_INVALID_ARGUMENT;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.count_out = counts;
    return siddon_launch<kCount>(p, (cudaStream_t)stream);
}

// No counterpart in the reference: the Siddon kernel family (0 automatic: the
// shared-memory slab path where a z-slice fits and the image has at most 32 slabs,
// 1 the same, 2 one thread per ray with L2 gathers and atomics).
extern "C" int srf_siddon_set_tuning(int path) {
    if (path < 0 || path > 2) return SRF_ERR_INVALID_ARGUMENT;
    g_sid_path.store(path);
    return SRF_OK;
}

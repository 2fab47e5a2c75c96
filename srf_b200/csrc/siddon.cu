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
// voxel uses float arithmetic for the Gaussian itself. The scatter ops reduce into four
// consecutive voxels at a time where a ray's run allows (siddon_kernel).

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
    // scatter ops with quads: rays whose |dy| exceeds |dx| accumulate into this y-fastest
    // copy [gz][gx][gy] (null: every ray into image_out), added to image_out afterwards
    float *image_yx;
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
    float nt0, nt1, nt2;  // next boundary along x, y, z (from the entry point)
    float dt0, dt1, dt2;  // boundary spacing along x, y, z
    int in0, in1, in2;    // voxels left along x, y, z
    int s1, s2;           // index steps of a y and a z move (an x move steps by +-1)
    int s0;
    int boffs;            // index of the current voxel (in image_out, or in image_yx)
    int yfast;            // the ray accumulates into image_yx
    float weight, t_tof;  // 1/L^2 (siddon.cu.cc:459), TOF position (:460)
    float oscale;         // back-projection / map: 1/value; adjoint: value
};

// CreateRay, IsThroughImage and SetupRayCast of ray t. Returns false when the ray
// contributes nothing (misses the box, value at/below 0 for back-projection and map,
// start voxel off the grid, a voxel counter already at 0).
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
    int pos[3], step[3], in_buf[3];
    float next_t[3], delta_t[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
        setup_axis(__fsub_rn(start[k], p.corner[k]), dir[k], tmin, p.v_res[k], p.g[k], pos[k],
                   next_t[k], delta_t[k], step[k], in_buf[k]);
    // A start voxel off the grid would make the reference read outside the image; such
    // a ray contributes nothing here.
    if (!(pos[0] >= 0 && pos[0] < p.g[0] && pos[1] >= 0 && pos[1] < p.g[1] && pos[2] >= 0 &&
          pos[2] < p.g[2]))
        return false;
    if (in_buf[0] * in_buf[1] * in_buf[2] == 0) return false;  // stillin = 0: no voxel
    R.nt0 = next_t[0]; R.nt1 = next_t[1]; R.nt2 = next_t[2];
    R.dt0 = delta_t[0]; R.dt1 = delta_t[1]; R.dt2 = delta_t[2];
    R.in0 = in_buf[0]; R.in1 = in_buf[1]; R.in2 = in_buf[2];
    // the voxel index in the layout the ray walks fastest through: x-fastest image_out,
    // or y-fastest image_yx for a ray that runs more along y than along x
    R.yfast = (p.image_yx && fabsf(dy) > fabsf(dx)) ? 1 : 0;
    const int ga = R.yfast ? p.g[1] : p.g[0], gb = R.yfast ? p.g[0] : p.g[1];
    const int pa = R.yfast ? pos[1] : pos[0], pb = R.yfast ? pos[0] : pos[1];
    R.s0 = step[0] * (R.yfast ? ga : 1);
    R.s1 = step[1] * (R.yfast ? 1 : ga);
    R.s2 = step[2] * ga * gb;
    R.boffs = pa + ga * (pb + gb * pos[2]);

    // weight (siddon.cu.cc:459, :514 and :557) and TOF position (:460).
    R.weight = (OP == kMap) ? __fdiv_rn(1.0f, __fmul_rn(length, length))
                            : __fdiv_rn(__fdiv_rn(1.0f, length), length);
    R.t_tof = 0.0f;
    if ((OP != kMap && OP != kCount) && p.tof_on)
        R.t_tof = __double2float_rn((double)length * 0.5 - (double)tmin -
                                    (double)__ldg(p.tof + o));
    R.oscale = (OP == kBack || OP == kMap) ? __fdiv_rn(1.0f, vscale) : vscale;
    return true;
}

// Adds four consecutive floats with one reduction (16-byte aligned address). Like a scalar
// float atomic add, it flushes subnormal inputs and results to zero. No memory clobber: the
// kernels that issue it never read the image they reduce into.
__device__ __forceinline__ void red_quad(float *q, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "l"(q), "f"(a), "f"(b), "f"(c), "f"(d));
}

// One thread per ray: RayTracing / BackRayTracing / Map (siddon.cu.cc:293-415) and the
// visit count. The walk takes the reference's next boundary with its tie order
// (siddon.cu.cc:305) and advances that axis with selects rather than a branch per axis,
// so the lanes of a warp (rays crossing boundaries along different axes) stay together.
//
// kQuad (scatter ops; the image 16-byte aligned, its voxel count a multiple of 4): a
// ray's consecutive voxels often share an aligned quad of four floats (runs along its
// dominant transverse axis: rays with |dy| > |dx| accumulate into a y-fastest copy of the
// image that is added to the output afterwards, 2.0 voxels per quad on average over the
// 64x64x32 workload against 1.6 with every ray in the x-fastest image), so the ray gathers its values
// for the current quad and adds them with one vector reduction when it leaves the quad
// (the L2 handles reductions at a fixed rate per request, whatever their width: measured
// 1.47e11 requests/s for 1, 2 or 4 floats). A ray visits each voxel once, so a quad's
// pending values are set, not summed, and the reduction adds the same value the scalar
// atomic would. The projection gathers one voxel at a time: its independent loads
// overlap better than a cached quad load the next voxels wait on (measured: 0.24 against
// 0.31 ms for 1M rays at 64x64x32; back-projection 0.40 against 0.61 ms with quads).
template <int OP, bool kQuad>
__global__ void __launch_bounds__(256) siddon_kernel(const SiddonParams p) {
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    const float sqrt2pi = 2.5066282746310002f;
    const bool tof = (OP != kMap && OP != kCount) && p.tof_on;
    for (int64_t t = tid0; t < p.n; t += nthreads) {
        Ray R;
        float acc = 0.0f;
        int n_visits = 0;
        if (ray_setup<OP>(p, t, R)) {
            float *const dst = R.yfast ? p.image_yx : p.image_out;  // kQuad scatter target
            float pend_v = 0.0f, pend_w = 0.0f;           // projection: the last gather
            int cur = -1;                                  // kQuad: current quad (index / 4)
            float4 qv = make_float4(0.f, 0.f, 0.f, 0.f);  // its values or pending adds
            float last_t = 0.0f;
            int stillin = 1;
            while (stillin) {
                // argmin with the reference's tie order (siddon.cu.cc:305)
                const bool ax = (R.nt0 <= R.nt1) && (R.nt0 <= R.nt2);
                const bool ay = !(R.nt0 <= R.nt1) && (R.nt1 <= R.nt2);
                const float nt = ax ? R.nt0 : (ay ? R.nt1 : R.nt2);
                const float l_len = __fsub_rn(nt, last_t);
                float val;  // weight * l_len * [TOF] for this voxel
                bool use = true;
                if (tof) {
                    const float tt = __fmaf_rn(-0.5f, __fadd_rn(nt, last_t), R.t_tof);
                    const float s2 = __double2float_rn(
                        (double)p.tof_sigma2 + (double)__fmaf_rn(l_len, l_len, p.bin2) / 12.0);
                    const float r = __fdiv_rn(__fmul_rn(tt, tt), s2);
                    use = r < 9.0f;
                    val = __fmul_rn(__fmul_rn(R.weight, l_len), p.tof_bin) *
                          (__expf(-0.5f * r) * rsqrtf(s2) * (1.0f / sqrt2pi));
                } else {
                    val = __fmul_rn(R.weight, l_len);
                }
                const int mi = R.boffs;
                if (OP != kCount && use) {
                    if (!kQuad) {
                        if (OP == kProj) {
                            // the gather is consumed one voxel later, so its latency
                            // overlaps the next step of the walk; same sum, same order
                            acc = fmaf(pend_v, pend_w, acc);
                            pend_v = __ldg(p.image_in + mi);
                            pend_w = val;
                        } else {
                            atomicAdd(p.image_out + mi, val * R.oscale);
                        }
                    } else {
                        const int qd = mi >> 2, r = mi & 3;
                        if (qd != cur) {
                            if (cur >= 0) red_quad(dst + 4 * (int64_t)cur, qv.x, qv.y, qv.z, qv.w);
                            qv = make_float4(0.f, 0.f, 0.f, 0.f);
                            cur = qd;
                        }
                        const float add = val * R.oscale;
                        qv.x = r == 0 ? add : qv.x;
                        qv.y = r == 1 ? add : qv.y;
                        qv.z = r == 2 ? add : qv.z;
                        qv.w = r == 3 ? add : qv.w;
                    }
                }
                n_visits++;
                last_t = nt;
                const bool az = !ax && !ay;
                R.nt0 = ax ? __fadd_rn(R.nt0, R.dt0) : R.nt0;
                R.nt1 = ay ? __fadd_rn(R.nt1, R.dt1) : R.nt1;
                R.nt2 = az ? __fadd_rn(R.nt2, R.dt2) : R.nt2;
                R.boffs += ax ? R.s0 : (ay ? R.s1 : R.s2);
                R.in0 -= ax ? 1 : 0;
                R.in1 -= ay ? 1 : 0;
                R.in2 -= az ? 1 : 0;
                stillin = ax ? R.in0 : (ay ? R.in1 : R.in2);
            }
            if (kQuad && OP != kProj && OP != kCount && cur >= 0)
                red_quad(dst + 4 * (int64_t)cur, qv.x, qv.y, qv.z, qv.w);
            if (OP == kProj) acc = fmaf(pend_v, pend_w, acc);
        }
        if (OP == kProj) p.proj_out[t] = acc;
        if (OP == kCount) p.count_out[t] = n_visits;
    }
}

// out[z][y][x] += t[z][x][y] for an [gz][gy][gx] image: 32 x 32 tiles through shared
// memory, so both the read of t and the update of out are coalesced.
__global__ void __launch_bounds__(1024) add_transposed_kernel(float *__restrict__ out,
                                                             const float *__restrict__ t,
                                                             int gx, int gy) {
    __shared__ float tile[32][33];
    const int64_t z = blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const float *tz = t + z * gx * gy;
    float *oz = out + z * gx * gy;
    {
        const int x = x0 + threadIdx.y, y = y0 + threadIdx.x;  // t[x][y], y fastest
        if (x < gx && y < gy) tile[threadIdx.y][threadIdx.x] = tz[(int64_t)x * gy + y];
    }
    __syncthreads();
    const int y = y0 + threadIdx.y, x = x0 + threadIdx.x;  // out[y][x], x fastest
    if (x < gx && y < gy) oz[(int64_t)y * gx + x] += tile[threadIdx.x][threadIdx.y];
}

// Kernel family (srf_siddon_set_tuning): 0 automatic (quads for the scatter ops where the
// image allows), 1 one load / atomic per voxel.
std::atomic<int> g_sid_path{0};

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

template <int OP>
int siddon_launch(const SiddonParams &p, cudaStream_t stream) {
    if (p.n == 0) return SRF_OK;
    const int block = 256;
    const int grid = stride_grid(p.n, block, 8);
    constexpr bool kScatter = OP == kBack || OP == kMap || OP == kAdj;
    const bool quad = kScatter && g_sid_path.load(std::memory_order_relaxed) == 0 &&
                      (reinterpret_cast<uintptr_t>(p.image_out) & 15u) == 0 &&
                      ((int64_t)p.g[0] * p.g[1] * p.g[2]) % 4 == 0;
    if (!quad) {
        siddon_kernel<OP, false><<<grid, block, 0, stream>>>(p);
        count_launches(1);
        return check_launch();
    }
    // the y-fastest accumulation image (stream-ordered scratch from the library's pool)
    const size_t n_vox = (size_t)p.g[0] * p.g[1] * p.g[2];
    SiddonParams q = p;
    cudaError_t e = scratch_alloc((void **)&q.image_yx, sizeof(float) * n_vox, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(q.image_yx, 0, sizeof(float) * n_vox, stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        if (q.image_yx) cudaFreeAsync(q.image_yx, stream);
        return SRF_ERR_CUDA;
    }
    siddon_kernel<OP, kScatter><<<grid, block, 0, stream>>>(q);
    const dim3 tg((p.g[0] + 31) / 32, (p.g[1] + 31) / 32, p.g[2]);
    add_transposed_kernel<<<tg, dim3(32, 32), 0, stream>>>(p.image_out, q.image_yx, p.g[0],
                                                            p.g[1]);
    count_launches(2);
    int st = check_launch();
    e = cudaFreeAsync(q.image_yx, stream);
    if (st == SRF_OK && e != cudaSuccess) {
        set_cuda_error(e);
        st = SRF_ERR_CUDA;
    }
    return st;
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

// No counterpart in the reference: the Siddon kernel family (0 automatic: the scatter ops
// reduce four consecutive voxels at a time where the image allows; 1 one per voxel).
extern "C" int srf_siddon_set_tuning(int path) {
    if (path < 0 || path > 1) return SRF_ERR_INVALID_ARGUMENT;
    g_sid_path.store(path);
    return SRF_OK;
}

// TOR (tube-of-response) listmode projector for sm_100a.
//
// Operator (reference: src/cpp/tf_custom_ops/tor.cu.cc): for every LOR and every image
// slice z_s strictly between the LOR's endpoints along the slice axis (:30-33), the
// LOR crosses the slice plane at X (:35-36); a patch x patch window of voxels starting
// `patch/2` voxels before the voxel holding X (:135-136) is weighted by
//   G(d^2) = exp(-d^2 / (2 tor_sigma2)) for d^2 < 9 tor_sigma2, else 0       (:61-71)
// with d the voxel centre's distance to the LOR, times, when TOF is on,
//   T = tof_bin exp(-(|C - X|^2 - d^2) / (2 (tof_sigma2 + tof_bin^2/12)))
//       / sqrt(2 pi tof_sigma2)                                               (:84-91)
// with C the LOR's TOF centre.
//
// Kernel structure (one launch per call instead of the reference's one launch per
// slice): one warp per LOR, lanes over the LOR's crossed slices. Each lane computes
// its slice's crossing point and window exactly as the reference does (the discrete
// choices), then walks the window. The two Gaussians are folded into one exponent
//   log2 w = d^2 * k1 + k0(slice),  k1 = log2(e)/2 (1/tse - 1/tsc),
//   k0 = -log2(e)/2 |C - X|^2 / tse,
// so each non-zero voxel costs one exp2; the constant tof_bin/sqrt(2 pi tof_sigma2)
// is applied once per LOR. Voxels outside the 3-sigma cut-off are skipped: their
// weight is exactly zero in the reference as well.

#include <cmath>

#include "srf_common.cuh"

namespace srf {
namespace {

enum TorOp { kProj = 0, kBack = 1, kMap = 2, kAdj = 3, kCount = 4 };

struct TorParams {
    const float *x1, *y1, *z1, *x2, *y2, *z2, *xc, *yc, *zc, *f;
    int64_t stride, n;
    int gx, gy, gz, patch, half, geo, tof_on;
    float inter_x, inter_y, inter_z, l_bound, b_bound;
    float slice0_f;   // cz - (lz - inter_z)/2 in float (projection launcher, tor.cu.cc:380)
    double slice0_d;  // cz - (lz - inter_z)/2.0 in double (back/map launchers, :423, :471)
    float tor_sigma2;
    float cut;        // float threshold equivalent to (double)d2 < 9.0*tor_sigma2
    float k1;         // exponent slope (log2 units) when geo_sigma2_flag is off
    float tse;        // tof_sigma2 + tof_bin^2/12, float as in tor.cu.cc:88
    float a_coef;     // log2(e) / (2 tse)
    float tof_scale;  // tof_bin / sqrt(2 pi tof_sigma2), or 1 without TOF
    const float *image_in;
    const float *values;
    float *image_out;
    float *proj_out;
    int *count_out;   // kCount: [n] voxels with non-zero weight, [n] window voxels visited
};

// slice_z of the reference launchers: float for projection (tor.cu.cc:380), a double
// intermediate for back-projection and map (:423, :471).
template <int OP>
__device__ __forceinline__ float slice_z(const TorParams &p, int s) {
    float step = __fmul_rn((float)s, p.inter_z);
    if (OP == kProj) return __fadd_rn(p.slice0_f, step);
    return __double2float_rn(p.slice0_d + (double)step);
}

template <int OP>
__global__ void __launch_bounds__(256) tor_kernel(const TorParams p) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t slice_mesh = (int64_t)p.gx * p.gy;

    for (int64_t t = warp; t < p.n; t += nwarps) {
        const int64_t o = t * p.stride;
        const float x1 = __ldg(p.x1 + o), y1 = __ldg(p.y1 + o), z1 = __ldg(p.z1 + o);
        const float x2 = __ldg(p.x2 + o), y2 = __ldg(p.y2 + o), z2 = __ldg(p.z2 + o);
        const float f = __ldg(p.f + o);

        // Per-LOR output scale and the early-outs of the reference's value tests.
        float scale = p.tof_scale;
        bool all_slots = false;  // map with a zero/non-finite divisor: every visited voxel gets w/v
        if (OP == kBack) {
            float v = __ldg(p.values + t);
            if (!((double)v > 1e-7)) continue;  // tor.cu.cc:203
            scale = __fdiv_rn(p.tof_scale, v);
        } else if (OP == kMap) {
            float v = __ldg(p.values + t);
            scale = __fdiv_rn(1.0f, v);  // tor.cu.cc:239 divides without a threshold
            all_slots = !(fabsf(scale) <= 3.0e38f);
        } else if (OP == kAdj) {
            scale = p.tof_scale * __ldg(p.values + t);
        }

        const float d0 = __fsub_rn(x2, x1), d1 = __fsub_rn(y2, y1), dz = __fsub_rn(z2, z1);
        const float dis = __fsqrt_rn(__fmaf_rn(dz, dz, __fmaf_rn(d0, d0, __fmul_rn(d1, d1))));
        const float ux = __fdiv_rn(d0, dis), uy = __fdiv_rn(d1, dis);

        float cut = p.cut, k1 = p.k1;
        if (p.geo) {
            const float tsc = __fmul_rn(p.tor_sigma2, f);  // tor.cu.cc:67
            cut = __double2float_ru(9.0 * (double)tsc);
            const float inv = 0.5f * kLog2e / tsc;
            k1 = (p.tof_on && OP != kMap) ? (p.a_coef - inv) : -inv;
        }

        // Candidate slices: every s whose plane lies strictly inside (z1, z2), with a
        // margin; each is then tested with the reference's own ratio.
        float acc = 0.0f;
        int n_useful = 0, n_slots = 0;
        const float zlo = fminf(z1, z2), zhi = fmaxf(z1, z2);
        if (dz != 0.0f && zlo == zlo && zhi == zhi && fabsf(zhi - zlo) <= 3.0e38f) {
            const float flo = floorf((zlo - p.slice0_f) / p.inter_z) - 2.0f;
            const float fhi = ceilf((zhi - p.slice0_f) / p.inter_z) + 2.0f;
            const int s_lo = (int)fmaxf(flo, 0.0f);
            const int s_hi = (int)fminf(fhi, (float)(p.gz - 1));
            float xc = 0.f, yc = 0.f, zc = 0.f;
            if (OP != kMap && p.tof_on) {
                xc = __ldg(p.xc + o);
                yc = __ldg(p.yc + o);
                zc = __ldg(p.zc + o);
            }
            for (int s = s_lo + lane; s <= s_hi; s += 32) {
                const float sz = slice_z<OP>(p, s);
                const float ratio = __fdiv_rn(__fsub_rn(sz, z1), dz);
                if (!(ratio > 0.0f && ratio < 1.0f)) continue;
                const float cx = __fmaf_rn(d0, ratio, x1);
                const float cy = __fmaf_rn(d1, ratio, y1);
                const int ix0 =
                    __float2int_rz(__fdiv_rn(__fsub_rn(cx, p.l_bound), p.inter_x)) - p.half;
                const int iy0 =
                    __float2int_rz(__fdiv_rn(__fsub_rn(cy, p.b_bound), p.inter_y)) - p.half;
                float k0 = 0.0f;
                if (OP != kMap && p.tof_on) {
                    const float ax = __fsub_rn(xc, cx), ay = __fsub_rn(yc, cy),
                                az = __fsub_rn(zc, sz);
                    const float a2 = __fmaf_rn(az, az, __fmaf_rn(ax, ax, __fmul_rn(ay, ay)));
                    k0 = -a2 * p.a_coef;
                }
                const int i_lo = max(0, -ix0), i_hi = min(p.patch, p.gx - ix0);
                const int j_lo = max(0, -iy0), j_hi = min(p.patch, p.gy - iy0);
                if (OP == kCount) n_slots += max(0, i_hi - i_lo) * max(0, j_hi - j_lo);
                const int64_t base = (int64_t)s * slice_mesh;
                for (int j = j_lo; j < j_hi; ++j) {
                    const int iy = iy0 + j;
                    const float my = __fmaf_rn(p.inter_y, (float)iy + 0.5f, p.b_bound);
                    const float dy = __fsub_rn(cy, my);
                    const float dyuy = __fmul_rn(dy, uy);
                    const float dy2 = __fmul_rn(dy, dy);
                    const int64_t row = base + (int64_t)iy * p.gx;
                    for (int i = i_lo; i < i_hi; ++i) {
                        const int ix = ix0 + i;
                        const float mx = __fmaf_rn(p.inter_x, (float)ix + 0.5f, p.l_bound);
                        const float dx = __fsub_rn(cx, mx);
                        const float rc = __fmaf_rn(dx, ux, dyuy);
                        const float d2 = __fmaf_rn(-rc, rc, __fmaf_rn(dx, dx, dy2));
                        if (d2 < cut) {
                            const float w = exp2f(fmaf(d2, k1, k0));
                            if (OP == kCount) {
                                n_useful++;
                            } else if (OP == kProj) {
                                acc = fmaf(w, __ldg(p.image_in + row + ix), acc);
                            } else {
                                atomicAdd(p.image_out + row + ix, w * scale);
                            }
                        } else if (OP == kMap && all_slots) {
                            atomicAdd(p.image_out + row + ix, 0.0f * scale);
                        }
                    }
                }
            }
        }
        if (OP == kProj) {
            acc = warp_sum(acc);
            if (lane == 0) p.proj_out[t] = acc * scale;
        }
        if (OP == kCount) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                n_useful += __shfl_xor_sync(0xffffffffu, n_useful, o);
                n_slots += __shfl_xor_sync(0xffffffffu, n_slots, o);
            }
            if (lane == 0) {
                p.count_out[t] = n_useful;
                p.count_out[p.n + t] = n_slots;
            }
        }
    }
}

int tor_setup(TorParams &p, const int *grid, const float *center, const float *size,
              float kernel_width, float tof_bin, float tof_sigma2, int64_t n,
              int64_t lor_stride) {
    if (!grid || !center || !size) return SRF_ERR_INVALID_ARGUMENT;
    if (n < 0 || lor_stride < 1) return SRF_ERR_INVALID_ARGUMENT;
    if (grid[0] <= 0 || grid[1] <= 0 || grid[2] <= 0) return SRF_ERR_INVALID_ARGUMENT;
    if (!finite3(center) || !finite3(size)) return SRF_ERR_INVALID_ARGUMENT;
    if (size[0] <= 0.f || size[1] <= 0.f || size[2] <= 0.f) return SRF_ERR_INVALID_ARGUMENT;
    if (!(kernel_width >= 0.f) || !(kernel_width < 1e30f)) return SRF_ERR_INVALID_ARGUMENT;
    if (!(tof_sigma2 == tof_sigma2) || !(tof_bin == tof_bin)) return SRF_ERR_INVALID_ARGUMENT;
    if ((int64_t)grid[0] * grid[1] * grid[2] > ((int64_t)1 << 31) - 1)
        return SRF_ERR_UNSUPPORTED;

    // Host set-up of tor.cu.cc:364-375, in the reference's float arithmetic.
    const unsigned int gx = grid[0], gy = grid[1], gz = grid[2];
    const float lx = size[0], ly = size[1], lz = size[2];
    p.gx = (int)gx;
    p.gy = (int)gy;
    p.gz = (int)gz;
    p.inter_x = lx / gx;
    p.inter_y = ly / gy;
    p.inter_z = lz / gz;
    p.l_bound = center[0] - lx / 2;
    p.b_bound = center[1] - ly / 2;
    p.tor_sigma2 = kernel_width * kernel_width / 36;
    const double patch_d = std::ceil((std::sqrt(2.0) * kernel_width + p.inter_z) / p.inter_x);
    if (!(patch_d >= 0.0) || patch_d > 4096.0) return SRF_ERR_UNSUPPORTED;
    p.patch = (int)patch_d;
    p.half = (int)((unsigned)p.patch / 2);
    p.slice0_f = center[2] - (lz - p.inter_z) / 2;
    p.slice0_d = (double)center[2] - (double)(lz - p.inter_z) / 2.0;
    p.geo = 0;
    p.tof_on = tof_sigma2 < kTofThreshold ? 1 : 0;
    p.tse = tof_sigma2 + (tof_bin * tof_bin) / 12;
    const double log2e = 1.4426950408889634;
    p.a_coef = (float)(0.5 * log2e / (double)p.tse);
    p.cut = (float)(9.0 * (double)p.tor_sigma2);
    if ((double)p.cut < 9.0 * (double)p.tor_sigma2) p.cut = std::nextafter(p.cut, INFINITY);
    const double tsc = p.tor_sigma2;
    p.k1 = (float)(p.tof_on ? (0.5 * log2e / (double)p.tse - 0.5 * log2e / tsc)
                            : -0.5 * log2e / tsc);
    p.tof_scale = p.tof_on ? (float)((double)tof_bin / std::sqrt(2.0 * M_PI * (double)tof_sigma2))
                           : 1.0f;
    p.n = n;
    p.stride = lor_stride;
    return SRF_OK;
}

template <int OP>
int tor_launch(TorParams &p, cudaStream_t stream) {
    if (p.n == 0) return SRF_OK;
    const int block = 256;
    const int grid = stride_grid(p.n, block / 32, 8);
    tor_kernel<OP><<<grid, block, 0, stream>>>(p);
    return check_launch();
}

int zero_image(float *image, const int *grid, cudaStream_t stream) {
    size_t bytes = sizeof(float) * (size_t)grid[0] * grid[1] * grid[2];
    cudaError_t e = cudaMemsetAsync(image, 0, bytes, stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    return SRF_OK;
}

bool cols_ok(std::initializer_list<const void *> cols) {
    for (const void *c : cols)
        if (!c) return false;
    return true;
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int srf_tor_projection(const float *x1, const float *y1, const float *z1,
                                  const float *x2, const float *y2, const float *z2,
                                  const float *xc, const float *yc, const float *zc,
                                  const float *sigma2_factor, int geo_sigma2_flag,
                                  float *projection_value, const int *grid, const float *center,
                                  const float *size, float kernel_width, float tof_bin,
                                  float tof_sigma2, const float *image, int64_t num_events,
                                  int64_t lor_stride, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value, image}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && p.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.xc = xc; p.yc = yc; p.zc = zc; p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.image_in = image;
    p.proj_out = projection_value;
    return tor_launch<kProj>(p, (cudaStream_t)stream);
}

extern "C" int srf_tor_backprojection(const float *x1, const float *y1, const float *z1,
                                      const float *x2, const float *y2, const float *z2,
                                      const float *xc, const float *yc, const float *zc,
                                      const float *sigma2_factor, int geo_sigma2_flag,
                                      const float *projection_value, const int *grid,
                                      const float *center, const float *size,
                                      float kernel_width, float tof_bin, float tof_sigma2,
                                      float *image, int64_t num_events, int64_t lor_stride,
                                      int accumulate, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && p.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_image(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.xc = xc; p.yc = yc; p.zc = zc; p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.values = projection_value;
    p.image_out = image;
    return tor_launch<kBack>(p, (cudaStream_t)stream);
}

extern "C" int srf_tor_maplors(const float *x1, const float *y1, const float *z1,
                               const float *x2, const float *y2, const float *z2,
                               const float *sigma2_factor, int geo_sigma2_flag,
                               const float *projection_value, const int *grid,
                               const float *center, const float *size, float kernel_width,
                               float *image, int64_t num_events, int64_t lor_stride,
                               int accumulate, void *stream) {
    TorParams p{};
    // The map op carries no TOF attributes (tor.cc:49-64): TOF is off.
    int st = tor_setup(p, grid, center, size, kernel_width, 0.0f, 1.0e30f, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_image(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.values = projection_value;
    p.image_out = image;
    return tor_launch<kMap>(p, (cudaStream_t)stream);
}

extern "C" int srf_tor_count_samples(const float *x1, const float *y1, const float *z1,
                                     const float *x2, const float *y2, const float *z2,
                                     const float *sigma2_factor, int geo_sigma2_flag,
                                     const int *grid, const float *center, const float *size,
                                     float kernel_width, int *counts, int64_t num_events,
                                     int64_t lor_stride, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, 0.0f, 1.0e30f, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (num_events > 0 && !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, counts}))
        return SRF_ERR_INVALID_ARGUMENT;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.count_out = counts;
    return tor_launch<kCount>(p, (cudaStream_t)stream);
}

extern "C" int srf_tor_backproject_adjoint(const float *x1, const float *y1, const float *z1,
                                           const float *x2, const float *y2, const float *z2,
                                           const float *xc, const float *yc, const float *zc,
                                           const float *sigma2_factor, int geo_sigma2_flag,
                                           const float *values, const int *grid,
                                           const float *center, const float *size,
                                           float kernel_width, float tof_bin, float tof_sigma2,
                                           float *image, int64_t num_events,
                                           int64_t lor_stride, int accumulate, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (!image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, values}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && p.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_image(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.xc = xc; p.yc = yc; p.zc = zc; p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.values = values;
    p.image_out = image;
    return tor_launch<kAdj>(p, (cudaStream_t)stream);
}

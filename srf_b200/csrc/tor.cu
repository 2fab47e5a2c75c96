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

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "lor_prep.cuh"
#include "srf_common.cuh"

namespace srf {
namespace {

enum TorOp { kProj = 0, kBack = 1, kMap = 2, kAdj = 3, kCount = 4 };

// Process-wide tuning (srf_tor_set_tuning): kernel family (0 auto, 1 slab with a lane per
// segment, 2 LOR-centric, 3 slab with items spread over lanes),
// slices per slab (0 = as many as fit), grid multiplier of the persistent slab kernel
// (CTAs = SMs x mult, one resident per SM: more, smaller shares of the segment list;
// 0 = automatic, see slab_grid_mult).
std::atomic<int> g_tune_path{0};
std::atomic<int> g_tune_nsl{0};
std::atomic<int> g_tune_mult{0};

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
    float inv_x, inv_y;  // 1/inter_x, 1/inter_y (window bounding boxes only)
    float box_e;         // d^2 margin of the bounding boxes, far above float d^2 error
    const float *image_in;
    const float *values;
    float *image_out;
    float *proj_out;
    int *count_out;   // kCount: [n] voxels with non-zero weight, [n] window voxels visited
    int use_slab;     // scatter ops: shared-memory slab kernel (1) or global atomics (0)
    int slab_expand;  // slab kernel: spread items over lanes (1) or a lane per segment (0)
    // Batched frames: LOR i belongs to frame frame[i] (null: one frame) whose image starts
    // frame_stride floats after the previous frame's.
    const int *frame;
    int64_t frame_stride;
    int n_frames;
    // Element strides of the kernel axes x, y, z inside a frame of image_in and image_out
    // (1, gx, gx gy for a contiguous image; any layout whose frame fits in frame_stride,
    // e.g. a permuted view of an image stack, through the strided entry point).
    int64_t sx, sy, sz;
    // Map LORs made on the fly (srf_tor_maplors_generated): gen = 0 LOR columns in memory;
    // 1 uniform random crystal pairs; 2 every crystal pair of the scanner's block pairs.
    // LOR t of the call is number gen_first + t of that sequence, taken through
    // map_process and kept when its dominant axis is gen_axis; its value is 1.
    int gen, gen_axis;
    int64_t gen_first;
    unsigned long long gen_seed;
    const float *crystals;  // [n_rings * n_blocks * n_per_block][3] crystal centres
    int n_rings, n_blocks, n_per_block;
};

// ---------------------------------------------------------------------------------
// Generated detector-pair LORs (map calls). The random pairs use SplitMix64 (Steele, Lea
// and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014): output k of
// the stream seeded s is the finaliser applied to s + (k + 1) * 0x9E3779B97F4A7C15.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long s,
                                                         unsigned long long k) {
    unsigned long long z = s + (k + 1ull) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Crystal indices (a, b) of LOR number g; false for a pair of one crystal with itself.
//   gen 1: random chords of a ring scanner (crystal a_pos of ring r at index
//          r * n_per_block + a_pos, angle 2 pi a_pos / n_per_block). LORs come in groups of
//          kChordGroup consecutive numbers that share the transverse direction (the chord
//          class s = a_pos + b_pos mod n) and the ring offset d = r_b - r_a: with
//          (h1, l1) the high and low halves of splitmix64(seed, 4 group) and h2 the high
//          half of splitmix64(seed, 4 group + 2), s = floor(h1 n / 2^32) and d = j2 - j1,
//          j1 = floor(l1 nr / 2^32), j2 = floor(h2 nr / 2^32); per LOR, with (h, l) the
//          halves of splitmix64(seed, 2 g + 1) and i = g mod kChordGroup, a_pos =
//          floor(n (i + h / 2^32) / kChordGroup) (stratified: a uniform position, LOR i of a
//          group in the i-th part of the ring), b_pos = s - a_pos mod n and r_a =
//          max(0, -d) + floor(l (nr - |d|) / 2^32). Every ordered pair of
//          crystals is equally likely (s and a_pos uniform; d distributed as the
//          difference of two uniform rings, r_a uniform given d), and a warp's LORs
//          share a direction, so the slab kernels walk fewer wasted voxel slots than for
//          pairs drawn one by one;
//   gen 2: the g-th pair of the reference's effmap enumeration (srfapp_new.py:153-157 over
//          scanner/pet/pet.py:149-177): ring pairs (ir1, ir2) ir1-major, in each the block
//          pairs i1 < i2 (same ring) or i1 != i2 (different rings) row-major, in each every
//          crystal of the first block (major) with every crystal of the second.
constexpr long long kChordGroup = 256;

__device__ __forceinline__ unsigned scale32(unsigned u, unsigned n) {
    return (unsigned)(((unsigned long long)u * n) >> 32);
}

__device__ __forceinline__ bool gen_pair(const TorParams &p, long long g, int &a, int &b) {
    if (p.gen == 1) {
        const unsigned n = (unsigned)p.n_per_block, nr = (unsigned)p.n_rings;
        const unsigned long long grp = (unsigned long long)(g / kChordGroup);
        const unsigned long long hg = splitmix64(p.gen_seed, 4ull * grp);
        const unsigned long long hg2 = splitmix64(p.gen_seed, 4ull * grp + 2ull);
        const unsigned s = scale32((unsigned)(hg >> 32), n);
        const int d = (int)scale32((unsigned)(hg2 >> 32), nr) - (int)scale32((unsigned)hg, nr);
        const unsigned long long h = splitmix64(p.gen_seed, 2ull * (unsigned long long)g + 1ull);
        // stratified over the group: LOR i of the group draws a_pos in the i-th of
        // kChordGroup equal parts of the ring, so neighbours are near-identical chords
        const unsigned long long i = (unsigned long long)(g % kChordGroup);
        const unsigned a_pos = (unsigned)((((i << 32) | (h >> 32)) * n) >> 40);
        const unsigned b_pos = (s + n - a_pos) % n;
        const int r_lo = max(0, -d);
        const int r_a = r_lo + (int)scale32((unsigned)h, nr - (unsigned)abs(d));
        a = r_a * (int)n + (int)a_pos;
        b = (r_a + d) * (int)n + (int)b_pos;
        return a != b;
    }
    const long long nb = p.n_blocks, cb = (long long)p.n_per_block * p.n_per_block;
    const long long n_same = nb * (nb - 1) / 2 * cb, n_cross = nb * (nb - 1) * cb;
    const long long row = (long long)(p.n_rings - 1) * n_cross + n_same;  // one ir1
    const long long ir1 = g / row;
    long long r = g - ir1 * row;
    long long ir2;
    if (r < ir1 * n_cross) {
        ir2 = r / n_cross;
        r -= ir2 * n_cross;
    } else if (r < ir1 * n_cross + n_same) {
        ir2 = ir1;
        r -= ir1 * n_cross;
    } else {
        const long long q = r - ir1 * n_cross - n_same;
        ir2 = ir1 + 1 + q / n_cross;
        r = q - (ir2 - ir1 - 1) * n_cross;
    }
    const long long bp = r / cb, rc = r - bp * cb;
    long long i1, i2;
    if (ir1 == ir2) {
        // row i of the strict upper triangle holds nb - 1 - i pairs and starts at
        // i (2 nb - i - 1) / 2; estimate i from the quadratic, then correct exactly
        const double bb = 2.0 * (double)nb - 1.0;
        long long i = (long long)floor((bb - sqrt(fmax(bb * bb - 8.0 * (double)bp, 0.0))) / 2.0);
        i = max(0ll, min(i, nb - 2));
        while (i > 0 && i * (2 * nb - i - 1) / 2 > bp) i--;
        while (i < nb - 2 && (i + 1) * (2 * nb - i - 2) / 2 <= bp) i++;
        i1 = i;
        i2 = i + 1 + (bp - i * (2 * nb - i - 1) / 2);
    } else {
        i1 = bp / (nb - 1);
        const long long j = bp - i1 * (nb - 1);
        i2 = j + (j >= i1 ? 1 : 0);
    }
    const long long c1 = rc / p.n_per_block, c2 = rc - c1 * p.n_per_block;
    a = (int)((ir1 * nb + i1) * p.n_per_block + c1);
    b = (int)((ir2 * nb + i2) * p.n_per_block + c2);
    return true;
}

// The map record columns of generated LOR t (x1, y1, z1, x2, y2, z2, f after
// map_process's swap and permutation); false when its dominant axis is another group's.
__device__ __forceinline__ bool gen_columns(const TorParams &p, int64_t t, float (&c)[7]) {
    int a, b;
    if (!gen_pair(p, (long long)(p.gen_first + t), a, b)) return false;
    float e[6];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        e[k] = __ldg(p.crystals + 3 * (int64_t)a + k);
        e[3 + k] = __ldg(p.crystals + 3 * (int64_t)b + k);
    }
    // the dominant axis first (process's own test): another group's LOR costs no more
    if (dominant_axis(e) != p.gen_axis) return false;
    const Rec r = process<false>(e, false, 0.0f);  // map_process (on_tor_lors.py:243-248)
    if (r.bucket >= kBuckets || (r.bucket >> 1) != p.gen_axis) return false;
#pragma unroll
    for (int k = 0; k < 7; k++) c[k] = r.v[k];
    return true;
}

// LOR t's endpoints and sigma^2 factor (from memory, or generated); false for a generated
// LOR of another axis group.
// kGen: the call's LORs are generated (TorParams::gen), map calls only.
template <int OP, bool kGen>
__device__ __forceinline__ bool lor_columns(const TorParams &p, int64_t t, float &x1, float &y1,
                                            float &z1, float &x2, float &y2, float &z2,
                                            float &f) {
    if constexpr (kGen) {
        static_assert(OP == kMap, "generated LORs are map LORs");
        static_assert(kChordGroup == 256, "the stratified draw shifts by 40 = 32 + log2(256)");
        float c[7];
        if (!gen_columns(p, t, c)) return false;
        x1 = c[0]; y1 = c[1]; z1 = c[2]; x2 = c[3]; y2 = c[4]; z2 = c[5]; f = c[6];
        return true;
    }
    const int64_t o = t * p.stride;
    x1 = __ldg(p.x1 + o); y1 = __ldg(p.y1 + o); z1 = __ldg(p.z1 + o);
    x2 = __ldg(p.x2 + o); y2 = __ldg(p.y2 + o); z2 = __ldg(p.z2 + o);
    f = __ldg(p.f + o);
    return true;
}

// The map's divisor of LOR t (the caller's lors_value; 1 for generated LORs).
__device__ __forceinline__ float map_value(const TorParams &p, int64_t t) {
    return p.values ? __ldg(p.values + t) : 1.0f;
}

__device__ __forceinline__ int64_t frame_offset(const TorParams &p, int64_t t) {
    return p.frame ? (int64_t)__ldg(p.frame + t) * p.frame_stride : 0;
}

// Batched calls: a LOR whose frame id lies outside [0, n_frames) contributes nothing
// (as a LOR with non-finite endpoints does) instead of indexing past the image stack.
__device__ __forceinline__ bool frame_ok(const TorParams &p, int64_t t) {
    return !p.frame || (unsigned)__ldg(p.frame + t) < (unsigned)p.n_frames;
}

// slice_z of the reference launchers: float for projection (tor.cu.cc:380), a double
// intermediate for back-projection and map (:423, :471).
template <int OP>
__device__ __forceinline__ float slice_z(const TorParams &p, int s) {
    float step = __fmul_rn((float)s, p.inter_z);
    if (OP == kProj) return __fadd_rn(p.slice0_f, step);
    return __double2float_rn(p.slice0_d + (double)step);
}

// 2^x with the hardware approximation (ex2.approx, relative error ~2^-22); the
// argument here is always <= ~0, results below 2^-126 flush to zero.
__device__ __forceinline__ float fast_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Generic per-LOR body (any patch size): the reference's loops as written, every
// in-slice window voxel visited. Used for patch sizes without a specialised kernel and
// for map calls whose divisor is zero or non-finite.
template <int OP>
__device__ __noinline__ void generic_lor(const TorParams &p, int64_t t, int lane) {
    if (!frame_ok(p, t)) {
        if (OP == kProj && lane == 0) p.proj_out[t] = 0.0f;
        if (OP == kCount && lane == 0) p.count_out[t] = p.count_out[p.n + t] = 0;
        return;
    }
    const int64_t img0 = frame_offset(p, t);
    const int64_t o = t * p.stride;
    float x1, y1, z1, x2, y2, z2, f;
    bool have;
    if constexpr (OP == kMap)
        have = p.gen ? lor_columns<OP, true>(p, t, x1, y1, z1, x2, y2, z2, f)
                     : lor_columns<OP, false>(p, t, x1, y1, z1, x2, y2, z2, f);
    else
        have = lor_columns<OP, false>(p, t, x1, y1, z1, x2, y2, z2, f);
    if (!have) {
        if (OP == kCount && lane == 0) p.count_out[t] = p.count_out[p.n + t] = 0;
        return;
    }

    // Per-LOR output scale and the early-outs of the reference's value tests.
    float scale = p.tof_scale;
    bool all_slots = false;  // map with a zero/non-finite divisor: every visited voxel gets w/v
    if (OP == kBack) {
        float v = __ldg(p.values + t);
        if (!((double)v > 1e-7)) return;  // tor.cu.cc:203
        scale = __fdiv_rn(p.tof_scale, v);
    } else if (OP == kMap) {
        float v = map_value(p, t);
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
            const int64_t base = (int64_t)s * p.sz;
            for (int j = j_lo; j < j_hi; ++j) {
                const int iy = iy0 + j;
                const float my = __fmaf_rn(p.inter_y, (float)iy + 0.5f, p.b_bound);
                const float dy = __fsub_rn(cy, my);
                const float dyuy = __fmul_rn(dy, uy);
                const float dy2 = __fmul_rn(dy, dy);
                const int64_t row = base + (int64_t)iy * p.sy;
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
                            acc = fmaf(w, __ldg(p.image_in + img0 + row + ix * p.sx), acc);
                        } else {
                            atomicAdd(p.image_out + img0 + row + ix * p.sx, w * scale);
                        }
                    } else if (OP == kMap && all_slots) {
                        atomicAdd(p.image_out + img0 + row + ix * p.sx, 0.0f * scale);
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

template <int OP>
__global__ void __launch_bounds__(256) tor_kernel(const TorParams p) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < p.n; t += nwarps) generic_lor<OP>(p, t, lane);
}

// ---------------------------------------------------------------------------------
// Fast path: per-LOR constants, per-slice visit, and two kernels built on them.
//
// Same traversal and the same float arithmetic for every quantity the reference
// rounds, with three changes that cut the instruction count per voxel slot:
//  * only the part of the P x P window inside the bounding box of the tube's section
//    is walked. With d^2 = dx^2 + dy^2 - (dx ux + dy uy)^2 and q = 1 - ux^2 - uy^2, the
//    set d^2 < c is an ellipse whose half-extents are sqrt(c (1 - uy^2) / q) along x and
//    sqrt(c (1 - ux^2) / q) along y. The box is taken for c = cut + box_e, box_e far
//    above the float error of d^2, so it holds every voxel the reference weights non-zero;
//    each voxel in it still takes the exact float test. For dominant-axis LOR groups
//    q >= 1/3 and the box is 4-5 voxels wide where the window is 6;
//  * the P column offsets dx_i = X_x - mesh_x(i) are computed once per slice;
//  * the weight is one raw ex2 and the slot test is predicated, not branched.

struct LorConst {
    float x1, y1, z1, d0, d1, dz, ux, uy;
    float cut, k1;
    float bxv, byv;  // bounding-box half-extents in voxels (margin included)
    float xc, yc, zc;
    float scale;
    float k0s;       // back-projection: log2(scale), folded into the exponent (else 0)
    int s_lo, s_hi;  // candidate slices (a superset; each is tested exactly)
    bool all;        // map with a zero / non-finite divisor: every window voxel gets w/v
};

// The per-LOR constants that do not depend on the op's values: direction, cut-off and
// exponent slope, bounding-box half-extents, TOF centre and candidate slices. Returns
// false when no crossing is possible (degenerate or non-finite LOR, bad frame id).
template <int OP, bool kGen = false>
__device__ __forceinline__ bool lor_geometry(const TorParams &p, int64_t t, LorConst &L) {
    L.all = false;
    L.scale = p.tof_scale;
    L.k0s = 0.0f;
    L.s_lo = 0;
    L.s_hi = -1;
    if (!frame_ok(p, t)) return false;
    const int64_t o = t * p.stride;
    float x1, y1, z1, x2, y2, z2, f;
    if (!lor_columns<OP, kGen>(p, t, x1, y1, z1, x2, y2, z2, f)) return false;
    L.x1 = x1;
    L.y1 = y1;
    L.z1 = z1;
    L.d0 = __fsub_rn(x2, x1);
    L.d1 = __fsub_rn(y2, y1);
    L.dz = __fsub_rn(z2, z1);
    const float dis =
        __fsqrt_rn(__fmaf_rn(L.dz, L.dz, __fmaf_rn(L.d0, L.d0, __fmul_rn(L.d1, L.d1))));
    L.ux = __fdiv_rn(L.d0, dis);
    L.uy = __fdiv_rn(L.d1, dis);
    L.cut = p.cut;
    L.k1 = p.k1;
    if (p.geo) {
        const float tsc = __fmul_rn(p.tor_sigma2, f);  // tor.cu.cc:67
        L.cut = __double2float_ru(9.0 * (double)tsc);
        const float inv = 0.5f * kLog2e / tsc;
        L.k1 = (p.tof_on && OP != kMap) ? (p.a_coef - inv) : -inv;
    }
    {
        const float om_x = 1.0f - L.ux * L.ux, om_y = 1.0f - L.uy * L.uy;
        const float q = om_x - L.uy * L.uy;
        const float c = L.cut * 1.0001f + p.box_e;
        const bool boxed = q > 1e-3f && c < 3.0e38f;
        // outside a box (nearly in-plane LOR): the whole window
        L.bxv = boxed ? sqrtf(c * om_y / q) * p.inv_x + (1.0f / 1024.0f) : 1.0e9f;
        L.byv = boxed ? sqrtf(c * om_x / q) * p.inv_y + (1.0f / 1024.0f) : 1.0e9f;
    }
    L.xc = L.yc = L.zc = 0.0f;
    if (OP != kMap && OP != kCount && p.tof_on) {
        L.xc = __ldg(p.xc + o);
        L.yc = __ldg(p.yc + o);
        L.zc = __ldg(p.zc + o);
    }
    const float zlo = fminf(z1, z2), zhi = fmaxf(z1, z2);
    if (!(L.dz != 0.0f && zlo == zlo && zhi == zhi && fabsf(zhi - zlo) <= 3.0e38f)) return false;
    const float flo = floorf((zlo - p.slice0_f) / p.inter_z) - 2.0f;
    const float fhi = ceilf((zhi - p.slice0_f) / p.inter_z) + 2.0f;
    L.s_lo = (int)fmaxf(flo, 0.0f);
    L.s_hi = (int)fminf(fhi, (float)(p.gz - 1));
    return L.s_lo <= L.s_hi;
}

// The op's per-LOR output scale from its value (back-projection: tof_scale / v, dropped
// at or below 1e-7, tor.cu.cc:203; map: 1 / v with no threshold, :239, where a zero or
// non-finite divisor lands w/v on every visited voxel; adjoint: tof_scale * v). Returns
// false when the LOR contributes nothing.
template <int OP>
__device__ __forceinline__ bool lor_value_scale(const TorParams &p, int64_t t, LorConst &L) {
    if (OP == kBack) {
        const float v = __ldg(p.values + t);
        if (!((double)v > 1e-7)) return false;  // tor.cu.cc:203
        L.scale = __fdiv_rn(p.tof_scale, v);
        // w * scale = 2^(log2 w + log2 scale): the scale joins the exponent (one add per
        // slice instead of one multiply per voxel). scale = m 2^e with m in [0.5, 1):
        // log2 m from the hardware approximation (absolute error ~2^-22) plus e exactly.
        int e;
        const float m = frexpf(L.scale, &e);
        L.k0s = (float)e + __log2f(m);
    } else if (OP == kMap) {
        L.scale = __fdiv_rn(1.0f, map_value(p, t));  // tor.cu.cc:239, no threshold
        L.all = !(fabsf(L.scale) <= 3.0e38f);  // w/0 or w/NaN lands on every visited voxel
        if (L.all) L.bxv = L.byv = 1.0e9f;     // ... so the whole window is walked
    } else if (OP == kAdj) {
        L.scale = p.tof_scale * __ldg(p.values + t);
    }
    return true;
}

// Loads LOR t and derives its constants. Returns false when the LOR contributes
// nothing (no crossing possible, or a back-projection value at/below 1e-7).
template <int OP, bool kGen = false>
__device__ __forceinline__ bool lor_prepare(const TorParams &p, int64_t t, LorConst &L) {
    if (!lor_geometry<OP, kGen>(p, t, L)) return false;
    return lor_value_scale<OP>(p, t, L);
}

// lor_geometry / lor_prepare for a call whose LORs may be generated (map calls).
template <int OP>
__device__ __forceinline__ bool geometry_any(const TorParams &p, int64_t t, LorConst &L) {
    if constexpr (OP == kMap) {
        if (p.gen) return lor_geometry<OP, true>(p, t, L);
    }
    return lor_geometry<OP, false>(p, t, L);
}

template <int OP>
__device__ __forceinline__ bool prepare_any(const TorParams &p, int64_t t, LorConst &L) {
    if constexpr (OP == kMap) {
        if (p.gen) return lor_prepare<OP, true>(p, t, L);
    }
    return lor_prepare<OP, false>(p, t, L);
}

// The binning pass stores each LOR's geometry once as a 64-byte record, so the slab
// kernels take it with four 16-byte loads per segment instead of re-deriving it from the
// ten columns in every slab the LOR meets:
//   {x1, y1, z1, d0}, {d1, dz, ux, uy}, {cut, k1, bxv, byv}, {xc, yc, zc, slices}
// with slices = s_lo | s_hi << 16, or -1 when the LOR contributes nothing.
struct __align__(16) LorRec {
    float4 a, b, c, d;
};

__device__ __forceinline__ LorRec make_rec(const LorConst &L, bool ok) {
    LorRec r;
    r.a = make_float4(L.x1, L.y1, L.z1, L.d0);
    r.b = make_float4(L.d1, L.dz, L.ux, L.uy);
    r.c = make_float4(L.cut, L.k1, L.bxv, L.byv);
    r.d = make_float4(L.xc, L.yc, L.zc, __int_as_float(ok ? (L.s_lo | (L.s_hi << 16)) : -1));
    return r;
}

__device__ __forceinline__ float4 ldg_f4(const float4 *q) {
    float4 v;
    asm("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(q));
    return v;
}

// LOR t's geometry from its record; false when the LOR contributes nothing.
__device__ __forceinline__ bool lor_rec_geometry(const LorRec *rec, int64_t t, LorConst &L) {
    const float4 *q = reinterpret_cast<const float4 *>(rec + t);
    const float4 d = ldg_f4(q + 3);
    const int sl = __float_as_int(d.w);
    const float4 a = ldg_f4(q), b = ldg_f4(q + 1), c = ldg_f4(q + 2);
    L.x1 = a.x; L.y1 = a.y; L.z1 = a.z; L.d0 = a.w;
    L.d1 = b.x; L.dz = b.y; L.ux = b.z; L.uy = b.w;
    L.cut = c.x; L.k1 = c.y; L.bxv = c.z; L.byv = c.w;
    L.xc = d.x; L.yc = d.y; L.zc = d.z;
    L.s_lo = sl & 0xffff;
    L.s_hi = sl >> 16;
    L.all = false;
    L.k0s = 0.0f;
    return sl >= 0;
}

// LOR t's constants from its record and the op's value (lor_prepare's result).
template <int OP>
__device__ __forceinline__ bool lor_load(const TorParams &p, const LorRec *rec, int64_t t,
                                         LorConst &L) {
    L.scale = p.tof_scale;
    if (!lor_rec_geometry(rec, t, L)) return false;
    return lor_value_scale<OP>(p, t, L);
}

// (int)(a / b) with a correctly rounded quotient, as the reference truncates it
// (tor.cu.cc:135-136). q = a * (1/b) is within 2^-22 |a/b| of the rounded quotient, so
// both truncate to the same integer unless q lies that close to an integer (or is 0);
// only then is the division itself evaluated.
__device__ __forceinline__ int trunc_div(float a, float b, float inv_b) {
    const float q = a * inv_b;
    if (fabsf(q - rintf(q)) <= fabsf(q) * 1.0e-6f) return __float2int_rz(__fdiv_rn(a, b));
    return __float2int_rz(q);
}

// One voxel slot: the reference's d^2 (tor.cu.cc:61-66, FMA-contracted as nvcc builds
// it) and cut-off decision, and the folded exponent.
// `cut` and `all` are the LOR's (L.cut, L.all) for a row the caller walks, -inf and false
// for a row it must leave out (so the row costs no branch).
template <int OP, typename F>
__device__ __forceinline__ void slot(const LorConst &L, float cut, bool all, float dx, float dyuy,
                                     float dy2, float k0, int ix, int iy, F &f) {
    const float rc = __fmaf_rn(dx, L.ux, dyuy);
    const float d2 = __fmaf_rn(-rc, rc, __fmaf_rn(dx, dx, dy2));
    const bool in_cut = d2 < cut;
    const float e = fast_exp2(fmaf(d2, L.k1, k0));
    if (OP == kMap)
        f(ix, iy, in_cut ? e : 0.0f, in_cut || all);
    else
        f(ix, iy, e, in_cut);
}

// W consecutive slots of one row.
template <int OP, int W, int P, typename F>
__device__ __forceinline__ void row_slots(const LorConst &L, float cut, bool all,
                                          const float (&dxs)[P], float dy, float k0, int xlo,
                                          int iy, F &f) {
    const float dyuy = __fmul_rn(dy, L.uy);
    const float dy2 = __fmul_rn(dy, dy);
#pragma unroll
    for (int i = 0; i < W; i++) slot<OP>(L, cut, all, dxs[i], dyuy, dy2, k0, xlo + i, iy, f);
}

// g(std::integral_constant<int, w>{}) for a runtime width 1 <= w <= P.
template <int P, typename G>
__device__ __forceinline__ void with_width(int w, G &&g) {
    if constexpr (P >= 1) {
        if (w >= P) {
            g(std::integral_constant<int, P>{});
        } else {
            with_width<P - 1>(w, g);
        }
    }
}

// One (LOR, slice): the reference's crossing test and window (tor.cu.cc:22-48,
// :135-136), then the voxels of the window's part inside the tube's bounding box:
// f(ix, iy, w, use) with w the unscaled weight and use the reference's decision (d^2
// below the cut-off; for a map LOR with L.all set, every in-slice window voxel, with
// w = 0 outside the cut-off, as the reference adds 0/0 there). Returns the number of
// in-slice window voxels (for kCount).
//
// Only rows R0 <= iy < R1 are walked (a band of rows of the grid, or all of it).
// kPadded: the caller's slice has P - 1 zero columns on both sides of the grid and P - 1
// spare rows above and below the band (the shared-memory slab), so window columns
// outside the grid need no test: a gather reads 0 there and a scatter lands in padding
// that is never flushed. The walked box is then widened to the warp's largest (kept
// inside the window), which makes the trip counts warp-uniform; rows the widening adds
// outside the band are masked. Otherwise the box is clipped to the grid.
template <int OP, int P, bool kPadded, bool kBand, typename F>
__device__ __forceinline__ int slice_visit(const TorParams &p, const LorConst &L, int s, int R0,
                                           int R1, F &&f) {
    const float sz = slice_z<OP>(p, s);
    const float ratio = __fdiv_rn(__fsub_rn(sz, L.z1), L.dz);
    if (!(ratio > 0.0f && ratio < 1.0f)) return 0;
    const float cx = __fmaf_rn(L.d0, ratio, L.x1);
    const float cy = __fmaf_rn(L.d1, ratio, L.y1);
    const float rx = __fsub_rn(cx, p.l_bound), ry = __fsub_rn(cy, p.b_bound);
    const int ix0 = trunc_div(rx, p.inter_x, p.inv_x) - p.half;
    const int iy0 = trunc_div(ry, p.inter_y, p.inv_y) - p.half;
    if (ix0 >= p.gx || iy0 >= p.gy || ix0 <= -P || iy0 <= -P) return 0;  // window off the grid
    int n_slots = 0;
    if (OP == kCount) {
        const int i_lo = max(0, -ix0), i_hi = min(P, p.gx - ix0);
        const int j_lo = max(0, -iy0), j_hi = min(P, p.gy - iy0);
        n_slots = (i_hi - i_lo) * (j_hi - j_lo);
    }
    // Bounding box in voxel-centre units (column i has its centre at i + 0.5 voxels).
    const float fx = __fmaf_rn(rx, p.inv_x, -0.5f), fy = __fmaf_rn(ry, p.inv_y, -0.5f);
    int xlo = max(ix0, __float2int_ru(fx - L.bxv));
    int xhi = min(ix0 + P - 1, __float2int_rd(fx + L.bxv));
    int ylo = max(iy0, __float2int_ru(fy - L.byv));
    int yhi = min(iy0 + P - 1, __float2int_rd(fy + L.byv));
    // A slab holding whole slices has zero padding rows too; only a band needs row limits.
    constexpr bool banded = !kPadded || kBand;
    if (banded) {
        ylo = max(ylo, R0);
        yhi = min(yhi, R1 - 1);
    }
    if (!kPadded) {
        xlo = max(xlo, 0);
        xhi = min(xhi, p.gx - 1);
    }
    int wx = xhi - xlo + 1, wy = yhi - ylo + 1;
    if (wx <= 0 || wy <= 0) return n_slots;
    if (kPadded) {
        const unsigned am = __activemask();
        const int mx = __reduce_max_sync(am, wx), my = __reduce_max_sync(am, wy);
        xlo = min(xlo, ix0 + P - mx);  // still inside the window, still covers the box
        ylo = min(ylo, iy0 + P - my);
        wx = mx;
        wy = my;
    }
    float k0 = OP == kBack ? L.k0s : 0.0f;
    if (OP != kMap && OP != kCount && p.tof_on) {
        const float ax = __fsub_rn(L.xc, cx), ay = __fsub_rn(L.yc, cy), az = __fsub_rn(L.zc, sz);
        const float a2 = __fmaf_rn(az, az, __fmaf_rn(ax, ax, __fmul_rn(ay, ay)));
        k0 = fmaf(-a2, p.a_coef, k0);
    }
    float dxs[P];
    const float fx0 = (float)xlo;
#pragma unroll
    for (int i = 0; i < P; i++) {
        const float mxi = __fmaf_rn(p.inter_x, fx0 + ((float)i + 0.5f), p.l_bound);
        dxs[i] = __fsub_rn(cx, mxi);
    }
    if (kPadded) {
        // wx, wy are warp-uniform: one fully unrolled row body per width, so that a row's
        // loads issue back to back. The gather picks the body once per slice; the scatter
        // (a compare-and-swap loop per voxel in shared memory) runs faster picking it per
        // row (measured).
        // In a band, rows the widening added outside [R0, R1) (another band's, or off
        // the grid) are masked through their cut-off; the walked rows stay within the
        // slab's padding rows. Whole slices need no mask (their padding rows read 0).
        const float fy0 = (float)ylo + 0.5f;
        auto walk = [&](auto masked) {
            constexpr bool kMask = decltype(masked)::value;
            auto row_cut = [&](int j, bool &all) {
                if constexpr (kMask) {
                    const bool in_band = (unsigned)(ylo + j - R0) < (unsigned)(R1 - R0);
                    all = in_band && L.all;
                    return in_band ? L.cut : -INFINITY;
                } else {
                    all = L.all;
                    return L.cut;
                }
            };
            // fj = ylo + j + 0.5 (a half-integer: adding 1 per row is exact)
            if (OP == kProj) {
                with_width<P>(wx, [&](auto W) {
                    float fj = fy0;
                    for (int j = 0; j < wy; j++, fj += 1.0f) {
                        bool all;
                        const float cut = row_cut(j, all);
                        const float dy = __fsub_rn(cy, __fmaf_rn(p.inter_y, fj, p.b_bound));
                        row_slots<OP, decltype(W)::value>(L, cut, all, dxs, dy, k0, xlo, ylo + j,
                                                          f);
                    }
                });
            } else {
                float fj = fy0;
                for (int j = 0; j < wy; j++, fj += 1.0f) {
                    bool all;
                    const float cut = row_cut(j, all);
                    const float dy = __fsub_rn(cy, __fmaf_rn(p.inter_y, fj, p.b_bound));
                    with_width<P>(wx, [&](auto W) {
                        row_slots<OP, decltype(W)::value>(L, cut, all, dxs, dy, k0, xlo, ylo + j,
                                                          f);
                    });
                }
            }
        };
        walk(std::integral_constant<bool, kBand>{});
    } else {
#pragma unroll
        for (int j = 0; j < P; j++) {
            if (j >= wy) break;
            const int iy = ylo + j;
            const float dy = __fsub_rn(cy, __fmaf_rn(p.inter_y, (float)iy + 0.5f, p.b_bound));
            const float dyuy = __fmul_rn(dy, L.uy);
            const float dy2 = __fmul_rn(dy, dy);
#pragma unroll
            for (int i = 0; i < P; i++) {
                if (i >= wx) break;
                slot<OP>(L, L.cut, L.all, dxs[i], dyuy, dy2, k0, xlo + i, iy, f);
            }
        }
    }
    return n_slots;
}

// LOR-centric kernel: one warp per LOR, lanes over its slices; projection gathers
// from the image in L2/L1, scatter ops use global atomics.
template <int OP, int P>
__global__ void __launch_bounds__(256) tor_kernel_p(const TorParams p) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t t = warp; t < p.n; t += nwarps) {
        LorConst L;
        const bool any = prepare_any<OP>(p, t, L);
        float acc = 0.0f;
        int n_useful = 0, n_slots = 0;
        if (any) {
            const int64_t img0 = frame_offset(p, t);
            for (int s = L.s_lo + lane; s <= L.s_hi; s += 32) {
                const int64_t base = img0 + (int64_t)s * p.sz;
                n_slots += slice_visit<OP, P, false, false>(p, L, s, 0, p.gy,
                                                     [&](int ix, int iy, float w, bool use) {
                    const int64_t idx = base + (int64_t)iy * p.sy + (int64_t)ix * p.sx;
                    if (OP == kCount) {
                        n_useful += use ? 1 : 0;
                    } else if (OP == kProj) {
                        if (use) acc = fmaf(w, __ldg(p.image_in + idx), acc);
                    } else {
                        // back-projection: the scale is in w's exponent already
                        if (use) atomicAdd(p.image_out + idx, OP == kBack ? w : w * L.scale);
                    }
                });
            }
        }
        if (OP == kProj) {
            acc = warp_sum(acc);
            if (lane == 0) p.proj_out[t] = any ? acc * L.scale : 0.0f;
        }
        if (OP == kCount) {
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) {
                n_useful += __shfl_xor_sync(0xffffffffu, n_useful, o2);
                n_slots += __shfl_xor_sync(0xffffffffu, n_slots, o2);
            }
            if (lane == 0) {
                p.count_out[t] = n_useful;
                p.count_out[p.n + t] = n_slots;
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Slab path for the scatter ops (back-projection, map, adjoint).
//
// The kernel-layout image is cut into slabs of `nsl` consecutive slices that fit in
// shared memory. Each LOR is binned into every slab its candidate slice range meets
// (a segment = (slab, LOR)); the segments are laid out slab by slab. A persistent grid
// then gives every CTA an equal, contiguous share of that list: the CTA accumulates its
// segments' voxel weights into the slab with shared-memory atomics and adds the slab to
// the output once per slab it touched (a share spans one or two slabs). Global atomics
// drop from one per non-zero voxel weight (5e9 per 10M-event pass) to one per slab voxel
// per CTA, and no SM waits on an overfull slab.
//
// Binning (three kernels, deterministic counts, order inside a slab unspecified):
//   seg_count  per LOR: slab range -> packed (k_lo, k_hi); per-tile slab histogram
//   seg_scan   per slab: scan over tiles; slab offsets; total
//   seg_fill   per LOR: write its index into each slab's list

constexpr int kSegThreads = 512;
constexpr int kSegItems = 8;
constexpr int kSegTile = kSegThreads * kSegItems;
constexpr int kMaxSlabs = 4096;
constexpr int kSlabThreads = 1024;
constexpr size_t kSlabSmemBytes = 220 * 1024;  // of the 227 KB a CTA can opt into
// Budget of the per-slab LOR lists of one chunk of LORs (srf_tor_set_scratch_limit). The
// lists are sized for the worst case (every slab of a frame), so the budget sets how many
// chunks a call over row-band slabs takes, each a full pass (slab loads and flushes again):
// 10M events at 256 x 256 x 128 24.1 ms per combined call with 1 GiB, 20.9 with 2, 19.0
// with 4 (5 -> 2 chunks per group); 50M generated map LORs 242 / 221 / 208 ms. 4 GiB is
// 2 % of a B200's memory, held by the library's pool once a call has needed it.
constexpr long long kSegScratchDefault = 4ll << 30;
std::atomic<long long> g_seg_scratch_bytes{kSegScratchDefault};

struct SegPlan {
    int nsl, n_slabs, ntiles;  // n_slabs counts slab ids over all frames
    int slabs_pf;              // slice ranges per frame
    int nbands, band_rows;     // row bands per slice range and rows per band (last: fewer)
    unsigned band_magic;       // ceil(2^32 / band_rows): r / band_rows = umulhi(r, magic)
    int *range;            // [n] packed k_lo | k_hi << 16, or -1
    int *tile_counts;      // [ntiles * n_slabs]
    int64_t *tile_offs;    // [ntiles * n_slabs]
    int64_t *slab_offs;    // [n_slabs + 1]
    int *seg;              // [capacity] LOR indices, slab-major
    LorRec *rec;           // [n] per-LOR records written by seg_count
};

// Slab ids (slice range k of a LOR's frame, row band b): id = k * nbands + b, with k
// counted over frames. With row bands, the bands of slice range k are those the LOR's
// window rows can reach in its slices there: the rows follow the crossing point's y, which
// is monotonic in the slice, so the rows of the range's two end slices, with two rows of
// margin and the window's extent, bound them. y1, z1, d1 = y2 - y1 and dz = z2 - z1 come
// from the LOR's record, so counting and filling agree bit for bit.
struct SlabIdLor {
    int k_lo, k_hi, s_lo, s_hi, f0;
    float y1, d1, r0, rs, z1, dz;
    int lin;  // y at slice s from r0 + s rs (else the division, where 1 / dz would overflow)
};

__device__ __forceinline__ SlabIdLor slab_id_lor(const TorParams &p, const SegPlan &sp,
                                                 int64_t t, int k_lo, int k_hi, int s_lo,
                                                 int s_hi, float y1, float z1, float d1,
                                                 float dz) {
    SlabIdLor c;
    c.k_lo = k_lo;
    c.k_hi = k_hi;
    c.s_lo = s_lo;
    c.s_hi = s_hi;
    c.f0 = p.frame ? __ldg(p.frame + t) * sp.slabs_pf : 0;
    // the crossing's position along the LOR at slice s, r(s) = (z_s - z1) / dz, as
    // r0 + s * rs: within a few ulps of the division, far inside the two rows of margin
    c.lin = fabsf(dz) > 1.0e-30f;
    const float inv_dz = c.lin ? 1.0f / dz : 0.0f;
    c.r0 = (p.slice0_f - z1) * inv_dz;
    c.rs = p.inter_z * inv_dz;
    c.y1 = y1;
    c.d1 = d1;
    c.z1 = z1;
    c.dz = dz;
    return c;
}

// LOR c's slab ids in slice range k: g(id) for each band its windows can reach.
template <bool kBand, typename G>
__device__ __forceinline__ void range_slab_ids(const TorParams &p, const SegPlan &sp,
                                               const SlabIdLor &c, int k, G &&g) {
    if constexpr (!kBand) {
        g(k);
        return;
    }
    auto y_at = [&](int s) {
        const float r = c.lin ? fmaf((float)s, c.rs, c.r0)
                              : (p.slice0_f + (float)s * p.inter_z - c.z1) / c.dz;
        return fmaf(c.d1, fminf(fmaxf(r, 0.0f), 1.0f), c.y1);
    };
    const int first = (k - c.f0) * sp.nsl;
    const float ya = y_at(max(c.s_lo, first)), yb = y_at(min(c.s_hi, first + sp.nsl - 1));
    const float lo = fminf(ya, yb), hi = fmaxf(ya, yb);
    int b_lo = 0, b_hi = sp.nbands - 1;
    if (lo == lo && hi == hi) {  // else: every band, left to the exact per-slice test
        const float flo = fminf(fmaxf(floorf((lo - p.b_bound) * p.inv_y), -1.0e8f), 1.0e8f);
        const float fhi = fminf(fmaxf(floorf((hi - p.b_bound) * p.inv_y), -1.0e8f), 1.0e8f);
        const int r_lo = max((int)flo - p.half - 2, 0);
        const int r_hi = min((int)fhi - p.half + p.patch + 1, p.gy - 1);
        if (r_lo > r_hi) return;
        // 0 <= r < 2^14 and band_rows < 2^14: the multiply-high quotient is exact
        b_lo = (int)__umulhi((unsigned)r_lo, sp.band_magic);
        b_hi = min((int)__umulhi((unsigned)r_hi, sp.band_magic), sp.nbands - 1);
    }
    for (int b = b_lo; b <= b_hi; b++) g(k * sp.nbands + b);
}

// The slab ids of the warp's LORs (lane l holds LOR t_l, `ok` when it enters the lists),
// as (LOR, slice range) items spread over the lanes 32 at a time: g(id, t) for each. A LOR
// meets tens of slice ranges, in numbers that differ from lane to lane, so one LOR per
// lane would leave most lanes idle. Called by all 32 lanes of the warp.
template <bool kBand, typename G>
__device__ __forceinline__ void warp_slab_ids(const TorParams &p, const SegPlan &sp,
                                              signed char (&owner)[32], bool ok, int t,
                                              const SlabIdLor &c, G &&g) {
    const int lane = threadIdx.x & 31;
    const int cnt = ok ? c.k_hi - c.k_lo + 1 : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int excl = incl - cnt;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int base = 0; base < total; base += 32) {
        for (int i = max(excl, base); i < min(incl, base + 32); ++i)
            owner[i - base] = (signed char)lane;
        __syncwarp();
        const int item = base + lane;
        const bool valid = item < total;
        const int o = valid ? (int)owner[lane] : 0;
        __syncwarp();
        SlabIdLor m;
        m.k_lo = __shfl_sync(0xffffffffu, c.k_lo, o);
        const int k = m.k_lo + item - __shfl_sync(0xffffffffu, excl, o);
        const int to = __shfl_sync(0xffffffffu, t, o);
        if constexpr (kBand) {
            m.s_lo = __shfl_sync(0xffffffffu, c.s_lo, o);
            m.s_hi = __shfl_sync(0xffffffffu, c.s_hi, o);
            m.f0 = __shfl_sync(0xffffffffu, c.f0, o);
            m.lin = __shfl_sync(0xffffffffu, c.lin, o);
            m.y1 = __shfl_sync(0xffffffffu, c.y1, o);
            m.d1 = __shfl_sync(0xffffffffu, c.d1, o);
            m.r0 = __shfl_sync(0xffffffffu, c.r0, o);
            m.rs = __shfl_sync(0xffffffffu, c.rs, o);
            m.z1 = __shfl_sync(0xffffffffu, c.z1, o);
            m.dz = __shfl_sync(0xffffffffu, c.dz, o);
        }
        if (valid) range_slab_ids<kBand>(p, sp, m, k, [&](int id) { g(id, to); });
    }
}

// atomicAdd(&counter[id], 1) for the calling lane, with one shared-memory update per
// distinct id among the warp's active lanes (neighbouring LORs mostly share slabs). Returns
// the lane's slot: the counter's old value plus its rank among the lanes with that id.
__device__ __forceinline__ int warp_increment(int *counter, int id) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, id);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int first = 0;
    if (lane == leader) first = atomicAdd(counter + id, __popc(peers));
    first = __shfl_sync(active, first, leader);
    return first + __popc(peers & ((1u << lane) - 1u));
}

// Counting. Map calls over row-band slabs spread the (LOR, slice range) items of a warp
// over its lanes (warp_slab_ids): their LORs span the whole field of view (tens of ranges
// each, in numbers that differ between lanes, with a band computation per range), and
// generated LORs of another axis group drop out here, idling their lanes in a loop per
// lane (generated random pairs at 256 x 256 x 128: 239 against 264 ms per 50M, tensor
// pairs 217 against 220 ms). Elsewhere a loop per lane measured faster: 1.4 % on the
// 128 x 128 x 64 combined call, 4 % on the 128 x 128 x 64 map, where a range costs one
// shared add.
template <int OP, bool kBand>
__global__ void __launch_bounds__(kSegThreads) seg_count_kernel(const TorParams p, SegPlan sp) {
    extern __shared__ int hist[];  // [n_slabs]
    __shared__ signed char owner_tab[kSegThreads / 32][32];
    for (int k = threadIdx.x; k < sp.n_slabs; k += kSegThreads) hist[k] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSegTile;
    for (int it = 0; it < kSegItems; it++) {
        const int64_t t = base + (int64_t)it * kSegThreads + threadIdx.x;
        if (base + (int64_t)it * kSegThreads >= p.n) break;  // warp-uniform (whole block)
        int packed = -1;
        LorConst L;
        bool ok = false;
        SlabIdLor c{};
        if (t < p.n) {
            ok = geometry_any<OP>(p, t, L);  // generated map LORs are made here
            if (ok) {  // only LORs that enter the slab lists are ever read back
                const LorRec r = make_rec(L, ok);
                float4 *q = reinterpret_cast<float4 *>(sp.rec + t);
                q[0] = r.a;
                q[1] = r.b;
                q[2] = r.c;
                q[3] = r.d;
            }
            if (ok && OP == kBack) ok = (double)__ldg(p.values + t) > 1e-7;  // tor.cu.cc:203
            if (ok) {
                const int f0 = p.frame ? __ldg(p.frame + t) * sp.slabs_pf : 0;
                const int k_lo = f0 + L.s_lo / sp.nsl, k_hi = f0 + L.s_hi / sp.nsl;
                packed = k_lo | (k_hi << 16);
                c = slab_id_lor(p, sp, t, k_lo, k_hi, L.s_lo, L.s_hi, L.y1, L.z1, L.d1, L.dz);
            }
            sp.range[t] = packed;
        }
        if (OP == kMap && kBand) {
            warp_slab_ids<kBand>(p, sp, owner_tab[threadIdx.x >> 5], ok, (int)t, c,
                                 [&](int id, int) { atomicAdd(&hist[id], 1); });
        } else if (ok) {
            for (int k = c.k_lo; k <= c.k_hi; k++)
                range_slab_ids<kBand>(p, sp, c, k, [&](int id) { atomicAdd(&hist[id], 1); });
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < sp.n_slabs; k += kSegThreads)
        sp.tile_counts[(int64_t)blockIdx.x * sp.n_slabs + k] = hist[k];
}

// Per slab (one block each): exclusive scan of the tile counts -> tile_offs, slab total
// -> slab_tot[k]. A second single-warp kernel turns the totals into slab offsets.
__global__ void __launch_bounds__(1024) seg_scan_kernel(SegPlan sp, int64_t *slab_tot) {
    __shared__ int64_t warp_sums[32];
    const int k = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t carry = 0;
    for (int start = 0; start < sp.ntiles; start += 1024) {
        const int tile = start + threadIdx.x;
        const int64_t v = tile < sp.ntiles ? sp.tile_counts[(int64_t)tile * sp.n_slabs + k] : 0;
        int64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int64_t w = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const int64_t before = (wid ? warp_sums[wid - 1] : 0) + carry;
        if (tile < sp.ntiles) sp.tile_offs[(int64_t)tile * sp.n_slabs + k] = before + x - v;
        const int64_t chunk = warp_sums[31];
        __syncthreads();
        carry += chunk;
    }
    if (threadIdx.x == 0) slab_tot[k] = carry;
}

__global__ void seg_offsets_kernel(SegPlan sp, const int64_t *slab_tot) {
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (int k = 0; k < sp.n_slabs; k++) {
            sp.slab_offs[k] = acc;
            acc += slab_tot[k];
        }
        sp.slab_offs[sp.n_slabs] = acc;
    }
}

// Filling: one LOR per lane, so that the lanes of a warp that meet a slab append their
// LORs to its list side by side, in LOR order (warp_increment). The slab kernels hand a warp
// 32 consecutive entries of a list and walk the largest box among them: runs of
// neighbouring LORs (records are ordered by direction) keep those warps coherent. Spread
// over the lanes like the counting, the entries interleave and the slab kernels ran 4-8 %
// slower (measured).
template <bool kBand>
__global__ void __launch_bounds__(kSegThreads) seg_fill_kernel(const TorParams p, SegPlan sp) {
    extern __shared__ int64_t tile_base[];  // [n_slabs] where this tile's run of each slab starts
    int *cursor = reinterpret_cast<int *>(tile_base + sp.n_slabs);  // [n_slabs]
    for (int k = threadIdx.x; k < sp.n_slabs; k += kSegThreads) {
        cursor[k] = 0;
        tile_base[k] = sp.slab_offs[k] + sp.tile_offs[(int64_t)blockIdx.x * sp.n_slabs + k];
    }
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSegTile;
    for (int it = 0; it < kSegItems; it++) {
        const int64_t t = base + (int64_t)it * kSegThreads + threadIdx.x;
        if (t >= p.n) break;
        const int packed = sp.range[t];
        if (packed < 0) continue;
        const int k_lo = packed & 0xffff, k_hi = packed >> 16;
        int s_lo = 0, s_hi = p.gz - 1;
        float y1 = 0.f, z1 = 0.f, d1 = 0.f, dz = 1.f;
        if (kBand) {  // the values seg_count used, from the LOR's record
            const float4 *q = reinterpret_cast<const float4 *>(sp.rec + t);
            const float4 a = q[0], b = q[1], d = q[3];
            const int sl = __float_as_int(d.w);
            s_lo = sl & 0xffff;
            s_hi = sl >> 16;
            y1 = a.y;
            z1 = a.z;
            d1 = b.x;
            dz = b.y;
        }
        const SlabIdLor c = slab_id_lor(p, sp, t, k_lo, k_hi, s_lo, s_hi, y1, z1, d1, dz);
        for (int k = k_lo; k <= k_hi; k++)
            range_slab_ids<kBand>(p, sp, c, k, [&](int id) {
                const int pos = warp_increment(cursor, id);
                sp.seg[tile_base[id] + pos] = (int)t;
            });
    }
}

// Shared-memory slab layout. Every slice of the slab has pad = P - 1 zero rows and
// columns around it, so a window that meets the grid never leaves the slab: row iy,
// column ix of slab slice sl sits at origin + sl * ss + iy * rs + ix with rs = gx + pad
// (a row's right padding is the next row's left padding) and pad rows between slices
// (the bottom padding of one slice is the top padding of the next). The slice stride is
// rounded up to 5 (mod 32) floats so that a warp's lanes, often consecutive slices of
// one LOR at the same (row, column), fall into different banks.
__host__ __device__ __forceinline__ int slab_row_stride(int gx, int pad) { return gx + pad; }
__host__ __device__ __forceinline__ int slab_slice_stride(int gx, int gy, int pad) {
    const int dense = (gy + pad) * (gx + pad);
    return dense + ((5 - dense % 32) + 32) % 32;
}
__host__ __device__ __forceinline__ int slab_origin(int gx, int pad) {
    return pad * (gx + pad) + pad;
}
__host__ __device__ __forceinline__ int slab_floats(int nsl, int gx, int gy, int pad) {
    return nsl * slab_slice_stride(gx, gy, pad) + slab_origin(gx, pad);
}

// Persistent pass over the slab-major segment list (all TOR ops but the count). Scatter
// ops accumulate into the slab with shared atomics and flush once per slab; the
// projection gathers from the slab (loaded from the image) and adds each LOR's partial
// sum to its output.
// kExpand: the (LOR, slice) items of a warp's 32 segments are spread over its lanes, 32
// at a time (one item per lane, the LOR's constants read from its record); otherwise
// each lane walks its own segment's slices.
// kBand: the slabs are bands of rows (sp.nbands > 1), so rows are limited to the band.
template <int OP, int P, bool kExpand, bool kBand>
__global__ void __launch_bounds__(kSlabThreads, 1) tor_slab_kernel(const TorParams p, SegPlan sp) {
    extern __shared__ float slab[];
    __shared__ signed char owner_tab[kSlabThreads / 32][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kSlabThreads / 32;
    constexpr int pad = P - 1;
    const int rs = slab_row_stride(p.gx, pad), ss = slab_slice_stride(p.gx, sp.band_rows, pad);
    const int origin = slab_origin(p.gx, pad);
    const int64_t total = sp.slab_offs[sp.n_slabs];
    const int64_t g = blockIdx.x, G = gridDim.x;
    const int64_t lo = total * g / G, hi = total * (g + 1) / G;
    if (lo >= hi) return;
    if (OP == kProj) {
        // The padding columns stay zero: the slab loads below write grid voxels only.
        const int n = slab_floats(sp.nsl, p.gx, sp.band_rows, pad);
        for (int i = threadIdx.x; i < n; i += kSlabThreads) slab[i] = 0.0f;
        __syncthreads();
    }
    int k = 0;
    {
        int a = 0, b = sp.n_slabs - 1;
        while (a < b) {
            const int m = (a + b + 1) >> 1;
            if (sp.slab_offs[m] <= lo) a = m; else b = m - 1;
        }
        k = a;
    }
    int64_t pos = lo;
    while (pos < hi) {
        while (sp.slab_offs[k + 1] <= pos) k++;  // skip empty slabs
        const int64_t end = min(hi, sp.slab_offs[k + 1]);
        // slab id -> frame, slice range, row band
        const int per_frame = sp.slabs_pf * sp.nbands;
        const int fr = k / per_frame;
        const int kk = (k - fr * per_frame) / sp.nbands, band = k - fr * per_frame - kk * sp.nbands;
        const int S0 = kk * sp.nsl, S1 = min(S0 + sp.nsl, p.gz);
        const int R0 = band * sp.band_rows, R1 = min(R0 + sp.band_rows, p.gy);
        const int nbr = R1 - R0;
        const int64_t img0 = (int64_t)fr * p.frame_stride;
        const int n_rows = (S1 - S0) * nbr;
        if (OP == kProj) {
            const float *src = p.image_in + img0 + (int64_t)S0 * p.sz + (int64_t)R0 * p.sy;
            for (int r = warp; r < n_rows; r += kWarps) {
                const int sl = r / nbr, iy = r - sl * nbr;
                const float *g = src + (int64_t)sl * p.sz + (int64_t)iy * p.sy;
                float *d = slab + origin + sl * ss + iy * rs;
                for (int ix = lane; ix < p.gx; ix += 32) d[ix] = __ldg(g + (int64_t)ix * p.sx);
            }
        } else {
            const int n = slab_floats(S1 - S0, p.gx, sp.band_rows, pad);
            for (int i = threadIdx.x; i < n; i += kSlabThreads) slab[i] = 0.0f;
        }
        __syncthreads();
        for (int64_t q0 = pos + (int64_t)warp * 32; q0 < end; q0 += (int64_t)kWarps * 32) {
            const int64_t q = q0 + lane;
            LorConst L;
            int a = 0, cnt = 0, t = -1;
            if (q < end) {
                t = sp.seg[q];
                if (lor_load<OP>(p, sp.rec, t, L)) {
                    a = max(L.s_lo, S0);
                    cnt = max(0, min(L.s_hi, S1 - 1) - a + 1);
                }
            }
            if (!kExpand) {
                float acc = 0.0f;
                for (int i = 0; i < cnt; i++) {
                    const int s = a + i;
                    float *sb = slab + origin + (s - S0) * ss;  // slice s, row R0
                    if (OP == kProj) {
                        slice_visit<OP, P, true, kBand>(p, L, s, R0, R1,
                                                 [&](int ix, int iy, float w, bool use) {
                            const float v = sb[(iy - R0) * rs + ix];
                            acc = use ? fmaf(w, v, acc) : acc;
                        });
                    } else {
                        slice_visit<OP, P, true, kBand>(p, L, s, R0, R1,
                                                 [&](int ix, int iy, float w, bool use) {
                            if (use)
                                atomicAdd(&sb[(iy - R0) * rs + ix], OP == kBack ? w : w * L.scale);
                        });
                    }
                }
                if (OP == kProj && cnt > 0) atomicAdd(p.proj_out + t, acc * L.scale);
                continue;
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int excl = incl - cnt;
            const int n_items = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < n_items; base += 32) {
                for (int i = max(excl, base); i < min(incl, base + 32); ++i)
                    owner_tab[warp][i - base] = (signed char)lane;
                __syncwarp();
                const int item = base + lane;
                const bool valid = item < n_items;
                const int o = valid ? (int)owner_tab[warp][lane] : 0;
                __syncwarp();
                const int a_o = __shfl_sync(0xffffffffu, a, o);
                const int excl_o = __shfl_sync(0xffffffffu, excl, o);
                const int t_o = __shfl_sync(0xffffffffu, t, o);
                // the item's LOR from its record (the lanes of one LOR read the same 64
                // bytes, served once by L1), its value scale from the owning lane
                LorConst M;
                const float scale_o = __shfl_sync(0xffffffffu, L.scale, o);
                const float k0s_o = __shfl_sync(0xffffffffu, L.k0s, o);
                const bool all_o = OP == kMap && __shfl_sync(0xffffffffu, (int)L.all, o);
                if (valid) {
                    lor_rec_geometry(sp.rec, t_o, M);
                    M.scale = scale_o;
                    M.k0s = k0s_o;
                    M.all = all_o;
                    if (all_o) M.bxv = M.byv = 1.0e9f;
                }
                float partial = 0.0f;
                if (valid) {
                    const int s = a_o + (item - excl_o);
                    float *sb = slab + origin + (s - S0) * ss;  // slice s, row R0
                    if (OP == kProj) {
                        float acc = 0.0f;
                        slice_visit<OP, P, true, kBand>(p, M, s, R0, R1,
                                                 [&](int ix, int iy, float w, bool use) {
                            const float v = sb[(iy - R0) * rs + ix];
                            acc = use ? fmaf(w, v, acc) : acc;
                        });
                        partial = acc * M.scale;
                    } else {
                        slice_visit<OP, P, true, kBand>(p, M, s, R0, R1,
                                                 [&](int ix, int iy, float w, bool use) {
                            if (use)
                                atomicAdd(&sb[(iy - R0) * rs + ix], OP == kBack ? w : w * M.scale);
                        });
                    }
                }
                if (OP == kProj) {
                    // items of one LOR sit in consecutive lanes: segmented suffix sum
                    const int key = valid ? o : -1 - lane;
                    float v = partial;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const float nv = __shfl_down_sync(0xffffffffu, v, d);
                        const int nk = __shfl_down_sync(0xffffffffu, key, d);
                        if (lane + d < 32 && nk == key) v += nv;
                    }
                    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
                    if (valid && (lane == 0 || prev != key)) atomicAdd(p.proj_out + t_o, v);
                }
            }
        }
        __syncthreads();
        if (OP != kProj) {
            float *out = p.image_out + img0 + (int64_t)S0 * p.sz + (int64_t)R0 * p.sy;
            for (int r = warp; r < n_rows; r += kWarps) {
                const int sl = r / nbr, iy = r - sl * nbr;
                const float *src = slab + origin + sl * ss + iy * rs;
                float *g = out + (int64_t)sl * p.sz + (int64_t)iy * p.sy;
                for (int ix = lane; ix < p.gx; ix += 32) {
                    const float v = src[ix];
                    if (v != 0.0f) atomicAdd(g + (int64_t)ix * p.sx, v);
                }
            }
            __syncthreads();
        }
        pos = end;
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
    p.inv_x = 1.0f / p.inter_x;
    p.inv_y = 1.0f / p.inter_y;
    p.sx = 1;
    p.sy = gx;
    p.sz = (int64_t)gx * gy;
    // |dx|, |dy| <= patch * inter inside a window; the float d^2 of such a voxel is within
    // ~1e-6 (patch * inter)^2 of the exact value, the margin is 2^-16 (patch * inter)^2.
    const float span = (float)p.patch * std::max(p.inter_x, p.inter_y);
    p.box_e = span * span * (1.0f / 65536.0f);
    p.n = n;
    p.stride = lor_stride;
    // Kernel family: the shared-memory slab kernels unless tuning selects the LOR-centric
    // ones (gathers from L2, global atomics; also the fallback when a slice does not fit).
    const int path = g_tune_path.load(std::memory_order_relaxed);
    p.use_slab = path == 2 ? 0 : 1;
    p.slab_expand = path == 3 ? 1 : 0;
    return SRF_OK;
}

template <int OP, int P>
void launch_p(const TorParams &p, int grid, int block, cudaStream_t stream) {
    tor_kernel_p<OP, P><<<grid, block, 0, stream>>>(p);
    count_launches(1);
}

// Slab shape: slices per slab, slice ranges per frame, row bands and rows per band.
// Whole slices when at least kMinSlabSlices of them fit in shared memory (or the tuned
// count fits); otherwise bands of rows, as tall as fit for that many slices (fewer
// slices if not even kMinBandRows rows fit). False when nothing fits or there are too
// many slab ids (the LOR-centric kernels are used then).
constexpr int kMinSlabSlices = 4;
constexpr int kMinBandRows = 8;

bool slab_geometry(const TorParams &p, int pad, SegPlan &sp) {
    if (p.gx > (1 << 14) || p.gy > (1 << 14)) return false;
    const size_t budget = kSlabSmemBytes / sizeof(float);
    auto fits = [&](int n, int rows) {
        return (size_t)slab_floats(n, p.gx, rows, pad) <= budget;
    };
    int full = 0;
    while (full < p.gz && fits(full + 1, p.gy)) full++;
    const int want = g_tune_nsl.load(std::memory_order_relaxed);
    if ((want == 0 && full >= std::min(kMinSlabSlices, p.gz)) || (want > 0 && want <= full)) {
        sp.nsl = want > 0 ? want : full;
        sp.band_rows = p.gy;
    } else {
        int n = std::min(want > 0 ? want : kMinSlabSlices, p.gz);
        sp.band_rows = 0;
        for (; n >= 1; n--) {
            int rows = std::min(p.gy, (int)((budget / n) / (size_t)slab_row_stride(p.gx, pad)));
            while (rows > 0 && !fits(n, rows)) rows--;
            if (rows >= std::min(p.gy, kMinBandRows)) {
                sp.band_rows = rows;
                break;
            }
        }
        if (sp.band_rows == 0) return false;
        sp.nsl = n;
    }
    sp.nbands = (p.gy + sp.band_rows - 1) / sp.band_rows;
    // floor(r / d) = (r * ceil(2^32 / d)) >> 32 for r, d < 2^14 (error term r (m d - 2^32)
    // < 2^28 stays below 2^32); band_rows >= 2 whenever there is more than one band
    sp.band_magic = sp.band_rows >= 2
                        ? (unsigned)((((uint64_t)1 << 32) + (uint64_t)sp.band_rows - 1) /
                                     (uint64_t)sp.band_rows)
                        : 0u;
    sp.slabs_pf = (p.gz + sp.nsl - 1) / sp.nsl;
    sp.n_slabs = sp.slabs_pf * sp.nbands * std::max(1, p.n_frames);
    return sp.n_slabs <= kMaxSlabs && sp.slabs_pf * std::max(1, p.n_frames) < (1 << 16) &&
           p.n < (int64_t)INT32_MAX;
}

// CTAs per SM of the persistent slab kernels: the tuned multiplier, or automatically 2 for
// projection and back-projection launches of at least 4M LORs over whole-slice slabs
// (smaller shares even out the end of the launch: 5M-LOR calls on 128 x 64 slices measured
// 1.5 % faster, 4.5M-LOR batched calls on 96 x 48 slices 3 %) and 1 otherwise (0.5M-LOR
// calls measured 1.8 % slower with 2; with row bands each extra share reloads and flushes
// more slabs, 11 % slower on 256 x 128 slices; the map keeps 1).
constexpr int64_t kGridMult2MinLors = 4 << 20;

int slab_grid_mult(int op, const SegPlan &sp, int64_t lors_per_launch) {
    const int tuned = g_tune_mult.load(std::memory_order_relaxed);
    if (tuned > 0) return std::min(8, tuned);
    return (sp.nbands == 1 && (op == kProj || op == kBack) &&
            lors_per_launch >= kGridMult2MinLors) ? 2 : 1;
}

// Events [c0, c0 + n) of p as a call of their own (same images and outputs' layout).
TorParams lor_chunk(const TorParams &p, int64_t c0, int64_t n) {
    TorParams q = p;
    const int64_t o = c0 * p.stride;
    for (const float **c : {&q.x1, &q.y1, &q.z1, &q.x2, &q.y2, &q.z2, &q.xc, &q.yc, &q.zc, &q.f})
        if (*c) *c += o;
    if (q.values) q.values += c0;
    if (q.proj_out) q.proj_out += c0;
    if (q.frame) q.frame += c0;
    q.gen_first += c0;
    q.n = n;
    return q;
}

// The slab kernel instance for p's variant, with its shared-memory limit raised once per
// device.
template <int OP, int P>
int slab_kernel(const TorParams &p, bool band, void (**kern)(const TorParams, SegPlan)) {
    *kern = p.slab_expand
                ? (band ? tor_slab_kernel<OP, P, true, true> : tor_slab_kernel<OP, P, true, false>)
                : (band ? tor_slab_kernel<OP, P, false, true> : tor_slab_kernel<OP, P, false, false>);
    static std::atomic<unsigned long long> attr_set[4];  // per kernel instance, per device
    std::atomic<unsigned long long> &done = attr_set[(p.slab_expand ? 2 : 0) + (band ? 1 : 0)];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    if (!(done.load() & (1ull << dev))) {
        const cudaError_t e = cudaFuncSetAttribute(
            *kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSlabSmemBytes);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return SRF_ERR_CUDA;
        }
        done.fetch_or(1ull << dev);
    }
    return SRF_OK;
}

// One TOR op over the slab path; with OP2 >= 0 a second op (p2: the same LORs and
// geometry) runs on the same per-slab LOR lists right after the first, chunk by chunk
// (the projection's lists serve the back-projection: it drops LORs below its value
// threshold itself). Returns -1 when the slab path does not apply.
template <int OP, int P, int OP2>
int launch_slab(const TorParams &p, const TorParams *p2, cudaStream_t stream) {
    SegPlan sp{};
    if (!slab_geometry(p, P - 1, sp)) return -1;
    // The segment list is sized for the worst case (every LOR in every slab of its frame);
    // with each LOR's record and slab range, LORs are taken in chunks small enough that
    // this stays within the scratch budget (at least one 4096-LOR tile per chunk).
    const int64_t max_slabs_per_lor = (int64_t)sp.slabs_pf * sp.nbands;
    const size_t budget = (size_t)g_seg_scratch_bytes.load(std::memory_order_relaxed);
    int64_t chunk = (int64_t)(budget / (sizeof(int) * (size_t)max_slabs_per_lor +
                                        sizeof(LorRec) + sizeof(int)));
    chunk = std::max<int64_t>(kSegTile, chunk / kSegTile * kSegTile);
    chunk = std::min<int64_t>(chunk, p.n);
    sp.ntiles = (int)((chunk + kSegTile - 1) / kSegTile);
    // Scratch from the library's stream-ordered pool: no host synchronisation, capturable.
    const size_t cap = (size_t)chunk * (size_t)max_slabs_per_lor;
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t b_range = al(sizeof(int) * chunk);
    const size_t b_counts = al(sizeof(int) * (size_t)sp.ntiles * sp.n_slabs);
    const size_t b_offs = al(sizeof(int64_t) * (size_t)sp.ntiles * sp.n_slabs);
    const size_t b_slab = al(sizeof(int64_t) * (2 * sp.n_slabs + 1));
    const size_t b_seg = al(sizeof(int) * cap);
    const size_t b_rec = al(sizeof(LorRec) * chunk);
    char *ws = nullptr;
    cudaError_t e = scratch_alloc((void **)&ws,
                                  b_rec + b_range + b_counts + b_offs + b_slab + b_seg, stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    sp.rec = reinterpret_cast<LorRec *>(ws);
    char *w2 = ws + b_rec;
    sp.range = reinterpret_cast<int *>(w2);
    sp.tile_counts = reinterpret_cast<int *>(w2 + b_range);
    sp.tile_offs = reinterpret_cast<int64_t *>(w2 + b_range + b_counts);
    sp.slab_offs = reinterpret_cast<int64_t *>(w2 + b_range + b_counts + b_offs);
    sp.seg = reinterpret_cast<int *>(w2 + b_range + b_counts + b_offs + b_slab);

    const bool band = sp.nbands > 1;
    void (*kern)(const TorParams, SegPlan) = nullptr;
    void (*kern2)(const TorParams, SegPlan) = nullptr;
    int st = slab_kernel<OP, P>(p, band, &kern);
    if constexpr (OP2 >= 0) {
        if (st == SRF_OK) st = slab_kernel<OP2, P>(*p2, band, &kern2);
    }
    if (st != SRF_OK) {
        cudaFreeAsync(ws, stream);
        return st;
    }
    const size_t smem = sizeof(float) * (size_t)slab_floats(sp.nsl, p.gx, sp.band_rows, P - 1);
    int64_t *slab_tot = sp.slab_offs + sp.n_slabs + 1;
    if (OP == kProj) {
        e = cudaMemsetAsync(p.proj_out, 0, sizeof(float) * p.n, stream);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            cudaFreeAsync(ws, stream);
            return SRF_ERR_CUDA;
        }
    }
    const int mult = slab_grid_mult(OP, sp, chunk);
    const size_t hist_bytes = sizeof(int) * (size_t)sp.n_slabs;  // <= 16 KB (kMaxSlabs)
    const size_t fill_bytes = (sizeof(int64_t) + sizeof(int)) * (size_t)sp.n_slabs;  // <= 48 KB
    for (int64_t c0 = 0; c0 < p.n && st == SRF_OK; c0 += chunk) {
        const TorParams q = lor_chunk(p, c0, std::min(chunk, p.n - c0));
        SegPlan sq = sp;
        sq.ntiles = (int)((q.n + kSegTile - 1) / kSegTile);
        if (band)
            seg_count_kernel<OP, true><<<sq.ntiles, kSegThreads, hist_bytes, stream>>>(q, sq);
        else
            seg_count_kernel<OP, false><<<sq.ntiles, kSegThreads, hist_bytes, stream>>>(q, sq);
        seg_scan_kernel<<<sq.n_slabs, 1024, 0, stream>>>(sq, slab_tot);
        seg_offsets_kernel<<<1, 32, 0, stream>>>(sq, slab_tot);
        if (band)
            seg_fill_kernel<true><<<sq.ntiles, kSegThreads, fill_bytes, stream>>>(q, sq);
        else
            seg_fill_kernel<false><<<sq.ntiles, kSegThreads, fill_bytes, stream>>>(q, sq);
        kern<<<num_sms() * mult, kSlabThreads, smem, stream>>>(q, sq);
        count_launches(5);
        if constexpr (OP2 >= 0) {
            kern2<<<num_sms() * mult, kSlabThreads, smem, stream>>>(
                lor_chunk(*p2, c0, std::min(chunk, p.n - c0)), sq);
            count_launches(1);
        }
        st = check_launch();
    }
    e = cudaFreeAsync(ws, stream);
    if (st == SRF_OK && e != cudaSuccess) {
        set_cuda_error(e);
        st = SRF_ERR_CUDA;
    }
    return st;
}

template <int OP>
int tor_launch(TorParams &p, cudaStream_t stream, bool generic = false) {
    if (p.n == 0) return SRF_OK;
    if ((OP == kProj || OP == kBack || OP == kMap || OP == kAdj) && !generic && p.use_slab) {
        int st = -1;
        switch (p.patch) {
            case 2: st = launch_slab<OP, 2, -1>(p, nullptr, stream); break;
            case 3: st = launch_slab<OP, 3, -1>(p, nullptr, stream); break;
            case 4: st = launch_slab<OP, 4, -1>(p, nullptr, stream); break;
            case 5: st = launch_slab<OP, 5, -1>(p, nullptr, stream); break;
            case 6: st = launch_slab<OP, 6, -1>(p, nullptr, stream); break;
            case 7: st = launch_slab<OP, 7, -1>(p, nullptr, stream); break;
            case 8: st = launch_slab<OP, 8, -1>(p, nullptr, stream); break;
            default: break;
        }
        if (st >= 0) return st;
    }
    const int block = 256;
    const int grid = stride_grid(p.n, block / 32, 8);
    switch (generic ? 0 : p.patch) {
        case 2: launch_p<OP, 2>(p, grid, block, stream); break;
        case 3: launch_p<OP, 3>(p, grid, block, stream); break;
        case 4: launch_p<OP, 4>(p, grid, block, stream); break;
        case 5: launch_p<OP, 5>(p, grid, block, stream); break;
        case 6: launch_p<OP, 6>(p, grid, block, stream); break;
        case 7: launch_p<OP, 7>(p, grid, block, stream); break;
        case 8: launch_p<OP, 8>(p, grid, block, stream); break;
        default:
            tor_kernel<OP><<<grid, block, 0, stream>>>(p);
            count_launches(1);
            break;
    }
    return check_launch();
}

// Projection pp then back-projection pb of its values (same LORs, geometry and tuning):
// on the slab path both ops share one set of per-slab LOR lists.
int tor_launch_pair(TorParams &pp, TorParams &pb, cudaStream_t stream) {
    if (pp.n == 0) return SRF_OK;
    int st = -1;
    if (pp.use_slab) {
        switch (pp.patch) {
            case 2: st = launch_slab<kProj, 2, kBack>(pp, &pb, stream); break;
            case 3: st = launch_slab<kProj, 3, kBack>(pp, &pb, stream); break;
            case 4: st = launch_slab<kProj, 4, kBack>(pp, &pb, stream); break;
            case 5: st = launch_slab<kProj, 5, kBack>(pp, &pb, stream); break;
            case 6: st = launch_slab<kProj, 6, kBack>(pp, &pb, stream); break;
            case 7: st = launch_slab<kProj, 7, kBack>(pp, &pb, stream); break;
            case 8: st = launch_slab<kProj, 8, kBack>(pp, &pb, stream); break;
            default: break;
        }
    }
    if (st >= 0) return st;
    st = tor_launch<kProj>(pp, stream);
    return st == SRF_OK ? tor_launch<kBack>(pb, stream) : st;
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

extern "C" int srf_tor_projection_backprojection(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, float *projection_value, const int *grid,
    const float *center, const float *size, float kernel_width, float tof_bin, float tof_sigma2,
    const float *image, float *back_image, int64_t num_events, int64_t lor_stride,
    int accumulate, void *stream) {
    TorParams pp{};
    int st = tor_setup(pp, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if (!back_image || back_image == image) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value, image}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && pp.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_image(back_image, grid, (cudaStream_t)stream)) != SRF_OK)
        return st;
    pp.x1 = x1; pp.y1 = y1; pp.z1 = z1; pp.x2 = x2; pp.y2 = y2; pp.z2 = z2;
    pp.xc = xc; pp.yc = yc; pp.zc = zc; pp.f = sigma2_factor;
    pp.geo = geo_sigma2_flag != 0;
    TorParams pb = pp;
    pp.image_in = image;
    pp.proj_out = projection_value;
    pb.values = projection_value;
    pb.image_out = back_image;
    return tor_launch_pair(pp, pb, (cudaStream_t)stream);
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

extern "C" int srf_tor_maplors_generated(int kind, const float *crystals, int n_rings,
                                         int n_blocks, int n_per_block,
                                         unsigned long long seed, int64_t first,
                                         int64_t count, int axis, int geo_sigma2_flag,
                                         const int *grid, const float *center,
                                         const float *size, float kernel_width, float *image,
                                         int accumulate, void *stream) {
    if (kind != 0 && kind != 1) return SRF_ERR_INVALID_ARGUMENT;
    if (axis < 0 || axis > 2 || first < 0 || count < 0) return SRF_ERR_INVALID_ARGUMENT;
    if (n_rings < 1 || n_blocks < 1 || n_per_block < 1) return SRF_ERR_INVALID_ARGUMENT;
    const int64_t n_cry = (int64_t)n_rings * n_blocks * n_per_block;
    if (n_cry < 2 || n_cry > ((int64_t)1 << 31) - 1) return SRF_ERR_INVALID_ARGUMENT;
    if (kind == 0 && n_blocks != 1) return SRF_ERR_INVALID_ARGUMENT;  // rings of crystals
    if (kind == 1) {
        if (n_blocks < 2) return SRF_ERR_INVALID_ARGUMENT;
        const double cb = (double)n_per_block * n_per_block;
        const double total = (double)n_rings * ((double)(n_rings - 1) * n_blocks *
                                                (n_blocks - 1) * cb +
                                                (double)n_blocks * (n_blocks - 1) / 2 * cb);
        if ((double)first + (double)count > total) return SRF_ERR_INVALID_ARGUMENT;
    }
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, 0.0f, 1.0e30f, count, 1);
    if (st != SRF_OK) return st;
    if (!image || (count > 0 && !crystals)) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate && (st = zero_image(image, grid, (cudaStream_t)stream)) != SRF_OK) return st;
    p.geo = geo_sigma2_flag != 0;
    p.values = nullptr;  // every LOR's value is 1
    p.image_out = image;
    p.gen = kind + 1;
    p.gen_axis = axis;
    p.gen_first = first;
    p.gen_seed = seed;
    p.crystals = crystals;
    p.n_rings = n_rings;
    p.n_blocks = n_blocks;
    p.n_per_block = n_per_block;
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

// ------------------------------------------------------------------ batched frames
// No counterpart in the reference: many independent reconstructions sharing one
// geometry in one launch. LOR i belongs to frame frame[i] in [0, n_frames); the images
// are n_frames consecutive blocks of frame_stride floats (frame_stride >= voxels).

namespace {
int set_frames(TorParams &p, const int *frame, int n_frames, int64_t frame_stride) {
    const int64_t nvox = (int64_t)p.gx * p.gy * p.gz;
    if (n_frames < 1 || (p.n > 0 && !frame) || frame_stride < nvox) return SRF_ERR_INVALID_ARGUMENT;
    if ((int64_t)n_frames * frame_stride > ((int64_t)1 << 40)) return SRF_ERR_UNSUPPORTED;
    p.frame = frame;
    p.n_frames = n_frames;
    p.frame_stride = frame_stride;
    return SRF_OK;
}

int zero_frames(float *image, int n_frames, int64_t frame_stride, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(image, 0, sizeof(float) * (size_t)n_frames * frame_stride,
                                    stream);
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return SRF_ERR_CUDA;
    }
    return SRF_OK;
}
}  // namespace

extern "C" int srf_tor_projection_batched(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, const float *images,
    int64_t num_events, int64_t lor_stride, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if ((st = set_frames(p, frame, n_frames, frame_stride)) != SRF_OK) return st;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value, images}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && p.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.xc = xc; p.yc = yc; p.zc = zc; p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.image_in = images;
    p.proj_out = projection_value;
    return tor_launch<kProj>(p, (cudaStream_t)stream);
}

namespace {
template <int OP>
int scatter_batched(const float *x1, const float *y1, const float *z1, const float *x2,
                    const float *y2, const float *z2, const float *xc, const float *yc,
                    const float *zc, const float *sigma2_factor, int geo_sigma2_flag,
                    const int *frame, int n_frames, int64_t frame_stride, const float *values,
                    const int *grid, const float *center, const float *size, float kernel_width,
                    float tof_bin, float tof_sigma2, float *images, int64_t num_events,
                    int64_t lor_stride, int accumulate, void *stream) {
    TorParams p{};
    int st = tor_setup(p, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if ((st = set_frames(p, frame, n_frames, frame_stride)) != SRF_OK) return st;
    if (!images) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, values}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && p.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate &&
        (st = zero_frames(images, n_frames, frame_stride, (cudaStream_t)stream)) != SRF_OK)
        return st;
    p.x1 = x1; p.y1 = y1; p.z1 = z1; p.x2 = x2; p.y2 = y2; p.z2 = z2;
    p.xc = xc; p.yc = yc; p.zc = zc; p.f = sigma2_factor;
    p.geo = geo_sigma2_flag != 0;
    p.values = values;
    p.image_out = images;
    return tor_launch<OP>(p, (cudaStream_t)stream);
}
}  // namespace

extern "C" int srf_tor_backprojection_batched(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, const float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, float *images,
    int64_t num_events, int64_t lor_stride, int accumulate, void *stream) {
    return scatter_batched<kBack>(x1, y1, z1, x2, y2, z2, xc, yc, zc, sigma2_factor,
                                  geo_sigma2_flag, frame, n_frames, frame_stride,
                                  projection_value, grid, center, size, kernel_width, tof_bin,
                                  tof_sigma2, images, num_events, lor_stride, accumulate,
                                  stream);
}

extern "C" int srf_tor_projection_backprojection_batched(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, const float *images,
    float *back_images, int64_t num_events, int64_t lor_stride, int accumulate, void *stream) {
    TorParams pp{};
    int st = tor_setup(pp, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if ((st = set_frames(pp, frame, n_frames, frame_stride)) != SRF_OK) return st;
    if (!back_images || back_images == images) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value, images}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && pp.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate &&
        (st = zero_frames(back_images, n_frames, frame_stride, (cudaStream_t)stream)) != SRF_OK)
        return st;
    pp.x1 = x1; pp.y1 = y1; pp.z1 = z1; pp.x2 = x2; pp.y2 = y2; pp.z2 = z2;
    pp.xc = xc; pp.yc = yc; pp.zc = zc; pp.f = sigma2_factor;
    pp.geo = geo_sigma2_flag != 0;
    TorParams pb = pp;
    pp.image_in = images;
    pp.proj_out = projection_value;
    pb.values = projection_value;
    pb.image_out = back_images;
    return tor_launch_pair(pp, pb, (cudaStream_t)stream);
}

// srf_tor_projection_backprojection_batched on image stacks in any axis order: voxel
// (ix, iy, iz) of frame f (kernel axes) is at f * frame_stride + ix image_strides[0] +
// iy image_strides[1] + iz image_strides[2] of both images and back_images, e.g. a
// permuted view of an [F, nx, ny, nz] stack, which then needs no copy into the kernel
// layout and back.
extern "C" int srf_tor_projection_backprojection_batched_strided(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, const float *images,
    float *back_images, const int64_t *image_strides, int64_t num_events, int64_t lor_stride,
    int accumulate, void *stream) {
    TorParams pp{};
    int st = tor_setup(pp, grid, center, size, kernel_width, tof_bin, tof_sigma2, num_events,
                       lor_stride);
    if (st != SRF_OK) return st;
    if ((st = set_frames(pp, frame, n_frames, frame_stride)) != SRF_OK) return st;
    if (!image_strides) return SRF_ERR_INVALID_ARGUMENT;
    const int64_t sx = image_strides[0], sy = image_strides[1], sz = image_strides[2];
    if (sx < 1 || sy < 1 || sz < 1) return SRF_ERR_INVALID_ARGUMENT;
    // a frame's voxels stay inside its frame_stride floats (and the offsets inside int64)
    const int64_t lim = (int64_t)1 << 40;
    if (sx > lim || sy > lim || sz > lim) return SRF_ERR_UNSUPPORTED;
    if ((int64_t)(pp.gx - 1) * sx + (int64_t)(pp.gy - 1) * sy + (int64_t)(pp.gz - 1) * sz >=
        frame_stride)
        return SRF_ERR_INVALID_ARGUMENT;
    if (!back_images || back_images == images) return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 &&
        !cols_ok({x1, y1, z1, x2, y2, z2, sigma2_factor, projection_value, images}))
        return SRF_ERR_INVALID_ARGUMENT;
    if (num_events > 0 && pp.tof_on && !cols_ok({xc, yc, zc})) return SRF_ERR_INVALID_ARGUMENT;
    if (!accumulate &&
        (st = zero_frames(back_images, n_frames, frame_stride, (cudaStream_t)stream)) != SRF_OK)
        return st;
    pp.x1 = x1; pp.y1 = y1; pp.z1 = z1; pp.x2 = x2; pp.y2 = y2; pp.z2 = z2;
    pp.xc = xc; pp.yc = yc; pp.zc = zc; pp.f = sigma2_factor;
    pp.geo = geo_sigma2_flag != 0;
    pp.sx = sx;
    pp.sy = sy;
    pp.sz = sz;
    TorParams pb = pp;
    pp.image_in = images;
    pp.proj_out = projection_value;
    pb.values = projection_value;
    pb.image_out = back_images;
    return tor_launch_pair(pp, pb, (cudaStream_t)stream);
}

extern "C" int srf_tor_backproject_adjoint_batched(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, const float *values, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, float *images,
    int64_t num_events, int64_t lor_stride, int accumulate, void *stream) {
    return scatter_batched<kAdj>(x1, y1, z1, x2, y2, z2, xc, yc, zc, sigma2_factor,
                                 geo_sigma2_flag, frame, n_frames, frame_stride, values, grid,
                                 center, size, kernel_width, tof_bin, tof_sigma2, images,
                                 num_events, lor_stride, accumulate, stream);
}

// No counterpart in the reference: process-wide kernel tuning for the TOR ops, used by
// the autotuner. path: 0 automatic (slab kernels when a slice fits in shared memory),
// 1 slab kernels, 2 LOR-centric kernels; slab_slices: slices per shared-memory slab
// (0 = as many as fit); grid_mult: persistent slab CTAs = SMs x grid_mult (1..8, 0 =
// automatic).
extern "C" int srf_tor_set_scratch_limit(int64_t bytes) {
    if (bytes < 0) return SRF_ERR_INVALID_ARGUMENT;
    g_seg_scratch_bytes.store(bytes == 0 ? kSegScratchDefault : (long long)bytes);
    return SRF_OK;
}

extern "C" int srf_tor_set_tuning(int path, int slab_slices, int grid_mult) {
    if (path < 0 || path > 3 || slab_slices < 0 || grid_mult < 0 || grid_mult > 8)
        return SRF_ERR_INVALID_ARGUMENT;
    g_tune_path.store(path);
    g_tune_nsl.store(slab_slices);
    g_tune_mult.store(grid_mult);
    return SRF_OK;
}

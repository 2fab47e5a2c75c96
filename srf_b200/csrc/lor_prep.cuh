// Per-event arithmetic of the reference's host preprocessing
// (src/python/srf/preprocess/function/on_tor_lors.py: recon_process :251-262, map_process
// :243-248), shared by the preprocessing kernels (preprocess.cu) and the TOR map kernels
// that make their LORs on the fly (tor.cu). Float32 in numpy's operation order: numpy never
// fuses a*b+c, so every product and sum is a separately rounded __fmul_rn / __fadd_rn.
#pragma once

#include <cuda_runtime.h>

namespace srf {

constexpr int kBuckets = 6;

struct Rec {
    float v[10];
    int bucket;  // 0..5, or 6 when no axis is dominant (NaN input)
};

__device__ __forceinline__ float sq(float a) { return __fmul_rn(a, a); }

__device__ __forceinline__ float pick(const float *a, int k) {
    return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]);
}

// The dominant axis of an event (dominentBy, :70-77): 0 x, 1 y, 2 z, -1 none (NaN).
__device__ __forceinline__ int dominant_axis(const float *e) {
    const float ax = fabsf(__fsub_rn(e[3], e[0])), ay = fabsf(__fsub_rn(e[4], e[1]));
    const float az = fabsf(__fsub_rn(e[5], e[2]));
    if (ax >= ay && ax >= az) return 0;
    if (ay > ax && ay >= az) return 1;
    if (az > ax && az > ay) return 2;
    return -1;
}

// One event -> its bucket and output record. RECON selects recon_process (10
// columns out) vs map_process (7 columns out).
template <bool RECON>
__device__ __forceinline__ Rec process(const float *e, bool cut, float limit) {
    constexpr bool recon = RECON;
    Rec r;
    const float x1 = e[0], y1 = e[1], z1 = e[2], x2 = e[3], y2 = e[4], z2 = e[5];
    const float t = recon ? e[6] : 0.0f;
    const float dx = __fsub_rn(x2, x1), dy = __fsub_rn(y2, y1), dz = __fsub_rn(z2, z1);
    // sigma2_factor
    const float p_dis2 = __fadd_rn(__fadd_rn(sq(dx), sq(dy)), sq(dz));
    const float dsq = __fadd_rn(sq(dx), sq(dy));
    const float rsq = __fadd_rn(__fadd_rn(__fadd_rn(sq(x1), sq(x2)), sq(y1)), sq(y2));
    const float f = __fdiv_rn(__fdiv_rn(__fdiv_rn(sq(dsq), rsq), p_dis2), 2.0f);
    // dominant axis (dominentBy)
    const int axis = dominant_axis(e);
    if (axis < 0) {
        r.bucket = kBuckets;
        return r;
    }
    const float d = axis == 0 ? dx : (axis == 1 ? dy : dz);  // SwapPointsOrder's test
    const bool swap = !(d >= 0.0f);
    r.bucket = axis * 2 + (swap ? 1 : 0);
    float p1[3] = {x1, y1, z1}, p2[3] = {x2, y2, z2};
    float tt = t;
    if (swap) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float s = p1[k];
            p1[k] = p2[k];
            p2[k] = s;
        }
        tt = __fsub_rn(0.0f, t);
    }
    float c[3] = {0.f, 0.f, 0.f};
    if (recon) {
        // CutLoRs
        float pd[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pd[k] = __fsub_rn(p2[k], p1[k]);
        const float p_dis = __fsqrt_rn(__fadd_rn(__fadd_rn(sq(pd[0]), sq(pd[1])), sq(pd[2])));
        float dc[3];
#pragma unroll
        for (int k = 0; k < 3; k++) dc[k] = __fdiv_rn(pd[k], p_dis);
        const float ratio = __fsub_rn(0.5f, __fdiv_rn(tt, p_dis));
#pragma unroll
        for (int k = 0; k < 3; k++) c[k] = __fadd_rn(__fmul_rn(ratio, pd[k]), p1[k]);
        const float dcs = __fsqrt_rn(__fadd_rn(
            __fadd_rn(sq(__fsub_rn(c[0], p1[0])), sq(__fsub_rn(c[1], p1[1]))),
            sq(__fsub_rn(c[2], p1[2]))));
        if (cut && dcs > limit) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const float m = __fmul_rn(limit, dc[k]);
                p1[k] = __fsub_rn(c[k], m);
                p2[k] = __fadd_rn(c[k], m);
            }
        }
    }
    // permutation: dominant axis last
    const int a0 = axis == 0 ? 1 : 0;
    const int a1 = axis == 2 ? 1 : 2;
    const int a2 = axis;
    r.v[0] = pick(p1, a0);
    r.v[1] = pick(p1, a1);
    r.v[2] = pick(p1, a2);
    r.v[3] = pick(p2, a0);
    r.v[4] = pick(p2, a1);
    r.v[5] = pick(p2, a2);
    if (recon) {
        r.v[6] = pick(c, a0);
        r.v[7] = pick(c, a1);
        r.v[8] = pick(c, a2);
        r.v[9] = f;
    } else {
        r.v[6] = f;
    }
    return r;
}

}  // namespace srf

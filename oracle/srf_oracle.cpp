// SRF listmode projector ORACLE — CPU restatement of the reference projectors.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the shipped library calls this code; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it, and only
// as the checker.
//
// What it restates (reference paths relative to the SRF project root):
//   TOR   : src/cpp/tf_custom_ops/tor.cu.cc    (host set-up :348-481, device math :22-346)
//   Siddon: src/cpp/tf_custom_ops/siddon.cu.cc (host set-up :583-675, device math :61-575)
//
// Two arithmetic modes:
//   * f32 mode  reproduces the reference's float arithmetic operation by operation,
//               including the places where the reference promotes to double (double
//               literals feeding exp/sqrt, tor.cu.cc:71,90; siddon.cu.cc:311-316,460).
//               `contract` selects how a*b+c is rounded: 1 = one rounding (fused
//               multiply-add, what nvcc emits for device code by default), 0 = two
//               roundings (the host compiler without FMA, i.e. the reference compiled
//               for the CPU through oracle/shim). With contract = 0 the f32 mode is
//               bit-identical to the reference compiled for the host; that pins it.
//   * f64 mode  the reference's operator evaluated exactly: every discrete choice the
//               reference makes in float is taken from the f32 path (with nvcc's
//               contraction) — for TOR which slices a LOR crosses (tor.cu.cc:30-33),
//               where the patch window starts (:135-136) and the 3-sigma cut-off test
//               (:71); for Siddon the voxel sequence of the walk (:302-330) and the
//               TOF 3-sigma test (:314) — while every weight, length and sum is
//               evaluated in double. The f64-vs-f32 difference is therefore pure
//               floating-point error of the values, not a different discretisation.
//
// Loop orders follow the reference so that float sums round identically: TOR
// projection per LOR over slices in ascending order (the host slice loop at
// tor.cu.cc:377 accumulates into projection_value[tid]); TOR back-projection and
// map slice-outer, LOR-inner (tor.cu.cc:420, :468); Siddon per LOR (siddon.cu.cc:443).
//
// LOR input layout: the reference's SoA layout, one contiguous column per field
// ([10,N] for TOR: x1,y1,z1,x2,y2,z2,xc,yc,zc,sigma2_factor; [7,N] for TOR map:
// x1..z2,sigma2_factor; [7,N] for Siddon: x1..z2,tof).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

constexpr float kTofThreshold = 405758.0f;  // tor.cu.cc:20, siddon.cu.cc:15

inline float madd(float a, float b, float c, bool contract) {
    // Built with -ffp-contract=off: the non-fused branch really rounds twice.
    return contract ? std::fmaf(a, b, c) : (a * b) + c;
}

// ---------------------------------------------------------------------------
// TOR
// ---------------------------------------------------------------------------

struct TorGeom {
    int gx, gy, gz;
    float cz, lz, inter_x, inter_y, inter_z, l_bound, b_bound, tor_sigma2;
    int patch;
    double d_inter_x, d_inter_y, d_inter_z, d_l_bound, d_b_bound, d_tor_sigma2, d_cz, d_lz;
};

// Host-side set-up of tor.cu.cc:364-375 (identical in the three launchers).
TorGeom tor_geom(const int *grid, const float *center, const float *size, float kernel_width) {
    TorGeom g;
    unsigned int gx = grid[0], gy = grid[1], gz = grid[2];
    float lx = size[0], ly = size[1], lz = size[2];
    g.gx = (int)gx;
    g.gy = (int)gy;
    g.gz = (int)gz;
    g.cz = center[2];
    g.lz = lz;
    g.inter_x = lx / gx;
    g.inter_y = ly / gy;
    g.inter_z = lz / gz;
    g.l_bound = center[0] - lx / 2;
    g.b_bound = center[1] - ly / 2;
    g.tor_sigma2 = kernel_width * kernel_width / 36;
    g.patch = (int)std::ceil((std::sqrt(2.0) * kernel_width + g.inter_z) / g.inter_x);
    g.d_inter_x = (double)lx / gx;
    g.d_inter_y = (double)ly / gy;
    g.d_inter_z = (double)lz / gz;
    g.d_l_bound = (double)center[0] - (double)lx / 2;
    g.d_b_bound = (double)center[1] - (double)ly / 2;
    g.d_tor_sigma2 = (double)kernel_width * kernel_width / 36;
    g.d_cz = center[2];
    g.d_lz = lz;
    return g;
}

// slice_z of the projection launcher (tor.cu.cc:380): all float.
inline float tor_slice_z_proj(const TorGeom &g, unsigned int s) {
    return g.cz - (g.lz - g.inter_z) / 2 + s * g.inter_z;
}
// slice_z of the back-projection and map launchers (tor.cu.cc:423, :471): the
// `/ 2.0` makes the first difference double before the result is stored as float.
inline float tor_slice_z_back(const TorGeom &g, unsigned int s) {
    return (float)(g.cz - (double)(g.lz - g.inter_z) / 2.0 + (double)(s * g.inter_z));
}
inline double tor_slice_z_f64(const TorGeom &g, unsigned int s) {
    return g.d_cz - (g.d_lz - g.d_inter_z) / 2.0 + s * g.d_inter_z;
}

struct TorCross {
    bool valid;
    float cross_x, cross_y, dcos_x, dcos_y;
};

// CalculateCrossPoint, tor.cu.cc:22-48.
inline TorCross tor_cross(float x1, float y1, float z1, float x2, float y2, float z2, float slice_z,
                          bool c) {
    TorCross r;
    float d0 = x2 - x1, d1 = y2 - y1, d2 = z2 - z1;
    float ratio = (slice_z - z1) / d2;
    r.valid = ratio > 0.0 && ratio < 1.0;
    r.cross_x = madd(d0, ratio, x1, c);
    r.cross_y = madd(d1, ratio, y1, c);
    float dis = std::sqrt(madd(d2, d2, madd(d0, d0, d1 * d1, c), c));
    r.dcos_x = d0 / dis;
    r.dcos_y = d1 / dis;
    return r;
}

struct TorCrossD {
    double cross_x, cross_y, dcos_x, dcos_y;
};

inline TorCrossD tor_cross_f64(float x1, float y1, float z1, float x2, float y2, float z2,
                               double slice_z) {
    TorCrossD r;
    double d0 = (double)x2 - x1, d1 = (double)y2 - y1, d2 = (double)z2 - z1;
    double ratio = (slice_z - z1) / d2;
    r.cross_x = x1 + d0 * ratio;
    r.cross_y = y1 + d1 * ratio;
    double dis = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    r.dcos_x = d0 / dis;
    r.dcos_y = d1 / dis;
    return r;
}

// Perpendicular squared distance of a mesh point to the LOR, float arithmetic of
// tor.cu.cc:57-61 (and the identical MapSMV lines :100-103).
inline float tor_d2_f32(float cross_x, float cross_y, float mesh_x, float mesh_y, float ux, float uy,
                        bool c) {
    float dx = cross_x - mesh_x;
    float dy = cross_y - mesh_y;
    float r_cos = madd(dx, ux, dy * uy, c);
    return madd(-r_cos, r_cos, madd(dx, dx, dy * dy, c), c);
}

// CalculateSMV, tor.cu.cc:50-92, float mode.
inline float tor_smv_f32(float xc, float yc, float zc, float f, bool geo, float slice_z,
                         float tof_bin, float tof_sigma2, float cross_x, float cross_y,
                         float mesh_x, float mesh_y, float ux, float uy, float tor_sigma2,
                         bool c) {
    float d2 = tor_d2_f32(cross_x, cross_y, mesh_x, mesh_y, ux, uy, c);
    float tsc = geo ? tor_sigma2 * f : tor_sigma2;
    float value = ((double)d2 < 9.0 * (double)tsc)
                      ? (float)std::exp(-0.5 * (double)d2 / (double)tsc)
                      : 0.0f;
    if (tof_sigma2 < kTofThreshold) {
        float ax = xc - cross_x, ay = yc - cross_y, az = zc - slice_z;
        float d2_tof = madd(az, az, madd(ax, ax, ay * ay, c), c) - d2;
        float tse = tof_sigma2 + (tof_bin * tof_bin) / 12;
        float t2 = d2_tof / tse;
        value = (float)((double)value * ((double)tof_bin * std::exp(-0.5 * (double)t2) /
                                         std::sqrt(2.0 * M_PI * (double)tof_sigma2)));
    }
    return value;
}

// MapSMV, tor.cu.cc:94-122, float mode.
inline float tor_map_smv_f32(float f, bool geo, float cross_x, float cross_y, float mesh_x,
                             float mesh_y, float ux, float uy, float tor_sigma2, bool c) {
    float d2 = tor_d2_f32(cross_x, cross_y, mesh_x, mesh_y, ux, uy, c);
    float tsc = geo ? tor_sigma2 * f : tor_sigma2;
    return ((double)d2 < 9.0 * (double)tsc) ? (float)std::exp(-0.5 * (double)d2 / (double)tsc)
                                            : 0.0f;
}

// Same weights in double.
// `inside` is the reference's float cut-off decision for this voxel.
inline double tor_smv_f64(double xc, double yc, double zc, double f, bool geo, double slice_z,
                          double tof_bin, double tof_sigma2, bool tof_on, double cross_x,
                          double cross_y, double mesh_x, double mesh_y, double ux, double uy,
                          double tor_sigma2, bool with_tof, bool inside) {
    double dx = cross_x - mesh_x, dy = cross_y - mesh_y;
    double r_cos = dx * ux + dy * uy;
    double d2 = dx * dx + dy * dy - r_cos * r_cos;
    double tsc = geo ? tor_sigma2 * f : tor_sigma2;
    double value = inside ? std::exp(-0.5 * d2 / tsc) : 0.0;
    if (with_tof && tof_on) {
        double ax = xc - cross_x, ay = yc - cross_y, az = zc - slice_z;
        double d2_tof = ax * ax + ay * ay + az * az - d2;
        double tse = tof_sigma2 + tof_bin * tof_bin / 12.0;
        value *= tof_bin * std::exp(-0.5 * d2_tof / tse) / std::sqrt(2.0 * M_PI * tof_sigma2);
    }
    return value;
}

struct TorLor {
    float x1, y1, z1, x2, y2, z2, xc, yc, zc, f;
};

inline TorLor tor_lor(const float *lors, int64_t n, int64_t i, bool with_center) {
    TorLor l;
    l.x1 = lors[0 * n + i];
    l.y1 = lors[1 * n + i];
    l.z1 = lors[2 * n + i];
    l.x2 = lors[3 * n + i];
    l.y2 = lors[4 * n + i];
    l.z2 = lors[5 * n + i];
    if (with_center) {
        l.xc = lors[6 * n + i];
        l.yc = lors[7 * n + i];
        l.zc = lors[8 * n + i];
        l.f = lors[9 * n + i];
    } else {  // Maplors layout [7,N]: x1..z2, sigma2_factor (tor.cc:310-321)
        l.xc = l.yc = l.zc = 0.0f;
        l.f = lors[6 * n + i];
    }
    return l;
}

// Visit the patch window of one (LOR, slice) exactly as LoopPatch / BackLoopPatch /
// MapLoopPatch do (tor.cu.cc:135-165, :180-208, :220-241): j outer, i inner, skipping
// out-of-slice indices. `cb(index, index0, index1)` is called for each visited voxel.
template <typename F>
inline void tor_visit_patch(const TorGeom &g, float cross_x, float cross_y, F &&cb) {
    int index_x = (int)((cross_x - g.l_bound) / g.inter_x) - (int)((unsigned)g.patch / 2);
    int index_y = (int)((cross_y - g.b_bound) / g.inter_y) - (int)((unsigned)g.patch / 2);
    for (int j = 0; j < g.patch; j++) {
        for (int i = 0; i < g.patch; i++) {
            int index0 = index_x + i;
            int index1 = index_y + j;
            if (index0 < 0 || index0 >= g.gx || index1 < 0 || index1 >= g.gy) continue;
            cb(index0 + index1 * g.gx, index0, index1);
        }
    }
}

// Mesh centre of LoopPatch/BackLoopPatch: `inter_x * (index0 + 0.5) + l_bound` is
// evaluated in double and is exact there, so one rounding to float gives it.
inline float tor_mesh(float inter, int k, float bound) {
    return (float)((double)inter * ((double)k + 0.5) + (double)bound);
}
// Mesh centre of MapLoopPatch (tor.cu.cc:235-236): float arithmetic.
inline float tor_mesh_map(float inter, int k, float bound, bool c) {
    return madd(inter, (float)(0.5 + k), bound, c);
}

// The reference's cut-off decision (tor.cu.cc:57-71) in its device float arithmetic.
inline bool tor_inside_f32(const TorGeom &g, const TorCross &x, int i0, int i1, float f,
                           bool geo) {
    float d2 = tor_d2_f32(x.cross_x, x.cross_y, tor_mesh(g.inter_x, i0, g.l_bound),
                          tor_mesh(g.inter_y, i1, g.b_bound), x.dcos_x, x.dcos_y, true);
    float tsc = geo ? g.tor_sigma2 * f : g.tor_sigma2;
    return (double)d2 < 9.0 * (double)tsc;
}

// ---------------------------------------------------------------------------
// Siddon
// ---------------------------------------------------------------------------

template <typename T>
struct Ray {
    T start[3], dir[3], length, min_t, max_t;
};

template <typename T>
struct RayCast {
    int boffs;
    T nextT[3], deltaT[3];
    int deltaBuf[3], inBuf[3];
};

template <typename T>
inline T madd_t(T a, T b, T c, bool contract);
template <>
inline float madd_t<float>(float a, float b, float c, bool contract) {
    return madd(a, b, c, contract);
}
template <>
inline double madd_t<double>(double a, double b, double c, bool) {
    return a * b + c;
}

template <typename T>
inline T sqrt_t(T v);
template <>
inline float sqrt_t<float>(float v) {
    return std::sqrt(v);
}
template <>
inline double sqrt_t<double>(double v) {
    return std::sqrt(v);
}

// CreateRay, siddon.cu.cc:61-81.
template <typename T>
inline Ray<T> create_ray(float x1, float y1, float z1, float x2, float y2, float z2, bool c) {
    Ray<T> r;
    T dx = (T)x2 - (T)x1, dy = (T)y2 - (T)y1, dz = (T)z2 - (T)z1;
    T length = sqrt_t<T>(madd_t<T>(dz, dz, madd_t<T>(dx, dx, dy * dy, c), c));
    r.length = length;
    r.start[0] = x1;
    r.start[1] = y1;
    r.start[2] = z1;
    r.dir[0] = dx / length;
    r.dir[1] = dy / length;
    r.dir[2] = dz / length;
    r.min_t = 0;
    r.max_t = length;
    return r;
}

// ClipRay, siddon.cu.cc:118-153.
template <typename T>
inline bool clip_ray(T toplim, T botlim, int comp, Ray<T> &ray) {
    T p0 = ray.start[comp];
    T delta_p = ray.dir[comp];
    T tmax = ray.max_t, tmin = ray.min_t, t;
    if (delta_p > 0.0) {
        t = (toplim - p0) / delta_p;
        if (t < tmax) tmax = t;
        t = (botlim - p0) / delta_p;
        if (t > tmin) tmin = t;
    } else if (delta_p < 0.0) {
        t = (botlim - p0) / delta_p;
        if (t < tmax) tmax = t;
        t = (toplim - p0) / delta_p;
        if (t > tmin) tmin = t;
    } else {
        if ((p0 < botlim) || (p0 > toplim)) return false;
    }
    ray.min_t = tmin;
    ray.max_t = tmax;
    return tmin < tmax;
}

template <typename T>
struct Box {
    int grid[3];
    T size[3], center[3];
};

// IsThroughImage, siddon.cu.cc:163-183.
template <typename T>
inline bool through_image(const Box<T> &b, Ray<T> &ray) {
    ray.min_t = 0;
    ray.max_t = ray.length;
    for (int i = 0; i < 3; i++) {
        if (!clip_ray<T>(b.center[i] + b.size[i] / 2, b.center[i] - b.size[i] / 2, i, ray))
            return false;
    }
    return ray.min_t < ray.max_t;
}

// SetupRayCastComponent, siddon.cu.cc:196-250.
template <typename T>
inline void setup_component(const Box<T> &b, const Ray<T> &ray, int comp, RayCast<T> &rc,
                            int &pos, bool c) {
    T p0 = ray.start[comp];
    T r_pdir = ray.dir[comp];
    T pt = madd_t<T>(ray.min_t, r_pdir, p0, c);
    T v_res = b.size[comp] / b.grid[comp];
    int v_count = b.grid[comp];
    if (r_pdir > 0.0) {
        pos = (int)(pt / v_res);
        rc.nextT[comp] = madd_t<T>((T)(pos + 1), v_res, -pt, c) / r_pdir;
        rc.deltaT[comp] = v_res / r_pdir;
        rc.deltaBuf[comp] = 1;
        rc.inBuf[comp] = v_count - pos;
    } else if (r_pdir < 0.0) {
        pos = v_count - 1 - (int)(v_count - pt / v_res);
        rc.nextT[comp] = madd_t<T>((T)pos, v_res, -pt, c) / r_pdir;
        rc.deltaT[comp] = -v_res / r_pdir;
        rc.deltaBuf[comp] = -1;
        rc.inBuf[comp] = pos + 1;
    } else {
        pos = (int)(pt / v_res);
        rc.nextT[comp] = std::numeric_limits<float>::max();
        rc.deltaT[comp] = std::numeric_limits<float>::max();
        rc.deltaBuf[comp] = 0;
        rc.inBuf[comp] = 1;
    }
    for (int i = comp - 1; i >= 0; i--) rc.deltaBuf[comp] *= b.grid[i];
}

// SetupRayCast, siddon.cu.cc:261-284. Returns false when the start voxel lies
// outside the grid while the walk would run (the reference then reads outside the
// image; the new kernels skip such a ray, and the oracle reports it).
template <typename T>
inline bool setup_raycast(const Box<T> &b, Ray<T> &ray, RayCast<T> &rc, bool c,
                          int *pos_out = nullptr) {
    for (int i = 0; i < 3; i++) ray.start[i] = ray.start[i] - (b.center[i] - b.size[i] / 2);
    int pos[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) setup_component<T>(b, ray, k, rc, pos[k], c);
    rc.boffs = pos[0] + b.grid[0] * (pos[1] + b.grid[1] * pos[2]);
    if (pos_out)
        for (int k = 0; k < 3; k++) pos_out[k] = pos[k];
    bool runs = rc.inBuf[0] * rc.inBuf[1] * rc.inBuf[2] != 0;
    bool inside = true;
    for (int k = 0; k < 3; k++) inside = inside && pos[k] >= 0 && pos[k] < b.grid[k];
    return !runs || inside;
}

template <typename T>
inline int argmin3(const T *n) {  // siddon.cu.cc:305, ties to the lower index
    return (n[0] <= n[1]) ? ((n[0] <= n[2]) ? 0 : 2) : ((n[1] <= n[2]) ? 1 : 2);
}

template <typename T>
Box<T> make_box(const int *grid, const float *center, const float *size) {
    Box<T> b;
    for (int i = 0; i < 3; i++) {
        b.grid[i] = grid[i];
        b.size[i] = size[i];
        b.center[i] = center[i];
    }
    return b;
}

// Walk one ray; `cb(index, l_len, t_mid_rel)` per visited voxel. t_mid_rel is the
// TOF offset `t` of siddon.cu.cc:311 already evaluated in the mode's arithmetic.
// Returns the number of visited voxels.
template <typename T, typename F>
inline int walk(RayCast<T> &rc, F &&cb) {
    T last_t = 0;
    int stillin = rc.inBuf[0] * rc.inBuf[1] * rc.inBuf[2];
    int visited = 0;
    while (stillin) {
        int i = argmin3<T>(rc.nextT);
        T l_len = rc.nextT[i] - last_t;
        cb(rc.boffs, l_len, rc.nextT[i], last_t);
        last_t = rc.nextT[i];
        rc.nextT[i] += rc.deltaT[i];
        rc.boffs += rc.deltaBuf[i];
        stillin = rc.inBuf[i] - 1;
        rc.inBuf[i] = stillin;
        visited++;
    }
    return visited;
}

struct SiddonLor {
    float x1, y1, z1, x2, y2, z2, tof;
};

inline SiddonLor siddon_lor(const float *lors, int64_t n, int64_t i) {
    return {lors[0 * n + i], lors[1 * n + i], lors[2 * n + i], lors[3 * n + i],
            lors[4 * n + i], lors[5 * n + i], lors[6 * n + i]};
}

// The f32 TOF terms of RayTracing / BackRayTracing (siddon.cu.cc:310-316, :356-362):
// `skip` when the 3-sigma test fails; e = exp(-t2/2) and s = sqrt(2*pi*sigma2) in
// double, so callers can evaluate `(P * e) / s` in the reference's order.
inline void siddon_tof_terms_f32(float t_tof, float nextT, float last_t, float l_len,
                                 float sigma2_tof, float bs, bool c, bool &skip, double &e,
                                 double &s) {
    float t = (float)((double)t_tof - 0.5 * (double)(nextT + last_t));
    float sigma2 = (float)((double)sigma2_tof + (double)madd(l_len, l_len, bs * bs, c) / 12.0);
    float t2_by_sigma2 = t * t / sigma2;
    skip = !(t2_by_sigma2 < 9);
    e = std::exp(-0.5 * (double)t2_by_sigma2);
    s = std::sqrt(2.0 * M_PI * (double)sigma2);
}


// ---- f64 mode for Siddon: the float walk decides, a double shadow measures.

// Entry/exit parameters of the ray in double, all three slabs (no early exit).
inline void clip_all_f64(const Box<double> &b, Ray<double> &ray) {
    double tmin = 0, tmax = ray.length;
    for (int k = 0; k < 3; k++) {
        double top = b.center[k] + b.size[k] / 2, bot = b.center[k] - b.size[k] / 2;
        double p0 = ray.start[k], dp = ray.dir[k];
        if (dp > 0) {
            tmax = std::min(tmax, (top - p0) / dp);
            tmin = std::max(tmin, (bot - p0) / dp);
        } else if (dp < 0) {
            tmax = std::min(tmax, (bot - p0) / dp);
            tmin = std::max(tmin, (top - p0) / dp);
        }
    }
    ray.min_t = tmin;
    ray.max_t = tmax;
}

struct ShadowRay {
    bool through = false, ok = true;
    RayCast<float> rc;  // the reference's float walk state
    double length = 0, min_t = 0, nextT[3] = {0, 0, 0}, deltaT[3] = {0, 0, 0};
    float lengthf = 0, min_tf = 0;
};

inline ShadowRay shadow_setup(const Box<float> &bf, const Box<double> &bd, const SiddonLor &l) {
    ShadowRay S;
    Ray<float> rf = create_ray<float>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, true);
    S.lengthf = rf.length;
    if (!through_image<float>(bf, rf)) return S;
    S.through = true;
    S.min_tf = rf.min_t;
    int pos[3];
    S.ok = setup_raycast<float>(bf, rf, S.rc, true, pos);
    Ray<double> rd = create_ray<double>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, true);
    clip_all_f64(bd, rd);
    S.length = rd.length;
    S.min_t = rd.min_t;
    for (int k = 0; k < 3; k++) {
        double v_res = bd.size[k] / bd.grid[k];
        double p0 = rd.start[k] - (bd.center[k] - bd.size[k] / 2);
        double pt = rd.min_t * rd.dir[k] + p0;
        double dir = rd.dir[k];
        if (rf.dir[k] > 0.0f && dir != 0) {
            S.nextT[k] = ((pos[k] + 1) * v_res - pt) / dir;
            S.deltaT[k] = v_res / dir;
        } else if (rf.dir[k] < 0.0f && dir != 0) {
            S.nextT[k] = (pos[k] * v_res - pt) / dir;
            S.deltaT[k] = -v_res / dir;
        } else {
            S.nextT[k] = std::numeric_limits<float>::max();
            S.deltaT[k] = std::numeric_limits<float>::max();
        }
    }
    return S;
}

// Walk the float state; cb(index, l_f, next_f, last_f, l_d, next_d, last_d).
template <typename F>
inline void shadow_walk(ShadowRay &S, F &&cb) {
    RayCast<float> &rc = S.rc;
    float last_t = 0;
    double last_d = 0;
    int stillin = rc.inBuf[0] * rc.inBuf[1] * rc.inBuf[2];
    while (stillin) {
        int i = argmin3<float>(rc.nextT);
        cb(rc.boffs, rc.nextT[i] - last_t, rc.nextT[i], last_t, S.nextT[i] - last_d, S.nextT[i],
           last_d);
        last_t = rc.nextT[i];
        last_d = S.nextT[i];
        rc.nextT[i] += rc.deltaT[i];
        S.nextT[i] += S.deltaT[i];
        rc.boffs += rc.deltaBuf[i];
        stillin = rc.inBuf[i] - 1;
        rc.inBuf[i] = stillin;
    }
}

// The TOF factor of one voxel: float 3-sigma decision (siddon.cu.cc:311-314 with
// nvcc contraction), double value bin*exp(-t^2/2s^2)/sqrt(2 pi s^2).
inline bool shadow_tof(float t_tof_f, double t_tof_d, float next_f, float last_f, float l_f,
                       double next_d, double last_d, double l_d, float tof_sigma2,
                       float tof_bin, double &factor) {
    bool skip;
    double e, sq;
    siddon_tof_terms_f32(t_tof_f, next_f, last_f, l_f, tof_sigma2, tof_bin, true, skip, e, sq);
    if (skip) return false;
    double t = t_tof_d - 0.5 * (next_d + last_d);
    double s2 = (double)tof_sigma2 + (l_d * l_d + (double)tof_bin * tof_bin) / 12.0;
    factor = (double)tof_bin * std::exp(-0.5 * t * t / s2) / std::sqrt(2.0 * M_PI * s2);
    return true;
}

}  // namespace

extern "C" {

int oracle_version() { return 3; }

// ---------------------------------------------------------------------------
// TOR entry points
// ---------------------------------------------------------------------------

// Projection (tor.cu.cc:348-392 + ComputeSlice/LoopPatch). out has n entries.
void oracle_tor_projection_f32(const float *lors, int64_t n, const int *grid, const float *center,
                               const float *size, float kernel_width, int geo_flag, float tof_bin,
                               float tof_sigma2, const float *image, int contract, float *out) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool c = contract != 0, geo = geo_flag != 0;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    for (int64_t t = 0; t < n; t++) {
        TorLor l = tor_lor(lors, n, t, true);
        float pv = 0.0f;
        for (int s = 0; s < g.gz; s++) {
            float sz = tor_slice_z_proj(g, (unsigned)s);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, c);
            if (!x.valid) continue;
            const float *slice = image + s * slice_mesh;
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                float v = tor_smv_f32(l.xc, l.yc, l.zc, l.f, geo, sz, tof_bin, tof_sigma2,
                                      x.cross_x, x.cross_y, tor_mesh(g.inter_x, i0, g.l_bound),
                                      tor_mesh(g.inter_y, i1, g.b_bound), x.dcos_x, x.dcos_y,
                                      g.tor_sigma2, c);
                pv = madd(v, slice[idx], pv, c);
            });
        }
        out[t] = pv;
    }
}

void oracle_tor_projection_f64(const float *lors, int64_t n, const int *grid, const float *center,
                               const float *size, float kernel_width, int geo_flag, float tof_bin,
                               float tof_sigma2, const float *image, double *out) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool geo = geo_flag != 0, tof_on = tof_sigma2 < kTofThreshold;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    for (int64_t t = 0; t < n; t++) {
        TorLor l = tor_lor(lors, n, t, true);
        double pv = 0.0;
        for (int s = 0; s < g.gz; s++) {
            float sz = tor_slice_z_proj(g, (unsigned)s);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, true);
            if (!x.valid) continue;
            double szd = tor_slice_z_f64(g, (unsigned)s);
            TorCrossD xd = tor_cross_f64(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, szd);
            const float *slice = image + s * slice_mesh;
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                double v = tor_smv_f64(l.xc, l.yc, l.zc, l.f, geo, szd, tof_bin, tof_sigma2,
                                       tof_on, xd.cross_x, xd.cross_y,
                                       g.d_inter_x * (i0 + 0.5) + g.d_l_bound,
                                       g.d_inter_y * (i1 + 0.5) + g.d_b_bound, xd.dcos_x,
                                       xd.dcos_y, g.d_tor_sigma2, true,
                                       tor_inside_f32(g, x, i0, i1, l.f, geo));
                pv += v * (double)slice[idx];
            });
        }
        out[t] = pv;
    }
}

// Back-projection (tor.cu.cc:394-433 + BackComputeSlice/BackLoopPatch): the output
// image is zeroed, then image += value / lors_value[t] where lors_value[t] > 1e-7.
void oracle_tor_backprojection_f32(const float *lors, const float *lors_value, int64_t n,
                                   const int *grid, const float *center, const float *size,
                                   float kernel_width, int geo_flag, float tof_bin,
                                   float tof_sigma2, int contract, float *image) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool c = contract != 0, geo = geo_flag != 0;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    std::memset(image, 0, sizeof(float) * slice_mesh * g.gz);
    for (int s = 0; s < g.gz; s++) {
        float sz = tor_slice_z_back(g, (unsigned)s);
        float *slice = image + s * slice_mesh;
        for (int64_t t = 0; t < n; t++) {
            TorLor l = tor_lor(lors, n, t, true);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, c);
            if (!x.valid) continue;
            float pv = lors_value[t];
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                float v = tor_smv_f32(l.xc, l.yc, l.zc, l.f, geo, sz, tof_bin, tof_sigma2,
                                      x.cross_x, x.cross_y, tor_mesh(g.inter_x, i0, g.l_bound),
                                      tor_mesh(g.inter_y, i1, g.b_bound), x.dcos_x, x.dcos_y,
                                      g.tor_sigma2, c);
                if ((double)pv > 1e-7) slice[idx] += v / pv;
            });
        }
    }
}

void oracle_tor_backprojection_f64(const float *lors, const float *lors_value, int64_t n,
                                   const int *grid, const float *center, const float *size,
                                   float kernel_width, int geo_flag, float tof_bin,
                                   float tof_sigma2, double *image) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool geo = geo_flag != 0, tof_on = tof_sigma2 < kTofThreshold;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    std::memset(image, 0, sizeof(double) * slice_mesh * g.gz);
    for (int s = 0; s < g.gz; s++) {
        float sz = tor_slice_z_back(g, (unsigned)s);
        double szd = tor_slice_z_f64(g, (unsigned)s);
        double *slice = image + s * slice_mesh;
        for (int64_t t = 0; t < n; t++) {
            TorLor l = tor_lor(lors, n, t, true);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, true);
            if (!x.valid) continue;
            double pv = lors_value[t];
            if (!(pv > 1e-7)) continue;
            TorCrossD xd = tor_cross_f64(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, szd);
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                double v = tor_smv_f64(l.xc, l.yc, l.zc, l.f, geo, szd, tof_bin, tof_sigma2,
                                       tof_on, xd.cross_x, xd.cross_y,
                                       g.d_inter_x * (i0 + 0.5) + g.d_l_bound,
                                       g.d_inter_y * (i1 + 0.5) + g.d_b_bound, xd.dcos_x,
                                       xd.dcos_y, g.d_tor_sigma2, true,
                                       tor_inside_f32(g, x, i0, i1, l.f, geo));
                slice[idx] += v / pv;
            });
        }
    }
}

// Map (tor.cu.cc:435-481 + Mapping/MapLoopPatch): lors layout [7,N]; image += value /
// lors_value[t] with no threshold and no TOF.
void oracle_tor_maplors_f32(const float *lors, const float *lors_value, int64_t n, const int *grid,
                            const float *center, const float *size, float kernel_width,
                            int geo_flag, int contract, float *image) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool c = contract != 0, geo = geo_flag != 0;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    std::memset(image, 0, sizeof(float) * slice_mesh * g.gz);
    for (int s = 0; s < g.gz; s++) {
        float sz = tor_slice_z_back(g, (unsigned)s);
        float *slice = image + s * slice_mesh;
        for (int64_t t = 0; t < n; t++) {
            TorLor l = tor_lor(lors, n, t, false);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, c);
            if (!x.valid) continue;
            float pv = lors_value[t];
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                float v = tor_map_smv_f32(l.f, geo, x.cross_x, x.cross_y,
                                          tor_mesh_map(g.inter_x, i0, g.l_bound, c),
                                          tor_mesh_map(g.inter_y, i1, g.b_bound, c), x.dcos_x,
                                          x.dcos_y, g.tor_sigma2, c);
                slice[idx] += v / pv;
            });
        }
    }
}

void oracle_tor_maplors_f64(const float *lors, const float *lors_value, int64_t n, const int *grid,
                            const float *center, const float *size, float kernel_width,
                            int geo_flag, double *image) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool geo = geo_flag != 0;
    int64_t slice_mesh = (int64_t)g.gx * g.gy;
    std::memset(image, 0, sizeof(double) * slice_mesh * g.gz);
    for (int s = 0; s < g.gz; s++) {
        float sz = tor_slice_z_back(g, (unsigned)s);
        double szd = tor_slice_z_f64(g, (unsigned)s);
        double *slice = image + s * slice_mesh;
        for (int64_t t = 0; t < n; t++) {
            TorLor l = tor_lor(lors, n, t, false);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, true);
            if (!x.valid) continue;
            double pv = lors_value[t];
            TorCrossD xd = tor_cross_f64(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, szd);
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int idx, int i0, int i1) {
                double v = tor_smv_f64(0, 0, 0, l.f, geo, szd, 0, 0, false, xd.cross_x,
                                       xd.cross_y, g.d_inter_x * (i0 + 0.5) + g.d_l_bound,
                                       g.d_inter_y * (i1 + 0.5) + g.d_b_bound, xd.dcos_x,
                                       xd.dcos_y, g.d_tor_sigma2, false,
                                       tor_inside_f32(g, x, i0, i1, l.f, geo));
                slice[idx] += v / pv;
            });
        }
    }
}

// Per-LOR work counts for the roofline: `slots` = voxels the reference visits (in
// slice bounds, all patch positions: the loop-body count of tor.cu.cc:138-165) and
// `useful` = those inside the 3-sigma tube cut-off (non-zero weight).
void oracle_tor_counts(const float *lors, int64_t n, int ncols, const int *grid,
                       const float *center, const float *size, float kernel_width, int geo_flag,
                       int64_t *slots, int64_t *useful, int64_t *slices) {
    TorGeom g = tor_geom(grid, center, size, kernel_width);
    bool geo = geo_flag != 0;
    for (int64_t t = 0; t < n; t++) {
        TorLor l = tor_lor(lors, n, t, ncols == 10);
        int64_t ns = 0, nu = 0, nsl = 0;
        for (int s = 0; s < g.gz; s++) {
            float sz = tor_slice_z_proj(g, (unsigned)s);
            TorCross x = tor_cross(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, sz, true);
            if (!x.valid) continue;
            nsl++;
            tor_visit_patch(g, x.cross_x, x.cross_y, [&](int, int i0, int i1) {
                ns++;
                float d2 = tor_d2_f32(x.cross_x, x.cross_y, tor_mesh(g.inter_x, i0, g.l_bound),
                                      tor_mesh(g.inter_y, i1, g.b_bound), x.dcos_x, x.dcos_y,
                                      true);
                float tsc = geo ? g.tor_sigma2 * l.f : g.tor_sigma2;
                if ((double)d2 < 9.0 * (double)tsc) nu++;
            });
        }
        slots[t] = ns;
        useful[t] = nu;
        slices[t] = nsl;
    }
}

// ---------------------------------------------------------------------------
// Siddon entry points
// ---------------------------------------------------------------------------

// Projection (siddon.cu.cc:583-606 + project/RayTracing). out has n entries.
// Returns the number of rays whose start voxel was outside the grid (skipped).
int64_t oracle_siddon_projection_f32(const float *lors, int64_t n, const int *grid,
                                     const float *center, const float *size, float tof_bin,
                                     float tof_sigma2, const float *image, int contract,
                                     float *out) {
    bool c = contract != 0;
    Box<float> box = make_box<float>(grid, center, size);
    bool tof_on = tof_sigma2 < kTofThreshold;
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        Ray<float> ray = create_ray<float>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, c);
        if (!through_image<float>(box, ray)) {
            out[t] = 0.0f;
            continue;
        }
        RayCast<float> rc;
        if (!setup_raycast<float>(box, ray, rc, c)) {
            bad++;
            out[t] = 0.0f;
            continue;
        }
        float weight = 1 / ray.length / ray.length;
        float t_tof = (float)((double)ray.length * 0.5 - (double)ray.min_t - (double)l.tof);
        float pv = 0.0f;
        walk<float>(rc, [&](int mi, float l_len, float next_t, float last_t) {
            if (tof_on) {
                bool skip;
                double e, s;
                siddon_tof_terms_f32(t_tof, next_t, last_t, l_len, tof_sigma2, tof_bin, c, skip,
                                     e, s);
                if (!skip)
                    pv = (float)((double)pv +
                                 (double)(image[mi] * weight * l_len * tof_bin) * e / s);
            } else {
                pv = madd(image[mi] * weight, l_len, pv, c);
            }
        });
        out[t] = pv;
    }
    return bad;
}

int64_t oracle_siddon_projection_f64(const float *lors, int64_t n, const int *grid,
                                     const float *center, const float *size, float tof_bin,
                                     float tof_sigma2, const float *image, double *out) {
    Box<float> bf = make_box<float>(grid, center, size);
    Box<double> bd = make_box<double>(grid, center, size);
    bool tof_on = tof_sigma2 < kTofThreshold;
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        ShadowRay S = shadow_setup(bf, bd, l);
        out[t] = 0.0;
        if (!S.through) continue;
        if (!S.ok) {
            bad++;
            continue;
        }
        double weight = 1.0 / (S.length * S.length);
        float t_tof_f = (float)((double)S.lengthf * 0.5 - (double)S.min_tf - (double)l.tof);
        double t_tof_d = S.length * 0.5 - S.min_t - (double)l.tof;
        double pv = 0.0;
        shadow_walk(S, [&](int mi, float lf, float nf, float la_f, double ld, double nd,
                           double la_d) {
            if (tof_on) {
                double fac;
                if (shadow_tof(t_tof_f, t_tof_d, nf, la_f, lf, nd, la_d, ld, tof_sigma2, tof_bin,
                               fac))
                    pv += image[mi] * weight * ld * fac;
            } else {
                pv += image[mi] * weight * ld;
            }
        });
        out[t] = pv;
    }
    return bad;
}

// Back-projection (siddon.cu.cc:614-641 + backproject/BackRayTracing): image zeroed,
// image += value / lors_value[t] where lors_value[t] > 0.
int64_t oracle_siddon_backprojection_f32(const float *lors, const float *lors_value, int64_t n,
                                         const int *grid, const float *center, const float *size,
                                         float tof_bin, float tof_sigma2, int contract,
                                         float *image) {
    bool c = contract != 0;
    Box<float> box = make_box<float>(grid, center, size);
    std::memset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    bool tof_on = tof_sigma2 < kTofThreshold;
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        Ray<float> ray = create_ray<float>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, c);
        if (!through_image<float>(box, ray)) continue;
        RayCast<float> rc;
        if (!setup_raycast<float>(box, ray, rc, c)) {
            bad++;
            continue;
        }
        float weight = 1 / ray.length / ray.length;
        float t_tof = (float)((double)ray.length * 0.5 - (double)ray.min_t - (double)l.tof);
        float pv = lors_value[t];
        walk<float>(rc, [&](int mi, float l_len, float next_t, float last_t) {
            if (tof_on) {
                bool skip;
                double e, s;
                siddon_tof_terms_f32(t_tof, next_t, last_t, l_len, tof_sigma2, tof_bin, c, skip,
                                     e, s);
                if (!skip) {
                    float value = (float)((double)(weight * l_len * tof_bin) * e / s);
                    if (pv > 0) image[mi] += value / pv;
                }
            } else {
                float value = weight * l_len;
                if (pv > 0) image[mi] += value / pv;
            }
        });
    }
    return bad;
}

int64_t oracle_siddon_backprojection_f64(const float *lors, const float *lors_value, int64_t n,
                                         const int *grid, const float *center, const float *size,
                                         float tof_bin, float tof_sigma2, double *image) {
    Box<float> bf = make_box<float>(grid, center, size);
    Box<double> bd = make_box<double>(grid, center, size);
    std::memset(image, 0, sizeof(double) * (int64_t)grid[0] * grid[1] * grid[2]);
    bool tof_on = tof_sigma2 < kTofThreshold;
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        double pv = lors_value[t];
        if (!(lors_value[t] > 0)) continue;
        ShadowRay S = shadow_setup(bf, bd, l);
        if (!S.through) continue;
        if (!S.ok) {
            bad++;
            continue;
        }
        double weight = 1.0 / (S.length * S.length);
        float t_tof_f = (float)((double)S.lengthf * 0.5 - (double)S.min_tf - (double)l.tof);
        double t_tof_d = S.length * 0.5 - S.min_t - (double)l.tof;
        shadow_walk(S, [&](int mi, float lf, float nf, float la_f, double ld, double nd,
                           double la_d) {
            if (tof_on) {
                double fac;
                if (shadow_tof(t_tof_f, t_tof_d, nf, la_f, lf, nd, la_d, ld, tof_sigma2, tof_bin,
                               fac))
                    image[mi] += weight * ld * fac / pv;
            } else {
                image[mi] += weight * ld / pv;
            }
        });
    }
    return bad;
}

// Map (siddon.cu.cc:650-675 + mapping/Map): weight 1/(L*L), no TOF, value / pv if pv > 0.
// lors layout [6+,N] (only x1..z2 are read).
int64_t oracle_siddon_maplors_f32(const float *lors, const float *lors_value, int64_t n,
                                  const int *grid, const float *center, const float *size,
                                  int contract, float *image) {
    bool c = contract != 0;
    Box<float> box = make_box<float>(grid, center, size);
    std::memset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        Ray<float> ray = create_ray<float>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, c);
        float weight = 1 / (ray.length * ray.length);
        if (!through_image<float>(box, ray)) continue;
        RayCast<float> rc;
        if (!setup_raycast<float>(box, ray, rc, c)) {
            bad++;
            continue;
        }
        float pv = lors_value[t];
        walk<float>(rc, [&](int mi, float l_len, float, float) {
            float value = weight * l_len;
            if (pv > 0) image[mi] += value / pv;
        });
    }
    return bad;
}

int64_t oracle_siddon_maplors_f64(const float *lors, const float *lors_value, int64_t n,
                                  const int *grid, const float *center, const float *size,
                                  double *image) {
    Box<float> bf = make_box<float>(grid, center, size);
    Box<double> bd = make_box<double>(grid, center, size);
    std::memset(image, 0, sizeof(double) * (int64_t)grid[0] * grid[1] * grid[2]);
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        double pv = lors_value[t];
        if (!(lors_value[t] > 0)) continue;
        ShadowRay S = shadow_setup(bf, bd, l);
        if (!S.through) continue;
        if (!S.ok) {
            bad++;
            continue;
        }
        double weight = 1.0 / (S.length * S.length);
        shadow_walk(S, [&](int mi, float, float, float, double ld, double, double) {
            image[mi] += weight * ld / pv;
        });
    }
    return bad;
}

// Per-LOR voxel-visit counts (the a18 loop trips) and a flag for rays whose start
// voxel is outside the grid.
int64_t oracle_siddon_counts(const float *lors, int64_t n, const int *grid, const float *center,
                             const float *size, int64_t *visits) {
    Box<float> box = make_box<float>(grid, center, size);
    int64_t bad = 0;
    for (int64_t t = 0; t < n; t++) {
        SiddonLor l = siddon_lor(lors, n, t);
        Ray<float> ray = create_ray<float>(l.x1, l.y1, l.z1, l.x2, l.y2, l.z2, true);
        visits[t] = 0;
        if (!through_image<float>(box, ray)) continue;
        RayCast<float> rc;
        if (!setup_raycast<float>(box, ray, rc, true)) {
            bad++;
            continue;
        }
        visits[t] = walk<float>(rc, [](int, float, float, float) {});
    }
    return bad;
}

}  // extern "C"

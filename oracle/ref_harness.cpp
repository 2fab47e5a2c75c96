// Driver for the reference's own projector host functions, compiled for the CPU
// through oracle/shim (TEST INFRASTRUCTURE: checker and CPU baseline only).
//
// Build one library per projector family (the reference TOR and Siddon libraries
// both define `projection` / `backprojection` / `maplors`, tor.cc:66-92 and
// siddon.cc:59-77, with different parameter lists):
//   -DSRF_REF_TOR    links src/cpp/tf_custom_ops/tor.cu.cc
//   -DSRF_REF_SIDDON links src/cpp/tf_custom_ops/siddon.cu.cc
//
// Each entry point splits the events into `nthreads` contiguous chunks, one
// std::thread per chunk. Projection writes disjoint output ranges; back-projection
// and map give each thread a private zeroed image and sum the images in thread
// order afterwards, so the result is deterministic. With nthreads == 1 the call is
// exactly the reference's serial order. Outputs are zeroed first, as the TF op
// wrappers do (tor.cc:132,222,310; siddon.cc:106).

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#if defined(SRF_REF_TOR)
// Prototypes as declared by the reference op wrapper, tor.cc:66-92.
void projection(const float *x1, const float *y1, const float *z1, const float *x2,
                const float *y2, const float *z2, const float *xc, const float *yc,
                const float *zc, const float *sigma2_factor, bool geo_sigma2_flag,
                float *projection_value, const int *grid, const float *center, const float *size,
                const float kernel_width, const float tof_bin, const float tof_sigma2,
                const float *image, const int num_events);
void backprojection(const float *x1, const float *y1, const float *z1, const float *x2,
                    const float *y2, const float *z2, const float *xc, const float *yc,
                    const float *zc, const float *sigma2_factor, bool geo_sigma2_flag,
                    const float *projection_value, const int *grid, const float *center,
                    const float *size, const float kernel_width, const float tof_bin,
                    const float tof_sigma2, float *image, const int num_events);
void maplors(const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
             const float *z2, const float *geo_sigma2_factor, bool geo_sigma2_flag,
             const float *projection_value, const int *grid, const float *center,
             const float *size, const float kernel_width, float *image, const int num_events);
#elif defined(SRF_REF_SIDDON)
// Prototypes as declared by the reference op wrapper, siddon.cc:59-77.
void projection(const float *x1, const float *y1, const float *z1, const float *x2,
                const float *y2, const float *z2, const float *tof_t, float *projection_value,
                const int *grid, const float *center, const float *size, const float tof_bin,
                const float tof_sigma2, const float *image, const int num_events);
void backprojection(const float *x1, const float *y1, const float *z1, const float *x2,
                    const float *y2, const float *z2, const float *tof_t,
                    const float *projection_value, const int *grid, const float *center,
                    const float *size, const float tof_bin, const float tof_sigma2, float *image,
                    const int num_events);
void maplors(const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
             const float *z2, const float *projection_value, const int *grid,
             const float *center, const float *size, float *image, const int num_events);
#else
#error "define SRF_REF_TOR or SRF_REF_SIDDON"
#endif

namespace {

template <typename F>
void run_chunks(int64_t n, int nthreads, F &&fn) {
    nthreads = std::max(1, nthreads);
    if (n < nthreads) nthreads = (int)std::max<int64_t>(1, n);
    int64_t per = (n + nthreads - 1) / nthreads;
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; t++) {
        int64_t b = t * per, e = std::min<int64_t>(n, b + per);
        if (b >= e) break;
        if (nthreads == 1) {
            fn(t, b, e);
        } else {
            pool.emplace_back([&fn, t, b, e]() { fn(t, b, e); });
        }
    }
    for (auto &th : pool) th.join();
}

// Back-projection style call: private images per thread, summed in thread order.
template <typename F>
void run_scatter(int64_t n, int nthreads, int64_t nvox, float *image, F &&fn) {
    nthreads = std::max(1, nthreads);
    if (n < nthreads) nthreads = (int)std::max<int64_t>(1, n);
    if (nthreads == 1) {
        std::memset(image, 0, sizeof(float) * nvox);
        if (n > 0) fn(image, 0, n);
        return;
    }
    std::vector<std::vector<float>> priv(nthreads, std::vector<float>(nvox, 0.0f));
    run_chunks(n, nthreads, [&](int t, int64_t b, int64_t e) { fn(priv[t].data(), b, e); });
    std::memset(image, 0, sizeof(float) * nvox);
    for (int t = 0; t < nthreads; t++)
        for (int64_t v = 0; v < nvox; v++) image[v] += priv[t][v];
}

}  // namespace

extern "C" {

#if defined(SRF_REF_TOR)

// lors: [10,N] SoA (x1,y1,z1,x2,y2,z2,xc,yc,zc,sigma2_factor).
void ref_tor_projection(const float *lors, int64_t n, const int *grid, const float *center,
                        const float *size, float kernel_width, int geo_flag, float tof_bin,
                        float tof_sigma2, const float *image, float *out, int nthreads) {
    std::memset(out, 0, sizeof(float) * n);
    const float *c[10];
    for (int k = 0; k < 10; k++) c[k] = lors + k * n;
    run_chunks(n, nthreads, [&](int, int64_t b, int64_t e) {
        projection(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, c[6] + b,
                   c[7] + b, c[8] + b, c[9] + b, geo_flag != 0, out + b, grid, center, size,
                   kernel_width, tof_bin, tof_sigma2, image, (int)(e - b));
    });
}

void ref_tor_backprojection(const float *lors, const float *lors_value, int64_t n,
                            const int *grid, const float *center, const float *size,
                            float kernel_width, int geo_flag, float tof_bin, float tof_sigma2,
                            float *image, int nthreads) {
    const float *c[10];
    for (int k = 0; k < 10; k++) c[k] = lors + k * n;
    int64_t nvox = (int64_t)grid[0] * grid[1] * grid[2];
    run_scatter(n, nthreads, nvox, image, [&](float *img, int64_t b, int64_t e) {
        backprojection(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, c[6] + b,
                       c[7] + b, c[8] + b, c[9] + b, geo_flag != 0, lors_value + b, grid, center,
                       size, kernel_width, tof_bin, tof_sigma2, img, (int)(e - b));
    });
}

// lors: [7,N] SoA (x1,y1,z1,x2,y2,z2,sigma2_factor).
void ref_tor_maplors(const float *lors, const float *lors_value, int64_t n, const int *grid,
                     const float *center, const float *size, float kernel_width, int geo_flag,
                     float *image, int nthreads) {
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    int64_t nvox = (int64_t)grid[0] * grid[1] * grid[2];
    run_scatter(n, nthreads, nvox, image, [&](float *img, int64_t b, int64_t e) {
        maplors(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, c[6] + b,
                geo_flag != 0, lors_value + b, grid, center, size, kernel_width, img,
                (int)(e - b));
    });
}

#else  // SRF_REF_SIDDON

// lors: [7,N] SoA (x1,y1,z1,x2,y2,z2,tof).
void ref_siddon_projection(const float *lors, int64_t n, const int *grid, const float *center,
                           const float *size, float tof_bin, float tof_sigma2,
                           const float *image, float *out, int nthreads) {
    std::memset(out, 0, sizeof(float) * n);
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    run_chunks(n, nthreads, [&](int, int64_t b, int64_t e) {
        projection(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, c[6] + b,
                   out + b, grid, center, size, tof_bin, tof_sigma2, image, (int)(e - b));
    });
}

void ref_siddon_backprojection(const float *lors, const float *lors_value, int64_t n,
                               const int *grid, const float *center, const float *size,
                               float tof_bin, float tof_sigma2, float *image, int nthreads) {
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    int64_t nvox = (int64_t)grid[0] * grid[1] * grid[2];
    run_scatter(n, nthreads, nvox, image, [&](float *img, int64_t b, int64_t e) {
        backprojection(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, c[6] + b,
                       lors_value + b, grid, center, size, tof_bin, tof_sigma2, img,
                       (int)(e - b));
    });
}

void ref_siddon_maplors(const float *lors, const float *lors_value, int64_t n, const int *grid,
                        const float *center, const float *size, float *image, int nthreads) {
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    int64_t nvox = (int64_t)grid[0] * grid[1] * grid[2];
    run_scatter(n, nthreads, nvox, image, [&](float *img, int64_t b, int64_t e) {
        maplors(c[0] + b, c[1] + b, c[2] + b, c[3] + b, c[4] + b, c[5] + b, lors_value + b, grid,
                center, size, img, (int)(e - b));
    });
}

#endif

}  // extern "C"

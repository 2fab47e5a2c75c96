// Driver for the reference's own CUDA projector kernels, compiled for sm_100a from
// src/cpp/tf_custom_ops/{tor,siddon}.cu.cc as they lie (TEST INFRASTRUCTURE: the GPU
// parity target and the GPU bar to beat; never part of the shipped library).
//
// The reference host launchers read grid/center/size from DEVICE memory with
// blocking copies (tor.cu.cc:361-363, siddon.cu.cc:593-595) and launch on the legacy
// default stream, so this driver stages the geometry on the device, zeroes the
// output like the TF op wrappers do (tor.cc:132,222,310; siddon.cc:106), calls the
// launcher and synchronises. Returns the CUDA error code (0 on success).
//
// Build one library per projector family (-DSRF_REF_TOR / -DSRF_REF_SIDDON).

#include <cuda_runtime.h>
#include <cstdint>

#if defined(SRF_REF_TOR)
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

struct DevGeom {
    int *grid = nullptr;
    float *center = nullptr, *size = nullptr;
    cudaError_t err = cudaSuccess;
    DevGeom(const int *g, const float *c, const float *s) {
        if ((err = cudaMalloc(&grid, 3 * sizeof(int))) != cudaSuccess) return;
        if ((err = cudaMalloc(&center, 3 * sizeof(float))) != cudaSuccess) return;
        if ((err = cudaMalloc(&size, 3 * sizeof(float))) != cudaSuccess) return;
        if ((err = cudaMemcpy(grid, g, 3 * sizeof(int), cudaMemcpyHostToDevice))) return;
        if ((err = cudaMemcpy(center, c, 3 * sizeof(float), cudaMemcpyHostToDevice))) return;
        err = cudaMemcpy(size, s, 3 * sizeof(float), cudaMemcpyHostToDevice);
    }
    ~DevGeom() {
        cudaFree(grid);
        cudaFree(center);
        cudaFree(size);
    }
};

int finish() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return (int)cudaDeviceSynchronize();
}

}  // namespace

extern "C" {

#if defined(SRF_REF_TOR)

// lors: device [10,N] SoA.
int refgpu_tor_projection(const float *lors, int64_t n, const int *grid, const float *center,
                          const float *size, float kernel_width, int geo_flag, float tof_bin,
                          float tof_sigma2, const float *image, float *out) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(out, 0, sizeof(float) * n);
    const float *c[10];
    for (int k = 0; k < 10; k++) c[k] = lors + k * n;
    projection(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9], geo_flag != 0, out,
               g.grid, g.center, g.size, kernel_width, tof_bin, tof_sigma2, image, (int)n);
    return finish();
}

int refgpu_tor_backprojection(const float *lors, const float *lors_value, int64_t n,
                              const int *grid, const float *center, const float *size,
                              float kernel_width, int geo_flag, float tof_bin, float tof_sigma2,
                              float *image) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    const float *c[10];
    for (int k = 0; k < 10; k++) c[k] = lors + k * n;
    backprojection(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9], geo_flag != 0,
                   lors_value, g.grid, g.center, g.size, kernel_width, tof_bin, tof_sigma2, image,
                   (int)n);
    return finish();
}

int refgpu_tor_maplors(const float *lors, const float *lors_value, int64_t n, const int *grid,
                       const float *center, const float *size, float kernel_width, int geo_flag,
                       float *image) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    maplors(c[0], c[1], c[2], c[3], c[4], c[5], c[6], geo_flag != 0, lors_value, g.grid,
            g.center, g.size, kernel_width, image, (int)n);
    return finish();
}

#else

int refgpu_siddon_projection(const float *lors, int64_t n, const int *grid, const float *center,
                             const float *size, float tof_bin, float tof_sigma2,
                             const float *image, float *out) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(out, 0, sizeof(float) * n);
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    projection(c[0], c[1], c[2], c[3], c[4], c[5], c[6], out, g.grid, g.center, g.size, tof_bin,
               tof_sigma2, image, (int)n);
    return finish();
}

int refgpu_siddon_backprojection(const float *lors, const float *lors_value, int64_t n,
                                 const int *grid, const float *center, const float *size,
                                 float tof_bin, float tof_sigma2, float *image) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    backprojection(c[0], c[1], c[2], c[3], c[4], c[5], c[6], lors_value, g.grid, g.center,
                   g.size, tof_bin, tof_sigma2, image, (int)n);
    return finish();
}

int refgpu_siddon_maplors(const float *lors, const float *lors_value, int64_t n, const int *grid,
                          const float *center, const float *size, float *image) {
    DevGeom g(grid, center, size);
    if (g.err) return (int)g.err;
    cudaDeviceSynchronize();
    cudaMemset(image, 0, sizeof(float) * (int64_t)grid[0] * grid[1] * grid[2]);
    const float *c[7];
    for (int k = 0; k < 7; k++) c[k] = lors + k * n;
    maplors(c[0], c[1], c[2], c[3], c[4], c[5], lors_value, g.grid, g.center, g.size, image,
            (int)n);
    return finish();
}

#endif

}  // extern "C"

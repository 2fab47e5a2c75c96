// Sparse transaxial point-spread function of the PSF reconstruction step
// (src/python/srf/model/recon_step.py:56-115): the image, seen as an [nx*ny, nz] matrix,
// is multiplied by a sparse [nx*ny, nx*ny] transaxial kernel (tf.sparse_tensor_dense_matmul
// there). Here: y = A x with A in CSR form and x, y dense row-major [rows, nz]; one warp per
// row of A, lanes over the nz columns, so a row's reads of x and its write of y are
// coalesced. The adjoint is the same product with the CSR of A^T (built once by the caller).

#include "srf_common.cuh"

namespace srf {
namespace {

constexpr int kSpmmThreads = 256;

__global__ void __launch_bounds__(kSpmmThreads)
csr_spmm_kernel(const int64_t *__restrict__ rowptr, const int *__restrict__ col,
                const float *__restrict__ val, int64_t nrows, int64_t ncols,
                const float *__restrict__ x, int nz, float *__restrict__ y, int accumulate) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < nrows; r += nwarps) {
        const int64_t k0 = __ldg(rowptr + r), k1 = __ldg(rowptr + r + 1);
        for (int z0 = 0; z0 < nz; z0 += 32) {
            const int z = z0 + lane;
            float acc = 0.0f;
            for (int64_t k = k0; k < k1; k++) {
                const int c = __ldg(col + k);
                const float a = __ldg(val + k);
                if (z < nz && (unsigned)c < (unsigned)ncols)
                    acc = fmaf(a, __ldg(x + (int64_t)c * nz + z), acc);
            }
            if (z < nz) {
                float *dst = y + r * nz + z;
                *dst = accumulate ? *dst + acc : acc;
            }
        }
    }
}

}  // namespace
}  // namespace srf

using namespace srf;

extern "C" int srf_csr_spmm(const int64_t *rowptr, const int *col, const float *val,
                            int64_t nrows, int64_t ncols, const float *x, int nz, float *y,
                            int accumulate, void *stream) {
    if (nrows < 0 || ncols < 0 || nz < 0) return SRF_ERR_INVALID_ARGUMENT;
    if (nrows == 0 || nz == 0) return SRF_OK;
    if (!rowptr || !y || (ncols > 0 && !x)) return SRF_ERR_INVALID_ARGUMENT;
    const int grid = stride_grid(nrows, kSpmmThreads / 32, 8);
    csr_spmm_kernel<<<grid, kSpmmThreads, 0, (cudaStream_t)stream>>>(rowptr, col, val, nrows,
                                                                       ncols, x, nz, y,
                                                                       accumulate);
    count_launches(1);
    return check_launch();
}

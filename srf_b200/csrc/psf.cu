// Point-spread function of the PSF reconstruction step (src/python/srf/model/
// recon_step.py:56-115). The image, seen as an [nx*ny, nz] matrix X, is multiplied by a
// dense axial kernel Pz [nz, nz] and a sparse transaxial kernel A [nx*ny, nx*ny]:
//   forward  (:78-87)   Y = A (X Pz^T)   (there: a dense matmul, then
//                                          tf.sparse_tensor_dense_matmul)
//   adjoint  (:95-101)  Y = A^T (B Pz)   (the same call with the CSR of A^T).
// The two products act on different sides, so A (X M) = (A X) M: csr_psf_kernel takes one
// row of A per warp, sums its neighbours' rows of X into U (lanes over the nz columns, so
// the reads of X are coalesced), stages U in shared memory and multiplies it by M = Pz^T
// (forward) or Pz (adjoint), kept in shared memory for the whole block: one launch per
// PSF application, no intermediate [nx*ny, nz] matrix. csr_spmm_kernel is the sparse
// product alone.

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

// Y = A X M with A in CSR form, X [ncols, nz], Y [nrows, nz] row-major, M[j][z] =
// Pz[z][j] (transpose_pz = 0, the forward PSF) or Pz[j][z] (transpose_pz = 1).
// Dynamic shared memory: M (nz * nz floats, laid out [j][z] so a warp's lanes read
// consecutive z) then one nz-float row per warp for U.
__global__ void __launch_bounds__(kSpmmThreads)
csr_psf_kernel(const int64_t *__restrict__ rowptr, const int *__restrict__ col,
               const float *__restrict__ val, int64_t nrows, int64_t ncols,
               const float *__restrict__ x, int nz, const float *__restrict__ pz,
               int transpose_pz, float *__restrict__ y, int accumulate) {
    extern __shared__ float sm[];
    float *m = sm;                                              // [nz][nz]
    float *u = sm + (size_t)nz * nz + (size_t)(threadIdx.x >> 5) * nz;  // this warp's U
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < nz * nz; i += blockDim.x) {
        const int j = i / nz, z = i - j * nz;  // m[j][z]
        m[i] = transpose_pz ? __ldg(pz + (int64_t)j * nz + z) : __ldg(pz + (int64_t)z * nz + j);
    }
    __syncthreads();
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < nrows; r += nwarps) {
        const int64_t k0 = __ldg(rowptr + r), k1 = __ldg(rowptr + r + 1);
        for (int z = lane; z < nz; z += 32) {
            float acc = 0.0f;
            for (int64_t k = k0; k < k1; k++) {
                const int c = __ldg(col + k);
                if ((unsigned)c < (unsigned)ncols)
                    acc = fmaf(__ldg(val + k), __ldg(x + (int64_t)c * nz + z), acc);
            }
            u[z] = acc;
        }
        __syncwarp();
        for (int z = lane; z < nz; z += 32) {
            float acc = 0.0f;
            for (int j = 0; j < nz; j++) acc = fmaf(u[j], m[j * nz + z], acc);
            float *dst = y + r * nz + z;
            *dst = accumulate ? *dst + acc : acc;
        }
        __syncwarp();  // u is rewritten for the warp's next row
    }
}

constexpr int kPsfMaxNz = 224;  // M and the U rows in shared memory: 224^2 + 8 * 224 floats

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

extern "C" int srf_psf_apply(const int64_t *rowptr, const int *col, const float *val,
                             int64_t nrows, int64_t ncols, const float *x, int nz,
                             const float *pz, int transpose_pz, float *y, int accumulate,
                             void *stream) {
    if (nrows < 0 || ncols < 0 || nz < 0) return SRF_ERR_INVALID_ARGUMENT;
    if (transpose_pz != 0 && transpose_pz != 1) return SRF_ERR_INVALID_ARGUMENT;
    if (nz > kPsfMaxNz) return SRF_ERR_UNSUPPORTED;
    if (nrows == 0 || nz == 0) return SRF_OK;
    if (!rowptr || !y || !pz || (ncols > 0 && !x)) return SRF_ERR_INVALID_ARGUMENT;
    const size_t smem = sizeof(float) * ((size_t)nz * nz + (size_t)(kSpmmThreads / 32) * nz);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(
            csr_psf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            set_cuda_error(e);
            return SRF_ERR_CUDA;
        }
    }
    const int grid = stride_grid(nrows, kSpmmThreads / 32, 4);
    csr_psf_kernel<<<grid, kSpmmThreads, smem, (cudaStream_t)stream>>>(
        rowptr, col, val, nrows, ncols, x, nz, pz, transpose_pz, y, accumulate);
    count_launches(1);
    return check_launch();
}

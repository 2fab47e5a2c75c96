/*
 * srf_b200 — C ABI of the B200 listmode PET projector library.
 *
 * Drop-in replacement for the native layer of SRF's listmode projector pair: the
 * host launchers of src/cpp/tf_custom_ops/tor.cu.cc and siddon.cu.cc (paths relative
 * to the SRF project root), which the TF op wrappers tor.cc / siddon.cc call.
 *
 * Conventions (all entry points):
 *   - LOR data is the reference's column layout: one pointer per field. Event i of a
 *     column is at column[i * lor_stride]; lor_stride = 1 is the reference's [C,N]
 *     layout (tor.cc:140-160), lor_stride = C is a row-major [N,C] array.
 *   - All data pointers are DEVICE pointers. grid / center / size are HOST arrays of
 *     three values (kernel order: fastest axis first), passed by value to the kernel:
 *     the reference instead copies them device-to-host on every call (tor.cu.cc:361).
 *   - Image layout is [grid[2]][grid[1]][grid[0]] (grid[0] fastest), as the reference.
 *   - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) and
 *     never synchronises the host, so calls can be captured in a CUDA graph.
 *   - Return value: SRF_OK or an srf_status_t code; nothing is launched on error.
 *     srf_status_string() names it; srf_last_cuda_error() gives the CUDA error of the
 *     calling thread's last failing call.
 *   - Outputs are overwritten (the reference op zeroes them first: tor.cc:132,222,310,
 *     siddon.cc:106) unless `accumulate` is non-zero, in which case results are added
 *     to what the output already holds.
 */
#ifndef SRF_B200_H
#define SRF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SRF_OK = 0,
    SRF_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, non-finite geometry */
    SRF_ERR_CUDA = 2,             /* a CUDA call failed; see srf_last_cuda_error() */
    SRF_ERR_UNSUPPORTED = 3       /* parameters outside what the kernels support */
} srf_status_t;

const char *srf_status_string(int status);
int srf_last_cuda_error(void);
int srf_version(void);
/* Number of kernels this library has launched in this process (all devices, all entry
 * points); a caller diffs it around a region to count that region's launches. */
int64_t srf_launch_count(void);
/* The TOR slab kernels take stream-ordered scratch (the per-slab LOR lists, up to
 * 4 bytes x LORs x slabs per frame) from a memory pool the library keeps per device;
 * the pool retains its memory between calls. This returns all of it that is not in use
 * to the driver. */
int srf_release_scratch(void);

/* ------------------------------------------------------------------ TOR (tube of response)
 * Field columns for TOR: x1,y1,z1,x2,y2,z2 (LOR endpoints, dominant axis last, as
 * produced by recon_process, src/python/srf/preprocess/function/on_tor_lors.py:251-262),
 * xc,yc,zc (TOF centre), sigma2_factor. TOF is on when tof_sigma2 < 405758
 * (tor.cu.cc:20,84). tor_sigma2 = kernel_width^2/36 and the patch edge is
 * ceil((sqrt(2)*kernel_width + voxel_z)/voxel_x) voxels (tor.cu.cc:374-375).
 */

/* Replaces projection(), tor.cu.cc:348-392 (TF op "Projection", tor.cc:14-28).
 * projection_value[i] = sum over crossed slices and patch voxels of weight * image. */
int srf_tor_projection(const float *x1, const float *y1, const float *z1, const float *x2,
                       const float *y2, const float *z2, const float *xc, const float *yc,
                       const float *zc, const float *sigma2_factor, int geo_sigma2_flag,
                       float *projection_value, const int *grid, const float *center,
                       const float *size, float kernel_width, float tof_bin, float tof_sigma2,
                       const float *image, int64_t num_events, int64_t lor_stride,
                       void *stream);

/* Replaces backprojection(), tor.cu.cc:394-433 (TF op "Backprojection", tor.cc:30-47).
 * image += weight / projection_value[i] for LORs with projection_value[i] > 1e-7. */
int srf_tor_backprojection(const float *x1, const float *y1, const float *z1, const float *x2,
                           const float *y2, const float *z2, const float *xc, const float *yc,
                           const float *zc, const float *sigma2_factor, int geo_sigma2_flag,
                           const float *projection_value, const int *grid, const float *center,
                           const float *size, float kernel_width, float tof_bin,
                           float tof_sigma2, float *image, int64_t num_events,
                           int64_t lor_stride, int accumulate, void *stream);

/* The reference's projection followed by its back-projection of the result, in one call
 * (the numerator of the reference's recon step, model/recon_step.py:38-40, done there as
 * two op calls): projection_value = A image (as srf_tor_projection) and
 * back_image = A^T(1 / projection_value) with the 1e-7 threshold (as
 * srf_tor_backprojection, `accumulate` likewise). No counterpart as one call in the
 * reference: both ops share one set of per-slab LOR lists. back_image must not alias image. */
int srf_tor_projection_backprojection(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, float *projection_value, const int *grid,
    const float *center, const float *size, float kernel_width, float tof_bin, float tof_sigma2,
    const float *image, float *back_image, int64_t num_events, int64_t lor_stride,
    int accumulate, void *stream);

/* Replaces maplors(), tor.cu.cc:435-481 (TF op "Maplors", tor.cc:49-64): geometric
 * weight only (no TOF), image += weight / projection_value[i] with no threshold. */
int srf_tor_maplors(const float *x1, const float *y1, const float *z1, const float *x2,
                    const float *y2, const float *z2, const float *sigma2_factor,
                    int geo_sigma2_flag, const float *projection_value, const int *grid,
                    const float *center, const float *size, float kernel_width, float *image,
                    int64_t num_events, int64_t lor_stride, int accumulate, void *stream);

/* No counterpart in the reference: the plain adjoint of srf_tor_projection,
 * image += weight * values[i] (no division, no threshold). Backward pass of the
 * differentiable projector and the OSEM numerator A^T(y/Ax) in its true form. */
int srf_tor_backproject_adjoint(const float *x1, const float *y1, const float *z1,
                                const float *x2, const float *y2, const float *z2,
                                const float *xc, const float *yc, const float *zc,
                                const float *sigma2_factor, int geo_sigma2_flag,
                                const float *values, const int *grid, const float *center,
                                const float *size, float kernel_width, float tof_bin,
                                float tof_sigma2, float *image, int64_t num_events,
                                int64_t lor_stride, int accumulate, void *stream);

/* No counterpart in the reference as one call: the effmap's Maplors (tor.cu.cc:435-481)
 * of detector-pair LORs that never exist in memory. LORs number first .. first+count-1 of
 * a generated sequence are taken through map_process (on_tor_lors.py:243-248) and those
 * of dominant-axis group `axis` (0 x, 1 y, 2 z) are mapped with lors_value = 1 into
 * `image`, in that group's kernel layout (grid / center / size as for srf_tor_maplors).
 * Every kernel of the call makes LOR t again from its number:
 *   kind 0: a random chord of a ring scanner (n_rings rings of n_per_block crystals,
 *           crystal k of ring r at index r * n_per_block + k, angle 2 pi k / n_per_block;
 *           n_blocks = 1): groups of 256 consecutive numbers share the chord class
 *           s = (k_a + k_b) mod n and the ring offset r_b - r_a, drawn from SplitMix64
 *           outputs 4 group and 4 group + 2 of the stream seeded `seed`; k_a and r_a come
 *           from output 2 g + 1 (g = first + t). Every ordered crystal pair is equally
 *           likely; a crystal paired with itself maps nothing;
 *   kind 1: the scanner's block-pair enumeration in the reference's order (ring pairs
 *           ir1-major, srfapp_new.py:153-157; block pairs i1 < i2 in a ring, i1 != i2
 *           across rings, scanner/pet/pet.py:149-168; every crystal of the first block,
 *           major, with every crystal of the second, :170-177).
 * crystals: DEVICE float32 [n_rings * n_blocks * n_per_block][3] crystal centres, ring
 * major, then block, then crystal in the block's mesh order. */
int srf_tor_maplors_generated(int kind, const float *crystals, int n_rings, int n_blocks,
                              int n_per_block, unsigned long long seed, int64_t first,
                              int64_t count, int axis, int geo_sigma2_flag, const int *grid,
                              const float *center, const float *size, float kernel_width,
                              float *image, int accumulate, void *stream);

/* No counterpart in the reference: per-LOR work counts of the TOR operator, used for
 * the roofline (algorithmic samples) and for work estimation. counts[i] = patch voxels
 * with non-zero weight (inside the 3-sigma tube), counts[num_events + i] = window
 * voxels visited (the reference's loop-body count). counts: DEVICE int32[2*N]. */
int srf_tor_count_samples(const float *x1, const float *y1, const float *z1, const float *x2,
                          const float *y2, const float *z2, const float *sigma2_factor,
                          int geo_sigma2_flag, const int *grid, const float *center,
                          const float *size, float kernel_width, int *counts,
                          int64_t num_events, int64_t lor_stride, void *stream);

/* srf_tor_projection_backprojection for batched frames (frame, n_frames, frame_stride as
 * in srf_tor_projection_batched): projection_value from the frames' images, then
 * back_images (same layout, must not alias images) += A^T(1 / projection_value) per frame.
 * No counterpart in the reference. */
int srf_tor_projection_backprojection_batched(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, const float *images,
    float *back_images, int64_t num_events, int64_t lor_stride, int accumulate, void *stream);

/* srf_tor_projection_backprojection_batched on image stacks in any axis order: voxel
 * (ix, iy, iz) of frame f (the kernel's axes, grid[0..2]) is element f * frame_stride +
 * ix * image_strides[0] + iy * image_strides[1] + iz * image_strides[2] (HOST int64[3],
 * each >= 1, a frame's last voxel below frame_stride) of both images and back_images,
 * e.g. a permuted view of an [F, nx, ny, nz] stack, which then needs no copy into the
 * kernel layout and back. accumulate = 0 zeroes all n_frames * frame_stride floats from
 * back_images first (the whole stack, not only the voxels the strides reach). No
 * counterpart in the reference. */
int srf_tor_projection_backprojection_batched_strided(
    const float *x1, const float *y1, const float *z1, const float *x2, const float *y2,
    const float *z2, const float *xc, const float *yc, const float *zc,
    const float *sigma2_factor, int geo_sigma2_flag, const int *frame, int n_frames,
    int64_t frame_stride, float *projection_value, const int *grid, const float *center,
    const float *size, float kernel_width, float tof_bin, float tof_sigma2, const float *images,
    float *back_images, const int64_t *image_strides, int64_t num_events, int64_t lor_stride,
    int accumulate, void *stream);

/* No counterpart in the reference: batched TOR for many reconstructions that share one
 * geometry (dynamic frames, many phantoms). LOR i belongs to frame frame[i] (DEVICE
 * int32[N], 0 <= frame[i] < n_frames; a LOR with a frame id outside that range
 * contributes nothing, as a LOR with non-finite endpoints does); images are n_frames
 * consecutive blocks of frame_stride floats (>= grid voxels). One launch covers every
 * frame. Semantics per
 * frame are those of srf_tor_projection / srf_tor_backprojection /
 * srf_tor_backproject_adjoint; `accumulate` = 0 zeroes all n_frames blocks first. */
int srf_tor_projection_batched(const float *x1, const float *y1, const float *z1,
                               const float *x2, const float *y2, const float *z2,
                               const float *xc, const float *yc, const float *zc,
                               const float *sigma2_factor, int geo_sigma2_flag,
                               const int *frame, int n_frames, int64_t frame_stride,
                               float *projection_value, const int *grid, const float *center,
                               const float *size, float kernel_width, float tof_bin,
                               float tof_sigma2, const float *images, int64_t num_events,
                               int64_t lor_stride, void *stream);
int srf_tor_backprojection_batched(const float *x1, const float *y1, const float *z1,
                                   const float *x2, const float *y2, const float *z2,
                                   const float *xc, const float *yc, const float *zc,
                                   const float *sigma2_factor, int geo_sigma2_flag,
                                   const int *frame, int n_frames, int64_t frame_stride,
                                   const float *projection_value, const int *grid,
                                   const float *center, const float *size, float kernel_width,
                                   float tof_bin, float tof_sigma2, float *images,
                                   int64_t num_events, int64_t lor_stride, int accumulate,
                                   void *stream);
int srf_tor_backproject_adjoint_batched(const float *x1, const float *y1, const float *z1,
                                        const float *x2, const float *y2, const float *z2,
                                        const float *xc, const float *yc, const float *zc,
                                        const float *sigma2_factor, int geo_sigma2_flag,
                                        const int *frame, int n_frames, int64_t frame_stride,
                                        const float *values, const int *grid,
                                        const float *center, const float *size,
                                        float kernel_width, float tof_bin, float tof_sigma2,
                                        float *images, int64_t num_events, int64_t lor_stride,
                                        int accumulate, void *stream);

/* No counterpart in the reference: process-wide tuning of the TOR kernels (used by the
 * autotuner; affects later calls from every thread). path: 0 automatic, 1 shared-memory
 * slab kernels with one lane per (LOR, slab) segment, 2 LOR-centric kernels (L2 gathers,
 * global atomics), 3 slab kernels with a segment's slices spread over lanes; slab_slices: slices
 * per slab, 0 = as many as fit; grid_mult: persistent slab CTAs = SMs x grid_mult (1..8;
 * 0 = automatic: 2 for projection and back-projection launches of at least 4M LORs over
 * whole-slice slabs, else 1). */
int srf_tor_set_tuning(int path, int slab_slices, int grid_mult);

/* No counterpart in the reference: the Siddon kernel family. path 0: automatic (the
 * scatter ops reduce four consecutive voxels at a time wherever the image is 16-byte
 * aligned and its voxel count is a multiple of 4); 1: one atomic per voxel. The projection
 * gathers one voxel at a time either way. Process-wide. */
int srf_siddon_set_tuning(int path);

/* No counterpart in the reference: upper bound, in bytes, of the per-slab LOR lists the
 * slab kernels build per call (0 = the default, 4 GiB). The lists are sized for the worst
 * case, 4 bytes x LORs x slabs per frame; a call with more LORs than fit is processed in
 * chunks of LORs (at least 4096 each), each chunk a complete pass. Process-wide. */
int srf_tor_set_scratch_limit(int64_t bytes);

/* ---------------------------------------------------------------------------------- Siddon
 * Field columns for Siddon: x1,y1,z1,x2,y2,z2,tof (tof in mm along the LOR, the
 * reference's convention, siddon.cu.cc:460). Weight 1/L^2 (siddon.cu.cc:459). TOF on
 * when tof_sigma2 < 405758 (siddon.cu.cc:15,308). A ray whose first voxel falls off
 * the grid (the reference then reads outside the image) contributes nothing.
 */

/* Replaces projection(), siddon.cu.cc:583-606 (TF op "Projection", siddon.cc:14-26). */
int srf_siddon_projection(const float *x1, const float *y1, const float *z1, const float *x2,
                          const float *y2, const float *z2, const float *tof_t,
                          float *projection_value, const int *grid, const float *center,
                          const float *size, float tof_bin, float tof_sigma2,
                          const float *image, int64_t num_events, int64_t lor_stride,
                          void *stream);

/* Replaces backprojection(), siddon.cu.cc:614-641 (TF op "Backprojection",
 * siddon.cc:28-43): image += weight / projection_value[i] where projection_value[i] > 0. */
int srf_siddon_backprojection(const float *x1, const float *y1, const float *z1,
                              const float *x2, const float *y2, const float *z2,
                              const float *tof_t, const float *projection_value,
                              const int *grid, const float *center, const float *size,
                              float tof_bin, float tof_sigma2, float *image,
                              int64_t num_events, int64_t lor_stride, int accumulate,
                              void *stream);

/* Replaces maplors(), siddon.cu.cc:650-675 (TF op "Maplors", siddon.cc:45-57): weight
 * 1/(L*L), no TOF, image += weight / projection_value[i] where projection_value[i] > 0. */
int srf_siddon_maplors(const float *x1, const float *y1, const float *z1, const float *x2,
                       const float *y2, const float *z2, const float *projection_value,
                       const int *grid, const float *center, const float *size, float *image,
                       int64_t num_events, int64_t lor_stride, int accumulate, void *stream);

/* No counterpart in the reference: plain adjoint of srf_siddon_projection,
 * image += weight * values[i]. */
int srf_siddon_backproject_adjoint(const float *x1, const float *y1, const float *z1,
                                   const float *x2, const float *y2, const float *z2,
                                   const float *tof_t, const float *values, const int *grid,
                                   const float *center, const float *size, float tof_bin,
                                   float tof_sigma2, float *image, int64_t num_events,
                                   int64_t lor_stride, int accumulate, void *stream);

/* No counterpart in the reference: per-ray work of the Siddon operator, used for the
 * roofline (algorithmic samples) and work estimation. counts[i] = voxels the ray's walk
 * visits (the loop trips of RayTracing, siddon.cu.cc:293-331; 0 for a ray that misses the
 * image). counts: DEVICE int32[N]. */
int srf_siddon_count_samples(const float *x1, const float *y1, const float *z1, const float *x2,
                             const float *y2, const float *z2, const int *grid,
                             const float *center, const float *size, int *counts,
                             int64_t num_events, int64_t lor_stride, void *stream);

/* ------------------------------------------------------------------ LOR preprocessing
 * The reference runs these in host numpy; here they run on the device with the same
 * float32 arithmetic and the same output order (x group, y group, z group; in each,
 * unswapped events then swapped ones, each in input order). Events with no dominant
 * axis (NaN coordinates) are dropped. The caller provides `workspace` of at least
 * srf_preprocess_workspace_size(num_events) bytes (device memory, 256-byte aligned).
 * group_counts is a DEVICE int64[3] receiving the sizes of the x, y and z groups.
 */
int64_t srf_preprocess_workspace_size(int64_t num_events);

/* Replaces recon_process, src/python/srf/preprocess/function/on_tor_lors.py:251-262:
 * events [N, >=7] rows (x1,y1,z1,x2,y2,z2,tof) with row stride event_stride floats ->
 * out [N, 10] rows (p1, p2, TOF centre, sigma2_factor; dominant axis last). tof_res is
 * the TOF resolution in ps (cut to +/-3 sigma when < 10000). */
int srf_recon_process(const float *events, int64_t num_events, int64_t event_stride,
                      double tof_res, float *out, int64_t *group_counts, void *workspace,
                      int64_t workspace_bytes, void *stream);

/* No counterpart in the reference: srf_recon_process for callers that cannot allocate
 * device memory when they preprocess (a service with a fixed memory budget that forbids
 * allocations after start-up, or a latency-critical path where cudaMalloc's implicit
 * device synchronisation is not acceptable). The partition's scratch comes from a
 * buffer inside the library (a file-scope __device__ array, 8.1 MiB, held by every GPU
 * that loads the library until exit) instead of a caller workspace; nothing is
 * allocated. Limits and rules:
 *   - num_events <= SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS, else SRF_ERR_UNSUPPORTED
 *     (nothing launched);
 *   - the first call on a device looks up the buffer's device address
 *     (cudaGetSymbolAddress) with that device current: make it before any stream
 *     capture;
 *   - all calls on a device share the buffer and it keeps the last call's contents
 *     (no part needs to start at zero); calls that overlap on the GPU race on it, so
 *     serialise them on one stream;
 *   - the looked-up address is kept for the life of the process, like the library's
 *     other per-device state (its scratch pool): after cudaDeviceReset of a device,
 *     do not call the library on that device again in the same process.
 * Same inputs, outputs and results as srf_recon_process. */
#define SRF_RECON_PROCESS_NOALLOC_MAX_EVENTS 8388608
int srf_recon_process_noalloc(const float *events, int64_t num_events, int64_t event_stride,
                              double tof_res, float *out, int64_t *group_counts, void *stream);

/* No counterpart in the reference: an optional step between preprocessing and the TOR
 * projectors. Copies records [num_records, ncols] (row-major, record_stride floats apart,
 * ncols >= 6: x1,y1,z1,x2,y2,z2 first) to `out` (same layout, must not alias `records`)
 * reordered inside each block of 4096 consecutive records by the shape of the LOR's tube
 * section, then by where it starts along the slice axis (a stable sort on a quantised
 * key). Records keep their block;
 * list-mode events being an unordered set, reconstructing from `out` gives the same sums
 * in another order, with fewer voxel slots walked by the slab kernels. */
int srf_order_by_direction(const float *records, int64_t num_records, int ncols,
                           int64_t record_stride, float *out, void *stream);

/* Replaces map_process, on_tor_lors.py:243-248: lors [N, >=6] -> out [N, 7] rows
 * (p1, p2 with the dominant axis last, sigma2_factor). */
int srf_map_process(const float *lors, int64_t num_lors, int64_t lor_stride, float *out,
                    int64_t *group_counts, void *workspace, int64_t workspace_bytes,
                    void *stream);

/* ------------------------------------------------------------------------- image algebra */

/* MLEM/OSEM update of model/recon_step.py:48-49: image[v] *= effinv[v] * bp[v]. */
int srf_mlem_update(float *image, const float *effinv, const float *bp, int64_t num_voxels,
                    void *stream);

/* Sparse transaxial PSF of the PSF reconstruction step (PSFReconStep,
 * src/python/srf/model/recon_step.py:56-115, there tf.sparse_tensor_dense_matmul):
 * y = A x, A an [nrows, ncols] CSR matrix (rowptr int64[nrows+1], col int32, val float32),
 * x a dense row-major [ncols, nz] matrix, y [nrows, nz] (y += A x with accumulate != 0).
 * All DEVICE pointers. The adjoint is the same call with the CSR of A^T. */
int srf_csr_spmm(const int64_t *rowptr, const int *col, const float *val, int64_t nrows,
                 int64_t ncols, const float *x, int nz, float *y, int accumulate, void *stream);

/* Separable PSF of the PSF reconstruction step in one launch (PSFReconStep,
 * src/python/srf/model/recon_step.py:78-87 and :95-101, there a dense matmul followed by
 * tf.sparse_tensor_dense_matmul): y = A (x Pz^T) (transpose_pz = 0, the forward PSF) or
 * y = A (x Pz) (transpose_pz = 1; with the CSR of A^T this is the adjoint), A an
 * [nrows, ncols] CSR matrix as in srf_csr_spmm, x [ncols, nz], Pz a dense row-major
 * [nz, nz] matrix, y [nrows, nz] (y += ... with accumulate != 0). nz <= 224
 * (SRF_ERR_UNSUPPORTED above). All DEVICE pointers. */
int srf_psf_apply(const int64_t *rowptr, const int *col, const float *val, int64_t nrows,
                  int64_t ncols, const float *x, int nz, const float *pz, int transpose_pz,
                  float *y, int accumulate, void *stream);

/* ------------------------------------------------------------------------ peak probes */

/* No counterpart in the reference: measurement kernels for the roofline denominators
 * that are not a plain HBM copy, timed by the caller with events on `stream`.
 * srf_probe_threads: threads per probe launch (the length of `sink` in floats).
 * srf_probe_l2_read: every thread reads a 16-byte-aligned buffer of n_floats (sized to
 *   stay L2-resident) `reps` times with L2-only loads; bytes read = reps * 4 * n_floats
 *   rounded down to 16-byte vectors.
 * srf_probe_ex2: every thread evaluates 8 * iters dependent-by-chain ex2.approx. */
int srf_probe_threads(int64_t *n_threads);
int srf_probe_l2_read(const float *buf, int64_t n_floats, int reps, float *sink, void *stream);
int srf_probe_ex2(int iters, float *sink, void *stream);
/* srf_probe_smem_threads: threads per shared-memory probe launch (the length of `sink`).
 * srf_probe_smem_read: every thread reads 16 bytes from a 32 KB shared buffer `iters`
 * times (a warp on consecutive addresses).
 * srf_probe_smem_atomic: every thread does `iters` float atomicAdd into a 32 KB shared
 * buffer; random = 0: a warp's lanes on 32 consecutive floats, 1: hashed addresses. */
int srf_probe_smem_threads(int64_t *n_threads);
int srf_probe_smem_read(int iters, float *sink, void *stream);
int srf_probe_smem_atomic(int iters, int random, float *sink, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SRF_B200_H */

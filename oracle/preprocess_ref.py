"""numpy restatement of SRF's host-side LOR preprocessing and effmap post-processing.

TEST INFRASTRUCTURE ONLY (the checker for the CUDA preprocessing kernels and the
source of expected values in the tests). Each function names the reference lines it
follows, relative to the SRF project root. Arithmetic stays in float32 when the input
is float32, exactly as the reference's numpy code does (numpy never fuses a*b+c, and
Python float scalars combine with float32 arrays in float32).
"""

import numpy as np

GAUSSIAN_FACTOR = 2.35482005  # srfapp_new.py:247, on_tor_lors.py:220

AXES = ("x", "y", "z")


def tof_info(tof_res_ps, tof_bin_ps):
    """``SRFApp._get_tof_info`` (src/python/srf/api/app/srfapp_new.py:244-251):
    returns (tof_bin [mm], tof_sigma2 [mm^2]) as Python floats."""
    limit = tof_res_ps * 0.15 / GAUSSIAN_FACTOR * 3
    return tof_bin_ps * 0.15, (limit ** 2) / 9


def sigma2_factor(lors):
    """on_tor_lors.py:137-166: (dx^2+dy^2)^2 / (x1^2+x2^2+y1^2+y2^2) / L^2 / 2."""
    p_start = lors[:, 0:3]
    p_end = lors[:, 3:6]
    p_diff = p_end - p_start
    p_dis2 = np.sum(np.square(p_diff), 1)
    dsq = p_diff[:, 0] ** 2 + p_diff[:, 1] ** 2
    rsq = p_start[:, 0] ** 2 + p_end[:, 0] ** 2 + p_start[:, 1] ** 2 + p_end[:, 1] ** 2
    return dsq ** 2 / rsq / p_dis2 / 2


def dominant_index(lors, axis):
    """``dominentBy`` + ``Partition`` (on_tor_lors.py:70-77, :97-107): ascending indices
    of the LORs whose |direction| is dominant along ``axis`` with the reference's tie
    rules (x wins |dx|=|dy|; y wins |dy|=|dz|; z needs a strict maximum)."""
    d = np.abs(lors[:, 3:6] - lors[:, 0:3])
    dx, dy, dz = d[:, 0], d[:, 1], d[:, 2]
    if axis == "x":
        m = (dx >= dy) & (dx >= dz)
    elif axis == "y":
        m = (dy > dx) & (dy >= dz)
    else:
        m = (dz > dx) & (dz > dy)
    return np.nonzero(m)[0]


def swap_points(lors, axis):
    """``SwapPointsOrder`` (on_tor_lors.py:175-193): rows with p2 >= p1 on ``axis``
    first (original order), then the others with their endpoints swapped; for
    records wider than 7 columns the TOF column is negated and the rest kept."""
    k = AXES.index(axis)
    d = lors[:, 3 + k] - lors[:, k]
    pos = lors[d >= 0]
    neg = lors[d < 0]
    parts = [neg[:, 3:6], neg[:, 0:3]]
    if lors.shape[1] > 7:
        parts += [0 - neg[:, 6:7], neg[:, 7:]]
    else:
        parts += [neg[:, 6:7]]
    return np.vstack((pos, np.hstack(parts)))


def cut_lors(lors, tof_res):
    """``CutLoRs`` (on_tor_lors.py:196-229) on [N,8] = (x1..z2, t, f): TOF centre
    C = p1 + (0.5 - t/L)(p2 - p1); when tof_res < 10000 ps and |C - p1| > 3 sigma,
    both endpoints move to C -/+ 3 sigma along the LOR. Returns [N,10] =
    (p1, p2, C, f)."""
    p_diff = lors[:, 3:6] - lors[:, 0:3]
    p_dis = np.sqrt(np.sum(np.square(p_diff), 1))
    dcos = np.array([p_diff[:, a] / p_dis for a in range(3)]).T.reshape((-1, 3))
    ratio = np.array(0.5 - (lors[:, 6] / p_dis))
    p0 = lors[:, 0:3].copy()
    p1 = lors[:, 3:6].copy()
    center = np.array([ratio * p_diff[:, a] for a in range(3)]).T + p0
    dcs = np.sqrt(np.sum(np.square(center - p0), 1))
    if tof_res < 10000:
        limit = tof_res * 0.15 / GAUSSIAN_FACTOR * 3
        idx = dcs > limit
        p0[idx] = center[idx] - limit * dcos[idx, :]
        p1[idx] = center[idx] + limit * dcos[idx, :]
    return np.hstack((p0, p1, center, lors[:, 7:]))


PERM_RECON = {"x": [1, 2, 0, 4, 5, 3, 7, 8, 6], "y": [0, 2, 1, 3, 5, 4, 6, 8, 7]}
PERM_MAP = {"x": [1, 2, 0, 4, 5, 3], "y": [0, 2, 1, 3, 5, 4]}


def recon_process(lors, tof_res):
    """``recon_process`` (on_tor_lors.py:251-262): [N,7] (x1..z2, t) -> dict axis ->
    [N_a,10] with the dominant axis moved to the kernel's third coordinate."""
    lors = np.hstack([lors, np.expand_dims(sigma2_factor(lors), 1)])
    out = {}
    for a in AXES:
        g = swap_points(lors[dominant_index(lors, a)].reshape((-1, lors.shape[1])), a)
        g = cut_lors(g, tof_res)
        if a in PERM_RECON:
            g[:, 0:9] = g[:, PERM_RECON[a]]
        out[a] = g
    return out


def map_process(lors):
    """``map_process`` (on_tor_lors.py:243-248): [N,6] -> dict axis -> [N_a,7]
    (endpoints permuted, column 6 = sigma2 factor)."""
    lors = np.hstack([lors, np.expand_dims(sigma2_factor(lors), 1)])
    out = {}
    for a in AXES:
        g = swap_points(lors[dominant_index(lors, a)].reshape((-1, lors.shape[1])), a)
        if a in PERM_MAP:
            g[:, 0:6] = g[:, PERM_MAP[a]]
        out[a] = g
    return out


# --------------------------------------------------------------- image bookkeeping

PERM = {"z": [2, 1, 0], "y": [1, 2, 0], "x": [0, 2, 1]}        # split_lors.py:54-61
PERM_BACK = {"z": [2, 1, 0], "y": [2, 0, 1], "x": [0, 2, 1]}   # split_lors.py:63-70


def axis_view(image, center, size, axis):
    """What ``SplitLoRsModel`` hands the TOR op for one axis group
    (split_lors.py:79-89 with ``transpose(Image)``, src/python/srf/data/image.py:17-22):
    the permuted image and the reversed grid/center/size."""
    p = PERM[axis]
    img = np.ascontiguousarray(np.transpose(image, p))
    c = [center[i] for i in p][::-1]
    s = [size[i] for i in p][::-1]
    return img, list(img.shape[::-1]), c, s


def crop_mask(grid, center, size, inner_radius, axial_length, crop_ratio=0.95):
    """``crop_image`` (src/python/srf/preprocess/merge_map.py:47-65) as a keep-mask over
    the [nx,ny,nz] image. The mesh list comes from ``RingBlock.get_meshes``
    (src/python/srf/scanner/pet/block.py:73-109): ``np.meshgrid`` in its default 'xy'
    indexing enumerates (iy, ix, iz), while the image is flattened as (ix, iy, iz);
    the mask reproduces that pairing."""
    grid = np.asarray(grid)
    center = np.asarray(center, dtype=np.float64)
    size = np.asarray(size, dtype=np.float64)
    interval = size / grid
    p_start = center - (size - interval) / 2
    p_end = center + (size - interval) / 2
    r = [np.linspace(p_start[i], p_end[i], grid[i]) for i in range(3)]
    meshes = np.array(np.meshgrid(r[0], r[1], r[2])).reshape((3, -1)).T
    xy = np.sqrt(meshes[:, 0] ** 2 + meshes[:, 1] ** 2)
    z = np.abs(meshes[:, 2])
    keep = np.ones(meshes.shape[0], bool)
    keep[xy > crop_ratio * inner_radius] = False
    keep[z >= axial_length / 2] = False
    return keep.reshape(tuple(grid))


def merge_effmap(total, keep, threshold=1e-6, zero_below=True):
    """Normalise and invert a summed efficiency map (merge_map.py:37-41 with
    threshold 1e-6 and zeroing; merge_map.py:85-87 ``_full`` with 1e-7 and no
    zeroing)."""
    m = np.where(keep, total, 0)
    m = m / np.max(m)
    out = m.copy()
    hi = m > threshold
    out[hi] = 1 / m[hi]
    if zero_below:
        out[~hi] = 0
    return out


def psf_forward(psf_xy, psf_z, image):
    """``PSFReconStep.kernel`` forward PSF (src/python/srf/model/recon_step.py:78-87): the
    image as an [nx*ny, nz] matrix, times psf_z^T (dense), then the sparse transaxial
    matrix from the left (tf.sparse_tensor_dense_matmul), reshaped back. ``psf_xy``: a
    scipy sparse or dense [nx*ny, nx*ny] matrix; arithmetic in the inputs' precision."""
    nx, ny, nz = image.shape
    v = image.reshape(nx * ny, nz) @ psf_z.T
    return np.asarray(psf_xy @ v).reshape(nx, ny, nz)


def psf_adjoint(psf_xy, psf_z, image):
    """The back-projection side of the same step (recon_step.py:95-101): the image as an
    [nx*ny, nz] matrix times psf_z, then the transposed sparse matrix from the left."""
    nx, ny, nz = image.shape
    v = image.reshape(nx * ny, nz) @ psf_z
    return np.asarray(psf_xy.T @ v).reshape(nx, ny, nz)

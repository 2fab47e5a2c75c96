"""Seeded test inputs shared by the CPU and GPU tests (small versions of the
benchmark workloads). Preprocessing for CPU-side checks uses the numpy restatement in
``oracle/preprocess_ref.py``; GPU tests feed the same events through the product's
preprocessing kernels and check those separately."""

import functools

import numpy as np
import torch

from oracle import preprocess_ref as P
from srf_b200.scanner import RingScanner, tof_info
from srf_b200.synthetic import (generate_events, large_fov_phantom, random_lors,
                                standard_phantom)

SCANNER = RingScanner(400.0, 400, 32, 3.2)
KW_CONFIG = 6 * 4.0 / 2.35482005  # TOR FWHM 4 mm -> kernel_width 10.19 mm


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


@functools.lru_cache(maxsize=None)
def events(n, seed, tof_res=530.0):
    _, sig2 = tof_info(tof_res, 40.0)
    ev = generate_events(n, SCANNER, standard_phantom(), seed,
                         tof_sigma_mm=float(np.sqrt(sig2)) if tof_res < 1e4 else None)
    return ev.numpy()


@functools.lru_cache(maxsize=None)
def phantom_image(grid, voxel, seed=3):
    size = [g * voxel for g in grid]
    img = standard_phantom().voxelize(grid, [0, 0, 0], size)
    rng = np.random.default_rng(seed)
    return (img + 0.25 * rng.random(img.shape, dtype=np.float32) + 0.05).astype(np.float32)


def box_events(n, seed, half=(260.0, 260.0, 260.0), tof_sigma=33.76):
    """Events with endpoints uniform in a box: populates all three dominant-axis
    groups (the ring scanner alone yields almost no z-dominant LORs)."""
    rng = np.random.default_rng(seed)
    h = np.array(half, np.float64)
    p1 = (rng.random((n, 3)) * 2 - 1) * h
    p2 = (rng.random((n, 3)) * 2 - 1) * h
    t = rng.normal(0.0, tof_sigma, n)
    return np.hstack([p1, p2, t[:, None]]).astype(np.float32)


def tor_case(n=2000, seed=11, grid=(64, 64, 32), voxel=6.4, tof_res=530.0, n_box=600):
    ev = events(n, seed, tof_res)
    if n_box:
        ev = np.vstack([ev, box_events(n_box, seed + 1)])
    groups = P.recon_process(ev, tof_res)
    size = [g * voxel for g in grid]
    image = phantom_image(tuple(grid), voxel)
    return dict(events=ev, groups=groups, image=image, grid=list(grid), center=[0.0, 0.0, 0.0],
                size=size, tof_res=tof_res)


def tor_axis(case, axis):
    """(lors [10,N] SoA, permuted image, kernel grid, center, size) for one group."""
    img, g, c, s = P.axis_view(case["image"], case["center"], case["size"], axis)
    lors = np.ascontiguousarray(case["groups"][axis].T.astype(np.float32))
    return lors, img, g, c, s


def map_case(n=3000, seed=5, grid=(64, 64, 32), voxel=6.4):
    lors = random_lors(n, SCANNER, seed).numpy()
    groups = P.map_process(lors)
    size = [g * voxel for g in grid]
    return dict(lors=lors, groups=groups, grid=list(grid), center=[0.0, 0.0, 0.0], size=size)


def siddon_case(n=3000, seed=21, grid=(64, 64, 32), voxel=3.4, tof_res=530.0):
    ev = events(n, seed, tof_res)
    size = [g * voxel for g in grid]
    image = phantom_image(tuple(grid), voxel)
    # CompleteLoRsModel hands the op the image transposed to [nz,ny,nx] (x fastest)
    # with the grid reversed back to (nx,ny,nz) (complete_lors.py:194-202).
    kimg = np.ascontiguousarray(np.transpose(image, (2, 1, 0)))
    return dict(events=ev, lors=np.ascontiguousarray(ev.T), image=image, kimage=kimg,
                grid=list(grid), center=[0.0, 0.0, 0.0], size=size)


def tof_params(tof_res, tof_bin_ps=40.0):
    b, s2 = tof_info(tof_res, tof_bin_ps)
    return float(np.float32(b)), float(np.float32(s2))


# The large axial FOV configuration: R 390 mm, 600 crystals x 320 rings over 1 m
# (3.125 mm pitch), 256x256x128 at 2.5 mm, 400 ps TOF.
LARGE_SCANNER = RingScanner(390.0, 600, 320, 3.125)


def large_case(n=3000, seed=71, n_box=800, tof_res=400.0):
    """Events of the large-FOV multi-cylinder phantom on the 1 m scanner plus box events
    (all three dominant-axis groups populated), preprocessed, with a noisy phantom image
    at 256x256x128 / 2.5 mm."""
    _, sig2 = tof_info(tof_res, 40.0)
    ph = large_fov_phantom(half_length=LARGE_SCANNER.axial_length / 2)
    ev = generate_events(n, LARGE_SCANNER, ph, seed, tof_sigma_mm=float(np.sqrt(sig2))).numpy()
    if n_box:
        ev = np.vstack([ev, box_events(n_box, seed + 1, half=(330.0, 330.0, 200.0),
                                       tof_sigma=float(np.sqrt(sig2)))])
    groups = P.recon_process(ev, tof_res)
    grid, voxel = (256, 256, 128), 2.5
    size = [g * voxel for g in grid]
    img = ph.voxelize(grid, [0.0, 0.0, 0.0], size)
    rng = np.random.default_rng(seed + 2)
    img = (img + 0.25 * rng.random(img.shape, dtype=np.float32) + 0.05).astype(np.float32)
    return dict(events=ev, groups=groups, image=img, grid=list(grid), center=[0.0, 0.0, 0.0],
                size=size, tof_res=tof_res)

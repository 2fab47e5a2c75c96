"""The effmap crop mask (merge_map.py:47-65 of SRF) built on a device with torch equals
the numpy restatement voxel for voxel, including the reference's pairing of the
meshgrid 'xy' mesh list with the (ix, iy, iz) image order (visible on non-cubic grids)."""

import numpy as np
import pytest
import torch

from srf_b200.preprocess import crop_mask, initial_image

CASES = [
    # grid, center, size, inner radius, axial length
    ((64, 64, 32), [0.0, 0.0, 0.0], [217.6, 217.6, 108.8], 400.0, 102.4),
    ((20, 12, 9), [3.0, -7.5, 11.0], [200.0, 120.0, 90.0], 60.0, 70.0),
    ((17, 33, 8), [0.0, 0.0, 0.0], [170.0, 330.0, 80.0], 150.0, 500.0),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_crop_mask_torch_equals_numpy(case):
    grid, center, size, radius, axial = CASES[case]
    host = crop_mask(grid, center, size, radius, axial)
    dev = crop_mask(grid, center, size, radius, axial, device="cpu")
    assert dev.dtype == torch.bool and tuple(dev.shape) == tuple(grid)
    assert host.any() and not host.all()
    np.testing.assert_array_equal(dev.numpy(), host)


def test_initial_image_is_the_cropped_ones():
    grid, center, size, radius, axial = CASES[1]
    img = initial_image(grid, center, size, radius, axial, "cpu")
    assert img.dtype == torch.float32
    np.testing.assert_array_equal(img.numpy(),
                                  crop_mask(grid, center, size, radius, axial).astype(np.float32))

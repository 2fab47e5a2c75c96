"""Host-side geometry of the projector models (CPU): the per-axis transposes of
SplitLoRsModel (split_lors.py:54-70) and the kernel view of an image (reversed grid,
center and size, split_lors.py:73-90 and complete_lors.py:59-98)."""

import torch

from srf_b200.data import Image
from srf_b200.physics import CompleteLoRsModel, SplitLoRsModel


def test_split_perms_are_the_reference_ones_and_inverse():
    M = SplitLoRsModel
    assert M.perm("x") == [0, 2, 1] and M.perm("y") == [1, 2, 0] and M.perm("z") == [2, 1, 0]
    x = torch.arange(2 * 3 * 5).reshape(2, 3, 5)
    for a in "xyz":
        assert torch.equal(x.permute(*M.perm(a)).permute(*M.perm_back(a)), x)


def test_kernel_geometry_reverses_the_permuted_axes():
    data = torch.arange(4 * 6 * 8, dtype=torch.float32).reshape(4, 6, 8)
    img = Image(data, [1.0, 2.0, 3.0], [40.0, 60.0, 80.0])
    for a in "xyz":
        kimg, g, c, s = SplitLoRsModel.kernel_geometry(img, a)
        p = SplitLoRsModel.perm(a)
        assert torch.equal(kimg, data.permute(*p))
        assert list(g) == [data.shape[k] for k in p][::-1]
        assert list(c) == [img.center[k] for k in p][::-1]
        assert list(s) == [img.size[k] for k in p][::-1]
        # the slice axis (slowest of the kernel layout) is the dominant axis a
        assert kimg.shape[0] == data.shape["xyz".index(a)]
    kimg, g, c, s = CompleteLoRsModel.kernel_geometry(img)
    assert torch.equal(kimg, data.permute(2, 1, 0))
    assert list(g) == [4, 6, 8] and list(c) == [1.0, 2.0, 3.0] and list(s) == [40.0, 60.0, 80.0]

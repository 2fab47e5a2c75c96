"""Data types of the reconstruction path, mirroring the reference's:

* ``Image`` — ``src/python/srf/data/image.py:4-28``: data + center + size; ``grid`` is
  the data's shape; ``transpose`` permutes data, center and size together.
* ``ListModeData`` / ``ListModeDataWithoutTOF`` — ``src/python/srf/data/listmode.py:52-77``:
  LOR records plus one value per LOR.
* ``ListModeDataSplit`` / ``ListModeDataSplitWithoutTOF`` — ``listmode.py:127-138``: one
  ``ListModeData`` per dominant axis, indexable by 'x' / 'y' / 'z'.

Tensors are torch tensors (CUDA for anything that reaches a projector).
"""

import torch


class Image:
    """Image data with center and size (kernel-independent, [nx, ny, nz] order)."""

    def __init__(self, data, center, size):
        self.data = data
        self.center = [float(c) for c in center]
        self.size = [float(s) for s in size]

    @property
    def grid(self):
        return list(self.data.shape)

    def fmap(self, f):
        return Image(f(self.data), self.center, self.size)

    def transpose(self, perm=None):
        """``transpose.register(Image)`` of image.py:17-22 (default perm [2, 1, 0])."""
        if perm is None:
            perm = [2, 1, 0]
        return Image(self.data.permute(*perm).contiguous(), [self.center[p] for p in perm],
                     [self.size[p] for p in perm])

    def __repr__(self):
        return f"Image(grid={self.grid}, center={self.center}, size={self.size})"


def transpose(x, perm=None):
    if isinstance(x, Image):
        return x.transpose(perm)
    if perm is None:
        perm = list(range(x.dim()))[::-1]
    return x.permute(*perm).contiguous()


class ListModeData:
    def __init__(self, lors, values):
        self._lors = lors
        self._values = values

    @property
    def lors(self):
        return self._lors

    @property
    def values(self):
        return self._values

    def __len__(self):
        return int(self._values.numel()) if self._values is not None else int(self._lors.shape[0])


class ListModeDataWithoutTOF(ListModeData):
    pass


class _XYZ:
    AXES = ("x", "y", "z")

    def __init__(self, x, y, z):
        self._x, self._y, self._z = x, y, z

    @property
    def x(self):
        return self._x

    @property
    def y(self):
        return self._y

    @property
    def z(self):
        return self._z

    def __getitem__(self, item):
        if item == "x":
            return self._x
        if item == "y":
            return self._y
        if item == "z":
            return self._z
        raise KeyError(item)

    def items(self):
        return [(a, self[a]) for a in self.AXES]


class ListModeDataSplit(_XYZ):
    pass


class ListModeDataSplitWithoutTOF(_XYZ):
    pass


def as_cuda_f32(a, device=None):
    """numpy / torch -> contiguous CUDA float32 tensor."""
    if not torch.is_tensor(a):
        a = torch.as_tensor(a)
    dev = device if device is not None else (a.device if a.is_cuda else torch.device("cuda"))
    return a.to(device=dev, dtype=torch.float32).contiguous()

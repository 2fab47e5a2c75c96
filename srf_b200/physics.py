"""Physics models: the drop-in for ``src/python/srf/physics/split_lors.py`` (TOR) and
``src/python/srf/physics/complete_lors.py`` (Siddon).

``projection(model, image, data)`` / ``backprojection(model, data, image)`` dispatch on
the model and data types exactly as the reference's multidispatch registrations do
(split_lors.py:73-133, complete_lors.py:192-231):

* ``SplitLoRsModel`` + ``ListModeDataSplit``: per dominant axis, transpose the image by
  ``perm(axis)``, call the TOR op with the reversed grid/center/size; back-projection
  transposes each result back by ``perm_back(axis)`` and sums the three.
* ``SplitLoRsModel`` + ``ListModeDataSplitWithoutTOF``: the same through ``Maplors``.
* ``CompleteLoRsModel`` + ``ListModeData``: transpose [2,1,0] (x fastest), Siddon op,
  transpose back; ``ListModeDataWithoutTOF`` goes through ``Maplors``.

Every call runs on the CUDA library; there is no other compute path.
"""

import torch

from . import ops
from .data import (Image, ListModeData, ListModeDataSplit, ListModeDataSplitWithoutTOF,
                   ListModeDataWithoutTOF)


class SplitLoRsModel:
    """TOR model on dominant-axis-split LORs (split_lors.py:28-70)."""

    AXIS = ("x", "y", "z")

    class KEYS:
        KERNEL_WIDTH = "kernel_width"
        TOF_BIN = "tof_bin"
        TOF_SIGMA2 = "tof_sigma2"
        GEO_SIGMA2_FLAG = "geo_sigma2_flag"

    def __init__(self, kernel_width, geo_sigma2_flag=False, tof_sigma2=None, tof_bin=None,
                 name="split_lor_model"):
        if tof_bin is None:
            tof_bin = 1.0e4
        if tof_sigma2 is None:
            tof_sigma2 = 1.0e4
        self.name = name
        self.config = {self.KEYS.KERNEL_WIDTH: float(kernel_width),
                       self.KEYS.GEO_SIGMA2_FLAG: bool(geo_sigma2_flag),
                       self.KEYS.TOF_SIGMA2: float(tof_sigma2),
                       self.KEYS.TOF_BIN: float(tof_bin)}

    @property
    def kernel_width(self):
        return self.config[self.KEYS.KERNEL_WIDTH]

    @property
    def geo_sigma2_flag(self):
        return self.config[self.KEYS.GEO_SIGMA2_FLAG]

    @property
    def tof_sigma2(self):
        return self.config[self.KEYS.TOF_SIGMA2]

    @property
    def tof_bin(self):
        return self.config[self.KEYS.TOF_BIN]

    @classmethod
    def perm(cls, axis):
        return {"z": [2, 1, 0], "y": [1, 2, 0], "x": [0, 2, 1]}[axis]

    @classmethod
    def perm_back(cls, axis):
        return {"z": [2, 1, 0], "y": [2, 0, 1], "x": [0, 2, 1]}[axis]

    @classmethod
    def kernel_geometry(cls, image, axis):
        """(image data permuted for ``axis``, grid, center, size in kernel order)."""
        img = image.transpose(cls.perm(axis))
        return img.data, img.grid[::-1], img.center[::-1], img.size[::-1]

    def projection(self, image, data):
        return projection(self, image, data)

    def backprojection(self, data, image):
        return backprojection(self, data, image)


class CompleteLoRsModel:
    """Siddon model on complete LORs (complete_lors.py:33-52)."""

    class KEYS:
        class CONFIG:
            TOF_SIGMA2 = "tof_sigma2"
            TOF_BIN = "tof_bin"

    def __init__(self, name="complete_lor_model", tof_sigma2=None, tof_bin=None):
        if tof_sigma2 is None:
            tof_sigma2 = 1.0e4
        if tof_bin is None:
            tof_bin = 1.0e4
        self.name = name
        self.config = {self.KEYS.CONFIG.TOF_SIGMA2: float(tof_sigma2),
                       self.KEYS.CONFIG.TOF_BIN: float(tof_bin)}

    @property
    def tof_sigma2(self):
        return self.config[self.KEYS.CONFIG.TOF_SIGMA2]

    @property
    def tof_bin(self):
        return self.config[self.KEYS.CONFIG.TOF_BIN]

    @staticmethod
    def kernel_geometry(image):
        img = image.transpose()
        return img.data, img.grid[::-1], img.center[::-1], img.size[::-1]

    def projection(self, image, data):
        return projection(self, image, data)

    def backprojection(self, data, image):
        return backprojection(self, data, image)


def _lors_of(d):
    return d.lors


def projection(model, image, data):
    """Forward projection; returns list-mode data holding the projected values."""
    if isinstance(model, SplitLoRsModel):
        if not isinstance(data, ListModeDataSplit):
            raise TypeError("SplitLoRsModel projects ListModeDataSplit")
        res = {}
        for a in model.AXIS:
            if data[a].lors.shape[0] == 0:  # nothing to launch
                res[a] = torch.zeros(0, dtype=torch.float32, device=data[a].lors.device)
                continue
            img, g, c, s = model.kernel_geometry(image, a)
            res[a] = ops.tor_projection(_lors_of(data[a]), img, g, c, s, model.kernel_width,
                                        model.geo_sigma2_flag, model.tof_bin, model.tof_sigma2,
                                        layout="nc")
        return ListModeDataSplit(*[ListModeData(data[a].lors, res[a]) for a in model.AXIS])
    if isinstance(model, CompleteLoRsModel):
        img, g, c, s = model.kernel_geometry(image)
        v = ops.siddon_projection(_lors_of(data), img, g, c, s, model.tof_bin, model.tof_sigma2,
                                  layout="nc")
        return ListModeData(data.lors, v)
    raise TypeError(f"no projection for {type(model).__name__}")


def _sum_back(model, parts, image):
    out = None
    for a, bp in parts:
        back = bp.permute(*model.perm_back(a))
        out = back.clone() if out is None else out.add_(back)
    if out is None:  # every group empty
        out = torch.zeros_like(image.data)
    return Image(out.contiguous(), image.center, image.size)


def backprojection(model, data, image):
    """Back-projection (Aᵀ(1/v), the reference's semantics) or, for *WithoutTOF data,
    the efficiency-map ``Maplors``; returns an ``Image`` in the input image's layout."""
    if isinstance(model, SplitLoRsModel):
        parts = []
        if isinstance(data, ListModeDataSplitWithoutTOF):
            for a in model.AXIS:
                if data[a].lors.shape[0] == 0:
                    continue
                img, g, c, s = model.kernel_geometry(image, a)
                parts.append((a, ops.tor_maplors(img, g, c, s, _lors_of(data[a]), data[a].values,
                                                 model.kernel_width, model.geo_sigma2_flag,
                                                 layout="nc")))
        elif isinstance(data, ListModeDataSplit):
            for a in model.AXIS:
                if data[a].lors.shape[0] == 0:
                    continue
                img, g, c, s = model.kernel_geometry(image, a)
                parts.append((a, ops.tor_backprojection(
                    img, _lors_of(data[a]), data[a].values, g, c, s, model.kernel_width,
                    model.geo_sigma2_flag, model.tof_bin, model.tof_sigma2, layout="nc")))
        else:
            raise TypeError("SplitLoRsModel back-projects ListModeDataSplit[WithoutTOF]")
        return _sum_back(model, parts, image)
    if isinstance(model, CompleteLoRsModel):
        img, g, c, s = model.kernel_geometry(image)
        if isinstance(data, ListModeDataWithoutTOF):
            r = ops.siddon_maplors(img, g, c, s, _lors_of(data), data.values, layout="nc")
        elif isinstance(data, ListModeData):
            r = ops.siddon_backprojection(img, _lors_of(data), data.values, g, c, s,
                                          model.tof_bin, model.tof_sigma2, layout="nc")
        else:
            raise TypeError("CompleteLoRsModel back-projects ListModeData[WithoutTOF]")
        return Image(r.permute(2, 1, 0).contiguous(), image.center, image.size)
    raise TypeError(f"no backprojection for {type(model).__name__}")


def projection_backprojection(model, image, data):
    """``backprojection(model, projection(model, image, data), image)`` with the projected
    data too; for TOR each axis group is one combined library call. Returns
    (projected list-mode data, back-projected ``Image``)."""
    if isinstance(model, SplitLoRsModel) and isinstance(data, ListModeDataSplit) \
            and not isinstance(data, ListModeDataSplitWithoutTOF):
        res, parts = {}, []
        for a in model.AXIS:
            if data[a].lors.shape[0] == 0:
                res[a] = torch.zeros(0, dtype=torch.float32, device=data[a].lors.device)
                continue
            img, g, c, s = model.kernel_geometry(image, a)
            res[a], bp = ops.tor_projection_backprojection(
                _lors_of(data[a]), img, g, c, s, model.kernel_width, model.geo_sigma2_flag,
                model.tof_bin, model.tof_sigma2, layout="nc")
            parts.append((a, bp))
        proj = ListModeDataSplit(*[ListModeData(data[a].lors, res[a]) for a in model.AXIS])
        return proj, _sum_back(model, parts, image)
    proj = projection(model, image, data)
    return proj, backprojection(model, proj, image)


def backproject_adjoint(model, data, image):
    """The plain transpose Aᵀ·values (no division): autograd's backward and the
    textbook OSEM numerator."""
    if isinstance(model, SplitLoRsModel):
        parts = []
        for a in model.AXIS:
            if data[a].lors.shape[0] == 0:
                continue
            img, g, c, s = model.kernel_geometry(image, a)
            parts.append((a, ops.tor_backproject_adjoint(
                data[a].values, _lors_of(data[a]), g, c, s, model.kernel_width,
                model.geo_sigma2_flag, model.tof_bin, model.tof_sigma2, layout="nc")))
        return _sum_back(model, parts, image)
    if isinstance(model, CompleteLoRsModel):
        img, g, c, s = model.kernel_geometry(image)
        r = ops.siddon_backproject_adjoint(data.values, _lors_of(data), g, c, s, model.tof_bin,
                                           model.tof_sigma2, layout="nc")
        return Image(r.permute(2, 1, 0).contiguous(), image.center, image.size)
    raise TypeError(f"no adjoint for {type(model).__name__}")


def map_lors(model, data, image):
    """Efficiency-map back-projection (``Maplors``) for either model."""
    if isinstance(model, SplitLoRsModel) and not isinstance(data, ListModeDataSplitWithoutTOF):
        data = ListModeDataSplitWithoutTOF(*[data[a] for a in model.AXIS])
    if isinstance(model, CompleteLoRsModel) and not isinstance(data, ListModeDataWithoutTOF):
        data = ListModeDataWithoutTOF(data.lors, data.values)
    return backprojection(model, data, image)


def map_generated(model, pairs, image, first=0, count=None):
    """Maplors of generated detector-pair LORs ``first .. first+count-1``
    (``synthetic.GeneratedPairs``) for the TOR model, with no LOR array in memory: per
    axis group one ``srf_tor_maplors_generated`` call, then the reference's transpose back
    and sum (split_lors.py:116-133). Returns an ``Image`` in the input image's layout."""
    if not isinstance(model, SplitLoRsModel):
        raise TypeError("generated LORs are mapped by the TOR model")
    count = len(pairs) - first if count is None else count
    parts = []
    for k, a in enumerate(model.AXIS):
        _, g, c, s = model.kernel_geometry(image, a)
        parts.append((a, ops.tor_maplors_generated(
            pairs.kind, pairs.crystals, pairs.n_rings, pairs.n_blocks, pairs.n_per_block,
            pairs.seed, first, count, k, g, c, s, model.kernel_width, model.geo_sigma2_flag)))
    return _sum_back(model, parts, image)

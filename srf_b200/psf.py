"""PSF-in-the-loop reconstruction step (``PSFReconStep``,
src/python/srf/model/recon_step.py:56-115, with the loader of
src/python/srf/data/loader.py:75-86).

The image [nx, ny, nz] is seen as an [nx*ny, nz] matrix X. The PSF applies a dense axial
kernel Pz [nz, nz] and a sparse transaxial kernel Axy [nx*ny, nx*ny]:

    psf(X)      = Axy (X Pz^T)        (recon_step.py:78-87)
    psf^T(B)    = Axy^T (B Pz)        (recon_step.py:95-101)

and one step is x <- update(x, psf^T(backprojection(projection(psf(x)))), effmap). Each
application is one launch of the library's fused kernel (``srf_psf_apply``): a warp per
row of Axy sums its neighbours' rows of X (lanes over z), then multiplies that row by
Pz^T (or Pz) held in shared memory, so no intermediate [nx*ny, nz] matrix is written.
Axy^T is built once on the host for the adjoint.
"""

import numpy as np
import torch

from . import _lib
from .data import Image
from .recon import mlem_update


def _csr(mat, device):
    """CSR device tensors (rowptr int64, col int32, val float32) of a scipy sparse matrix."""
    import scipy.sparse as sp
    m = sp.csr_matrix(mat, dtype=np.float32)
    m.sum_duplicates()
    m.sort_indices()
    return (torch.as_tensor(m.indptr.astype(np.int64), device=device),
            torch.as_tensor(m.indices.astype(np.int32), device=device),
            torch.as_tensor(m.data.astype(np.float32), device=device), m.shape)


class PSF:
    """Separable PSF: ``psf_xy`` a (scipy) sparse or dense [nx*ny, nx*ny] matrix, ``psf_z``
    a dense [nz, nz] matrix."""

    def __init__(self, psf_xy, psf_z, device="cuda"):
        dev = torch.device(device)
        self.fwd = _csr(psf_xy, dev)
        import scipy.sparse as sp
        self.adj = _csr(sp.csr_matrix(psf_xy, dtype=np.float32).T, dev)
        self.pz = torch.as_tensor(np.asarray(psf_z, np.float32), device=dev)
        if self.pz.dim() != 2 or self.pz.shape[0] != self.pz.shape[1]:
            raise ValueError("psf_z must be a square [nz, nz] matrix")
        if self.fwd[3][0] != self.fwd[3][1]:
            raise ValueError("psf_xy must be a square [nx*ny, nx*ny] matrix")

    def _psf(self, csr, x, transpose_pz):
        """csr (x Pz^T) (transpose_pz = 0) or csr (x Pz) (1), x a contiguous [rows, nz]."""
        rowptr, col, val, shape = csr
        y = torch.empty((shape[0], x.shape[1]), dtype=torch.float32, device=x.device)
        with torch.cuda.device(x.device):
            _lib.call("srf_psf_apply", rowptr.data_ptr(), col.data_ptr(), val.data_ptr(),
                      shape[0], shape[1], x.data_ptr(), x.shape[1], self.pz.data_ptr(),
                      int(transpose_pz), y.data_ptr(), 0,
                      torch.cuda.current_stream(x.device).cuda_stream)
        return y

    def _check(self, data):
        nx, ny, nz = data.shape
        if nx * ny != self.fwd[3][0] or nz != self.pz.shape[0]:
            raise ValueError(f"image {tuple(data.shape)} does not match the PSF "
                             f"({self.fwd[3][0]} transaxial, {self.pz.shape[0]} axial)")
        return nx, ny, nz

    def apply(self, image):
        """psf(image): Axy (X Pz^T) (recon_step.py:78-87), as an Image."""
        nx, ny, nz = self._check(image.data)
        x = image.data.reshape(nx * ny, nz).contiguous()
        out = self._psf(self.fwd, x, 0).reshape(nx, ny, nz)
        return Image(out, image.center, image.size)

    def adjoint(self, image):
        """psf^T(image): Axy^T (B Pz) (recon_step.py:95-101), as an Image."""
        nx, ny, nz = self._check(image.data)
        b = image.data.reshape(nx * ny, nz).contiguous()
        out = self._psf(self.adj, b, 1).reshape(nx, ny, nz)
        return Image(out, image.center, image.size)


def load_psf(xy_path, z_path, device="cuda"):
    """``WorkerLoader._load_psf``: the transaxial matrix from a MATLAB file's ``matrix``
    entry, the axial matrix from ``.npy``."""
    import scipy.io as scio
    xy = scio.loadmat(xy_path)["matrix"]
    return PSF(xy, np.load(z_path), device)


class PSFReconStep:
    """``PSFReconStep.kernel``: x <- update(x, psf^T(A^T(1/(A psf(x)))), effmap)."""

    def __init__(self, model, psf, update=mlem_update):
        self.model = model
        self.psf = psf
        self.update = update

    def __call__(self, image, efficiency_map, projection_data):
        from .physics import backprojection, projection
        image_psf = self.psf.apply(image)
        proj = projection(self.model, image_psf, projection_data)
        back = backprojection(self.model, proj, image_psf)
        return self.update(image, self.psf.adjoint(back), efficiency_map)

"""PSF reconstruction step: the fused PSF kernel against the numpy restatement of
recon_step.py:78-87 / :95-101 (oracle, float32 and float64), its adjoint identity, the
loader (MATLAB + .npy files), and the step with an identity PSF equal to the plain
reconstruction step."""

import numpy as np
import pytest
import scipy.io as scio
import scipy.sparse as sp
import torch

from srf_b200.psf import PSF, PSFReconStep, load_psf


def _psf_mats(nx, ny, nz, seed=2):
    """A local transaxial blur (3x3 neighbourhood, random weights) and an axial band."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for ix in range(nx):
        for iy in range(ny):
            r = ix * ny + iy
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    jx, jy = ix + dx, iy + dy
                    if 0 <= jx < nx and 0 <= jy < ny:
                        rows.append(r)
                        cols.append(jx * ny + jy)
                        vals.append(rng.uniform(0.1, 1.0))
    xy = sp.coo_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))
    z = np.zeros((nz, nz), np.float32)
    for i in range(nz):
        for j in range(max(0, i - 2), min(nz, i + 3)):
            z[i, j] = rng.uniform(0.1, 1.0)
    return xy, z


def test_load_psf_files(tmp_path):
    xy, z = _psf_mats(6, 5, 4)
    scio.savemat(tmp_path / "xy.mat", {"matrix": xy.tocsc()})
    np.save(tmp_path / "z.npy", z)
    p = load_psf(str(tmp_path / "xy.mat"), str(tmp_path / "z.npy"), device="cpu")
    assert p.fwd[3] == (30, 30) and tuple(p.pz.shape) == (4, 4)
    assert int(p.fwd[0][-1]) == xy.nnz == int(p.adj[0][-1])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 12, 8), (20, 18, 64), (9, 7, 130)])
def test_psf_matches_the_oracle_and_is_adjoint(shape):
    from oracle import preprocess_ref as P
    nx, ny, nz = shape
    xy, z = _psf_mats(nx, ny, nz)
    p = PSF(xy, z)
    rng = np.random.default_rng(4)
    x = rng.random((nx, ny, nz)).astype(np.float32)
    yv = rng.random((nx, ny, nz)).astype(np.float32)
    from srf_b200.data import Image
    X = Image(torch.as_tensor(x).cuda(), [0, 0, 0], [1, 1, 1])
    Y = Image(torch.as_tensor(yv).cuda(), [0, 0, 0], [1, 1, 1])
    A32 = xy.tocsr().astype(np.float32)
    A64 = xy.tocsr().astype(np.float64)
    got = p.apply(X).data.cpu().numpy()
    gota = p.adjoint(Y).data.cpu().numpy()

    def rel(a, b):
        return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))

    # float32: the reference's product order; float64: the exact value
    assert rel(got, P.psf_forward(A32, z, x)) < 1e-6
    assert rel(got, P.psf_forward(A64, z.astype(np.float64), x.astype(np.float64))) < 1e-6
    assert rel(gota, P.psf_adjoint(A32, z, yv)) < 1e-6
    assert rel(gota, P.psf_adjoint(A64, z.astype(np.float64), yv.astype(np.float64))) < 1e-6
    lhs = float((p.apply(X).data.double() * Y.data.double()).sum())
    rhs = float((X.data.double() * p.adjoint(Y).data.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_psf_oracle_restatement_is_separable():
    """The oracle's product order (dense axial first) equals the other association."""
    from oracle import preprocess_ref as P
    xy, z = _psf_mats(5, 4, 6)
    x = np.random.default_rng(1).random((5, 4, 6))
    A = xy.toarray()
    np.testing.assert_allclose(P.psf_forward(xy.tocsr(), z.astype(np.float64), x),
                               ((A @ x.reshape(20, 6)) @ z.T).reshape(5, 4, 6), rtol=1e-12)
    np.testing.assert_allclose(P.psf_adjoint(xy.tocsr(), z.astype(np.float64), x),
                               ((A.T @ x.reshape(20, 6)) @ z).reshape(5, 4, 6), rtol=1e-12)


@pytest.mark.gpu
def test_psf_step_with_identity_psf_is_the_plain_step():
    from srf_b200 import SplitLoRsModel
    from srf_b200 import preprocess as PP
    from srf_b200.data import Image
    from srf_b200.recon import ReconStep
    from tests import _cases as K
    grid, voxel = (32, 32, 16), 6.4
    size = [g * voxel for g in grid]
    ev = K.events(20_000, 13, 530.0).astype(np.float32)
    data = PP.split_listmode(PP.recon_process(torch.as_tensor(ev).cuda(), 530.0))
    b, s2 = K.tof_params(530.0)
    model = SplitLoRsModel(K.KW_CONFIG, False, tof_sigma2=s2, tof_bin=b)
    x = Image(torch.rand(grid, device="cuda") + 0.5, [0, 0, 0], size)
    eff = Image(torch.rand(grid, device="cuda") + 0.5, [0, 0, 0], size)
    ident = PSF(sp.identity(grid[0] * grid[1], format="csr"), np.eye(grid[2]))
    a = PSFReconStep(model, ident)(x, eff, data).data
    r = ReconStep(model)(x, eff, data).data
    assert torch.count_nonzero(r) > 0
    assert float((a - r).norm() / r.norm()) < 1e-6

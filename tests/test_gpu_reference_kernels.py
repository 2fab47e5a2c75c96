"""The product kernels against the reference's OWN CUDA kernels (src/cpp/tf_custom_ops/
tor.cu.cc and siddon.cu.cc built for sm_100a by oracle/Makefile), on the same B200 and
the same inputs: the parity target (rel-L2 <= 1e-5 in float32).

Skipped where oracle/_ref was not built. Siddon inputs are first walked by the oracle:
a ray whose first voxel falls off the grid would make the reference read outside the
image, so such inputs are never handed to it.
"""

import numpy as np
import pytest
import torch

from oracle import pyoracle as O
from srf_b200 import ops
from tests import _cases as K
from tests.test_gpu_parity import TOL, TOR_PATHS, cu, host, record

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refgpu():
    if not O.ReferenceGPU.available():
        pytest.skip("reference GPU build not present")
    return O.ReferenceGPU()


@pytest.fixture(scope="module")
def tcase():
    return K.tor_case(n=20000, seed=51, grid=(128, 128, 64), voxel=3.2, n_box=2000)


@pytest.fixture(params=list(TOR_PATHS))
def tor_path(request):
    from srf_b200 import tuning
    tuning.set_tuning(*TOR_PATHS[request.param])
    yield request.param
    tuning.set_tuning()


@pytest.mark.parametrize("kw,geo", [(K.KW_CONFIG, False), (4.0, True)])
@pytest.mark.parametrize("axis", ["x", "y", "z"])
def test_tor_against_reference_gpu(refgpu, tcase, kw, geo, axis, tor_path):
    b, s2 = K.tof_params(530.0)
    lors, img, g, c, s = K.tor_axis(tcase, axis)
    L, I = cu(lors), cu(img)
    ref = host(refgpu.tor_projection(L, I, g, c, s, kw, geo, b, s2))
    got = host(ops.tor_projection(L, I, g, c, s, kw, geo, b, s2, layout="cn"))
    e = K.rel_l2(got, ref)
    exact = float(np.mean(got == ref))
    record("tor_vs_reference_gpu", kw=kw, geo=geo, axis=axis, n=int(lors.shape[1]), rel_l2=e,
           bit_equal_fraction=exact, path=tor_path)
    assert e <= TOL, e
    pv = ref.copy()
    pv[::13] = 0.0
    refb = host(refgpu.tor_backprojection(L, cu(pv), g, c, s, kw, geo, b, s2))
    gotb = host(ops.tor_backprojection(I, L, cu(pv), g, c, s, kw, geo, b, s2, layout="cn"))
    eb = K.rel_l2(gotb, refb)
    record("tor_bproj_vs_reference_gpu", kw=kw, geo=geo, axis=axis, rel_l2=eb)
    assert eb <= TOL, eb


def test_tor_map_against_reference_gpu(refgpu):
    mc = K.map_case(n=20000, seed=9, grid=(128, 128, 64), voxel=3.2)
    for axis in "xyz":
        lors7 = np.ascontiguousarray(mc["groups"][axis].T.astype(np.float32))
        _, g, c, s = K.P.axis_view(np.zeros(mc["grid"], np.float32), mc["center"], mc["size"],
                                   axis)
        ones = cu(np.ones(lors7.shape[1], np.float32))
        L = cu(lors7)
        ref = host(refgpu.tor_maplors(L, ones, g, c, s, K.KW_CONFIG, False))
        got = host(ops.tor_maplors(L, g, c, s, L, ones, K.KW_CONFIG, False, layout="cn"))
        e = K.rel_l2(got, ref)
        record("tor_map_vs_reference_gpu", axis=axis, rel_l2=e)
        assert e <= TOL, (axis, e)


@pytest.mark.parametrize("tof", [True, False])
def test_siddon_against_reference_gpu(refgpu, tof):
    sc = K.siddon_case(n=30000, seed=61, grid=(64, 64, 32), voxel=3.4)
    args = (sc["grid"], sc["center"], sc["size"])
    visits, bad = O.siddon_counts(sc["lors"], *args)
    assert bad == 0, "input would make the reference read outside the image"
    b, s2 = K.tof_params(530.0)
    if not tof:
        s2 = 1.0e6
    L, I = cu(sc["lors"]), cu(sc["kimage"])
    ref = host(refgpu.siddon_projection(L, I, *args, b, s2))
    got = host(ops.siddon_projection(L, I, *args, b, s2, layout="cn"))
    e = K.rel_l2(got, ref)
    record("siddon_vs_reference_gpu", tof=tof, rel_l2=e, bit_equal_fraction=float(np.mean(got == ref)))
    assert e <= TOL, e
    refb = host(refgpu.siddon_backprojection(L, cu(ref), *args, b, s2))
    gotb = host(ops.siddon_backprojection(I, L, cu(ref), *args, b, s2, layout="cn"))
    assert K.rel_l2(gotb, refb) <= TOL
    ones = cu(np.ones(sc["lors"].shape[1], np.float32))
    refm = host(refgpu.siddon_maplors(L, ones, *args))
    gotm = host(ops.siddon_maplors(I, *args, L, ones, layout="cn"))
    assert K.rel_l2(gotm, refm) <= TOL
